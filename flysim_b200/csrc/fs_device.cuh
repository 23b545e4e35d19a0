// Device-side data of the flysim step engine (shared by the kernels and the
// C ABI implementation).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "flysim_b200.h"

namespace fsd {

constexpr uint32_t kFull = 0xffffffffu;

// Reference-order layout of one receptor on the device (fs_rec_layout).
struct RecDev {
  uint32_t n_gates;
  const uint32_t *gate_pre, *gate_post0;
  const float *gate_g;
  float *gate_st, *gate_xt;
  const uint32_t *grow, *ggate;  // gather CSR by post
  uint32_t n_recs;
  const uint32_t *rpre, *rpost;
  float *rg, *rst, *rxt;
  const uint32_t *rrow;  // records CSR by post
};

// Everything the compat kernels touch; passed by value.
struct CompatDev {
  uint32_t n;
  uint32_t glob;  // global ActCtr (STP/STD/LTP)
  // parameters
  const float *Vth, *El, *gl, *Cm, *Vreset, *df, *ef, *dVmax;
  const int32_t *RfPed, *SpiDy;
  const float *Vrev, *dfst, *nmda_dfxt, *nmda_efst, *nmda_as, *nmda_mg, *ext_g;
  const float *pb;
  const uint32_t *act;
  const float *inj_mean, *inj_std;
  const float *stp_pv, *stp_dfD, *stp_efD, *stp_aF, *stp_dfF, *stp_efF, *stp_aCap, *stp_dfCap,
      *stp_aCar, *stp_dfCar, *stp_efCar;
  const float *ltp_dfLP, *ltp_Pos, *ltp_Neg;
  const int32_t *ltp_SpiLPDy;
  // state
  float *V, *Isyn, *G, *ext_st, *ext_xt_n, *ext_st_n, *Irep, *D, *F, *Cap, *Car, *LP;
  int32_t *Count, *CountLP;
  uint32_t *NS;
  RecDev R[FS_NREC];
  uint32_t gate_off[FS_NREC + 1];  // prefix of n_gates (gate kernel index space)
  uint32_t rec_off[FS_NREC + 1];   // prefix of n_recs (LTP kernel index space)
  const uint32_t *gap_row, *gap_other;
  const float *gap_g;
  // random streams of one batch
  const uint32_t *drawoff;  // [n] first draw of neuron i within a step
  const uint32_t *injoff;   // [n] rank of neuron i among injected neurons
  uint32_t draws_per_step, inj_per_step;
  const uint32_t *draws;    // raw mt19937 outputs of the batch
  uint32_t jcong_base;      // congruential state before the batch's first Gaussian
  // glibc-exact expf / logf exception tables
  const uint32_t *expf_keys;
  const float *expf_vals;
  uint32_t expf_n;
  const uint32_t *logf_keys;
  const float *logf_vals;
  uint32_t logf_n;
  // per-step outputs of the batch
  uint32_t *spikebits;      // [nsteps][words]
  uint32_t words;
  float *outV, *outIrep;
  uint32_t *outNS;
  const uint32_t *gv_sel;
  uint32_t gv_n;
  float *gv_st, *gv_xt;
  int *err;                 // device error word
};

// Launch wrappers (fs_compat.cu)
void compat_set_tables(const uint32_t kn[128], const float fn[128], const float wn[128],
                       const uint32_t jump_a[32], const uint32_t jump_c[32], cudaStream_t st);
cudaError_t compat_step(const CompatDev &d, uint32_t s, uint32_t sm_count, cudaStream_t st,
                        uint64_t *launches);
cudaError_t compat_varinit(const CompatDev &d, cudaStream_t st);
cudaError_t mt_generate(uint32_t *state, uint32_t *pos, uint32_t *out, uint64_t count, cudaStream_t st);
cudaError_t spikes_compact(const uint32_t *bits, uint32_t nsteps, uint32_t words, uint32_t *counts,
                           uint32_t *offsets, uint32_t *idx, cudaStream_t st, uint64_t *launches);
// test hooks
cudaError_t expf_ref_eval(const float *x, float *y, uint64_t k, const uint32_t *keys, const float *vals,
                          uint32_t nk, cudaStream_t st);

}  // namespace fsd
