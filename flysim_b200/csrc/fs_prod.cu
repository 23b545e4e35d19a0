// Production engine of the flysim step (FS_MODE_FP32 / FS_MODE_FP64).
//
// Same neuron model as the reference (VmEul + firing, code/EqsGnl2.cpp:152-251;
// external Bernoulli drive per receptor, code/EqsGnl2.cpp:284-337), with the
// synapse side restructured for the GPU:
//
//  * Linear receptors (AMPA, GABA, ACh, GluCl).  Every synapse gate of the
//    reference obeys st <- st + inc on a presynaptic spike, st <- st*df
//    otherwise (code/EqsGnl2.cpp:404-480, :866-917), and the post-synaptic
//    conductance is sum(g*st).  With df shared by all targets of a presynaptic
//    neuron, that sum obeys G(t) = df*G(t-1) + sum_spikes g*c, with
//    c = inc + st_pre(t-1)*(1-df) computed once per spike from a per-neuron
//    gate st_pre.  So a spike pushes g*c into a delay ring
//    ring[receptor][post][(t+delay) mod S] (64-bit fixed point, 2^-40 nS:
//    integer atomics make the sum independent of arrival order), and each post
//    folds its slot into G once per step.
//  * NMDA.  The gate s is nonlinear in its own state (code/EqsGnl2.cpp:493) but
//    depends only on the presynaptic spike train, so x_pre/s_pre are kept per
//    presynaptic neuron, s_pre(t) is stored in a history ring
//    s_hist[pre][t mod S], and each post pulls sum(g * s_pre(t-1-delay)) over
//    its NMDA in-edges.
//  * Drive: counter-based Philox-4x32-10 (Salmon et al., SC'11) keyed by
//    (step, neuron), so no generator state is shared.
//
// Scheduling.  Every value a neuron reads from another neuron was produced
// at least min_delay steps earlier.  The steps are therefore cut into
// intervals of max(min_delay, 1) steps separated by a bounded-wait grid
// barrier; inside an interval the neurons are independent.  A block owns a
// contiguous range of post neurons and, per interval, (1) pulls the NMDA
// conductances of all the interval's steps at once (one warp per post, the
// in-edges split over the lanes, a butterfly reduction per step: the loads of
// many steps overlap), then (2) advances its neurons one thread each through
// the interval's steps with their state in registers, pushing the spikes of
// each step into the delay ring (one warp per spike).  The ring depth
// S = next power of two >= max_delay + min_delay + 2 keeps the reuse of a
// slot out of any interval that still reads it.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <numeric>
#include <string>
#include <thread>
#include <vector>
#include <cuda_runtime.h>
#include "fs_prod.cuh"
#include "fs_device.cuh"

namespace fsp {

constexpr double kFix = 1099511627776.0;           // 2^40
constexpr double kInvFix = 9.094947017729282e-13;  // 2^-40
constexpr uint32_t kThreads = 256;
constexpr uint32_t kTile = 256;  // post neurons advanced together (one per thread)
constexpr uint32_t kLB = 16;     // steps per NMDA pull batch
// posts per tile (FP64 tiles are half as wide so the per-tile buffers stay
// in static shared memory); per-tile buffers are step-major, [step][post],
// so the per-step reads of consecutive threads hit consecutive banks
template <class T>
struct TileW { static constexpr uint32_t W = sizeof(T) == 4 ? kTile : kTile / 2; };

enum { PL_NONE = 0, PL_STD = 1, PL_STP = 2, PL_TM = 3 };

struct Params {
  uint32_t n, slots, mask, interval, nlin;
  uint32_t dmax0;                        // every delay is 0 (single-step pull order)
  int lin_of_rec[4];
  const float *Vth, *El, *gl, *Cm, *Vreset, *df, *ef, *dVmax;
  const int32_t *RfPed, *SpiDy;
  const float *Vrev, *dfst, *nmda_dfxt, *nmda_efst, *nmda_as, *nmda_mg, *ext_g, *pb;
  const uint32_t *act;
  const float *inj_mean, *inj_std;
  const float *pdf;                      // [4n] decay of st_pre per linear receptor
  const float *p_dfxt, *p_dfst, *p_efas; // NMDA presynaptic kinetics
  const uint8_t *proj;                   // receptors a neuron projects with (bit r)
  int plast;
  const float *stp_pv, *stp_dfD, *stp_efD, *stp_aF, *stp_dfF, *stp_efF, *stp_aCap, *stp_dfCap,
      *stp_aCar, *stp_dfCar, *stp_efCar;
  const uint8_t *tm_on;
  const float *tm_U, *tm_dfr, *tm_dff;
  void *V, *G, *ext_st, *ext_x, *ext_s, *st_pre, *x_pre, *s_pre, *s_hist;
  int32_t *Count;
  uint32_t *NS;
  float *D, *F, *Cap, *Car, *tm_u, *tm_x;
  unsigned long long *ring;              // [nlin][n][S]
  const uint32_t *out_row, *out_code;
  const float *out_w;
  const uint32_t *in_row, *in_code;
  const float *in_w;
  const uint32_t *block_post;            // [blocks+1] post range of each block
  uint32_t key0, key1;
  uint64_t t0;
  uint32_t nsteps;
  uint32_t *bits;
  uint32_t words;
  uint32_t *counts;
  float *outV;
  unsigned int *bar;
  int *err;
  unsigned long long *spike_total;  // spikes since reset
  uint32_t *nspk;                   // per-neuron spike counts since reset (or null)
  float *Irep;                      // [5][n] receptor currents of each neuron's last integrated step
  float *outI;                      // [steps][5][n] Irep per step (or null)
  uint32_t *outNS;                  // [steps][n] LIF state word per step (or null)
  float rg[5];                      // synaptic gain per receptor (scales every weight; 1 = as built)
  // gap junctions (or null): terms of neuron p are [gap_row[p], gap_row[p+1])
  // (other neuron, conductance); Vg [2][n] holds V at the end of the last two
  // steps (parity of the step), which the next step's gap currents read
  const uint32_t *gap_row, *gap_other;
  const float *gap_w;
  void *Vg;
  // long-term plasticity (k_prod_ltp; null unless the network has LTP):
  // per neuron the trace LP and its delay counter with their parameters;
  // copies of the last two steps' LP, spike flag and presynaptic gates by
  // step parity (the LTP phase of step t - 1 reads them while the owners
  // advance step t); the LTP records of each neuron as presynaptic
  // (ltp_orow: entry = post | receptor << 24, index of its weight in out_w
  // or, for NMDA, in_w) and as postsynaptic (ltp_irow: pre | receptor <<
  // 24, index); the NMDA sums of a step ([n]) and the spike lists of the
  // last two steps (id, step slot, c per linear receptor; counts [2])
  void *ltp_lp;
  int32_t *ltp_clp;
  const float *ltp_dflp, *ltp_pos, *ltp_neg;
  const int32_t *ltp_spd;
  void *ltp_lp2, *ltp_sp2;
  uint8_t *ltp_spk2;
  const uint32_t *ltp_orow, *ltp_oent, *ltp_oidx, *ltp_irow, *ltp_ient, *ltp_iidx;
  void *ltp_gn;
  uint32_t *ltp_cnt, *ltp_id;
  uint16_t *ltp_tm;
  void *ltp_c;
  // single-step kernel k_prod1 (null unless the network takes it): per
  // block, the presynaptic neurons it tracks (sorted ids, NMDA kinetics
  // class, rows of their linear synapses onto the block's posts), the NMDA
  // in-edges of its posts as (tracked index, weight) in CSR order, and the
  // spike lists of the last two steps
  const struct Blk1 *b1;
  const uint32_t *t1_gid, *t1_lin, *t1_grow;
  const uint16_t *t1_lrow, *t1_perm;
  const uint8_t *t1_cls;
  const float *t1_linw, *t1_ew, *t1_cls_tab;
  const uint16_t *t1_eidx;
  const uint32_t *t1_bits;   // per block: bitmap of its tracked neurons' ids
  const uint16_t *t1_rank;   // per block: tracked neurons in the bitmap's earlier words
  uint32_t t1_ncls, t1_smem;
  // GatingVariable output (or null): selections of neuron p are entries
  // [gv_row[p], gv_row[p+1]) of gv_ent (output column | receptor << 28)
  void *gn_buf;          // tile kernels: NMDA sums of a batch of steps, [L][n]
  unsigned long long *phase;  // phase clock: [blocks][16] SM cycles per phase, or null
  const uint32_t *gv_row, *gv_ent;
  uint32_t gv_n;
  float *gv_st, *gv_xt;  // [steps][gv_n]
  uint32_t *t1_cnt;      // [4] overflow entries of step t, slot t mod 4
  uint32_t t1_slots;     // entries per block region of a step's list
  uint32_t t1_w;         // 16-byte words per list entry: 1 or 2
  uint4 *t1_list;        // [2][blocks][t1_slots][t1_w]: (id, inc, c, step + 1) when every neuron
                         // projects onto at most one linear receptor (c: that receptor's),
                         // else (id, inc, c0, c1), (c2, c3, step + 1, 0)
  uint4 *t1_ovf;         // [2][n][t1_w] the overflow lists
};

// Block plan of k_prod1: posts [post0, post0 + np); tracked neurons [trk0,
// trk0 + ntrk) of the per-tracked t1 arrays (their slots in t1_perm, their
// linear rows at lrow0, ntrk + 1 offsets); NMDA edge entries [e0, e0 + ne)
// (groups of four posts in rows of 32, the groups' first rows at grow0,
// (np + 3) / 4 + 1 of them); linear delivery entries from l0.
struct Blk1 {
  uint32_t post0, np, trk0, ntrk, lrow0, e0, ne, grow0, l0;
  uint32_t bm0, w0, nwd;  // bitmap: words [w0, w0 + nwd) of the id space, at t1_bits + bm0
  uint32_t s0, nslot;     // slot tables (t1_gid, t1_cls) at s0, nslot of them (a multiple of 32)
};

// ---- Philox-4x32-10 -------------------------------------------------------
__device__ __forceinline__ void philox(uint32_t c[4], uint32_t k0, uint32_t k1) {
#pragma unroll
  for (int r = 0; r < 10; r++) {
    const uint32_t hi0 = __umulhi(0xD2511F53u, c[0]), lo0 = 0xD2511F53u * c[0];
    const uint32_t hi1 = __umulhi(0xCD9E8D57u, c[2]), lo1 = 0xCD9E8D57u * c[2];
    const uint32_t n0 = hi1 ^ c[1] ^ k0, n2 = hi0 ^ c[3] ^ k1;
    c[0] = n0; c[1] = lo1; c[2] = n2; c[3] = lo0;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
}
__device__ __forceinline__ float u24(uint32_t x) { return (float)(x >> 8) * 5.9604644775390625e-08f; }

// Delay ring slot of (linear receptor index ri, post, slot): slot-major,
// [ri][slot][post], so the posts a warp advances read one slot's
// consecutive words.
__device__ __forceinline__ unsigned long long *ring_at(const Params &P, int ri, uint32_t post, uint32_t slot) {
  return P.ring + ((size_t)ri * P.slots + slot) * P.n + post;
}

// ---- bounded grid barrier ---------------------------------------------------
// Over the `count` blocks that share `bar` (the whole grid).  The first 8
// bytes of bar are a 64-bit arrival counter that the host zeroes before each
// launch and that only grows: barrier k of a launch is passed when the
// counter reaches k * count.  Each block's thread 0, after bar.sync (which
// orders the block's writes before it), adds its arrival with a release
// reduction and polls the counter with acquire loads; a load that sees the
// full count synchronises with every arrival (the reductions form one
// release sequence), and the closing bar.sync hands that on to the block.
// No block resets anything and there is no second hop through a
// generation word.  Every wait is bounded: after ~2^24 polls the block sets
// the error word and all blocks leave.  `target` is thread 0's count of the
// arrivals expected so far.
__device__ __forceinline__ unsigned long long ld_acquire_gpu(const unsigned long long *p) {
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void red_release_gpu(unsigned long long *p, unsigned long long v) {
  asm volatile("red.release.gpu.global.add.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

__device__ __forceinline__ bool arrive_and_wait(unsigned int *bar, int *err, uint32_t count,
                                                unsigned long long &target, unsigned int limit) {
  unsigned long long *ctr = (unsigned long long *)bar;
  target += count;
  red_release_gpu(ctr, 1ull);
  // the error word is looked at every 64 polls only: a load after an acquire
  // load waits for it, so checking it on every poll would double the time
  // between polls
  unsigned int spins = 0;
  while (ld_acquire_gpu(ctr) < target) {
    if ((++spins & 63u) == 0u) {
      if (*(volatile int *)err) return false;
      if (spins > limit) {
        atomicExch(err, 2);
        return false;
      }
    }
  }
  return true;
}

// A block leaves when thread 0's wait failed (its own limit, or the error
// word set by another block); thread 0 hands the outcome to the block
// through shared memory, so no thread reads global memory after the
// barrier.  A block that passed a barrier which another block gave up on
// finds the error word set while it waits at the next one (that block never
// arrives there), so every block leaves within 64 polls of the failure.
__device__ __forceinline__ bool grid_sync(unsigned int *bar, int *err, uint32_t count, unsigned long long &target,
                                          unsigned int limit = 1u << 24) {
  __shared__ int ok;
  __syncthreads();
  if (threadIdx.x == 0) ok = count > 1 ? arrive_and_wait(bar, err, count, target, limit) : 1;
  __syncthreads();
  return ok != 0;
}

// Loads of the NMDA s history may be served by L1 (ld.global.ca): a block
// reads only slots written in earlier intervals, and every interval ends
// with the grid barrier above, whose fences (release before the arrival,
// acquire after the wait, then bar.sync) order those writes before the
// reads in the PTX memory model; the vector windows of one edge and the
// edges of different posts that share a presynaptic neuron then hit L1.
template <class T>
__device__ __forceinline__ T ldhist_t(const T *p);
template <>
__device__ __forceinline__ float ldhist_t<float>(const float *p) { return __ldca(p); }
template <>
__device__ __forceinline__ double ldhist_t<double>(const double *p) { return __ldca(p); }

template <class T>
__device__ __forceinline__ T exp_t(T x);
template <>
__device__ __forceinline__ float exp_t<float>(float x) { return expf(x); }
template <>
__device__ __forceinline__ double exp_t<double>(double x) { return exp(x); }

template <class T>
__device__ __forceinline__ T fma_t(T a, T b, T c);
template <>
__device__ __forceinline__ float fma_t<float>(float a, float b, float c) { return __fmaf_rn(a, b, c); }
template <>
__device__ __forceinline__ double fma_t<double>(double a, double b, double c) { return __fma_rn(a, b, c); }

template <class T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(fsd::kFull, v, o);
  return v;
}

// ---- NMDA pull for L steps of a tile: gn[j][q] = sum_e w_e s_pre(tb+j-1-d_e)
// FP32: every neuron keeps its s history as 4 rows, row k shifted by k
// slots (row k, element i = slot (i + k) mod S).  The L consecutive values an
// edge needs then start on a 16-byte boundary of row (start mod 4), so they
// arrive as ceil(L/4) aligned vector loads with every value in a fixed
// register; each lane keeps four edges' loads in flight.
constexpr uint32_t kSH = 4;  // shifted copies of the s history (FP32)

__device__ __forceinline__ float comp4(const float4 &q, int k) {
  return k == 0 ? q.x : k == 1 ? q.y : k == 2 ? q.z : q.w;
}

// Lanes work in groups that each take one edge, lane k of a group loading
// vector k of the edge's window (steps 4k..4k+3), so one warp load covers a
// group's worth of edges whose vectors share a cache line per edge (about
// 1.25 L1 wavefronts per edge instead of 3 for a lane per edge); each lane
// keeps U edges in flight, and the next round's edge codes and weights are
// fetched while the current windows are in flight.  Networks whose interval
// is at most 12 steps (batches of at most 12 steps: three vectors) use
// triads, lanes 3g + k for g < 10 (lanes 30 and 31 idle), so a warp load
// covers ten edges; the others use quads, lanes 4g + k for g < 8.  Group g
// sums the post's edges g, g + G, g + 2G, ... (G = 10 or 8) in that order
// whatever U is (U only sets how many are in flight); then triads are
// combined in a fixed tree (g + 5 onto g, then g + 3, g + 2 and g + 1) and
// quads by an xor butterfly over the eight groups.  The group size depends
// on the network's interval alone, so the sums depend on neither U, the
// block plan, the kernel nor the length of a batch.
template <int U>
__device__ __forceinline__ void nmda_pull_f32(const Params &P, uint32_t p0, uint32_t np, uint64_t tb, uint32_t L,
                                              float (*gn)[kTile], uint32_t wid, uint32_t lane) {
  const float4 *sh = (const float4 *)P.s_hist;
  const uint32_t S4 = P.slots >> 2, qmask = S4 - 1, mask = P.mask;
  const uint32_t nvl = (L + 3u) >> 2;  // vectors needed for L steps
  const uint32_t nw = kThreads / 32;
  const bool tri = P.interval <= 12u;
  const uint32_t G = tri ? 10u : 8u;   // groups (edges per warp load)
  const uint32_t CH = G * U;           // edges per warp round
  const uint32_t g = tri ? lane / 3u : lane >> 2, k = tri ? lane - 3u * g : lane & 3u;
  const bool gv = g < G, kv = gv && k < nvl;
  uint32_t code[U];
  float w[U];
  auto fetch = [&](uint32_t base, uint32_t end) {
#pragma unroll
    for (int u = 0; u < U; u++) {
      const uint32_t eu = base + g + G * u;
      code[u] = gv && eu < end ? __ldg(P.in_code + eu) : 0u;
      w[u] = gv && eu < end ? __ldg(P.in_w + eu) : 0.0f;
    }
  };
  uint32_t q = wid, b0 = 0, b1 = 0;
  if (P.in_row && q < np) {
    b0 = __ldg(P.in_row + p0 + q);
    b1 = __ldg(P.in_row + p0 + q + 1);
    fetch(b0, b1);
  }
  for (; q < np; q += nw) {
    const uint32_t qn = q + nw;
    uint32_t n0 = 0, n1 = 0;
    if (P.in_row && qn < np) {
      n0 = __ldg(P.in_row + p0 + qn);
      n1 = __ldg(P.in_row + p0 + qn + 1);
    }
    float acc[4] = {0.0f, 0.0f, 0.0f, 0.0f};
    const uint32_t nch = (b1 - b0 + CH - 1) / CH;
    for (uint32_t c = 0; c < nch; c++) {
      const uint32_t e = b0 + c * CH + g;
      float4 v[U];
#pragma unroll
      for (int u = 0; u < U; u++) {
        const bool ok = kv && e + G * u < b1;
        const uint32_t pre = code[u] & 0xffffffu, d = code[u] >> 24;
        const uint32_t a = (uint32_t)(tb - 1u - d) & mask;
        const float4 *row = sh + ((size_t)pre * kSH + (a & 3u)) * S4;
        v[u] = ok ? __ldca(row + (((a >> 2) + k) & qmask)) : make_float4(0.f, 0.f, 0.f, 0.f);
      }
      float wc[U];
#pragma unroll
      for (int u = 0; u < U; u++) wc[u] = w[u];
      if (c + 1 < nch) fetch(b0 + (c + 1) * CH, b1);
      else if (qn < np) fetch(n0, n1);
#pragma unroll
      for (int u = 0; u < U; u++) {
        acc[0] += wc[u] * v[u].x;
        acc[1] += wc[u] * v[u].y;
        acc[2] += wc[u] * v[u].z;
        acc[3] += wc[u] * v[u].w;
      }
    }
    if (nch == 0 && qn < np) fetch(n0, n1);
    if (tri) {
      // g + 5 onto g (g < 5), g + 3 onto g (g < 2), then g + 2 and g + 1
      // onto g = 0: lane k ends with its four steps' sums
#pragma unroll
      for (int i = 0; i < 4; i++) {
        float t = __shfl_down_sync(fsd::kFull, acc[i], 15);
        if (g < 5u) acc[i] += t;
        t = __shfl_down_sync(fsd::kFull, acc[i], 9);
        if (g < 2u) acc[i] += t;
        t = __shfl_down_sync(fsd::kFull, acc[i], 6);
        if (g == 0u) acc[i] += t;
        t = __shfl_down_sync(fsd::kFull, acc[i], 3);
        if (g == 0u) acc[i] += t;
      }
    } else {
#pragma unroll
      for (int o = 4; o < 32; o <<= 1)
#pragma unroll
        for (int i = 0; i < 4; i++) acc[i] += __shfl_xor_sync(fsd::kFull, acc[i], o);
    }
    if (lane < (tri ? 3u : 4u)) {
#pragma unroll
      for (int i = 0; i < 4; i++) {
        const uint32_t j = 4u * lane + (uint32_t)i;
        if (j < L) gn[j][q] = acc[i];
      }
    }
    b0 = n0;
    b1 = n1;
  }
}

// Single-step pull of networks whose delays are all 0 (every network in the
// reference's own format): the eight lanes of a quarter warp sum one post,
// lane l of the quarter its edges l, l + 8, l + 16, ... in order (fused
// multiply-adds), then an xor butterfly over 4, 2, 1.  The single-step
// persistent kernel (k_prod1) sums its shared-memory copy of the same edges
// in the same order, so the two kernels, and a batch instance and its solo
// run, give the same sums bit for bit.
template <bool kMW = false>
__device__ __forceinline__ void nmda_pull1_f32(const Params &P, uint32_t p0, uint32_t np, uint64_t tb,
                                               float (*gn)[kTile], uint32_t wid, uint32_t lane) {
  const float *sh = (const float *)P.s_hist;
  const uint32_t S = P.slots, mask = P.mask;
  const uint32_t nw = kThreads / 32;
  if (!P.in_row) {
    for (uint32_t q = wid * 32 + lane; q < np; q += nw * 32) gn[0][q] = 0.0f;
    return;
  }
  const uint32_t slot = (uint32_t)(tb - 1u) & mask;
  const uint32_t h = lane >> 3, l8 = lane & 7u;
  for (uint32_t q0 = wid * 4u; q0 < np; q0 += nw * 4u) {
    const uint32_t q = q0 + h;
    const bool has = q < np;
    const uint32_t b0 = has ? __ldg(P.in_row + p0 + q) : 0u, b1 = has ? __ldg(P.in_row + p0 + q + 1) : 0u;
    float acc = 0.0f;
    for (uint32_t e = b0 + l8; e < b1; e += 8) {
      const uint32_t pre = __ldg(P.in_code + e) & 0xffffffu;
      // row 0 of the shifted copies holds slot i at element i
      const float w = kMW ? __ldcg(P.in_w + e) : __ldg(P.in_w + e);
      acc = __fmaf_rn(w, __ldca(sh + (size_t)pre * kSH * S + slot), acc);
    }
#pragma unroll
    for (int o = 4; o; o >>= 1) acc += __shfl_xor_sync(fsd::kFull, acc, o);
    if (l8 == 0 && has) gn[0][q] = acc;
  }
}

template <class T, bool kMW = false>
__device__ __forceinline__ void nmda_pull(const Params &P, uint32_t p0, uint32_t np, uint64_t tb, uint32_t L,
                                          T (*gn)[TileW<T>::W], uint32_t wid, uint32_t lane) {
  const T *sh = (const T *)P.s_hist;
  const uint32_t S = P.slots, mask = P.mask;
  const uint32_t nw = kThreads / 32;
  for (uint32_t q = wid; q < np; q += nw) {
    T acc[kLB];
#pragma unroll
    for (uint32_t j = 0; j < kLB; j++) acc[j] = (T)0;
    if (P.in_row) {
      const uint32_t p = p0 + q;
      const uint32_t e0 = __ldg(P.in_row + p), e1 = __ldg(P.in_row + p + 1);
      for (uint32_t e = e0 + lane; e < e1; e += 32) {
        const uint32_t code = __ldg(P.in_code + e);
        const T w = (T)(kMW ? __ldcg(P.in_w + e) : __ldg(P.in_w + e));
        const uint32_t pre = code & 0xffffffu, d = code >> 24;
        const T *row = sh + (size_t)pre * S;
        const uint32_t a = (uint32_t)(tb - 1u - d) & mask;
#pragma unroll
        for (uint32_t j = 0; j < kLB; j++)
          if (j < L) acc[j] += w * ldhist_t<T>(row + ((a + j) & mask));
      }
    }
#pragma unroll
    for (uint32_t j = 0; j < kLB; j++) {
      if (j < L) {
        const T v = warp_sum<T>(acc[j]);
        if (lane == j) gn[j][q] = v;
      }
    }
  }
}

// ---- spike pushes into the delay ring --------------------------------------
// Threads start, start+stride, ... of a group walk the out-edges of neuron q
// (four edges per thread per round, loads issued before the atomics) and add
// w*c[receptor] as 2^-40 fixed point to ring[receptor][post][(tm+delay) mod S].
// kMW: the weights change during the launch (LTP), so they are read
// through L2 rather than the read-only path.
template <class T, bool kMW = false>
__device__ __forceinline__ void push_spike(const Params &P, uint32_t q, uint32_t tm, const T (&cj)[4],
                                           uint32_t start, uint32_t stride) {
  const uint32_t mask = P.mask;
  const uint32_t ob = __ldg(P.out_row + q), oe = __ldg(P.out_row + q + 1);
  for (uint32_t e = ob + start; e < oe; e += 4 * stride) {
    uint32_t code[4];
    float w[4];
#pragma unroll
    for (int u = 0; u < 4; u++) {
      const uint32_t eu = e + u * stride;
      code[u] = eu < oe ? __ldg(P.out_code + eu) : 0u;
      w[u] = eu < oe ? (kMW ? __ldcg(P.out_w + eu) : __ldg(P.out_w + eu)) : 0.0f;
    }
#pragma unroll
    for (int u = 0; u < 4; u++) {
      if (e + u * stride < oe) {
        const uint32_t post = code[u] & 0x3fffffu, r = (code[u] >> 22) & 3u, d = code[u] >> 24;
        const T cv = ((r == 0) ? cj[0] : (r == 1) ? cj[1] : (r == 2) ? cj[2] : cj[3]) * (T)P.rg[r];
        const long long fx = __double2ll_rn((double)((T)w[u] * cv) * kFix);
        const int ri = P.lin_of_rec[r];
        atomicAdd(ring_at(P, ri, post, (tm + d) & mask), (unsigned long long)fx);
      }
    }
  }
}

// spikes of a block awaiting their push (shared memory)
template <class T>
struct SpikeList {
  uint32_t *n, *p;
  uint16_t *tm;
  T (*c)[4];
  uint32_t cap;
};

// ---- drive draws -----------------------------------------------------------
// The external Bernoulli outcomes (bit r: receptor r hit this step) and the
// injection noise of neuron p at step t depend on no state: Philox block 0
// keyed by (t, p) gives the four linear receptors' uniforms, block 1 (drawn
// only for a neuron with NMDA drive or injection) the NMDA uniform and the
// Box-Muller pair.
template <class T>
__device__ __forceinline__ uint32_t draw_one(const Params &P, uint32_t p, uint64_t t, T &gauss) {
  const uint32_t n = P.n;
  const uint32_t a = __ldg(P.act + p);
  uint32_t rnd[4] = {(uint32_t)t, (uint32_t)(t >> 32), p, 0u};
  philox(rnd, P.key0, P.key1);
  uint32_t h = 0;
#pragma unroll
  for (int r = 0; r < 4; r++)
    if (__ldg(P.pb + (size_t)r * n + p) > u24(rnd[r])) h |= 1u << r;
  // a drive probability that is not positive never draws a hit
  const float pbn = __ldg(P.pb + (size_t)FS_NMDA * n + p);
  if (((a & FS_ACT_NMDA) && pbn > 0.0f) || (a & FS_ACT_INJ)) {
    uint32_t r2[4] = {(uint32_t)t, (uint32_t)(t >> 32), p, 1u};
    philox(r2, P.key0, P.key1);
    if (pbn > u24(r2[0])) h |= 1u << FS_NMDA;
    if (a & FS_ACT_INJ) {  // Box-Muller normal
      const double u1 = ((double)(r2[1] >> 8) + 1.0) * 5.9604644775390625e-08;
      const double u2 = (double)(r2[2] >> 8) * 5.9604644775390625e-08;
      const double z = sqrt(-2.0 * log(u1)) * cospi(2.0 * u2);
      gauss = fma_t<T>((T)__ldg(P.inj_std + p), (T)z, (T)__ldg(P.inj_mean + p));
    }
  }
  return h;
}

// Draws of L steps for a tile, by all threads at once, off the neurons'
// per-step dependency chain.
template <class T>
__device__ __forceinline__ void draw_inputs(const Params &P, uint32_t p0, uint32_t np, uint64_t tb, uint32_t L,
                                            uint8_t (*hits)[TileW<T>::W], T (*gauss)[TileW<T>::W]) {
  for (uint32_t idx = threadIdx.x; idx < np * L; idx += kThreads) {
    const uint32_t j = idx / np, q = idx - j * np;
    T gv = (T)0;
    hits[j][q] = (uint8_t)draw_one<T>(P, p0 + q, tb + j, gv);
    gauss[j][q] = gv;
  }
}

// ---- phase clock (debug aid) -------------------------------------------------
// When P.phase is set, thread 0 of each block adds the SM cycles between
// consecutive marks to its block's counter k (a relaxed add per mark).
constexpr uint32_t kPhaseSlots = 16;  // counters per block
struct PhaseClock {
  unsigned long long *out;
  long long t;
  __device__ __forceinline__ void start(const Params &P) {
    out = (P.phase && threadIdx.x == 0) ? P.phase + (size_t)blockIdx.x * kPhaseSlots : nullptr;
    if (out) t = clock64();
  }
  // adds the cycles since the last mark to counter k and restarts the count
  __device__ __forceinline__ void mark(int k) {
    if (out) {
      const long long now = clock64();
      atomicAdd(out + k, (unsigned long long)(now - t));
      t = now;
    }
  }
  // adds the cycles since the last mark to counter k once `dep` is known
  // (a branch on it comes first), without restarting the count; `dep` is
  // never 0xffffffff at a call
  __device__ __forceinline__ void lap(int k, uint32_t dep = 0u) {
    if (out && dep != 0xffffffffu) atomicAdd(out + k, (unsigned long long)(clock64() - t));
  }
};

// ---- one neuron's step (shared by every kernel) ----------------------------
// Parameters and state of one neuron, held in registers while its thread
// advances it; the per-step arithmetic below is the single definition used
// by the interval kernel (k_prod / k_prod_batch) and the single-step kernel
// (k_prod1), so the two give bit-identical neurons.
constexpr uint8_t kPjTM = 0x80;  // NeuronPar::pj: Tsodyks-Markram plasticity on (next to the receptor bits)

template <class T>
struct NeuronPar {
  uint32_t a;
  uint8_t pj;  // bit r: the neuron projects onto receptor r; kPjTM
  int32_t rf, sd;
  T vth, vreset, df, ef, dvm;
  T icm;   // 1e-3 / Cm: the membrane current's scale (one division per launch, not per step)
  T leak;
  T mg;    // Mg / 3.57 of the NMDA Mg block
  T vrev[5], dfs[5], extg[5];
  T ndfxt, nefas;
  T pdf[4];
  T pdfxt, pdfst, pefas;
};

template <class T>
struct NeuronState {
  T V;
  int32_t cnt;
  uint32_t ns;
  T G[4], est[4], sp[4];
  T ex, es, xp, spre;
  float tmu, tmx;  // Tsodyks-Markram u, x (float between steps)
};

// kTM = false: the caller never runs a Tsodyks-Markram network (no
// registers are spent on its state).
template <class T, bool kTM = true>
__device__ __forceinline__ void load_neuron(const Params &P, uint32_t p, NeuronPar<T> &q, NeuronState<T> &st) {
  const uint32_t n = P.n;
  q.a = P.act[p];
  q.pj = P.proj[p];
  q.rf = __ldg(P.RfPed + p);
  q.sd = __ldg(P.SpiDy + p);
  q.vth = (T)__ldg(P.Vth + p);
  q.vreset = (T)__ldg(P.Vreset + p);
  q.df = (T)__ldg(P.df + p);
  q.ef = (T)__ldg(P.ef + p);
  q.dvm = (T)__ldg(P.dVmax + p);
  q.icm = (T)1e-3 / (T)__ldg(P.Cm + p);
  q.leak = (T)__ldg(P.gl + p) * (T)__ldg(P.El + p) * (T)1e3;
  q.mg = (T)__ldg(P.nmda_mg + p) / (T)3.57;
#pragma unroll
  for (int r = 0; r < 5; r++) {
    q.vrev[r] = (T)__ldg(P.Vrev + (size_t)r * n + p);
    q.dfs[r] = (T)__ldg(P.dfst + (size_t)r * n + p);
    q.extg[r] = (T)__ldg(P.ext_g + (size_t)r * n + p);
  }
  q.ndfxt = (T)__ldg(P.nmda_dfxt + p);
  q.nefas = (T)__ldg(P.nmda_efst + p) * (T)__ldg(P.nmda_as + p);
#pragma unroll
  for (int r = 0; r < 4; r++) q.pdf[r] = (T)__ldg(P.pdf + (size_t)r * n + p);
  q.pdfxt = (T)__ldg(P.p_dfxt + p);
  q.pdfst = (T)__ldg(P.p_dfst + p);
  q.pefas = (T)__ldg(P.p_efas + p);
  // the Tsodyks-Markram state lives in registers for the launch (or batch;
  // its parameters are read-only loads of each step); a neuron without
  // projections has no presynaptic state
  st.tmu = st.tmx = 0.0f;
  if (kTM && P.plast == PL_TM && q.pj && P.tm_on[p]) {
    q.pj |= kPjTM;
    st.tmu = P.tm_u[p];
    st.tmx = P.tm_x[p];
  }
  st.V = ((T *)P.V)[p];
  st.cnt = P.Count[p];
  st.ns = P.NS[p];
#pragma unroll
  for (int r = 0; r < 4; r++) {
    st.G[r] = ((T *)P.G)[(size_t)r * n + p];
    st.est[r] = ((T *)P.ext_st)[(size_t)r * n + p];
    st.sp[r] = ((T *)P.st_pre)[(size_t)r * n + p];
  }
  st.ex = ((T *)P.ext_x)[p];
  st.es = ((T *)P.ext_s)[p];
  st.xp = ((T *)P.x_pre)[p];
  st.spre = ((T *)P.s_pre)[p];
}

template <class T, bool kTM = true>
__device__ __forceinline__ void store_neuron(const Params &P, uint32_t p, const NeuronPar<T> &q,
                                             const NeuronState<T> &st) {
  const uint32_t n = P.n;
  if (kTM && (q.pj & kPjTM)) {
    P.tm_u[p] = st.tmu;
    P.tm_x[p] = st.tmx;
  }
  ((T *)P.V)[p] = st.V;
  P.Count[p] = st.cnt;
  P.NS[p] = st.ns;
#pragma unroll
  for (int r = 0; r < 4; r++) {
    ((T *)P.G)[(size_t)r * n + p] = st.G[r];
    ((T *)P.ext_st)[(size_t)r * n + p] = st.est[r];
    ((T *)P.st_pre)[(size_t)r * n + p] = st.sp[r];
  }
  ((T *)P.ext_x)[p] = st.ex;
  ((T *)P.ext_s)[p] = st.es;
  ((T *)P.x_pre)[p] = st.xp;
  ((T *)P.s_pre)[p] = st.spre;
}

// NMDA presynaptic kinetics of one step (code/EqsGnl2.cpp:493): x jumps by
// inc on a spike and decays otherwise, s follows with its (1 - s)
// saturation.  The neuron's owner and every block that tracks a copy of it
// (k_prod1) call this one function with the same operands.
template <class T>
__device__ __forceinline__ void nmda_pre_step(T &xp, T &spre, bool spk, T inc, T pdfxt, T pdfst, T pefas) {
  xp = spk ? xp + inc : xp * pdfxt;
  spre = fma_t<T>(pdfst, spre, (pefas * xp) * ((T)1 - spre));
}

// Long-term plasticity trace of one neuron (k_prod_ltp): LP and its
// back-propagation delay counter, with their parameters.  LP is float in
// both modes, as the reference keeps it, so the weights LTP writes depend
// only on the spike times (FP32 and FP64 runs rewrite them alike).
template <class T>
struct LtpTrace {
  float lp, dflp;
  int32_t clp, spd;
};

// One step of neuron p: fold the linear conductances' delivered sums
// (rv: 2^-40 fixed point) into G, add the external drive (hit bits, injection
// current) and the NMDA sum gnmda, VmEul + firing (code/EqsGnl2.cpp:152-251),
// per-step outputs of step s, then the presynaptic state: the increment inc of
// a spike and, per linear receptor, c = inc + st(t-1)(1 - df) for the push.
// kLTP: also the LP trace of a neuron with LTP on (lt; firLP and ltpEul,
// code/EqsGnl2.cpp:207-216, :254-280).  Returns whether the neuron spiked.
template <class T, bool kTM = true, bool kLTP = false>
__device__ __forceinline__ bool neuron_step(const Params &P, const NeuronPar<T> &q, NeuronState<T> &st,
                                            const long long (&rv)[4], T gnmda, uint32_t hit, T gauss, T gapI,
                                            uint32_t p, bool own, uint32_t s, T (&cinc)[4], T &inc_out,
                                            const float *tm = nullptr, LtpTrace<T> *lt = nullptr) {
  const uint32_t n = P.n;
  T g[5];
#pragma unroll
  for (int r = 0; r < 4; r++) {
    g[r] = (T)0;
    if (P.lin_of_rec[r] >= 0) {
      st.G[r] = fma_t<T>(q.dfs[r], st.G[r], (T)rv[r] * (T)kInvFix);  // exact power-of-two scale
      g[r] = st.G[r];
    }
  }
  g[FS_NMDA] = gnmda * (T)P.rg[FS_NMDA];
  // external drive (BgInit): bit r of hit = receptor r's Bernoulli outcome
  const uint32_t bitsr[4] = {FS_ACT_AMPA, FS_ACT_GABA, FS_ACT_ACH, FS_ACT_GCL};
#pragma unroll
  for (int r = 0; r < 4; r++) {
    if (q.a & bitsr[r]) {
      st.est[r] = (hit & (1u << r)) ? st.est[r] + (T)1 : st.est[r] * q.dfs[r];
      g[r] = fma_t<T>(q.extg[r], st.est[r], g[r]);
    }
  }
  T isyn = (T)0;
  if (q.a & FS_ACT_NMDA) {
    st.ex = (hit & (1u << FS_NMDA)) ? st.ex + (T)1 : st.ex * q.ndfxt;
    st.es = fma_t<T>(q.dfs[FS_NMDA], st.es, (q.nefas * st.ex) * ((T)1 - st.es));
    g[FS_NMDA] = fma_t<T>(q.extg[FS_NMDA], st.es, g[FS_NMDA]);
  }
  if (q.a & FS_ACT_INJ) isyn = gauss;
  if (P.gap_row) isyn = isyn + gapI;  // steps of networks with gap junctions come one at a time
  // VmEul + firing (code/EqsGnl2.cpp:152-251); the production modes scale
  // the Mg block and the current by per-neuron constants formed once
  // (Mg / 3.57, 1e-3 / Cm), where the reference divides every step: two
  // divisions off each step's dependency chain (775 -> 664 SM cycles per
  // step for one warp), at a rounding difference the FP32 and FP64 modes
  // share
  uint32_t ns = st.ns;
  bool fire_now = false;
  if (ns & FS_NS_FIRE) {
    fire_now = true;
  } else {
    const T v = st.V;
    const T Ir0 = g[FS_AMPA] * (q.vrev[FS_AMPA] - v);
    const T Ir1 = g[FS_GABA] * (q.vrev[FS_GABA] - v);
    const T Ir2 = g[FS_NMDA] * (q.vrev[FS_NMDA] - v) / ((T)1 + q.mg * exp_t<T>((T)-0.062 * v));
    const T Ir3 = g[FS_ACH] * (q.vrev[FS_ACH] - v);
    const T Ir4 = g[FS_GCL] * (q.vrev[FS_GCL] - v);
    T I = fma_t<T>(isyn, (T)1e3, Ir0 + Ir1 + Ir2 + Ir3 + Ir4) + q.leak;
    I = I * q.icm;
    if (I > q.dvm) {
      I = q.dvm;
      ns = (ns | FS_NS_MEMDV_OVF) & ~FS_NS_MEMDV_UDF;
    } else if (I < -q.dvm) {
      I = -q.dvm;
      ns = (ns & ~FS_NS_MEMDV_OVF) | FS_NS_MEMDV_UDF;
    } else {
      ns &= ~(FS_NS_MEMDV_OVF | FS_NS_MEMDV_UDF);
    }
    st.V = fma_t<T>(q.df, v, q.ef * I);
    if (P.outI && own) {  // kept only while requested (code/EqsGnl2.cpp:196-206)
      P.Irep[p] = (float)Ir0;
      P.Irep[(size_t)n + p] = (float)Ir1;
      P.Irep[(size_t)FS_NMDA * n + p] = (float)Ir2;
      P.Irep[(size_t)FS_ACH * n + p] = (float)Ir3;
      P.Irep[(size_t)FS_GCL * n + p] = (float)Ir4;
    }
    if (st.V > q.vth) {
      ns |= FS_NS_FIRE;
      fire_now = true;
      if constexpr (kLTP) {
        if (q.a & FS_ACT_LTP) ns |= FS_NS_LP_FIRE;
      }
    }
  }
  if (fire_now) {
    if (st.cnt < q.rf) {
      st.V = (st.cnt == 0) ? (T)0 : q.vreset;
      if (st.cnt == q.sd) ns |= FS_NS_SPIKE;
      else ns &= ~FS_NS_SPIKE;
      st.cnt++;
    } else {
      st.cnt = 0;
      ns &= ~FS_NS_FIRE;
    }
  }
  if constexpr (kLTP) {
    if (q.a & FS_ACT_LTP) {  // firLP + ltpEul
      if (ns & FS_NS_LP_FIRE) {
        if (lt->clp == lt->spd) {
          ns = (ns | FS_NS_LP_SPIKE) & ~FS_NS_LP_FIRE;
          lt->clp = 0;
        } else {
          ns &= ~FS_NS_LP_SPIKE;
          lt->clp++;
        }
      } else {
        ns &= ~FS_NS_LP_SPIKE;
      }
      lt->lp = (ns & FS_NS_LP_SPIKE) ? __fadd_rn(lt->lp, 1.0f) : __fmul_rn(lt->dflp, lt->lp);
    }
  }
  st.ns = ns;
  if (own && P.outV) P.outV[(size_t)s * n + p] = (float)st.V;
  if (own && P.outNS) P.outNS[(size_t)s * n + p] = ns;
  if (own && P.outI)
#pragma unroll
    for (int r = 0; r < 5; r++) P.outI[(size_t)s * 5 * n + (size_t)r * n + p] = P.Irep[(size_t)r * n + p];
  const bool spk = own && (ns & FS_NS_SPIKE) != 0;
  // presynaptic state: increment per spike, then plasticity update
#pragma unroll
  for (int r = 0; r < 4; r++) cinc[r] = (T)0;
  T inc = (T)1;
  if (q.pj && own) {
    if (P.plast == PL_STD) inc = (T)P.D[p];
    else if (P.plast == PL_STP) inc = (T)P.D[p] * (T)P.F[p];
    else if (kTM && (q.pj & kPjTM)) {
      T u = (T)st.tmu, x = (T)st.tmx;
      // parameters from the caller's per-thread copy (tm: U, dff, dfr) or
      // from global memory
      const T U = (T)(tm ? tm[0] : __ldg(P.tm_U + p));
      if (spk) {
        u = u + U * ((T)1 - u);
        const T rel = u * x;
        inc = rel;
        x = x - rel;
      } else {
        u = U + (u - U) * (T)(tm ? tm[1] : __ldg(P.tm_dff + p));
        x = (T)1 + (x - (T)1) * (T)(tm ? tm[2] : __ldg(P.tm_dfr + p));
      }
      st.tmu = (float)u;
      st.tmx = (float)x;
    }
#pragma unroll
    for (int r = 0; r < 4; r++) {
      if (q.pj & (1u << r)) {
        if (spk) {
          cinc[r] = inc + st.sp[r] * ((T)1 - q.pdf[r]);
          st.sp[r] = st.sp[r] + inc;
        } else {
          st.sp[r] = st.sp[r] * q.pdf[r];
        }
      }
    }
    if (q.pj & (1u << FS_NMDA)) nmda_pre_step<T>(st.xp, st.spre, spk, inc, q.pdfxt, q.pdfst, q.pefas);
    if (P.plast == PL_STD) {
      P.D[p] = spk ? P.D[p] * (1.0f - P.stp_pv[p]) : P.stp_dfD[p] * P.D[p] + P.stp_efD[p];
    } else if (P.plast == PL_STP) {
      float Dv = P.D[p], Fv = P.F[p], Cp = P.Cap[p], Cr = P.Car[p];
      if (spk) {
        Cr += P.stp_aCar[p];
        Cp += P.stp_aCap[p];
        Fv += (Cp + Cr) * (1.0f - Fv) * P.stp_aF[p];
        Dv *= (1.0f - P.stp_pv[p] * Fv);
      } else {
        Cr = P.stp_dfCar[p] * Cr + P.stp_efCar[p];
        Cp = P.stp_dfCap[p] * Cp;
        Fv = P.stp_dfF[p] * Fv + P.stp_efF[p] * (Cp + Cr) * (1.0f - Fv) * P.stp_aF[p];
        Dv = P.stp_dfD[p] * Dv + P.stp_efD[p];
      }
      P.D[p] = Dv; P.F[p] = Fv; P.Cap[p] = Cp; P.Car[p] = Cr;
    }
  }
  inc_out = inc;
  return spk;
}

// Spike outputs of a warp's step: the per-step bitmap and count, the total.
// total = false: the caller adds its spikes to the total itself (once).
__device__ __forceinline__ void spike_outputs(const Params &P, uint32_t m, bool spk, uint32_t p, uint32_t s,
                                              uint32_t lane, bool total = true) {
  if (spk && P.bits) atomicOr(P.bits + (size_t)s * P.words + (p >> 5), 1u << (p & 31));
  if (lane == 0) {
    if (P.counts) atomicAdd(P.counts + s, (unsigned)__popc(m));
    if (total) atomicAdd(P.spike_total, (unsigned long long)__popc(m));
  }
}

// GatingVariable columns of neuron p after step s: a single-target record's
// gate is its presynaptic neuron's gate of the receptor; NMDA records take
// the neuron's x and s (code/NetSimGnl2_info.cpp:701-758 prints st, and xt
// for NMDA).
template <class T>
__device__ __forceinline__ void gv_write(const Params &P, uint32_t p, uint32_t s, const NeuronState<T> &st) {
  for (uint32_t e = __ldg(P.gv_row + p), e1 = __ldg(P.gv_row + p + 1); e < e1; e++) {
    const uint32_t code = __ldg(P.gv_ent + e), col = code & 0x0fffffffu, r = code >> 28;
    const size_t o = (size_t)s * P.gv_n + col;
    if (r == FS_NMDA) {
      P.gv_st[o] = (float)st.spre;
      P.gv_xt[o] = (float)st.xp;
    } else {
      P.gv_st[o] = (float)(r == 0 ? st.sp[0] : r == 1 ? st.sp[1] : r == 2 ? st.sp[2] : st.sp[3]);
      P.gv_xt[o] = 0.0f;
    }
  }
}

// ---- L steps of a tile's neurons (thread per neuron), with the pushes ----
// Per-neuron parameters and state stay in registers for the L steps; the
// ring slots of the next PD steps are in flight while the current step
// computes (they are final: every push into them happened before the
// interval began); a warp pushes the spikes of its own lanes, so a step
// needs no block barrier.  neuron_load issues a thread's loads (parameters,
// state, Tsodyks-Markram parameters into its shared-memory copy, the first
// ring slots).  (Issuing them before the batch's drive draws, to overlap
// the draws, measured the same on the 1 M network: 0.7538 -> 0.7541.)
template <class T>
struct StepRegs {
  NeuronPar<T> q;
  NeuronState<T> st;
  long long rv[4], rv2[4];  // ring slots of the first steps (step 0, step 1)
};

template <class T, int PD>
__device__ __forceinline__ void neuron_load(const Params &P, uint32_t p0, uint32_t np, uint32_t sb, uint32_t L,
                                            StepRegs<T> &R, float *tm3) {
  static_assert(PD == 1 || PD == 2, "ring prefetch distance 1 or 2");
  const uint32_t tid = threadIdx.x, mask = P.mask;
  const bool own = tid < np;
  const uint32_t p = own ? p0 + tid : p0;  // non-owners read a valid neuron, write nothing
  load_neuron<T>(P, p, R.q, R.st);
  if (R.q.pj & kPjTM) {
    tm3[3 * tid] = P.tm_U[p];
    tm3[3 * tid + 1] = P.tm_dff[p];
    tm3[3 * tid + 2] = P.tm_dfr[p];
  }
  const uint32_t tprev = (uint32_t)(P.t0 + sb - 1u) & mask, tn = (uint32_t)(P.t0 + sb) & mask;
#pragma unroll
  for (int r = 0; r < 4; r++) {
    const int ri = P.lin_of_rec[r];
    R.rv[r] = (ri >= 0 && own) ? (long long)__ldcg(ring_at(P, ri, p, tprev)) : 0ll;
    R.rv2[r] = (PD == 2 && ri >= 0 && own && L > 1) ? (long long)__ldcg(ring_at(P, ri, p, tn)) : 0ll;
  }
}

// The L steps of neuron_load's neuron; tm3: the thread's Tsodyks-Markram
// parameters (read every step from shared memory rather than from global
// memory on the step's dependency chain).
template <class T, int PD, bool kLTP = false>
__device__ __forceinline__ void neuron_steps(const Params &P, uint32_t p0, uint32_t np, uint32_t sb, uint32_t L,
                                             T (*gn)[TileW<T>::W], const uint8_t (*hits)[TileW<T>::W],
                                             const T (*gauss)[TileW<T>::W], const SpikeList<T> &lst,
                                             const T *gapI, StepRegs<T> &R, const float *tm3) {
  const uint32_t tid = threadIdx.x, lane = tid & 31;
  const uint32_t n = P.n, S = P.slots, mask = P.mask;
  const bool own = tid < np;
  const uint32_t p = own ? p0 + tid : p0;
  NeuronPar<T> &q = R.q;
  NeuronState<T> &st = R.st;
  long long(&rv)[4] = R.rv, (&rv2)[4] = R.rv2;
  uint32_t nsp = 0;
  LtpTrace<T> lt;
  if constexpr (kLTP) {
    lt.lp = ((float *)P.ltp_lp)[p];
    lt.clp = P.ltp_clp[p];
    lt.dflp = __ldg(P.ltp_dflp + p);
    lt.spd = __ldg(P.ltp_spd + p);
  }
  for (uint32_t j = 0; j < L; j++) {
    const uint32_t s = sb + j;
    const uint64_t t = P.t0 + s;
    const uint32_t tm = (uint32_t)t & mask, tprev = (uint32_t)(t - 1u) & mask;
    // the slots this step folds in; the ones of step j + PD go in flight
    long long cur[4];
#pragma unroll
    for (int r = 0; r < 4; r++) {
      cur[r] = rv[r];
      const int ri = P.lin_of_rec[r];
      if (ri >= 0) {
        if (own && rv[r]) __stcg(ring_at(P, ri, p, tprev), 0ull);
        if constexpr (PD == 2) {
          rv[r] = rv2[r];
          rv2[r] = (own && j + 2 < L) ? (long long)__ldcg(ring_at(P, ri, p, (tm + 1u) & mask)) : 0ll;
        } else {
          rv[r] = (own && j + 1 < L) ? (long long)__ldcg(ring_at(P, ri, p, tm)) : 0ll;
        }
      }
    }
    const uint32_t qs = tid < np ? tid : 0;
    T cinc[4], inc;
    const bool spk = neuron_step<T, true, kLTP>(P, q, st, cur, gn[j][qs], hits[j][qs], gauss[j][qs],
                                                P.gap_row ? gapI[qs] : (T)0, p, own, s, cinc, inc, tm3 + 3 * tid,
                                                &lt);
    nsp += spk ? 1u : 0u;
    if constexpr (kLTP) {
      // what the LTP phase of this step reads while the owners run the next
      if (own) {
        const uint32_t par = (uint32_t)t & 1u;
        ((float *)P.ltp_lp2)[(size_t)par * n + p] = lt.lp;
        P.ltp_spk2[(size_t)par * n + p] = spk ? 1 : 0;
#pragma unroll
        for (int r = 0; r < 4; r++) ((T *)P.ltp_sp2)[((size_t)par * 4 + r) * n + p] = st.sp[r];
      }
    }
    if (own && P.gv_row) gv_write<T>(P, p, s, st);
    if (own && (q.pj & (1u << FS_NMDA))) {
      if constexpr (sizeof(T) == 4) {
#pragma unroll
        for (uint32_t k = 0; k < kSH; k++)
          __stcg((T *)P.s_hist + ((size_t)p * kSH + k) * S + ((tm - k) & mask), st.spre);
      } else {
        __stcg((T *)P.s_hist + (size_t)p * S + tm, st.spre);
      }
    }
    // spikes of this warp: outputs, and the spike list the block pushes at
    // the end of the batch (a push lands >= min_delay steps ahead, so it may
    // wait until the interval's end); a full list falls back to a push by
    // this warp right away
    uint32_t m = __ballot_sync(fsd::kFull, spk);
    if (m) {
      spike_outputs(P, m, spk, p, s, lane);
      bool listed = false;
      if (spk) {
        const uint32_t k = atomicAdd(lst.n, 1u);
        if (k < lst.cap) {
          lst.p[k] = p;
          lst.tm[k] = (uint16_t)tm;
#pragma unroll
          for (int r = 0; r < 4; r++) lst.c[k][r] = cinc[r];
          listed = true;
        }
      }
      uint32_t over = __ballot_sync(fsd::kFull, spk && !listed);
      while (over) {
        const int jl = __ffs(over) - 1;
        over &= over - 1;
        const uint32_t qq = __shfl_sync(fsd::kFull, p, jl);
        T cj[4];
#pragma unroll
        for (int r = 0; r < 4; r++) cj[r] = __shfl_sync(fsd::kFull, cinc[r], jl);
        push_spike<T>(P, qq, tm, cj, lane, 32);
      }
    }
  }
  if (own) {
    store_neuron<T>(P, p, q, st);
    if (P.gap_row) ((T *)P.Vg)[(size_t)((P.t0 + sb) & 1u) * n + p] = st.V;
    if (P.nspk && nsp) P.nspk[p] += nsp;
    if constexpr (kLTP) {
      ((float *)P.ltp_lp)[p] = lt.lp;
      P.ltp_clp[p] = lt.clp;
    }
  }
}

// Shared-memory buffers of one tile (the posts a block advances together).
template <class T>
struct TileBufs {
  static constexpr uint32_t kT = TileW<T>::W;
  static constexpr uint32_t kCap = sizeof(T) == 4 ? 320 : 192;
  T gn[kLB][kT];
  T gauss[kLB][kT];
  T gapI[kT];
  uint8_t hits[kLB][kT];
  uint32_t l_n, l_p[kCap];
  uint16_t l_tm[kCap];
  T l_c[kCap][4];
};

// NMDA sums of L steps for a tile's posts into B.gn.
template <class T, int PU>
__device__ __forceinline__ void tile_pull(const Params &P, uint32_t tp0, uint32_t np, uint32_t bs, uint32_t L,
                                          TileBufs<T> &B) {
  const uint32_t tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  if constexpr (sizeof(T) == 4) {
    if (P.dmax0) nmda_pull1_f32(P, tp0, np, P.t0 + bs, (float (*)[kTile])B.gn, wid, lane);
    else nmda_pull_f32<PU>(P, tp0, np, P.t0 + bs, L, (float (*)[kTile])B.gn, wid, lane);
  } else {
    nmda_pull<T>(P, tp0, np, P.t0 + bs, L, B.gn, wid, lane);
  }
}

// Gap currents of step bs of a tile's posts (interval 1): g (V_other -
// V_self) over V at the end of the previous step (none before the first).
template <class T>
__device__ __forceinline__ void tile_gap(const Params &P, uint32_t tp0, uint32_t np, uint32_t bs, T *gapI) {
  const uint64_t t = P.t0 + bs;
  for (uint32_t q = threadIdx.x; q < np; q += kThreads) {
    T acc = (T)0;
    if (t > 0) {
      const T *vp = (const T *)P.Vg + (size_t)((t - 1u) & 1u) * P.n;
      const uint32_t pq = tp0 + q;
      const T vs = __ldcg(vp + pq);
      for (uint32_t e = __ldg(P.gap_row + pq), e1 = __ldg(P.gap_row + pq + 1); e < e1; e++)
        acc = acc + (T)__ldg(P.gap_w + e) * (__ldcg(vp + __ldg(P.gap_other + e)) - vs);
    }
    gapI[q] = acc;
  }
}

// The rest of a tile's batch of L steps once its NMDA sums are in B.gn: the
// drive draws, gap currents, the neurons' steps and the spikes' pushes.
template <class T, int PD>
__device__ __forceinline__ void tile_steps(const Params &P, uint32_t tp0, uint32_t np, uint32_t bs, uint32_t L,
                                           TileBufs<T> &B, PhaseClock &pc) {
  constexpr uint32_t kCap = TileBufs<T>::kCap;
  const SpikeList<T> lst{&B.l_n, B.l_p, B.l_tm, B.l_c, kCap};
  const uint32_t tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  // warps without neurons in this tile skip the steps
  const bool act = (tid & ~31u) < np;
  __shared__ float tm3[kThreads * 3];
  StepRegs<T> R;
  draw_inputs<T>(P, tp0, np, P.t0 + bs, L, B.hits, B.gauss);
  if (P.gap_row) tile_gap<T>(P, tp0, np, bs, B.gapI);
  __syncthreads();
  pc.mark(1);
  if (act) neuron_load<T, PD>(P, tp0, np, bs, L, R, tm3);
  if (act) neuron_steps<T, PD>(P, tp0, np, bs, L, B.gn, B.hits, B.gauss, lst, B.gapI, R, tm3);
  __syncthreads();
  pc.mark(2);
  // the batch's spikes: with fewer spikes than warps the whole block
  // walks each spike's out-edges (a hub's hundreds of edges in one or
  // two rounds); with more, one spike per warp, eight in flight
  const uint32_t nl = min(B.l_n, kCap);
  if (nl < kThreads / 32) {
    for (uint32_t k = 0; k < nl; k++) {
      T cj[4];
#pragma unroll
      for (int r = 0; r < 4; r++) cj[r] = B.l_c[k][r];
      push_spike<T>(P, B.l_p[k], B.l_tm[k], cj, tid, kThreads);
    }
  } else {
    for (uint32_t k = wid; k < nl; k += kThreads / 32) {
      T cj[4];
#pragma unroll
      for (int r = 0; r < 4; r++) cj[r] = B.l_c[k][r];
      push_spike<T>(P, B.l_p[k], B.l_tm[k], cj, lane, 32);
    }
  }
  __syncthreads();
  pc.mark(3);
  if (tid == 0) B.l_n = 0;
}

// The steps of one block: posts [B0, B1) of the network P, whose blocks
// (nblk of them) meet at a barrier after every interval.  PU: NMDA edges in
// flight per lane in the pull; PD: ring slots in flight per neuron in the
// steps (results depend on neither).
template <class T, int PU, int PD>
__device__ __forceinline__ void prod_blocks(const Params &P, uint32_t B0, uint32_t B1, uint32_t nblk) {
  constexpr uint32_t kT = TileW<T>::W;
  __shared__ TileBufs<T> B;
  PhaseClock pc;
  pc.start(P);
  unsigned long long target = 0;  // barrier arrivals so far (thread 0)
  if (threadIdx.x == 0) B.l_n = 0;
  __syncthreads();
  uint32_t s = 0;
  while (s < P.nsteps) {
    const uint32_t iv_end = min(P.nsteps, s + P.interval);
    for (uint32_t bs = s; bs < iv_end; bs += kLB) {
      const uint32_t L = min(kLB, iv_end - bs);
      for (uint32_t tp0 = B0; tp0 < B1; tp0 += kT) {
        const uint32_t np = min(kT, B1 - tp0);
        tile_pull<T, PU>(P, tp0, np, bs, L, B);
        pc.mark(0);
        tile_steps<T, PD>(P, tp0, np, bs, L, B, pc);
      }
    }
    s = iv_end;
    if (s < P.nsteps) {
      if (!grid_sync(P.bar, P.err, nblk, target)) return;
      pc.mark(4);
    }
  }
}

// FP32: two blocks per SM (128 registers); FP64 runs one block per SM.  PU
// NMDA edges in flight per lane: four when a block's posts fit one tile
// (20k connectome: 4.05 us per timestep against 4.71 with eight), eight when
// they span several (250k network: 43.3 against 46.3 us); ring slots two
// steps ahead (4.60 us with one).  Batches of small networks run eight edges
// and one step ahead (their kernel has fewer registers to spare).
template <class T, int PU>
__global__ void __launch_bounds__(kThreads, sizeof(T) == 4 ? 2 : 1) k_prod(const __grid_constant__ Params P) {
  prod_blocks<T, PU, 2>(P, P.block_post[blockIdx.x], P.block_post[blockIdx.x + 1], gridDim.x);
}

// ---- long-term plasticity (networks with LTP, delays 0) ---------------------
// The reference's LTP (code/EqsGnl2.cpp:1005-1044) rewrites the weight g of
// a single-target record after the step's gather: on a presynaptic spike
// g += LP(post)·NegISI(pre) (NegISI > 0) or g *= 1 + LP(post)·NegISI(pre),
// then on a postsynaptic spike the same with LP(pre) and PosISI(pre).  The
// record's contribution to its post is g·st, with st its gate.  The
// production engine keeps one conductance per (post, receptor), G(t) =
// df·G(t-1) + pushes, which holds sum(g·st) only while g is fixed; a weight
// change dg after step t makes the next conductance df·(G + dg·st(t)) +
// pushes, so the LTP phase adds df·dg·st(t) (st(t): the presynaptic
// neuron's gate after step t, the production gate of every record of that
// neuron and receptor) to the slot the post folds at step t + 2, as the
// pushes of step t + 1's spikes do.  NMDA records need no correction: the
// pull sums g·s_pre over the current weights every step.  Only the records
// of neurons that spiked are touched (~(out + in degree) per spike).
// float arithmetic, one rounding per operation (no fused multiply-add), as
// the reference computes it
__device__ __forceinline__ float ltp_rule(float g, float lp, float x) {
  return x > 0.0f ? __fadd_rn(g, __fmul_rn(lp, x)) : __fmul_rn(g, __fadd_rn(1.0f, __fmul_rn(lp, x)));
}

template <class T>
__device__ __forceinline__ void ltp_correct(const Params &P, uint32_t post, uint32_t r, T dg, T stv, uint32_t slot) {
  const T v = (T)__ldg(P.dfst + (size_t)r * P.n + post) * dg * stv * (T)P.rg[r];
  const long long fx = __double2ll_rn((double)v * kFix);
  if (fx) atomicAdd(ring_at(P, P.lin_of_rec[r], post, slot), (unsigned long long)fx);
}

// LTP of record k of neuron a's out-records (a spiked at the step of parity
// par) and of record k of its in-records; the corrections go to ring slot
// `slot` (that step + 1).  Each record is rewritten once: by its presynaptic
// neuron's item when only that neuron spiked, by its postsynaptic neuron's
// item otherwise (both rules, the presynaptic one first, as the reference
// applies them).
template <class T>
__device__ __forceinline__ void ltp_out_record(const Params &P, uint32_t a, uint32_t k, uint32_t par, uint32_t slot) {
  const uint32_t n = P.n;
  const uint32_t ent = __ldg(P.ltp_oent + k), idx = __ldg(P.ltp_oidx + k);
  const uint32_t b = ent & 0xffffffu, r = ent >> 24;
  if (__ldcg(P.ltp_spk2 + (size_t)par * n + b)) return;
  float *wp = (r == FS_NMDA ? (float *)P.in_w : (float *)P.out_w) + idx;
  const float g0 = __ldcg(wp);
  const float g1 = ltp_rule(g0, __ldcg((const float *)P.ltp_lp2 + (size_t)par * n + b), __ldg(P.ltp_neg + a));
  __stcg(wp, g1);
  if (r != FS_NMDA)
    ltp_correct<T>(P, b, r, (T)g1 - (T)g0, __ldcg((const T *)P.ltp_sp2 + ((size_t)par * 4 + r) * n + a), slot);
}

template <class T>
__device__ __forceinline__ void ltp_in_record(const Params &P, uint32_t a, uint32_t k, uint32_t par, uint32_t slot) {
  const uint32_t n = P.n;
  const float *lp = (const float *)P.ltp_lp2 + (size_t)par * n;
  const uint32_t ent = __ldg(P.ltp_ient + k), idx = __ldg(P.ltp_iidx + k);
  const uint32_t c = ent & 0xffffffu, r = ent >> 24;
  float *wp = (r == FS_NMDA ? (float *)P.in_w : (float *)P.out_w) + idx;
  const float g0 = __ldcg(wp);
  float g = g0;
  if (__ldcg(P.ltp_spk2 + (size_t)par * n + c)) g = ltp_rule(g, __ldcg(lp + a), __ldg(P.ltp_neg + c));
  g = ltp_rule(g, __ldcg(lp + c), __ldg(P.ltp_pos + c));
  __stcg(wp, g);
  if (r != FS_NMDA)
    ltp_correct<T>(P, a, r, (T)g - (T)g0, __ldcg((const T *)P.ltp_sp2 + ((size_t)par * 4 + r) * n + c), slot);
}

// The LTP of a step's nl listed spikes (ids; parity par), over all warps of
// the grid: spike j contributes ceil(out_j / 32) + ceil(in_j / 32) items of
// 32 records, and warp gw takes items gw, gw + nwarps, ...  Every warp
// forms the same prefix over the spikes, 32 at a time (one spike per lane).
template <class T>
__device__ __forceinline__ void ltp_phase(const Params &P, const uint32_t *ids, uint32_t nl, uint32_t par,
                                          uint32_t slot, uint32_t gw, uint32_t nwarps, uint32_t lane) {
  uint32_t acc = 0;  // items of the earlier rounds
  for (uint32_t base = 0; base < nl; base += 32) {
    const uint32_t j = base + lane;
    uint32_t a = 0, o0 = 0, co = 0, i0 = 0, ci = 0;
    if (j < nl) {
      a = __ldcg(ids + j);
      o0 = __ldg(P.ltp_orow + a);
      i0 = __ldg(P.ltp_irow + a);
      co = (__ldg(P.ltp_orow + a + 1) - o0 + 31u) >> 5;
      ci = (__ldg(P.ltp_irow + a + 1) - i0 + 31u) >> 5;
    }
    uint32_t incl = co + ci;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t v = __shfl_up_sync(fsd::kFull, incl, o);
      if (lane >= (uint32_t)o) incl += v;
    }
    const uint32_t total = __shfl_sync(fsd::kFull, incl, 31);
    // first item of this round that is this warp's
    uint32_t it = gw >= acc ? gw - acc : (nwarps - (acc - gw) % nwarps) % nwarps;
    for (; it < total; it += nwarps) {
      const uint32_t jl = __ffs(__ballot_sync(fsd::kFull, incl > it)) - 1;  // the spike of item it
      const uint32_t aj = __shfl_sync(fsd::kFull, a, jl), coj = __shfl_sync(fsd::kFull, co, jl);
      const uint32_t first = __shfl_sync(fsd::kFull, incl - co - ci, jl);
      const uint32_t c = it - first;
      if (c < coj) {
        const uint32_t b0 = __shfl_sync(fsd::kFull, o0, jl), k = b0 + 32u * c + lane;
        if (k < __ldg(P.ltp_orow + aj + 1)) ltp_out_record<T>(P, aj, k, par, slot);
      } else {
        const uint32_t b0 = __shfl_sync(fsd::kFull, i0, jl), k = b0 + 32u * (c - coj) + lane;
        if (k < __ldg(P.ltp_irow + aj + 1)) ltp_in_record<T>(P, aj, k, par, slot);
      }
    }
    acc += total;
  }
}

// Persistent kernel of networks with LTP (every delay 0, so every step ends
// at a grid barrier).  Step t of a block: (1) the NMDA sums of its posts
// over the weights as they were after step t - 1's gather; (2) the pushes of
// step t - 1's spikes (the network's list, any warp takes any spike) over
// the linear weights of step t - 1; a grid barrier; (3) the LTP of step t -
// 1's spikes (no block reads a weight it rewrites until the next barrier);
// (4) the neurons' steps, which list step t's spikes; a grid barrier.  A
// launch of steps [t0, t1) ends with (1)-(3) of step t1: the NMDA sums of
// step t1 (kept in ltp_gn for the next launch, whose first step pulls
// nothing), the pushes and the LTP of step t1 - 1.  So between launches the
// weights are those after the last step's LTP, as the reference's are, and
// nothing else is pending.
template <class T>
__global__ void __launch_bounds__(kThreads, sizeof(T) == 4 ? 2 : 1) k_prod_ltp(const __grid_constant__ Params P) {
  constexpr uint32_t kT = TileW<T>::W;
  __shared__ TileBufs<T> B;
  __shared__ float tm3[kThreads * 3];
  const uint32_t B0 = P.block_post[blockIdx.x], B1 = P.block_post[blockIdx.x + 1];
  const uint32_t nblk = gridDim.x, tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  const uint32_t gw = blockIdx.x * (kThreads / 32) + wid, nwarps = nblk * (kThreads / 32);
  const uint32_t n = P.n, mask = P.mask;
  PhaseClock pc;
  pc.start(P);
  unsigned long long target = 0;
  for (uint32_t s = 0; s <= P.nsteps; s++) {
    const uint64_t t = P.t0 + s;
    const bool last = s == P.nsteps;
    if (s > 0) {
      for (uint32_t tp0 = B0; tp0 < B1; tp0 += kT) {
        const uint32_t np = min(kT, B1 - tp0);
        T(*gn)[kT] = (T(*)[kT])((T *)P.ltp_gn + tp0);
        if constexpr (sizeof(T) == 4) nmda_pull1_f32<true>(P, tp0, np, t, (float(*)[kTile])gn, wid, lane);
        else nmda_pull<T, true>(P, tp0, np, t, 1, gn, wid, lane);
      }
      pc.mark(0);
    }
    if (s > 0) {
      const uint32_t par = (uint32_t)(t - 1u) & 1u;
      const uint32_t nl = __ldcg(P.ltp_cnt + par);
      const uint32_t *ids = P.ltp_id + (size_t)par * n;
      const uint16_t *tms = P.ltp_tm + (size_t)par * n;
      const T *cs = (const T *)P.ltp_c + (size_t)par * n * 4;
      for (uint32_t k = gw; k < nl; k += nwarps) {
        T cj[4];
#pragma unroll
        for (int r = 0; r < 4; r++) cj[r] = __ldcg(cs + (size_t)k * 4 + r);
        push_spike<T, true>(P, __ldcg(ids + k), __ldcg(tms + k), cj, lane, 32);
      }
      // step t's list starts empty: its last readers (step t - 2's pushes
      // and LTP) passed the barrier of step t - 1, its writers come after
      // the next one (or in the next launch)
      if (blockIdx.x == 0 && tid == 0) P.ltp_cnt[(uint32_t)t & 1u] = 0u;
      pc.mark(5);
      if (!grid_sync(P.bar, P.err, nblk, target)) return;
      pc.mark(6);
      ltp_phase<T>(P, ids, nl, par, (uint32_t)t & mask, gw, nwarps, lane);
      pc.mark(7);
    }
    if (last) break;
    const uint32_t par = (uint32_t)t & 1u;
    const SpikeList<T> lst{P.ltp_cnt + par, P.ltp_id + (size_t)par * n, P.ltp_tm + (size_t)par * n,
                           (T(*)[4])((T *)P.ltp_c + (size_t)par * n * 4), n};
    for (uint32_t tp0 = B0; tp0 < B1; tp0 += kT) {
      const uint32_t np = min(kT, B1 - tp0);
      draw_inputs<T>(P, tp0, np, t, 1, B.hits, B.gauss);
      if (P.gap_row) tile_gap<T>(P, tp0, np, s, B.gapI);
      __syncthreads();
      pc.mark(1);
      if ((tid & ~31u) < np) {
        StepRegs<T> R;
        neuron_load<T, 1>(P, tp0, np, s, 1, R, tm3);
        neuron_steps<T, 1, true>(P, tp0, np, s, 1, (T(*)[kT])((T *)P.ltp_gn + tp0), B.hits, B.gauss, lst, B.gapI, R,
                                 tm3);
      }
      __syncthreads();
      pc.mark(2);
    }
    if (!grid_sync(P.bar, P.err, nblk, target)) return;
    pc.mark(4);
  }
}

// ---- single-step persistent kernel (networks whose delays are all 0) -------
// Every network in the reference's own format has no synaptic delays, so a
// spike of step t acts in step t + 1 and every step ends at a grid barrier.
// k_prod1 keeps everything a block reads from other neurons in its own
// shared memory, so the only traffic between blocks per step is the list of
// the step's spikes:
//  * each block tracks the presynaptic neurons of its posts (one block per
//    SM, up to 512 posts): for those with NMDA synapses it keeps a copy of
//    x and s, advanced every step by nmda_pre_step from the spike list (the
//    same function and operands as the neuron's owner, so every copy equals
//    the owner's value bit for bit);
//  * the NMDA in-edges of its posts live in shared memory as (tracked index,
//    weight), summed per post by eight lanes (lane-strided, then an xor
//    butterfly: the order of nmda_pull1_f32);
//  * a listed spike is matched to the block's tracked neurons through a
//    bitmap of their ids with per-word ranks (two shared-memory loads);
//  * a spike's linear synapses are delivered by the blocks of its targets:
//    each block walks the rows of its tracked neurons that spiked and adds
//    w*c (2^-40 fixed point, integer atomics: any order gives the same sum)
//    into per-post accumulators, the same integers the interval kernel's
//    delay ring sums;
//  * the owner of a neuron that spikes appends (id, inc, c[4]) to the step's
//    list; lists alternate by step parity and the last block at a barrier
//    empties the next step's list.
// Across launches the pending deliveries travel through the delay ring as
// in the interval kernel: the last step pushes its spikes into the ring and
// the first step of the next launch folds its ring slot.  The drive draws
// of step t + 1 are made while a block waits at the barrier of step t.
constexpr uint32_t kT1 = 512;   // threads of k_prod1 (= max posts per block)
constexpr uint32_t kT1F = 512;  // listed spikes looked up per pass

// Tracked index of neuron id in a block (or -1): bit id of the block's
// bitmap (words [w0, w0 + nwd) of the id space) says whether it is
// tracked, and its index is the number of tracked neurons below it: the
// count of the earlier words (rank) plus the set bits below it in its word.
__device__ __forceinline__ int find_tracked(const uint32_t *bits, const uint16_t *rank, uint32_t w0, uint32_t nwd,
                                            uint32_t id) {
  const uint32_t w = (id >> 5) - w0;  // ids below the first word wrap to >= nwd
  if (w >= nwd) return -1;
  const uint32_t word = bits[w], b = id & 31u;
  if (!((word >> b) & 1u)) return -1;
  return (int)rank[w] + __popc(word & ((1u << b) - 1u));
}

// Deliveries of a pass of listed spikes onto a block (k_prod1): warp w of
// nw takes listed spikes w, w + nw, ... and walks the spike's synapse row
// onto the block's posts, adding w * c (receptor gain applied) as 2^-40
// fixed point into the per-post accumulators.
constexpr uint32_t kDelW = 4;  // warps that deliver the last pass
__device__ __forceinline__ void deliver_listed(const Params &P, const Blk1 &me, uint32_t nf, const uint32_t *f_j,
                                               const float (*f_c)[4], const uint16_t *lrow, long long *acc,
                                               uint32_t w, uint32_t lane, uint32_t nw) {
  for (uint32_t k = w; k < nf; k += nw) {
    const uint32_t j = f_j[k];
    for (uint32_t e = lrow[j] + lane; e < lrow[j + 1]; e += 32) {
      const uint32_t code = __ldg(P.t1_lin + me.l0 + e);
      const float wt = __ldg(P.t1_linw + me.l0 + e);
      const uint32_t r = code >> 16, ql = code & 0xffffu;
      const float cv = f_c[k][r] * P.rg[r];
      const long long fx = __double2ll_rn((double)(wt * cv) * kFix);
      atomicAdd((unsigned long long *)&acc[(size_t)P.lin_of_rec[r] * kT1 + ql], (unsigned long long)fx);
    }
  }
}

// Grid barrier of k_prod1: as grid_sync, with threads of warps 1.. running
// work() while thread 0 waits.
template <class F>
__device__ __forceinline__ bool grid_sync_work(unsigned int *bar, int *err, uint32_t count,
                                               unsigned long long &target, PhaseClock &pc, F &&work,
                                               unsigned int limit = 1u << 24) {
  __shared__ int ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    ok = count > 1 ? arrive_and_wait(bar, err, count, target, limit) : 1;
    pc.mark(6);  // thread 0's wait for the other blocks
  } else if (threadIdx.x >= 32) {
    work();
  }
  __syncthreads();
  return ok != 0;
}

// kTM: the network has Tsodyks-Markram plasticity (an instance without it
// spends no registers on its state).
template <bool kTM>
__global__ void __launch_bounds__(kT1, 1) k_prod1(const __grid_constant__ Params P) {
  extern __shared__ __align__(16) unsigned char sm1[];
  __shared__ float gn[kT1], d_gauss[kT1], f_c[kT1F][4], nf_inc[kT1F];
  __shared__ uint8_t d_hits[kT1];
  __shared__ uint32_t f_j[kT1F], f_n, nf_j[kT1F], nf_n, next_grp, blk_n;
  const Blk1 me = P.b1[blockIdx.x];
  const uint32_t tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  const uint32_t n = P.n, mask = P.mask, NT = me.ntrk, NS = me.nslot, np = me.np, ng = (np + 3) / 4;
  // shared-memory layout (16-byte aligned pieces first); the NMDA copies are
  // per slot (a tracked neuron's slot is perm[j]) and double-buffered by
  // step parity: buffer s & 1 holds the values after step t0 + s - 1
  long long *acc = (long long *)sm1;                           // [nlin][kT1]
  float *const cx0 = (float *)(acc + (size_t)max(1u, P.nlin) * kT1);  // [NS] NMDA x copies
  float *const cs0 = cx0 + NS;                                 // [NS] NMDA s copies
  float *const cx1 = cs0 + NS;
  float *const cs1 = cx1 + NS;
  float *ctab = cs1 + NS;                                      // [ncls][3]
  float *ew = ctab + 3 * P.t1_ncls;                            // [ne] edge weights, group rows
  uint32_t *bits = (uint32_t *)(ew + me.ne);                   // [nwd] tracked-neuron bitmap
  uint32_t *grow = bits + me.nwd;                              // [ng + 1] first row of each group
  uint16_t *eidx = (uint16_t *)(grow + ng + 1);                // [ne] edge sources' slots
  uint16_t *rank = eidx + me.ne;                               // [nwd]
  uint16_t *lrow = rank + me.nwd;                              // [NT + 1] linear rows
  uint16_t *perm = lrow + NT + 1;                              // [NT] slots
  uint8_t *cls = (uint8_t *)(perm + NT);                       // [NS] kinetics class, 255: none
  // ---- tables ----
  for (uint32_t i = tid; i < max(1u, P.nlin) * kT1; i += kT1) acc[i] = 0ll;
  for (uint32_t i = tid; i < 3 * P.t1_ncls; i += kT1) ctab[i] = __ldg(P.t1_cls_tab + i);
  for (uint32_t i = tid; i < NS; i += kT1) {
    const uint32_t g = __ldg(P.t1_gid + me.s0 + i);
    const uint8_t c = __ldg(P.t1_cls + me.s0 + i);
    cls[i] = c;
    // the copies start from the owners' values after the last step before
    // this launch (written back by the previous launch); every other slot
    // holds 0 in both buffers (the zero-weight fillers read them)
    cx0[i] = c != 255 ? __ldcg((const float *)P.x_pre + g) : 0.0f;
    cs0[i] = c != 255 ? __ldcg((const float *)P.s_pre + g) : 0.0f;
    cx1[i] = 0.0f;
    cs1[i] = 0.0f;
  }
  for (uint32_t w = tid; w < me.nwd; w += kT1) {
    bits[w] = __ldg(P.t1_bits + me.bm0 + w);
    rank[w] = __ldg(P.t1_rank + me.bm0 + w);
  }
  for (uint32_t j = tid; j <= NT; j += kT1) lrow[j] = __ldg(P.t1_lrow + me.lrow0 + j);
  for (uint32_t j = tid; j < NT; j += kT1) perm[j] = __ldg(P.t1_perm + me.trk0 + j);
  for (uint32_t g = tid; g <= ng; g += kT1) grow[g] = __ldg(P.t1_grow + me.grow0 + g);
  for (uint32_t e = tid; e < me.ne; e += kT1) {
    ew[e] = __ldg(P.t1_ew + me.e0 + e);
    eidx[e] = __ldg(P.t1_eidx + me.e0 + e);
  }
  // ---- own neuron (thread tid owns post post0 + tid) ----
  const bool own = tid < np;
  const bool active = (tid & ~31u) < np;  // warps with posts
  const uint32_t p = own ? me.post0 + tid : me.post0;
  NeuronPar<float> q;
  NeuronState<float> st;
  if (active) load_neuron<float, kTM>(P, p, q, st);
  uint32_t nsp = 0;
  if (own) {
    float gv = 0.0f;
    d_hits[tid] = (uint8_t)draw_one<float>(P, p, P.t0, gv);
    d_gauss[tid] = gv;
  }
  PhaseClock pc;
  pc.start(P);
  unsigned long long target = 0;  // barrier arrivals so far (thread 0)
  if (tid == 0) {
    f_n = 0;
    next_grp = 0;
  }
  __syncthreads();
  pc.mark(5);
  for (uint32_t s = 0; s < P.nsteps; s++) {
    const uint64_t t = P.t0 + s;
    float *X = (s & 1u) ? cx1 : cx0, *Sv = (s & 1u) ? cs1 : cs0;
    // spike counts rotate over four slots: the slot of step t + 2 was last
    // read in step t - 1, so it can be emptied now (every append to it comes
    // after two more barriers)
    if (blockIdx.x == 0 && tid == 0) __stcg(P.t1_cnt + ((uint32_t)(t + 2u) & 3u), 0u);
    if (tid == 0) blk_n = 0;  // this step's spikes of the block (read after the NMDA sums' barrier)
    if (s > 0) {
      // ---- spikes of step t - 1 ----
      // the buffer of this step already holds every copy advanced as if its
      // neuron had not spiked (made during the barrier wait); the listed
      // spikes are redone from the previous buffer, and their linear
      // synapses onto this block are delivered
      const float *Xo = (s & 1u) ? cx0 : cx1, *So = (s & 1u) ? cs0 : cs1;
      const uint32_t par = (uint32_t)(t - 1u) & 1u;
      const uint32_t tag = (uint32_t)(t - 1u) + 1u;  // entries of step t - 1 carry it
      const uint32_t nreg = gridDim.x * P.t1_slots;   // block-region entries (<= kT1F)
      const uint32_t W = P.t1_w;
      const uint4 *reg = P.t1_list + (size_t)par * nreg * W;
      const uint4 *ovf = P.t1_ovf + (size_t)par * n * W;
      // the regions' entries are loaded with the overflow count (one round
      // trip); stale entries carry another step's tag
      uint4 a0 = make_uint4(0u, 0u, 0u, 0u), b0 = a0;
      if (tid < nreg) {
        a0 = __ldcg(reg + W * (size_t)tid);
        if (W == 2) b0 = __ldcg(reg + 2 * (size_t)tid + 1);
      }
      const uint32_t cnt = nreg + __ldcg(P.t1_cnt + ((uint32_t)(t - 1u) & 3u));
      pc.lap(8, cnt);    // the list's entry count is in
      pc.lap(12, a0.x);  // thread 0's entries are in
      for (uint32_t c0 = 0; c0 < cnt; c0 += kT1F) {
        if (tid == 0) {
          f_n = 0;
          nf_n = 0;
        }
        __syncthreads();
        const uint32_t i = c0 + tid;
        if (tid < kT1F && i < cnt) {
          uint4 a = a0, b = b0;
          const bool over = i >= nreg;  // an overflow entry: every one is of step t - 1
          if (over) {
            a = __ldcg(ovf + W * (size_t)(i - nreg));
            if (W == 2) b = __ldcg(ovf + 2 * (size_t)(i - nreg) + 1);
          }
          const bool cur = over || (W == 2 ? b.z : a.w) == tag;
          const int j = cur ? find_tracked(bits, rank, me.w0, me.nwd, a.x) : -1;
          if (j >= 0) {
            const uint32_t sl = perm[j];
            if (cls[sl] != 255) {
              const uint32_t k = atomicAdd(&nf_n, 1u);
              nf_j[k] = sl;
              nf_inc[k] = __uint_as_float(a.y);
            }
            if (lrow[j + 1] > lrow[j]) {
              const uint32_t k = atomicAdd(&f_n, 1u);
              f_j[k] = (uint32_t)j;
              f_c[k][0] = __uint_as_float(a.z);
              f_c[k][1] = __uint_as_float(W == 2 ? a.w : a.z);
              f_c[k][2] = __uint_as_float(W == 2 ? b.x : a.z);
              f_c[k][3] = __uint_as_float(W == 2 ? b.y : a.z);
            }
          }
        }
        __syncthreads();
        pc.lap(9);  // the look-ups are done
        // the NMDA copies of the listed neurons (by slot), from their
        // previous values
        for (uint32_t k = tid; k < nf_n; k += kT1) {
          const uint32_t sl = nf_j[k], c = cls[sl];
          float xv = Xo[sl], sv = So[sl];
          nmda_pre_step<float>(xv, sv, true, nf_inc[k], ctab[3 * c], ctab[3 * c + 1], ctab[3 * c + 2]);
          X[sl] = xv;
          Sv[sl] = sv;
        }
        // the deliveries of all but the last pass (the last pass's are made
        // by the first warps while the others start the NMDA sums)
        if (c0 + kT1F < cnt) {
          deliver_listed(P, me, f_n, f_j, f_c, lrow, acc, wid, lane, kT1 / 32);
          __syncthreads();
          if (tid == 0) f_n = 0;
        }
        __syncthreads();
      }
      pc.mark(0);
      pc.mark(1);
    }
    // ---- NMDA sums of the block's posts (order of nmda_pull1_f32) ----
    // the first kDelW warps deliver the last pass's listed spikes (their
    // synapse rows come from L2) and then join; every warp takes groups of
    // four posts from a shared counter and walks the group's rows of 32
    // entries: lane l of quarter h sums post 4g + h's edges l, l + 8, ... in
    // order (then zero-weight fillers, which leave the sum unchanged), four
    // rows loaded ahead, then the butterfly over 4, 2, 1
    if (wid < kDelW) {
      deliver_listed(P, me, f_n, f_j, f_c, lrow, acc, wid, lane, kDelW);
      pc.lap(10);  // warp 0's deliveries are issued
    }
    for (;;) {
      uint32_t g = 0;
      if (lane == 0) g = atomicAdd(&next_grp, 1u);
      g = __shfl_sync(fsd::kFull, g, 0);
      if (g >= ng) break;
      const uint32_t iend = grow[g + 1] * 32u;
      uint32_t i = grow[g] * 32u + lane;
      float sum = 0.0f;
      for (; i + 96u < iend; i += 128u) {
        const float w0 = ew[i], w1 = ew[i + 32], w2 = ew[i + 64], w3 = ew[i + 96];
        const float v0 = Sv[eidx[i]], v1 = Sv[eidx[i + 32]], v2 = Sv[eidx[i + 64]], v3 = Sv[eidx[i + 96]];
        sum = __fmaf_rn(w0, v0, sum);
        sum = __fmaf_rn(w1, v1, sum);
        sum = __fmaf_rn(w2, v2, sum);
        sum = __fmaf_rn(w3, v3, sum);
      }
      for (; i < iend; i += 32u) sum = __fmaf_rn(ew[i], Sv[eidx[i]], sum);
#pragma unroll
      for (int o = 4; o; o >>= 1) sum += __shfl_xor_sync(fsd::kFull, sum, o);
      const uint32_t qq = 4 * g + (lane >> 3);
      if ((lane & 7u) == 0 && qq < np) gn[qq] = sum;
    }
    pc.lap(11);  // warp 0 found no more posts to sum
    __syncthreads();
    pc.mark(2);
    // (the pass counters are reset behind the barrier above, for the next step)
    if (tid == 0) {
      f_n = 0;
      next_grp = 0;
    }
    // ---- the neurons' step ----
    if (active) {
      long long rv[4];
#pragma unroll
      for (int r = 0; r < 4; r++) {
        rv[r] = 0ll;
        const int ri = P.lin_of_rec[r];
        if (ri >= 0 && own) {
          if (s == 0) {  // deliveries of the step before this launch: the ring
            long long *slot = (long long *)ring_at(P, ri, p, (uint32_t)(t - 1u) & mask);
            rv[r] = __ldcg(slot);
            if (rv[r]) __stcg(slot, 0ll);
          } else {
            rv[r] = acc[(size_t)ri * kT1 + tid];
            acc[(size_t)ri * kT1 + tid] = 0ll;
          }
        }
      }
      const uint32_t qs = own ? tid : 0;
      float cinc[4], inc;
      const bool spk =
          neuron_step<float, kTM>(P, q, st, rv, gn[qs], d_hits[qs], d_gauss[qs], 0.0f, p, own, s, cinc, inc);
      pc.lap(13, spk ? 1u : 0u);  // warp 0's neurons have stepped
      nsp += spk ? 1u : 0u;
      if (own && P.gv_row) gv_write<float>(P, p, s, st);
      const uint32_t m = __ballot_sync(fsd::kFull, spk);
      if (m) {
        spike_outputs(P, m, spk, p, s, lane, false);
        // the spike goes to this block's region of the step's list (a
        // shared-memory counter); past the region's slots, to the overflow
        // list (a global counter)
        const uint32_t par = (uint32_t)t & 1u;
        const int leader = __ffs(m) - 1;
        uint32_t base = 0;
        if ((int)lane == leader) base = atomicAdd(&blk_n, (uint32_t)__popc(m));
        base = __shfl_sync(fsd::kFull, base, leader);
        if (spk) {
          const uint32_t k = base + __popc(m & ((1u << lane) - 1u));
          const uint32_t W = P.t1_w;
          uint4 *e;
          if (k < P.t1_slots) {
            e = P.t1_list + (((size_t)par * gridDim.x + blockIdx.x) * P.t1_slots + k) * W;
          } else {
            const uint32_t o = atomicAdd(P.t1_cnt + ((uint32_t)t & 3u), 1u);
            e = P.t1_ovf + ((size_t)par * n + o) * W;
          }
          if (W == 2) {
            __stcg(e, make_uint4(p, __float_as_uint(inc), __float_as_uint(cinc[0]), __float_as_uint(cinc[1])));
            __stcg(e + 1, make_uint4(__float_as_uint(cinc[2]), __float_as_uint(cinc[3]), (uint32_t)t + 1u, 0u));
          } else {
            // at most one receptor's c is not 0: the sum is that c exactly
            const float cl = ((cinc[0] + cinc[1]) + cinc[2]) + cinc[3];
            __stcg(e, make_uint4(p, __float_as_uint(inc), __float_as_uint(cl), (uint32_t)t + 1u));
          }
        }
        if (s + 1 == P.nsteps) {
          // the launch's last step: its spikes go into the delay ring, which
          // the next launch's first step folds
          const uint32_t tm = (uint32_t)t & mask;
          uint32_t rem = m;
          while (rem) {
            const int jl = __ffs(rem) - 1;
            rem &= rem - 1;
            const uint32_t qq = __shfl_sync(fsd::kFull, p, jl);
            float cj[4];
#pragma unroll
            for (int r = 0; r < 4; r++) cj[r] = __shfl_sync(fsd::kFull, cinc[r], jl);
            push_spike<float>(P, qq, tm, cj, lane, 32);
          }
        }
      }
    }
    pc.mark(3);
    if (s + 1 < P.nsteps) {
      // while the barrier is awaited: the next step's drive draws, and every
      // NMDA copy advanced into the other buffer as if its neuron had not
      // spiked (the listed spikes are redone after the barrier)
      const uint64_t tn = t + 1;
      float *Xn = (s & 1u) ? cx0 : cx1, *Sn = (s & 1u) ? cs0 : cs1;
      const bool ok = grid_sync_work(P.bar, P.err, gridDim.x, target, pc, [&]() {
        for (uint32_t qq = tid - 32; qq < np; qq += kT1 - 32) {
          float gv = 0.0f;
          d_hits[qq] = (uint8_t)draw_one<float>(P, me.post0 + qq, tn, gv);
          d_gauss[qq] = gv;
        }
        if (P.t1_ncls == 1) {  // one class (the usual case): its constants in registers
          const float k0 = ctab[0], k1 = ctab[1], k2 = ctab[2];
          for (uint32_t j = tid - 32; j < NS; j += kT1 - 32) {
            if (cls[j] != 255) {
              float xv = X[j], sv = Sv[j];
              nmda_pre_step<float>(xv, sv, false, 1.0f, k0, k1, k2);
              Xn[j] = xv;
              Sn[j] = sv;
            }
          }
        } else {
          for (uint32_t j = tid - 32; j < NS; j += kT1 - 32) {
            const uint32_t c = cls[j];
            if (c != 255) {
              float xv = X[j], sv = Sv[j];
              nmda_pre_step<float>(xv, sv, false, 1.0f, ctab[3 * c], ctab[3 * c + 1], ctab[3 * c + 2]);
              Xn[j] = xv;
              Sn[j] = sv;
            }
          }
        }
      });
      if (!ok) return;
      pc.mark(4);
    }
  }
  if (own) {
    store_neuron<float, kTM>(P, p, q, st);
    if (P.nspk && nsp) P.nspk[p] += nsp;
  }
  // the launch's spikes, added to the total once per warp
  if (active) {
    uint32_t w = nsp;
#pragma unroll
    for (int o = 16; o; o >>= 1) w += __shfl_xor_sync(fsd::kFull, w, o);
    if (lane == 0 && w) atomicAdd(P.spike_total, (unsigned long long)w);
  }
}

// ---- tile kernels: networks too large for one persistent launch, batches --
// A launch pair advances every tile (up to TileW posts of one network) by a
// batch of L steps: k_tile_pull writes the tiles' NMDA sums of the batch to
// gn_buf, k_tile_step draws the drive, runs the neurons' steps and pushes
// the spikes.  The kernel boundary is the barrier between batches, so
// blocks are scheduled freely over the tiles of all networks (no block
// waits for another), the pull runs at the occupancy its registers allow,
// and L never exceeds the smallest interval of the networks (every value a
// batch reads was final before it began).  A chunk of steps is one CUDA
// graph of these pairs.  Per post the arithmetic and the order of every sum
// are those of the persistent kernel, so the results are identical.
struct IvTile {
  uint32_t inst, p0, np, pad;
};

__device__ __forceinline__ void params_to_smem(Params &Psh, const Params *__restrict__ Ps, uint32_t inst) {
  const uint32_t *src = (const uint32_t *)(Ps + inst);
  uint32_t *dst = (uint32_t *)&Psh;
  for (uint32_t i = threadIdx.x; i < sizeof(Params) / 4; i += blockDim.x) dst[i] = src[i];
}

template <class T, int U>
__global__ void __launch_bounds__(kThreads, U == 4 ? 4 : 2) k_tile_pull(const Params *__restrict__ Ps,
                                                          const IvTile *__restrict__ tiles, uint32_t bs,
                                                          uint32_t L) {
  __shared__ __align__(16) Params Psh;
  __shared__ T gn[kLB][TileW<T>::W];
  const IvTile tl = tiles[blockIdx.x];
  params_to_smem(Psh, Ps, tl.inst);
  __syncthreads();
  const Params &P = Psh;
  const uint32_t tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  if constexpr (sizeof(T) == 4) {
    if (P.dmax0) nmda_pull1_f32(P, tl.p0, tl.np, P.t0 + bs, (float (*)[kTile])gn, wid, lane);
    else nmda_pull_f32<U>(P, tl.p0, tl.np, P.t0 + bs, L, (float (*)[kTile])gn, wid, lane);
  } else {
    nmda_pull<T>(P, tl.p0, tl.np, P.t0 + bs, L, gn, wid, lane);
  }
  __syncthreads();
  T *out = (T *)P.gn_buf;
  for (uint32_t i = tid; i < tl.np * L; i += kThreads) {
    const uint32_t j = i / tl.np, q = i - j * tl.np;
    out[(size_t)j * P.n + tl.p0 + q] = gn[j][q];
  }
}

template <class T, int PD>
__global__ void __launch_bounds__(kThreads, sizeof(T) == 4 ? 2 : 1) k_tile_step(const Params *__restrict__ Ps,
                                                                              const IvTile *__restrict__ tiles,
                                                                              uint32_t bs, uint32_t L) {
  __shared__ __align__(16) Params Psh;
  __shared__ TileBufs<T> B;
  const IvTile tl = tiles[blockIdx.x];
  params_to_smem(Psh, Ps, tl.inst);
  if (threadIdx.x == 0) B.l_n = 0;
  __syncthreads();
  const Params &P = Psh;
  const T *in = (const T *)P.gn_buf;
  for (uint32_t i = threadIdx.x; i < tl.np * L; i += kThreads) {
    const uint32_t j = i / tl.np, q = i - j * tl.np;
    B.gn[j][q] = in[(size_t)j * P.n + tl.p0 + q];
  }
  PhaseClock pc;
  pc.out = nullptr;
  tile_steps<T, PD>(P, tl.p0, tl.np, bs, L, B, pc);  // its first barrier orders the loads above
}


// ---- host side -------------------------------------------------------------
struct Tiles;
struct Prod {
  bool fp64 = false;
  bool single = false;     // runs on the single-step kernel k_prod1
  struct Tiles *tiles = nullptr;  // runs on the tile kernels (large networks)
  uint32_t b1_blocks = 0;  // its blocks (one per SM at most)
  unsigned long long *phase_buf = nullptr;  // phase clock counters (debug aid)
  bool wide = false;  // some block's posts span several tiles: eight NMDA edges in flight
  bool ltp = false;   // long-term plasticity: runs on k_prod_ltp
  uint32_t n = 0, sm = 148;
  Params P{};
  std::vector<void *> allocs;
  uint64_t t = 0;  // steps done since reset
  uint32_t d_min = 0, d_max = 0;
  uint32_t blocks = 0, chunks = 0;
  uint64_t lin_edges = 0, nmda_edges = 0;
  uint32_t nlin = 0;
  uint32_t chunk_steps = 1000;
  // per-launch buffers
  uint32_t *counts = nullptr, *bits = nullptr, *offsets = nullptr, *idx = nullptr;
  float *outV = nullptr, *outI = nullptr;
  uint32_t *outNS = nullptr;
  uint64_t cap_steps = 0, outv_steps = 0, outi_steps = 0, outns_steps = 0;
  unsigned int *bar = nullptr;
  int *err = nullptr;
  unsigned long long *spike_total = nullptr;
  // one event pair per launch since the last accounting: finish() adds up
  // the device time of every launch in order, however many chunks ran
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev;
  size_t ev_used = 0;
  double ms = 0.0;
  uint64_t kl = 0;
  uint64_t key = 0;
  std::vector<uint32_t> host_counts;
  // GatingVariable selections: presynaptic neuron of each record, per
  // receptor (from the compat layout), and the device buffers of a call
  std::vector<uint32_t> rec_src[FS_NREC];
  uint32_t *gv_row = nullptr, *gv_ent = nullptr;
  float *gv_st = nullptr, *gv_xt = nullptr;
  uint64_t gv_out_cap = 0;
  uint32_t gv_ent_cap = 0;
  std::vector<uint32_t> in_row_h;  // NMDA in-degree prefix (block partitioning)
  // networks with LTP: where each synapse-list entry's weight lives (index
  // in out_w, or in in_w with the top bit set)
  std::vector<uint32_t> wpos;
};

namespace {

template <class X>
int dal(Prod *p, X **ptr, size_t count, std::string &err) {
  *ptr = nullptr;
  if (!count) return FS_OK;
  void *q = nullptr;
  cudaError_t e = cudaMalloc(&q, count * sizeof(X));
  if (e != cudaSuccess) {
    err = std::string("cudaMalloc: ") + cudaGetErrorString(e);
    return FS_ERR_NOMEM;
  }
  p->allocs.push_back(q);
  *ptr = (X *)q;
  return FS_OK;
}
template <class X>
int dup(Prod *p, X **ptr, const X *src, size_t count, cudaStream_t st, std::string &err) {
  int rc = dal(p, ptr, count, err);
  if (rc || !count) return rc;
  cudaError_t e = src ? cudaMemcpyAsync(*ptr, src, count * sizeof(X), cudaMemcpyHostToDevice, st)
                      : cudaMemsetAsync(*ptr, 0, count * sizeof(X), st);
  if (e != cudaSuccess) {
    err = std::string("upload: ") + cudaGetErrorString(e);
    return FS_ERR_CUDA;
  }
  return FS_OK;
}

int ensure_buffers(Prod *p, uint32_t steps, bool wantV, bool wantI, bool wantNS, std::string &err) {
  int rc;
  if (steps > p->cap_steps) {
    const uint32_t words = (p->n + 31) / 32;
    if ((rc = dal(p, &p->counts, steps, err)) || (rc = dal(p, &p->bits, (size_t)steps * words, err)) ||
        (rc = dal(p, &p->offsets, (size_t)steps + 1, err)) || (rc = dal(p, &p->idx, (size_t)steps * p->n, err)))
      return rc;
    p->cap_steps = steps;
  }
  if (wantV && steps > p->outv_steps) {
    if ((rc = dal(p, &p->outV, (size_t)steps * p->n, err))) return rc;
    p->outv_steps = steps;
  }
  if (wantI && steps > p->outi_steps) {
    if ((rc = dal(p, &p->outI, (size_t)steps * 5 * p->n, err))) return rc;
    p->outi_steps = steps;
  }
  if (wantNS && steps > p->outns_steps) {
    if ((rc = dal(p, &p->outNS, (size_t)steps * p->n, err))) return rc;
    p->outns_steps = steps;
  }
  return FS_OK;
}

}  // namespace

// tile runner of a single network (defined with the tile runner below)
int tiles_solo_launch(Prod *p, const Params &P, uint32_t nsteps, cudaStream_t st, uint64_t *kernels,
                      std::string &err);
void tiles_delete(Tiles *T);
int tiles_solo_create(Prod *p, std::string &err);

namespace {

int launch(Prod *p, uint32_t nsteps, bool want_bits, bool wantV, cudaStream_t st, uint64_t *launches,
           std::string &err, bool wantI = false, bool wantNS = false, bool wantGV = false) {
  int rc = ensure_buffers(p, nsteps, wantV, wantI, wantNS, err);
  if (rc) return rc;
  const uint32_t words = (p->n + 31) / 32;
  cudaError_t e = cudaMemsetAsync(p->counts, 0, (size_t)nsteps * 4, st);
  if (e == cudaSuccess && want_bits) e = cudaMemsetAsync(p->bits, 0, (size_t)nsteps * words * 4, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(p->bar, 0, 64 * 4, st);
  if (e != cudaSuccess) {
    err = std::string("memset: ") + cudaGetErrorString(e);
    return FS_ERR_CUDA;
  }
  Params P = p->P;
  P.t0 = p->t;
  P.nsteps = nsteps;
  P.bits = want_bits ? p->bits : nullptr;
  P.words = words;
  P.counts = p->counts;
  P.outV = wantV ? p->outV : nullptr;
  P.outI = wantI ? p->outI : nullptr;
  P.outNS = wantNS ? p->outNS : nullptr;
  if (p->gv_out_cap && wantGV) {
    P.gv_row = p->gv_row;
    P.gv_ent = p->gv_ent;
    P.gv_st = p->gv_st;
    P.gv_xt = p->gv_xt;
  } else {
    P.gv_row = P.gv_ent = nullptr;
    P.gv_st = P.gv_xt = nullptr;
    P.gv_n = 0;
  }
  P.bar = p->bar;
  P.err = p->err;
  P.spike_total = p->spike_total;
  void *args[] = {&P};
  if (p->ev_used == p->ev.size()) {
    cudaEvent_t a = nullptr, b = nullptr;
    if (cudaEventCreate(&a) != cudaSuccess || cudaEventCreate(&b) != cudaSuccess) {
      if (a) cudaEventDestroy(a);
      err = "event create";
      return FS_ERR_CUDA;
    }
    p->ev.push_back({a, b});
  }
  // the single-step kernel's lists start empty (region entries are told
  // apart by their step tag; a reset or a restored checkpoint moves the
  // step counter back)
  if (p->single && (cudaMemsetAsync(P.t1_cnt, 0, 16, st) != cudaSuccess ||
                    cudaMemsetAsync(P.t1_list, 0, (size_t)2 * p->b1_blocks * P.t1_slots * 16 * P.t1_w, st) != cudaSuccess)) {
    err = "memset";
    return FS_ERR_CUDA;
  }
  const auto &evp = p->ev[p->ev_used];
  cudaEventRecord(evp.first, st);
  if (p->tiles) {
    uint64_t k = 0;
    int trc = tiles_solo_launch(p, P, nsteps, st, &k, err);
    cudaEventRecord(evp.second, st);
    if (trc) return trc;
    p->ev_used++;
    p->t += nsteps;
    if (launches) *launches += k;
    return FS_OK;
  }
  if (p->ltp) {
    // both spike lists start empty (a launch leaves none pending)
    e = cudaMemsetAsync(P.ltp_cnt, 0, 8, st);
    if (e == cudaSuccess)
      e = cudaLaunchCooperativeKernel(p->fp64 ? (const void *)k_prod_ltp<double> : (const void *)k_prod_ltp<float>,
                                      p->blocks, kThreads, args, 0, st);
  } else if (p->single) {
    const void *k1 = P.plast == PL_TM ? (const void *)k_prod1<true> : (const void *)k_prod1<false>;
    e = cudaLaunchCooperativeKernel(k1, p->b1_blocks, kT1, args, P.t1_smem, st);
  } else {
    // (the FP64 pull does not take the edges-in-flight parameter)
    const void *k = p->fp64 ? (const void *)k_prod<double, 4>
                            : (p->wide ? (const void *)k_prod<float, 8> : (const void *)k_prod<float, 4>);
    e = cudaLaunchCooperativeKernel(k, p->blocks, kThreads, args, 0, st);
  }
  cudaEventRecord(evp.second, st);
  if (e != cudaSuccess) {
    err = std::string("cooperative launch: ") + cudaGetErrorString(e);
    return FS_ERR_CUDA;
  }
  p->ev_used++;
  p->t += nsteps;
  if (launches) *launches += 1;
  return FS_OK;
}

int finish(Prod *p, cudaStream_t st, std::string &err) {
  cudaError_t e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    err = std::string("kernel: ") + cudaGetErrorString(e);
    return FS_ERR_CUDA;
  }
  for (size_t i = 0; i < p->ev_used; i++) {
    float ms = 0;
    if (cudaEventElapsedTime(&ms, p->ev[i].first, p->ev[i].second) == cudaSuccess) p->ms += ms;
    p->kl += 1;
  }
  p->ev_used = 0;
  int h = 0;
  e = cudaMemcpy(&h, p->err, 4, cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) {
    err = std::string("error word: ") + cudaGetErrorString(e);
    return FS_ERR_CUDA;
  }
  if (h) {
    err = "grid barrier wait gave up (device error word set)";
    return FS_ERR_TIMEOUT;
  }
  return FS_OK;
}

}  // namespace

// ---- host tables of a production network -----------------------------------
// From the flat synapse list: the receptor kinetics each presynaptic neuron
// imposes on its gates (production modes need one per (neuron, receptor)),
// the receptors each neuron projects with, the delay range, and the two CSR
// tables (linear out-edges by pre: code = post | receptor << 22 | delay <<
// 24; NMDA in-edges by post: code = pre | delay << 24) in synapse-list order.
struct HostNet {
  uint32_t n = 0, nlin = 0, dmin = 0, dmax = 0;
  int lin_of_rec[4] = {-1, -1, -1, -1};
  uint64_t nlin_e = 0, nnm_e = 0;
  std::vector<float> pdf, p_dfxt, p_dfst, p_efas;
  std::vector<uint8_t> proj;
  std::vector<uint32_t> out_row, in_row, out_code, in_code;
  std::vector<float> out_w, in_w;
};

static int host_net(const fs_net_desc *d, HostNet &H, std::string &err) {
  const fs_neurons &v = d->neurons;
  const uint32_t n = v.n;
  H.n = n;
  const fs_syn_list &S = *d->syn;
  std::vector<float> &pdf = H.pdf, &p_dfxt = H.p_dfxt, &p_dfst = H.p_dfst, &p_efas = H.p_efas;
  pdf.assign((size_t)4 * n, -1.0f);
  p_dfxt.assign(n, -1.0f);
  p_dfst.assign(n, -1.0f);
  p_efas.assign(n, -1.0f);
  std::vector<uint8_t> &proj = H.proj;
  proj.assign(n, 0);
  bool present[5] = {false, false, false, false, false};
  uint32_t dmin = 0xffffffffu, dmax = 0;
  uint64_t nlin_e = 0, nnm_e = 0;
  for (uint64_t e = 0; e < S.n; e++) {
    const uint32_t a = S.pre[e], b = S.post[e], r = S.rec[e];
    const uint32_t dl = S.delay ? S.delay[e] : 0;
    if (a >= n || b >= n || r >= FS_NREC) {
      err = "synapse list: index out of range";
      return FS_ERR_ARG;
    }
    if (dl > 255) {
      err = "synapse delays above 255 steps are not supported";
      return FS_ERR_UNSUPPORTED;
    }
    dmin = std::min(dmin, dl);
    dmax = std::max(dmax, dl);
    present[r] = true;
    proj[a] |= (uint8_t)(1u << r);
    auto same = [&](float &slot, float val) -> bool {
      if (slot < 0.0f) { slot = val; return true; }
      return slot == val;
    };
    bool ok;
    if (r != FS_NMDA) {
      ok = same(pdf[(size_t)r * n + a], v.dfst[(size_t)r * n + b]);
      nlin_e++;
    } else {
      ok = same(p_dfxt[a], v.nmda_dfxt[b]) && same(p_dfst[a], v.dfst[(size_t)FS_NMDA * n + b]) &&
           same(p_efas[a], v.nmda_efst[b] * v.nmda_as[b]);
      nnm_e++;
    }
    if (!ok) {
      err = "production modes need one receptor time constant per (presynaptic neuron, receptor); "
            "targets of a neuron differ (use FS_MODE_COMPAT)";
      return FS_ERR_UNSUPPORTED;
    }
  }
  if (S.n == 0) dmin = 0;
  H.dmin = dmin;
  H.dmax = dmax;
  H.nlin_e = nlin_e;
  H.nnm_e = nnm_e;
  for (int r = 0; r < 4; r++) H.lin_of_rec[r] = present[r] ? (int)(H.nlin++) : -1;
  for (auto &x : pdf) if (x < 0) x = 0;
  for (auto *vv : {&p_dfxt, &p_dfst, &p_efas}) for (auto &x : *vv) if (x < 0) x = 0;
  // ---- CSR of linear out-edges (by pre) and NMDA in-edges (by post) ----
  std::vector<uint32_t> &out_row = H.out_row, &in_row = H.in_row;
  out_row.assign(n + 1, 0);
  in_row.assign(n + 1, 0);
  for (uint64_t e = 0; e < S.n; e++) {
    if (S.rec[e] == FS_NMDA) in_row[S.post[e] + 1]++;
    else out_row[S.pre[e] + 1]++;
  }
  for (uint32_t i = 0; i < n; i++) { out_row[i + 1] += out_row[i]; in_row[i + 1] += in_row[i]; }
  H.out_code.assign(nlin_e, 0);
  H.in_code.assign(nnm_e, 0);
  H.out_w.assign(nlin_e, 0.0f);
  H.in_w.assign(nnm_e, 0.0f);
  {
    std::vector<uint32_t> fo(out_row.begin(), out_row.end() - 1), fi(in_row.begin(), in_row.end() - 1);
    for (uint64_t e = 0; e < S.n; e++) {
      const uint32_t dl = S.delay ? S.delay[e] : 0;
      if (S.rec[e] == FS_NMDA) {
        const uint32_t q = fi[S.post[e]]++;
        H.in_code[q] = S.pre[e] | (dl << 24);
        H.in_w[q] = S.g[e];
      } else {
        const uint32_t q = fo[S.pre[e]]++;
        H.out_code[q] = S.post[e] | ((uint32_t)S.rec[e] << 22) | (dl << 24);
        H.out_w[q] = S.g[e];
      }
    }
  }
  return FS_OK;
}

// ---- plan of the single-step kernel ------------------------------------------
// Posts are cut into at most one block per SM, in whole warps (32 posts) and
// at most kT1 posts per block, balanced by a cost of 24 per post plus its
// NMDA in-edges plus a quarter of its linear in-edges.  Per block: the sorted
// presynaptic neurons of its posts' synapses, their NMDA kinetics classes,
// their linear synapses onto the block grouped by neuron, and the NMDA
// in-edges in CSR order with the presynaptic neuron as a tracked index.
// Returns false (and the interval kernel runs) when a block's tables do not
// fit in shared memory or there are more than 255 NMDA kinetics classes.
struct Single {
  std::vector<Blk1> blk;
  std::vector<uint32_t> gid, lin, grow, bits;  // gid, cls: per slot
  std::vector<uint8_t> cls;
  std::vector<float> linw, ew, tab;
  std::vector<uint16_t> eidx, rank, lrow, perm;  // lrow, perm: per tracked neuron
  uint32_t smem = 0;
};

// Shared memory of k_prod1's tables for one block (the kernel's layout):
// accumulators | x, s copies x2 (per slot) | class table | edge weights |
// bitmap | group rows | edge slots | ranks | linear rows | slots of the
// tracked neurons | classes (per slot).
static size_t single_smem(uint32_t nlin, uint32_t ncls, const Blk1 &k) {
  const size_t ng = ((size_t)k.np + 3) / 4;
  return (size_t)std::max(1u, nlin) * kT1 * 8 + (size_t)k.nslot * 16 + 3 * (size_t)ncls * 4 + (size_t)k.ne * 4 +
         (size_t)k.nwd * 4 + (ng + 1) * 4 + (size_t)k.ne * 2 + (size_t)k.nwd * 2 + ((size_t)k.ntrk + 1) * 2 +
         (size_t)k.ntrk * 2 + (size_t)k.nslot;
}

// Slots of a block's tracked neurons in its shared-memory copies, so that
// the gathers of one row of NMDA edges (32 tracked indices, `rows` lists
// them) fall in as few lanes of the same bank as a greedy pass finds: the
// neurons in the most rows first, each into the bank (slot mod 32) that
// least raises the rows' largest bank counts, at most cap per bank.  The
// slots change where values live, not which values a sum adds or in which
// order.  Returns the slot count (a multiple of 32).
static uint32_t color_slots(uint32_t nt, const std::vector<std::vector<uint32_t>> &rows, std::vector<uint16_t> &slot) {
  slot.assign(nt, 0);
  if (nt == 0) return 0;
  std::vector<std::vector<uint32_t>> in_rows(nt);
  for (uint32_t i = 0; i < rows.size(); i++)
    for (uint32_t j : rows[i])
      if (in_rows[j].empty() || in_rows[j].back() != i) in_rows[j].push_back(i);
  std::vector<uint32_t> order(nt);
  for (uint32_t j = 0; j < nt; j++) order[j] = j;
  std::stable_sort(order.begin(), order.end(),
                   [&](uint32_t a, uint32_t b) { return in_rows[a].size() > in_rows[b].size(); });
  const uint32_t cap = (nt + 31) / 32 + 2;
  std::vector<std::array<uint16_t, 32>> cnt(rows.size());
  std::vector<uint16_t> mx(rows.size(), 0);
  for (auto &c : cnt) c.fill(0);
  std::vector<uint32_t> fill(32, 0), bank(nt, 0);
  for (uint32_t j : order) {
    uint64_t best = ~0ull;
    uint32_t bb = 0;
    for (uint32_t b = 0; b < 32; b++) {
      if (fill[b] >= cap) continue;
      uint64_t score = 0;
      for (uint32_t i : in_rows[j]) score += (cnt[i][b] + 1u > mx[i] ? 1024u : 0u) + cnt[i][b];
      if (score < best) {
        best = score;
        bb = b;
      }
    }
    bank[j] = bb;
    fill[bb]++;
    for (uint32_t i : in_rows[j]) {
      cnt[i][bb]++;
      mx[i] = std::max<uint16_t>(mx[i], cnt[i][bb]);
    }
  }
  std::vector<uint32_t> next(32, 0);
  uint32_t maxfill = 0;
  for (uint32_t j = 0; j < nt; j++) {
    slot[j] = (uint16_t)(next[bank[j]]++ * 32 + bank[j]);
    maxfill = std::max(maxfill, next[bank[j]]);
  }
  return 32 * maxfill;
}

static bool plan_single(uint32_t n, uint32_t nlin, uint32_t sm_count, const std::vector<uint32_t> &in_row,
                        const std::vector<uint32_t> &in_code, const std::vector<float> &in_w,
                        const std::vector<uint32_t> &out_row, const std::vector<uint32_t> &out_code,
                        const std::vector<float> &out_w, const std::vector<float> &p_dfxt,
                        const std::vector<float> &p_dfst, const std::vector<float> &p_efas, const uint8_t *proj,
                        Single &S1, std::string &why) {
  // the posts are cut into blocks at groups of four (the NMDA sums' unit),
  // balancing the rows of 32 edge entries the groups take (each group's
  // longest post) plus one row's worth per group for its other work: the
  // sums phase, proportional to the rows, is the longest of a step
  const uint32_t units = (n + 3) / 4, per = kT1 / 4;
  uint32_t B = std::min<uint32_t>(sm_count, units);
  if (B == 0 || (uint64_t)B * per < units) {
    why = "more than 512 posts per block would be needed";
    return false;
  }
  std::vector<double> pre(units + 1, 0.0);
  for (uint32_t u = 0; u < units; u++) {
    uint32_t R = 0;
    for (uint32_t q = u * 4; q < std::min(n, u * 4 + 4); q++) R = std::max(R, (in_row[q + 1] - in_row[q] + 7) / 8);
    pre[u + 1] = pre[u] + 1.0 + (double)R;
  }
  std::vector<uint32_t> cut(B + 1, units);
  cut[0] = 0;
  for (uint32_t b = 1; b < B; b++) {
    const double want = pre[units] * b / B;
    uint32_t c = (uint32_t)(std::lower_bound(pre.begin(), pre.end(), want) - pre.begin());
    c = std::max(c, cut[b - 1] + 1);
    c = std::min(c, cut[b - 1] + per);
    c = std::max<uint32_t>(c, units > per * (B - b) ? units - per * (B - b) : 0);
    c = std::min(c, units - (B - b));  // every later block keeps at least one unit
    cut[b] = c;
  }
  for (uint32_t b = 0; b < B; b++)
    if (cut[b + 1] - cut[b] > per || cut[b + 1] == cut[b]) {
      why = "no balanced cut of the posts";
      return false;
    }
  // NMDA kinetics classes of the presynaptic neurons
  std::vector<int> cls_of(n, -1);
  std::vector<std::array<uint32_t, 3>> tabs;
  for (uint32_t i = 0; i < n; i++) {
    if (!(proj[i] & (1u << FS_NMDA))) continue;
    std::array<uint32_t, 3> k;
    std::memcpy(&k[0], &p_dfxt[i], 4);
    std::memcpy(&k[1], &p_dfst[i], 4);
    std::memcpy(&k[2], &p_efas[i], 4);
    size_t c = 0;
    while (c < tabs.size() && tabs[c] != k) c++;
    if (c == tabs.size()) {
      if (tabs.size() == 255) {
        why = "more than 255 NMDA kinetics classes";
        return false;
      }
      tabs.push_back(k);
    }
    cls_of[i] = (int)c;
  }
  S1.tab.clear();
  for (auto &k : tabs)
    for (int j = 0; j < 3; j++) {
      float f;
      std::memcpy(&f, &k[j], 4);
      S1.tab.push_back(f);
    }
  // linear synapses grouped by the block of their post
  std::vector<uint32_t> blk_of_unit(units);
  for (uint32_t b = 0; b < B; b++)
    for (uint32_t u = cut[b]; u < cut[b + 1]; u++) blk_of_unit[u] = b;
  std::vector<std::vector<uint64_t>> lin_b(B);  // (pre << 32) | edge index
  for (uint32_t a = 0; a < n; a++)
    for (uint32_t e = out_row[a]; e < out_row[a + 1]; e++) {
      const uint32_t post = out_code[e] & 0x3fffffu;
      lin_b[blk_of_unit[post >> 2]].push_back(((uint64_t)a << 32) | e);
    }
  std::vector<int32_t> loc(n, -1);
  S1.blk.clear();
  S1.gid.clear(); S1.lrow.clear(); S1.lin.clear(); S1.grow.clear(); S1.cls.clear(); S1.perm.clear();
  S1.linw.clear(); S1.ew.clear(); S1.eidx.clear(); S1.bits.clear(); S1.rank.clear();
  size_t smax = 0;
  bool big_lin = false;
  for (uint32_t b = 0; b < B; b++) {
    const uint32_t P0 = cut[b] * 4, P1 = std::min(n, cut[b + 1] * 4);
    std::vector<uint64_t> &L = lin_b[b];
    std::sort(L.begin(), L.end());
    std::vector<uint32_t> trk;
    for (uint32_t q = P0; q < P1; q++)
      for (uint32_t e = in_row[q]; e < in_row[q + 1]; e++) trk.push_back(in_code[e] & 0xffffffu);
    for (uint64_t x : L) trk.push_back((uint32_t)(x >> 32));
    std::sort(trk.begin(), trk.end());
    trk.erase(std::unique(trk.begin(), trk.end()), trk.end());
    if (trk.size() > 65535 - 95) {
      why = "a block tracks more than 65440 presynaptic neurons";
      return false;
    }
    big_lin |= L.size() > 65535;  // (reported after the shared-memory check)
    Blk1 bk{};
    bk.post0 = P0;
    bk.np = P1 - P0;
    bk.trk0 = (uint32_t)S1.perm.size();
    bk.ntrk = (uint32_t)trk.size();
    bk.lrow0 = (uint32_t)S1.lrow.size();
    bk.e0 = (uint32_t)S1.ew.size();
    bk.grow0 = (uint32_t)S1.grow.size();
    bk.l0 = (uint32_t)S1.lin.size();
    for (uint32_t j = 0; j < trk.size(); j++) loc[trk[j]] = (int32_t)j;
    // bitmap of the tracked ids over the words they span, and per word the
    // tracked neurons in the words before it
    bk.bm0 = (uint32_t)S1.bits.size();
    bk.w0 = trk.empty() ? 0u : trk.front() >> 5;
    bk.nwd = trk.empty() ? 0u : (trk.back() >> 5) - bk.w0 + 1;
    S1.bits.resize((size_t)bk.bm0 + bk.nwd, 0u);
    S1.rank.resize((size_t)bk.bm0 + bk.nwd, 0u);
    for (uint32_t a : trk) S1.bits[bk.bm0 + (a >> 5) - bk.w0] |= 1u << (a & 31u);
    for (uint32_t w = 0, c = 0; w < bk.nwd; w++) {
      S1.rank[bk.bm0 + w] = (uint16_t)c;
      c += (uint32_t)__builtin_popcount(S1.bits[bk.bm0 + w]);
    }
    // NMDA in-edges: posts in groups of four, a group's edges in rows of 32
    // (row r, quarter h, lane l: edge 8r + l of post 4g + h in CSR order, or
    // a zero-weight filler), as many rows as its longest post needs
    const uint32_t npb = P1 - P0, ng = (npb + 3) / 4;
    std::vector<uint32_t> grow(ng + 1, 0);
    for (uint32_t g = 0; g < ng; g++) {
      uint32_t R = 0;
      for (uint32_t h = 0; h < 4 && 4 * g + h < npb; h++) {
        const uint32_t q = P0 + 4 * g + h;
        R = std::max(R, (in_row[q + 1] - in_row[q] + 7) / 8);
      }
      grow[g + 1] = grow[g] + R;
    }
    const uint32_t nrow = grow[ng];
    std::vector<int32_t> ent((size_t)nrow * 32, -1);  // tracked index per entry, -1: filler
    std::vector<std::vector<uint32_t>> rows(nrow);
    for (uint32_t g = 0; g < ng; g++)
      for (uint32_t h = 0; h < 4 && 4 * g + h < npb; h++) {
        const uint32_t q = P0 + 4 * g + h;
        for (uint32_t e = 0; e < in_row[q + 1] - in_row[q]; e++) {
          const uint32_t r = grow[g] + e / 8, x = r * 32 + 8 * h + (e & 7u);
          ent[x] = loc[in_code[in_row[q] + e] & 0xffffffu];
          rows[r].push_back((uint32_t)ent[x]);
        }
      }
    for (auto &rw : rows) std::sort(rw.begin(), rw.end());
    std::vector<uint16_t> slot;
    bk.nslot = color_slots(bk.ntrk, rows, slot);
    if (bk.nslot > 65535) {
      why = "a block needs more than 65535 slots";
      return false;
    }
    bk.s0 = (uint32_t)S1.gid.size();
    S1.gid.resize((size_t)bk.s0 + bk.nslot, 0xffffffffu);
    S1.cls.resize((size_t)bk.s0 + bk.nslot, 255);
    for (uint32_t j = 0; j < trk.size(); j++) {
      S1.perm.push_back(slot[j]);
      S1.gid[bk.s0 + slot[j]] = trk[j];
    }
    for (uint32_t g = 0; g <= ng; g++) S1.grow.push_back(grow[g]);
    for (uint32_t x = 0; x < nrow * 32; x++) {
      if (ent[x] < 0) {
        S1.eidx.push_back(0);
        S1.ew.push_back(0.0f);
        continue;
      }
      const uint32_t r = x / 32, h = (x & 31u) / 8, g = (uint32_t)(std::upper_bound(grow.begin(), grow.end(), r) -
                                                                     grow.begin()) - 1;
      const uint32_t q = P0 + 4 * g + h, e = in_row[q] + 8 * (r - grow[g]) + (x & 7u);
      const uint32_t a = in_code[e] & 0xffffffu, sl = slot[(uint32_t)ent[x]];
      S1.eidx.push_back((uint16_t)sl);
      S1.ew.push_back(in_w[e]);
      S1.cls[bk.s0 + sl] = (uint8_t)cls_of[a];
    }
    bk.ne = nrow * 32;
    // linear rows per tracked neuron (L is sorted by neuron)
    size_t k = 0;
    for (uint32_t j = 0; j < trk.size(); j++) {
      S1.lrow.push_back((uint16_t)(S1.lin.size() - bk.l0));
      while (k < L.size() && (uint32_t)(L[k] >> 32) == trk[j]) {
        const uint32_t e = (uint32_t)L[k];
        const uint32_t post = out_code[e] & 0x3fffffu, r = (out_code[e] >> 22) & 3u;
        S1.lin.push_back((post - P0) | (r << 16));
        S1.linw.push_back(out_w[e]);
        k++;
      }
    }
    S1.lrow.push_back((uint16_t)(S1.lin.size() - bk.l0));
    for (uint32_t a : trk) loc[a] = -1;
    S1.blk.push_back(bk);
    smax = std::max(smax, single_smem(nlin, (uint32_t)tabs.size(), bk));
  }
  // dynamic shared memory next to the kernel's ~15 KB of static arrays
  if (smax > (size_t)200 * 1024) {
    why = "a block's tables need " + std::to_string(smax) + " bytes of shared memory";
    return false;
  }
  if (big_lin) {
    why = "a block receives more than 65535 linear synapses";
    return false;
  }
  S1.smem = (uint32_t)((smax + 15) & ~(size_t)15);
  return true;
}

// Host-side check of a single-step plan: every index k_prod1 forms from the
// plan stays inside the arrays and the shared memory it sizes, and the plan
// holds each synapse of the network exactly once.
static bool validate_single(const HostNet &H, const Single &S1, std::string &err) {
  const uint32_t n = H.n;
  auto fail = [&](uint32_t b, const char *what) {
    err = "single-step plan, block " + std::to_string(b) + ": " + what;
    return false;
  };
  const uint32_t ncls = (uint32_t)(S1.tab.size() / 3);
  uint32_t next_post = 0;
  uint64_t lin_total = 0, nmda_total = 0;
  for (uint32_t b = 0; b < S1.blk.size(); b++) {
    const Blk1 &k = S1.blk[b];
    if (k.post0 != next_post || k.post0 % 4 || k.np == 0 || k.np > kT1 || k.post0 + k.np > n)
      return fail(b, "post range");
    next_post = k.post0 + k.np;
    const uint32_t ng = (k.np + 3) / 4;
    if (k.ntrk > k.nslot || k.nslot % 32 || k.nslot > 65535 || (size_t)k.trk0 + k.ntrk > S1.perm.size() ||
        (size_t)k.s0 + k.nslot > S1.gid.size() || (size_t)k.s0 + k.nslot > S1.cls.size() ||
        (size_t)k.lrow0 + k.ntrk + 1 > S1.lrow.size() || (size_t)k.grow0 + ng + 1 > S1.grow.size() ||
        (size_t)k.e0 + k.ne > S1.ew.size() || (size_t)k.e0 + k.ne > S1.eidx.size() ||
        (size_t)k.bm0 + k.nwd > S1.bits.size() || (size_t)k.bm0 + k.nwd > S1.rank.size() ||
        ((uint64_t)k.w0 + k.nwd) * 32 > (uint64_t)n + 31)
      return fail(b, "table range");
    // slots: a one-to-one map of the tracked neurons into [0, nslot), the
    // other slots empty; tracked ids ascending (the bitmap's rank order)
    std::vector<int32_t> trk_of(k.nslot, -1);
    std::vector<uint32_t> trk(k.ntrk);
    for (uint32_t j = 0; j < k.ntrk; j++) {
      const uint32_t sl = S1.perm[k.trk0 + j];
      if (sl >= k.nslot || trk_of[sl] >= 0) return fail(b, "slots");
      trk_of[sl] = (int32_t)j;
      trk[j] = S1.gid[k.s0 + sl];
      if (trk[j] >= n || (j && trk[j] <= trk[j - 1])) return fail(b, "tracked ids not sorted");
    }
    for (uint32_t sl = 0; sl < k.nslot; sl++) {
      const uint8_t c = S1.cls[k.s0 + sl];
      if (trk_of[sl] < 0 && (c != 255 || S1.gid[k.s0 + sl] != 0xffffffffu)) return fail(b, "empty slot");
      if (c != 255 && c >= ncls) return fail(b, "kinetics class");
    }
    // the bitmap look-up the kernel makes gives every tracked neuron its
    // index, and the bitmap holds no other neuron
    uint32_t set = 0;
    for (uint32_t w = 0; w < k.nwd; w++) set += (uint32_t)__builtin_popcount(S1.bits[k.bm0 + w]);
    if (set != k.ntrk) return fail(b, "bitmap");
    for (uint32_t j = 0; j < k.ntrk; j++) {
      const uint32_t g = trk[j], w = (g >> 5) - k.w0;
      if (w >= k.nwd) return fail(b, "bitmap");
      const uint32_t word = S1.bits[k.bm0 + w];
      if (!((word >> (g & 31u)) & 1u) ||
          S1.rank[k.bm0 + w] + (uint32_t)__builtin_popcount(word & ((1u << (g & 31u)) - 1u)) != j)
        return fail(b, "bitmap");
    }
    const uint16_t *lr = &S1.lrow[k.lrow0];
    if (lr[0] != 0) return fail(b, "linear rows");
    for (uint32_t j = 0; j < k.ntrk; j++)
      if (lr[j + 1] < lr[j]) return fail(b, "linear rows");
    if ((size_t)k.l0 + lr[k.ntrk] > S1.lin.size() || (size_t)k.l0 + lr[k.ntrk] > S1.linw.size())
      return fail(b, "linear entries");
    for (uint32_t e = 0; e < lr[k.ntrk]; e++) {
      const uint32_t code = S1.lin[k.l0 + e], r = code >> 16, q = code & 0xffffu;
      if (q >= k.np || r > 3 || H.lin_of_rec[r] < 0) return fail(b, "linear entry");
    }
    lin_total += lr[k.ntrk];
    // NMDA edges: every edge of every post at its entry (row grow[g] + e / 8,
    // quarter h, lane e mod 8) with its weight and its source's slot, every
    // other entry of the group's rows a zero-weight filler on a valid slot
    const uint32_t *gr = &S1.grow[k.grow0];
    if (gr[0] != 0 || (uint64_t)gr[ng] * 32 != k.ne) return fail(b, "group rows");
    std::vector<uint8_t> used(k.ne, 0);
    for (uint32_t g = 0; g < ng; g++) {
      if (gr[g + 1] < gr[g]) return fail(b, "group rows");
      for (uint32_t h = 0; h < 4 && 4 * g + h < k.np; h++) {
        const uint32_t q = k.post0 + 4 * g + h, b0 = H.in_row[q], len = H.in_row[q + 1] - b0;
        if ((len + 7) / 8 > gr[g + 1] - gr[g]) return fail(b, "group rows");
        for (uint32_t e = 0; e < len; e++) {
          const uint32_t x = (gr[g] + e / 8) * 32 + 8 * h + (e & 7u);
          const uint16_t sl = S1.eidx[k.e0 + x];
          if (sl >= k.nslot || trk_of[sl] < 0 || S1.cls[k.s0 + sl] == 255) return fail(b, "edge slot");
          if (trk[trk_of[sl]] != (H.in_code[b0 + e] & 0xffffffu)) return fail(b, "edge source");
          if (std::memcmp(&S1.ew[k.e0 + x], &H.in_w[b0 + e], 4) != 0) return fail(b, "edge weight");
          used[x] = 1;
        }
      }
    }
    for (uint32_t x = 0; x < k.ne; x++) {
      if (used[x]) {
        nmda_total++;
      } else if (S1.ew[k.e0 + x] != 0.0f || std::signbit(S1.ew[k.e0 + x]) || S1.eidx[k.e0 + x] >= k.nslot) {
        return fail(b, "filler");
      }
    }
    if (single_smem(H.nlin, ncls, k) > S1.smem) return fail(b, "shared memory");
  }
  if (next_post != n) return fail((uint32_t)S1.blk.size(), "posts not covered");
  if (lin_total != H.nlin_e || nmda_total != H.nnm_e) return fail(0, "synapse count");
  return true;
}

int prod_check_single_plan(const fs_net_desc *d, uint32_t sm_count, uint64_t *stats, std::string &err) {
  HostNet H;
  int rc = host_net(d, H, err);
  if (rc) return rc;
  for (int i = 0; i < 8; i++) stats[i] = 0;
  if (H.dmax != 0) return FS_OK;
  Single S1;
  if (!plan_single(H.n, H.nlin, sm_count, H.in_row, H.in_code, H.in_w, H.out_row, H.out_code, H.out_w, H.p_dfxt,
                   H.p_dfst, H.p_efas, H.proj.data(), S1, err))
    return FS_OK;
  if (!validate_single(H, S1, err)) return FS_ERR_ARG;
  stats[0] = 1;
  stats[1] = S1.blk.size();
  for (const Blk1 &k : S1.blk) {
    stats[2] = std::max<uint64_t>(stats[2], k.np);
    stats[3] = std::max<uint64_t>(stats[3], k.ntrk);
    stats[4] = std::max<uint64_t>(stats[4], H.in_row[k.post0 + k.np] - H.in_row[k.post0]);
  }
  stats[5] = S1.smem;
  stats[6] = S1.lin.size();
  stats[7] = H.nnm_e;
  return FS_OK;
}

static int prod_create_from(Prod **out, const fs_net_desc *d, const fs_run_opts &o, uint32_t sm_count,
                            cudaStream_t st, std::string &err, bool allow_single, HostNet *pre);

// Tables and state of long-term plasticity (k_prod_ltp).  The LTP records
// are the synapse-list entries with ltp[e] set (all of them when the list
// has no flags): the reference's single-target records (SynFst1 and
// SynSlo1, code/EqsGnl2.cpp:1005-1044), whose presynaptic neuron here is
// the true one.  Each record is located by the index of its weight in
// out_w or in_w, replaying host_net's fill order.
static int ltp_create(Prod *p, const fs_net_desc *d, const HostNet &H, size_t T, cudaStream_t st, std::string &err) {
  const fs_neurons &v = d->neurons;
  const fs_syn_list &S = *d->syn;
  const uint32_t n = p->n;
  Params &P = p->P;
  std::vector<uint32_t> fo(H.out_row.begin(), H.out_row.end() - 1), fi(H.in_row.begin(), H.in_row.end() - 1);
  std::vector<uint32_t> orow(n + 1, 0), irow(n + 1, 0), pos(S.n);
  for (uint64_t e = 0; e < S.n; e++) {
    pos[e] = S.rec[e] == FS_NMDA ? fi[S.post[e]]++ : fo[S.pre[e]]++;
    if (!S.ltp || S.ltp[e]) {
      orow[S.pre[e] + 1]++;
      irow[S.post[e] + 1]++;
    }
  }
  for (uint32_t i = 0; i < n; i++) {
    orow[i + 1] += orow[i];
    irow[i + 1] += irow[i];
  }
  const uint32_t nr = orow[n];
  if (H.nlin_e >= (1ull << 31) || H.nnm_e >= (1ull << 31)) {
    err = "networks with LTP: at most 2^31 - 1 synapses per receptor class";
    return FS_ERR_UNSUPPORTED;
  }
  p->wpos.resize(S.n);
  for (uint64_t e = 0; e < S.n; e++) p->wpos[e] = pos[e] | (S.rec[e] == FS_NMDA ? 0x80000000u : 0u);
  std::vector<uint32_t> oent(nr), oidx(nr), ient(nr), iidx(nr);
  {
    std::vector<uint32_t> a(orow.begin(), orow.end() - 1), b(irow.begin(), irow.end() - 1);
    for (uint64_t e = 0; e < S.n; e++) {
      if (S.ltp && !S.ltp[e]) continue;
      const uint32_t r = S.rec[e], x = a[S.pre[e]]++, y = b[S.post[e]]++;
      oent[x] = S.post[e] | (r << 24);
      oidx[x] = pos[e];
      ient[y] = S.pre[e] | (r << 24);
      iidx[y] = pos[e];
    }
  }
  std::vector<float> zf(n, 0.0f);
  std::vector<int32_t> zi(n, 0);
  int rc;
  if ((rc = dup(p, (uint32_t **)&P.ltp_orow, orow.data(), orow.size(), st, err)) ||
      (rc = dup(p, (uint32_t **)&P.ltp_irow, irow.data(), irow.size(), st, err)) ||
      (rc = dup(p, (uint32_t **)&P.ltp_oent, oent.data(), nr, st, err)) ||
      (rc = dup(p, (uint32_t **)&P.ltp_oidx, oidx.data(), nr, st, err)) ||
      (rc = dup(p, (uint32_t **)&P.ltp_ient, ient.data(), nr, st, err)) ||
      (rc = dup(p, (uint32_t **)&P.ltp_iidx, iidx.data(), nr, st, err)) ||
      (rc = dup(p, (float **)&P.ltp_dflp, v.ltp_dfLP ? v.ltp_dfLP : zf.data(), n, st, err)) ||
      (rc = dup(p, (float **)&P.ltp_pos, v.ltp_PosISI ? v.ltp_PosISI : zf.data(), n, st, err)) ||
      (rc = dup(p, (float **)&P.ltp_neg, v.ltp_NegISI ? v.ltp_NegISI : zf.data(), n, st, err)) ||
      (rc = dup(p, (int32_t **)&P.ltp_spd, v.ltp_SpiLPDy ? v.ltp_SpiLPDy : zi.data(), n, st, err)) ||
      (rc = dup(p, (uint8_t **)&P.ltp_lp, (const uint8_t *)nullptr, (size_t)n * 4, st, err)) ||
      (rc = dup(p, &P.ltp_clp, (const int32_t *)nullptr, n, st, err)) ||
      (rc = dup(p, (uint8_t **)&P.ltp_lp2, (const uint8_t *)nullptr, (size_t)2 * n * 4, st, err)) ||
      (rc = dup(p, (uint8_t **)&P.ltp_sp2, (const uint8_t *)nullptr, 8 * n * T, st, err)) ||
      (rc = dup(p, &P.ltp_spk2, (const uint8_t *)nullptr, 2 * (size_t)n, st, err)) ||
      (rc = dup(p, (uint8_t **)&P.ltp_gn, (const uint8_t *)nullptr, n * T, st, err)) ||
      (rc = dup(p, &P.ltp_cnt, (const uint32_t *)nullptr, 2, st, err)) ||
      (rc = dup(p, &P.ltp_id, (const uint32_t *)nullptr, 2 * (size_t)n, st, err)) ||
      (rc = dup(p, &P.ltp_tm, (const uint16_t *)nullptr, 2 * (size_t)n, st, err)) ||
      (rc = dup(p, (uint8_t **)&P.ltp_c, (const uint8_t *)nullptr, 8 * n * T, st, err)))
    return rc;
  return FS_OK;
}

int prod_create(Prod **out, const fs_net_desc *d, const fs_run_opts &o, uint32_t sm_count, cudaStream_t st,
                std::string &err, bool allow_single) {
  return prod_create_from(out, d, o, sm_count, st, err, allow_single, nullptr);
}

// pre: host tables already built by host_net (moved from), or null
static int prod_create_from(Prod **out, const fs_net_desc *d, const fs_run_opts &o, uint32_t sm_count,
                            cudaStream_t st, std::string &err, bool allow_single, HostNet *pre) {
  *out = nullptr;
  const fs_neurons &v = d->neurons;
  const uint32_t n = v.n;
  if (n >= (1u << 22)) {
    err = "production modes support up to 4,194,303 neurons per handle";
    return FS_ERR_UNSUPPORTED;
  }
  // long-term plasticity runs on its own persistent kernel (k_prod_ltp):
  // not in batches, not on the tile kernels, and only without delays (the
  // reference has none; a weight change would otherwise have to reach
  // every delayed copy of the record's gate)
  const bool ltp = (d->act_ctr & FS_ACT_LTP) != 0;
  if (ltp && !allow_single) {
    err = "batches do not run networks with LTP (create them one by one)";
    return FS_ERR_UNSUPPORTED;
  }
  if (ltp && (o.flags & FS_RUN_TILE_KERNELS)) {
    err = "networks with LTP run on their own persistent kernel, not on the tile kernels";
    return FS_ERR_UNSUPPORTED;
  }
  // gap junctions: the per-neuron term lists of the compat layout (other
  // neuron, conductance), applied with a one-step lag as the reference does
  // (its Spike phase adds them to Isyn for the next step's VmEul,
  // code/EqsGnl2.cpp:705-725, :982-999)
  const bool gap = d->compat && d->compat->gap_rowptr && d->compat->gap_rowptr[n] != 0;
  Prod *p = new Prod();
  p->fp64 = (o.mode == FS_MODE_FP64);
  p->n = n;
  p->sm = sm_count;
  p->key = o.philox_key;
  p->chunk_steps = o.chunk_steps ? o.chunk_steps : 1000;
  Params &P = p->P;
  P.n = n;
  for (int r = 0; r < 5; r++) P.rg[r] = 1.0f;
  const size_t nr = (size_t)FS_NREC * n;
  HostNet H;
  if (pre) {
    H = std::move(*pre);
  } else {
    int hrc = host_net(d, H, err);
    if (hrc) {
      delete p;
      return hrc;
    }
  }
  const uint32_t dmin = H.dmin, dmax = H.dmax;
  const uint64_t nlin_e = H.nlin_e, nnm_e = H.nnm_e;
  if (ltp && dmax != 0) {
    delete p;
    err = "networks with LTP need every synaptic delay 0 in the production modes";
    return FS_ERR_UNSUPPORTED;
  }
  p->ltp = ltp;
  std::vector<float> &pdf = H.pdf, &p_dfxt = H.p_dfxt, &p_dfst = H.p_dfst, &p_efas = H.p_efas;
  std::vector<uint8_t> &proj = H.proj;
  std::vector<uint32_t> &out_row = H.out_row, &in_row = H.in_row, &out_code = H.out_code, &in_code = H.in_code;
  std::vector<float> &out_w = H.out_w, &in_w = H.in_w;
  const fs_syn_list &S = *d->syn;
  p->d_min = dmin;
  p->d_max = dmax;
  p->lin_edges = nlin_e;
  p->nmda_edges = nnm_e;
  {
    uint32_t need = dmax + dmin + 2, S = 8;
    while (S < need) S <<= 1;
    P.slots = S;
    P.mask = S - 1;
  }
  P.interval = std::max<uint32_t>(1, dmin);
  P.dmax0 = dmax == 0 ? 1u : 0u;
  if (gap) P.interval = 1;  // a gap current reads every neuron's V of the step before
  p->nlin = H.nlin;
  for (int r = 0; r < 4; r++) P.lin_of_rec[r] = H.lin_of_rec[r];
  P.nlin = p->nlin;
  // ---- grid: all blocks co-resident; posts split by estimated cost ----
  int occ = 0;
  {
    const void *kq = ltp ? (p->fp64 ? (const void *)k_prod_ltp<double> : (const void *)k_prod_ltp<float>)
                         : (p->fp64 ? (const void *)k_prod<double, 4> : (const void *)k_prod<float, 4>);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kq, kThreads, 0);
  }
  if (occ < 1) occ = 1;
  int per_sm = std::min(occ, 4);
  if (o.blocks_per_sm) per_sm = std::min<int>(occ, (int)o.blocks_per_sm);
  uint32_t blocks = sm_count * (uint32_t)per_sm;
  blocks = std::max<uint32_t>(1, std::min<uint32_t>(blocks, (n + 7) / 8));
  p->blocks = blocks;
  std::vector<uint32_t> block_post(blocks + 1, n);
  block_post[0] = 0;
  {
    // cost of a post: its NMDA in-edges (pull) plus a fixed update cost
    const double upd = 24.0;
    const double total = (double)nnm_e + upd * n;
    double acc = 0;
    uint32_t b = 1;
    for (uint32_t q = 0; q < n && b < blocks; q++) {
      acc += upd + (double)(in_row[q + 1] - in_row[q]);
      while (b < blocks && acc >= total * b / blocks) block_post[b++] = q + 1;
    }
    for (; b < blocks; b++) block_post[b] = n;
  }
  p->chunks = blocks;
  for (uint32_t b = 0; b < blocks; b++)
    if (block_post[b + 1] - block_post[b] > kTile) p->wide = true;
  p->in_row_h = in_row;
  // ---- device arrays ----
  int rc = 0;
  const size_t T = p->fp64 ? 8 : 4;
#define UPF(field, src, cnt) if ((rc = dup(p, (float **)&P.field, src, cnt, st, err))) goto fail
#define UPI(field, src, cnt) if ((rc = dup(p, (int32_t **)&P.field, src, cnt, st, err))) goto fail
#define UPU(field, src, cnt) if ((rc = dup(p, (uint32_t **)&P.field, src, cnt, st, err))) goto fail
  UPF(Vth, v.Vth, n); UPF(El, v.El, n); UPF(gl, v.gl, n); UPF(Cm, v.Cm, n); UPF(Vreset, v.Vreset, n);
  UPF(df, v.df, n); UPF(ef, v.ef, n); UPF(dVmax, v.dVmax, n); UPI(RfPed, v.RfPed, n); UPI(SpiDy, v.SpiDy, n);
  UPF(Vrev, v.Vrev, nr); UPF(dfst, v.dfst, nr); UPF(nmda_dfxt, v.nmda_dfxt, n); UPF(nmda_efst, v.nmda_efst, n);
  UPF(nmda_as, v.nmda_as, n); UPF(nmda_mg, v.nmda_mg, n); UPF(ext_g, v.ext_g, nr);
  UPF(pb, v.pb, nr); UPU(act, v.act, n); UPF(inj_mean, v.inj_mean, n); UPF(inj_std, v.inj_std, n);
  UPF(pdf, pdf.data(), pdf.size()); UPF(p_dfxt, p_dfxt.data(), n); UPF(p_dfst, p_dfst.data(), n);
  UPF(p_efas, p_efas.data(), n);
  if ((rc = dup(p, (uint8_t **)&P.proj, proj.data(), n, st, err))) goto fail;
  UPF(stp_pv, v.stp_pv, n); UPF(stp_dfD, v.stp_dfD, n); UPF(stp_efD, v.stp_efD, n); UPF(stp_aF, v.stp_aF, n);
  UPF(stp_dfF, v.stp_dfF, n); UPF(stp_efF, v.stp_efF, n); UPF(stp_aCap, v.stp_aCap, n);
  UPF(stp_dfCap, v.stp_dfCap, n); UPF(stp_aCar, v.stp_aCar, n); UPF(stp_dfCar, v.stp_dfCar, n);
  UPF(stp_efCar, v.stp_efCar, n);
  P.plast = (d->act_ctr & FS_ACT_STP) ? PL_STP : (d->act_ctr & FS_ACT_STD) ? PL_STD : PL_NONE;
  if (d->tm && d->tm->enabled) {
    if (P.plast != PL_NONE) {
      err = "Tsodyks-Markram parameters and the reference STD/STP flags are exclusive";
      rc = FS_ERR_ARG;
      goto fail;
    }
    P.plast = PL_TM;
    std::vector<float> U(n), dfr(n), dff(n);
    for (uint32_t i = 0; i < n; i++) {
      U[i] = d->tm->U ? d->tm->U[i] : 0.2f;
      const float tr = d->tm->tau_rec ? d->tm->tau_rec[i] : 200.0f, tf = d->tm->tau_fac ? d->tm->tau_fac[i] : 600.0f;
      dfr[i] = tr > 0 ? std::exp(-d->dt / tr) : 0.0f;
      dff[i] = tf > 0 ? std::exp(-d->dt / tf) : 0.0f;
    }
    if ((rc = dup(p, (uint8_t **)&P.tm_on, d->tm->enabled, n, st, err))) goto fail;
    UPF(tm_U, U.data(), n); UPF(tm_dfr, dfr.data(), n); UPF(tm_dff, dff.data(), n);
  }
  // state
  if ((rc = dup(p, (uint8_t **)&P.V, (const uint8_t *)nullptr, n * T, st, err)) ||
      (rc = dup(p, (uint8_t **)&P.G, (const uint8_t *)nullptr, 4 * n * T, st, err)) ||
      (rc = dup(p, (uint8_t **)&P.ext_st, (const uint8_t *)nullptr, 4 * n * T, st, err)) ||
      (rc = dup(p, (uint8_t **)&P.ext_x, (const uint8_t *)nullptr, n * T, st, err)) ||
      (rc = dup(p, (uint8_t **)&P.ext_s, (const uint8_t *)nullptr, n * T, st, err)) ||
      (rc = dup(p, (uint8_t **)&P.st_pre, (const uint8_t *)nullptr, 4 * n * T, st, err)) ||
      (rc = dup(p, (uint8_t **)&P.x_pre, (const uint8_t *)nullptr, n * T, st, err)) ||
      (rc = dup(p, (uint8_t **)&P.s_pre, (const uint8_t *)nullptr, n * T, st, err)) ||
      (rc = dup(p, (uint8_t **)&P.s_hist, (const uint8_t *)nullptr, (size_t)P.slots * n * T * (p->fp64 ? 1 : kSH), st, err)) ||
      (rc = dup(p, &P.Count, (const int32_t *)nullptr, n, st, err)) ||
      (rc = dup(p, &P.NS, (const uint32_t *)nullptr, n, st, err)) ||
      (rc = dup(p, &P.D, (const float *)nullptr, n, st, err)) || (rc = dup(p, &P.F, (const float *)nullptr, n, st, err)) ||
      (rc = dup(p, &P.Cap, (const float *)nullptr, n, st, err)) || (rc = dup(p, &P.Car, (const float *)nullptr, n, st, err)) ||
      (rc = dup(p, &P.tm_u, (const float *)nullptr, n, st, err)) || (rc = dup(p, &P.tm_x, (const float *)nullptr, n, st, err)) ||
      (rc = dup(p, &P.nspk, (const uint32_t *)nullptr, n, st, err)) ||
      (rc = dup(p, &P.Irep, (const float *)nullptr, (size_t)5 * n, st, err)) ||
      (rc = dup(p, &P.ring, (const unsigned long long *)nullptr, (size_t)std::max<uint32_t>(1, p->nlin) * P.slots * n, st, err)))
    goto fail;
  // edges
  UPU(out_row, out_row.data(), (size_t)n + 1); UPU(out_code, out_code.data(), out_code.size());
  UPF(out_w, out_w.data(), out_w.size());
  if (nnm_e) {
    UPU(in_row, in_row.data(), (size_t)n + 1); UPU(in_code, in_code.data(), in_code.size());
    UPF(in_w, in_w.data(), in_w.size());
  } else {
    P.in_row = nullptr;
  }
  UPU(block_post, block_post.data(), block_post.size());
  if (d->compat)
    for (int r = 0; r < FS_NREC; r++) {
      const fs_rec_layout &L = d->compat->rec[r];
      const uint32_t *src = L.rec_src ? L.rec_src : L.rec_pre;
      if (L.n_recs && src) p->rec_src[r].assign(src, src + L.n_recs);
    }
  // single-step kernel: FP32, every delay 0, no gap junctions
  if (allow_single && !ltp && !p->fp64 && dmax == 0 && !gap && S.n > 0 && !(o.flags & FS_RUN_INTERVAL_KERNEL)) {
    Single S1;
    std::string why;
    if (plan_single(n, p->nlin, sm_count, in_row, in_code, in_w, out_row, out_code, out_w, p_dfxt, p_dfst, p_efas,
                    proj.data(), S1, why)) {
      if (!validate_single(H, S1, err)) {
        rc = FS_ERR_ARG;
        goto fail;
      }
      // the attribute is per kernel, not per handle: always the largest
      // dynamic size any plan may take
      int dev = 0, maxsm = 0;
      cudaGetDevice(&dev);
      cudaDeviceGetAttribute(&maxsm, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
      cudaFuncAttributes fa{};
      cudaFuncGetAttributes(&fa, (const void *)k_prod1<true>);
      const int dyn_max = std::min<int>(200 * 1024, maxsm - (int)fa.sharedSizeBytes);
      if ((int)S1.smem <= dyn_max &&
          cudaFuncSetAttribute((const void *)k_prod1<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn_max) ==
              cudaSuccess &&
          cudaFuncSetAttribute((const void *)k_prod1<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn_max) ==
              cudaSuccess) {
        if ((rc = dup(p, (Blk1 **)&P.b1, S1.blk.data(), S1.blk.size(), st, err))) goto fail;
        UPU(t1_gid, S1.gid.data(), S1.gid.size());
        if ((rc = dup(p, (uint16_t **)&P.t1_lrow, S1.lrow.data(), S1.lrow.size(), st, err))) goto fail;
        if ((rc = dup(p, (uint16_t **)&P.t1_perm, S1.perm.data(), S1.perm.size(), st, err))) goto fail;
        UPU(t1_lin, S1.lin.data(), S1.lin.size());
        UPU(t1_grow, S1.grow.data(), S1.grow.size());
        if ((rc = dup(p, (uint8_t **)&P.t1_cls, S1.cls.data(), S1.cls.size(), st, err))) goto fail;
        UPF(t1_linw, S1.linw.data(), S1.linw.size());
        UPF(t1_ew, S1.ew.data(), S1.ew.size());
        UPF(t1_cls_tab, S1.tab.data(), S1.tab.size());
        if ((rc = dup(p, (uint16_t **)&P.t1_eidx, S1.eidx.data(), S1.eidx.size(), st, err))) goto fail;
        UPU(t1_bits, S1.bits.data(), S1.bits.size());
        if ((rc = dup(p, (uint16_t **)&P.t1_rank, S1.rank.data(), S1.rank.size(), st, err))) goto fail;
        if ((rc = dup(p, &P.t1_cnt, (const uint32_t *)nullptr, 4, st, err))) goto fail;
        P.t1_slots = std::min<uint32_t>(16, kT1F / (uint32_t)S1.blk.size());
        // one 16-byte word per listed spike when no neuron projects onto two
        // linear receptors (its one c travels alone), else two
        P.t1_w = 1;
        for (uint32_t i = 0; i < n; i++)
          if (__builtin_popcount(proj[i] & 15u) > 1) P.t1_w = 2;
        if ((rc = dup(p, &P.t1_list, (const uint4 *)nullptr, (size_t)2 * S1.blk.size() * P.t1_slots * 2, st, err)) ||
            (rc = dup(p, &P.t1_ovf, (const uint4 *)nullptr, (size_t)4 * n, st, err)))
          goto fail;
        P.t1_ncls = (uint32_t)(S1.tab.size() / 3);
        P.t1_smem = S1.smem;
        p->single = true;
        p->b1_blocks = (uint32_t)S1.blk.size();
      }
      cudaGetLastError();
    }
  }
  // tile kernels: networks whose blocks would each walk more than two tiles
  // of posts per batch (at 2 blocks per SM: above ~150,000 neurons)
  if (allow_single && !ltp && !p->single && !(o.flags & FS_RUN_INTERVAL_KERNEL) &&
      ((o.flags & FS_RUN_TILE_KERNELS) || (uint64_t)n > (uint64_t)p->blocks * 2 * (p->fp64 ? TileW<double>::W : kTile))) {
    if ((rc = tiles_solo_create(p, err))) goto fail;
  }
  if (gap) {
    const uint32_t ng = d->compat->gap_rowptr[n];
    UPU(gap_row, d->compat->gap_rowptr, (size_t)n + 1);
    UPU(gap_other, d->compat->gap_other, ng);
    UPF(gap_w, d->compat->gap_g, ng);
    if ((rc = dup(p, (uint8_t **)&P.Vg, (const uint8_t *)nullptr, 2 * n * T, st, err))) goto fail;
  } else {
    P.gap_row = P.gap_other = nullptr;
    P.gap_w = nullptr;
    P.Vg = nullptr;
  }
  if (ltp && (rc = ltp_create(p, d, H, T, st, err))) goto fail;
  if ((rc = dal(p, &p->bar, 64, err)) || (rc = dal(p, &p->err, 1, err)) ||
      (rc = dup(p, &p->spike_total, (const unsigned long long *)nullptr, 1, st, err)))
    goto fail;
  if (cudaMemsetAsync(p->err, 0, 4, st) != cudaSuccess) { rc = FS_ERR_CUDA; err = "memset"; goto fail; }
  if (cudaStreamSynchronize(st) != cudaSuccess) { rc = FS_ERR_CUDA; err = "upload sync"; goto fail; }
#undef UPF
#undef UPI
#undef UPU
  *out = p;
  return FS_OK;
fail:
  prod_destroy(p);
  return rc ? rc : FS_ERR_CUDA;
}

void prod_destroy(Prod *p) {
  if (!p) return;
  if (p->tiles) tiles_delete(p->tiles);
  for (void *q : p->allocs) cudaFree(q);
  for (auto &x : p->ev) {
    cudaEventDestroy(x.first);
    cudaEventDestroy(x.second);
  }
  delete p;
}

int prod_upload_params(Prod *p, const float *pb, const uint32_t *act, const float *inj_mean, const float *inj_std,
                       cudaStream_t st, std::string &err) {
  const size_t n = p->n;
  cudaError_t e = cudaMemcpyAsync((void *)p->P.pb, pb, FS_NREC * n * 4, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync((void *)p->P.act, act, n * 4, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync((void *)p->P.inj_mean, inj_mean, n * 4, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync((void *)p->P.inj_std, inj_std, n * 4, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    err = std::string("parameter upload: ") + cudaGetErrorString(e);
    return FS_ERR_CUDA;
  }
  return FS_OK;
}

__global__ void k_prod_init(const __grid_constant__ Params P, int fp64) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P.n) return;
  if (fp64) ((double *)P.V)[i] = -70.0;
  else ((float *)P.V)[i] = -70.0f;
  const uint32_t a = P.act[i];
  if (a & FS_ACT_STP) { P.D[i] = 1.0f; P.F[i] = 1.0f; P.Cap[i] = 0.0f; P.Car[i] = 20.0f; }
  else { P.D[i] = 1.0f; P.F[i] = 0.0f; }
  if (P.tm_U) { P.tm_u[i] = P.tm_U[i]; P.tm_x[i] = 1.0f; }
}

int prod_reset(Prod *p, uint32_t seed, cudaStream_t st, std::string &err) {
  const size_t n = p->n, T = p->fp64 ? 8 : 4;
  Params &P = p->P;
  cudaError_t e = cudaSuccess;
  auto z = [&](void *ptr, size_t bytes) {
    if (e == cudaSuccess && ptr && bytes) e = cudaMemsetAsync(ptr, 0, bytes, st);
  };
  z(P.G, 4 * n * T); z(P.ext_st, 4 * n * T); z(P.ext_x, n * T); z(P.ext_s, n * T);
  z(P.st_pre, 4 * n * T); z(P.x_pre, n * T); z(P.s_pre, n * T); z(P.s_hist, (size_t)P.slots * n * T * (p->fp64 ? 1 : kSH));
  z(P.Count, n * 4); z(P.NS, n * 4); z(P.Cap, n * 4); z(P.Car, n * 4); z(P.nspk, n * 4); z(P.Irep, (size_t)5 * n * 4);
  z(P.ring, (size_t)std::max<uint32_t>(1, p->nlin) * P.slots * n * 8);
  z(P.Vg, 2 * n * T);
  // LTP: trace and counter (VarInit, code/EqsGnl2.cpp:363-367); the weights
  // keep what earlier runs made of them, as the reference's records do
  z(P.ltp_lp, n * 4);
  z(P.ltp_clp, n * 4);
  z(P.ltp_gn, n * T);  // the NMDA sums of step 0 (the history is empty)
  z(P.ltp_cnt, 8);
  z(p->err, 4);
  z(p->spike_total, 8);
  if (e == cudaSuccess) {
    k_prod_init<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(P, p->fp64 ? 1 : 0);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    err = std::string("reset: ") + cudaGetErrorString(e);
    return FS_ERR_CUDA;
  }
  // stream key: user key and the run seed
  P.key0 = (uint32_t)p->key ^ seed;
  P.key1 = (uint32_t)(p->key >> 32) ^ 0x5eed5eedu;
  p->t = 0;
  p->ms = 0.0;
  p->kl = 0;
  p->ev_used = 0;
  return FS_OK;
}

// Device tables of a GatingVariable selection (out->gv_sel: receptor << 28
// | record index): per presynaptic neuron, its output columns; output
// buffers for chunks of up to `steps` steps.
static int gv_prepare(Prod *p, const fs_step_out *out, uint32_t steps, cudaStream_t st, std::string &err) {
  const uint32_t n = p->n, k = out->gv_n;
  std::vector<uint32_t> row(n + 1, 0), ent(k);
  std::vector<uint32_t> src(k);
  for (uint32_t i = 0; i < k; i++) {
    const uint32_t r = out->gv_sel[i] >> 28, e = out->gv_sel[i] & 0x0fffffffu;
    if (r >= FS_NREC || e >= p->rec_src[r].size() || p->rec_src[r][e] >= n) {
      err = "GatingVariable selection " + std::to_string(i) + " names no single-target record of the network";
      return FS_ERR_ARG;
    }
    src[i] = p->rec_src[r][e];
    row[src[i] + 1]++;
  }
  for (uint32_t i = 0; i < n; i++) row[i + 1] += row[i];
  {
    std::vector<uint32_t> fill(row.begin(), row.end() - 1);
    for (uint32_t i = 0; i < k; i++) ent[fill[src[i]]++] = i | ((out->gv_sel[i] >> 28) << 28);
  }
  int rc;
  if (!p->gv_row && (rc = dal(p, &p->gv_row, (size_t)n + 1, err))) return rc;
  if (k > p->gv_ent_cap) {
    if ((rc = dal(p, &p->gv_ent, k, err))) return rc;
    p->gv_ent_cap = k;
  }
  if ((uint64_t)steps * k > p->gv_out_cap) {
    if ((rc = dal(p, &p->gv_st, (size_t)steps * k, err)) || (rc = dal(p, &p->gv_xt, (size_t)steps * k, err)))
      return rc;
    p->gv_out_cap = (uint64_t)steps * k;
  }
  cudaError_t e = cudaMemcpyAsync(p->gv_row, row.data(), (size_t)(n + 1) * 4, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(p->gv_ent, ent.data(), (size_t)k * 4, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    err = std::string("GatingVariable tables: ") + cudaGetErrorString(e);
    return FS_ERR_CUDA;
  }
  p->P.gv_n = k;
  return FS_OK;
}

int prod_step(Prod *p, uint32_t nsteps, fs_step_out *out, uint64_t *written, cudaStream_t st, uint64_t *launches,
              uint64_t *spikes_total, std::string &err) {
  const uint32_t n = p->n, words = (n + 31) / 32;
  uint32_t chunk = p->chunk_steps;
  if ((uint64_t)chunk * n > (64ull << 20)) chunk = (uint32_t)std::max<uint64_t>(1, (64ull << 20) / n);
  uint32_t done = 0;
  while (done < nsteps) {
    const uint32_t b = std::min(chunk, nsteps - done);
    const bool wantV = out && out->V, wantI = out && out->Irep, wantNS = out && out->nstate;
    const bool wantGV = out && out->gv_n && out->gv_sel && out->gv_st;
    if (wantGV && done == 0) {
      int grc = gv_prepare(p, out, b, st, err);
      if (grc) return grc;
    }
    int rc = launch(p, b, true, wantV, st, launches, err, wantI, wantNS, wantGV);
    if (rc) return rc;
    cudaError_t e = fsd::spikes_compact(p->bits, b, words, p->counts, p->offsets, p->idx, st, launches);
    if (e != cudaSuccess) { err = cudaGetErrorString(e); return FS_ERR_CUDA; }
    if ((rc = finish(p, st, err))) return rc;
    uint32_t total = 0;
    e = cudaMemcpyAsync(&total, p->offsets + b, 4, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess && out && out->spike_count)
      e = cudaMemcpyAsync(out->spike_count + done, p->counts, (size_t)b * 4, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) { err = cudaGetErrorString(e); return FS_ERR_CUDA; }
    if (out && out->spike_idx) {
      if (*written + total > out->spike_cap) {
        err = "spike_idx buffer too small";
        return FS_ERR_CAPACITY;
      }
      e = cudaMemcpy(out->spike_idx + *written, p->idx, (size_t)total * 4, cudaMemcpyDeviceToHost);
      if (e != cudaSuccess) { err = cudaGetErrorString(e); return FS_ERR_CUDA; }
    }
    if (wantV) {
      e = cudaMemcpy(out->V + (size_t)done * n, p->outV, (size_t)b * n * 4, cudaMemcpyDeviceToHost);
      if (e != cudaSuccess) { err = cudaGetErrorString(e); return FS_ERR_CUDA; }
    }
    if (wantI) {
      e = cudaMemcpy(out->Irep + (size_t)done * 5 * n, p->outI, (size_t)b * 5 * n * 4, cudaMemcpyDeviceToHost);
      if (e != cudaSuccess) { err = cudaGetErrorString(e); return FS_ERR_CUDA; }
    }
    if (wantNS) {
      e = cudaMemcpy(out->nstate + (size_t)done * n, p->outNS, (size_t)b * n * 4, cudaMemcpyDeviceToHost);
      if (e != cudaSuccess) { err = cudaGetErrorString(e); return FS_ERR_CUDA; }
    }
    if (wantGV) {
      e = cudaMemcpy(out->gv_st + (size_t)done * out->gv_n, p->gv_st, (size_t)b * out->gv_n * 4,
                     cudaMemcpyDeviceToHost);
      if (e == cudaSuccess && out->gv_xt)
        e = cudaMemcpy(out->gv_xt + (size_t)done * out->gv_n, p->gv_xt, (size_t)b * out->gv_n * 4,
                       cudaMemcpyDeviceToHost);
      if (e != cudaSuccess) { err = cudaGetErrorString(e); return FS_ERR_CUDA; }
    }
    *written += total;
    if (spikes_total) *spikes_total += total;
    done += b;
  }
  return FS_OK;
}

int prod_run(Prod *p, uint32_t nsteps, cudaStream_t st, uint64_t *launches, std::string &err) {
  uint32_t done = 0;
  while (done < nsteps) {
    const uint32_t b = std::min(p->chunk_steps, nsteps - done);
    int rc = launch(p, b, false, false, st, launches, err);
    if (rc) return rc;
    done += b;
  }
  return FS_OK;
}

int prod_check(Prod *p, cudaStream_t st, uint64_t *spikes_total, std::string &err) {
  int rc = finish(p, st, err);
  if (rc) return rc;
  unsigned long long tot = 0;
  cudaError_t e = cudaMemcpy(&tot, p->spike_total, 8, cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) {
    err = cudaGetErrorString(e);
    return FS_ERR_CUDA;
  }
  if (spikes_total) *spikes_total = tot;
  return FS_OK;
}

void prod_kernel_time(Prod *p, double *ms_per_launch, uint64_t *launches) {
  if (ms_per_launch) *ms_per_launch = p->kl ? p->ms / (double)p->kl : 0.0;
  if (launches) *launches = p->kl;
}

int prod_get_state(Prod *p, float *V, int32_t *Count, uint32_t *NState, cudaStream_t st, std::string &err) {
  const size_t n = p->n;
  cudaError_t e = cudaStreamSynchronize(st);
  if (e == cudaSuccess && V) {
    if (p->fp64) {
      std::vector<double> tmp(n);
      e = cudaMemcpy(tmp.data(), p->P.V, n * 8, cudaMemcpyDeviceToHost);
      for (size_t i = 0; i < n; i++) V[i] = (float)tmp[i];
    } else {
      e = cudaMemcpy(V, p->P.V, n * 4, cudaMemcpyDeviceToHost);
    }
  }
  if (e == cudaSuccess && Count) e = cudaMemcpy(Count, p->P.Count, n * 4, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess && NState) e = cudaMemcpy(NState, p->P.NS, n * 4, cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) {
    err = cudaGetErrorString(e);
    return FS_ERR_CUDA;
  }
  return FS_OK;
}

void prod_info(const Prod *p, ProdInfo *info) {
  info->n = p->n;
  info->d_min = p->d_min;
  info->d_max = p->d_max;
  info->slots = p->P.slots;
  info->interval = p->P.interval;
  info->blocks = p->single ? p->b1_blocks : p->blocks;
  info->threads = p->single ? kT1 : kThreads;
  info->single_step = p->single ? 1 : 0;
  info->tiles = p->tiles ? 1 : 0;
  info->ltp = p->ltp ? 1 : 0;
  info->chunks = p->chunks;
  info->lin_edges = p->lin_edges;
  info->nmda_edges = p->nmda_edges;
  info->lin_receptors = p->nlin;
  info->fp64 = p->fp64 ? 1 : 0;
}


int prod_spike_counts(Prod *p, uint32_t *counts, cudaStream_t st, std::string &err) {
  cudaError_t e = cudaStreamSynchronize(st);
  if (e == cudaSuccess) e = cudaMemcpy(counts, p->P.nspk, (size_t)p->n * 4, cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) {
    err = cudaGetErrorString(e);
    return FS_ERR_CUDA;
  }
  return FS_OK;
}

// ---- tile runner (batches; single networks too large for one launch) ---------
// Device tile plan and parameter array over one or more production
// networks, and the CUDA graph of a chunk of steps.
struct Tiles {
  bool fp64 = false;
  uint32_t count = 0;
  Params *dP = nullptr;        // [count] parameters as the kernels read them
  IvTile *dT = nullptr;        // [ntiles]
  uint32_t ntiles = 0, dT_cap = 0;
  uint32_t tile_w = kTile;     // posts per tile
  int U = 8;                   // NMDA edges in flight per lane in the pull
  uint32_t Lmax = 1;           // steps per launch pair
  uint32_t dev_nsteps = 0;     // nsteps the device parameters hold (0: stale)
  cudaGraphExec_t exec = nullptr;
  uint32_t graph_steps = 0;
  bool graph_ok = true, graph_used = false;
};

namespace {

template <class X>
cudaError_t bal(X **p, size_t count) {
  return cudaMalloc((void **)p, count * sizeof(X));
}

void tiles_free(Tiles &T) {
  if (T.exec) cudaGraphExecDestroy(T.exec);
  if (T.dP) cudaFree(T.dP);
  if (T.dT) cudaFree(T.dT);
  T = Tiles();
}

// Tiles of tile_w posts, network by network (a network's tiles run
// together and share its s history in L2).
int tiles_plan(Tiles &T, const std::vector<Prod *> &inst, uint32_t tile_w, int U, std::string &err) {
  const uint32_t W = T.fp64 ? TileW<double>::W : TileW<float>::W;
  tile_w = std::max<uint32_t>(32, std::min(tile_w, W));
  std::vector<IvTile> plan;
  uint32_t L = kLB;
  for (uint32_t i = 0; i < inst.size(); i++) {
    for (uint32_t p0 = 0; p0 < inst[i]->n; p0 += tile_w)
      plan.push_back(IvTile{i, p0, std::min(tile_w, inst[i]->n - p0), 0});
    L = std::min(L, inst[i]->P.interval);
  }
  if (plan.size() > T.dT_cap) {
    if (T.dT) cudaFree(T.dT);
    T.dT = nullptr;
    T.dT_cap = 0;
    cudaError_t e = bal(&T.dT, plan.size());
    if (e != cudaSuccess) {
      err = std::string("cudaMalloc: ") + cudaGetErrorString(e);
      return FS_ERR_NOMEM;
    }
    T.dT_cap = (uint32_t)plan.size();
  }
  cudaError_t e = cudaMemcpy(T.dT, plan.data(), plan.size() * sizeof(IvTile), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    err = std::string("tile plan upload: ") + cudaGetErrorString(e);
    return FS_ERR_CUDA;
  }
  T.ntiles = (uint32_t)plan.size();
  T.tile_w = tile_w;
  T.U = U;
  T.Lmax = std::max<uint32_t>(1, L);
  if (T.exec) cudaGraphExecDestroy(T.exec);
  T.exec = nullptr;
  T.graph_steps = 0;
  return FS_OK;
}

int tiles_upload(Tiles &T, const Params *hp, uint32_t count, uint32_t nsteps, cudaStream_t st, std::string &err) {
  if (!T.dP || count != T.count) {
    if (T.dP) cudaFree(T.dP);
    T.dP = nullptr;
    cudaError_t e = bal(&T.dP, count);
    if (e != cudaSuccess) {
      err = std::string("cudaMalloc: ") + cudaGetErrorString(e);
      return FS_ERR_NOMEM;
    }
    T.count = count;
  }
  cudaError_t e = cudaMemcpyAsync(T.dP, hp, count * sizeof(Params), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    err = std::string("parameter upload: ") + cudaGetErrorString(e);
    return FS_ERR_CUDA;
  }
  T.dev_nsteps = nsteps;
  return FS_OK;
}

// Advances every instance's step counter after a chunk (graph node).
__global__ void k_tiles_advance(Params *Ps, uint32_t count, uint32_t nsteps) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < count) Ps[i].t0 += nsteps;
}

cudaError_t tiles_enqueue(const Tiles &T, uint32_t nsteps, cudaStream_t st) {
  for (uint32_t bs = 0; bs < nsteps; bs += T.Lmax) {
    const uint32_t L = std::min(T.Lmax, nsteps - bs);
    if (T.fp64) {
      k_tile_pull<double, 4><<<T.ntiles, kThreads, 0, st>>>(T.dP, T.dT, bs, L);
      k_tile_step<double, 1><<<T.ntiles, kThreads, 0, st>>>(T.dP, T.dT, bs, L);
    } else {
      if (T.U == 4) k_tile_pull<float, 4><<<T.ntiles, kThreads, 0, st>>>(T.dP, T.dT, bs, L);
      else k_tile_pull<float, 8><<<T.ntiles, kThreads, 0, st>>>(T.dP, T.dT, bs, L);
      k_tile_step<float, 2><<<T.ntiles, kThreads, 0, st>>>(T.dP, T.dT, bs, L);
    }
  }
  k_tiles_advance<<<(T.count + 255) / 256, 256, 0, st>>>(T.dP, T.count, nsteps);
  return cudaGetLastError();
}

// kernels of one chunk
uint64_t tiles_kernels(const Tiles &T, uint32_t nsteps) { return 2ull * ((nsteps + T.Lmax - 1) / T.Lmax) + 1; }

// One chunk of nsteps: a replay of the captured graph when one exists for
// this step count, else a direct launch.
int tiles_launch(Tiles &T, uint32_t nsteps, cudaStream_t st, std::string &err) {
  cudaError_t e = cudaSuccess;
  if (T.graph_ok && T.graph_steps != nsteps) {
    if (T.exec) cudaGraphExecDestroy(T.exec);
    T.exec = nullptr;
    T.graph_steps = 0;
    cudaGraph_t g = nullptr;
    e = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
      cudaError_t le = tiles_enqueue(T, nsteps, st);
      e = cudaStreamEndCapture(st, &g);
      if (le != cudaSuccess) e = le;
    }
    if (e == cudaSuccess) e = cudaGraphInstantiate(&T.exec, g, 0);
    if (g) cudaGraphDestroy(g);
    if (e == cudaSuccess) {
      T.graph_steps = nsteps;
    } else {
      cudaGetLastError();
      T.graph_ok = false;
      if (T.exec) cudaGraphExecDestroy(T.exec);
      T.exec = nullptr;
    }
  }
  if (T.exec && T.graph_steps == nsteps) {
    e = cudaGraphLaunch(T.exec, st);
    T.graph_used = true;
  } else {
    e = tiles_enqueue(T, nsteps, st);
  }
  if (e != cudaSuccess) {
    err = std::string("tile launch: ") + cudaGetErrorString(e);
    return FS_ERR_CUDA;
  }
  return FS_OK;
}

}  // namespace

// ---- batch of independent networks ------------------------------------------
struct Batch {
  bool fp64 = false;
  uint32_t sm = 148;
  std::vector<Prod *> inst;
  std::vector<uint32_t> seeds;
  Tiles T;
  uint32_t chunk = 10000;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  double ms = 0.0;
  uint64_t launches = 0;
};

namespace {

int batch_upload(Batch *B, uint32_t nsteps, cudaStream_t st, std::string &err) {
  const uint32_t count = (uint32_t)B->inst.size();
  std::vector<Params> hp(count);
  for (uint32_t i = 0; i < count; i++) {
    Params P = B->inst[i]->P;
    P.t0 = B->inst[i]->t;
    P.nsteps = nsteps;
    P.bits = nullptr;
    P.counts = nullptr;
    P.outV = nullptr;
    P.outI = nullptr;
    P.outNS = nullptr;
    P.gv_row = P.gv_ent = nullptr;
    P.gv_st = P.gv_xt = nullptr;
    P.spike_total = B->inst[i]->spike_total;
    hp[i] = P;
  }
  return tiles_upload(B->T, hp.data(), count, nsteps, st, err);
}

int batch_launch(Batch *B, uint32_t nsteps, cudaStream_t st, std::string &err) {
  int rc;
  if (B->T.dev_nsteps != nsteps && (rc = batch_upload(B, nsteps, st, err))) return rc;
  if ((rc = tiles_launch(B->T, nsteps, st, err))) return rc;
  for (Prod *p : B->inst) p->t += nsteps;
  B->launches += tiles_kernels(B->T, nsteps);
  return FS_OK;
}

int batch_check(Batch *B, cudaStream_t st, std::string &err) {
  cudaError_t e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    err = std::string("batch kernel: ") + cudaGetErrorString(e);
    return FS_ERR_CUDA;
  }
  return FS_OK;
}

}  // namespace

void batch_destroy(Batch *B) {
  if (!B) return;
  for (Prod *p : B->inst) prod_destroy(p);
  tiles_free(B->T);
  if (B->e0) cudaEventDestroy(B->e0);
  if (B->e1) cudaEventDestroy(B->e1);
  delete B;
}

int batch_create(Batch **out, uint32_t count, const fs_net_desc *const *descs, const fs_run_opts &o,
                 uint32_t sm_count, cudaStream_t st, std::string &err) {
  *out = nullptr;
  if (!count || !descs) {
    err = "batch: no instances";
    return FS_ERR_ARG;
  }
  Batch *B = new Batch();
  B->fp64 = (o.mode == FS_MODE_FP64);
  B->T.fp64 = B->fp64;
  B->sm = sm_count;
  B->chunk = o.chunk_steps ? o.chunk_steps : 10000;
  int rc = FS_OK;
  for (uint32_t i = 0; i < count && rc == FS_OK; i++)
    if (!descs[i]) {
      err = "batch: null network description " + std::to_string(i);
      rc = FS_ERR_ARG;
    }
  // the host tables of a wave of instances are built on all host threads,
  // then the instances are uploaded one by one
  const uint32_t wave = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
  for (uint32_t i0 = 0; i0 < count && rc == FS_OK; i0 += wave) {
    const uint32_t k = std::min(wave, count - i0);
    std::vector<HostNet> hn(k);
    std::vector<int> hrc(k, FS_OK);
    std::vector<std::string> herr(k);
    std::vector<std::thread> th;
    for (uint32_t j = 0; j < k; j++)
      th.emplace_back([&, j]() { hrc[j] = host_net(descs[i0 + j], hn[j], herr[j]); });
    for (auto &x : th) x.join();
    for (uint32_t j = 0; j < k && rc == FS_OK; j++) {
      const uint32_t i = i0 + j;
      Prod *p = nullptr;
      if (hrc[j]) {
        rc = hrc[j];
        err = "instance " + std::to_string(i) + ": " + herr[j];
        break;
      }
      rc = prod_create_from(&p, descs[i], o, sm_count, st, err, false, &hn[j]);
      if (rc) err = "instance " + std::to_string(i) + ": " + err;
      else {
        B->inst.push_back(p);
        rc = prod_tile_buffers(p, st, err);
      }
    }
  }
  if (rc == FS_OK) {
    cudaError_t e = cudaEventCreate(&B->e0);
    if (e == cudaSuccess) e = cudaEventCreate(&B->e1);
    if (e != cudaSuccess) {
      err = std::string("batch events: ") + cudaGetErrorString(e);
      rc = FS_ERR_CUDA;
    }
  }
  if (rc == FS_OK) rc = tiles_plan(B->T, B->inst, B->fp64 ? TileW<double>::W : kTile, 4, err);
  if (rc) {
    batch_destroy(B);
    return rc;
  }
  B->seeds.assign(count, 1);
  *out = B;
  return FS_OK;
}

int batch_reset(Batch *B, const uint32_t *seeds, cudaStream_t st, std::string &err) {
  for (size_t i = 0; i < B->inst.size(); i++) {
    const uint32_t s = seeds ? seeds[i] : B->seeds[i];
    B->seeds[i] = s;
    int rc = prod_reset(B->inst[i], s, st, err);
    if (rc) {
      err = "instance " + std::to_string(i) + ": " + err;
      return rc;
    }
  }
  B->T.dev_nsteps = 0;
  B->ms = 0.0;
  return FS_OK;
}

int batch_run(Batch *B, uint32_t nsteps, cudaStream_t st, double *device_ms, std::string &err) {
  cudaEventRecord(B->e0, st);
  uint32_t done = 0;
  while (done < nsteps) {
    const uint32_t k = std::min(B->chunk, nsteps - done);
    int rc = batch_launch(B, k, st, err);
    if (rc) return rc;
    done += k;
  }
  cudaEventRecord(B->e1, st);
  int rc = batch_check(B, st, err);
  if (rc) return rc;
  float ms = 0;
  cudaEventElapsedTime(&ms, B->e0, B->e1);
  B->ms += ms;
  if (device_ms) *device_ms = ms;
  return FS_OK;
}

// Autotuner: times a sample of the batch for each tile width (posts per
// block) and number of NMDA edges in flight per lane, keeps the fastest and
// resets every instance (its seed unchanged).  Results never depend on the
// choice.
int batch_tune(Batch *B, uint32_t sample_steps, cudaStream_t st, BatchPlan *out, std::string &err) {
  if (!sample_steps) sample_steps = 200;
  double best = -1.0;
  uint32_t best_w = B->T.tile_w;
  int best_u = B->T.U;
  uint32_t tried = 0;
  const uint32_t widths[3] = {64, 128, 256};
  const int us[2] = {4, 8};
  for (uint32_t w : widths) {
    if (B->fp64 && w > TileW<double>::W) continue;
    for (int u : us) {
      if (B->fp64 && u != 4) continue;  // the FP64 pull has no edges-in-flight parameter
      int rc = tiles_plan(B->T, B->inst, w, u, err);
      if (rc) return rc;
      if ((rc = batch_reset(B, nullptr, st, err))) return rc;
      double ms = 0;
      if ((rc = batch_run(B, sample_steps, st, nullptr, err))) return rc;  // warm-up (graph capture)
      if ((rc = batch_run(B, sample_steps, st, &ms, err))) return rc;
      tried++;
      if (best < 0 || ms < best) {
        best = ms;
        best_w = w;
        best_u = u;
      }
    }
  }
  int rc = tiles_plan(B->T, B->inst, best_w, best_u, err);
  if (rc == FS_OK) rc = batch_reset(B, nullptr, st, err);
  if (rc) return rc;
  B->ms = 0.0;
  if (out) {
    batch_info(B, out);
    out->sample_ms = best;
    out->candidates = tried;
  }
  return FS_OK;
}

void batch_info(const Batch *B, BatchPlan *out) {
  int occ = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(
      &occ, B->fp64 ? (const void *)k_tile_step<double, 1> : (const void *)k_tile_step<float, 2>, kThreads, 0);
  out->blocks = B->T.ntiles;
  out->blocks_per_sm = (uint32_t)std::max(0, occ);
  out->tile_posts = B->T.tile_w;
  out->edges_in_flight = (uint32_t)B->T.U;
  out->sample_ms = 0.0;
  out->candidates = 0;
  out->graph = B->T.graph_used ? 1 : 0;
  out->launches = B->launches;
  out->total_ms = B->ms;
}

int batch_spike_counts(Batch *B, uint32_t i, uint32_t *counts, cudaStream_t st, std::string &err) {
  if (i >= B->inst.size()) {
    err = "batch: instance index out of range";
    return FS_ERR_ARG;
  }
  return prod_spike_counts(B->inst[i], counts, st, err);
}

int batch_spike_totals(Batch *B, uint64_t *totals, cudaStream_t st, std::string &err) {
  cudaError_t e = cudaStreamSynchronize(st);
  for (size_t i = 0; i < B->inst.size() && e == cudaSuccess; i++) {
    unsigned long long t = 0;
    e = cudaMemcpy(&t, B->inst[i]->spike_total, 8, cudaMemcpyDeviceToHost);
    totals[i] = t;
  }
  if (e != cudaSuccess) {
    err = cudaGetErrorString(e);
    return FS_ERR_CUDA;
  }
  return FS_OK;
}

uint32_t batch_size(const Batch *B) { return (uint32_t)B->inst.size(); }

int prod_tile_buffers(Prod *p, cudaStream_t st, std::string &err) {
  (void)st;
  if (p->P.gn_buf) return FS_OK;
  return dal(p, (uint8_t **)&p->P.gn_buf, (size_t)kLB * p->n * (p->fp64 ? 8 : 4), err);
}

int tiles_solo_create(Prod *p, std::string &err) {
  int rc = prod_tile_buffers(p, nullptr, err);
  if (rc) return rc;
  p->tiles = new Tiles();
  p->tiles->fp64 = p->fp64;
  std::vector<Prod *> one{p};
  return tiles_plan(*p->tiles, one, p->fp64 ? TileW<double>::W : kTile, 4, err);
}

void tiles_delete(Tiles *T) {
  if (!T) return;
  tiles_free(*T);
  delete T;
}

int tiles_solo_launch(Prod *p, const Params &P, uint32_t nsteps, cudaStream_t st, uint64_t *kernels,
                      std::string &err) {
  int rc = tiles_upload(*p->tiles, &P, 1, nsteps, st, err);
  if (rc) return rc;
  if ((rc = tiles_launch(*p->tiles, nsteps, st, err))) return rc;
  if (kernels) *kernels = tiles_kernels(*p->tiles, nsteps);
  return FS_OK;
}

// ---- failure detection check ---------------------------------------------
// One block waits at a barrier of two blocks that the second never reaches:
// the bounded wait gives up after `limit` polls, sets the error word and
// returns, and the context stays usable.
__global__ void k_barrier_probe(unsigned int *bar, int *err, unsigned int limit) {
  unsigned long long target = 0;
  grid_sync(bar, err, 2, target, limit);
}

int prod_barrier_probe(unsigned int limit, int *err_word, std::string &err) {
  unsigned int *bar = nullptr;
  int *ew = nullptr;
  cudaError_t e = cudaMalloc(&bar, 64 * 4);
  if (e == cudaSuccess) e = cudaMalloc(&ew, 4);
  if (e == cudaSuccess) e = cudaMemset(bar, 0, 64 * 4);
  if (e == cudaSuccess) e = cudaMemset(ew, 0, 4);
  if (e == cudaSuccess) {
    k_barrier_probe<<<1, 32>>>(bar, ew, limit);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (e == cudaSuccess) e = cudaMemcpy(err_word, ew, 4, cudaMemcpyDeviceToHost);
  if (bar) cudaFree(bar);
  if (ew) cudaFree(ew);
  if (e != cudaSuccess) {
    err = std::string("barrier probe: ") + cudaGetErrorString(e);
    return FS_ERR_CUDA;
  }
  return FS_OK;
}

// ---- checks of the drive draws --------------------------------------------
// The device Philox on k arbitrary (counter, key) pairs, and the drive draws
// of a step and neuron range through draw_inputs itself (the function the
// engine's kernels call), so the CPU restatement can be compared with both.
__global__ void k_debug_philox(const uint32_t *ctr, const uint32_t *key, uint64_t k, uint32_t *out) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= k) return;
  uint32_t c[4] = {ctr[4 * i], ctr[4 * i + 1], ctr[4 * i + 2], ctr[4 * i + 3]};
  philox(c, key[2 * i], key[2 * i + 1]);
  for (int w = 0; w < 4; w++) out[4 * i + w] = c[w];
}

template <class T>
__global__ void __launch_bounds__(kThreads) k_debug_drive(const __grid_constant__ Params P, uint32_t first,
                                                          uint32_t count, uint64_t t0, uint32_t nsteps,
                                                          uint8_t *hits_out, double *gauss_out) {
  constexpr uint32_t kT = TileW<T>::W;
  __shared__ T gauss[kLB][kT];
  __shared__ uint8_t hits[kLB][kT];
  const uint32_t q0 = blockIdx.x * kT;
  if (q0 >= count) return;
  const uint32_t np = min(kT, count - q0), p0 = first + q0;
  for (uint32_t j0 = 0; j0 < nsteps; j0 += kLB) {
    const uint32_t L = min(kLB, nsteps - j0);
    draw_inputs<T>(P, p0, np, t0 + j0, L, hits, gauss);
    __syncthreads();
    for (uint32_t idx = threadIdx.x; idx < np * L; idx += kThreads) {
      const uint32_t j = idx / np, q = idx - j * np;
      const size_t o = (size_t)(j0 + j) * count + q0 + q;
      hits_out[o] = hits[j][q];
      gauss_out[o] = (__ldg(P.act + p0 + q) & FS_ACT_INJ) ? (double)gauss[j][q] : 0.0;
    }
    __syncthreads();
  }
}

int prod_debug_philox(const uint32_t *ctr, const uint32_t *key, uint64_t k, uint32_t *out, std::string &err) {
  uint32_t *dc = nullptr, *dk = nullptr, *dout = nullptr;
  cudaError_t e = cudaMalloc(&dc, k * 16);
  if (e == cudaSuccess) e = cudaMalloc(&dk, k * 8);
  if (e == cudaSuccess) e = cudaMalloc(&dout, k * 16);
  if (e == cudaSuccess) e = cudaMemcpy(dc, ctr, k * 16, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(dk, key, k * 8, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    k_debug_philox<<<(unsigned)((k + 255) / 256), 256>>>(dc, dk, k, dout);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpy(out, dout, k * 16, cudaMemcpyDeviceToHost);
  if (dc) cudaFree(dc);
  if (dk) cudaFree(dk);
  if (dout) cudaFree(dout);
  if (e != cudaSuccess) {
    err = std::string("philox check: ") + cudaGetErrorString(e);
    return FS_ERR_CUDA;
  }
  return FS_OK;
}

int prod_debug_drive(Prod *p, uint64_t t0, uint32_t nsteps, uint32_t first, uint32_t count, uint8_t *hits,
                     double *gauss, cudaStream_t st, std::string &err) {
  const size_t m = (size_t)nsteps * count;
  uint8_t *dh = nullptr;
  double *dg = nullptr;
  cudaError_t e = cudaStreamSynchronize(st);
  if (e == cudaSuccess) e = cudaMalloc(&dh, m);
  if (e == cudaSuccess) e = cudaMalloc(&dg, m * 8);
  if (e == cudaSuccess) {
    const uint32_t W = p->fp64 ? TileW<double>::W : TileW<float>::W;
    const unsigned blocks = (count + W - 1) / W;
    if (p->fp64) k_debug_drive<double><<<blocks, kThreads, 0, st>>>(p->P, first, count, t0, nsteps, dh, dg);
    else k_debug_drive<float><<<blocks, kThreads, 0, st>>>(p->P, first, count, t0, nsteps, dh, dg);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(hits, dh, m, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(gauss, dg, m * 8, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (dh) cudaFree(dh);
  if (dg) cudaFree(dg);
  if (e != cudaSuccess) {
    err = std::string("drive check: ") + cudaGetErrorString(e);
    return FS_ERR_CUDA;
  }
  return FS_OK;
}

// Phase clock: per block, SM cycles spent in each phase of the persistent
// kernels since it was switched on (k_prod1: 0 spike-list lookups, 1 NMDA
// copies of listed spikes, 2 last deliveries and NMDA sums, 3 neuron steps
// and spike lists, 6 thread 0's barrier wait, 4 the rest of the barrier,
// 5 set-up; k_prod: 0 NMDA pull, 1 drive draws, 2 neuron steps, 3 pushes,
// 4 grid barrier).
int prod_phase_clock(Prod *p, int enable, cudaStream_t st, std::string &err) {
  const uint32_t nb = std::max(p->blocks, p->b1_blocks);
  if (!enable) {
    p->P.phase = nullptr;
    return FS_OK;
  }
  if (!p->phase_buf) {
    int rc = dal(p, &p->phase_buf, (size_t)nb * kPhaseSlots, err);
    if (rc) return rc;
  }
  cudaError_t e = cudaMemsetAsync(p->phase_buf, 0, (size_t)nb * kPhaseSlots * 8, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    err = std::string("phase clock: ") + cudaGetErrorString(e);
    return FS_ERR_CUDA;
  }
  p->P.phase = p->phase_buf;
  return FS_OK;
}

int prod_phase_times(Prod *p, uint64_t *out, uint32_t cap, uint32_t *blocks, cudaStream_t st, std::string &err) {
  const uint32_t nb = p->single ? p->b1_blocks : p->blocks;
  if (blocks) *blocks = nb;
  if (!p->phase_buf) {
    err = "phase clock was never switched on";
    return FS_ERR_ARG;
  }
  const size_t k = std::min<size_t>(cap, (size_t)nb * kPhaseSlots);
  cudaError_t e = cudaStreamSynchronize(st);
  if (e == cudaSuccess && k) e = cudaMemcpy(out, p->phase_buf, k * 8, cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) {
    err = std::string("phase clock: ") + cudaGetErrorString(e);
    return FS_ERR_CUDA;
  }
  return FS_OK;
}

int prod_inject_wait_failure(Prod *p, cudaStream_t st, std::string &err) {
  const int word = 2;  // the value a barrier wait that gave up stores
  cudaError_t e = cudaMemcpyAsync(p->err, &word, 4, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    err = std::string("error word: ") + cudaGetErrorString(e);
    return FS_ERR_CUDA;
  }
  return FS_OK;
}

// ---- checkpoints --------------------------------------------------------
// The state a production engine carries from one step to the next, in the
// order it is saved: neuron and receptor state, presynaptic gates and NMDA
// kinetics, the s history, spike counters, plasticity state and the delay
// ring (pushes already made for future steps), then the spike total.
namespace {
struct StateHead {
  uint64_t t;
  uint32_t key0, key1;
  float rg[5];
  uint32_t pad;
};
void state_regions(Prod *p, std::vector<std::pair<void *, size_t>> &r) {
  const size_t n = p->n, T = p->fp64 ? 8 : 4;
  Params &P = p->P;
  r.clear();
  r.push_back({P.V, n * T});
  r.push_back({P.G, 4 * n * T});
  r.push_back({P.ext_st, 4 * n * T});
  r.push_back({P.ext_x, n * T});
  r.push_back({P.ext_s, n * T});
  r.push_back({P.st_pre, 4 * n * T});
  r.push_back({P.x_pre, n * T});
  r.push_back({P.s_pre, n * T});
  r.push_back({P.s_hist, (size_t)P.slots * n * T * (p->fp64 ? 1 : kSH)});
  r.push_back({P.Count, n * 4});
  r.push_back({P.NS, n * 4});
  r.push_back({P.D, n * 4});
  r.push_back({P.F, n * 4});
  r.push_back({P.Cap, n * 4});
  r.push_back({P.Car, n * 4});
  r.push_back({P.tm_u, n * 4});
  r.push_back({P.tm_x, n * 4});
  r.push_back({P.nspk, n * 4});
  r.push_back({P.Irep, (size_t)5 * n * 4});
  r.push_back({P.ring, (size_t)std::max<uint32_t>(1, p->nlin) * P.slots * n * 8});
  if (P.Vg) r.push_back({P.Vg, 2 * n * T});
  if (p->ltp) {  // the weights LTP rewrites, and the traces
    r.push_back({(void *)P.out_w, p->lin_edges * 4});
    r.push_back({(void *)P.in_w, p->nmda_edges * 4});
    r.push_back({P.ltp_lp, n * 4});
    r.push_back({P.ltp_clp, n * 4});
    r.push_back({P.ltp_gn, n * T});  // the next step's NMDA sums
  }
  r.push_back({p->spike_total, 8});
}
}  // namespace

uint64_t prod_state_bytes(Prod *p) {
  std::vector<std::pair<void *, size_t>> r;
  state_regions(p, r);
  uint64_t b = sizeof(StateHead);
  for (auto &x : r) b += x.second;
  return b;
}

int prod_state_save(Prod *p, uint8_t *buf, cudaStream_t st, std::string &err) {
  cudaError_t e = cudaStreamSynchronize(st);
  StateHead h{};
  h.t = p->t;
  h.key0 = p->P.key0;
  h.key1 = p->P.key1;
  std::memcpy(h.rg, p->P.rg, sizeof h.rg);
  std::memcpy(buf, &h, sizeof h);
  std::vector<std::pair<void *, size_t>> r;
  state_regions(p, r);
  size_t off = sizeof h;
  for (auto &x : r) {
    if (e == cudaSuccess) e = cudaMemcpyAsync(buf + off, x.first, x.second, cudaMemcpyDeviceToHost, st);
    off += x.second;
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    err = std::string("checkpoint save: ") + cudaGetErrorString(e);
    return FS_ERR_CUDA;
  }
  return FS_OK;
}

int prod_state_load(Prod *p, const uint8_t *buf, cudaStream_t st, std::string &err) {
  cudaError_t e = cudaStreamSynchronize(st);
  StateHead h;
  std::memcpy(&h, buf, sizeof h);
  std::vector<std::pair<void *, size_t>> r;
  state_regions(p, r);
  size_t off = sizeof h;
  for (auto &x : r) {
    if (e == cudaSuccess) e = cudaMemcpyAsync(x.first, buf + off, x.second, cudaMemcpyHostToDevice, st);
    off += x.second;
  }
  if (e == cudaSuccess) e = cudaMemsetAsync(p->err, 0, 4, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    err = std::string("checkpoint load: ") + cudaGetErrorString(e);
    return FS_ERR_CUDA;
  }
  p->t = h.t;
  p->P.key0 = h.key0;
  p->P.key1 = h.key1;
  std::memcpy(p->P.rg, h.rg, sizeof h.rg);
  p->ms = 0.0;
  p->kl = 0;
  p->ev_used = 0;
  return FS_OK;
}

int prod_get_weights(Prod *p, float *g, uint64_t n, cudaStream_t st, std::string &err) {
  if (!p->ltp) {
    err = "fs_get_weights: the network has no LTP (its weights are the description's)";
    return FS_ERR_UNSUPPORTED;
  }
  if (n != p->wpos.size()) {
    err = "fs_get_weights: n must be the synapse list's length (" + std::to_string(p->wpos.size()) + ")";
    return FS_ERR_ARG;
  }
  std::vector<float> ow(p->lin_edges), iw(p->nmda_edges);
  cudaError_t e = cudaStreamSynchronize(st);
  if (e == cudaSuccess && !ow.empty()) e = cudaMemcpy(ow.data(), p->P.out_w, ow.size() * 4, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess && !iw.empty()) e = cudaMemcpy(iw.data(), p->P.in_w, iw.size() * 4, cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) {
    err = std::string("fs_get_weights: ") + cudaGetErrorString(e);
    return FS_ERR_CUDA;
  }
  for (uint64_t i = 0; i < n; i++) {
    const uint32_t w = p->wpos[i];
    g[i] = (w & 0x80000000u) ? iw[w & 0x7fffffffu] : ow[w];
  }
  return FS_OK;
}

void prod_set_gains(Prod *p, const float *g) {
  for (int r = 0; r < 5; r++) p->P.rg[r] = g[r];
}

int prod_set_pb(Prod *p, const float *pb, cudaStream_t st, std::string &err) {
  cudaError_t e = cudaMemcpyAsync((void *)p->P.pb, pb, (size_t)FS_NREC * p->n * 4, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    err = std::string("drive upload: ") + cudaGetErrorString(e);
    return FS_ERR_CUDA;
  }
  return FS_OK;
}

int batch_set_gains(Batch *B, uint32_t i, const float *g, std::string &err) {
  if (i >= B->inst.size()) {
    err = "batch: instance index out of range";
    return FS_ERR_ARG;
  }
  prod_set_gains(B->inst[i], g);
  B->T.dev_nsteps = 0;  // the device copy of the parameters is stale
  return FS_OK;
}

int batch_set_drive(Batch *B, uint32_t i, const float *pb, cudaStream_t st, std::string &err) {
  if (i >= B->inst.size()) {
    err = "batch: instance index out of range";
    return FS_ERR_ARG;
  }
  return prod_set_pb(B->inst[i], pb, st, err);
}
uint32_t batch_neurons(const Batch *B, uint32_t i) { return i < B->inst.size() ? B->inst[i]->n : 0; }

}  // namespace fsp
