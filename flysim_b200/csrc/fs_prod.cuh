// Production engine (FS_MODE_FP32 / FS_MODE_FP64): interface used by the C ABI.
#pragma once
#include <cstdint>
#include <string>
#include <cuda_runtime.h>
#include "flysim_b200.h"

namespace fsp {

struct Prod;

// allow_single: a network that qualifies may run on the single-step kernel
// (batch instances never do: the batch kernel advances them)
int prod_create(Prod **out, const fs_net_desc *d, const fs_run_opts &o, uint32_t sm_count,
                cudaStream_t st, std::string &err, bool allow_single = true);
// NMDA-sum buffer of the tile kernels (allocated once per network)
int prod_tile_buffers(Prod *p, cudaStream_t st, std::string &err);
void prod_destroy(Prod *p);
int prod_upload_params(Prod *p, const float *pb, const uint32_t *act, const float *inj_mean,
                       const float *inj_std, cudaStream_t st, std::string &err);
int prod_reset(Prod *p, uint32_t seed, cudaStream_t st, std::string &err);
int prod_step(Prod *p, uint32_t nsteps, fs_step_out *out, uint64_t *written, cudaStream_t st,
              uint64_t *launches, uint64_t *spikes_total, std::string &err);
int prod_run(Prod *p, uint32_t nsteps, cudaStream_t st, uint64_t *launches, std::string &err);
int prod_check(Prod *p, cudaStream_t st, uint64_t *spikes_total, std::string &err);
void prod_kernel_time(Prod *p, double *ms_per_launch, uint64_t *launches);
int prod_get_state(Prod *p, float *V, int32_t *Count, uint32_t *NState, cudaStream_t st, std::string &err);
// Current weights in synapse-list order (networks with LTP: n = list size).
int prod_get_weights(Prod *p, float *g, uint64_t n, cudaStream_t st, std::string &err);

// Builds the single-step plan of a network on the host (no device needed)
// and checks every index the kernel derives from it; stats[0] = 1 when the
// network qualifies, then blocks, max posts, max tracked neurons, max NMDA
// edges per block, shared-memory bytes, linear entries, NMDA edges.
int prod_check_single_plan(const fs_net_desc *d, uint32_t sm_count, uint64_t *stats, std::string &err);
// Layout facts for measurement (algorithmic bytes).
struct ProdInfo {
  uint32_t n, d_min, d_max, slots, interval, blocks, threads, chunks;
  uint64_t lin_edges, nmda_edges;
  uint32_t lin_receptors;
  int fp64;
  int single_step;  // the network runs on the single-step kernel
  int tiles;        // the network runs on the tile kernels
  int ltp;          // the network runs on the LTP kernel (long-term plasticity)
};
void prod_info(const Prod *p, ProdInfo *info);
int prod_spike_counts(Prod *p, uint32_t *counts, cudaStream_t st, std::string &err);
// Runs the bounded barrier wait to its limit (see k_barrier_probe).
int prod_barrier_probe(unsigned int limit, int *err_word, std::string &err);
// Checks of the drive draws: the device Philox on k (counter[4], key[2])
// pairs, and the draws of steps [t0, t0 + nsteps) for neurons [first,
// first + count) with the handle's key and parameters (hits [nsteps][count]
// bit r = receptor r hit, gauss the injection current, 0 where it is off).
int prod_debug_philox(const uint32_t *ctr, const uint32_t *key, uint64_t k, uint32_t *out, std::string &err);
int prod_debug_drive(Prod *p, uint64_t t0, uint32_t nsteps, uint32_t first, uint32_t count, uint8_t *hits,
                     double *gauss, cudaStream_t st, std::string &err);
// Phase clock of the persistent kernels (debug aid): per block, SM cycles
// per phase; out holds [blocks][8].
int prod_phase_clock(Prod *p, int enable, cudaStream_t st, std::string &err);
int prod_phase_times(Prod *p, uint64_t *out, uint32_t cap, uint32_t *blocks, cudaStream_t st, std::string &err);
// Stores into the device error word what a bounded wait that gave up stores.
int prod_inject_wait_failure(Prod *p, cudaStream_t st, std::string &err);
// Checkpoint blob of the engine's step-to-step state (step counter, drive
// stream key, gains, every state array and the delay ring).
uint64_t prod_state_bytes(Prod *p);
int prod_state_save(Prod *p, uint8_t *buf, cudaStream_t st, std::string &err);
int prod_state_load(Prod *p, const uint8_t *buf, cudaStream_t st, std::string &err);

// Batch: independent production networks advanced by one persistent launch.
struct Batch;
struct BatchPlan {
  uint32_t blocks, blocks_per_sm, candidates, tile_posts, edges_in_flight;
  double sample_ms;
  int graph;
  uint64_t launches;
  double total_ms;
};
int batch_create(Batch **out, uint32_t count, const fs_net_desc *const *descs, const fs_run_opts &o,
                 uint32_t sm_count, cudaStream_t st, std::string &err);
void batch_destroy(Batch *b);
int batch_reset(Batch *b, const uint32_t *seeds, cudaStream_t st, std::string &err);
int batch_run(Batch *b, uint32_t nsteps, cudaStream_t st, double *device_ms, std::string &err);
int batch_tune(Batch *b, uint32_t sample_steps, cudaStream_t st, BatchPlan *out, std::string &err);
void batch_info(const Batch *b, BatchPlan *out);
int batch_spike_counts(Batch *b, uint32_t inst, uint32_t *counts, cudaStream_t st, std::string &err);
int batch_spike_totals(Batch *b, uint64_t *totals, cudaStream_t st, std::string &err);
uint32_t batch_size(const Batch *b);
uint32_t batch_neurons(const Batch *b, uint32_t inst);
void prod_set_gains(Prod *p, const float *gains);
int prod_set_pb(Prod *p, const float *pb, cudaStream_t st, std::string &err);
int batch_set_gains(Batch *b, uint32_t inst, const float *gains, std::string &err);
int batch_set_drive(Batch *b, uint32_t inst, const float *pb, cudaStream_t st, std::string &err);

}  // namespace fsp
