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
#include <cmath>
#include <cstring>
#include <numeric>
#include <string>
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

// ---- bounded grid barrier ---------------------------------------------------
// Over the `count` blocks that share `bar` (the whole grid, or the blocks of
// one network instance in a batch).  bar[0] counts arrivals, bar[32] (its
// own 128-byte line) is the generation the waiting blocks poll; the last
// block to arrive resets the count and advances the generation.  Ordering
// (PTX memory model): after bar.sync, thread 0's acq_rel arrival releases
// the whole block's writes (release is cumulative) and, for the last block,
// acquires every earlier arrival's; the last block publishes the count reset
// and all writes with a release add on the generation, which the others
// observe with relaxed polls followed by one acquire fence; the closing
// bar.sync hands that on to the block.  Every wait is bounded: after ~2^24
// polls the block sets the error word and all blocks leave.
__device__ __forceinline__ unsigned int ld_relaxed_gpu(const unsigned int *p) {
  unsigned int v;
  asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ unsigned int atom_add_acq_rel_gpu(unsigned int *p, unsigned int v) {
  unsigned int old;
  asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
  return old;
}
__device__ __forceinline__ void red_release_gpu(unsigned int *p, unsigned int v) {
  asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ void fence_acquire_gpu() { asm volatile("fence.acq_rel.gpu;" ::: "memory"); }

__device__ __forceinline__ bool grid_sync(unsigned int *bar, int *err, uint32_t count,
                                          unsigned int limit = 1u << 24) {
  __syncthreads();
  if (count <= 1) return *(volatile int *)err == 0;
  if (threadIdx.x == 0) {
    unsigned int *gen = bar + 32;
    const unsigned int g = ld_relaxed_gpu(gen);
    const unsigned int arrived = atom_add_acq_rel_gpu(bar, 1u);
    if (arrived == count - 1) {
      atomicExch(bar, 0u);
      red_release_gpu(gen, 1u);
    } else {
      unsigned int spins = 0;
      while (ld_relaxed_gpu(gen) == g) {
        if (*(volatile int *)err) break;
        if (++spins > limit) {
          atomicExch(err, 2);
          break;
        }
      }
      fence_acquire_gpu();
    }
  }
  __syncthreads();
  return *(volatile int *)err == 0;
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

// Lanes work in quads: the four lanes of a quad take the same edge and each
// loads one of its window's 16-byte vectors (lane k: steps 4k..4k+3), so one
// warp load instruction covers eight edges whose vectors share a cache line
// per edge (about 1.25 L1 wavefronts per edge instead of 3 for a lane per
// edge); each lane keeps U edges in flight.  The next round's edge codes
// and weights are fetched while the current windows are in flight.  Quad g
// sums the post's edges g, g + 8, g + 16, ... in that order whatever U is
// (U only sets how many are in flight), then the eight quads are combined
// by a butterfly, so the sums depend on neither U nor the block plan.
template <int U>
__device__ __forceinline__ void nmda_pull_f32(const Params &P, uint32_t p0, uint32_t np, uint64_t tb, uint32_t L,
                                              float (*gn)[kTile], uint32_t wid, uint32_t lane) {
  constexpr uint32_t CH = 8u * U;      // edges per warp round
  const float4 *sh = (const float4 *)P.s_hist;
  const uint32_t S4 = P.slots >> 2, qmask = S4 - 1, mask = P.mask;
  const uint32_t nvl = (L + 3u) >> 2;  // vectors needed for L steps
  const uint32_t nw = kThreads / 32;
  const uint32_t k = lane & 3u, g = lane >> 2;
  const bool kv = k < nvl;
  uint32_t code[U];
  float w[U];
  auto fetch = [&](uint32_t base, uint32_t end) {
#pragma unroll
    for (int u = 0; u < U; u++) {
      const uint32_t eu = base + g + 8u * u;
      code[u] = eu < end ? __ldg(P.in_code + eu) : 0u;
      w[u] = eu < end ? __ldg(P.in_w + eu) : 0.0f;
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
        const bool ok = kv && e + 8u * u < b1;
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
#pragma unroll
    for (int o = 4; o < 32; o <<= 1)
#pragma unroll
      for (int i = 0; i < 4; i++) acc[i] += __shfl_xor_sync(fsd::kFull, acc[i], o);
    if (lane < 4) {
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

// Single-step batches (networks whose minimum delay is 0 or 1 step pull
// every step, and the last step of a call that ends one step into an
// interval): each edge needs one value, so a warp takes four posts at once
// with scalar loads, four times the edges in flight of the window path.
// Lane (g, k) of the warp (lane = 4g + k) sums post k's edges g, g + 8,
// g + 16, ... in order and the same xor 4, 8, 16 butterfly combines the
// eight g, which is exactly the quad path's order for step 0: a step's
// NMDA sum does not depend on the batch it falls in.
__device__ __forceinline__ void nmda_pull1_f32(const Params &P, uint32_t p0, uint32_t np, uint64_t tb,
                                               float (*gn)[kTile], uint32_t wid, uint32_t lane) {
  constexpr int PG = 4;             // posts per warp at once
  constexpr int U = 4;              // edges per lane per round
  constexpr uint32_t CH = 8u * U;   // edges of a post per round
  const float *sh = (const float *)P.s_hist;
  const uint32_t S = P.slots, mask = P.mask;
  const uint32_t nw = kThreads / 32;
  const uint32_t k = lane & 3u, g = lane >> 2;
  if (!P.in_row) {
    for (uint32_t q = wid * 32 + lane; q < np; q += nw * 32) gn[0][q] = 0.0f;
    return;
  }
  for (uint32_t q0 = wid * PG; q0 < np; q0 += nw * PG) {
    const uint32_t q = q0 + k;
    const bool qv = q < np;
    const uint32_t b0 = qv ? __ldg(P.in_row + p0 + q) : 0u, b1 = qv ? __ldg(P.in_row + p0 + q + 1) : 0u;
    uint32_t nch = (b1 - b0 + CH - 1) / CH;
#pragma unroll
    for (int o = 1; o < PG; o <<= 1) nch = max(nch, __shfl_xor_sync(fsd::kFull, nch, o));
    float acc = 0.0f;
    for (uint32_t c = 0; c < nch; c++) {
      uint32_t code[U];
      float w[U], v[U];
#pragma unroll
      for (int u = 0; u < U; u++) {
        const uint32_t e = b0 + c * CH + g + 8u * u;
        const bool ok = e < b1;
        code[u] = ok ? __ldg(P.in_code + e) : 0u;
        w[u] = ok ? __ldg(P.in_w + e) : 0.0f;
      }
#pragma unroll
      for (int u = 0; u < U; u++) {
        const uint32_t e = b0 + c * CH + g + 8u * u;
        const uint32_t pre = code[u] & 0xffffffu, d = code[u] >> 24;
        // row 0 of the shifted copies holds slot i at element i
        v[u] = e < b1 ? __ldca(sh + (size_t)pre * kSH * S + ((uint32_t)(tb - 1u - d) & mask)) : 0.0f;
      }
#pragma unroll
      for (int u = 0; u < U; u++) acc += w[u] * v[u];
    }
#pragma unroll
    for (int o = 4; o < 32; o <<= 1) acc += __shfl_xor_sync(fsd::kFull, acc, o);
    if (g == 0 && qv) gn[0][q] = acc;
  }
}

template <class T>
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
        const T w = (T)__ldg(P.in_w + e);
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
template <class T>
__device__ __forceinline__ void push_spike(const Params &P, uint32_t q, uint32_t tm, const T (&cj)[4],
                                           uint32_t start, uint32_t stride) {
  const uint32_t n = P.n, S = P.slots, mask = P.mask;
  const uint32_t ob = __ldg(P.out_row + q), oe = __ldg(P.out_row + q + 1);
  for (uint32_t e = ob + start; e < oe; e += 4 * stride) {
    uint32_t code[4];
    float w[4];
#pragma unroll
    for (int u = 0; u < 4; u++) {
      const uint32_t eu = e + u * stride;
      code[u] = eu < oe ? __ldg(P.out_code + eu) : 0u;
      w[u] = eu < oe ? __ldg(P.out_w + eu) : 0.0f;
    }
#pragma unroll
    for (int u = 0; u < 4; u++) {
      if (e + u * stride < oe) {
        const uint32_t post = code[u] & 0x3fffffu, r = (code[u] >> 22) & 3u, d = code[u] >> 24;
        const T cv = ((r == 0) ? cj[0] : (r == 1) ? cj[1] : (r == 2) ? cj[2] : cj[3]) * (T)P.rg[r];
        const long long fx = __double2ll_rn((double)((T)w[u] * cv) * kFix);
        const int ri = P.lin_of_rec[r];
        atomicAdd(P.ring + ((size_t)ri * n + post) * S + ((tm + d) & mask), (unsigned long long)fx);
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

// ---- drive draws of L steps for a tile -------------------------------------
// The external Bernoulli outcomes (bit r: receptor r hit this step) and the
// injection noise depend on no state, so they are drawn for the whole batch
// by all threads at once, off the neurons' per-step dependency chain.
template <class T>
__device__ __forceinline__ void draw_inputs(const Params &P, uint32_t p0, uint32_t np, uint64_t tb, uint32_t L,
                                            uint8_t (*hits)[TileW<T>::W], T (*gauss)[TileW<T>::W]) {
  const uint32_t n = P.n;
  for (uint32_t idx = threadIdx.x; idx < np * L; idx += kThreads) {
    const uint32_t j = idx / np, q = idx - j * np, p = p0 + q;
    const uint64_t t = tb + j;
    const uint32_t a = __ldg(P.act + p);
    uint32_t rnd[4] = {(uint32_t)t, (uint32_t)(t >> 32), p, 0u};
    philox(rnd, P.key0, P.key1);
    uint32_t h = 0;
#pragma unroll
    for (int r = 0; r < 4; r++)
      if (__ldg(P.pb + (size_t)r * n + p) > u24(rnd[r])) h |= 1u << r;
    // the second block serves the NMDA drive and the injection noise; a
    // drive probability that is not positive never draws a hit
    const float pbn = __ldg(P.pb + (size_t)FS_NMDA * n + p);
    if (((a & FS_ACT_NMDA) && pbn > 0.0f) || (a & FS_ACT_INJ)) {
      uint32_t r2[4] = {(uint32_t)t, (uint32_t)(t >> 32), p, 1u};
      philox(r2, P.key0, P.key1);
      if (pbn > u24(r2[0])) h |= 1u << FS_NMDA;
      if (a & FS_ACT_INJ) {  // Box-Muller normal
        const double u1 = ((double)(r2[1] >> 8) + 1.0) * 5.9604644775390625e-08;
        const double u2 = (double)(r2[2] >> 8) * 5.9604644775390625e-08;
        const double z = sqrt(-2.0 * log(u1)) * cospi(2.0 * u2);
        gauss[j][q] = (T)__ldg(P.inj_mean + p) + (T)__ldg(P.inj_std + p) * (T)z;
      }
    }
    hits[j][q] = (uint8_t)h;
  }
}

// ---- L steps of a tile's neurons (thread per neuron), with the pushes ----
// Per-neuron parameters and state stay in registers for the L steps; the
// ring slots of the next PD steps are in flight while the current step
// computes (they are final: every push into them happened before the
// interval began); a warp pushes the spikes of its own lanes, so a step
// needs no block barrier.
template <class T, int PD>
__device__ __forceinline__ void neuron_steps(const Params &P, uint32_t p0, uint32_t np, uint32_t sb, uint32_t L,
                                             T (*gn)[TileW<T>::W], const uint8_t (*hits)[TileW<T>::W],
                                             const T (*gauss)[TileW<T>::W], const SpikeList<T> &lst,
                                             const T *gapI) {
  const uint32_t tid = threadIdx.x, lane = tid & 31;
  const uint32_t n = P.n, S = P.slots, mask = P.mask;
  const bool own = tid < np;
  const uint32_t p = own ? p0 + tid : p0;  // non-owners read a valid neuron, write nothing
  // ---- parameters ----
  const uint32_t a = P.act[p];
  const uint8_t pj = P.proj[p];
  const int32_t rf = __ldg(P.RfPed + p), sd = __ldg(P.SpiDy + p);
  const T vth = (T)__ldg(P.Vth + p), vreset = (T)__ldg(P.Vreset + p), df = (T)__ldg(P.df + p),
          ef = (T)__ldg(P.ef + p), dvm = (T)__ldg(P.dVmax + p), cm = (T)__ldg(P.Cm + p),
          leak = (T)__ldg(P.gl + p) * (T)__ldg(P.El + p) * (T)1e3, mg = (T)__ldg(P.nmda_mg + p);
  T vrev[5], dfs[5], extg[5];
#pragma unroll
  for (int r = 0; r < 5; r++) {
    vrev[r] = (T)__ldg(P.Vrev + (size_t)r * n + p);
    dfs[r] = (T)__ldg(P.dfst + (size_t)r * n + p);
    extg[r] = (T)__ldg(P.ext_g + (size_t)r * n + p);
  }
  const T ndfxt = (T)__ldg(P.nmda_dfxt + p), nefas = (T)__ldg(P.nmda_efst + p) * (T)__ldg(P.nmda_as + p);
  T pdf[4];
#pragma unroll
  for (int r = 0; r < 4; r++) pdf[r] = (T)__ldg(P.pdf + (size_t)r * n + p);
  const T pdfxt = (T)__ldg(P.p_dfxt + p), pdfst = (T)__ldg(P.p_dfst + p), pefas = (T)__ldg(P.p_efas + p);
  // ---- state ----
  T V = ((T *)P.V)[p];
  int32_t cnt = P.Count[p];
  uint32_t ns = P.NS[p];
  T G[4], est[4], sp[4];
#pragma unroll
  for (int r = 0; r < 4; r++) {
    G[r] = ((T *)P.G)[(size_t)r * n + p];
    est[r] = ((T *)P.ext_st)[(size_t)r * n + p];
    sp[r] = ((T *)P.st_pre)[(size_t)r * n + p];
  }
  T ex = ((T *)P.ext_x)[p], es = ((T *)P.ext_s)[p], xp = ((T *)P.x_pre)[p], spre = ((T *)P.s_pre)[p];
  uint32_t nsp = 0;
  // ring slots of the first steps: rv for step 0, rv2 for step 1 (PD == 2)
  static_assert(PD == 1 || PD == 2, "ring prefetch distance 1 or 2");
  long long rv[4], rv2[4];
  {
    const uint32_t tprev = (uint32_t)(P.t0 + sb - 1u) & mask, tn = (uint32_t)(P.t0 + sb) & mask;
#pragma unroll
    for (int r = 0; r < 4; r++) {
      const int ri = P.lin_of_rec[r];
      rv[r] = (ri >= 0 && own) ? (long long)__ldcg(P.ring + ((size_t)ri * n + p) * S + tprev) : 0ll;
      rv2[r] = (PD == 2 && ri >= 0 && own && L > 1) ? (long long)__ldcg(P.ring + ((size_t)ri * n + p) * S + tn) : 0ll;
    }
  }
  for (uint32_t j = 0; j < L; j++) {
    const uint32_t s = sb + j;
    const uint64_t t = P.t0 + s;
    const uint32_t tm = (uint32_t)t & mask, tprev = (uint32_t)(t - 1u) & mask;
    bool spk = false;
    T cinc[4] = {0, 0, 0, 0};
    // conductances of the previous step's spike phase
    T g[5];
#pragma unroll
    for (int r = 0; r < 4; r++) {
      g[r] = (T)0;
      const int ri = P.lin_of_rec[r];
      if (ri >= 0) {
        if (own && rv[r]) __stcg(P.ring + ((size_t)ri * n + p) * S + tprev, 0ull);
        G[r] = dfs[r] * G[r] + (T)rv[r] * (T)kInvFix;  // exact power-of-two scale
        g[r] = G[r];
        // the slot of step j + PD (final since the interval began)
        if constexpr (PD == 2) {
          rv[r] = rv2[r];
          rv2[r] = (own && j + 2 < L) ? (long long)__ldcg(P.ring + ((size_t)ri * n + p) * S + ((tm + 1u) & mask)) : 0ll;
        } else {
          rv[r] = (own && j + 1 < L) ? (long long)__ldcg(P.ring + ((size_t)ri * n + p) * S + tm) : 0ll;
        }
      }
    }
    const uint32_t qs = tid < np ? tid : 0;
    g[FS_NMDA] = gn[j][qs] * (T)P.rg[FS_NMDA];
    // external drive (BgInit): the Bernoulli outcomes of this step were drawn
    // in the pull phase (bit r: receptor r hit)
    const uint32_t hit = hits[j][qs];
    const uint32_t bitsr[4] = {FS_ACT_AMPA, FS_ACT_GABA, FS_ACT_ACH, FS_ACT_GCL};
#pragma unroll
    for (int r = 0; r < 4; r++) {
      if (a & bitsr[r]) {
        if (hit & (1u << r)) est[r] = est[r] + (T)1;
        else est[r] = est[r] * dfs[r];
        g[r] = g[r] + extg[r] * est[r];
      }
    }
    T isyn = (T)0;
    if (a & FS_ACT_NMDA) {
      if (hit & (1u << FS_NMDA)) ex = ex + (T)1;
      else ex = ex * ndfxt;
      es = dfs[FS_NMDA] * es + nefas * ex * ((T)1 - es);
      g[FS_NMDA] = g[FS_NMDA] + extg[FS_NMDA] * es;
    }
    if (a & FS_ACT_INJ) isyn = (T)gauss[j][qs];
    if (P.gap_row) isyn = isyn + gapI[qs];  // batches of one step (interval 1)
    // VmEul + firing (code/EqsGnl2.cpp:152-251)
    bool fire_now = false;
    if (ns & FS_NS_FIRE) {
      fire_now = true;
    } else {
      const T v = V;
      const T Ir0 = g[FS_AMPA] * (vrev[FS_AMPA] - v);
      const T Ir1 = g[FS_GABA] * (vrev[FS_GABA] - v);
      const T Ir2 = g[FS_NMDA] * (vrev[FS_NMDA] - v) / ((T)1 + mg * exp_t<T>((T)-0.062 * v) / (T)3.57);
      const T Ir3 = g[FS_ACH] * (vrev[FS_ACH] - v);
      const T Ir4 = g[FS_GCL] * (vrev[FS_GCL] - v);
      T I = Ir0 + Ir1 + Ir2 + Ir3 + Ir4 + isyn * (T)1e3 + leak;
      I = (T)1e-3 * I / cm;
      if (I > dvm) {
        I = dvm;
        ns = (ns | FS_NS_MEMDV_OVF) & ~FS_NS_MEMDV_UDF;
      } else if (I < -dvm) {
        I = -dvm;
        ns = (ns & ~FS_NS_MEMDV_OVF) | FS_NS_MEMDV_UDF;
      } else {
        ns &= ~(FS_NS_MEMDV_OVF | FS_NS_MEMDV_UDF);
      }
      V = df * v + ef * I;
      if (P.outI && own) {  // kept only while requested (code/EqsGnl2.cpp:196-206)
        P.Irep[p] = (float)Ir0;
        P.Irep[(size_t)n + p] = (float)Ir1;
        P.Irep[(size_t)FS_NMDA * n + p] = (float)Ir2;
        P.Irep[(size_t)FS_ACH * n + p] = (float)Ir3;
        P.Irep[(size_t)FS_GCL * n + p] = (float)Ir4;
      }
      if (V > vth) {
        ns |= FS_NS_FIRE;
        fire_now = true;
      }
    }
    if (fire_now) {
      if (cnt < rf) {
        V = (cnt == 0) ? (T)0 : vreset;
        if (cnt == sd) ns |= FS_NS_SPIKE;
        else ns &= ~FS_NS_SPIKE;
        cnt++;
      } else {
        cnt = 0;
        ns &= ~FS_NS_FIRE;
      }
    }
    if (own && P.outV) P.outV[(size_t)s * n + p] = (float)V;
    if (own && P.outNS) P.outNS[(size_t)s * n + p] = ns;
    if (own && P.outI)
#pragma unroll
      for (int r = 0; r < 5; r++) P.outI[(size_t)s * 5 * n + (size_t)r * n + p] = P.Irep[(size_t)r * n + p];
    spk = own && (ns & FS_NS_SPIKE) != 0;
    nsp += spk ? 1u : 0u;
    // presynaptic state: increment per spike, then plasticity update
    if (pj && own) {
      T inc = (T)1;
      if (P.plast == PL_STD) inc = (T)P.D[p];
      else if (P.plast == PL_STP) inc = (T)P.D[p] * (T)P.F[p];
      else if (P.plast == PL_TM && P.tm_on[p]) {
        T u = (T)P.tm_u[p], x = (T)P.tm_x[p];
        const T U = (T)P.tm_U[p];
        if (spk) {
          u = u + U * ((T)1 - u);
          const T rel = u * x;
          inc = rel;
          x = x - rel;
        } else {
          u = U + (u - U) * (T)P.tm_dff[p];
          x = (T)1 + (x - (T)1) * (T)P.tm_dfr[p];
        }
        P.tm_u[p] = (float)u;
        P.tm_x[p] = (float)x;
      }
#pragma unroll
      for (int r = 0; r < 4; r++) {
        if (pj & (1u << r)) {
          if (spk) {
            cinc[r] = inc + sp[r] * ((T)1 - pdf[r]);
            sp[r] = sp[r] + inc;
          } else {
            sp[r] = sp[r] * pdf[r];
          }
        }
      }
      if (pj & (1u << FS_NMDA)) {
        if (spk) xp = xp + inc;
        else xp = xp * pdfxt;
        spre = pdfst * spre + pefas * xp * ((T)1 - spre);
        if constexpr (sizeof(T) == 4) {
#pragma unroll
          for (uint32_t k = 0; k < kSH; k++)
            __stcg((T *)P.s_hist + ((size_t)p * kSH + k) * S + ((tm - k) & mask), spre);
        } else {
          __stcg((T *)P.s_hist + (size_t)p * S + tm, spre);
        }
      }
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
    // spikes of this warp: outputs, and the spike list the block pushes at
    // the end of the batch (a push lands >= min_delay steps ahead, so it may
    // wait until the interval's end); a full list falls back to a push by
    // this warp right away
    uint32_t m = __ballot_sync(fsd::kFull, spk);
    if (m) {
      if (spk && P.bits) atomicOr(P.bits + (size_t)s * P.words + (p >> 5), 1u << (p & 31));
      if (lane == 0) {
        if (P.counts) atomicAdd(P.counts + s, (unsigned)__popc(m));
        atomicAdd(P.spike_total, (unsigned long long)__popc(m));
      }
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
        const uint32_t q = __shfl_sync(fsd::kFull, p, jl);
        T cj[4];
#pragma unroll
        for (int r = 0; r < 4; r++) cj[r] = __shfl_sync(fsd::kFull, cinc[r], jl);
        push_spike<T>(P, q, tm, cj, lane, 32);
      }
    }
  }
  if (own) {
    ((T *)P.V)[p] = V;
    if (P.gap_row) ((T *)P.Vg)[(size_t)((P.t0 + sb) & 1u) * n + p] = V;
    P.Count[p] = cnt;
    P.NS[p] = ns;
#pragma unroll
    for (int r = 0; r < 4; r++) {
      ((T *)P.G)[(size_t)r * n + p] = G[r];
      ((T *)P.ext_st)[(size_t)r * n + p] = est[r];
      ((T *)P.st_pre)[(size_t)r * n + p] = sp[r];
    }
    ((T *)P.ext_x)[p] = ex;
    ((T *)P.ext_s)[p] = es;
    ((T *)P.x_pre)[p] = xp;
    ((T *)P.s_pre)[p] = spre;
    if (P.nspk && nsp) P.nspk[p] += nsp;
  }
}

// The steps of one block: posts [B0, B1) of the network P, whose blocks
// (nblk of them) meet at a barrier after every interval.  PU: NMDA edges in
// flight per lane in the pull; PD: ring slots in flight per neuron in the
// steps (results depend on neither).
template <class T, int PU, int PD>
__device__ __forceinline__ void prod_blocks(const Params &P, uint32_t B0, uint32_t B1, uint32_t nblk) {
  // FP64 tiles are half as wide so the per-tile buffers stay in static
  // shared memory
  constexpr uint32_t kT = TileW<T>::W;
  constexpr uint32_t kCap = sizeof(T) == 4 ? 448 : 192;
  __shared__ T gn[kLB][kT];
  __shared__ T gauss[kLB][kT];
  __shared__ T gapI[kT];
  __shared__ uint8_t hits[kLB][kT];
  __shared__ uint32_t l_n, l_p[kCap];
  __shared__ uint16_t l_tm[kCap];
  __shared__ T l_c[kCap][4];
  const SpikeList<T> lst{&l_n, l_p, l_tm, l_c, kCap};
  const uint32_t tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  if (tid == 0) l_n = 0;
  __syncthreads();
  uint32_t s = 0;
  while (s < P.nsteps) {
    const uint32_t iv_end = min(P.nsteps, s + P.interval);
    for (uint32_t bs = s; bs < iv_end; bs += kLB) {
      const uint32_t L = min(kLB, iv_end - bs);
      for (uint32_t tp0 = B0; tp0 < B1; tp0 += kT) {
        const uint32_t np = min(kT, B1 - tp0);
        if constexpr (sizeof(T) == 4) {
          if (L == 1) nmda_pull1_f32(P, tp0, np, P.t0 + bs, (float (*)[kTile])gn, wid, lane);
          else nmda_pull_f32<PU>(P, tp0, np, P.t0 + bs, L, (float (*)[kTile])gn, wid, lane);
        }
        else nmda_pull<T>(P, tp0, np, P.t0 + bs, L, gn, wid, lane);
        draw_inputs<T>(P, tp0, np, P.t0 + bs, L, hits, gauss);
        if (P.gap_row) {
          // gap currents of this step (interval 1): g (V_other - V_self) over
          // V at the end of the previous step (none before the first step)
          const uint64_t t = P.t0 + bs;
          for (uint32_t q = tid; q < np; q += kThreads) {
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
        __syncthreads();
        // warps without neurons in this tile skip the steps
        if ((tid & ~31u) < np) neuron_steps<T, PD>(P, tp0, np, bs, L, gn, hits, gauss, lst, gapI);
        __syncthreads();
        // the batch's spikes: with fewer spikes than warps the whole block
        // walks each spike's out-edges (a hub's hundreds of edges in one or
        // two rounds); with more, one spike per warp, eight in flight
        const uint32_t nl = min(l_n, kCap);
        if (nl < kThreads / 32) {
          for (uint32_t k = 0; k < nl; k++) {
            T cj[4];
#pragma unroll
            for (int r = 0; r < 4; r++) cj[r] = l_c[k][r];
            push_spike<T>(P, l_p[k], l_tm[k], cj, tid, kThreads);
          }
        } else {
          for (uint32_t k = wid; k < nl; k += kThreads / 32) {
            T cj[4];
#pragma unroll
            for (int r = 0; r < 4; r++) cj[r] = l_c[k][r];
            push_spike<T>(P, l_p[k], l_tm[k], cj, lane, 32);
          }
        }
        __syncthreads();
        if (tid == 0) l_n = 0;
      }
    }
    s = iv_end;
    if (s < P.nsteps) {
      if (!grid_sync(P.bar, P.err, nblk)) return;
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

// ---- batch: many independent networks in one persistent launch -----------
// Block b works on instance blk[b].inst, posts [b0, b1), and meets only the
// other blocks of that instance (blk[b].nblk of them) at its barriers, so
// instances of different sizes and intervals advance independently.
struct BatchBlock {
  uint32_t inst, b0, b1, nblk;
};

template <class T>
__global__ void __launch_bounds__(kThreads) k_prod_batch(const Params *__restrict__ Ps,
                                                         const BatchBlock *__restrict__ blk) {
  __shared__ __align__(16) Params Psh;
  const BatchBlock me = blk[blockIdx.x];
  {
    const uint32_t *src = (const uint32_t *)(Ps + me.inst);
    uint32_t *dst = (uint32_t *)&Psh;
    for (uint32_t i = threadIdx.x; i < sizeof(Params) / 4; i += blockDim.x) dst[i] = src[i];
  }
  __syncthreads();
  prod_blocks<T, 8, 1>(Psh, me.b0, me.b1, me.nblk);
}

// Advances every instance's step counter after a batch launch (graph node).
__global__ void k_batch_advance(Params *Ps, uint32_t count, uint32_t nsteps) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < count) Ps[i].t0 += nsteps;
}

// ---- host side -------------------------------------------------------------
struct Prod {
  bool fp64 = false;
  bool wide = false;  // some block's posts span several tiles: eight NMDA edges in flight
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
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  double ms = 0.0;
  uint64_t kl = 0;
  uint64_t key = 0;
  std::vector<uint32_t> host_counts;
  std::vector<uint32_t> in_row_h;  // NMDA in-degree prefix (block partitioning)
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

int launch(Prod *p, uint32_t nsteps, bool want_bits, bool wantV, cudaStream_t st, uint64_t *launches,
           std::string &err, bool wantI = false, bool wantNS = false) {
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
  P.bar = p->bar;
  P.err = p->err;
  P.spike_total = p->spike_total;
  void *args[] = {&P};
  cudaEventRecord(p->e0, st);
  // (the FP64 pull does not take the edges-in-flight parameter)
  const void *k = p->fp64 ? (const void *)k_prod<double, 4>
                          : (p->wide ? (const void *)k_prod<float, 8> : (const void *)k_prod<float, 4>);
  e = cudaLaunchCooperativeKernel(k, p->blocks, kThreads, args, 0, st);
  cudaEventRecord(p->e1, st);
  if (e != cudaSuccess) {
    err = std::string("cooperative launch: ") + cudaGetErrorString(e);
    return FS_ERR_CUDA;
  }
  p->t += nsteps;
  if (launches) *launches += 1;
  p->kl += 1;
  return FS_OK;
}

int finish(Prod *p, cudaStream_t st, std::string &err) {
  cudaError_t e = cudaEventSynchronize(p->e1);
  if (e != cudaSuccess) {
    err = std::string("kernel: ") + cudaGetErrorString(e);
    return FS_ERR_CUDA;
  }
  float ms = 0;
  cudaEventElapsedTime(&ms, p->e0, p->e1);
  p->ms += ms;
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

int prod_create(Prod **out, const fs_net_desc *d, const fs_run_opts &o, uint32_t sm_count, cudaStream_t st,
                std::string &err) {
  *out = nullptr;
  const fs_neurons &v = d->neurons;
  const uint32_t n = v.n;
  if (n >= (1u << 22)) {
    err = "production modes support up to 4,194,303 neurons per handle";
    return FS_ERR_UNSUPPORTED;
  }
  if (d->act_ctr & FS_ACT_LTP) {
    err = "production modes do not implement LTP (use FS_MODE_COMPAT)";
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
  const fs_syn_list &S = *d->syn;
  // ---- receptor kinetics seen by each presynaptic neuron ----
  std::vector<float> pdf((size_t)4 * n, -1.0f), p_dfxt(n, -1.0f), p_dfst(n, -1.0f), p_efas(n, -1.0f);
  std::vector<uint8_t> proj(n, 0);
  bool present[5] = {false, false, false, false, false};
  uint32_t dmin = 0xffffffffu, dmax = 0;
  uint64_t nlin_e = 0, nnm_e = 0;
  for (uint64_t e = 0; e < S.n; e++) {
    const uint32_t a = S.pre[e], b = S.post[e], r = S.rec[e];
    const uint32_t dl = S.delay ? S.delay[e] : 0;
    if (a >= n || b >= n || r >= FS_NREC) {
      err = "synapse list: index out of range";
      delete p;
      return FS_ERR_ARG;
    }
    if (dl > 255) {
      err = "synapse delays above 255 steps are not supported";
      delete p;
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
      delete p;
      return FS_ERR_UNSUPPORTED;
    }
  }
  if (S.n == 0) dmin = 0;
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
  if (gap) P.interval = 1;  // a gap current reads every neuron's V of the step before
  for (int r = 0; r < 4; r++) P.lin_of_rec[r] = present[r] ? (int)(p->nlin++) : -1;
  P.nlin = p->nlin;
  for (auto &x : pdf) if (x < 0) x = 0;
  for (auto *vv : {&p_dfxt, &p_dfst, &p_efas}) for (auto &x : *vv) if (x < 0) x = 0;
  // ---- CSR of linear out-edges (by pre) and NMDA in-edges (by post) ----
  std::vector<uint32_t> out_row(n + 1, 0), in_row(n + 1, 0);
  for (uint64_t e = 0; e < S.n; e++) {
    if (S.rec[e] == FS_NMDA) in_row[S.post[e] + 1]++;
    else out_row[S.pre[e] + 1]++;
  }
  for (uint32_t i = 0; i < n; i++) { out_row[i + 1] += out_row[i]; in_row[i + 1] += in_row[i]; }
  std::vector<uint32_t> out_code(nlin_e), in_code(nnm_e);
  std::vector<float> out_w(nlin_e), in_w(nnm_e);
  {
    std::vector<uint32_t> fo(out_row.begin(), out_row.end() - 1), fi(in_row.begin(), in_row.end() - 1);
    for (uint64_t e = 0; e < S.n; e++) {
      const uint32_t dl = S.delay ? S.delay[e] : 0;
      if (S.rec[e] == FS_NMDA) {
        const uint32_t q = fi[S.post[e]]++;
        in_code[q] = S.pre[e] | (dl << 24);
        in_w[q] = S.g[e];
      } else {
        const uint32_t q = fo[S.pre[e]]++;
        out_code[q] = S.post[e] | ((uint32_t)S.rec[e] << 22) | (dl << 24);
        out_w[q] = S.g[e];
      }
    }
  }
  // ---- grid: all blocks co-resident; posts split by estimated cost ----
  int occ = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, p->fp64 ? (const void *)k_prod<double, 4> : (const void *)k_prod<float, 4>,
                                                kThreads, 0);
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
  if ((rc = dal(p, &p->bar, 64, err)) || (rc = dal(p, &p->err, 1, err)) ||
      (rc = dup(p, &p->spike_total, (const unsigned long long *)nullptr, 1, st, err)))
    goto fail;
  if (cudaMemsetAsync(p->err, 0, 4, st) != cudaSuccess) { rc = FS_ERR_CUDA; err = "memset"; goto fail; }
  if (cudaEventCreate(&p->e0) != cudaSuccess || cudaEventCreate(&p->e1) != cudaSuccess) {
    rc = FS_ERR_CUDA;
    err = "event create";
    goto fail;
  }
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
  for (void *q : p->allocs) cudaFree(q);
  if (p->e0) cudaEventDestroy(p->e0);
  if (p->e1) cudaEventDestroy(p->e1);
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
    if (out && out->gv_n) {
      err = "production modes aggregate the synapse gates: GatingVariable output needs FS_MODE_COMPAT";
      return FS_ERR_UNSUPPORTED;
    }
    int rc = launch(p, b, true, wantV, st, launches, err, wantI, wantNS);
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
  info->blocks = p->blocks;
  info->threads = kThreads;
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

// ---- batch of independent networks ------------------------------------------
struct Batch {
  bool fp64 = false;
  uint32_t sm = 148, occ = 1;
  std::vector<Prod *> inst;
  std::vector<uint32_t> seeds;
  Params *dP = nullptr;          // [count] parameters as the kernel reads them
  BatchBlock *dB = nullptr;      // [blocks]
  uint32_t dB_cap = 0;
  unsigned int *bars = nullptr;  // [count][64]
  int *errs = nullptr;           // [count]
  uint32_t blocks = 0, per_sm = 0;
  double upd = 24.0;
  uint32_t chunk = 10000;
  uint32_t dev_nsteps = 0;       // nsteps the device parameter array holds (0: stale)
  cudaGraphExec_t exec = nullptr;
  uint32_t graph_steps = 0;
  bool graph_ok = true;          // capture works for this launch
  bool graph_used = false;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  double ms = 0.0;
  uint64_t launches = 0;
};

namespace {

template <class X>
cudaError_t bal(X **p, size_t count) {
  return cudaMalloc((void **)p, count * sizeof(X));
}

// cost-balanced split of an instance's posts into k contiguous ranges
void split_posts(const Prod *p, uint32_t k, double upd, std::vector<uint32_t> &bp) {
  const uint32_t n = p->n;
  bp.assign(k + 1, n);
  bp[0] = 0;
  const std::vector<uint32_t> &in = p->in_row_h;
  const double total = (double)p->nmda_edges + upd * n;
  double acc = 0;
  uint32_t b = 1;
  for (uint32_t q = 0; q < n && b < k; q++) {
    acc += upd + (double)(in[q + 1] - in[q]);
    while (b < k && acc >= total * b / k) bp[b++] = q + 1;
  }
  for (; b < k; b++) bp[b] = n;
}

int batch_plan(Batch *B, uint32_t per_sm, double upd, std::string &err) {
  const uint32_t count = (uint32_t)B->inst.size();
  const uint32_t total = B->sm * per_sm;
  if (count > total) {
    err = "batch of " + std::to_string(count) + " instances exceeds the " + std::to_string(total) +
          " co-resident blocks of one launch";
    return FS_ERR_CAPACITY;
  }
  std::vector<double> c(count);
  double sum = 0;
  for (uint32_t i = 0; i < count; i++) sum += (c[i] = upd * B->inst[i]->n + (double)B->inst[i]->nmda_edges);
  // one block each, the rest by cost (largest remainder), at most n/8 blocks
  std::vector<uint32_t> k(count, 1);
  std::vector<std::pair<double, uint32_t>> rem;
  uint32_t used = count;
  for (uint32_t i = 0; i < count; i++) {
    const double want = (double)(total - count) * c[i] / sum;
    const uint32_t cap = std::max<uint32_t>(1, (B->inst[i]->n + 7) / 8);
    const uint32_t add = std::min<uint32_t>((uint32_t)want, cap - 1);
    k[i] += add;
    used += add;
    rem.push_back({want - (double)add, i});
  }
  std::sort(rem.begin(), rem.end(), [](const std::pair<double, uint32_t> &a, const std::pair<double, uint32_t> &b) {
    return a.first > b.first || (a.first == b.first && a.second < b.second);
  });
  for (size_t r = 0; r < rem.size() && used < total; r++) {
    const uint32_t i = rem[r].second;
    if (k[i] < std::max<uint32_t>(1, (B->inst[i]->n + 7) / 8)) { k[i]++; used++; }
  }
  std::vector<BatchBlock> plan;
  std::vector<uint32_t> bp;
  for (uint32_t i = 0; i < count; i++) {
    split_posts(B->inst[i], k[i], upd, bp);
    for (uint32_t j = 0; j < k[i]; j++) plan.push_back(BatchBlock{i, bp[j], bp[j + 1], k[i]});
  }
  if (plan.size() > B->dB_cap) {
    if (B->dB) cudaFree(B->dB);
    B->dB = nullptr;
    B->dB_cap = 0;
    cudaError_t e = bal(&B->dB, plan.size());
    if (e != cudaSuccess) {
      err = std::string("cudaMalloc: ") + cudaGetErrorString(e);
      return FS_ERR_NOMEM;
    }
    B->dB_cap = (uint32_t)plan.size();
  }
  cudaError_t e = cudaMemcpy(B->dB, plan.data(), plan.size() * sizeof(BatchBlock), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    err = std::string("plan upload: ") + cudaGetErrorString(e);
    return FS_ERR_CUDA;
  }
  B->blocks = (uint32_t)plan.size();
  B->per_sm = per_sm;
  B->upd = upd;
  if (B->exec) cudaGraphExecDestroy(B->exec);
  B->exec = nullptr;
  B->graph_steps = 0;
  return FS_OK;
}

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
    P.bar = B->bars + 64 * (size_t)i;
    P.err = B->errs + i;
    P.spike_total = B->inst[i]->spike_total;
    hp[i] = P;
  }
  cudaError_t e = cudaMemcpyAsync(B->dP, hp.data(), count * sizeof(Params), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    err = std::string("batch parameter upload: ") + cudaGetErrorString(e);
    return FS_ERR_CUDA;
  }
  B->dev_nsteps = nsteps;
  return FS_OK;
}

cudaError_t batch_enqueue(Batch *B, uint32_t nsteps, cudaStream_t st) {
  void *args[] = {&B->dP, &B->dB};
  cudaError_t e = B->fp64 ? cudaLaunchCooperativeKernel((void *)k_prod_batch<double>, B->blocks, kThreads, args, 0, st)
                          : cudaLaunchCooperativeKernel((void *)k_prod_batch<float>, B->blocks, kThreads, args, 0, st);
  if (e != cudaSuccess) return e;
  const uint32_t count = (uint32_t)B->inst.size();
  k_batch_advance<<<(count + 255) / 256, 256, 0, st>>>(B->dP, count, nsteps);
  return cudaGetLastError();
}

// one launch of nsteps for every instance: a replay of the captured graph
// when one exists for this step count, else a direct launch
int batch_launch(Batch *B, uint32_t nsteps, cudaStream_t st, std::string &err) {
  int rc;
  if (B->dev_nsteps != nsteps && (rc = batch_upload(B, nsteps, st, err))) return rc;
  cudaError_t e = cudaSuccess;
  if (B->graph_ok && B->graph_steps != nsteps) {
    if (B->exec) cudaGraphExecDestroy(B->exec);
    B->exec = nullptr;
    B->graph_steps = 0;
    cudaGraph_t g = nullptr;
    e = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
      cudaError_t le = batch_enqueue(B, nsteps, st);
      e = cudaStreamEndCapture(st, &g);
      if (le != cudaSuccess) e = le;
    }
    if (e == cudaSuccess) e = cudaGraphInstantiate(&B->exec, g, 0);
    if (g) cudaGraphDestroy(g);
    if (e == cudaSuccess) {
      B->graph_steps = nsteps;
    } else {
      // this launch form cannot be captured here: launch it directly
      cudaGetLastError();
      B->graph_ok = false;
      if (B->exec) cudaGraphExecDestroy(B->exec);
      B->exec = nullptr;
    }
  }
  if (B->exec && B->graph_steps == nsteps) {
    e = cudaGraphLaunch(B->exec, st);
    B->graph_used = true;
  } else {
    e = batch_enqueue(B, nsteps, st);
  }
  if (e != cudaSuccess) {
    err = std::string("batch launch: ") + cudaGetErrorString(e);
    return FS_ERR_CUDA;
  }
  for (Prod *p : B->inst) p->t += nsteps;
  B->launches++;
  return FS_OK;
}

int batch_check(Batch *B, cudaStream_t st, std::string &err) {
  cudaError_t e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    err = std::string("batch kernel: ") + cudaGetErrorString(e);
    return FS_ERR_CUDA;
  }
  std::vector<int> h(B->inst.size());
  e = cudaMemcpy(h.data(), B->errs, h.size() * 4, cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) {
    err = std::string("error words: ") + cudaGetErrorString(e);
    return FS_ERR_CUDA;
  }
  for (size_t i = 0; i < h.size(); i++)
    if (h[i]) {
      err = "instance " + std::to_string(i) + ": barrier wait gave up (device error word set)";
      return FS_ERR_TIMEOUT;
    }
  return FS_OK;
}

}  // namespace

void batch_destroy(Batch *B) {
  if (!B) return;
  for (Prod *p : B->inst) prod_destroy(p);
  if (B->exec) cudaGraphExecDestroy(B->exec);
  if (B->dP) cudaFree(B->dP);
  if (B->dB) cudaFree(B->dB);
  if (B->bars) cudaFree(B->bars);
  if (B->errs) cudaFree(B->errs);
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
  B->sm = sm_count;
  B->chunk = o.chunk_steps ? o.chunk_steps : 10000;
  int rc = FS_OK;
  for (uint32_t i = 0; i < count && rc == FS_OK; i++) {
    Prod *p = nullptr;
    if (!descs[i]) {
      err = "batch: null network description " + std::to_string(i);
      rc = FS_ERR_ARG;
      break;
    }
    rc = prod_create(&p, descs[i], o, sm_count, st, err);
    if (rc) err = "instance " + std::to_string(i) + ": " + err;
    else B->inst.push_back(p);
  }
  int occ = 0;
  if (rc == FS_OK) {
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        &occ, B->fp64 ? (const void *)k_prod_batch<double> : (const void *)k_prod_batch<float>, kThreads, 0);
    B->occ = (uint32_t)std::max(1, occ);
    cudaError_t e = bal(&B->dP, count);
    if (e == cudaSuccess) e = bal(&B->bars, (size_t)count * 64);
    if (e == cudaSuccess) e = bal(&B->errs, count);
    if (e == cudaSuccess) e = cudaMemset(B->bars, 0, (size_t)count * 64 * 4);
    if (e == cudaSuccess) e = cudaMemset(B->errs, 0, (size_t)count * 4);
    if (e == cudaSuccess) e = cudaEventCreate(&B->e0);
    if (e == cudaSuccess) e = cudaEventCreate(&B->e1);
    if (e != cudaSuccess) {
      err = std::string("batch buffers: ") + cudaGetErrorString(e);
      rc = FS_ERR_NOMEM;
    }
  }
  if (rc == FS_OK) {
    uint32_t per_sm = std::min<uint32_t>(B->occ, 2);
    if (o.blocks_per_sm) per_sm = std::min<uint32_t>(B->occ, o.blocks_per_sm);
    while (per_sm < B->occ && B->sm * per_sm < count) per_sm++;
    rc = batch_plan(B, per_sm, 24.0, err);
  }
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
  cudaError_t e = cudaMemsetAsync(B->bars, 0, B->inst.size() * 64 * 4, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(B->errs, 0, B->inst.size() * 4, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    err = std::string("batch reset: ") + cudaGetErrorString(e);
    return FS_ERR_CUDA;
  }
  B->dev_nsteps = 0;
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

int batch_tune(Batch *B, uint32_t sample_steps, cudaStream_t st, BatchPlan *out, std::string &err) {
  if (!sample_steps) sample_steps = 200;
  double best = -1.0;
  uint32_t best_ps = B->per_sm;
  double best_upd = B->upd;
  const double upds[3] = {8.0, 24.0, 64.0};
  uint32_t tried = 0;
  for (uint32_t ps = 1; ps <= std::min<uint32_t>(B->occ, 4); ps++) {
    if (B->sm * ps < B->inst.size()) continue;
    for (double u : upds) {
      int rc = batch_plan(B, ps, u, err);
      if (rc) return rc;
      if ((rc = batch_reset(B, nullptr, st, err))) return rc;
      double ms = 0;
      if ((rc = batch_run(B, sample_steps, st, nullptr, err))) return rc;   // warm-up (graph capture)
      if ((rc = batch_run(B, sample_steps, st, &ms, err))) return rc;
      tried++;
      if (best < 0 || ms < best) {
        best = ms;
        best_ps = ps;
        best_upd = u;
      }
    }
  }
  int rc = batch_plan(B, best_ps, best_upd, err);
  if (rc == FS_OK) rc = batch_reset(B, nullptr, st, err);
  if (rc) return rc;
  B->ms = 0.0;
  if (out) {
    out->blocks = B->blocks;
    out->blocks_per_sm = B->per_sm;
    out->cost_update = best_upd;
    out->sample_ms = best;
    out->candidates = tried;
  }
  return FS_OK;
}

void batch_info(const Batch *B, BatchPlan *out) {
  out->blocks = B->blocks;
  out->blocks_per_sm = B->per_sm;
  out->cost_update = B->upd;
  out->sample_ms = 0.0;
  out->candidates = 0;
  out->graph = B->graph_used ? 1 : 0;
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

// ---- failure detection check ---------------------------------------------
// One block waits at a barrier of two blocks that the second never reaches:
// the bounded wait gives up after `limit` polls, sets the error word and
// returns, and the context stays usable.
__global__ void k_barrier_probe(unsigned int *bar, int *err, unsigned int limit) { grid_sync(bar, err, 2, limit); }

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
  B->dev_nsteps = 0;  // the device copy of the parameters is stale
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
