// Reference-order FP32 kernels of the flysim step (FS_MODE_COMPAT).
//
// Compiled with -fmad=false and IEEE division/denormals (no fast math): every
// floating-point expression below is evaluated with the operand order and
// rounding of the reference's g++ -O3 SSE2 build, so the spike raster equals
// the reference's bit for bit.  Kernel map (reference code they replace):
//   k_activation  EqsGnl2::Activation = BgInit + VmEul + firing (+ firLP/ltpEul)
//                 (code/EqsGnl2.cpp:152-337, :1098-1105); one thread per neuron,
//                 spike flags ballot-packed into a per-step bitmap
//   k_gates       ThdPGatVar / STD / STP: group gate updates (code/EqsGnl2.cpp:728-932)
//   k_gather      ThdPSynapse + ThdSynapse* + ThdGapSyn (code/EqsGnl2.cpp:404-725,
//                 :937-1002); one warp per post-synaptic neuron: terms are formed
//                 lane-parallel and then added in the reference's order
//   k_plasticity  STP / STD / LTP (code/EqsGnl2.cpp:1005-1090)
//   k_mt19937     the std::mt19937 output stream the reference draws from
//   k_count / k_write   ordered spike-list compaction (ballot bitmaps, block prefix)
#include <cstdint>
#include <cuda_runtime.h>
#include "fs_device.cuh"

namespace fsd {

__constant__ uint32_t c_kn[128];
__constant__ float c_fn[128];
__constant__ float c_wn[128];
__constant__ uint32_t c_jump_a[32];  // congruential map x -> a*x + c raised to 2^i
__constant__ uint32_t c_jump_c[32];

// ---- glibc-exact float exp/log ----------------------------------------
// (float)exp((double)x) rounds correctly except when e^x lies within a few
// double ulps of a float rounding boundary; glibc's expf itself is not always
// correctly rounded.  The exception table holds glibc's result for every
// input of the tabulated range where the two may differ (generated at build
// time by calling glibc, see fs_tables.cpp).
__device__ __forceinline__ float table_patch(float r, float x, const uint32_t *keys, const float *vals,
                                             uint32_t n) {
  const uint32_t k = __float_as_uint(x);
  uint32_t lo = 0, hi = n;
  while (lo < hi) {
    const uint32_t mid = (lo + hi) >> 1;
    if (__ldg(keys + mid) < k) lo = mid + 1;
    else hi = mid;
  }
  if (lo < n && __ldg(keys + lo) == k) r = __ldg(vals + lo);
  return r;
}
__device__ __forceinline__ float expf_ref(float x, const CompatDev &d) {
  return table_patch((float)exp((double)x), x, d.expf_keys, d.expf_vals, d.expf_n);
}
__device__ __forceinline__ float logf_ref(float x, const CompatDev &d) {
  return table_patch((float)log((double)x), x, d.logf_keys, d.logf_vals, d.logf_n);
}

// ---- random streams ----------------------------------------------------
// uniform_real_distribution<float>(0,1) over mt19937 (libstdc++
// generate_canonical<float,24>: one 32-bit draw, float(x) * 2^-32, values
// rounding up to 1 replaced by the largest float below 1).
__device__ __forceinline__ float u01(uint32_t x) {
  float u = __uint2float_rn(x) * 2.3283064365386963e-10f;
  return (u >= 1.0f) ? 0.99999994f : u;
}

__device__ __forceinline__ uint32_t shr3(uint32_t &jsr) {
  const uint32_t in = jsr;
  jsr = jsr ^ (jsr << 13);
  jsr = jsr ^ (jsr >> 17);
  jsr = jsr ^ (jsr << 5);
  return in + jsr;
}
__device__ __forceinline__ float zuni(uint32_t &jsr) {
  const uint32_t in = jsr;
  jsr = jsr ^ (jsr << 13);
  jsr = jsr ^ (jsr >> 17);
  jsr = jsr ^ (jsr << 5);
  return (float)fmod(0.5 + (double)__uint2float_rn(in + jsr) / 65536.0 / 65536.0, 1.0);
}
// Marsaglia–Tsang ziggurat normal (code/StiExt.h:262-319).
__device__ float zig_nor(uint32_t &jsr, const CompatDev &d) {
  const float r = 3.442620f;
  int hz = (int)shr3(jsr);
  uint32_t iz = (uint32_t)(hz & 127);
  if (fabs((double)hz) < (double)c_kn[iz]) return (float)hz * c_wn[iz];
  for (int guard = 0; guard < 100000; guard++) {
    if (iz == 0) {
      float x, y;
      for (int g2 = 0; g2 < 100000; g2++) {
        x = (float)(-0.2904764 * (double)logf_ref(zuni(jsr), d));
        y = -logf_ref(zuni(jsr), d);
        if (x * x <= y + y) break;
      }
      return (hz <= 0) ? -r - x : r + x;
    }
    const float x = (float)hz * c_wn[iz];
    const float lhs = c_fn[iz] + zuni(jsr) * (c_fn[iz - 1] - c_fn[iz]);
    if ((double)lhs < exp(-0.5 * (double)x * (double)x)) return x;
    hz = (int)shr3(jsr);
    iz = (uint32_t)(hz & 127);
    if (fabs((double)hz) < (double)c_kn[iz]) return (float)hz * c_wn[iz];
  }
  if (d.err) atomicOr(d.err, 1);
  return 0.0f;
}
// jcong after k further congruential steps
__device__ __forceinline__ uint32_t jcong_jump(uint32_t x, uint32_t k) {
#pragma unroll 1
  for (int i = 0; k; i++, k >>= 1)
    if (k & 1) x = c_jump_a[i] * x + c_jump_c[i];
  return x;
}

// ---- firing (code/EqsGnl2.cpp:229-251) ----------------------------------
__device__ __forceinline__ void firing(float &V, int32_t &cnt, uint32_t &ns, int32_t rf, int32_t sd,
                                       float vreset) {
  if (cnt < rf) {
    V = (cnt == 0) ? 0.0f : vreset;
    if (cnt == sd) ns |= FS_NS_SPIKE;
    else ns &= ~FS_NS_SPIKE;
    cnt++;
  } else {
    cnt = 0;
    ns &= ~FS_NS_FIRE;
  }
}

// ---- Activation ---------------------------------------------------------
__global__ void __launch_bounds__(256) k_activation(const __grid_constant__ CompatDev d, uint32_t s) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t n = d.n;
  bool spk = false;
  if (i < n) {
    const uint32_t a = d.act[i];
    float g[FS_NREC];
#pragma unroll
    for (int r = 0; r < FS_NREC; r++) g[r] = d.G[(size_t)r * n + i];
    float isyn = d.Isyn[i];
    // BgInit (code/EqsGnl2.cpp:284-337): one draw per enabled receptor
    uint32_t pos = s * d.draws_per_step + d.drawoff[i];
    const uint32_t bits[4] = {FS_ACT_AMPA, FS_ACT_GABA, FS_ACT_ACH, FS_ACT_GCL};
#pragma unroll
    for (int r = 0; r < 4; r++) {
      if (a & bits[r]) {
        const float u = u01(d.draws[pos++]);
        float st = d.ext_st[(size_t)r * n + i];
        if (d.pb[(size_t)r * n + i] > u) st = st + 1.0f;
        else st = st * d.dfst[(size_t)r * n + i];
        d.ext_st[(size_t)r * n + i] = st;
        g[r] = g[r] + d.ext_g[(size_t)r * n + i] * st;
      }
    }
    if (a & FS_ACT_NMDA) {
      const float u = u01(d.draws[pos++]);
      float xt = d.ext_xt_n[i], st = d.ext_st_n[i];
      if (d.pb[(size_t)FS_NMDA * n + i] > u) xt = xt + 1.0f;
      else xt = xt * d.nmda_dfxt[i];
      st = d.dfst[(size_t)FS_NMDA * n + i] * st + d.nmda_efst[i] * d.nmda_as[i] * xt * (1.0f - st);
      d.ext_xt_n[i] = xt;
      d.ext_st_n[i] = st;
      g[FS_NMDA] = g[FS_NMDA] + d.ext_g[(size_t)FS_NMDA * n + i] * st;
    }
    if (a & FS_ACT_INJ) {
      const uint32_t k = s * d.inj_per_step + d.injoff[i] + 1u;
      uint32_t jsr = jcong_jump(d.jcong_base, k);
      isyn = isyn + (d.inj_mean[i] + d.inj_std[i] * zig_nor(jsr, d));
    }
    // VmEul (code/EqsGnl2.cpp:152-225)
    float V = d.V[i];
    int32_t cnt = d.Count[i];
    uint32_t ns = d.NS[i];
    const int32_t rf = d.RfPed[i], sd = d.SpiDy[i];
    const float vreset = d.Vreset[i];
    if (ns & FS_NS_FIRE) {
      firing(V, cnt, ns, rf, sd, vreset);
    } else {
      const float v = V;
      float Ir[5];
      Ir[0] = g[FS_AMPA] * (d.Vrev[(size_t)FS_AMPA * n + i] - v);
      Ir[1] = g[FS_GABA] * (d.Vrev[(size_t)FS_GABA * n + i] - v);
      Ir[2] = g[FS_NMDA] * (d.Vrev[(size_t)FS_NMDA * n + i] - v) /
              (1.0f + d.nmda_mg[i] * expf_ref(-0.062f * v, d) / 3.57f);
      Ir[3] = g[FS_ACH] * (d.Vrev[(size_t)FS_ACH * n + i] - v);
      Ir[4] = g[FS_GCL] * (d.Vrev[(size_t)FS_GCL * n + i] - v);
      float I = Ir[0] + Ir[1] + Ir[2] + Ir[3] + Ir[4] + isyn * 1e3f + d.gl[i] * d.El[i] * 1e3f;
      I = 1e-3f * I / d.Cm[i];
      const float dv = d.dVmax[i];
      if (I > dv) {
        I = dv;
        ns |= FS_NS_MEMDV_OVF;
        ns &= ~FS_NS_MEMDV_UDF;
      } else if (I < -dv) {
        I = -dv;
        ns &= ~FS_NS_MEMDV_OVF;
        ns |= FS_NS_MEMDV_UDF;
      } else {
        ns &= ~(FS_NS_MEMDV_OVF | FS_NS_MEMDV_UDF);
      }
      V = d.df[i] * v + d.ef[i] * I;
#pragma unroll
      for (int r = 0; r < 5; r++) d.Irep[(size_t)r * n + i] = Ir[r];
      if (V > d.Vth[i]) {
        ns |= FS_NS_FIRE;
        firing(V, cnt, ns, rf, sd, vreset);
        if (a & FS_ACT_LTP) ns |= FS_NS_LP_FIRE;
      }
    }
    if (a & FS_ACT_LTP) {  // firLP + ltpEul (code/EqsGnl2.cpp:254-280)
      int32_t clp = d.CountLP[i];
      if (ns & FS_NS_LP_FIRE) {
        if (clp == d.ltp_SpiLPDy[i]) {
          ns |= FS_NS_LP_SPIKE;
          ns &= ~FS_NS_LP_FIRE;
          clp = 0;
        } else {
          ns &= ~FS_NS_LP_SPIKE;
          clp++;
        }
      } else {
        ns &= ~FS_NS_LP_SPIKE;
      }
      d.CountLP[i] = clp;
      if (ns & FS_NS_LP_SPIKE) d.LP[i] = d.LP[i] + 1.0f;
      else d.LP[i] = d.ltp_dfLP[i] * d.LP[i];
    }
    d.V[i] = V;
    d.Count[i] = cnt;
    d.NS[i] = ns;
#pragma unroll
    for (int r = 0; r < FS_NREC; r++) d.G[(size_t)r * n + i] = 0.0f;
    d.Isyn[i] = 0.0f;
    spk = (ns & FS_NS_SPIKE) != 0;
    if (d.outV) d.outV[(size_t)s * n + i] = V;
    if (d.outNS) d.outNS[(size_t)s * n + i] = ns;
    if (d.outIrep)
#pragma unroll
      for (int r = 0; r < 5; r++) d.outIrep[(size_t)s * FS_NREC * n + (size_t)r * n + i] = d.Irep[(size_t)r * n + i];
  }
  const uint32_t b = __ballot_sync(kFull, spk);
  if ((threadIdx.x & 31) == 0 && (i >> 5) < d.words) d.spikebits[(size_t)s * d.words + (i >> 5)] = b;
}

// ---- group gates --------------------------------------------------------
__device__ __forceinline__ float gate_inc(const CompatDev &d, uint32_t pre, bool nmda) {
  if (d.glob & FS_ACT_STP) return d.D[pre] * d.F[pre];
  if (d.glob & FS_ACT_STD) return nmda ? d.D[pre] * d.F[pre] : d.D[pre];
  return 1.0f;
}

__global__ void __launch_bounds__(256) k_gates(const __grid_constant__ CompatDev d) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= d.gate_off[FS_NREC]) return;
  int r = 0;
#pragma unroll
  for (int q = 1; q < FS_NREC; q++)
    if (t >= d.gate_off[q]) r = q;
  const uint32_t n = d.n;
  const uint32_t k = t - d.gate_off[r];
  // select the receptor's arrays with static indices
  const RecDev *R = nullptr;
  switch (r) {
    case 0: R = &d.R[0]; break;
    case 1: R = &d.R[1]; break;
    case 2: R = &d.R[2]; break;
    case 3: R = &d.R[3]; break;
    default: R = &d.R[4]; break;
  }
  const uint32_t pre = R->gate_pre[k], p0 = R->gate_post0[k];
  const bool spk = (d.NS[pre] & FS_NS_SPIKE) != 0;
  const bool plastic = (d.glob & (FS_ACT_STP | FS_ACT_STD)) != 0;
  if (r != FS_NMDA) {
    float st = R->gate_st[k];
    if (spk) st = plastic ? st + gate_inc(d, pre, false) : st + 1.0f;
    else st = st * d.dfst[(size_t)r * n + p0];
    R->gate_st[k] = st;
  } else {
    float xt = R->gate_xt[k], st = R->gate_st[k];
    if (spk) xt = plastic ? xt + gate_inc(d, pre, true) : xt + 1.0f;
    else xt = xt * d.nmda_dfxt[p0];
    st = d.dfst[(size_t)FS_NMDA * n + p0] * st + d.nmda_efst[p0] * d.nmda_as[p0] * xt * (1.0f - st);
    R->gate_xt[k] = xt;
    R->gate_st[k] = st;
  }
}

// ---- ordered gather: warp per post ---------------------------------------
// Adds the lane terms t (lane j holds term j of this chunk) to acc in lane
// order; every lane ends with the same acc.
__device__ __forceinline__ float ordered_add(float acc, float t, uint32_t cnt) {
#pragma unroll 8
  for (uint32_t j = 0; j < cnt; j++) acc = acc + __shfl_sync(kFull, t, (int)j);
  return acc;
}

template <int r>
__device__ __forceinline__ void gather_rec(const CompatDev &d, uint32_t p, uint32_t lane) {
  const RecDev &R = d.R[r];
  const uint32_t n = d.n;
  const uint32_t gb = R.grow ? R.grow[p] : 0, ge = R.grow ? R.grow[p + 1] : 0;
  const uint32_t rb = R.rrow ? R.rrow[p] : 0, re = R.rrow ? R.rrow[p + 1] : 0;
  if (gb == ge && rb == re) return;
  float acc = d.G[(size_t)r * n + p];
  for (uint32_t base = gb; base < ge; base += 32) {
    const uint32_t e = base + lane;
    float t = 0.0f;
    if (e < ge) {
      const uint32_t k = R.ggate[e];
      t = R.gate_st[k] * R.gate_g[k];
    }
    acc = ordered_add(acc, t, min(32u, ge - base));
  }
  if (rb != re) {
    const bool plastic = (d.glob & (FS_ACT_STP | FS_ACT_STD)) != 0;
    const float dfp = d.dfst[(size_t)r * n + p];
    for (uint32_t base = rb; base < re; base += 32) {
      const uint32_t e = base + lane;
      float t = 0.0f;
      if (e < re) {
        const uint32_t pre = R.rpre[e];
        const bool spk = (d.NS[pre] & FS_NS_SPIKE) != 0;
        if (r != FS_NMDA) {
          float st = R.rst[e];
          if (spk) st = plastic ? st + gate_inc(d, pre, false) : st + 1.0f;
          else st = st * dfp;
          t = st * R.rg[e];
          R.rst[e] = st;
        } else {
          float xt = R.rxt[e], st = R.rst[e];
          if (spk) {
            if (d.glob & FS_ACT_STP) xt = xt + d.D[pre] * d.F[pre];
            else if (d.glob & FS_ACT_STD) xt = xt + d.D[pre];
            else xt = xt + 1.0f;
          } else {
            xt = xt * d.nmda_dfxt[p];
          }
          st = dfp * st + d.nmda_efst[p] * d.nmda_as[p] * xt * (1.0f - st);
          t = st * R.rg[e];
          R.rxt[e] = xt;
          R.rst[e] = st;
        }
      }
      acc = ordered_add(acc, t, min(32u, re - base));
    }
  }
  if (lane == 0) d.G[(size_t)r * n + p] = acc;
}

__global__ void __launch_bounds__(256) k_gather(const __grid_constant__ CompatDev d) {
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t p = warp; p < d.n; p += nw) {
    gather_rec<FS_AMPA>(d, p, lane);
    gather_rec<FS_GABA>(d, p, lane);
    gather_rec<FS_ACH>(d, p, lane);
    gather_rec<FS_GCL>(d, p, lane);
    gather_rec<FS_NMDA>(d, p, lane);
    if (d.gap_row) {
      const uint32_t b = d.gap_row[p], e = d.gap_row[p + 1];
      if (b != e) {
        float acc = d.Isyn[p];
        const float vp = d.V[p];
        for (uint32_t base = b; base < e; base += 32) {
          const uint32_t q = base + lane;
          float t = 0.0f;
          if (q < e) t = d.gap_g[q] * (d.V[d.gap_other[q]] - vp);
          acc = ordered_add(acc, t, min(32u, e - base));
        }
        if (lane == 0) d.Isyn[p] = acc;
      }
    }
  }
}

// ---- plasticity ---------------------------------------------------------
__global__ void __launch_bounds__(256) k_stp(const __grid_constant__ CompatDev d) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.n) return;
  const bool spk = (d.NS[i] & FS_NS_SPIKE) != 0;
  if (d.glob & FS_ACT_STP) {
    float Dv = d.D[i], Fv = d.F[i], Cp = d.Cap[i], Cr = d.Car[i];
    if (spk) {
      Cr = Cr + d.stp_aCar[i];
      Cp = Cp + d.stp_aCap[i];
      Fv = Fv + (Cp + Cr) * (1.0f - Fv) * d.stp_aF[i];
      Dv = Dv * (1.0f - d.stp_pv[i] * Fv);
    } else {
      Cr = d.stp_dfCar[i] * Cr + d.stp_efCar[i];
      Cp = d.stp_dfCap[i] * Cp;
      Fv = d.stp_dfF[i] * Fv + d.stp_efF[i] * (Cp + Cr) * (1.0f - Fv) * d.stp_aF[i];
      Dv = d.stp_dfD[i] * Dv + d.stp_efD[i];
    }
    d.D[i] = Dv; d.F[i] = Fv; d.Cap[i] = Cp; d.Car[i] = Cr;
  } else {
    if (spk) d.D[i] = d.D[i] * (1.0f - d.stp_pv[i]);
    else d.D[i] = d.stp_dfD[i] * d.D[i] + d.stp_efD[i];
  }
}

__global__ void __launch_bounds__(256) k_ltp(const __grid_constant__ CompatDev d) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= d.rec_off[FS_NREC]) return;
  int r = 0;
#pragma unroll
  for (int q = 1; q < FS_NREC; q++)
    if (t >= d.rec_off[q]) r = q;
  const RecDev *R;
  switch (r) {
    case 0: R = &d.R[0]; break;
    case 1: R = &d.R[1]; break;
    case 2: R = &d.R[2]; break;
    case 3: R = &d.R[3]; break;
    default: R = &d.R[4]; break;
  }
  const uint32_t e = t - d.rec_off[r];
  const uint32_t pre = R->rpre[e], post = R->rpost[e];
  float g = R->rg[e];
  if (d.NS[pre] & FS_NS_SPIKE) {
    const float ni = d.ltp_Neg[pre];
    if (ni > 0) g = g + d.LP[post] * ni;
    else g = g * (1.0f + d.LP[post] * ni);
  }
  if (d.NS[post] & FS_NS_SPIKE) {
    const float pi = d.ltp_Pos[pre];
    if (pi > 0) g = g + d.LP[pre] * pi;
    else g = g * (1.0f + d.LP[pre] * pi);
  }
  R->rg[e] = g;
}

__global__ void k_gv_snapshot(const __grid_constant__ CompatDev d, uint32_t s) {
  const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= d.gv_n) return;
  const uint32_t code = d.gv_sel[q], r = code >> 28, e = code & 0x0fffffffu;
  const RecDev *R;
  switch (r) {
    case 0: R = &d.R[0]; break;
    case 1: R = &d.R[1]; break;
    case 2: R = &d.R[2]; break;
    case 3: R = &d.R[3]; break;
    default: R = &d.R[4]; break;
  }
  d.gv_st[(size_t)s * d.gv_n + q] = R->rst[e];
  d.gv_xt[(size_t)s * d.gv_n + q] = R->rxt[e];
}

// ---- VarInit (code/EqsGnl2.cpp:339-401) -----------------------------------
// Group gates are not reset here, as in the reference (they are zeroed only
// when the network is built).
__global__ void __launch_bounds__(256) k_varinit(const __grid_constant__ CompatDev d) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t n = d.n;
  if (t < n) {
    const uint32_t i = t, a = d.act[i];
    d.Isyn[i] = 0.0f;
    d.V[i] = -70.0f;
    d.Count[i] = 0;
    d.NS[i] = 0u;
    if (a & FS_ACT_STP) {
      d.D[i] = 1.0f; d.F[i] = 1.0f; d.Cap[i] = 0.0f; d.Car[i] = 20.0f;
    } else if (a & FS_ACT_STD) {
      d.D[i] = 1.0f;
    }
    if (a & FS_ACT_LTP) { d.LP[i] = 0.0f; d.CountLP[i] = 0; }
#pragma unroll
    for (int r = 0; r < FS_NREC; r++) {
      d.G[(size_t)r * n + i] = 0.0f;
      d.Irep[(size_t)r * n + i] = 0.0f;
    }
#pragma unroll
    for (int r = 0; r < 4; r++) d.ext_st[(size_t)r * n + i] = 0.0f;
    d.ext_xt_n[i] = 0.0f;
    d.ext_st_n[i] = 0.0f;
  }
  if (t < d.rec_off[FS_NREC]) {
    int r = 0;
#pragma unroll
    for (int q = 1; q < FS_NREC; q++)
      if (t >= d.rec_off[q]) r = q;
    const RecDev &R = d.R[r];
    const uint32_t e = t - d.rec_off[r];
    R.rst[e] = 0.0f;
    R.rxt[e] = 0.0f;
  }
}

cudaError_t compat_varinit(const CompatDev &d, cudaStream_t st) {
  const uint64_t work = d.n > d.rec_off[FS_NREC] ? d.n : d.rec_off[FS_NREC];
  if (work == 0) return cudaSuccess;
  k_varinit<<<(unsigned)((work + 255) / 256), 256, 0, st>>>(d);
  return cudaGetLastError();
}

// ---- one reference step ---------------------------------------------------
static inline uint32_t blocks_for(uint64_t threads, uint32_t bs) {
  return (uint32_t)((threads + bs - 1) / bs);
}

cudaError_t compat_step(const CompatDev &d, uint32_t s, uint32_t sm_count, cudaStream_t st,
                        uint64_t *launches) {
  const uint32_t bs = 256;
  k_activation<<<blocks_for(((uint64_t)d.n + 31) / 32 * 32, bs), bs, 0, st>>>(d, s);
  uint64_t L = 1;
  if (d.gate_off[FS_NREC]) {
    k_gates<<<blocks_for(d.gate_off[FS_NREC], bs), bs, 0, st>>>(d);
    L++;
  }
  {
    // one warp per post; cap the grid at a few waves of resident blocks
    uint32_t blocks = blocks_for((uint64_t)d.n * 32, bs);
    const uint32_t cap = sm_count * 8;
    if (blocks > cap) blocks = cap;
    k_gather<<<blocks, bs, 0, st>>>(d);
    L++;
  }
  if (d.glob & (FS_ACT_STP | FS_ACT_STD)) {
    k_stp<<<blocks_for(d.n, bs), bs, 0, st>>>(d);
    L++;
  }
  if ((d.glob & FS_ACT_LTP) && d.rec_off[FS_NREC]) {
    k_ltp<<<blocks_for(d.rec_off[FS_NREC], bs), bs, 0, st>>>(d);
    L++;
  }
  if (d.gv_n) {
    k_gv_snapshot<<<blocks_for(d.gv_n, bs), bs, 0, st>>>(d, s);
    L++;
  }
  if (launches) *launches += L;
  return cudaGetLastError();
}

// ---- mt19937 stream -------------------------------------------------------
// The standard MT19937 recurrence (Matsumoto & Nishimura 1998; the
// parameters are those std::mt19937 fixes): x[k+624] = x[k+397] ^ A(x[k], x[k+1]).
// One CTA keeps the 624-word state in shared memory and regenerates it in
// three dependency waves (words 0..226 need only old words, 227..453 need
// wave one, 454..623 need wave two), then tempers and stores the words.
// state[0..623] holds the last untempered block, *pos how many of its words
// were already used.
__device__ __forceinline__ uint32_t mt_twist(uint32_t xi, uint32_t xi1, uint32_t xm) {
  const uint32_t y = (xi & 0x80000000u) | (xi1 & 0x7fffffffu);
  return xm ^ (y >> 1) ^ ((y & 1u) ? 0x9908b0dfu : 0u);
}
__device__ __forceinline__ uint32_t mt_temper(uint32_t y) {
  y ^= (y >> 11);
  y ^= (y << 7) & 0x9d2c5680u;
  y ^= (y << 15) & 0xefc60000u;
  y ^= (y >> 18);
  return y;
}

__global__ void __launch_bounds__(640) k_mt19937(uint32_t *state, uint32_t *pos, uint32_t *out, uint64_t count) {
  __shared__ uint32_t buf[2][624];
  const uint32_t t = threadIdx.x;
  if (t < 624) buf[0][t] = state[t];
  __syncthreads();
  uint32_t p = *pos;
  int cur = 0;
  uint64_t w = 0;
  // words left in the current block
  if (p < 624) {
    const uint64_t take = min((uint64_t)(624 - p), count);
    for (uint64_t k = t; k < take; k += blockDim.x) out[k] = mt_temper(buf[0][p + k]);
    w = take;
    p += (uint32_t)take;
  }
  while (w < count) {
    const uint32_t *o = buf[cur];
    uint32_t *nw = buf[cur ^ 1];
    if (t < 227) nw[t] = mt_twist(o[t], o[t + 1], o[t + 397]);
    __syncthreads();
    if (t >= 227 && t < 454) nw[t] = mt_twist(o[t], o[t + 1], nw[t - 227]);
    __syncthreads();
    if (t >= 454 && t < 623) nw[t] = mt_twist(o[t], o[t + 1], nw[t - 227]);
    if (t == 623) nw[623] = mt_twist(o[623], nw[0], nw[396]);
    __syncthreads();
    cur ^= 1;
    const uint64_t take = min((uint64_t)624, count - w);
    if (t < take) out[w + t] = mt_temper(buf[cur][t]);
    w += take;
    p = (uint32_t)take;
  }
  __syncthreads();
  if (t < 624) state[t] = buf[cur][t];
  if (t == 0) *pos = p;
}

cudaError_t mt_generate(uint32_t *state, uint32_t *pos, uint32_t *out, uint64_t count, cudaStream_t st) {
  if (count == 0) return cudaSuccess;
  k_mt19937<<<1, 640, 0, st>>>(state, pos, out, count);
  return cudaGetLastError();
}

// ---- ordered spike compaction ----------------------------------------------
// bits[s][w] are the warp ballots of step s.  k_count: one block per step sums
// the population counts.  k_write: one block per step computes a block-wide
// exclusive prefix of per-word counts and writes ascending neuron ids.
__global__ void __launch_bounds__(256) k_count(const uint32_t *bits, uint32_t words, uint32_t *counts) {
  const uint32_t s = blockIdx.x;
  uint32_t c = 0;
  for (uint32_t w = threadIdx.x; w < words; w += blockDim.x) c += __popc(bits[(size_t)s * words + w]);
  for (int o = 16; o; o >>= 1) c += __shfl_down_sync(kFull, c, o);
  __shared__ uint32_t part[8];
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = c;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t tot = 0;
    for (int k = 0; k < 8; k++) tot += part[k];
    counts[s] = tot;
  }
}
__global__ void k_scan_counts(const uint32_t *counts, uint32_t nsteps, uint32_t *offsets) {
  // single block, sequential over chunks of 1024
  __shared__ uint32_t sh[1024];
  __shared__ uint32_t carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (uint32_t base = 0; base < nsteps; base += 1024) {
    const uint32_t i = base + threadIdx.x;
    const uint32_t v = (i < nsteps) ? counts[i] : 0;
    sh[threadIdx.x] = v;
    __syncthreads();
    for (uint32_t o = 1; o < 1024; o <<= 1) {
      const uint32_t a = (threadIdx.x >= o) ? sh[threadIdx.x - o] : 0;
      __syncthreads();
      sh[threadIdx.x] += a;
      __syncthreads();
    }
    if (i < nsteps) offsets[i] = carry + sh[threadIdx.x] - v;
    __syncthreads();
    if (threadIdx.x == 1023) carry += sh[1023];
    __syncthreads();
  }
  if (threadIdx.x == 0) offsets[nsteps] = carry;
}
__global__ void __launch_bounds__(256) k_write(const uint32_t *bits, uint32_t words, const uint32_t *offsets,
                                               uint32_t *idx) {
  const uint32_t s = blockIdx.x;
  __shared__ uint32_t warp_tot[8];
  __shared__ uint32_t run;
  if (threadIdx.x == 0) run = offsets[s];
  __syncthreads();
  const uint32_t lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (uint32_t base = 0; base < words; base += blockDim.x) {
    const uint32_t w = base + threadIdx.x;
    const uint32_t b = (w < words) ? bits[(size_t)s * words + w] : 0u;
    const uint32_t c = __popc(b);
    // warp inclusive scan of c
    uint32_t x = c;
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(kFull, x, o);
      if (lane >= (uint32_t)o) x += y;
    }
    if (lane == 31) warp_tot[wid] = x;
    __syncthreads();
    uint32_t before = 0;
    for (uint32_t k = 0; k < wid; k++) before += warp_tot[k];
    uint32_t o0 = run + before + x - c;
    uint32_t bb = b;
    while (bb) {
      const int bit = __ffs(bb) - 1;
      idx[o0++] = w * 32u + (uint32_t)bit;
      bb &= bb - 1;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      uint32_t tot = 0;
      for (int k = 0; k < 8; k++) tot += warp_tot[k];
      run += tot;
    }
    __syncthreads();
  }
}

cudaError_t spikes_compact(const uint32_t *bits, uint32_t nsteps, uint32_t words, uint32_t *counts,
                           uint32_t *offsets, uint32_t *idx, cudaStream_t st, uint64_t *launches) {
  if (nsteps == 0) return cudaSuccess;
  k_count<<<nsteps, 256, 0, st>>>(bits, words, counts);
  k_scan_counts<<<1, 1024, 0, st>>>(counts, nsteps, offsets);
  k_write<<<nsteps, 256, 0, st>>>(bits, words, offsets, idx);
  if (launches) *launches += 3;
  return cudaGetLastError();
}

void compat_set_tables(const uint32_t kn[128], const float fn[128], const float wn[128],
                       const uint32_t jump_a[32], const uint32_t jump_c[32], cudaStream_t st) {
  cudaMemcpyToSymbolAsync(c_kn, kn, sizeof(uint32_t) * 128, 0, cudaMemcpyHostToDevice, st);
  cudaMemcpyToSymbolAsync(c_fn, fn, sizeof(float) * 128, 0, cudaMemcpyHostToDevice, st);
  cudaMemcpyToSymbolAsync(c_wn, wn, sizeof(float) * 128, 0, cudaMemcpyHostToDevice, st);
  cudaMemcpyToSymbolAsync(c_jump_a, jump_a, sizeof(uint32_t) * 32, 0, cudaMemcpyHostToDevice, st);
  cudaMemcpyToSymbolAsync(c_jump_c, jump_c, sizeof(uint32_t) * 32, 0, cudaMemcpyHostToDevice, st);
}

// test hook: the device expf used by the NMDA Mg block
__global__ void k_expf_eval(const float *x, float *y, uint64_t k, const uint32_t *keys, const float *vals,
                            uint32_t nk) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= k) return;
  CompatDev d{};
  d.expf_keys = keys;
  d.expf_vals = vals;
  d.expf_n = nk;
  y[i] = expf_ref(x[i], d);
}
cudaError_t expf_ref_eval(const float *x, float *y, uint64_t k, const uint32_t *keys, const float *vals,
                          uint32_t nk, cudaStream_t st) {
  if (k == 0) return cudaSuccess;
  k_expf_eval<<<(unsigned)((k + 255) / 256), 256, 0, st>>>(x, y, k, keys, vals, nk);
  return cudaGetLastError();
}

}  // namespace fsd
