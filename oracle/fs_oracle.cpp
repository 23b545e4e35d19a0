// ORACLE — test infrastructure only.  Nothing in the product links, loads or
// runs this file; only tests/, __graft_entry__.smoke() and bench.py's
// cpu_baseline leg use it, as what the engine's results are compared with.
//
// A CPU restatement of the reference's per-step integration, one step at a
// time in the reference's own order and FP32 arithmetic, over the structure of
// arrays of fs_net_desc.  Each function names the reference code it follows.
// Parity is pinned by tests/test_oracle_ref.py, which runs this oracle and
// the reference compiled from its own sources (oracle/Makefile.ref) on the
// same .conf/.pro files and requires byte-identical output files.
//
// Third-party algorithms used as the reference uses them (GCC 13.3.0
// libstdc++, glibc 2.39 libm):
//   std::mt19937 + std::uniform_real_distribution<float> — the drive draws
//     (code/EqsGnl2.cpp:290-326);
//   Marsaglia–Tsang ziggurat as written by J. Burkardt (r4_nor/r4_nor_setup),
//     restated from the algorithm description (code/StiExt.h:214-351).
#include <cmath>
#include <cstdint>
#include <cstring>
#include <random>
#include <string>
#include <vector>
#include "flysim_b200.h"

namespace {

struct Ziggurat {  // code/StiExt.h:191-351
  uint32_t kn[128];
  float fn[128], wn[128];
  uint32_t jcong = 0;
  Ziggurat() { setup(); }
  void setup() {
    double dn = 3.442619855899, tn = dn;
    const double m1 = 2147483648.0, vn = 9.91256303526217E-03;
    double q = vn / std::exp(-0.5 * dn * dn);
    kn[0] = (uint32_t)((dn / q) * m1);
    kn[1] = 0;
    wn[0] = (float)(q / m1);
    wn[127] = (float)(dn / m1);
    fn[0] = 1.0f;
    fn[127] = (float)std::exp(-0.5 * dn * dn);
    for (int i = 126; 1 <= i; i--) {
      dn = std::sqrt(-2.0 * std::log(vn / dn + std::exp(-0.5 * dn * dn)));
      kn[i + 1] = (uint32_t)((dn / tn) * m1);
      tn = dn;
      fn[i] = (float)std::exp(-0.5 * dn * dn);
      wn[i] = (float)(dn / m1);
    }
  }
  static uint32_t shr3(uint32_t &jsr) {
    uint32_t in = jsr;
    jsr = jsr ^ (jsr << 13);
    jsr = jsr ^ (jsr >> 17);
    jsr = jsr ^ (jsr << 5);
    return in + jsr;
  }
  static float uni(uint32_t &jsr) {
    uint32_t in = jsr;
    jsr = jsr ^ (jsr << 13);
    jsr = jsr ^ (jsr >> 17);
    jsr = jsr ^ (jsr << 5);
    return (float)std::fmod(0.5 + (float)(in + jsr) / 65536.0 / 65536.0, 1.0);
  }
  float nor(uint32_t &jsr) const {
    const float r = 3.442620f;
    int hz = (int)shr3(jsr);
    uint32_t iz = (uint32_t)(hz & 127);
    float value, x, y;
    if (std::fabs((double)hz) < kn[iz]) return (float)hz * wn[iz];
    for (;;) {
      if (iz == 0) {
        for (;;) {
          // log of a float argument is logf here (std::log(float) overload)
          x = (float)(-0.2904764 * std::log(uni(jsr)));
          y = -std::log(uni(jsr));
          if (x * x <= y + y) break;
        }
        value = (hz <= 0) ? -r - x : r + x;
        break;
      }
      x = (float)hz * wn[iz];
      if (fn[iz] + uni(jsr) * (fn[iz - 1] - fn[iz]) < std::exp(-0.5 * x * x)) {
        value = x;
        break;
      }
      hz = (int)shr3(jsr);
      iz = (uint32_t)(hz & 127);
      if (std::fabs((double)hz) < kn[iz]) {
        value = (float)hz * wn[iz];
        break;
      }
    }
    return value;
  }
  float gauss(float mean, float sd) {  // Igauss: one congruential step per draw
    jcong = 69069u * jcong + 1234567u;
    uint32_t jsr = jcong;
    return mean + sd * nor(jsr);
  }
};

struct Oracle {
  uint32_t n = 0;
  float dt = 0.1f;
  uint32_t glob = 0;  // global ActCtr (STP/STD/LTP mode)
  // parameters
  std::vector<float> Vth, El, gl, Cm, Vreset, df, ef, dVmax, Vrev, dfst, nmda_dfxt, nmda_efst,
      nmda_as, nmda_mg, ext_g, pb, inj_mean, inj_std;
  std::vector<int32_t> RfPed, SpiDy;
  std::vector<uint32_t> act;
  std::vector<float> stp[11];
  std::vector<float> ltp_dfLP, ltp_Pos, ltp_Neg;
  std::vector<int32_t> ltp_SpiLPDy;
  // synapses
  struct Rec {
    std::vector<uint32_t> gate_pre, gate_post0, grow, ggate, rpre, rpost, rrow;
    std::vector<float> gate_g, gate_st, gate_xt, rg, rst, rxt;
  } R[FS_NREC];
  std::vector<uint32_t> gap_row, gap_other;
  std::vector<float> gap_g;
  // state
  std::vector<float> V, Isyn, G, ext_st, ext_xt_n, ext_st_n, Irep, D, F, Cap, Car, LP;
  std::vector<int32_t> Count, CountLP;
  std::vector<uint32_t> NS;
  std::mt19937 mt;
  std::uniform_real_distribution<float> uni{0.0f, 1.0f};
  Ziggurat zig;
  std::string err;
};

template <class T>
std::vector<T> vec(const T *p, size_t k) {
  return p ? std::vector<T>(p, p + k) : std::vector<T>(k, T());
}

// EqsGnl2::firing (code/EqsGnl2.cpp:229-251)
void firing(Oracle &o, uint32_t i) {
  if (o.Count[i] < o.RfPed[i]) {
    o.V[i] = (o.Count[i] == 0) ? 0.0f : o.Vreset[i];
    if (o.Count[i] == o.SpiDy[i]) o.NS[i] |= FS_NS_SPIKE;
    else o.NS[i] &= ~FS_NS_SPIKE;
    o.Count[i]++;
  } else {
    o.Count[i] = 0;
    o.NS[i] &= ~FS_NS_FIRE;
  }
}

// EqsGnl2::BgInit (code/EqsGnl2.cpp:284-337)
void bg_init(Oracle &o, uint32_t i) {
  const uint32_t n = o.n, a = o.act[i];
  const uint32_t bits[4] = {FS_ACT_AMPA, FS_ACT_GABA, FS_ACT_ACH, FS_ACT_GCL};
  for (int r = 0; r < 4; r++) {
    if (!(a & bits[r])) continue;
    float &st = o.ext_st[(size_t)r * n + i];
    if (o.pb[(size_t)r * n + i] > o.uni(o.mt)) st++;
    else st *= o.dfst[(size_t)r * n + i];
    o.G[(size_t)r * n + i] += o.ext_g[(size_t)r * n + i] * st;
  }
  if (a & FS_ACT_NMDA) {
    float &xt = o.ext_xt_n[i], &st = o.ext_st_n[i];
    if (o.pb[(size_t)FS_NMDA * n + i] > o.uni(o.mt)) xt++;
    else xt *= o.nmda_dfxt[i];
    st = o.dfst[(size_t)FS_NMDA * n + i] * st + o.nmda_efst[i] * o.nmda_as[i] * xt * (1.0f - st);
    o.G[(size_t)FS_NMDA * n + i] += o.ext_g[(size_t)FS_NMDA * n + i] * st;
  }
  if (a & FS_ACT_INJ) o.Isyn[i] += o.zig.gauss(o.inj_mean[i], o.inj_std[i]);
}

// EqsGnl2::VmEul (code/EqsGnl2.cpp:152-225) with firLP/ltpEul (:254-280)
void vm_eul(Oracle &o, uint32_t i) {
  const uint32_t n = o.n;
  if (o.NS[i] & FS_NS_FIRE) {
    firing(o, i);
  } else {
    const float v = o.V[i];
    float Ir[5];
    Ir[0] = o.G[(size_t)FS_AMPA * n + i] * (o.Vrev[(size_t)FS_AMPA * n + i] - v);
    Ir[1] = o.G[(size_t)FS_GABA * n + i] * (o.Vrev[(size_t)FS_GABA * n + i] - v);
    Ir[2] = o.G[(size_t)FS_NMDA * n + i] * (o.Vrev[(size_t)FS_NMDA * n + i] - v) /
            (1.0f + o.nmda_mg[i] * (float)std::exp(-0.062f * v) / 3.57f);
    Ir[3] = o.G[(size_t)FS_ACH * n + i] * (o.Vrev[(size_t)FS_ACH * n + i] - v);
    Ir[4] = o.G[(size_t)FS_GCL * n + i] * (o.Vrev[(size_t)FS_GCL * n + i] - v);
    float I = Ir[0] + Ir[1] + Ir[2] + Ir[3] + Ir[4] + o.Isyn[i] * 1e3f + o.gl[i] * o.El[i] * 1e3f;
    I = 1e-3f * I / o.Cm[i];
    if (I > o.dVmax[i]) {
      I = o.dVmax[i];
      o.NS[i] |= FS_NS_MEMDV_OVF;
      o.NS[i] &= ~FS_NS_MEMDV_UDF;
    } else if (I < -o.dVmax[i]) {
      I = -o.dVmax[i];
      o.NS[i] &= ~FS_NS_MEMDV_OVF;
      o.NS[i] |= FS_NS_MEMDV_UDF;
    } else {
      o.NS[i] &= ~(FS_NS_MEMDV_OVF | FS_NS_MEMDV_UDF);
    }
    o.V[i] = o.df[i] * v + o.ef[i] * I;
    // Irep is stored receptor-major in the reference's order AMPA, GABA, NMDA, ACH, GCL
    for (int r = 0; r < 5; r++) o.Irep[(size_t)r * n + i] = Ir[r];
    if (o.V[i] > o.Vth[i]) {
      o.NS[i] |= FS_NS_FIRE;
      firing(o, i);
      if (o.act[i] & FS_ACT_LTP) o.NS[i] |= FS_NS_LP_FIRE;
    }
  }
  if (o.act[i] & FS_ACT_LTP) {
    // firLP
    if (o.NS[i] & FS_NS_LP_FIRE) {
      if (o.CountLP[i] == o.ltp_SpiLPDy[i]) {
        o.NS[i] |= FS_NS_LP_SPIKE;
        o.NS[i] &= ~FS_NS_LP_FIRE;
        o.CountLP[i] = 0;
      } else {
        o.NS[i] &= ~FS_NS_LP_SPIKE;
        o.CountLP[i]++;
      }
    } else {
      o.NS[i] &= ~FS_NS_LP_SPIKE;
    }
    // ltpEul
    if (o.NS[i] & FS_NS_LP_SPIKE) o.LP[i]++;
    else o.LP[i] = o.ltp_dfLP[i] * o.LP[i];
  }
  for (int r = 0; r < FS_NREC; r++) o.G[(size_t)r * n + i] = 0.0f;
  o.Isyn[i] = 0.0f;
}

inline bool spk(const Oracle &o, uint32_t i) { return (o.NS[i] & FS_NS_SPIKE) != 0; }

// increment of a gate on a presynaptic spike (ThdPGatVar/STD/STP and
// ThdSynapse/STD/STP): 1, D, or D*F
inline float inc(const Oracle &o, uint32_t pre, bool nmda) {
  if (o.glob & FS_ACT_STP) return o.D[pre] * o.F[pre];
  if (o.glob & FS_ACT_STD) return nmda ? o.D[pre] * o.F[pre] : o.D[pre];
  return 1.0f;
}

// EqsGnl2::Spike (code/EqsGnl2.cpp:1107-1131)
void spike_phase(Oracle &o) {
  const uint32_t n = o.n;
  const bool plastic = (o.glob & (FS_ACT_STP | FS_ACT_STD)) != 0;
  // gate updates (ThdPGatVar*, code/EqsGnl2.cpp:728-932)
  for (int r = 0; r < FS_NREC; r++) {
    Oracle::Rec &R = o.R[r];
    const bool nmda = (r == FS_NMDA);
    for (size_t k = 0; k < R.gate_pre.size(); k++) {
      const uint32_t pre = R.gate_pre[k], p0 = R.gate_post0[k];
      if (!nmda) {
        if (spk(o, pre)) {
          if (plastic) R.gate_st[k] += inc(o, pre, false);
          else R.gate_st[k]++;
        } else {
          R.gate_st[k] *= o.dfst[(size_t)r * n + p0];
        }
      } else {
        if (spk(o, pre)) {
          if (plastic) R.gate_xt[k] += inc(o, pre, true);
          else R.gate_xt[k]++;
        } else {
          R.gate_xt[k] *= o.nmda_dfxt[p0];
        }
        R.gate_st[k] = o.dfst[(size_t)FS_NMDA * n + p0] * R.gate_st[k] +
                       o.nmda_efst[p0] * o.nmda_as[p0] * R.gate_xt[k] * (1.0f - R.gate_st[k]);
      }
    }
  }
  // group gather (ThdPSynapse, code/EqsGnl2.cpp:941-979); RVs is 0 here
  for (int r = 0; r < FS_NREC; r++) {
    Oracle::Rec &R = o.R[r];
    for (uint32_t p = 0; p < n; p++) {
      if (R.grow[p] == R.grow[p + 1]) continue;
      float g = o.G[(size_t)r * n + p];
      for (uint32_t e = R.grow[p]; e < R.grow[p + 1]; e++) {
        const uint32_t k = R.ggate[e];
        g += R.gate_st[k] * R.gate_g[k];
      }
      o.G[(size_t)r * n + p] = g;
    }
  }
  // single-target records (ThdSynapse*, code/EqsGnl2.cpp:404-703)
  const int order[5] = {FS_AMPA, FS_GABA, FS_ACH, FS_GCL, FS_NMDA};
  for (int oi = 0; oi < 5; oi++) {
    const int r = order[oi];
    Oracle::Rec &R = o.R[r];
    const bool nmda = (r == FS_NMDA);
    for (uint32_t p = 0; p < n; p++) {
      if (R.rrow[p] == R.rrow[p + 1]) continue;
      float g = o.G[(size_t)r * n + p];
      for (uint32_t e = R.rrow[p]; e < R.rrow[p + 1]; e++) {
        const uint32_t pre = R.rpre[e];
        if (!nmda) {
          float st = R.rst[e];
          if (spk(o, pre)) {
            if (plastic) st += inc(o, pre, false);
            else st++;
          } else {
            st *= o.dfst[(size_t)r * n + p];
          }
          g += st * R.rg[e];
          R.rst[e] = st;
        } else {
          float xt = R.rxt[e], st = R.rst[e];
          if (spk(o, pre)) {
            if (o.glob & FS_ACT_STP) xt += o.D[pre] * o.F[pre];
            else if (o.glob & FS_ACT_STD) xt += o.D[pre];
            else xt++;
          } else {
            xt *= o.nmda_dfxt[p];
          }
          st = o.dfst[(size_t)FS_NMDA * n + p] * st + o.nmda_efst[p] * o.nmda_as[p] * xt * (1.0f - st);
          g += st * R.rg[e];
          R.rxt[e] = xt;
          R.rst[e] = st;
        }
      }
      o.G[(size_t)r * n + p] = g;
    }
  }
  // gap junctions (code/EqsGnl2.cpp:982-999 and ThdGapSyn :705-724)
  if (!o.gap_row.empty()) {
    for (uint32_t p = 0; p < n; p++) {
      if (o.gap_row[p] == o.gap_row[p + 1]) continue;
      float acc = o.Isyn[p];
      const float vp = o.V[p];
      for (uint32_t e = o.gap_row[p]; e < o.gap_row[p + 1]; e++)
        acc += o.gap_g[e] * (o.V[o.gap_other[e]] - vp);
      o.Isyn[p] = acc;
    }
  }
  // STP / STD (code/EqsGnl2.cpp:1048-1090)
  if (o.glob & FS_ACT_STP) {
    for (uint32_t i = 0; i < n; i++) {
      float Dv = o.D[i], Fv = o.F[i], Cp = o.Cap[i], Cr = o.Car[i];
      if (spk(o, i)) {
        Cr += o.stp[8][i];
        Cp += o.stp[6][i];
        Fv += (Cp + Cr) * (1.0f - Fv) * o.stp[3][i];
        Dv *= (1.0f - o.stp[0][i] * Fv);
      } else {
        Cr = o.stp[9][i] * Cr + o.stp[10][i];
        Cp = o.stp[7][i] * Cp;
        Fv = o.stp[4][i] * Fv + o.stp[5][i] * (Cp + Cr) * (1.0f - Fv) * o.stp[3][i];
        Dv = o.stp[1][i] * Dv + o.stp[2][i];
      }
      o.D[i] = Dv; o.F[i] = Fv; o.Cap[i] = Cp; o.Car[i] = Cr;
    }
  } else if (o.glob & FS_ACT_STD) {
    for (uint32_t i = 0; i < n; i++) {
      if (spk(o, i)) o.D[i] *= (1.0f - o.stp[0][i]);
      else o.D[i] = o.stp[1][i] * o.D[i] + o.stp[2][i];
    }
  }
  // LTP on single-target records (code/EqsGnl2.cpp:1005-1044)
  if (o.glob & FS_ACT_LTP) {
    for (int oi = 0; oi < 5; oi++) {
      Oracle::Rec &R = o.R[order[oi]];
      for (size_t e = 0; e < R.rpre.size(); e++) {
        const uint32_t pre = R.rpre[e], post = R.rpost[e];
        if (spk(o, pre)) {
          if (o.ltp_Neg[pre] > 0) R.rg[e] += o.LP[post] * o.ltp_Neg[pre];
          else R.rg[e] *= (1.0f + o.LP[post] * o.ltp_Neg[pre]);
        }
        if (spk(o, post)) {
          if (o.ltp_Pos[pre] > 0) R.rg[e] += o.LP[pre] * o.ltp_Pos[pre];
          else R.rg[e] *= (1.0f + o.LP[pre] * o.ltp_Pos[pre]);
        }
      }
    }
  }
}

// ---- engine table ----
int o_reset(void *ctx, uint32_t mt_seed, uint32_t jcong_seed) {
  Oracle &o = *(Oracle *)ctx;
  const uint32_t n = o.n;
  // VarInit (code/EqsGnl2.cpp:339-401)
  std::fill(o.Isyn.begin(), o.Isyn.end(), 0.0f);
  std::fill(o.V.begin(), o.V.end(), -70.0f);
  std::fill(o.Count.begin(), o.Count.end(), 0);
  std::fill(o.NS.begin(), o.NS.end(), 0u);
  for (uint32_t i = 0; i < n; i++) {
    if (o.act[i] & FS_ACT_STP) {
      o.D[i] = 1.0f; o.F[i] = 1.0f; o.Cap[i] = 0.0f; o.Car[i] = 20.0f;
    } else if (o.act[i] & FS_ACT_STD) {
      o.D[i] = 1.0f;  // F keeps its value: never initialised by the reference, 0 here
    }
    if (o.act[i] & FS_ACT_LTP) { o.LP[i] = 0.0f; o.CountLP[i] = 0; }
  }
  std::fill(o.G.begin(), o.G.end(), 0.0f);
  std::fill(o.Irep.begin(), o.Irep.end(), 0.0f);
  std::fill(o.ext_st.begin(), o.ext_st.end(), 0.0f);
  std::fill(o.ext_xt_n.begin(), o.ext_xt_n.end(), 0.0f);
  std::fill(o.ext_st_n.begin(), o.ext_st_n.end(), 0.0f);
  for (int r = 0; r < FS_NREC; r++) {
    // group gates are reset only by SetPp, not by VarInit (code/NetSimGnl2_BulPp.cpp:404,460-461)
    std::fill(o.R[r].rst.begin(), o.R[r].rst.end(), 0.0f);
    std::fill(o.R[r].rxt.begin(), o.R[r].rxt.end(), 0.0f);
  }
  o.mt.seed(mt_seed);
  o.uni.reset();
  o.zig.jcong = jcong_seed;
  return FS_OK;
}
int o_set_drive(void *ctx, uint32_t first, uint32_t count, int rec, float pb) {
  Oracle &o = *(Oracle *)ctx;
  if (rec < 0 || rec >= FS_NREC || (uint64_t)first + count > o.n) return FS_ERR_ARG;
  for (uint32_t i = first; i < first + count; i++) o.pb[(size_t)rec * o.n + i] = pb;
  return FS_OK;
}
int o_set_act(void *ctx, uint32_t first, uint32_t count, uint32_t clr, uint32_t set) {
  Oracle &o = *(Oracle *)ctx;
  if ((uint64_t)first + count > o.n) return FS_ERR_ARG;
  for (uint32_t i = first; i < first + count; i++) o.act[i] = (o.act[i] & ~clr) | set;
  return FS_OK;
}
int o_set_inj(void *ctx, uint32_t first, uint32_t count, float mean, float sd) {
  Oracle &o = *(Oracle *)ctx;
  if ((uint64_t)first + count > o.n) return FS_ERR_ARG;
  for (uint32_t i = first; i < first + count; i++) { o.inj_mean[i] = mean; o.inj_std[i] = sd; }
  return FS_OK;
}
int o_step(void *ctx, uint32_t nsteps, fs_step_out *out) {
  Oracle &o = *(Oracle *)ctx;
  const uint32_t n = o.n;
  uint64_t w = 0;
  for (uint32_t s = 0; s < nsteps; s++) {
    // Activation (code/EqsGnl2.cpp:1098-1105)
    for (uint32_t i = 0; i < n; i++) {
      bg_init(o, i);
      vm_eul(o, i);
    }
    spike_phase(o);
    if (out) {
      uint32_t c = 0;
      for (uint32_t i = 0; i < n; i++)
        if (spk(o, i)) {
          if (out->spike_idx) {
            if (w >= out->spike_cap) { o.err = "spike buffer too small"; return FS_ERR_CAPACITY; }
            out->spike_idx[w] = i;
          }
          w++;
          c++;
        }
      if (out->spike_count) out->spike_count[s] = c;
      if (out->V) std::memcpy(out->V + (size_t)s * n, o.V.data(), n * sizeof(float));
      if (out->Irep)
        std::memcpy(out->Irep + (size_t)s * FS_NREC * n, o.Irep.data(), (size_t)FS_NREC * n * sizeof(float));
      if (out->nstate) std::memcpy(out->nstate + (size_t)s * n, o.NS.data(), n * sizeof(uint32_t));
      for (uint32_t q = 0; q < out->gv_n; q++) {
        const uint32_t r = out->gv_sel[q] >> 28, e = out->gv_sel[q] & 0x0fffffffu;
        if (r >= FS_NREC || e >= o.R[r].rst.size()) { o.err = "bad record selection"; return FS_ERR_ARG; }
        if (out->gv_st) out->gv_st[(size_t)s * out->gv_n + q] = o.R[r].rst[e];
        if (out->gv_xt) out->gv_xt[(size_t)s * out->gv_n + q] = o.R[r].rxt[e];
      }
    }
  }
  if (out) out->spike_total = w;
  return FS_OK;
}
const char *o_error(void *ctx) { return ctx ? ((Oracle *)ctx)->err.c_str() : "no oracle"; }

const fs_engine_vtbl kOracleEngine = {o_reset, o_set_drive, o_set_act, o_set_inj, o_step, o_error};

}  // namespace

extern "C" {

const fs_engine_vtbl *oracle_engine(void) { return &kOracleEngine; }

void *oracle_create(const fs_net_desc *d) {
  if (!d || !d->compat) return nullptr;
  Oracle *o = new Oracle();
  const fs_neurons &nv = d->neurons;
  const uint32_t n = nv.n;
  o->n = n;
  o->dt = d->dt;
  o->glob = d->act_ctr;
  const size_t nr = (size_t)FS_NREC * n;
  o->Vth = vec(nv.Vth, n); o->El = vec(nv.El, n); o->gl = vec(nv.gl, n); o->Cm = vec(nv.Cm, n);
  o->Vreset = vec(nv.Vreset, n); o->df = vec(nv.df, n); o->ef = vec(nv.ef, n); o->dVmax = vec(nv.dVmax, n);
  o->RfPed = vec(nv.RfPed, n); o->SpiDy = vec(nv.SpiDy, n);
  o->Vrev = vec(nv.Vrev, nr); o->dfst = vec(nv.dfst, nr);
  o->nmda_dfxt = vec(nv.nmda_dfxt, n); o->nmda_efst = vec(nv.nmda_efst, n);
  o->nmda_as = vec(nv.nmda_as, n); o->nmda_mg = vec(nv.nmda_mg, n);
  o->ext_g = vec(nv.ext_g, nr); o->pb = vec(nv.pb, nr); o->act = vec(nv.act, n);
  o->inj_mean = vec(nv.inj_mean, n); o->inj_std = vec(nv.inj_std, n);
  const float *sp[11] = {nv.stp_pv, nv.stp_dfD, nv.stp_efD, nv.stp_aF, nv.stp_dfF, nv.stp_efF,
                         nv.stp_aCap, nv.stp_dfCap, nv.stp_aCar, nv.stp_dfCar, nv.stp_efCar};
  for (int k = 0; k < 11; k++) o->stp[k] = vec(sp[k], n);
  o->ltp_dfLP = vec(nv.ltp_dfLP, n); o->ltp_Pos = vec(nv.ltp_PosISI, n);
  o->ltp_Neg = vec(nv.ltp_NegISI, n); o->ltp_SpiLPDy = vec(nv.ltp_SpiLPDy, n);
  for (int r = 0; r < FS_NREC; r++) {
    const fs_rec_layout &L = d->compat->rec[r];
    Oracle::Rec &R = o->R[r];
    R.gate_pre = vec(L.gate_pre, L.n_gates);
    R.gate_post0 = vec(L.gate_post0, L.n_gates);
    R.gate_g = vec(L.gate_g, L.n_gates);
    R.gate_st.assign(L.n_gates, 0.0f);
    R.gate_xt.assign(L.n_gates, 0.0f);
    R.grow = vec(L.gather_rowptr, (size_t)n + 1);
    R.ggate = vec(L.gather_gate, R.grow[n]);
    R.rpre = vec(L.rec_pre, L.n_recs);
    R.rpost = vec(L.rec_post, L.n_recs);
    R.rg = vec(L.rec_g, L.n_recs);
    R.rst.assign(L.n_recs, 0.0f);
    R.rxt.assign(L.n_recs, 0.0f);
    R.rrow = vec(L.rec_rowptr, (size_t)n + 1);
  }
  if (d->compat->gap_rowptr) {
    o->gap_row = vec(d->compat->gap_rowptr, (size_t)n + 1);
    o->gap_other = vec(d->compat->gap_other, o->gap_row[n]);
    o->gap_g = vec(d->compat->gap_g, o->gap_row[n]);
  }
  o->V.assign(n, -70.0f); o->Isyn.assign(n, 0.0f); o->G.assign(nr, 0.0f);
  o->ext_st.assign((size_t)4 * n, 0.0f); o->ext_xt_n.assign(n, 0.0f); o->ext_st_n.assign(n, 0.0f);
  o->Irep.assign(nr, 0.0f);
  o->D.assign(n, 0.0f); o->F.assign(n, 0.0f); o->Cap.assign(n, 0.0f); o->Car.assign(n, 0.0f);
  o->LP.assign(n, 0.0f); o->Count.assign(n, 0); o->CountLP.assign(n, 0); o->NS.assign(n, 0u);
  return o;
}

void oracle_destroy(void *o) { delete (Oracle *)o; }

// state views for element-wise checks
int oracle_get_state(void *ctx, float *V, int32_t *Count, uint32_t *NState, float *G, float *Isyn) {
  Oracle &o = *(Oracle *)ctx;
  if (V) std::memcpy(V, o.V.data(), o.n * sizeof(float));
  if (Count) std::memcpy(Count, o.Count.data(), o.n * sizeof(int32_t));
  if (NState) std::memcpy(NState, o.NS.data(), o.n * sizeof(uint32_t));
  if (G) std::memcpy(G, o.G.data(), (size_t)FS_NREC * o.n * sizeof(float));
  if (Isyn) std::memcpy(Isyn, o.Isyn.data(), o.n * sizeof(float));
  return 0;
}

// glibc expf, for the device-exp checks
void oracle_expf(const float *x, float *y, uint64_t k) {
  for (uint64_t i = 0; i < k; i++) y[i] = std::exp(x[i]);
}

}  // extern "C"
