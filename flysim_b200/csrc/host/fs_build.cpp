// Network construction for the flysim drop-in: the work of
// NetSimGnl2::SetPp / PostSetPp (code/NetSimGnl2_BulPp.cpp:27-727) done again
// from the parsed model, producing structure-of-arrays buffers for the device
// engine.
//
// Bit-exact connectivity needs the reference's random draws: the set-up
// generator is std::mt19937 seeded with rseeds[0]; the post-synaptic target
// sets come from std::shuffle over the whole target population followed by
// std::sort of the first k entries (code/NetSim.h:431-454, PosBuild) or the
// first entry only (code/NetSim.h:403-429, PosBuild1).  Both calls go to the
// same libstdc++ here, so the draws, and the order std::sort leaves equal keys
// in, are those of the reference built with the same toolchain.
#include <cmath>
#include <climits>
#include <algorithm>
#include <numeric>
#include "fs_host.hpp"

namespace fsh {
namespace {

uint16_t act_of(uint8_t kw) {  // Parser::GetAct (code/parser.cpp:1467-1485)
  switch (kw) {
    case KW_AMPA: return FS_ACT_AMPA;
    case KW_GABA: return FS_ACT_GABA;
    case KW_NMDA: return FS_ACT_NMDA;
    case KW_GAP: return FS_ACT_GAP;
    case KW_CUBA: return 16;
    case KW_ACH: return FS_ACT_ACH;
    case KW_GCL: return FS_ACT_GCL;
    default: return 0;
  }
}
int rec_of_act(uint16_t act) {
  switch (act) {
    case FS_ACT_AMPA: return FS_AMPA;
    case FS_ACT_GABA: return FS_GABA;
    case FS_ACT_ACH: return FS_ACH;
    case FS_ACT_GCL: return FS_GCL;
    case FS_ACT_NMDA: return FS_NMDA;
    default: return -1;
  }
}

struct SynIdx { uint32_t pre, post; };
struct SynRec { uint32_t pre, post; float g; };

// Segments of equal post id in a post-sorted array (BulBiasDNeuMap,
// code/Eqs.h:1120-1165): returns [beg, end] pairs.
template <class T>
std::vector<std::pair<uint32_t, uint32_t>> segments(const std::vector<T> &a) {
  std::vector<std::pair<uint32_t, uint32_t>> s;
  if (a.empty()) return s;
  uint32_t beg = 0;
  for (uint32_t i = 1; i <= a.size(); i++) {
    if (i == a.size() || a[i].post != a[beg].post) {
      s.emplace_back(beg, i - 1);
      beg = i;
    }
  }
  return s;
}

// target set of one (presynaptic neuron, link): PosBuild
std::vector<uint32_t> pos_build(std::mt19937 &rng, uint32_t j, uint32_t k, uint32_t first,
                                uint32_t num, bool selcon) {
  std::vector<uint32_t> ary(num);
  bool self = false;
  const uint32_t js = j - first;
  for (uint32_t q = 0; q < num; q++) {
    ary[q] = first + q;
    if (js == q && !selcon) self = true;
  }
  if (self) ary.erase(ary.begin() + js);
  std::shuffle(ary.begin(), ary.end(), rng);
  if (k > ary.size()) throw ParseError("internal: more targets than candidates");
  std::sort(ary.begin(), ary.begin() + k);
  ary.resize(k);
  return ary;
}

uint32_t pos_build1(std::mt19937 &rng, uint32_t j, uint32_t first, uint32_t num, bool selcon) {
  if (num == 1) return first;
  std::vector<uint32_t> ary(num);
  bool self = false;
  const uint32_t js = j - first;
  for (uint32_t q = 0; q < num; q++) {
    ary[q] = first + q;
    if (js == q && !selcon) self = true;
  }
  if (self) ary.erase(ary.begin() + js);
  std::shuffle(ary.begin(), ary.end(), rng);
  return ary[0];
}

}  // namespace

void build_network(Model &m) {
  Network &net = m.net;
  const float dt = m.dt;
  const uint32_t np = (uint32_t)m.pops.size();
  net.nidx.assign(np, 0);
  uint32_t q = 0;
  for (uint32_t i = 0; i < np; i++) {
    net.nidx[i] = q;
    q += m.pops[i].N;
  }
  const uint32_t n = q;
  net.n = n;
  if (n == 0) throw ParseError("network has no neurons");

  // ---- seeds (code/NetSimGnl2_BulPp.cpp:80-127) ----
  const int rp = std::max(1, m.opts.repeats);
  m.rseeds.assign(rp, 0);
  // UDFRDSEED_ACT shares its bit with STD_ACT (code/Inc.h:275,280), so -STD
  // alone also selects the user seed, which is then 0 (code/NetSimGnl2_BulPp.cpp:83-84).
  if (m.act_ctr & FS_ACT_STD) m.rseeds[0] = m.opts.user_seed;
  else if (!m.macro_seeds.empty()) m.rseeds[0] = m.macro_seeds[0];
  else m.rseeds[0] = std::random_device()();
  std::mt19937 rng;
  rng.seed(m.rseeds[0]);
  std::uniform_int_distribution<unsigned int> dist(0, RAND_MAX);
  for (int i = 1; i < std::max(1, m.opts.threads); i++) (void)dist(rng);  // zig[i].jcong
  for (unsigned i = 1; i < (unsigned)rp; i++) {
    if (i < m.macro_seeds.size()) {
      m.rseeds[i] = m.macro_seeds[i];
    } else {
      unsigned s;
      bool found = true;
      while (found) {
        found = false;
        s = dist(rng);
        for (unsigned j = 0; j < i; j++)
          if (s == m.rseeds[j]) { found = true; break; }
      }
      m.rseeds[i] = s;
    }
  }

  // ---- per-neuron parameters (code/NetSimGnl2_BulPp.cpp:159-278) ----
  auto fill = [n](std::vector<float> &v, float x) { v.assign(n, x); };
  fill(net.Vth, 0); fill(net.El, 0); fill(net.gl, 0); fill(net.Cm, 0); fill(net.Vreset, 0);
  fill(net.df, 0); fill(net.ef, 0); fill(net.dVmax, 0);
  net.RfPed.assign(n, 0); net.SpiDy.assign(n, 0);
  net.Vrev.assign((size_t)FS_NREC * n, 0.0f);
  net.dfst.assign((size_t)FS_NREC * n, 0.0f);
  net.ext_g.assign((size_t)FS_NREC * n, 0.0f);
  net.pb.assign((size_t)FS_NREC * n, 0.0f);
  fill(net.nmda_dfxt, 0); fill(net.nmda_efst, 0); fill(net.nmda_as, 0); fill(net.nmda_mg, 0);
  net.act.assign(n, m.act_ctr);
  fill(net.inj_mean, 0.0f); fill(net.inj_std, 0.0f);
  for (auto *v : {&net.stp_pv, &net.stp_dfD, &net.stp_efD, &net.stp_aF, &net.stp_dfF, &net.stp_efF,
                  &net.stp_aCap, &net.stp_dfCap, &net.stp_aCar, &net.stp_dfCar, &net.stp_efCar,
                  &net.ltp_dfLP, &net.ltp_PosISI, &net.ltp_NegISI})
    fill(*v, 0.0f);
  net.ltp_SpiLPDy.assign(n, 0);

  for (uint32_t i = 0; i < np; i++) {
    const Pop &p = m.pops[i];
    for (uint32_t j = net.nidx[i]; j < net.nidx[i] + p.N; j++) {
      net.Vth[j] = p.Vth;
      net.El[j] = p.El;
      net.gl[j] = p.Cm / p.Taum;
      net.Cm[j] = p.Cm;
      net.Vreset[j] = p.Vreset;
      net.df[j] = std::exp(-dt / p.Taum);
      net.ef[j] = p.Taum * (1.0f - net.df[j]);
      net.RfPed[j] = p.RfPed;
      net.SpiDy[j] = p.SpiDy;
      net.ltp_dfLP[j] = std::exp(-dt / p.tLP);
      net.ltp_SpiLPDy[j] = p.SpiLPDy;
      net.ltp_PosISI[j] = p.PosISI;
      net.ltp_NegISI[j] = p.NegISI;
      net.stp_pv[j] = p.pv;
      net.stp_dfD[j] = std::exp(-dt / p.tD);
      net.stp_efD[j] = 1.0f - net.stp_dfD[j];
      net.stp_aF[j] = p.aF;
      net.stp_dfF[j] = std::exp(-dt / p.tF);
      net.stp_efF[j] = p.tF * (1.0f - net.stp_dfF[j]);
      net.stp_aCap[j] = p.aCap;
      net.stp_dfCap[j] = std::exp(-dt / p.tCap);
      net.stp_aCar[j] = p.aCar;
      net.stp_dfCar[j] = std::exp(-dt / p.tCar);
      net.stp_efCar[j] = (1.0f - net.stp_dfCar[j]) * kCarBase * 1e-6f;
      // receptor defaults for receptors a population does not declare
      net.Vrev[FS_AMPA * n + j] = 0.0f;   net.dfst[FS_AMPA * n + j] = 0.1f;
      net.Vrev[FS_GABA * n + j] = -90.0f; net.dfst[FS_GABA * n + j] = 0.1f;
      net.dVmax[j] = (net.Vth[j] - net.Vrev[FS_GABA * n + j]) / net.ef[j];
      net.nmda_as[j] = 0.6332f;
      net.nmda_dfxt[j] = 0.1f;
      net.dfst[FS_NMDA * n + j] = 0.1f;
      net.nmda_efst[j] = 0.01f;
      net.Vrev[FS_NMDA * n + j] = 0.0f;
      net.nmda_mg[j] = 1.0f;
      net.Vrev[FS_ACH * n + j] = 0.0f;   net.dfst[FS_ACH * n + j] = 0.1f;
      net.Vrev[FS_GCL * n + j] = -90.0f; net.dfst[FS_GCL * n + j] = 0.1f;
      for (const Receptor &r : p.reps) {
        int ri = -1;
        switch (r.name) {
          case KW_AMPA: ri = FS_AMPA; break;
          case KW_GABA: ri = FS_GABA; break;
          case KW_ACH: ri = FS_ACH; break;
          case KW_GCL: ri = FS_GCL; break;
          case KW_NMDA: ri = FS_NMDA; break;
          default: break;
        }
        if (ri < 0) continue;
        if (ri == FS_GABA) net.dVmax[j] = (p.Vth - r.Vrev) / net.ef[j];
        net.Vrev[ri * n + j] = r.Vrev;
        net.dfst[ri * n + j] = std::exp(-dt / r.Tau);
        net.pb[ri * n + j] = r.FExt * dt * 1e-3f;
        net.ext_g[ri * n + j] = r.MnExtEff * r.MnExtCon;
        if (ri == FS_NMDA) {
          net.nmda_as[j] = 0.6332f;
          net.nmda_dfxt[j] = std::exp(-dt / r.TauXT);
          net.nmda_efst[j] = r.Tau * (1.0f - net.dfst[ri * n + j]);
          net.nmda_mg[j] = 1.0f;
        }
      }
    }
  }

  // ---- group connections: one gate per (pre neuron, link) with >= 2 targets
  //      (code/NetSimGnl2_BulPp.cpp:289-567) ----
  std::vector<SynIdx> tsyn[FS_NREC];
  std::vector<SynIdx> tgap;                       // gap entries (gate, post)
  std::vector<uint32_t> gap_gate_pre;             // PSynCndP[].PreID
  std::vector<float> gap_gate_g;
  for (int r = 0; r < FS_NREC; r++) {
    net.rec[r] = Network::RecArrays();
  }
  uint64_t total = 0;
  for (uint32_t i = 0; i < np; i++) {
    const Pop &p = m.pops[i];
    for (uint32_t k = net.nidx[i]; k < net.nidx[i] + p.N; k++) {
      for (uint32_t j = p.link_beg; j < p.link_beg + p.link_num; j++) {
        const Link &l = m.links[j];
        const uint16_t act = act_of(l.rep);
        const uint32_t tn = m.pops[l.tgt].N;
        uint32_t num = (uint32_t)std::ceil((double)tn * l.conn);
        if (i == l.tgt && tn == num && !p.selcon) num--;
        std::vector<uint32_t> pos = pos_build(rng, k, num, net.nidx[l.tgt], tn, p.selcon);
        const float g = l.eff * l.weight;
        if (num < 2) continue;
        if (act == FS_ACT_GAP) {
          const uint32_t gate = (uint32_t)gap_gate_pre.size();
          for (uint32_t kk = 0; kk < num; kk++) tgap.push_back({gate, pos[kk]});
          gap_gate_pre.push_back(k);
          gap_gate_g.push_back(g);
          total += num;
          continue;
        }
        const int r = rec_of_act(act);
        if (r < 0) continue;
        Network::RecArrays &ra = net.rec[r];
        const uint32_t gate = (uint32_t)ra.gate_pre.size();
        for (uint32_t kk = 0; kk < num; kk++) tsyn[r].push_back({gate, pos[kk]});
        ra.gate_pre.push_back(k);
        ra.gate_post0.push_back(pos[0]);
        ra.gate_g.push_back(g);
        total += num;
      }
    }
  }
  // Sort entries by post (unstable, same keys as the reference's SynIdx sort).
  for (int r = 0; r < FS_NREC; r++)
    std::sort(tsyn[r].begin(), tsyn[r].end(), [](SynIdx a, SynIdx b) { return a.post < b.post; });
  std::sort(tgap.begin(), tgap.end(), [](SynIdx a, SynIdx b) { return a.post < b.post; });

  // Gather lists per post.  Each segment of equal post in the sorted array is
  // summed into RVs[post] (code/EqsGnl2.cpp:941-979); the GluCl segments are
  // addressed through the AMPA-independent ACh segment table, as the
  // reference's MapPLPosID is (code/NetSimGnl2_BulPp.cpp:549-550).
  std::vector<std::pair<uint32_t, uint32_t>> seg[FS_NREC];
  for (int r = 0; r < FS_NREC; r++) seg[r] = segments(tsyn[r]);
  for (int r = 0; r < FS_NREC; r++) {
    Network::RecArrays &ra = net.rec[r];
    std::vector<std::vector<uint32_t>> per_post;  // built lazily only if needed
    std::vector<uint32_t> seg_post(seg[r].size());
    for (size_t s = 0; s < seg[r].size(); s++) {
      uint32_t src;
      if (r == FS_GCL) {
        if (s >= seg[FS_ACH].size() || seg[FS_ACH][s].first >= tsyn[FS_GCL].size())
          throw ParseError(
              "GluCl group connections whose post-synaptic map the reference reads out of range "
              "(it indexes them through the Ach map); not reproducible");
        src = tsyn[FS_GCL][seg[FS_ACH][s].first].post;
      } else {
        src = tsyn[r][seg[r][s].first].post;
      }
      seg_post[s] = src;
    }
    // order of summation into a post: its segments in segment order
    std::vector<uint32_t> cnt(n + 1, 0);
    for (size_t s = 0; s < seg[r].size(); s++)
      cnt[seg_post[s] + 1] += seg[r][s].second - seg[r][s].first + 1;
    for (uint32_t i = 0; i < n; i++) cnt[i + 1] += cnt[i];
    ra.gather_rowptr = cnt;
    ra.seg_post = seg_post;
    ra.seg_len.resize(seg[r].size());
    for (size_t s = 0; s < seg[r].size(); s++) ra.seg_len[s] = seg[r][s].second - seg[r][s].first + 1;
    ra.gather_gate.assign(cnt[n], 0);
    std::vector<uint32_t> fillp(cnt.begin(), cnt.end() - 1);
    for (size_t s = 0; s < seg[r].size(); s++) {
      uint32_t post = seg_post[s];
      for (uint32_t e = seg[r][s].first; e <= seg[r][s].second; e++)
        ra.gather_gate[fillp[post]++] = tsyn[r][e].pre;
    }
  }

  // delay of each link in steps
  auto delay_steps = [&](float ms) -> uint16_t {
    if (!(ms > 0.0f)) return 0;
    long v = std::lround(ms / dt);
    if (v > 65535) v = 65535;
    return (uint16_t)v;
  };

  // ---- single-target connections (code/NetSimGnl2_BulPp.cpp:571-695) ----
  std::vector<SynRec> srec[FS_NREC];
  std::vector<SynRec> sgap;
  std::vector<uint32_t> src_neuron[FS_NREC];  // presynaptic neuron k (production modes)
  std::vector<uint16_t> src_delay[FS_NREC];   // link delay in steps (production modes)
  for (uint32_t i = 0; i < np; i++) {
    const Pop &p = m.pops[i];
    for (uint32_t k = net.nidx[i]; k < net.nidx[i] + p.N; k++) {
      for (uint32_t j = p.link_beg; j < p.link_beg + p.link_num; j++) {
        const Link &l = m.links[j];
        const uint32_t tn = m.pops[l.tgt].N;
        const uint32_t num = (uint32_t)std::ceil((double)tn * l.conn);
        if (num != 1) continue;
        const uint16_t act = act_of(l.rep);
        if (act == FS_ACT_GAP) {
          uint32_t post = pos_build1(rng, k, net.nidx[l.tgt], tn, p.selcon);
          sgap.push_back({i, post, l.eff * l.weight});
          continue;
        }
        const int r = rec_of_act(act);
        if (r < 0) continue;
        uint32_t post = pos_build1(rng, k, net.nidx[l.tgt], tn, p.selcon);
        srec[r].push_back({i, post, l.eff * l.weight});  // PreID = population index
        src_neuron[r].push_back(k);
        src_delay[r].push_back(delay_steps(l.delay_ms));
      }
    }
  }
  // PostSetPp sorts (code/NetSimGnl2_BulPp.cpp:706-712).  The production
  // modes need the true presynaptic neuron of each record too; it rides
  // along in a permutation sorted with the same comparator.
  std::vector<uint32_t> srec_src[FS_NREC];
  std::vector<uint16_t> rec_delay[FS_NREC];
  for (int r = 0; r < FS_NREC; r++) {
    struct Tagged { uint32_t pre, post; float g; uint32_t src; uint16_t d; };
    std::vector<Tagged> t(srec[r].size());
    for (size_t e = 0; e < t.size(); e++)
      t[e] = {srec[r][e].pre, srec[r][e].post, srec[r][e].g, src_neuron[r][e], src_delay[r][e]};
    std::sort(t.begin(), t.end(), [](const Tagged &a, const Tagged &b) { return a.post < b.post; });
    Network::RecArrays &ra = net.rec[r];
    ra.rec_pre.resize(t.size());
    ra.rec_post.resize(t.size());
    ra.rec_g.resize(t.size());
    srec_src[r].resize(t.size());
    rec_delay[r].resize(t.size());
    for (size_t e = 0; e < t.size(); e++) {
      ra.rec_pre[e] = t[e].pre;
      ra.rec_post[e] = t[e].post;
      ra.rec_g[e] = t[e].g;
      srec_src[r][e] = t[e].src;
      rec_delay[r][e] = t[e].d;
    }
    ra.rec_src = srec_src[r];
    ra.rec_rowptr.assign(n + 1, 0);
    for (size_t e = 0; e < t.size(); e++) ra.rec_rowptr[t[e].post + 1]++;
    for (uint32_t x = 0; x < n; x++) ra.rec_rowptr[x + 1] += ra.rec_rowptr[x];
    total += t.size();
  }
  std::sort(sgap.begin(), sgap.end(), [](const SynRec &a, const SynRec &b) { return a.post < b.post; });
  total += sgap.size();
  net.gap1_pre.resize(sgap.size());
  net.gap1_post.resize(sgap.size());
  net.gap1_g.resize(sgap.size());
  for (size_t e = 0; e < sgap.size(); e++) {
    net.gap1_pre[e] = sgap[e].pre;
    net.gap1_post[e] = sgap[e].post;
    net.gap1_g[e] = sgap[e].g;
  }
  net.gap_ngroup.clear();
  net.total_synapses = total;

  // ---- gap-junction terms per neuron, in accumulation order ----
  // 1) group gap, as post (code/EqsGnl2.cpp:982-989); the reverse direction
  //    loop (:991-999) runs over PCndOCntSize, which the reference never sets
  //    (it stays 0), so it adds nothing.
  // 2) single-target gap as post (code/EqsGnl2.cpp:708-715), records by post.
  // 3) single-target gap as pre (code/EqsGnl2.cpp:717-724), by PreID then
  //    record index (BulDPreNeuMap, code/Eqs.h:1167-1203).
  {
    std::vector<std::vector<std::pair<uint32_t, float>>> terms;
    bool any = !tgap.empty() || !sgap.empty();
    if (any) {
      terms.assign(n, {});
      for (const SynIdx &e : tgap) terms[e.post].push_back({gap_gate_pre[e.pre], gap_gate_g[e.pre]});
      net.gap_ngroup.resize(n);
      for (uint32_t i = 0; i < n; i++) net.gap_ngroup[i] = (uint32_t)terms[i].size();
      for (const SynRec &e : sgap) terms[e.post].push_back({e.pre, e.g});
      std::vector<std::vector<uint32_t>> by_pre(n);
      for (uint32_t e = 0; e < sgap.size(); e++) {
        if (sgap[e].pre < n) by_pre[sgap[e].pre].push_back(e);
      }
      for (uint32_t i = 0; i < n; i++)
        for (uint32_t e : by_pre[i]) terms[i].push_back({sgap[e].post, sgap[e].g});
      net.gap_rowptr.assign(n + 1, 0);
      for (uint32_t i = 0; i < n; i++) net.gap_rowptr[i + 1] = net.gap_rowptr[i] + (uint32_t)terms[i].size();
      net.gap_other.clear();
      net.gap_g.clear();
      for (uint32_t i = 0; i < n; i++)
        for (auto &t : terms[i]) {
          net.gap_other.push_back(t.first);
          net.gap_g.push_back(t.second);
        }
    } else {
      net.gap_rowptr.clear();
      net.gap_other.clear();
      net.gap_g.clear();
    }
  }

  // ---- flat synapse list for the production modes ----
  net.syn_pre.clear(); net.syn_post.clear(); net.syn_rec.clear(); net.syn_g.clear(); net.syn_delay.clear();
  net.syn_ltp.clear();
  // group gates carry their link's delay: rebuild the link of each gate
  std::vector<uint16_t> gate_delay[FS_NREC];
  {
    uint32_t gcount[FS_NREC] = {0, 0, 0, 0, 0};
    for (uint32_t i = 0; i < np; i++) {
      const Pop &p = m.pops[i];
      for (uint32_t k = net.nidx[i]; k < net.nidx[i] + p.N; k++)
        for (uint32_t j = p.link_beg; j < p.link_beg + p.link_num; j++) {
          const Link &l = m.links[j];
          const uint32_t tn = m.pops[l.tgt].N;
          uint32_t num = (uint32_t)std::ceil((double)tn * l.conn);
          if (i == l.tgt && tn == num && !p.selcon) num--;
          if (num < 2) continue;
          const int r = rec_of_act(act_of(l.rep));
          if (r < 0) continue;
          gate_delay[r].push_back(delay_steps(l.delay_ms));
          gcount[r]++;
        }
    }
  }
  for (int r = 0; r < FS_NREC; r++) {
    const Network::RecArrays &ra = net.rec[r];
    for (uint32_t post = 0; post < n; post++)
      for (uint32_t e = ra.gather_rowptr[post]; e < ra.gather_rowptr[post + 1]; e++) {
        uint32_t gate = ra.gather_gate[e];
        net.syn_pre.push_back(ra.gate_pre[gate]);
        net.syn_post.push_back(post);
        net.syn_rec.push_back((uint8_t)r);
        net.syn_g.push_back(ra.gate_g[gate]);
        net.syn_delay.push_back(gate_delay[r][gate]);
        net.syn_ltp.push_back(0);
      }
    for (uint32_t e = 0; e < ra.rec_pre.size(); e++) {
      net.syn_pre.push_back(srec_src[r][e]);
      net.syn_post.push_back(ra.rec_post[e]);
      net.syn_rec.push_back((uint8_t)r);
      net.syn_g.push_back(ra.rec_g[e]);
      net.syn_delay.push_back(rec_delay[r][e]);
      net.syn_ltp.push_back(1);
    }
  }
  net.make_views(dt, m.act_ctr);
}

void Network::make_views(float dt, uint32_t act_ctr) {
  fs_neurons &nv = desc.neurons;
  nv.n = n;
  nv.Vth = Vth.data(); nv.El = El.data(); nv.gl = gl.data(); nv.Cm = Cm.data();
  nv.Vreset = Vreset.data(); nv.df = df.data(); nv.ef = ef.data(); nv.dVmax = dVmax.data();
  nv.RfPed = RfPed.data(); nv.SpiDy = SpiDy.data();
  nv.Vrev = Vrev.data(); nv.dfst = dfst.data();
  nv.nmda_dfxt = nmda_dfxt.data(); nv.nmda_efst = nmda_efst.data();
  nv.nmda_as = nmda_as.data(); nv.nmda_mg = nmda_mg.data();
  nv.ext_g = ext_g.data(); nv.pb = pb.data(); nv.act = act.data();
  nv.inj_mean = inj_mean.data(); nv.inj_std = inj_std.data();
  nv.stp_pv = stp_pv.data(); nv.stp_dfD = stp_dfD.data(); nv.stp_efD = stp_efD.data();
  nv.stp_aF = stp_aF.data(); nv.stp_dfF = stp_dfF.data(); nv.stp_efF = stp_efF.data();
  nv.stp_aCap = stp_aCap.data(); nv.stp_dfCap = stp_dfCap.data(); nv.stp_aCar = stp_aCar.data();
  nv.stp_dfCar = stp_dfCar.data(); nv.stp_efCar = stp_efCar.data();
  nv.ltp_dfLP = ltp_dfLP.data(); nv.ltp_PosISI = ltp_PosISI.data();
  nv.ltp_NegISI = ltp_NegISI.data(); nv.ltp_SpiLPDy = ltp_SpiLPDy.data();
  for (int r = 0; r < FS_NREC; r++) {
    fs_rec_layout &L = compat.rec[r];
    RecArrays &ra = rec[r];
    L.n_gates = (uint32_t)ra.gate_pre.size();
    L.gate_pre = ra.gate_pre.data(); L.gate_post0 = ra.gate_post0.data(); L.gate_g = ra.gate_g.data();
    L.gather_rowptr = ra.gather_rowptr.data(); L.gather_gate = ra.gather_gate.data();
    L.n_recs = (uint32_t)ra.rec_pre.size();
    L.rec_pre = ra.rec_pre.data(); L.rec_post = ra.rec_post.data(); L.rec_g = ra.rec_g.data();
    L.rec_rowptr = ra.rec_rowptr.data();
    L.rec_src = ra.rec_src.empty() ? nullptr : ra.rec_src.data();
  }
  compat.gap_rowptr = gap_rowptr.empty() ? nullptr : gap_rowptr.data();
  compat.gap_other = gap_other.data();
  compat.gap_g = gap_g.data();
  syn.n = syn_pre.size();
  syn.pre = syn_pre.data(); syn.post = syn_post.data(); syn.rec = syn_rec.data();
  syn.g = syn_g.data(); syn.delay = syn_delay.data(); syn.ltp = syn_ltp.data();
  desc.dt = dt;
  desc.act_ctr = act_ctr;
  desc.compat = &compat;
  desc.syn = &syn;
  desc.tm = nullptr;
}

}  // namespace fsh
