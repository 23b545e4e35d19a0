// network.log: the per-neuron parameters, every synapse, the time events and
// the output controls of a built network, in the text layout of the
// reference's NetSimGnl2::logDataWrite (code/NetSimGnl2_info.cpp:93-546),
// which its RunInit writes once before the first repeat
// (code/NetSimGnl2.cpp:143-157).  Numbers go through the same iostream
// formatting (6 significant digits), and synapses are listed in the
// reference's internal orders, so the file is byte-identical.
#include <cmath>
#include <fstream>
#include <memory>
#include <string>
#include <vector>
#include "fs_host.hpp"

namespace fsh {
namespace {

// TmEvt::TexInfo (code/parser_affi.cpp:30-47)
void event_info(std::ostream &o, const Event &e) {
  o << "Event Time=" << e.TimEv;
  if (e.Type == EVT_EXTFREQ) o << ", type:ChangeExtFreq";
  else if (e.Type == EVT_CURINJ) o << ", type:CurrentInjec";
  o << ", Target population:" << e.Pp << ", Receptor:" << (unsigned)e.SubTyp
    << ", Variable1=" << e.Var1 << ", Variable2=" << e.Var2 << "\n";
}

// OutCtr::TexInfo (code/parser_affi.cpp:76-91)
void output_info(std::ostream &o, const OutCtl &c) {
  o << "Output File Name:" << c.FileName << ", Type:" << c.Type << "\n" << "Population:";
  for (size_t i = 0; i < c.ParList.size(); i++) {
    o << c.ParList[i] << ", ";
    if (i % 10 == 0) o << "\n";
  }
  o << "\n";
}

// single-target records of one receptor ("SynAMPA1" ...): `base` is the
// record's index in the reference's shared array, which decides the breaks
void single_records(std::ostream &o, const char *name, const std::vector<uint32_t> &pre,
                    const std::vector<uint32_t> &post, const std::vector<float> &g, size_t base) {
  if (pre.empty()) return;
  o << name << ":Num;PreID,PosID,g;PreID,PosID,g...\n" << name << ":" << pre.size();
  write_ordered(o, pre.size(), 4096, [&](size_t a, size_t b, std::ostream &s) {
    for (size_t e = a; e < b; e++) {
      s << ";" << pre[e] << "," << post[e] << "," << g[e];
      if ((base + e) % 10 == 0) s << "\n";
    }
  });
  o << "\n";
}

// group connections of one receptor ("PSynAMPA" ...), segment by segment
void group_records(std::ostream &o, const char *name, const Network::RecArrays &ra, uint32_t n) {
  const size_t total = ra.gather_gate.size();
  if (!total) return;
  o << name << ":" << name << "size;PreID,PosID,g;PreID,PosID,g...\n" << name << ":" << total << ";";
  // where each segment starts in the gather list and in the reference's array
  const size_t ns = ra.seg_post.size();
  std::vector<uint32_t> cur(ra.gather_rowptr.begin(), ra.gather_rowptr.begin() + n);
  std::vector<uint32_t> at(ns);
  std::vector<size_t> i0(ns);
  size_t i = 0;
  for (size_t s = 0; s < ns; s++) {
    at[s] = cur[ra.seg_post[s]];
    cur[ra.seg_post[s]] += ra.seg_len[s];
    i0[s] = i;
    i += ra.seg_len[s];
  }
  write_ordered(o, ns, 256, [&](size_t a, size_t b, std::ostream &os) {
    for (size_t s = a; s < b; s++)
      for (uint32_t q = 0; q < ra.seg_len[s]; q++) {
        const uint32_t gate = ra.gather_gate[at[s] + q];
        os << ra.gate_pre[gate] << "," << ra.seg_post[s] << "," << ra.gate_g[gate] << ";";
        if ((i0[s] + q) % 10 == 0) os << "\n";
      }
  });
  o << "\n";
}

}  // namespace

bool write_network_log(const Model &m, const std::string &path) {
  const Network &net = m.net;
  const uint32_t n = net.n;
  std::unique_ptr<char[]> buf(new char[1 << 22]);
  std::ofstream o;
  o.rdbuf()->pubsetbuf(buf.get(), 1 << 22);
  o.open(path.c_str());
  if (!o) return false;

  // SInfo (code/NetSimGnl2_info.cpp:24-59)
  o << "\ncapable mode of sim07_21 leaky integrate and fire model"
    << "\ntime step:" << m.dt << ", total neurons=" << n
    << ", total synapses=" << net.total_synapses << "\n" << "\n";
  if (m.act_ctr & FS_ACT_STD) o << "User define random seed enable!\n";  // UDFRDSEED_ACT
  else o << "internal random seed enable!\n";
  o << "repeats=" << m.opts.repeats << ",each repeat random seed=";
  for (int r = 0; r < m.opts.repeats && r < (int)m.rseeds.size(); r++) o << " " << m.rseeds[r];
  o << "\n\npopulation information:-------------------------------------------\n";

  // The reference's SetPp stores each population's normalised noise std in
  // BgSt[population index] (code/NetSimGnl2_BulPp.cpp:177), so the first
  // populations-many neurons show 0 times that factor (-0 for the usual
  // negative factor) and the rest the initial 0 (:143).
  std::vector<float> noise_std(n, 0.0f);
  for (uint32_t i = 0; i < m.pops.size() && i < n; i++) {
    const Pop &p = m.pops[i];
    if (p.N == 0) continue;
    const float df = net.df[net.nidx[i]];
    noise_std[i] = 0.0f * (1.0f + (float)std::log(1.0f - std::exp(-0.1f / p.Taum)) / (1.0f - df));
  }
  auto R = [n](int r, uint32_t i) { return (size_t)r * n + i; };
  write_ordered(o, n, 256, [&](size_t a, size_t b, std::ostream &o) {
    for (uint32_t i = (uint32_t)a; i < b; i++) {
      const uint32_t act = net.act[i];
      o << "-------------------------------------------\n" << "neuron:" << i << "\n";
      o << "ActCtr=" << act << " Vth=" << net.Vth[i] << "mv" << " El=" << net.El[i] << "mv"
        << " g=" << net.gl[i] << "uS" << " Cm=" << net.Cm[i] << "nF" << " Vreset=" << net.Vreset[i]
        << "mv" << " df=" << net.df[i] << " ef=" << net.ef[i] << " dVmax=" << net.dVmax[i] << "mv\n";
      o << "AMPA df=" << net.dfst[R(FS_AMPA, i)] << " Vrev=" << net.Vrev[R(FS_AMPA, i)] << "mV"
        << " GABA df=" << net.dfst[R(FS_GABA, i)] << " Vrev=" << net.Vrev[R(FS_GABA, i)] << "mV\n"
        << "NMDA dfxt=" << net.nmda_dfxt[i] << " dfst=" << net.dfst[R(FS_NMDA, i)]
        << " efst=" << net.nmda_efst[i] << " Vrev=" << net.Vrev[R(FS_NMDA, i)] << "mV"
        << " as=" << net.nmda_as[i] << " mg=" << net.nmda_mg[i] << "\n"
        << "ACH df=" << net.dfst[R(FS_ACH, i)] << " Vrev=" << net.Vrev[R(FS_ACH, i)] << "mV"
        << " GCL df=" << net.dfst[R(FS_GCL, i)] << " Vrev=" << net.Vrev[R(FS_GCL, i)] << "mV\n";
      if (act & FS_ACT_LIF)
        o << "LIF:" << " RfPed=" << net.RfPed[i] * m.dt << "ms" << " SpiDy=" << net.SpiDy[i] * m.dt << "ms\n";
      if (act & FS_ACT_STP)
        o << "STP:" << " pv=" << net.stp_pv[i] << " dfD=" << net.stp_dfD[i] << " efD=" << net.stp_efD[i]
          << " aF=" << net.stp_aF[i] << " dfF=" << net.stp_dfF[i] << " efF=" << net.stp_efF[i]
          << " aCap=" << net.stp_aCap[i] << " dfCap=" << net.stp_dfCap[i] << " aCar=" << net.stp_aCar[i]
          << " dfCar=" << net.stp_dfCar[i] << " efCar=" << net.stp_efCar[i] << "\n";
      if (act & FS_ACT_LTP)
        o << "LTP:" << " df=" << net.ltp_dfLP[i] << " SpiLPDy=" << net.ltp_SpiLPDy[i]
          << " PosISI=" << net.ltp_PosISI[i] << " NegISI=" << net.ltp_NegISI[i] << "\n";
      o << "noise parameters:" << "\n";
      o << "Injection current:" << "mean=" << 0.0f << " stddev=" << noise_std[i] << "\n";
      o << "Ext AMPA:prob=" << net.pb[R(FS_AMPA, i)] << ",g=" << net.ext_g[R(FS_AMPA, i)] << "\n";
      o << "Ext GABA:prob=" << net.pb[R(FS_GABA, i)] << ",g=" << net.ext_g[R(FS_GABA, i)] << "\n";
      o << "Ext Ach:prob=" << net.pb[R(FS_ACH, i)] << ",g=" << net.ext_g[R(FS_ACH, i)] << "\n";
      o << "Ext GluCl:prob=" << net.pb[R(FS_GCL, i)] << ",g=" << net.ext_g[R(FS_GCL, i)] << "\n";
      o << "Ext NMDA:prob=" << net.pb[R(FS_NMDA, i)] << ",g=" << net.ext_g[R(FS_NMDA, i)] << "\n";
    }
  });

  o << "\nsynapse connection information----------------------------------\n";
  // SynFst1 holds AMPA, GABA, ACH, GCL records back to back
  size_t base = 0;
  const int fast[4] = {FS_AMPA, FS_GABA, FS_ACH, FS_GCL};
  const char *fast_name[4] = {"SynAMPA1", "SynGABA1", "SynACH1", "SynGCL1"};
  for (int q = 0; q < 4; q++) {
    const Network::RecArrays &ra = net.rec[fast[q]];
    single_records(o, fast_name[q], ra.rec_pre, ra.rec_post, ra.rec_g, base);
    base += ra.rec_pre.size();
  }
  {
    const Network::RecArrays &ra = net.rec[FS_NMDA];
    single_records(o, "SynNMDA1", ra.rec_pre, ra.rec_post, ra.rec_g, 0);
  }
  single_records(o, "SynCnd1", net.gap1_pre, net.gap1_post, net.gap1_g, 0);
  group_records(o, "PSynAMPA", net.rec[FS_AMPA], n);
  group_records(o, "PSynGABA", net.rec[FS_GABA], n);
  group_records(o, "PSynNMDA", net.rec[FS_NMDA], n);
  group_records(o, "PSynACH", net.rec[FS_ACH], n);
  group_records(o, "PSynGCL", net.rec[FS_GCL], n);
  if (!net.gap_ngroup.empty()) {  // group gap terms open each post's gap row
    size_t total = 0;
    for (uint32_t p = 0; p < n; p++) total += net.gap_ngroup[p];
    if (total) {
      o << "PSynCnd:PSynCndsize;PreID,PosID,g;PreID,PosID,g...\n" << "PSynCnd:" << total << ";";
      std::vector<size_t> i0(n);
      size_t i = 0;
      for (uint32_t p = 0; p < n; p++) {
        i0[p] = i;
        i += net.gap_ngroup[p];
      }
      write_ordered(o, n, 256, [&](size_t a, size_t b, std::ostream &os) {
        for (size_t p = a; p < b; p++)
          for (uint32_t q = 0; q < net.gap_ngroup[p]; q++) {
            const uint32_t e = net.gap_rowptr[p] + q;
            os << net.gap_other[e] << "," << p << "," << net.gap_g[e] << ";";
            if ((i0[p] + q) % 10 == 0) os << "\n";
          }
      });
      o << "\n";
    }
  }

  o << "\ntime event information:-------------------------------------------\n";
  for (const Event &e : m.events) event_info(o, e);

  o << "\noutput files information:-----------------------------------------\n";
  // single-target records by presynaptic id, in record order (BulDPreNeuMap,
  // code/Eqs.h:1167-1203); PreID is the population index of the source
  auto by_pre = [n](const std::vector<uint32_t> &pre) {
    std::vector<std::vector<uint32_t>> b(n);
    for (uint32_t e = 0; e < pre.size(); e++)
      if (pre[e] < n) b[pre[e]].push_back(e);
    return b;
  };
  std::vector<std::vector<uint32_t>> pre_map[FS_NREC];
  bool have_pre_map = false;
  for (const OutCtl &c : m.outs) {
    output_info(o, c);
    switch (c.TypeID) {
      case OUT_ISYNSEP: {
        o << "1:Time";
        uint32_t kk = 2;
        for (uint32_t pp : c.ParList)
          for (uint32_t k = net.nidx[pp]; k < net.nidx[pp] + m.pops[pp].N; k++) {
            o << " NID=" << k;
            o << " " << kk++ << ":AMPA ";
            o << " " << kk++ << ":GABA ";
            o << " " << kk++ << ":NMDA ";
            o << " " << kk++ << ":ACH ";
            o << " " << kk++ << ":GCL ";
          }
        o << "\n";
        break;
      }
      case OUT_MEMPOT: {
        o << "1:Time";
        uint32_t kk = 2;
        for (uint32_t pp : c.ParList)
          for (uint32_t k = net.nidx[pp]; k < net.nidx[pp] + m.pops[pp].N; k++) o << " " << kk++ << ":NID=" << k;
        o << "\n";
        break;
      }
      case OUT_FRATE: {
        o << "FiringRateWinodw=" << c.RWin << "ms PrintStep=" << c.FPnt << "ms\n";
        o << "1:Time";
        if (c.Status & OF_SUMALL) {
          o << "2:total firing rate";
        } else {
          uint32_t kk = 2;
          for (uint32_t j = 0; j < c.ParList.size(); j++) o << " " << kk++ << ":NID=" << j;
        }
        o << "\n";
        break;
      }
      case OUT_GATVAR: {
        if (!have_pre_map) {
          for (int r = 0; r < FS_NREC; r++) pre_map[r] = by_pre(net.rec[r].rec_pre);
          have_pre_map = true;
        }
        o << "1:Time ";
        uint32_t kk = 2;
        const int order[4] = {FS_AMPA, FS_GABA, FS_ACH, FS_GCL};
        const char *tag[4] = {"_AMAP_st ", "_GABA_st ", "_ACH_st ", "_GCL_st "};
        for (uint32_t pp : c.ParList)
          for (uint32_t k = net.nidx[pp]; k < net.nidx[pp] + m.pops[pp].N; k++) {
            for (int q = 0; q < 4; q++)
              for (uint32_t e : pre_map[order[q]][k])
                o << kk++ << ":NID=" << k << "_PosID=" << net.rec[order[q]].rec_post[e] << tag[q];
            for (uint32_t e : pre_map[FS_NMDA][k]) {
              o << kk++ << ":NID=" << k << "_PosID=" << net.rec[FS_NMDA].rec_post[e] << "_NMDA_xt ";
              o << kk++ << ":NID=" << k << "_PosID=" << net.rec[FS_NMDA].rec_post[e] << "_NMDA_st ";
            }
          }
        break;
      }
      default:
        break;
    }
    o << "\n";
  }
  o.flush();
  return bool(o);
}

}  // namespace fsh
