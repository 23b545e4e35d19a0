// network.conf / network.pro parsing for the flysim drop-in.
//
// The file formats and every parsing rule below follow the reference's
// finite-state parsers (code/parser.cpp), written anew:
//   - tokens are separated by any of " :;,'=\t\r\n" (code/parser.cpp:28);
//   - the file is consumed in pieces of at most 65535 bytes exactly as
//     ifstream::get(ch, 65536, EOF) returns them (code/parser.cpp:63,151-169),
//     which matters because a piece that starts with a delimiter after a piece
//     that ended on one yields an empty token (the reference processes it);
//   - population, group and event look-ups take the FIRST matching name
//     (code/parser.cpp:806-814, :986-993, :1128-1147, :1316-1333); here they
//     use hash maps instead of linear scans (same result, O(1) per look-up);
//   - numbers go through std::stoi/std::stof like the reference.
#include <cmath>
#include <climits>
#include <cfloat>
#include <fstream>
#include <memory>
#include <sstream>
#include <unordered_map>
#include <algorithm>
#include "fs_host.hpp"

namespace fsh {
namespace {

// FSM states (values are internal; names follow code/Inc.h:67-173)
enum {
  ST_Initial = 0, ST_NeuPopuName, ST_NeuPopu, ST_N, ST_Taum, ST_Vth, ST_gl, ST_Cm, ST_Vresting,
  ST_Vreset, ST_RfPed, ST_SpiDy, ST_SelfCon, ST_HH, ST_STP_pv, ST_STP_tD, ST_STP_aF, ST_STP_tF,
  ST_STP_aCap, ST_STP_tCap, ST_STP_aCar, ST_STP_tCar, ST_LTP_tLP, ST_LTP_SpiLPDy, ST_LTP_PosISI,
  ST_LTP_NegISI, ST_RepName, ST_Receptor, ST_RepTauST, ST_RepTauXT, ST_RepVrv, ST_RepFExt,
  ST_RepMnExtEff, ST_RepMnExtCon, ST_NeuConName, ST_NeuCon, ST_NeuCon_Conct, ST_NeuCon_TarRep,
  ST_NeuCon_MnEff, ST_NeuCon_weight, ST_NeuCon_Delay, ST_VthSod,
  // .pro
  ST_TimEv = 100, ST_TimEvDef, ST_TimTyp, ST_TimLbl, ST_TimPp, ST_TimSubTyp, ST_TimVar1, ST_TimVar2,
  ST_OutCtr, ST_OutName, ST_OutType, ST_OutRWin, ST_OutFPnt, ST_OutTimEv, ST_OutPopu, ST_OutSumAllPp,
  ST_OutAlign, ST_DefMac, ST_MacGpName, ST_MacGpMbs, ST_MacRndSeds
};

const char *const kDelims = " :;,'=\t\r\n";

// Token stream with the reference's piece-wise reading (see file comment).
class TokenReader {
 public:
  explicit TokenReader(const std::string &path) {
    fin_.open(path.c_str());
    if (fin_) {
      read_piece(str_);
    } else {
      opened_ = false;
    }
    startpos_ = 0;
    pos_ = str_.find_first_of(kDelims, startpos_);
  }
  bool opened() const { return opened_; }
  bool next(std::string &tok) {
    if (!((pos_ != std::string::npos) || (startpos_ != std::string::npos))) return false;
    tok = str_.substr(startpos_, pos_ - startpos_);
    startpos_ = str_.find_first_not_of(kDelims, pos_);
    pos_ = str_.find_first_of(kDelims, startpos_);
    if (!opened_ || fin_.eof()) {
      // whole input consumed: keep scanning the current piece
    } else if (startpos_ == std::string::npos) {
      read_piece(str_);
      startpos_ = 0;
      pos_ = str_.find_first_of(kDelims, startpos_);
    } else if (pos_ == std::string::npos) {
      std::string carry = str_.substr(startpos_, str_.size() - 1);
      std::string piece;
      read_piece(piece);
      str_ = carry + piece;
      startpos_ = 0;
      pos_ = str_.find_first_of(kDelims, startpos_);
    }
    return true;
  }

 private:
  void read_piece(std::string &out) {
    buf_.assign(65536, '\0');
    fin_.get(&buf_[0], 65536, EOF);
    out.assign(buf_.c_str());
  }
  std::ifstream fin_;
  bool opened_ = true;
  std::string str_, buf_;
  std::string::size_type startpos_ = 0, pos_ = 0;
};

int to_i(const std::string &s, const char *what) {
  try {
    return std::stoi(s);
  } catch (...) {
    throw ParseError(std::string("expected an integer for ") + what + ", got '" + s + "'");
  }
}
float to_f(const std::string &s, const char *what) {
  try {
    return std::stof(s);
  } catch (...) {
    throw ParseError(std::string("expected a number for ") + what + ", got '" + s + "'");
  }
}

// Values the reference uses as sizes, divisors or step counts without a
// check (a negative N wraps its allocation, a zero FiringRateWindow divides
// by zero, a NaN event time breaks the event sort): here they are errors
// that name the keyword, where the reference crashes or runs undefined.
uint32_t to_count(const std::string &s, const char *what) {
  const int v = to_i(s, what);
  if (v < 0) throw ParseError(std::string(what) + " must not be negative, got '" + s + "'");
  return (uint32_t)v;
}
// a duration in ms rounded up to whole ms, at least 1
uint32_t to_whole_ms(const std::string &s, const char *what) {
  const float x = to_f(s, what);
  if (!(x > 0.0f) || !(x < 2147483648.0f))
    throw ParseError(std::string(what) + " must be a positive number of ms, got '" + s + "'");
  return (uint32_t)std::ceil(x);
}
// a finite number
float to_finite(const std::string &s, const char *what) {
  const float x = to_f(s, what);
  if (!std::isfinite(x)) throw ParseError(std::string(what) + " must be a finite number, got '" + s + "'");
  return x;
}
// floor(x / dt) (+ add) as the reference's int members take it
int to_steps(const std::string &s, const char *what, float dt, float add = 0.0f) {
  const float v = std::floor(to_finite(s, what) / dt) + add;
  if (!(v > -2147483648.0f && v < 2147483648.0f))
    throw ParseError(std::string(what) + " is out of range, got '" + s + "'");
  return (int)v;
}

// Receptor names of STATE_RepName / STATE_NeuCon_TarRep (code/parser.cpp:732-745, :844-857);
// unknown names leave kw unchanged, as the reference's shared KwTmp does.
void receptor_kw(const std::string &s, unsigned &kw) {
  if (s == "AMPA") kw = KW_AMPA;
  else if (s == "GABA") kw = KW_GABA;
  else if (s == "NMDA") kw = KW_NMDA;
  else if (s == "GAP") kw = KW_GAP;
  else if (s == "Sine") kw = KW_SINE;
  else if (s == "Ach") kw = KW_ACH;
  else if (s == "GluCl") kw = KW_GCL;
}

std::unordered_map<std::string, uint32_t> pop_index(const Model &m) {
  std::unordered_map<std::string, uint32_t> idx;
  idx.reserve(m.pops.size() * 2);
  for (uint32_t i = 0; i < m.pops.size(); i++) idx.emplace(m.pops[i].name, i);  // first wins
  return idx;
}

}  // namespace

// Parser::CSta (code/parser.cpp:51-294): count populations, receptors and
// links, then set every default.
void parse_conf_counts(Model &m, const std::string &path, int &state) {
  TokenReader rd(path);
  if (!rd.opened()) throw ParseError(".conf open file error: " + path);
  std::string s1;
  while (rd.next(s1)) {
    switch (state) {
      case ST_Initial:
        if (s1 == "NeuralPopulation") {
          m.pops.emplace_back();
          state = ST_NeuPopuName;
        }
        break;
      case ST_NeuPopuName:
        m.pops.back().name = s1;
        state = ST_NeuPopu;
        break;
      case ST_NeuPopu:
        if (s1 == "Receptor") {
          m.pops.back().nrep++;
          state = ST_Receptor;
        } else if (s1 == "TargetPopulation") {
          m.pops.back().link_num++;
          state = ST_NeuCon;
        } else if (s1 == "SelfConnection") {
          state = ST_SelfCon;
        } else if (s1 == "EndNeuralPopulation") {
          state = ST_Initial;
        }
        break;
      case ST_Receptor:
        if (s1 == "EndReceptor") state = ST_NeuPopu;
        break;
      case ST_NeuCon:
        if (s1 == "EndTargetPopulation") state = ST_NeuPopu;
        break;
      case ST_SelfCon:
        m.pops.back().selcon = (s1 == "true");
        state = ST_NeuPopu;
        break;
      default:
        break;
    }
  }
  uint32_t nl = 0;
  const float dt = m.dt;
  for (auto &p : m.pops) {
    p.reps.assign(p.nrep, Receptor());
    p.link_beg = nl;
    nl += p.link_num;
    p.RfPed = (int)(1.8f / dt + dt);  // code/parser.cpp:214
    p.SpiDy = (int)0.0f;
  }
  m.links.assign(nl, Link());
}

// Parser::parse(conf) (code/parser.cpp:297-907).
void parse_conf(Model &m, const std::string &path, int &state) {
  TokenReader rd(path);
  if (!rd.opened()) throw ParseError(".conf open file error: " + path);
  auto idx = pop_index(m);
  std::string s1;
  unsigned kw = KW_AMPA;
  uint32_t Ni = 0, Ri = 0, Li = 0;
  const float dt = m.dt;
  auto pop = [&]() -> Pop & {
    if (Ni >= m.pops.size()) throw ParseError("population count mismatch in .conf");
    return m.pops[Ni];
  };
  auto rep = [&]() -> Receptor & {
    Pop &p = pop();
    if (Ri >= p.reps.size()) throw ParseError("receptor count mismatch in population " + p.name);
    return p.reps[Ri];
  };
  auto link = [&]() -> Link & {
    Pop &p = pop();
    if (Li >= p.link_num) throw ParseError("link count mismatch in population " + p.name);
    return m.links[p.link_beg + Li];
  };
  while (rd.next(s1)) {
    switch (state) {
      case ST_Initial:
        if (s1 == "NeuralPopulation") state = ST_NeuPopuName;
        break;
      case ST_NeuPopuName:
        state = ST_NeuPopu;
        break;
      case ST_NeuPopu:
        if (s1 == "N") state = ST_N;
        else if (s1 == "Taum") state = ST_Taum;
        else if (s1 == "Threshold") state = ST_Vth;
        else if (s1 == "LeakyConductance") state = ST_gl;
        else if (s1 == "C") state = ST_Cm;
        else if (s1 == "RevPot" || s1 == "RestPot") state = ST_Vresting;
        else if (s1 == "ResetPot") state = ST_Vreset;
        else if (s1 == "RefractoryPeriod") state = ST_RfPed;
        else if (s1 == "SpikeDly") state = ST_SpiDy;
        else if (s1 == "STP_pv") state = ST_STP_pv;
        else if (s1 == "STP_tD") state = ST_STP_tD;
        else if (s1 == "STP_aF") state = ST_STP_aF;
        else if (s1 == "STP_tF") state = ST_STP_tF;
        else if (s1 == "STP_aCap") state = ST_STP_aCap;
        else if (s1 == "STP_tCap") state = ST_STP_tCap;
        else if (s1 == "STP_aCar") state = ST_STP_aCar;
        else if (s1 == "STP_tCar") state = ST_STP_tCar;
        else if (s1 == "LTP_tLP") state = ST_LTP_tLP;
        else if (s1 == "LTP_SpiLPDy") state = ST_LTP_SpiLPDy;
        else if (s1 == "LTP_PosISI") state = ST_LTP_PosISI;
        else if (s1 == "LTP_NegISI") state = ST_LTP_NegISI;
        else if (s1 == "VthSodium") state = ST_VthSod;
        else if (s1.size() > 3 && s1.compare(0, 3, "HH_") == 0 &&
                 (s1 == "HH_Ek" || s1 == "HH_gk" || s1 == "HH_Ena" || s1 == "HH_gna" ||
                  (s1.size() == 6 && std::string("AB").find(s1[3]) != std::string::npos &&
                   std::string("nmh").find(s1[4]) != std::string::npos &&
                   std::string("ABCD").find(s1[5]) != std::string::npos)))
          state = ST_HH;  // Hodgkin-Huxley parameters: parsed, unused by GNL2
        else if (s1 == "Receptor") state = ST_RepName;
        else if (s1 == "TargetPopulation") state = ST_NeuConName;
        else if (s1 == "EndNeuralPopulation") {
          Ni++;
          Ri = 0;
          Li = 0;
          state = ST_Initial;
        }
        break;
      case ST_N: pop().N = to_count(s1, "N"); state = ST_NeuPopu; break;
      case ST_Taum: pop().Taum = to_f(s1, "Taum"); state = ST_NeuPopu; break;
      case ST_Vth: pop().Vth = to_f(s1, "Threshold"); state = ST_NeuPopu; break;
      case ST_gl: pop().gl = to_f(s1, "LeakyConductance"); state = ST_NeuPopu; break;
      case ST_Cm: pop().Cm = to_f(s1, "C"); state = ST_NeuPopu; break;
      case ST_Vreset: pop().Vreset = to_f(s1, "ResetPot"); state = ST_NeuPopu; break;
      case ST_Vresting: pop().El = to_f(s1, "RestPot"); state = ST_NeuPopu; break;
      case ST_RfPed:  // int member assigned floor(x/dt)+dt (code/parser.cpp:508)
        pop().RfPed = to_steps(s1, "RefractoryPeriod", dt, dt);
        state = ST_NeuPopu;
        break;
      case ST_SpiDy:
        pop().SpiDy = to_steps(s1, "SpikeDly", dt);
        state = ST_NeuPopu;
        break;
      case ST_STP_pv: pop().pv = to_f(s1, "STP_pv"); state = ST_NeuPopu; break;
      case ST_STP_tD: pop().tD = to_f(s1, "STP_tD"); state = ST_NeuPopu; break;
      case ST_STP_aF: pop().aF = to_f(s1, "STP_aF"); state = ST_NeuPopu; break;
      case ST_STP_tF: pop().tF = to_f(s1, "STP_tF"); state = ST_NeuPopu; break;
      case ST_STP_aCap: pop().aCap = to_f(s1, "STP_aCap"); state = ST_NeuPopu; break;
      case ST_STP_tCap: pop().tCap = to_f(s1, "STP_tCap"); state = ST_NeuPopu; break;
      case ST_STP_aCar: pop().aCar = to_f(s1, "STP_aCar"); state = ST_NeuPopu; break;
      case ST_STP_tCar: pop().tCar = to_f(s1, "STP_tCar"); state = ST_NeuPopu; break;
      case ST_LTP_tLP: pop().tLP = to_f(s1, "LTP_tLP"); state = ST_NeuPopu; break;
      case ST_LTP_SpiLPDy:
        pop().SpiLPDy = to_steps(s1, "LTP_SpiLPDy", dt);
        state = ST_NeuPopu;
        break;
      case ST_LTP_PosISI: pop().PosISI = to_f(s1, "LTP_PosISI"); state = ST_NeuPopu; break;
      case ST_LTP_NegISI: pop().NegISI = to_f(s1, "LTP_NegISI"); state = ST_NeuPopu; break;
      case ST_VthSod:
      case ST_HH:
        (void)to_f(s1, "HH parameter");
        state = ST_NeuPopu;
        break;
      case ST_RepName:
        receptor_kw(s1, kw);
        rep().name = (uint8_t)kw;
        state = ST_Receptor;
        break;
      case ST_Receptor:
        if (s1 == "Tau") state = ST_RepTauST;
        else if (s1 == "TauXT") state = ST_RepTauXT;
        else if (s1 == "RevPot") state = ST_RepVrv;
        else if (s1 == "FreqExt") state = ST_RepFExt;
        else if (s1 == "MeanExtEff") state = ST_RepMnExtEff;
        else if (s1 == "MeanExtCon") state = ST_RepMnExtCon;
        else if (s1 == "EndReceptor") {
          Ri++;
          state = ST_NeuPopu;
        }
        break;
      case ST_RepTauST: rep().Tau = to_f(s1, "Tau"); state = ST_Receptor; break;
      case ST_RepTauXT: rep().TauXT = to_f(s1, "TauXT"); state = ST_Receptor; break;
      case ST_RepVrv: rep().Vrev = to_f(s1, "RevPot"); state = ST_Receptor; break;
      case ST_RepFExt: rep().FExt = to_f(s1, "FreqExt"); state = ST_Receptor; break;
      case ST_RepMnExtEff: rep().MnExtEff = to_f(s1, "MeanExtEff"); state = ST_Receptor; break;
      case ST_RepMnExtCon: rep().MnExtCon = to_f(s1, "MeanExtCon"); state = ST_Receptor; break;
      case ST_NeuConName: {
        auto it = idx.find(s1);
        if (it != idx.end()) link().tgt = it->second;
        state = ST_NeuCon;
        break;
      }
      case ST_NeuCon:
        if (s1 == "Connectivity") state = ST_NeuCon_Conct;
        else if (s1 == "TargetReceptor") state = ST_NeuCon_TarRep;
        else if (s1 == "MeanEff") state = ST_NeuCon_MnEff;
        else if (s1 == "weight") state = ST_NeuCon_weight;
        else if (s1 == "Delay") state = ST_NeuCon_Delay;
        else if (s1 == "EndTargetPopulation") {
          Li++;
          state = ST_NeuPopu;
        }
        break;
      case ST_NeuCon_Conct: {
        float c = to_f(s1, "Connectivity");
        if (!(c >= 0.0f))  // the target count ceil(N*c) would wrap (the reference's does)
          throw ParseError("Connectivity must be a number in [0, 1], got '" + s1 + "'");
        if (c > 1.0f) c = 1.0f;  // code/parser.cpp:836
        link().conn = c;
        state = ST_NeuCon;
        break;
      }
      case ST_NeuCon_TarRep:
        receptor_kw(s1, kw);
        link().rep = (uint8_t)kw;
        state = ST_NeuCon;
        break;
      case ST_NeuCon_MnEff: link().eff = to_f(s1, "MeanEff"); state = ST_NeuCon; break;
      case ST_NeuCon_weight: link().weight = to_f(s1, "weight"); state = ST_NeuCon; break;
      case ST_NeuCon_Delay: link().delay_ms = to_f(s1, "Delay"); state = ST_NeuCon; break;
      default:
        break;
    }
  }
}

// Parser::DefMacro (code/parser.cpp:911-1029): groups and random seeds.
void parse_macros(Model &m, const std::string &path, int &state) {
  TokenReader rd(path);
  if (!rd.opened()) throw ParseError(".pro open file error: " + path);
  auto idx = pop_index(m);
  std::string s1;
  Group g;
  while (rd.next(s1)) {
    switch (state) {
      case ST_Initial:
        if (s1 == "DefineMacro") state = ST_DefMac;
        break;
      case ST_DefMac:
        if (s1 == "GroupName") state = ST_MacGpName;
        else if (s1 == "GroupMembers") state = ST_MacGpMbs;
        else if (s1 == "RandomSeeds") state = ST_MacRndSeds;
        else if (s1 == "EndDefineMacro") state = ST_Initial;
        break;
      case ST_MacGpName:
        g.name = s1;
        state = ST_DefMac;
        break;
      case ST_MacRndSeds:
        if (s1 == "EndRandomSeeds") {
          state = ST_DefMac;
        } else {
          unsigned v = (unsigned)to_i(s1, "RandomSeeds");
          if (v <= (unsigned)RAND_MAX) m.macro_seeds.push_back(v);
        }
        break;
      case ST_MacGpMbs:
        if (s1 == "EndGroupMembers") {
          m.groups.push_back(g);
          g.pops.clear();
          state = ST_DefMac;
        } else {
          auto it = idx.find(s1);
          if (it != idx.end()) g.pops.push_back(it->second);
        }
        break;
      default:
        break;
    }
  }
}

// Parser::parse(pro) (code/parser.cpp:1032-1407): events and outputs.
void parse_pro(Model &m, const std::string &path, int &state) {
  TokenReader rd(path);
  if (!rd.opened()) throw ParseError(".pro open file error: " + path);
  auto idx = pop_index(m);
  std::unordered_map<std::string, uint32_t> gidx;
  for (uint32_t i = 0; i < m.groups.size(); i++) gidx.emplace(m.groups[i].name, i);
  const uint32_t npop = (uint32_t)m.pops.size();
  std::vector<Event> unsolved;
  Event ev;
  OutCtl of;
  std::string s1;
  unsigned kw = KW_AMPA;
  while (rd.next(s1)) {
    switch (state) {
      case ST_Initial:
        if (s1 == "EventTime") state = ST_TimEv;
        else if (s1 == "OutControl") state = ST_OutCtr;
        break;
      case ST_TimEv:
        if (s1 == "NoLimit") {
          ev.NoLmt = true;
          ev.TimEv = FLT_MAX;
        } else {
          ev.NoLmt = false;
          ev.TimEv = to_finite(s1, "EventTime") * 1e-3f;
        }
        state = ST_TimEvDef;
        break;
      case ST_TimEvDef:
        if (s1 == "Type") state = ST_TimTyp;
        else if (s1 == "Label" || s1 == "InFile") state = ST_TimLbl;
        else if (s1 == "Population") state = ST_TimPp;
        else if (s1 == "Receptor" || s1 == "SubType") state = ST_TimSubTyp;
        else if (s1 == "FreqExt" || s1 == "GaussMean") state = ST_TimVar1;
        else if (s1 == "GaussSTD") state = ST_TimVar2;
        else if (s1 == "EndEvent") {
          unsolved.push_back(ev);
          ev = Event();
          state = ST_Initial;
        }
        break;
      case ST_TimTyp:
        if (s1 == "ChangeExtFreq") ev.Type = EVT_EXTFREQ;
        else if (s1 == "ChangeMembraneNoise" || s1 == "CurrentInjec") ev.Type = EVT_CURINJ;
        state = ST_TimEvDef;
        break;
      case ST_TimLbl:
        state = ST_TimEvDef;
        break;
      case ST_TimPp: {
        auto it = idx.find(s1);
        if (it != idx.end()) ev.Pp = it->second;
        auto gt = gidx.find(s1);
        if (gt != gidx.end()) ev.Pp = gt->second + npop;
        if (s1 == "AllPopulation") ev.Pp = UINT_MAX;
        state = ST_TimEvDef;
        break;
      }
      case ST_TimSubTyp:
        if (s1 == "AMPA") kw = KW_AMPA;
        else if (s1 == "GABA") kw = KW_GABA;
        else if (s1 == "NMDA") kw = KW_NMDA;
        else if (s1 == "Ach") kw = KW_ACH;
        else if (s1 == "GluCl") kw = KW_GCL;
        else if (s1 == "GAP") kw = KW_GAP;
        else if (s1 == "Sine") kw = KW_SINE;
        else if (s1 == "ResumeSynCdt") kw = RSM_SYNCOND;
        else if (s1 == "ResumeGatingVariable") kw = RSM_GATVAR;
        else if (s1 == "ResumeMemPot") kw = RSM_MEMPOT;
        else if (s1 == "ResumeRndSeed") kw = RSM_RNDSED;
        else if (s1 == "ResumeAll") kw = RSM_ALL;
        ev.SubTyp = (uint8_t)kw;
        state = ST_TimEvDef;
        break;
      case ST_TimVar1: ev.Var1 = to_f(s1, "FreqExt/GaussMean"); state = ST_TimEvDef; break;
      case ST_TimVar2: ev.Var2 = to_f(s1, "GaussSTD"); state = ST_TimEvDef; break;
      case ST_OutCtr:
        if (s1 == "FileName") state = ST_OutName;
        else if (s1 == "Type") state = ST_OutType;
        else if (s1 == "FiringRateWindow") state = ST_OutRWin;
        else if (s1 == "PrintStep") state = ST_OutFPnt;
        else if (s1 == "SumAllPopulation") state = ST_OutSumAllPp;
        else if (s1 == "Align") state = ST_OutAlign;
        else if (s1 == "EventTime") state = ST_OutTimEv;
        else if (s1 == "population") state = ST_OutPopu;
        else if (s1 == "EndOutputFile") {
          if (of.Type != "Non") m.outs.push_back(of);
          std::vector<uint32_t> keep_win = of.SpiRWin;  // OutCtr::init leaves SpiRWin alone
          of = OutCtl();
          of.SpiRWin = keep_win;
          state = ST_OutCtr;
        } else if (s1 == "EndOutControl") {
          state = ST_Initial;
        }
        break;
      case ST_OutName: of.FileName = s1; state = ST_OutCtr; break;
      case ST_OutType:
        if (s1 == "MemPot" && !m.comm_mem) { of.Type = s1; of.TypeID = OUT_MEMPOT; }
        else if (s1 == "Spike" && !m.comm_spike) { of.Type = s1; of.TypeID = OUT_SPIKE; }
        else if (s1 == "FiringRate" && !m.comm_rate) { of.Type = s1; of.TypeID = OUT_FRATE; }
        else if (s1 == "GatingVariable") { of.Type = s1; of.TypeID = OUT_GATVAR; }
        else if (s1 == "IsynSeparatedSum") { of.Type = s1; of.TypeID = OUT_ISYNSEP; }
        else if (s1 == "SaveAllStates") { of.Type = s1; of.TypeID = OUT_SAVE; }
        else if (s1 == "SynapticWeight") { of.Type = s1; of.TypeID = OUT_SYNWGT; }
        else if (s1 == "DeltaMemPotLimit") { of.Type = s1; of.TypeID = OUT_DVOVF; }
        state = ST_OutCtr;
        break;
      case ST_OutRWin: of.RWin = to_whole_ms(s1, "FiringRateWindow"); state = ST_OutCtr; break;
      case ST_OutFPnt: of.FPnt = to_whole_ms(s1, "PrintStep"); state = ST_OutCtr; break;
      case ST_OutSumAllPp:
        if (s1 == "true") of.Status |= OF_SUMALL; else of.Status &= ~(uint32_t)OF_SUMALL;
        state = ST_OutCtr;
        break;
      case ST_OutAlign:
        if (s1 == "true") of.Status |= OF_ALIGN; else of.Status &= ~(uint32_t)OF_ALIGN;
        state = ST_OutCtr;
        break;
      case ST_OutTimEv: of.TimEv = to_f(s1, "EventTime") * 1e-3f; state = ST_OutCtr; break;
      case ST_OutPopu:
        if (s1 == "AllPopulation") {
          for (uint32_t i = 0; i < npop; i++) of.ParList.push_back(i);
        } else {
          auto it = idx.find(s1);
          if (it != idx.end()) of.ParList.push_back(it->second);
          auto gt = gidx.find(s1);
          if (gt != gidx.end()) {
            const auto &gp = m.groups[gt->second].pops;
            of.ParList.insert(of.ParList.end(), gp.begin(), gp.end());
          }
        }
        state = ST_OutCtr;
        break;
      default:
        break;
    }
  }
  // Macro expansion of events (code/parser.cpp:1368-1392).
  for (const Event &e : unsolved) {
    if (e.Pp < npop) {
      m.events.push_back(e);
    } else if (e.Pp == UINT_MAX) {
      for (uint32_t p = 0; p < npop; p++) {
        m.events.push_back(e);
        m.events.back().Pp = p;
      }
    } else {
      for (uint32_t j = 0; j < m.groups.size(); j++) {
        if (e.Pp == npop + j) {
          for (uint32_t p : m.groups[j].pops) {
            m.events.push_back(e);
            m.events.back().Pp = p;
          }
        }
      }
    }
  }
  // Same (unstable) libstdc++ sort on the same keys: same order of ties.
  std::sort(m.events.begin(), m.events.end(),
            [](const Event &a, const Event &b) { return a.TimEv < b.TimEv; });
}

// Parser::Comm (code/parser.cpp:1424-1464).
void add_command_outputs(Model &m) {
  const uint32_t npop = (uint32_t)m.pops.size();
  auto add = [&](const char *type, int id, const std::string &name) {
    OutCtl o;
    o.Type = type;
    o.TypeID = id;
    o.FileName = name;
    for (uint32_t i = 0; i < npop; i++) o.ParList.push_back(i);
    m.outs.push_back(o);
  };
  if (m.comm_mem) add("MemPot", OUT_MEMPOT, m.out_mem);
  if (m.comm_spike) add("Spike", OUT_SPIKE, m.out_spike);
  if (m.comm_rate) add("FiringRate", OUT_FRATE, m.out_rate);
}

static const char *rep_name(uint8_t kw, bool with_gap) {
  switch (kw) {
    case KW_AMPA: return "AMPA";
    case KW_GABA: return "GABA";
    case KW_NMDA: return "NMDA";
    case KW_ACH: return "Ach";
    case KW_GCL: return "GluCl";
    case KW_GAP: return with_gap ? "GAP" : "";
    default: return "";
  }
}

// Parser::ConfsInfo (code/parser.cpp:1488-1631): ConfsInfo.log.  The
// Hodgkin-Huxley block prints the reference's defaults (HH is not simulated).
bool write_confs_info(const Model &m, const std::string &path) {
  std::unique_ptr<char[]> buf(new char[1 << 22]);
  std::ofstream o;
  o.rdbuf()->pubsetbuf(buf.get(), 1 << 22);
  o.open(path.c_str());
  if (!o) return false;
  o << "configuration information:----------------------------------------\n";
  write_ordered(o, m.pops.size(), 256, [&m](size_t a, size_t b, std::ostream &o) {
    for (size_t i = a; i < b; i++) {
      const Pop &p = m.pops[i];
      o << "population:" << i << "\n"
        << "NeuPopuName:" << p.name << ", N=" << p.N << " Taum=" << p.Taum << " Vth=" << p.Vth
        << " El=" << p.El << " g=" << p.gl << " Cm=" << p.Cm << " Vreset=" << p.Vreset << "\n";
      o << "Ek=0 gk=0 Ena=0 gna=0\n"
        << "AnA=0.01 AnB=-60 AnC=10 AnD=-1\n"
        << "BnA=0.125 BnB=-70 BnC=80 BnD=0\n"
        << "AmA=0.1 AmB=-45 AmC=10 AmD=-1\n"
        << "BmA=4 BmB=-70 BmC=18 BmD=0\n"
        << "AhA=0.07 AhB=-70 AhC=20 AhD=0\n"
        << "BhA=1 BhB=-40 BhC=10 BhD=1\n";
      o << "pv=" << p.pv << " tD=" << p.tD << " aF=" << p.aF << " tF=" << p.tF << " aCap=" << p.aCap
        << " tCap=" << p.tCap << " aCar=" << p.aCar << " tCar=" << p.tCar << "\n";
      o << "tLP=" << p.tLP << " SpiLPDy=" << p.SpiLPDy << " PosISI=" << p.PosISI
        << " NegISI=" << p.NegISI << "\n";
      for (const Receptor &r : p.reps) {
        o << "NeuRepName:" << rep_name(r.name, false) << ", Tau=" << r.Tau;
        if (r.name == KW_NMDA) o << ", TauXT=" << r.TauXT;
        o << " Vrv=" << r.Vrev << " FExt=" << r.FExt << " MnExtEff=" << r.MnExtEff
          << " MnExtCon=" << r.MnExtCon << "\n";
      }
      o << "\n";
      for (uint32_t j = p.link_beg; j < p.link_beg + p.link_num; j++) {
        const Link &l = m.links[j];
        o << "TarPopuName:" << m.pops[l.tgt].name << " TarReceptor:" << rep_name(l.rep, true)
          << ", Connectivity=" << l.conn << " MeanEff=" << l.eff << " weight=" << l.weight << "\n";
      }
      o << "------------------------------------------------------------------\n";
    }
  });
  o.flush();
  return bool(o);
}

}  // namespace fsh
