// Internal host-side types of the flysim drop-in: configuration model,
// built network, protocol driver.  Not part of the C ABI.
#pragma once
#include <cstdint>
#include <string>
#include <vector>
#include <random>
#include <sstream>
#include <thread>
#include "flysim_b200.h"

namespace fsh {

// Parser keyword ids (same values as code/Inc.h:35-47).
enum : uint8_t { KW_AMPA = 0, KW_GABA = 1, KW_NMDA = 2, KW_GAP = 3, KW_CUBA = 4, KW_SINE = 5,
                 RSM_SYNCOND = 6, RSM_GATVAR = 7, RSM_MEMPOT = 8, RSM_RNDSED = 9, RSM_ALL = 10,
                 KW_ACH = 11, KW_GCL = 12 };
// Output type ids (code/Inc.h:183-193).
enum { OUT_MEMPOT = 1, OUT_SPIKE = 2, OUT_FRATE = 3, OUT_GATVAR = 5, OUT_ISYNSEP = 6,
       OUT_SAVE = 7, OUT_SYNWGT = 9, OUT_DVOVF = 10 };
enum { OF_ALIGN = 1, OF_SUMALL = 2 };
enum { EVT_EXTFREQ = 1, EVT_CURINJ = 2 };

constexpr float kVResting = -70.0f;  // code/Inc.h:25
constexpr float kVReset = -50.0f;    // code/Inc.h:26
constexpr float kCarBase = 20.0f;    // code/Inc.h:27

struct Receptor {  // NeuRep, defaults of code/parser.cpp:187-193
  uint8_t name = KW_AMPA;
  float Tau = 5.0f, TauXT = 2.0f, Vrev = 0.0f, FExt = 0.0f, MnExtEff = 2.1f, MnExtCon = 1.0f;
};

struct Link {  // NeuCon, defaults of code/parser.cpp:220-224
  uint32_t tgt = 0;
  uint8_t rep = KW_AMPA;
  float conn = 1.0f, eff = 0.0f, weight = 1.0f;
  float delay_ms = 0.0f;  // extension keyword "Delay" (ignored by the reference parser)
};

struct Pop {  // NetConfSta + NetConf + ParStp + ParLP
  std::string name;
  uint32_t N = 0, nrep = 0, link_beg = 0, link_num = 0;
  bool selcon = false;
  std::vector<Receptor> reps;
  float Taum = 2.0f, Vth = -50.0f, El = kVResting, gl = 2.5f, Cm = 1.0f, Vreset = kVReset;
  int RfPed = 0, SpiDy = 0;
  float pv = 0.6f, tD = 300.0f, aF = 0.0035f, tF = 7000.0f, aCap = 250.0f, tCap = 2.0f,
        aCar = 0.1f, tCar = 2000.0f;
  float tLP = 50.0f;
  int SpiLPDy = 0;
  float PosISI = 1e-5f, NegISI = 1e-5f;
};

struct Event {  // TmEvt (code/parser_affi.cpp:17-28)
  float TimEv = 0.0f;
  bool NoLmt = false;
  uint32_t Type = 0, Pp = 0;
  uint8_t SubTyp = KW_AMPA;
  float Var1 = 0.0f, Var2 = 0.0f;
};

struct OutCtl {  // OutCtr (code/parser_affi.cpp:55-65)
  uint32_t Status = 0;
  std::string Type = "Non";
  int TypeID = 0;
  std::string FileName = "Non";
  std::vector<uint32_t> ParList;
  uint32_t RWin = 50, FPnt = 100;
  float TimEv = 0.0f;
  std::vector<uint32_t> SpiRWin;
};

struct Group { std::string name; std::vector<uint32_t> pops; };

// Built network: the SoA arrays handed to the engines.
struct Network {
  uint32_t n = 0;
  std::vector<uint32_t> nidx;  // first neuron of each population
  std::vector<float> Vth, El, gl, Cm, Vreset, df, ef, dVmax;
  std::vector<int32_t> RfPed, SpiDy;
  std::vector<float> Vrev, dfst, ext_g, pb;  // [FS_NREC*n]
  std::vector<float> nmda_dfxt, nmda_efst, nmda_as, nmda_mg;
  std::vector<uint32_t> act;
  std::vector<float> inj_mean, inj_std;
  std::vector<float> stp_pv, stp_dfD, stp_efD, stp_aF, stp_dfF, stp_efF, stp_aCap, stp_dfCap,
      stp_aCar, stp_dfCar, stp_efCar;
  std::vector<float> ltp_dfLP, ltp_PosISI, ltp_NegISI;
  std::vector<int32_t> ltp_SpiLPDy;

  struct RecArrays {
    std::vector<uint32_t> gate_pre, gate_post0;
    std::vector<float> gate_g;
    std::vector<uint32_t> gather_rowptr, gather_gate;
    std::vector<uint32_t> rec_pre, rec_post;
    std::vector<float> rec_g;
    std::vector<uint32_t> rec_rowptr;
    std::vector<uint32_t> rec_src;  // presynaptic neuron of each record
    // group segments in the reference's order (posts ascending; for GluCl the
    // post read through the Ach map): segment s holds seg_len[s] gather
    // entries of post seg_post[s].  Only network.log reads these.
    std::vector<uint32_t> seg_post, seg_len;
  } rec[FS_NREC];
  std::vector<uint32_t> gap_rowptr, gap_other;
  std::vector<float> gap_g;
  // for network.log: single-target gap records sorted by post (PreID is the
  // population index) and, per post, how many group gap terms open its
  // gap_other row
  std::vector<uint32_t> gap1_pre, gap1_post, gap_ngroup;
  std::vector<float> gap1_g;

  // flat synapse list for the production modes
  std::vector<uint32_t> syn_pre, syn_post;
  std::vector<uint8_t> syn_rec;
  std::vector<float> syn_g;
  std::vector<uint16_t> syn_delay;
  std::vector<uint8_t> syn_ltp;  // 1: a single-target record (LTP rewrites its weight)

  uint64_t total_synapses = 0;  // TolSynp of the reference
  // C views
  fs_compat_layout compat{};
  fs_syn_list syn{};
  fs_net_desc desc{};
  void make_views(float dt, uint32_t act_ctr);
};

struct Model {
  fs_model_opts opts{};
  float dt = 0.1f;
  uint32_t act_ctr = 0;
  std::vector<Pop> pops;
  std::vector<Link> links;
  std::vector<Group> groups;
  std::vector<uint32_t> macro_seeds;
  std::vector<Event> events;
  std::vector<OutCtl> outs;
  std::vector<uint32_t> rseeds;
  std::string out_mem = "MemPot.dat", out_spike = "Spikes.dat", out_rate = "FRate.dat";
  bool comm_mem = false, comm_spike = false, comm_rate = false;
  Network net;
};

// Parsing (code/parser.cpp) and building (code/NetSimGnl2_BulPp.cpp).
void parse_conf_counts(Model &m, const std::string &path, int &state);
void parse_conf(Model &m, const std::string &path, int &state);
void parse_macros(Model &m, const std::string &path, int &state);
void parse_pro(Model &m, const std::string &path, int &state);
void add_command_outputs(Model &m);
bool write_confs_info(const Model &m, const std::string &path);
bool write_network_log(const Model &m, const std::string &path);
void build_network(Model &m);

// Formats items [0, count) in blocks of `block` on the host cores and writes
// the blocks to o in item order; fmt(a, b, os) formats items [a, b).  Used by
// the text logs, whose number formatting dominates their cost.
template <class F>
void write_ordered(std::ostream &o, size_t count, size_t block, F fmt) {
  unsigned hw = std::thread::hardware_concurrency();
  const unsigned T = hw < 1 ? 1 : (hw > 16 ? 16 : hw);
  std::vector<std::string> out(T);
  for (size_t base = 0; base < count; base += (size_t)T * block) {
    std::vector<std::thread> th;
    for (unsigned t = 0; t < T; t++) {
      const size_t a = base + (size_t)t * block;
      if (a >= count) break;
      const size_t b = a + block < count ? a + block : count;
      th.emplace_back([&out, &fmt, t, a, b] {
        std::ostringstream s;
        fmt(a, b, s);
        out[t] = s.str();
      });
    }
    for (auto &x : th) x.join();
    for (size_t t = 0; t < th.size(); t++) o << out[t];
  }
}

// Binary network cache (fs_cache.cpp).
bool cache_key(const char *conf, const char *pro, const fs_model_opts &o, uint64_t &key);
bool cache_read(const std::string &path, uint64_t key, Model &m);
bool cache_write(const std::string &path, uint64_t key, Model &m, std::string &err);

// Protocol driver: NetSimGnl2::Run/DoEvt/FileOut over any engine.
int run_protocol(Model &m, const fs_engine_vtbl *eng, void *ctx, const std::string &out_dir,
                 uint32_t chunk_steps, double *run_seconds, std::string &err);

struct ParseError : std::exception {
  std::string msg;
  explicit ParseError(std::string s) : msg(std::move(s)) {}
  const char *what() const noexcept override { return msg.c_str(); }
};

}  // namespace fsh
