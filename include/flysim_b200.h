/*
 * flysim_b200.h — C ABI of the B200-native flysim step engine.
 *
 * The reference (yc-h/flysim) has no plugin or FFI layer.  Its seam for the
 * per-timestep integration is the abstract class NetSim (code/NetSim.h:80-109:
 * DoEvt, SetPp, RunInit, Run, FileOut), created by GetNewSim
 * (code/main.cpp:259-266).  Inside Run() the hot path is the pair
 * EqsGnl2::Activation / EqsGnl2::Spike (code/Eqs.h:928-930), called once per
 * step on state held in raw heap arrays owned by EqsGnl2 (code/Eqs.h:973-1118).
 *
 * This header replaces that seam with plain C entry points:
 *   - fs_model_*   host side: parse network.conf / network.pro and build the
 *                  network exactly as Parser::CSta/parse/DefMacro
 *                  (code/parser.cpp:51-1407) and NetSimGnl2::SetPp/PostSetPp
 *                  (code/NetSimGnl2_BulPp.cpp:27-727) do.  No GPU needed.
 *   - fs_create / fs_step / ...  device side: one handle owns all device
 *                  memory of one network instance on one GPU.
 *   - fs_batch_*   many independent instances advanced together (one CUDA
 *                  graph of tile-kernel launches per chunk of steps).
 *
 * Conventions: every call returns an int status (FS_OK = 0, >0 error codes
 * below); fs_last_error() gives a message.  No exceptions cross the ABI.
 * One host thread per handle.  No torch types anywhere.
 */
#ifndef FLYSIM_B200_H
#define FLYSIM_B200_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* 2: fs_syn_list gained ltp (the struct grew); fs_get_weights */
#define FS_ABI_VERSION 2

/* ---- status codes ------------------------------------------------------ */
enum {
  FS_OK = 0,
  FS_ERR_ARG = 1,          /* bad argument / inconsistent description      */
  FS_ERR_CUDA = 2,         /* CUDA runtime error (message has details)     */
  FS_ERR_NOMEM = 3,        /* device or host allocation failed             */
  FS_ERR_CAPACITY = 4,     /* an output buffer was too small               */
  FS_ERR_PARSE = 5,        /* .conf/.pro could not be parsed               */
  FS_ERR_UNSUPPORTED = 6,  /* network uses a feature the chosen mode lacks */
  FS_ERR_TIMEOUT = 7,      /* a bounded device wait gave up                */
  FS_ERR_IO = 8,           /* file open / write failed                     */
  FS_ERR_NODEVICE = 9      /* no CUDA device visible                       */
};

/* ---- receptor indices (order of EqsGnl2::BgInit, code/EqsGnl2.cpp:288-332) */
enum { FS_AMPA = 0, FS_GABA = 1, FS_ACH = 2, FS_GCL = 3, FS_NMDA = 4, FS_NREC = 5 };

/* ---- ActCtr bits: same values as code/Inc.h:253-280 --------------------- */
#define FS_ACT_AMPA 1u
#define FS_ACT_GABA 2u
#define FS_ACT_NMDA 4u
#define FS_ACT_GAP 8u
#define FS_ACT_ACH 32u
#define FS_ACT_GCL 64u
#define FS_ACT_INJ 128u
#define FS_ACT_LIF 256u
#define FS_ACT_LTP 8192u
#define FS_ACT_STD 16384u
#define FS_ACT_STP 32768u

/* ---- NState bits: same values as code/Inc.h:225-231 --------------------- */
#define FS_NS_FIRE 1u
#define FS_NS_SPIKE 2u
#define FS_NS_LP_FIRE 4u
#define FS_NS_LP_SPIKE 8u
#define FS_NS_MEMDV_OVF 16u
#define FS_NS_MEMDV_UDF 32u

/* ---- numeric modes ------------------------------------------------------ */
enum {
  /* FP32, reference operation order, std::mt19937 drive stream, ziggurat
   * injection noise: the spike raster equals the reference's (-t 1) bit for
   * bit.  Synaptic delays must be 0. */
  FS_MODE_COMPAT = 0,
  /* FP32 state, Philox drive, aggregated conductances with per-synapse
   * integer delays (delay ring), deterministic fixed-point delivery. */
  FS_MODE_FP32 = 1,
  /* Same algorithm as FS_MODE_FP32 with FP64 state: accuracy reference. */
  FS_MODE_FP64 = 2
};

/* ---- network description (plain arrays; copied at fs_create) ----------- */

/* Per-neuron parameters, all arrays of length n_neurons.  They are the fields
 * of ParBase2/ParLIF/NeuRepPar2<RP3,RP4>/ParStp2/ParLP2 of the reference
 * (code/neuron_affi.h:97-221, code/receptor.h:167-182) stored as structure of
 * arrays.  Receptor-indexed arrays are receptor-major: a[r * n + i]. */
typedef struct fs_neurons {
  uint32_t n;
  const float *Vth, *El, *gl, *Cm, *Vreset, *df, *ef, *dVmax;
  const int32_t *RfPed, *SpiDy;
  const float *Vrev;   /* [FS_NREC*n] */
  const float *dfst;   /* [FS_NREC*n] */
  const float *nmda_dfxt, *nmda_efst, *nmda_as, *nmda_mg;
  const float *ext_g;  /* [FS_NREC*n] efficacy of the external drive synapse */
  const float *pb;     /* [FS_NREC*n] initial drive probability per step     */
  const uint32_t *act; /* initial ActCtr bits                                */
  const float *inj_mean, *inj_std; /* initial injection current (nA)        */
  /* short-term plasticity (code/NetSimGnl2_BulPp.cpp:186-200) */
  const float *stp_pv, *stp_dfD, *stp_efD, *stp_aF, *stp_dfF, *stp_efF,
              *stp_aCap, *stp_dfCap, *stp_aCar, *stp_dfCar, *stp_efCar;
  /* long-term plasticity (code/NetSimGnl2_BulPp.cpp:180-183) */
  const float *ltp_dfLP, *ltp_PosISI, *ltp_NegISI;
  const int32_t *ltp_SpiLPDy;
} fs_neurons;

/* Reference-order synapse layout of one receptor (FS_MODE_COMPAT).
 *  group gates: one gate per (presynaptic neuron, link) with >=2 targets,
 *    (PSynFstGatA..L and PSynSloGat, code/NetSimGnl2_BulPp.cpp:393-464); the gate
 *    decays with dfst of its first target gate_post0.
 *  gather CSR by post: the gate indices summed into each post, in the order
 *    of the reference's sorted PSyn* arrays (code/EqsGnl2.cpp:941-979).
 *  single-target records: SynFst1/SynSlo1 (code/NetSimGnl2_BulPp.cpp:577-695)
 *    after PostSetPp's sort by PosID; rec_pre is the reference's PreID (the
 *    presynaptic POPULATION index, kept as the reference uses it). */
typedef struct fs_rec_layout {
  uint32_t n_gates;
  const uint32_t *gate_pre, *gate_post0;
  const float *gate_g;
  const uint32_t *gather_rowptr; /* [n+1] */
  const uint32_t *gather_gate;   /* [gather_rowptr[n]] */
  uint32_t n_recs;
  const uint32_t *rec_pre, *rec_post;
  const float *rec_g;
  const uint32_t *rec_rowptr;    /* [n+1] records of post i: [rowptr[i], rowptr[i+1]) */
  /* the presynaptic NEURON of each record (the production modes' gate of a
   * record is that neuron's); NULL: rec_pre read as a neuron index */
  const uint32_t *rec_src;
} fs_rec_layout;

typedef struct fs_compat_layout {
  fs_rec_layout rec[FS_NREC];
  /* gap junction terms per neuron, in the order the reference accumulates
   * them into Isyn (code/EqsGnl2.cpp:982-999 then :705-724):
   *   Isyn[i] += g * (V[other] - V[i]) */
  const uint32_t *gap_rowptr; /* [n+1] (may be NULL when there are none) */
  const uint32_t *gap_other;
  const float *gap_g;
} fs_compat_layout;

/* Flat synapse list for the production modes: one entry per (pre, post,
 * receptor).  delay is in steps (0 = effect on the next step, as the
 * reference).  ltp marks the entries whose weight long-term plasticity
 * rewrites when act_ctr has FS_ACT_LTP: the reference's single-target
 * records (SynFst1 / SynSlo1, code/EqsGnl2.cpp:1005-1044), not the links
 * of a population to several targets. */
typedef struct fs_syn_list {
  uint64_t n;
  const uint32_t *pre, *post;
  const uint8_t *rec;
  const float *g;
  const uint16_t *delay;     /* may be NULL: all zero */
  const uint8_t *ltp;        /* may be NULL: every entry */
} fs_syn_list;

/* Tsodyks-Markram short-term plasticity for the production modes, per
 * presynaptic neuron (arrays of length n, NULL = off for everybody).  The TM
 * state (u, x) of a synapse depends only on its presynaptic spike train and
 * these parameters, so it is kept once per presynaptic neuron. */
typedef struct fs_tm_params {
  const uint8_t *enabled;
  const float *U, *tau_rec, *tau_fac; /* ms */
} fs_tm_params;

typedef struct fs_net_desc {
  float dt;                 /* ms */
  uint32_t act_ctr;         /* global ActCtr (STP/STD/LTP mode bits)      */
  fs_neurons neurons;
  const fs_compat_layout *compat; /* required by FS_MODE_COMPAT           */
  const fs_syn_list *syn;         /* required by FS_MODE_FP32/FP64        */
  const fs_tm_params *tm;         /* optional (production modes)          */
} fs_net_desc;

typedef struct fs_run_opts {
  int mode;            /* FS_MODE_*                                       */
  int device;          /* CUDA device ordinal                             */
  uint32_t chunk_steps;/* steps per device launch batch (0 = default 1000)*/
  uint64_t philox_key; /* production modes: drive stream key              */
  uint32_t blocks_per_sm; /* production modes: resident blocks per SM of the
                             persistent kernel (0 = as many as fit, <= 4)  */
  uint32_t flags;      /* FS_RUN_* bits (0 = defaults)                     */
} fs_run_opts;

/* fs_run_opts.flags: run an FS_MODE_FP32 network whose delays are all 0 on
 * the interval kernel rather than the single-step kernel (for checks and
 * A/B timing; results are identical). */
#define FS_RUN_INTERVAL_KERNEL 1u
/* fs_run_opts.flags: run the network on the tile kernels (one launch pair
 * per batch of steps, blocks scheduled freely over tiles of posts), which
 * networks above ~150,000 neurons take by default; results are identical
 * to the persistent kernel's. */
#define FS_RUN_TILE_KERNELS 2u

/* Per-call step outputs (host memory, caller owned; NULL = not wanted). */
typedef struct fs_step_out {
  uint32_t *spike_count;   /* [nsteps]: number of neurons with SPIKE set   */
  uint32_t *spike_idx;     /* ascending neuron ids, steps concatenated     */
  uint64_t spike_cap;      /* capacity of spike_idx                         */
  uint64_t spike_total;    /* out: number written                           */
  float *V;                /* [nsteps*n] membrane potential after the step */
  float *Irep;             /* [nsteps*FS_NREC*n] receptor currents (Nets.Irep) */
  uint32_t *nstate;        /* [nsteps*n] NState after the step             */
  /* gating variables of selected single-target records (GatingVariable
   * output, code/NetSimGnl2_info.cpp:701-758).  In the production modes a
   * record's st is its presynaptic neuron's gate for the receptor (every
   * record of one neuron and receptor obeys the same recurrence) and an
   * NMDA record's (xt, st) are that neuron's NMDA x and s; the selection
   * needs the compat layout of the description (fs_net_desc.compat). */
  const uint32_t *gv_sel;  /* (receptor << 28) | record index in fs_rec_layout order */
  uint32_t gv_n;
  float *gv_st;            /* [nsteps*gv_n] st after the step              */
  float *gv_xt;            /* [nsteps*gv_n] xt after the step (NMDA)       */
} fs_step_out;

typedef struct fs_handle fs_handle;

/* ---- library ------------------------------------------------------------ */
int fs_abi_version(void);
const char *fs_last_error(const fs_handle *h); /* h may be NULL: global error */
int fs_device_count(int *count);

/* ---- device engine: replaces EqsGnl2's state + Activation/Spike -------- */
/* Allocates and uploads one network (code/NetSimGnl2_BulPp.cpp:27-727 is the
 * reference's equivalent set-up). */
int fs_create(const fs_net_desc *desc, const fs_run_opts *opts, fs_handle **out);
int fs_destroy(fs_handle *h);
/* VarInit + reseed (code/EqsGnl2.cpp:339-401, code/NetSimGnl2.cpp:313-330):
 * mt_seed seeds the std::mt19937 drive stream (compat), jcong_seed the
 * ziggurat congruential state (compat); production modes use philox_key and
 * mt_seed as the stream counter offset. */
int fs_reset(fs_handle *h, uint32_t mt_seed, uint32_t jcong_seed);
/* DoEvt (code/NetSimGnl2.cpp:52-141) expressed as parameter writes on the
 * neuron range [first, first+count).  They take effect at the next fs_step. */
int fs_set_drive(fs_handle *h, uint32_t first, uint32_t count, int rec, float pb);
int fs_set_act(fs_handle *h, uint32_t first, uint32_t count, uint32_t clear_mask, uint32_t set_mask);
int fs_set_injection(fs_handle *h, uint32_t first, uint32_t count, float mean, float std);
/* Runs nsteps steps of Activation+Spike (code/NetSimGnl2.cpp:231-264 minus
 * events and output) and returns what the output writers need.  The steps
 * run in chunks; FS_ERR_CAPACITY (spike_idx too small) is found after the
 * chunk that overflowed has run, so the handle has then advanced past what
 * was returned: reset it (fs_reset) or restore a checkpoint before going on. */
int fs_step(fs_handle *h, uint32_t nsteps, fs_step_out *out);
/* Device-resident variant for timing: runs nsteps with no host copies; the
 * per-step spike counts stay on the device. */
int fs_run(fs_handle *h, uint32_t nsteps);
/* fs_run bracketed by CUDA events on the engine stream; returns the device
 * time of the whole call (ms) after synchronising. */
int fs_run_timed(fs_handle *h, uint32_t nsteps, double *device_ms);
/* Launch layout of a production-mode handle: thread blocks and threads per
 * block of its persistent kernel, the steps between grid barriers, and
 * which kernels run it (kernel): 0 the persistent interval kernel, 1 the
 * single-step kernel (FS_MODE_FP32 networks whose delays are all 0 and that
 * have no gap junctions), 2 the tile kernels (large networks), 3 the
 * long-term plasticity kernel (networks with FS_ACT_LTP).  No counterpart
 * in the reference. */
int fs_engine_layout(fs_handle *h, uint32_t *blocks, uint32_t *threads, uint32_t *interval, int *kernel);
/* Synchronise and report counters. */
int fs_sync(fs_handle *h);
int fs_stats(fs_handle *h, uint64_t *steps_done, uint64_t *spikes_total, uint64_t *kernel_launches);
/* Average device duration (ms) of the dominant kernel over the launches
 * since the last fs_reset that a synchronising call (fs_sync, fs_run_timed,
 * fs_step) has accounted, measured with CUDA events on the engine stream
 * (one event pair per launch); launches = how many. */
int fs_kernel_time(fs_handle *h, double *ms_per_launch, uint64_t *launches);
/* Evaluates the device's glibc-exact float exp (the NMDA Mg-block exp of
 * FS_MODE_COMPAT) on k host values, for checks against the host libm. */
int fs_debug_expf(const float *x, float *y, uint64_t k);
/* Allocation-free variant of fs_debug_expf; no counterpart in the reference.
 * For callers that must not allocate device memory per call: a process whose
 * caching allocator already holds the device's free memory, or a host thread
 * checking expf while a long fs_run is in flight (fs_debug_expf's cudaFree
 * waits for the work in flight on the device).  Same kernel and results as
 * fs_debug_expf, staged through one fixed 4 MiB static device array, so at
 * most FS_NOALLOC_MAX_K values per call; a larger k returns FS_ERR_ARG.
 * The first call on each device does a one-time set-up (scratch address
 * lookup, upload of the expf exception table): make it before any stream
 * capture begins.  All calls on one device share the scratch: overlapping
 * calls (several host threads at once) race, so serialise them.  Nothing in
 * the scratch has to start at zero.  Runs on the calling thread's default
 * stream (cudaStreamPerThread) and returns when y is written. */
#define FS_NOALLOC_MAX_K 262144u
int fs_debug_expf_noalloc(const float *x, float *y, uint64_t k);
/* Failure-detection check: a kernel waits at a grid barrier that a missing
 * block never reaches.  Every device wait in this library is bounded (the
 * production kernels' interval barrier gives up after 2^24 polls); here the
 * bound is poll_limit (1 .. 2^24), after which the kernel sets its error word
 * and returns.  Returns FS_ERR_TIMEOUT (the expected outcome), and the device
 * stays usable for the next call.  The reference has no counterpart: its
 * step threads meet at condition-variable waits with no time limit
 * (code/NetSimGnl2.cpp:198-224) and are joined at the end (:348). */
int fs_debug_barrier_timeout(uint32_t poll_limit);
/* Checks of the production modes' external drive against a CPU restatement;
 * no counterpart in the reference, whose drive is one sequential
 * std::mt19937 stream (code/EqsGnl2.cpp:284-337) and ziggurat normal
 * (code/StiExt.h:214-218).
 * fs_debug_philox: the device Philox-4x32-10 on k blocks, ctr [k][4] and
 * key [k][2] in, out [k][4].
 * fs_debug_drive: the drive draws of steps [t0, t0 + nsteps) (t counted from
 * the last fs_reset) of neurons [first, first + count) with the handle's
 * stream key and current drive and injection parameters, computed by the
 * function the engine's kernels call: hits [nsteps][count], bit r set when
 * receptor r (FS_AMPA .. FS_NMDA) is hit; gauss [nsteps][count], the
 * injection current (nA, 0 where injection is off).  Production modes. */
int fs_debug_philox(const uint32_t *ctr, const uint32_t *key, uint64_t k, uint32_t *out);
int fs_debug_drive(fs_handle *h, uint64_t t0, uint32_t nsteps, uint32_t first, uint32_t count, uint8_t *hits,
                   double *gauss);
/* Host-only check of the single-step kernel's plan for a network (no device
 * needed): builds the per-block tables for sm_count blocks and verifies every
 * index the kernel forms from them.  stats[8]: [0] 1 if the network takes
 * the single-step kernel, [1] blocks, [2] max posts, [3] max tracked
 * neurons, [4] max NMDA edges per block, [5] shared-memory bytes, [6]
 * linear delivery entries, [7] NMDA edges.  FS_ERR_ARG names a violated
 * bound.  No counterpart in the reference. */
int fs_debug_single_step_plan(const fs_net_desc *desc, uint32_t sm_count, uint64_t *stats);
/* Phase clock of the persistent kernels (a profiling aid; no counterpart in
 * the reference).  fs_debug_phase_clock(h, 1) zeroes and switches on
 * per-block counters of SM cycles per phase, 0 switches them off;
 * fs_debug_phase_times copies up to cap counters, [blocks][16], and the
 * block count.  Phases: single-step kernel 0 spike-list lookups, 1 NMDA
 * copies of listed spikes, 2 last deliveries and NMDA sums, 3 neuron steps,
 * 6 thread 0's wait at the grid barrier, 4 the rest of the barrier (the
 * other warps' drive draws and NMDA copies), 5 set-up, and laps inside a
 * phase (cycles from its start): 8 the list's entry count loaded, 9 the
 * look-ups done, 10 warp 0's deliveries issued, 11 warp 0 out of posts to
 * sum, 12 thread 0's list entries loaded, 13 warp 0's neuron steps done; interval kernel 0 NMDA pull, 1 drive draws, 2 neuron steps,
 * 3 pushes, 4 grid barrier.  The tile kernels have no phase clock. */
int fs_debug_phase_clock(fs_handle *h, int enable);
int fs_debug_phase_times(fs_handle *h, uint64_t *out, uint32_t cap, uint32_t *blocks);
/* Failure detection on the host side: stores into the handle's device error
 * word what a bounded device wait that gave up stores, without running or
 * stopping any kernel, so that the paths which must notice it (fs_sync,
 * fs_checkpoint_save) can be checked.  Production modes; the handle's next
 * fs_reset or fs_checkpoint_load clears it. */
int fs_debug_inject_wait_failure(fs_handle *h);
/* Checkpoints of a production-mode handle (FS_MODE_FP32 / FS_MODE_FP64).
 * The reference parses a SaveAllStates output and Resume event subtypes
 * (code/parser.cpp:1167-1176, :1254-1258) but implements neither; here a
 * checkpoint holds everything a step reads from the steps before it: the
 * step counter and drive stream key, the event-set parameters (drive,
 * receptor switches, injection), the synaptic gains, every neuron, receptor,
 * plasticity and spike-count state array, the NMDA s history and the delay
 * ring with the pushes already made for future steps.  A handle created
 * from the same description and mode continues from fs_checkpoint_load
 * exactly as the saved handle would (bit for bit: the drive draws are a
 * function of the step counter and key).  fs_checkpoint_size gives the
 * buffer size; loading a checkpoint of another network or mode returns
 * FS_ERR_ARG; the compat mode returns FS_ERR_UNSUPPORTED.  fs_checkpoint_save
 * first waits for the work in flight and returns FS_ERR_TIMEOUT, saving
 * nothing, when a device wait of that work gave up. */
int fs_checkpoint_size(fs_handle *h, uint64_t *bytes);
int fs_checkpoint_save(fs_handle *h, void *buf, uint64_t cap, uint64_t *bytes);
int fs_checkpoint_load(fs_handle *h, const void *buf, uint64_t bytes);
/* Copy state out (V, Count, NState) for checks; arrays of length n. */
int fs_get_state(fs_handle *h, float *V, int32_t *Count, uint32_t *NState);
/* The synaptic weights as long-term plasticity has made them, in the order
 * of the description's fs_syn_list (n = its length): the g of the
 * reference's records (code/EqsGnl2.cpp:1005-1044), which it never writes
 * out.  Production modes, networks with FS_ACT_LTP (the weights of other
 * networks do not change); otherwise FS_ERR_UNSUPPORTED. */
int fs_get_weights(fs_handle *h, float *g, uint64_t n);
/* Full conductance view for checks: RVs (FS_NREC*n) after the last step and
 * Isyn (n). */
int fs_get_syn_state(fs_handle *h, float *g, float *Isyn);

/* ---- host model: parser + network builder (no GPU) --------------------- */
typedef struct fs_model fs_model;
typedef struct fs_model_opts {
  float dt;              /* -dt (ms), default 0.1 */
  uint32_t flags;        /* FS_ACT_STP / FS_ACT_STD / FS_ACT_LTP as on the CLI */
  int user_seed_set;     /* -udfsed given (sets the STD bit too, as the reference) */
  uint32_t user_seed;
  int threads;           /* -t (affects set-up RNG draws only)          */
  int repeats;           /* -rp                                          */
  const char *out_mem, *out_spike, *out_rate; /* -om/-os/-or or NULL     */
} fs_model_opts;

int fs_model_load(const char *conf_path, const char *pro_path, const fs_model_opts *opts, fs_model **out);
/* fs_model_load through a binary network cache at cache_path (no
 * counterpart in the reference, which parses and builds from text on every
 * run, code/main.cpp:216-249).  The cache is keyed by the bytes of both files
 * and by opts: when the key matches, the model is read back without parsing
 * or building; otherwise the files are parsed and built and the cache is
 * (re)written.  A cache that cannot be written does not fail the load.
 * cache_status (may be NULL) receives one of FS_CACHE_*.  cache_path NULL or
 * "" behaves as fs_model_load. */
enum { FS_CACHE_OFF = 0, FS_CACHE_HIT = 1, FS_CACHE_STORED = 2, FS_CACHE_UNWRITABLE = 3, FS_CACHE_UNSEEDED = 4 };
/* FS_CACHE_UNSEEDED: the network has no fixed seed (neither -udfsed nor a
 * RandomSeeds macro), so, as in the reference, every load draws a new seed
 * from std::random_device and builds new connectivity from it; such a model
 * is loaded from the text files and never cached. */
int fs_model_load_cached(const char *conf_path, const char *pro_path, const fs_model_opts *opts,
                         const char *cache_path, fs_model **out, int *cache_status);
int fs_model_free(fs_model *m);
const char *fs_model_error(void);
/* Writes ConfsInfo.log for the parsed model (Parser::ConfsInfo,
 * code/parser.cpp:1488-1631); the reference CLI writes it on every run
 * (code/main.cpp:247). */
int fs_model_confs_info(fs_model *m, const char *path);
/* Writes network.log for the built network (NetSimGnl2::logDataWrite,
 * code/NetSimGnl2_info.cpp:93-546: per-neuron parameters, every synapse,
 * events, output columns); the reference writes it before the first repeat
 * (code/NetSimGnl2.cpp:143-157).  Text of O(neurons + synapses) size. */
int fs_model_network_log(fs_model *m, const char *path);
/* View of the built network (valid until fs_model_free). */
int fs_model_desc(fs_model *m, const fs_net_desc **desc);
int fs_model_info(fs_model *m, uint32_t *n_neurons, uint32_t *n_pops, uint64_t *n_syn_entries,
                  uint32_t *n_events, uint32_t *n_outputs);
/* Seed used by repeat r (1-based), as rseeds[r-1] of the reference. */
int fs_model_seed(fs_model *m, int repeat, uint32_t *seed);
/* Runs the full protocol (all repeats) on the device engine and writes the
 * output files of the .pro, exactly as NetSimGnl2::Run/FileOut
 * (code/NetSimGnl2.cpp:266-358, code/NetSimGnl2_info.cpp:548-769). */
int fs_model_run(fs_model *m, const fs_run_opts *opts, const char *out_dir, double *run_seconds);

/* Engine plug-in: the NetSim seam as a table of C function pointers.  The
 * protocol driver (events, repeats, output files) calls these; fs_model_run
 * plugs in the device engine. */
typedef struct fs_engine_vtbl {
  int (*reset)(void *ctx, uint32_t mt_seed, uint32_t jcong_seed);
  int (*set_drive)(void *ctx, uint32_t first, uint32_t count, int rec, float pb);
  int (*set_act)(void *ctx, uint32_t first, uint32_t count, uint32_t clear_mask, uint32_t set_mask);
  int (*set_injection)(void *ctx, uint32_t first, uint32_t count, float mean, float std);
  int (*step)(void *ctx, uint32_t nsteps, fs_step_out *out);
  const char *(*error)(void *ctx);
} fs_engine_vtbl;
int fs_model_run_with(fs_model *m, const fs_engine_vtbl *eng, void *ctx, const char *out_dir,
                      uint32_t chunk_steps, double *run_seconds);
/* The device engine's table (ctx = fs_handle*). */
const fs_engine_vtbl *fs_device_engine(void);

/* Per-neuron spike counts since the last fs_reset (production modes; n
 * entries).  The per-population rates of a FiringRate output are sums of
 * these (code/NetSimGnl2_info.cpp:660-700). */
int fs_spike_counts(fs_handle *h, uint32_t *counts);

/* ---- batches: many independent networks advanced together --------------
 * The generalisation of the reference's repeat loop (-rp, code/main.cpp:
 * 251-252) to instances that differ in size, parameters and seed, as the
 * seizure-like E/I-gain scans need.  Every instance is a production-mode
 * network (FP32 or FP64) with its own state.  All instances' posts are cut
 * into tiles; each batch of steps (at most the smallest interval of the
 * instances, and 16) is one pair of launches over every tile of every
 * instance (NMDA pull, then the neurons' steps and spike pushes), the blocks
 * scheduled freely over the tiles, and a chunk of steps is captured once
 * into a CUDA graph and replayed.  Any number of instances fits.  An
 * instance's results are identical to running it alone with fs_create /
 * fs_run (same seed and philox_key). */
typedef struct fs_batch fs_batch;
typedef struct fs_batch_plan {
  uint32_t blocks;        /* thread blocks of each launch: tiles of posts    */
  uint32_t blocks_per_sm; /* resident step-kernel blocks per SM              */
  uint32_t candidates;    /* configurations the tuner timed                  */
  uint32_t tile_posts;    /* posts per tile                                  */
  uint32_t edges_in_flight; /* NMDA edges in flight per lane in the pull     */
  double sample_ms;       /* device time of the chosen plan's sample run     */
} fs_batch_plan;
/* opts: mode FS_MODE_FP32 (default) or FS_MODE_FP64, device, chunk_steps
 * (steps per graph replay, default 10000), philox_key. */
int fs_batch_create(uint32_t count, const fs_net_desc *const *descs, const fs_run_opts *opts, fs_batch **out);
int fs_batch_destroy(fs_batch *b);
const char *fs_batch_error(const fs_batch *b); /* b may be NULL */
/* seeds: one per instance (NULL = the previous seeds, initially 1). */
int fs_batch_reset(fs_batch *b, const uint32_t *seeds);
/* Autotuner: times sample_steps (0 = 200) for each candidate plan (posts
 * per tile 64 / 128 / 256 x NMDA edges in flight per lane 4 / 8), keeps the
 * fastest and resets every instance (its seed unchanged).  Results never
 * depend on the plan. */
int fs_batch_tune(fs_batch *b, uint32_t sample_steps, fs_batch_plan *plan);
/* Advances every instance by nsteps; device_ms = device time of the call. */
int fs_batch_run(fs_batch *b, uint32_t nsteps, double *device_ms);
int fs_batch_info(fs_batch *b, uint32_t *count, uint32_t *blocks, uint32_t *blocks_per_sm, int *graph,
                  uint64_t *launches);
/* Per-neuron spike counts of instance inst since its reset. */
int fs_batch_spike_counts(fs_batch *b, uint32_t inst, uint32_t *counts);
/* Total spikes of every instance since its reset (count entries). */
int fs_batch_spike_totals(fs_batch *b, uint64_t *totals);
/* Synaptic gains per receptor (FS_AMPA .. FS_NMDA; 1 = the weights as
 * built): every recurrent weight of receptor r is scaled by gains[r], the
 * analogue of the reference's per-population efficacy factors that its
 * seizure scans vary (experiment/seizure/readme:1-6).  Production modes;
 * takes effect at the next run. */
int fs_set_gains(fs_handle *h, const float *gains);
int fs_batch_set_gains(fs_batch *b, uint32_t inst, const float *gains);
/* Drive probabilities of every neuron of instance inst, pb[FS_NREC * n]
 * (receptor-major, as fs_neurons.pb). */
int fs_batch_set_drive(fs_batch *b, uint32_t inst, const float *pb);

/* ---- mean-field surrogate (no counterpart in the reference) -------------
 * A multilayer perceptron with ReLU hidden layers, BF16 weights and
 * activations and FP32 accumulation on the tensor cores (tcgen05), trained
 * with Adam on rates the batched engine produced.  dims = {inputs, hidden...,
 * outputs}, every width in [1, 256]; the last output is a hyperactivity
 * logit and the others regress log(1 + rate).  Loss per batch: mean squared
 * error over the rate outputs plus binary cross-entropy of the logit.
 * Parameters in the host-side vectors are, per layer, W [out x in]
 * row-major followed by b [out].  Errors: fs_mlp_error(). */
typedef struct fs_mlp fs_mlp;
const char *fs_mlp_error(void);
int fs_mlp_create(const uint32_t *dims, uint32_t ndims, int device, uint64_t seed, fs_mlp **out);
int fs_mlp_destroy(fs_mlp *m);
uint64_t fs_mlp_param_count(const fs_mlp *m);
int fs_mlp_get_params(fs_mlp *m, float *params);
int fs_mlp_set_params(fs_mlp *m, const float *params);
/* y[rows x outputs] = network(x[rows x inputs]); host arrays. */
int fs_mlp_forward(fs_mlp *m, const float *x, uint64_t rows, float *y, double *device_ms);
/* Gradients of the loss over one batch (rows a multiple of 16, <= 256),
 * targets t[rows x outputs]; no update. */
int fs_mlp_grad(fs_mlp *m, const float *x, const float *t, uint32_t rows, float *grads, float *loss);
/* Adam, batches of 256 rows in a fresh shuffle per epoch (rows beyond a
 * multiple of 256 are left out of that epoch); epoch_loss[epochs] or NULL. */
int fs_mlp_train(fs_mlp *m, const float *x, const float *t, uint64_t rows, uint32_t epochs, float lr,
                 uint64_t seed, float *epoch_loss, double *device_ms);
/* One tensor-core GEMM for checks: c[m x n] = a[m x k] . b[n x k]^T (+ bias,
 * ReLU), a and b BF16 bit patterns, n and k multiples of 16 up to 256. */
int fs_mlp_gemm(const uint16_t *a, const uint16_t *b, uint32_t m, uint32_t n, uint32_t k, const float *bias,
                int relu, float *c);

#ifdef __cplusplus
}
#endif
#endif
