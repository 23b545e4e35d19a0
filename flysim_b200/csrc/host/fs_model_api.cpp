// C ABI of the host model (parser + builder + protocol driver).
#include <cmath>
#include <cstring>
#include <string>
#include <mutex>
#include "fs_host.hpp"

struct fs_model {
  fsh::Model m;
  std::string err;
};

namespace {
thread_local std::string g_model_err;
}

extern "C" {

const char *fs_model_error(void) { return g_model_err.c_str(); }

// main.cpp:216-249 order: CSta, parse(conf), Comm, DefMacro, parse(pro), SetPp.
int fs_model_load(const char *conf_path, const char *pro_path, const fs_model_opts *opts,
                  fs_model **out) {
  return fs_model_load_cached(conf_path, pro_path, opts, nullptr, out, nullptr);
}

int fs_model_load_cached(const char *conf_path, const char *pro_path, const fs_model_opts *opts,
                         const char *cache_path, fs_model **out, int *cache_status) {
  if (cache_status) *cache_status = FS_CACHE_OFF;
  if (!conf_path || !pro_path || !out) {
    g_model_err = "fs_model_load: null argument";
    return FS_ERR_ARG;
  }
  *out = nullptr;
  fs_model *fm = new (std::nothrow) fs_model();
  if (!fm) return FS_ERR_NOMEM;
  fsh::Model &m = fm->m;
  fs_model_opts o{};
  o.dt = 0.1f;
  o.threads = 1;
  o.repeats = 1;
  if (opts) o = *opts;
  if (!(o.dt > 0.0f) || !std::isfinite(o.dt)) o.dt = 0.1f;
  if (o.threads < 1) o.threads = 1;
  if (o.repeats < 1) o.repeats = 1;
  uint64_t key = 0;
  bool use_cache = cache_path && *cache_path && fsh::cache_key(conf_path, pro_path, o, key);
  if (use_cache && fsh::cache_read(cache_path, key, m)) {
    m.opts.out_mem = m.opts.out_spike = m.opts.out_rate = nullptr;
    if (cache_status) *cache_status = FS_CACHE_HIT;
    *out = fm;
    return FS_OK;
  }
  if (use_cache) {  // a miss may have left part of a damaged file in m
    delete fm;
    fm = new (std::nothrow) fs_model();
    if (!fm) return FS_ERR_NOMEM;
  }
  fsh::Model &mm = fm->m;
  mm.opts = o;
  mm.dt = o.dt;
  // GetNewSim's ActCtr and the CLI flags (code/main.cpp:220-231, :263)
  mm.act_ctr = FS_ACT_AMPA | FS_ACT_GABA | FS_ACT_NMDA | FS_ACT_ACH | FS_ACT_GCL | FS_ACT_GAP | FS_ACT_LIF;
  if (o.user_seed_set) mm.act_ctr |= FS_ACT_STD;  // UDFRDSEED_ACT == STD_ACT
  else mm.act_ctr &= ~FS_ACT_STD;
  mm.act_ctr |= (o.flags & (FS_ACT_STP | FS_ACT_STD | FS_ACT_LTP));
  if (o.out_mem) { mm.comm_mem = true; mm.out_mem = o.out_mem; }
  if (o.out_spike) { mm.comm_spike = true; mm.out_spike = o.out_spike; }
  if (o.out_rate) { mm.comm_rate = true; mm.out_rate = o.out_rate; }
  try {
    int state = 0;
    fsh::parse_conf_counts(mm, conf_path, state);
    fsh::parse_conf(mm, conf_path, state);
    fsh::add_command_outputs(mm);
    fsh::parse_macros(mm, pro_path, state);
    fsh::parse_pro(mm, pro_path, state);
    fsh::build_network(mm);
  } catch (const std::exception &e) {
    g_model_err = e.what();
    delete fm;
    return FS_ERR_PARSE;
  }
  // keep views valid for the model's life; options strings are not kept
  mm.opts.out_mem = mm.opts.out_spike = mm.opts.out_rate = nullptr;
  // A network seeded by std::random_device (no -udfsed, no RandomSeeds
  // macro) gets a fresh seed, and with it fresh connectivity and drive, on
  // every run of the reference (code/NetSimGnl2_BulPp.cpp:80-88); a cached
  // copy would replay one draw forever, so such a model is never stored.
  const bool random_seed = !(mm.act_ctr & FS_ACT_STD) && mm.macro_seeds.empty();
  if (use_cache && random_seed) {
    if (cache_status) *cache_status = FS_CACHE_UNSEEDED;
  } else if (use_cache) {
    std::string err;
    bool stored = fsh::cache_write(cache_path, key, mm, err);
    if (!stored) g_model_err = err;
    if (cache_status) *cache_status = stored ? FS_CACHE_STORED : FS_CACHE_UNWRITABLE;
  } else if (cache_path && *cache_path) {
    if (cache_status) *cache_status = FS_CACHE_UNWRITABLE;
    g_model_err = "network cache: cannot read the .conf or .pro for the cache key";
  }
  *out = fm;
  return FS_OK;
}

int fs_model_free(fs_model *m) {
  delete m;
  return FS_OK;
}

int fs_model_confs_info(fs_model *m, const char *path) {
  if (!m || !path) return FS_ERR_ARG;
  bool ok = false;
  try {
    ok = fsh::write_confs_info(m->m, path);
  } catch (const std::exception &e) {
    g_model_err = e.what();
    return FS_ERR_IO;
  }
  if (!ok) {
    g_model_err = std::string("cannot write ") + path;
    return FS_ERR_IO;
  }
  return FS_OK;
}

int fs_model_network_log(fs_model *m, const char *path) {
  if (!m || !path) return FS_ERR_ARG;
  bool ok = false;
  try {
    ok = fsh::write_network_log(m->m, path);
  } catch (const std::exception &e) {
    g_model_err = e.what();
    return FS_ERR_IO;
  }
  if (!ok) {
    g_model_err = std::string("cannot write ") + path;
    return FS_ERR_IO;
  }
  return FS_OK;
}

int fs_model_desc(fs_model *m, const fs_net_desc **desc) {
  if (!m || !desc) return FS_ERR_ARG;
  *desc = &m->m.net.desc;
  return FS_OK;
}

int fs_model_info(fs_model *m, uint32_t *n_neurons, uint32_t *n_pops, uint64_t *n_syn_entries,
                  uint32_t *n_events, uint32_t *n_outputs) {
  if (!m) return FS_ERR_ARG;
  if (n_neurons) *n_neurons = m->m.net.n;
  if (n_pops) *n_pops = (uint32_t)m->m.pops.size();
  if (n_syn_entries) *n_syn_entries = m->m.net.total_synapses;
  if (n_events) *n_events = (uint32_t)m->m.events.size();
  if (n_outputs) *n_outputs = (uint32_t)m->m.outs.size();
  return FS_OK;
}

int fs_model_seed(fs_model *m, int repeat, uint32_t *seed) {
  if (!m || !seed || repeat < 1 || repeat > (int)m->m.rseeds.size()) return FS_ERR_ARG;
  *seed = m->m.rseeds[repeat - 1];
  return FS_OK;
}

int fs_model_run_with(fs_model *m, const fs_engine_vtbl *eng, void *ctx, const char *out_dir,
                      uint32_t chunk_steps, double *run_seconds) {
  if (!m || !eng) {
    g_model_err = "fs_model_run_with: null argument";
    return FS_ERR_ARG;
  }
  std::string err;
  int rc = fsh::run_protocol(m->m, eng, ctx, out_dir ? out_dir : "", chunk_steps, run_seconds, err);
  if (rc) g_model_err = err;
  return rc;
}

int fs_model_run(fs_model *m, const fs_run_opts *opts, const char *out_dir, double *run_seconds) {
  if (!m) return FS_ERR_ARG;
  fs_run_opts o{};
  if (opts) o = *opts;
  fs_handle *h = nullptr;
  int rc = fs_create(&m->m.net.desc, &o, &h);
  if (rc) {
    g_model_err = fs_last_error(nullptr);
    return rc;
  }
  rc = fs_model_run_with(m, fs_device_engine(), h, out_dir, o.chunk_steps, run_seconds);
  fs_destroy(h);
  return rc;
}

}  // extern "C"
