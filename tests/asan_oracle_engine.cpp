// Test infrastructure for the sanitizer build of the host code
// (tests/test_host_sanitizers.py): the four device-side entry points of the
// C ABI that the host code calls (fs_create, fs_destroy, fs_device_engine,
// fs_last_error), served by the CPU oracle (oracle/fs_oracle.cpp) instead of
// the GPU engine, so that the flysim command line, the parser, the network
// builder, the cache, the protocol loop and the output writers can run
// under AddressSanitizer and UndefinedBehaviorSanitizer on a machine without
// a GPU.  Only FS_MODE_COMPAT exists here (the oracle is its restatement).
#include <cstdlib>
#include "flysim_b200.h"

// Failure injection: with FLYSIM_TEST_FAIL_STEP=k the k-th step call of a
// run returns FS_ERR_CUDA after doing nothing, as a device error would.
namespace {
int g_calls = 0;
int (*g_step)(void *, uint32_t, fs_step_out *) = nullptr;
int failing_step(void *ctx, uint32_t n, fs_step_out *out) {
  const char *k = std::getenv("FLYSIM_TEST_FAIL_STEP");
  if (k && ++g_calls == std::atoi(k)) return FS_ERR_CUDA;
  return g_step(ctx, n, out);
}
fs_engine_vtbl g_engine;
}  // namespace

extern "C" {
void *oracle_create(const fs_net_desc *d);
void oracle_destroy(void *o);
const fs_engine_vtbl *oracle_engine(void);

int fs_create(const fs_net_desc *desc, const fs_run_opts *opts, fs_handle **out) {
  if (!desc || !opts || !out) return FS_ERR_ARG;
  *out = nullptr;
  if (opts->mode != FS_MODE_COMPAT) return FS_ERR_UNSUPPORTED;
  void *o = oracle_create(desc);
  if (!o) return FS_ERR_ARG;
  *out = static_cast<fs_handle *>(o);
  return FS_OK;
}

int fs_destroy(fs_handle *h) {
  oracle_destroy(h);
  return FS_OK;
}

const fs_engine_vtbl *fs_device_engine(void) {
  g_engine = *oracle_engine();
  g_step = g_engine.step;
  g_engine.step = failing_step;
  return &g_engine;
}

const char *fs_last_error(const fs_handle *) { return "CPU oracle engine (sanitizer build)"; }
}
