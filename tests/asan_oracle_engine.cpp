// Test infrastructure for the sanitizer build of the host code
// (tests/test_host_sanitizers.py): the four device-side entry points of the
// C ABI that the host code calls (fs_create, fs_destroy, fs_device_engine,
// fs_last_error), served by the CPU oracle (oracle/fs_oracle.cpp) instead of
// the GPU engine, so that the flysim command line, the parser, the network
// builder, the cache, the protocol loop and the output writers can run
// under AddressSanitizer and UndefinedBehaviorSanitizer on a machine without
// a GPU.  Only FS_MODE_COMPAT exists here (the oracle is its restatement).
#include "flysim_b200.h"

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

const fs_engine_vtbl *fs_device_engine(void) { return oracle_engine(); }

const char *fs_last_error(const fs_handle *) { return "CPU oracle engine (sanitizer build)"; }
}
