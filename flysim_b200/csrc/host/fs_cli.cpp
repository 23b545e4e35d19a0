// flysim — command line of the B200 drop-in.  Same options and file contract
// as the reference CLI (code/main.cpp:26-256): reads network.conf and
// network.pro, writes the output files named in the .pro, ConfsInfo.log and
// network.log.
// Extra options: -mode compat|fp32|fp64 (default compat: the reference's
// raster bit for bit), -gpu N (CUDA device), -chunk N (steps per launch batch),
// -cache FILE (binary network cache: a rerun on unchanged files skips parsing
// and building), -nolog (skip network.log, a text copy of every synapse).
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include "flysim_b200.h"
#include "fs_host.hpp"

static void usage() {
  std::printf(
      "B200 flysim: per-timestep network integration on one GPU\n\n"
      "flysim -option parameters\n\n"
      "-pro network.pro      # read protocal file: default=network.pro\n"
      "-conf network.conf    # read configuration file: default=network.conf\n"
      "-om my_membrane.dat   # output membrane potential file\n"
      "-os my_spike.dat      # output spikes file\n"
      "-or my_rate.dat       # output firing rate: default rate window=50ms, print out=100ms\n"
      "-rp 1                 # set repeat times: default=1\n"
      "-t 4                  # accepted; one GPU runs the network (affects set-up draws only)\n"
      "-dt 0.1               # time step(default=0.1ms)\n"
      "-udfsed 7             # user random seed (also enables STD, as the reference)\n"
      "-STP / -STD / -LTP    # short-term / depression-only / long-term plasticity\n"
      "-nmodel GNL2          # accepted and ignored (GNL2 is the only model)\n"
      "-mode compat|fp32|fp64 # numeric mode (default compat)\n"
      "-gpu 0                # CUDA device\n"
      "-cache net.cache      # binary network cache (reused while .conf/.pro/options are unchanged)\n"
      "-nolog                # do not write network.log\n");
}

int main(int argc, char **argv) {
  std::string conf = "network.conf", pro = "network.pro";
  std::string om, os, orr, cache;
  fs_model_opts mo{};
  mo.dt = 0.1f;
  mo.threads = 1;
  mo.repeats = 1;
  fs_run_opts ro{};
  ro.mode = FS_MODE_COMPAT;
  bool help = false, netlog = true;
  for (int i = 1; i < argc && !help; i++) {
    std::string a = argv[i];
    auto val = [&](void) -> const char * {
      if (i + 1 >= argc) { help = true; return ""; }
      return argv[++i];
    };
    if (a == "-pro") pro = val();
    else if (a == "-conf") conf = val();
    else if (a == "-om") om = val();
    else if (a == "-os") os = val();
    else if (a == "-or") orr = val();
    else if (a == "-rp") mo.repeats = std::atoi(val());
    else if (a == "-t") mo.threads = std::atoi(val());
    else if (a == "-s") (void)val();
    else if (a == "-nmodel") (void)val();
    else if (a == "-dt") mo.dt = (float)std::atof(val());
    else if (a == "-udfsed") { mo.user_seed = (uint32_t)std::atoi(val()); mo.user_seed_set = 1; }
    else if (a == "-STP") mo.flags |= FS_ACT_STP;
    else if (a == "-STD") mo.flags |= FS_ACT_STD;
    else if (a == "-LTP") mo.flags |= FS_ACT_LTP;
    else if (a == "-gpu") ro.device = std::atoi(val());
    else if (a == "-chunk") ro.chunk_steps = (uint32_t)std::atoi(val());
    else if (a == "-cache") cache = val();
    else if (a == "-nolog") netlog = false;
    else if (a == "-daemon") return 0;  // the reference parses it, then stops without a run or a message (code/main.cpp:86, :205-208)
    else if (a == "-mode") {
      std::string v = val();
      if (v == "compat") ro.mode = FS_MODE_COMPAT;
      else if (v == "fp32") ro.mode = FS_MODE_FP32;
      else if (v == "fp64") ro.mode = FS_MODE_FP64;
      else help = true;
    } else help = true;
  }
  if (help) {
    usage();
    return 0;
  }
  if (!om.empty()) mo.out_mem = om.c_str();
  if (!os.empty()) mo.out_spike = os.c_str();
  if (!orr.empty()) mo.out_rate = orr.c_str();
  fs_model *m = nullptr;
  int cache_status = FS_CACHE_OFF;
  int rc = fs_model_load_cached(conf.c_str(), pro.c_str(), &mo, cache.c_str(), &m, &cache_status);
  if (rc) {
    std::fprintf(stderr, "flysim: %s\n", fs_model_error());
    return 1;
  }
  if (cache_status == FS_CACHE_HIT) std::printf("network read from cache %s\n", cache.c_str());
  else if (cache_status == FS_CACHE_UNWRITABLE) std::fprintf(stderr, "flysim: %s\n", fs_model_error());
  // main.cpp:247 writes ConfsInfo.log after parsing, before the network is set up
  if (fs_model_confs_info(m, "ConfsInfo.log")) std::fprintf(stderr, "flysim: %s\n", fs_model_error());
  uint32_t nn = 0;
  uint64_t ns = 0;
  fs_model_info(m, &nn, nullptr, &ns, nullptr, nullptr);
  std::printf("time step:%g, total neurons=%u, total synapses=%llu\n", (double)mo.dt, nn,
              (unsigned long long)ns);
  // RunInit (code/NetSimGnl2.cpp:143-157) writes network.log before the first repeat
  if (netlog && fs_model_network_log(m, "network.log")) std::fprintf(stderr, "flysim: %s\n", fs_model_error());
  double secs = 0.0;
  rc = fs_model_run(m, &ro, "", &secs);
  if (rc) {
    std::fprintf(stderr, "flysim: %s\n", fs_model_error());
    fs_model_free(m);
    return 1;
  }
  fs_model_free(m);
  return 0;
}
