// Protocol driver of the flysim drop-in: the per-trial loop of
// NetSimGnl2::Run/SimOne (code/NetSimGnl2.cpp:231-358), the event application
// of DoEvt (code/NetSimGnl2.cpp:52-141) and the output writers of FileOut
// (code/NetSimGnl2_info.cpp:548-769), over any engine behind fs_engine_vtbl.
//
// Steps run in batches on the engine; a batch ends before any step whose
// events change parameters, so each step sees exactly the parameters the
// reference would.  The engine returns per-step spike lists (and, when an
// output needs them, V / receptor currents / NState), from which the text
// lines are produced per step in the reference's format: numbers go through
// "%.6g", which is what the reference's default-precision ostringstream does.
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <functional>
#include <thread>
#include <iostream>
#include <algorithm>
#include "fs_host.hpp"

namespace fsh {
namespace {

struct OutFile {
  FILE *f = nullptr;
  std::string buf;
};

inline void put_g(std::string &s, float v) {
  char b[48];
  int k = std::snprintf(b, sizeof b, "%.6g", (double)v);
  s.append(b, (size_t)k);
}
inline void put_u(std::string &s, unsigned long long v) {
  char b[32];
  int k = std::snprintf(b, sizeof b, "%llu", v);
  s.append(b, (size_t)k);
}

int rec_of_kw(uint8_t kw, uint32_t &bit) {
  switch (kw) {
    case KW_AMPA: bit = FS_ACT_AMPA; return FS_AMPA;
    case KW_GABA: bit = FS_ACT_GABA; return FS_GABA;
    case KW_ACH: bit = FS_ACT_ACH; return FS_ACH;
    case KW_GCL: bit = FS_ACT_GCL; return FS_GCL;
    case KW_NMDA: bit = FS_ACT_NMDA; return FS_NMDA;
    default: bit = 0; return -1;
  }
}

}  // namespace

int run_protocol(Model &m, const fs_engine_vtbl *eng, void *ctx, const std::string &out_dir,
                 uint32_t chunk_steps, double *run_seconds, std::string &err) {
  Network &net = m.net;
  const uint32_t n = net.n;
  const float dt = m.dt;
  const uint32_t np = (uint32_t)m.pops.size();
  if (m.events.empty()) {
    err = "the protocol has no events (an EndTrial event sets the trial length)";
    return FS_ERR_PARSE;
  }
  if (chunk_steps == 0) chunk_steps = 1000;
  // a batch holds at most 64 M spike slots (worst case: every neuron every step)
  if ((uint64_t)chunk_steps * n > (64ull << 20)) chunk_steps = (uint32_t)std::max<uint64_t>(1, (64ull << 20) / n);
  auto fail = [&](int rc) {
    err = eng->error ? eng->error(ctx) : "engine error";
    return rc;
  };
  // SetOut: firing-rate windows (code/NetSim.cpp:32-42)
  for (OutCtl &o : m.outs)
    if (o.TypeID == OUT_FRATE) o.SpiRWin.assign(o.ParList.size() * (o.RWin + 2), 0);
  bool need_V = false, need_Irep = false, need_ns = false;
  for (const OutCtl &o : m.outs) {
    if (o.TypeID == OUT_MEMPOT) need_V = true;
    if (o.TypeID == OUT_ISYNSEP) need_Irep = true;
    if (o.TypeID == OUT_DVOVF) need_ns = true;
  }
  // GatingVariable outputs: single-target records whose (population-index)
  // PreID equals a listed neuron, per receptor in record order
  // (code/NetSimGnl2_info.cpp:443-470 builds these maps, :701-758 prints).
  std::vector<std::vector<uint32_t>> gv_of(m.outs.size());
  std::vector<uint32_t> gv_all;
  {
    const int order[5] = {FS_AMPA, FS_GABA, FS_ACH, FS_GCL, FS_NMDA};
    std::vector<std::vector<uint32_t>> by_pre[5];
    bool any = false;
    for (const OutCtl &o : m.outs) any |= (o.TypeID == OUT_GATVAR);
    if (any)
      for (int oi = 0; oi < 5; oi++) {
        const auto &ra = net.rec[order[oi]];
        by_pre[oi].assign(n, {});
        for (uint32_t e = 0; e < ra.rec_pre.size(); e++)
          if (ra.rec_pre[e] < n) by_pre[oi][ra.rec_pre[e]].push_back(((uint32_t)order[oi] << 28) | e);
      }
    for (size_t i = 0; i < m.outs.size(); i++) {
      if (m.outs[i].TypeID != OUT_GATVAR) continue;
      for (uint32_t pp : m.outs[i].ParList)
        for (uint32_t k = net.nidx[pp]; k < net.nidx[pp] + m.pops[pp].N; k++)
          for (int oi = 0; oi < 5; oi++)
            for (uint32_t code : by_pre[oi][k]) {
              gv_of[i].push_back((uint32_t)gv_all.size());
              gv_all.push_back(code);
            }
    }
  }
  const uint32_t gv_n = (uint32_t)gv_all.size();
  // Spike and FiringRate outputs over many populations: per-neuron maps so
  // that a step costs O(spikes) instead of a search per listed population.
  // Used when the list is ascending and has no repeats (then walking the
  // sorted spikes emits the lines in the list's order); other lists take the
  // general loop.
  std::vector<uint32_t> pop_of(n, 0xffffffffu);
  for (uint32_t pp = 0; pp < np; pp++)
    for (uint32_t k = net.nidx[pp]; k < net.nidx[pp] + m.pops[pp].N; k++) pop_of[k] = pp;
  std::vector<std::vector<int64_t>> spike_map(m.outs.size());  // neuron -> printed index, -1 = not listed
  std::vector<std::vector<int32_t>> rate_pos(m.outs.size());   // population -> list position, -1
  for (size_t i = 0; i < m.outs.size(); i++) {
    const OutCtl &o = m.outs[i];
    if (o.TypeID != OUT_SPIKE && o.TypeID != OUT_FRATE) continue;
    bool ascending = true;
    for (size_t j = 1; j < o.ParList.size(); j++) ascending &= o.ParList[j] > o.ParList[j - 1];
    bool in_range = true;
    for (uint32_t pp : o.ParList) in_range &= pp < np;
    if (!ascending || !in_range) continue;
    if (o.TypeID == OUT_SPIKE) {
      std::vector<int64_t> &mp = spike_map[i];
      mp.assign(n, -1);
      unsigned long long cnt = 0;
      for (uint32_t pp : o.ParList) {
        const uint32_t b = net.nidx[pp];
        for (uint32_t k = b; k < b + m.pops[pp].N; k++)
          mp[k] = (o.Status & OF_ALIGN) ? (int64_t)(cnt + (k - b)) : (int64_t)k;
        cnt += m.pops[pp].N;
      }
    } else {
      std::vector<int32_t> &rp = rate_pos[i];
      rp.assign(np, -1);
      for (size_t j = 0; j < o.ParList.size(); j++) rp[o.ParList[j]] = (int32_t)j;
    }
  }
  const int rp = std::max(1, m.opts.repeats);
  double total_run = 0.0;
  // Output pipeline: two buffer sets; while a formatter thread writes the
  // files of chunk k from one set, the engine computes chunk k+1 into the
  // other.  Chunks are formatted strictly in order (the next formatter starts
  // after the previous one joined), so the files are those of a serial run.
  struct ChunkBuf {
    std::vector<uint32_t> counts, spikes, NS;
    std::vector<float> V, I, gst, gxt;
    unsigned long long first = 0;
    uint32_t steps = 0;
  };
  ChunkBuf bufs[2];
  for (ChunkBuf &b : bufs) {
    b.counts.resize(chunk_steps);
    b.spikes.resize((size_t)chunk_steps * n);
    if (need_V) b.V.resize((size_t)chunk_steps * n);
    if (need_Irep) b.I.resize((size_t)chunk_steps * FS_NREC * n);
    if (need_ns) b.NS.resize((size_t)chunk_steps * n);
    if (gv_n) {
      b.gst.resize((size_t)chunk_steps * gv_n);
      b.gxt.resize((size_t)chunk_steps * gv_n);
    }
  }

  for (int rep = 1; rep <= rp; rep++) {
    const Event &last = m.events.back();
    const bool nolmt = last.NoLmt;
    // Endtime = floor(T*1e3f/dt) (code/NetSimGnl2.cpp:270); a NoLimit run's
    // FLT_MAX time overflows it, and the loop ignores it then
    const float endf = std::floor(last.TimEv * 1e3f / dt);
    const unsigned long long endtime =
        (endf >= 0.0f && endf < 1.8e19f) ? (unsigned long long)endf : (endf >= 0.0f ? ~0ull : 0ull);
    // steps per ms (1/dt); at least 1, so a step above 1 ms divides by 1 in
    // the rate writer where the reference would divide by 0
    const unsigned one_ms = std::max(1u, (unsigned)(1u / dt));
    // VarInit + reseed (code/NetSimGnl2.cpp:277, :319-323)
    int rc = eng->reset(ctx, m.rseeds[rep - 1], m.rseeds[rep - 1]);
    if (rc) return fail(rc);
    // pb reset from the configuration (code/NetSimGnl2.cpp:279-297)
    for (uint32_t i = 0; i < np; i++) {
      const Pop &p = m.pops[i];
      if (p.N == 0) continue;
      for (const Receptor &r : p.reps) {
        uint32_t bit;
        int ri = rec_of_kw(r.name, bit);
        if (ri < 0) continue;
        rc = eng->set_drive(ctx, net.nidx[i], p.N, ri, r.FExt * dt * 1e-3f);
        if (rc) return fail(rc);
      }
    }
    if (rep > 1)
      for (OutCtl &o : m.outs) std::fill(o.SpiRWin.begin(), o.SpiRWin.end(), 0u);
    unsigned iEvt = 0;
    if (rep > 1) iEvt = 0;
    // FileOpen (code/NetSim.cpp:45-66)
    std::vector<OutFile> files(m.outs.size());
    for (size_t i = 0; i < m.outs.size(); i++) {
      std::string name = m.outs[i].FileName;
      if (rep > 1) name += "_" + std::to_string((long long)rep);
      std::string path = out_dir.empty() ? name : out_dir + "/" + name;
      files[i].f = std::fopen(path.c_str(), "w");
      if (!files[i].f) {
        err = "cannot open output file " + path;
        for (auto &of : files)
          if (of.f) std::fclose(of.f);
        return FS_ERR_IO;
      }
    }
    // every return from here on closes the files with what was computed
    // written out (an engine error mid-run leaves complete files up to the
    // last finished chunk); it runs after the formatter thread has joined
    // (the joiner below is destroyed first)
    struct Closer {
      std::vector<OutFile> &v;
      ~Closer() {
        for (OutFile &x : v) {
          if (!x.f) continue;
          if (!x.buf.empty()) std::fwrite(x.buf.data(), 1, x.buf.size(), x.f);
          std::fclose(x.f);
          x.f = nullptr;
        }
      }
    } closer{files};
    std::printf("Iteration:%d\n", rep);

    // FileOut for one step
    auto file_out = [&](unsigned long long step, const uint32_t *sp, uint32_t nsp, const float *V,
                        const float *Irep, const uint32_t *ns, const float *gst, const float *gxt) {
      const float evtime = (float)step * dt;
      const float tsec = evtime * 1e-3f;
      for (size_t i = 0; i < m.outs.size(); i++) {
        OutCtl &o = m.outs[i];
        std::string &s = files[i].buf;
        switch (o.TypeID) {
          case OUT_ISYNSEP:
            put_g(s, tsec);
            for (uint32_t pp : o.ParList)
              for (uint32_t k = net.nidx[pp]; k < net.nidx[pp] + m.pops[pp].N; k++)
                for (int r = 0; r < FS_NREC; r++) {
                  s.push_back(' ');
                  put_g(s, Irep[(size_t)r * n + k] * 1e-12f);
                }
            s.push_back('\n');
            break;
          case OUT_MEMPOT:
            put_g(s, tsec);
            for (uint32_t pp : o.ParList)
              for (uint32_t k = net.nidx[pp]; k < net.nidx[pp] + m.pops[pp].N; k++) {
                s.push_back(' ');
                put_g(s, V[k] * 1e-3f);
              }
            s.push_back('\n');
            break;
          case OUT_DVOVF: {
            unsigned long long cnt = 0;
            for (uint32_t pp : o.ParList)
              for (uint32_t k = net.nidx[pp]; k < net.nidx[pp] + m.pops[pp].N; k++, cnt++) {
                if (ns[k] & FS_NS_MEMDV_OVF) {
                  put_g(s, tsec);
                  s.push_back(' ');
                  put_u(s, (o.Status & OF_ALIGN) ? cnt + 1 : (unsigned long long)k + 1);
                  s.push_back('\n');
                } else if (ns[k] & FS_NS_MEMDV_UDF) {
                  put_g(s, tsec);
                  s.append(" -");
                  put_u(s, (o.Status & OF_ALIGN) ? cnt + 1 : (unsigned long long)k + 1);
                  s.push_back('\n');
                }
              }
            break;
          }
          case OUT_SPIKE: {
            if (!spike_map[i].empty()) {
              const std::vector<int64_t> &mp = spike_map[i];
              for (uint32_t q = 0; q < nsp; q++) {
                const int64_t v = mp[sp[q]];
                if (v < 0) continue;
                put_g(s, tsec);
                s.push_back(' ');
                put_u(s, (unsigned long long)v);
                s.push_back('\n');
              }
              break;
            }
            unsigned long long cnt = 0;
            for (uint32_t pp : o.ParList) {
              const uint32_t b = net.nidx[pp], e = b + m.pops[pp].N;
              const uint32_t *lo = std::lower_bound(sp, sp + nsp, b);
              const uint32_t *hi = std::lower_bound(lo, sp + nsp, e);
              for (const uint32_t *q = lo; q < hi; q++) {
                put_g(s, tsec);
                s.push_back(' ');
                put_u(s, (o.Status & OF_ALIGN) ? cnt + (*q - b) : (unsigned long long)*q);
                s.push_back('\n');
              }
              cnt += m.pops[pp].N;
            }
            break;
          }
          case OUT_FRATE: {
            const size_t P = o.ParList.size();
            std::vector<uint32_t> &w = o.SpiRWin;
            if (!rate_pos[i].empty()) {
              for (uint32_t q = 0; q < nsp; q++) {
                const uint32_t pp = pop_of[sp[q]];
                const int32_t j = pp < np ? rate_pos[i][pp] : -1;
                if (j >= 0) w[P * o.RWin + j] += 1;
              }
            } else {
              for (size_t j = 0; j < P; j++) {
                const uint32_t pp = o.ParList[j];
                const uint32_t b = net.nidx[pp], e = b + m.pops[pp].N;
                const uint32_t *lo = std::lower_bound(sp, sp + nsp, b);
                const uint32_t *hi = std::lower_bound(lo, sp + nsp, e);
                w[P * o.RWin + j] += (uint32_t)(hi - lo);
              }
            }
            if (step % one_ms == 0) {
              const unsigned long long s1ms = step / one_ms;
              const unsigned mm = (unsigned)(s1ms % o.RWin);
              if (s1ms % o.FPnt == 0) {
                put_g(s, tsec);
                if (o.Status & OF_SUMALL) {
                  unsigned a = 0, nn = 0;
                  for (size_t j = 0; j < P; j++) {
                    a += w[P * (o.RWin + 1) + j];
                    nn += m.pops[j < np ? j : np - 1].N;  // list position, as code/NetSimGnl2_info.cpp:676
                  }
                  s.push_back(' ');
                  put_g(s, 1e3f * a / o.RWin / nn);
                } else {
                  for (size_t j = 0; j < P; j++) {
                    s.push_back(' ');
                    put_g(s, 1e3f * w[P * (o.RWin + 1) + j] / o.RWin / m.pops[j < np ? j : np - 1].N);
                  }
                }
                s.push_back('\n');
              }
              for (size_t j = 0; j < P; j++) {
                w[P * (o.RWin + 1) + j] -= w[j * o.RWin + mm];
                w[P * (o.RWin + 1) + j] += w[P * o.RWin + j];
                w[j * o.RWin + mm] = w[P * o.RWin + j];
                w[P * o.RWin + j] = 0;
              }
            }
            break;
          }
          case OUT_GATVAR:
            put_g(s, tsec);
            s.push_back(' ');
            for (uint32_t q : gv_of[i]) {
              if ((gv_all[q] >> 28) == FS_NMDA) {
                put_g(s, gxt[q]);
                s.push_back(' ');
              }
              put_g(s, gst[q]);
              s.push_back(' ');
            }
            s.push_back('\n');
            break;
          default:
            break;
        }
        if (s.size() > (1u << 20)) {
          std::fwrite(s.data(), 1, s.size(), files[i].f);
          s.clear();
        }
      }
    };

    // event application (DoEvt) for step i; returns true if any event matched
    auto events_at = [&](unsigned long long i, bool apply, int &erc) -> bool {
      const float evtime = (float)i * dt;
      bool any = false;
      for (unsigned e = iEvt; e < m.events.size(); e++) {
        const Event &ev = m.events[e];
        const float t = ev.TimEv * 1e3f;
        if (t >= evtime && t < (evtime + dt)) {
          any = true;
          if (!apply) return true;
          iEvt = e;
          if (ev.Pp >= np) continue;
          const uint32_t first = net.nidx[ev.Pp], cnt = m.pops[ev.Pp].N;
          if (cnt == 0) continue;
          if (ev.Type == EVT_EXTFREQ) {
            uint32_t bit;
            int ri = rec_of_kw(ev.SubTyp, bit);
            if (ri < 0) continue;
            if (ev.Var1 == 0.0f) {
              erc = eng->set_act(ctx, first, cnt, bit, 0);
            } else {
              erc = eng->set_act(ctx, first, cnt, 0, bit);
              if (!erc) erc = eng->set_drive(ctx, first, cnt, ri, (float)(ev.Var1 * dt * 1e-3f));
            }
          } else if (ev.Type == EVT_CURINJ) {
            const float sd =
                ev.Var2 * (1.0f + (float)std::log((1.0f - std::exp(-0.1f / m.pops[ev.Pp].Taum)) /
                                                  (1.0f - net.df[first])));
            erc = eng->set_injection(ctx, first, cnt, ev.Var1, sd);
            if (!erc) {
              if (ev.Var1 == 0.0f && ev.Var2 == 0.0f) erc = eng->set_act(ctx, first, cnt, FS_ACT_INJ, 0);
              else erc = eng->set_act(ctx, first, cnt, 0, FS_ACT_INJ);
            }
          }
          if (erc) return true;
        } else if (t >= (evtime + dt)) {
          break;
        }
      }
      return any;
    };

    auto t1 = std::chrono::high_resolution_clock::now();
    unsigned long long i = 0, batch_first = 0;
    uint32_t pending = 0;
    int cur = 0;
    std::thread formatter;
    auto join = [&]() {
      if (formatter.joinable()) formatter.join();
    };
    auto format_chunk = [&](ChunkBuf *b) {
      uint64_t off = 0;
      for (uint32_t s = 0; s < b->steps; s++) {
        file_out(b->first + s, b->spikes.data() + off, b->counts[s],
                 need_V ? b->V.data() + (size_t)s * n : nullptr,
                 need_Irep ? b->I.data() + (size_t)s * FS_NREC * n : nullptr,
                 need_ns ? b->NS.data() + (size_t)s * n : nullptr,
                 gv_n ? b->gst.data() + (size_t)s * gv_n : nullptr,
                 gv_n ? b->gxt.data() + (size_t)s * gv_n : nullptr);
        off += b->counts[s];
      }
    };
    auto flush = [&]() -> int {
      if (pending == 0) return FS_OK;
      ChunkBuf &b = bufs[cur];  // its previous formatter (two chunks ago) has joined
      fs_step_out so{};
      so.spike_count = b.counts.data();
      so.spike_idx = b.spikes.data();
      so.spike_cap = b.spikes.size();
      so.V = need_V ? b.V.data() : nullptr;
      so.Irep = need_Irep ? b.I.data() : nullptr;
      so.nstate = need_ns ? b.NS.data() : nullptr;
      so.gv_sel = gv_n ? gv_all.data() : nullptr;
      so.gv_n = gv_n;
      so.gv_st = gv_n ? b.gst.data() : nullptr;
      so.gv_xt = gv_n ? b.gxt.data() : nullptr;
      int r = eng->step(ctx, pending, &so);
      join();  // the previous chunk's files are complete
      if (r) return r;
      b.first = batch_first;
      b.steps = pending;
      formatter = std::thread(format_chunk, &b);
      cur ^= 1;
      batch_first += pending;
      pending = 0;
      return FS_OK;
    };
    // every return below joins the formatter first
    struct Joiner {
      std::function<void()> f;
      ~Joiner() { f(); }
    } joiner{join};
    // progress every 100 ms simulated, as the reference prints it
    // (code/NetSimGnl2.cpp:169-188, :238-257, ReportStep = 100/dt at :271)
    const unsigned long long report_step = std::max(1u, (unsigned)(100.0f / dt));
    for (; (i < endtime) || nolmt; i++) {
      int erc = 0;
      if (i % report_step == 0) {
        const double el = std::chrono::duration_cast<std::chrono::nanoseconds>(
                              std::chrono::high_resolution_clock::now() - t1).count() * 1e-9;
        const float evt = (float)i * dt;
        if (nolmt)
          std::printf("Expertment time=%.7gs real time=%.7gs :infinity End time             \r",
                      (double)(evt * 1e-3f), el);
        else
          std::printf("Expertment time=%.7gs real time=%.7gs %.7g%%             \r", (double)(evt * 1e-3f), el,
                      (double)(100.0f * (float)(i + 1) / (float)endtime));
        std::fflush(stdout);
      }
      if (events_at(i, false, erc)) {
        int r = flush();
        if (r) return fail(r);
        events_at(i, true, erc);
        if (erc) return fail(erc);
      }
      if (pending == 0) batch_first = i;
      pending++;
      if (pending == chunk_steps) {
        int r = flush();
        if (r) return fail(r);
      }
    }
    {
      int r = flush();
      if (r) return fail(r);
    }
    join();
    auto t2 = std::chrono::high_resolution_clock::now();
    const double secs = std::chrono::duration_cast<std::chrono::nanoseconds>(t2 - t1).count() * 1e-9;
    total_run += secs;
    const float evlast = (endtime > 0 ? (float)(endtime - 1) * dt : 0.0f);
    std::printf("Expertment time=%.7gs real time=%.7gs 100%%                 \n",
                (double)(evlast * 1e-3f), secs);
    std::fflush(stdout);
    for (size_t k = 0; k < files.size(); k++) {
      if (!files[k].buf.empty()) std::fwrite(files[k].buf.data(), 1, files[k].buf.size(), files[k].f);
      std::fclose(files[k].f);
      files[k].f = nullptr;
      files[k].buf.clear();
    }
  }
  if (run_seconds) *run_seconds = total_run;
  return FS_OK;
}

}  // namespace fsh
