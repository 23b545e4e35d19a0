// Binary network cache: a parsed and built Model (populations, links, groups,
// events, output controls, repeat seeds and every array of the built network)
// stored in one file under a key made from the bytes of the .conf and .pro
// files and the load options.  A later load of the same files with the same
// options reads the arrays back instead of parsing and building again; any
// change of either file, of an option or of the format makes the key differ
// and the cache is rebuilt.
//
// The reference has no cache: every run parses (code/parser.cpp:297-907,
// :1032-1407) and builds (code/NetSimGnl2_BulPp.cpp) from text.
//
// File layout (native byte order, written on the machine that reads it):
//   magic "FSB2NET\0", u32 format, u32 sizeof checks, u64 key,
//   payload (fields in the order of visit_model), u64 payload hash.
// The file is written to "<path>.tmp<pid>" and renamed into place, so a
// reader never sees a half-written cache.
#include <cstdio>
#include <cstring>
#include <string>
#include <type_traits>
#include <vector>
#include <unistd.h>
#include "fs_host.hpp"

namespace fsh {
namespace {

constexpr char kMagic[8] = {'F', 'S', 'B', '2', 'N', 'E', 'T', '\0'};
constexpr uint32_t kFormat = 5;  // 3: unseeded models are never stored; 4: record sources; 5: LTP record flags
constexpr uint32_t kSizes = (uint32_t)(sizeof(Receptor) | sizeof(Link) << 8 | sizeof(Event) << 16);

// 64-bit streaming hash for cache keys and the payload check (not a
// cryptographic hash): 8-byte words folded with a multiply-rotate step, the
// tail and the length folded last, and the SplitMix64 finaliser (Steele,
// Lea, Flood 2014) for avalanche.
struct Hash64 {
  uint64_t h = 0x6a09e667f3bcc908ull, len = 0;
  uint8_t tail[8];
  unsigned nt = 0;
  static uint64_t rotl(uint64_t x, int r) { return (x << r) | (x >> (64 - r)); }
  void word(uint64_t w) {
    w *= 0x87c37b91114253d5ull;
    w = rotl(w, 31);
    w *= 0x4cf5ad432745937full;
    h ^= w;
    h = rotl(h, 27) * 5 + 0x52dce729;
  }
  void add(const void *p, size_t n) {
    const uint8_t *b = (const uint8_t *)p;
    len += n;
    while (nt && n) {
      tail[nt++] = *b++;
      n--;
      if (nt == 8) {
        uint64_t w;
        std::memcpy(&w, tail, 8);
        word(w);
        nt = 0;
      }
    }
    for (; n >= 8; n -= 8, b += 8) {
      uint64_t w;
      std::memcpy(&w, b, 8);
      word(w);
    }
    while (n--) tail[nt++] = *b++;
  }
  uint64_t done() const {
    uint64_t x = h;
    uint64_t w = 0;
    std::memcpy(&w, tail, nt);
    x ^= w * 0x9e3779b97f4a7c15ull;
    x ^= len;
    x += 0x9e3779b97f4a7c15ull;
    x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
    x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
    return x ^ (x >> 31);
  }
};

bool hash_file(Hash64 &hs, const char *path) {
  std::FILE *f = std::fopen(path, "rb");
  if (!f) return false;
  std::vector<char> buf(1 << 20);
  size_t k;
  uint64_t total = 0;
  while ((k = std::fread(buf.data(), 1, buf.size(), f)) > 0) {
    hs.add(buf.data(), k);
    total += k;
  }
  bool ok = !std::ferror(f);
  std::fclose(f);
  hs.add(&total, sizeof total);  // separates the two files' bytes
  return ok;
}

void hash_str(Hash64 &hs, const char *s) {
  uint64_t n = s ? std::strlen(s) + 1 : 0;  // NULL and "" differ
  hs.add(&n, sizeof n);
  if (s) hs.add(s, n);
}

struct Writer {
  std::FILE *f;
  Hash64 hs;
  bool ok = true;
  void raw(const void *p, size_t n) {
    if (!n) return;
    hs.add(p, n);
    if (ok && std::fwrite(p, 1, n, f) != n) ok = false;
  }
  template <class T> void operator()(T &v) {
    static_assert(std::is_trivially_copyable<T>::value, "plain field");
    raw(&v, sizeof v);
  }
  void operator()(std::string &s) {
    uint64_t n = s.size();
    raw(&n, sizeof n);
    raw(s.data(), n);
  }
  template <class T> void operator()(std::vector<T> &v) {
    static_assert(std::is_trivially_copyable<T>::value, "plain elements");
    uint64_t n = v.size();
    raw(&n, sizeof n);
    raw(v.data(), n * sizeof(T));
  }
  template <class T, class F> void seq(std::vector<T> &v, F &&each) {
    uint64_t n = v.size();
    raw(&n, sizeof n);
    for (T &x : v) each(x);
  }
};

struct Reader {
  std::FILE *f;
  uint64_t left;  // payload bytes the file still holds
  Hash64 hs;
  bool ok = true;
  void raw(void *p, size_t n) {
    if (!n || !ok) return;
    if (n > left || std::fread(p, 1, n, f) != n) {
      ok = false;
      return;
    }
    left -= n;
    hs.add(p, n);
  }
  uint64_t count(size_t elem) {
    uint64_t n = 0;
    raw(&n, sizeof n);
    if (elem && n > left / elem) ok = false;  // a length no file this size can hold
    return ok ? n : 0;
  }
  template <class T> void operator()(T &v) {
    static_assert(std::is_trivially_copyable<T>::value, "plain field");
    raw(&v, sizeof v);
  }
  void operator()(std::string &s) {
    uint64_t n = count(1);
    s.resize(n);
    raw(&s[0], n);
  }
  template <class T> void operator()(std::vector<T> &v) {
    uint64_t n = count(sizeof(T));
    v.resize(n);
    raw(v.data(), n * sizeof(T));
  }
  template <class T, class F> void seq(std::vector<T> &v, F &&each) {
    uint64_t n = count(1);
    v.resize(n);
    for (T &x : v) {
      if (!ok) break;
      each(x);
    }
  }
};

// One list of the fields, walked by both the writer and the reader.
template <class A> void visit_model(A &a, Model &m) {
  a(m.opts.dt); a(m.opts.flags); a(m.opts.user_seed_set); a(m.opts.user_seed);
  a(m.opts.threads); a(m.opts.repeats);
  a(m.dt); a(m.act_ctr);
  a.seq(m.pops, [&](Pop &p) {
    a(p.name); a(p.N); a(p.nrep); a(p.link_beg); a(p.link_num); a(p.selcon); a(p.reps);
    a(p.Taum); a(p.Vth); a(p.El); a(p.gl); a(p.Cm); a(p.Vreset); a(p.RfPed); a(p.SpiDy);
    a(p.pv); a(p.tD); a(p.aF); a(p.tF); a(p.aCap); a(p.tCap); a(p.aCar); a(p.tCar);
    a(p.tLP); a(p.SpiLPDy); a(p.PosISI); a(p.NegISI);
  });
  a(m.links);
  a.seq(m.groups, [&](Group &g) { a(g.name); a(g.pops); });
  a(m.macro_seeds);
  a(m.events);
  a.seq(m.outs, [&](OutCtl &o) {
    a(o.Status); a(o.Type); a(o.TypeID); a(o.FileName); a(o.ParList); a(o.RWin); a(o.FPnt);
    a(o.TimEv); a(o.SpiRWin);
  });
  a(m.rseeds);
  a(m.out_mem); a(m.out_spike); a(m.out_rate);
  a(m.comm_mem); a(m.comm_spike); a(m.comm_rate);
  Network &n = m.net;
  a(n.n); a(n.nidx);
  a(n.Vth); a(n.El); a(n.gl); a(n.Cm); a(n.Vreset); a(n.df); a(n.ef); a(n.dVmax);
  a(n.RfPed); a(n.SpiDy);
  a(n.Vrev); a(n.dfst); a(n.ext_g); a(n.pb);
  a(n.nmda_dfxt); a(n.nmda_efst); a(n.nmda_as); a(n.nmda_mg);
  a(n.act); a(n.inj_mean); a(n.inj_std);
  a(n.stp_pv); a(n.stp_dfD); a(n.stp_efD); a(n.stp_aF); a(n.stp_dfF); a(n.stp_efF);
  a(n.stp_aCap); a(n.stp_dfCap); a(n.stp_aCar); a(n.stp_dfCar); a(n.stp_efCar);
  a(n.ltp_dfLP); a(n.ltp_PosISI); a(n.ltp_NegISI); a(n.ltp_SpiLPDy);
  for (int r = 0; r < FS_NREC; r++) {
    Network::RecArrays &ra = n.rec[r];
    a(ra.gate_pre); a(ra.gate_post0); a(ra.gate_g); a(ra.gather_rowptr); a(ra.gather_gate);
    a(ra.rec_pre); a(ra.rec_post); a(ra.rec_g); a(ra.rec_rowptr); a(ra.seg_post); a(ra.seg_len); a(ra.rec_src);
  }
  a(n.gap_rowptr); a(n.gap_other); a(n.gap_g);
  a(n.gap1_pre); a(n.gap1_post); a(n.gap_ngroup); a(n.gap1_g);
  a(n.syn_pre); a(n.syn_post); a(n.syn_rec); a(n.syn_g); a(n.syn_delay); a(n.syn_ltp);
  a(n.total_synapses);
}

}  // namespace

bool cache_key(const char *conf, const char *pro, const fs_model_opts &o, uint64_t &key) {
  Hash64 hs;
  hs.add(kMagic, sizeof kMagic);
  hs.add(&kFormat, sizeof kFormat);
  if (!hash_file(hs, conf) || !hash_file(hs, pro)) return false;
  hs.add(&o.dt, sizeof o.dt);
  hs.add(&o.flags, sizeof o.flags);
  hs.add(&o.user_seed_set, sizeof o.user_seed_set);
  uint32_t us = o.user_seed_set ? o.user_seed : 0;
  hs.add(&us, sizeof us);
  hs.add(&o.threads, sizeof o.threads);
  hs.add(&o.repeats, sizeof o.repeats);
  hash_str(hs, o.out_mem);
  hash_str(hs, o.out_spike);
  hash_str(hs, o.out_rate);
  key = hs.done();
  return true;
}

// Reads a cache written for `key` into m (views made); false on a missing
// file, another key or format, or any damage (m is then left unspecified).
bool cache_read(const std::string &path, uint64_t key, Model &m) {
  std::FILE *f = std::fopen(path.c_str(), "rb");
  if (!f) return false;
  std::setvbuf(f, nullptr, _IOFBF, 1 << 22);
  char mg[8];
  uint32_t fmt = 0, sz = 0;
  uint64_t k = 0;
  bool ok = std::fread(mg, 1, 8, f) == 8 && std::memcmp(mg, kMagic, 8) == 0 &&
            std::fread(&fmt, 4, 1, f) == 1 && fmt == kFormat && std::fread(&sz, 4, 1, f) == 1 &&
            sz == kSizes && std::fread(&k, 8, 1, f) == 1 && k == key;
  long start = ok ? std::ftell(f) : -1;
  if (ok && std::fseek(f, 0, SEEK_END) == 0) {
    long end = std::ftell(f);
    ok = end >= start + 8 && std::fseek(f, start, SEEK_SET) == 0;
    Reader rd{f, ok ? (uint64_t)(end - start - 8) : 0};
    if (ok) visit_model(rd, m);
    uint64_t want = 0;
    ok = ok && rd.ok && rd.left == 0 && std::fread(&want, 8, 1, f) == 1 && want == rd.hs.done();
  } else {
    ok = false;
  }
  std::fclose(f);
  if (ok) m.net.make_views(m.dt, m.act_ctr);
  return ok;
}

// Writes m under `key`; false (with err set) when the file cannot be written.
bool cache_write(const std::string &path, uint64_t key, Model &m, std::string &err) {
  std::string tmp = path + ".tmp" + std::to_string((long)getpid());
  std::FILE *f = std::fopen(tmp.c_str(), "wb");
  if (!f) {
    err = "cannot write network cache " + tmp;
    return false;
  }
  std::setvbuf(f, nullptr, _IOFBF, 1 << 22);
  bool ok = std::fwrite(kMagic, 1, 8, f) == 8 && std::fwrite(&kFormat, 4, 1, f) == 1 &&
            std::fwrite(&kSizes, 4, 1, f) == 1 && std::fwrite(&key, 8, 1, f) == 1;
  Writer wr{f};
  if (ok) visit_model(wr, m);
  uint64_t h = wr.hs.done();
  ok = ok && wr.ok && std::fwrite(&h, 8, 1, f) == 1;
  ok = (std::fclose(f) == 0) && ok;
  if (ok && std::rename(tmp.c_str(), path.c_str()) != 0) ok = false;
  if (!ok) {
    std::remove(tmp.c_str());
    err = "cannot write network cache " + path;
  }
  return ok;
}

}  // namespace fsh
