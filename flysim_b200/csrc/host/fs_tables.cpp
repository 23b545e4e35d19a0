// Exception tables that make the device's float exp/log agree with glibc's
// expf/logf, the functions the reference calls (NMDA Mg block,
// code/EqsGnl2.cpp:165; ziggurat tail, code/StiExt.h:284-285).
//
// The device evaluates (float)exp((double)x) / (float)log((double)x).  With a
// double result within 1 ulp of the true value (the documented bound of the
// device's double exp/log), rounding it to float gives the correctly rounded
// float unless the true value lies within a couple of double ulps of a float
// rounding boundary.  glibc's expf/logf are not correctly rounded everywhere.
// So the table lists every input of the covered range where
//   glibc_f(x) != (float)glibc_d((double)x),   or
//   glibc_d((double)x) lies within 4 double ulps of a float rounding boundary,
// with glibc_f(x) as the value.  Everything here calls glibc; no library
// internals are reproduced.
//
// Covered ranges: expf over |x| <= 12.4 (membrane potential within +-200 mV,
// x = -0.062 V); logf over the 2^24 values k * 2^-24 that the ziggurat's
// uniform r4_uni can produce.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <cstdint>
#include <string>
#include <thread>
#include <vector>
#include <algorithm>

namespace fsh {

namespace {
inline float u2f(uint32_t u) { float f; std::memcpy(&f, &u, 4); return f; }
inline uint32_t f2u(float f) { uint32_t u; std::memcpy(&u, &f, 4); return u; }

bool near_boundary(double v, float c) {
  if (!std::isfinite(v) || v == 0.0) return false;
  const double ulp = std::nextafter(std::fabs(v), INFINITY) - std::fabs(v);
  const float up = std::nextafterf(c, INFINITY), dn = std::nextafterf(c, -INFINITY);
  const double m1 = ((double)c + (double)up) * 0.5, m2 = ((double)c + (double)dn) * 0.5;
  return std::fabs(v - m1) <= 4.0 * ulp || std::fabs(v - m2) <= 4.0 * ulp;
}

struct Entry { uint32_t key; float val; };

void gen_exp(std::vector<Entry> &out) {
  const float lim = 12.4f;
  const uint32_t top = f2u(lim);
  const int T = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
  std::vector<std::vector<Entry>> part(T);
  std::vector<std::thread> th;
  for (int t = 0; t < T; t++)
    th.emplace_back([&, t]() {
      for (int sgn = 0; sgn < 2; sgn++)
        for (uint32_t u = (uint32_t)t; u <= top; u += (uint32_t)T) {
          const float x = u2f(u | (sgn ? 0x80000000u : 0u));
          const float g = std::exp(x);  // expf
          const double dv = std::exp((double)x);
          const float c = (float)dv;
          if (f2u(g) != f2u(c) || near_boundary(dv, c)) part[t].push_back({f2u(x), g});
        }
    });
  for (auto &x : th) x.join();
  for (auto &p : part) out.insert(out.end(), p.begin(), p.end());
  std::sort(out.begin(), out.end(), [](const Entry &a, const Entry &b) { return a.key < b.key; });
}

void gen_log(std::vector<Entry> &out) {
  for (uint32_t k = 1; k < (1u << 24); k++) {
    const float x = (float)k * 5.9604644775390625e-08f;  // k * 2^-24, exact
    const float g = std::log(x);                         // logf
    const double dv = std::log((double)x);
    const float c = (float)dv;
    if (f2u(g) != f2u(c) || near_boundary(dv, c)) out.push_back({f2u(x), g});
  }
  std::sort(out.begin(), out.end(), [](const Entry &a, const Entry &b) { return a.key < b.key; });
}

bool write_table(const std::string &path, const std::vector<Entry> &t) {
  FILE *f = std::fopen(path.c_str(), "wb");
  if (!f) return false;
  const uint32_t magic = 0x46534554u, n = (uint32_t)t.size();
  std::fwrite(&magic, 4, 1, f);
  std::fwrite(&n, 4, 1, f);
  for (const Entry &e : t) std::fwrite(&e.key, 4, 1, f);
  for (const Entry &e : t) std::fwrite(&e.val, 4, 1, f);
  return std::fclose(f) == 0;
}
}  // namespace

bool read_table(const std::string &path, std::vector<uint32_t> &keys, std::vector<float> &vals) {
  FILE *f = std::fopen(path.c_str(), "rb");
  if (!f) return false;
  uint32_t magic = 0, n = 0;
  bool ok = std::fread(&magic, 4, 1, f) == 1 && std::fread(&n, 4, 1, f) == 1 && magic == 0x46534554u;
  if (ok) {
    keys.resize(n);
    vals.resize(n);
    ok = std::fread(keys.data(), 4, n, f) == n && std::fread(vals.data(), 4, n, f) == n;
  }
  std::fclose(f);
  return ok;
}

int generate_tables(const std::string &dir) {
  std::vector<Entry> e, l;
  gen_exp(e);
  gen_log(l);
  if (!write_table(dir + "/expf_glibc.bin", e)) return 1;
  if (!write_table(dir + "/logf_glibc.bin", l)) return 1;
  std::printf("expf exceptions: %zu, logf exceptions: %zu\n", e.size(), l.size());
  return 0;
}

}  // namespace fsh

#ifdef FS_TABLES_MAIN
int main(int argc, char **argv) {
  if (argc < 2) {
    std::fprintf(stderr, "usage: fs_gen_tables <dir>\n");
    return 2;
  }
  return fsh::generate_tables(argv[1]);
}
#endif
