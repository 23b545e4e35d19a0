// C ABI of the device engine (include/flysim_b200.h): one fs_handle owns the
// device memory of one network instance and a CUDA stream.  Host code above
// this layer never sees a CUDA type.
#include <dlfcn.h>
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>
#include <cuda_runtime.h>
#include "flysim_b200.h"
#include "fs_device.cuh"
#include "fs_prod.cuh"

namespace fsh {
bool read_table(const std::string &path, std::vector<uint32_t> &keys, std::vector<float> &vals);
}

struct fs_handle {
  int mode = FS_MODE_COMPAT;
  int device = 0;
  cudaStream_t st = nullptr;
  uint32_t sm_count = 148;
  uint32_t n = 0;
  float dt = 0.1f;
  uint32_t glob = 0;
  uint32_t chunk = 1000;
  std::string err;
  std::vector<void *> allocs;
  // host mirrors of the event-driven parameters
  std::vector<float> pb, inj_mean, inj_std;
  std::vector<uint32_t> act;
  bool dirty = true;
  // compat
  fsd::CompatDev cd{};
  uint32_t *mt_state = nullptr, *mt_pos = nullptr, *draws = nullptr;
  uint64_t draws_cap = 0;
  uint32_t *drawoff = nullptr, *injoff = nullptr;
  uint32_t jcong = 0;
  // batch buffers
  uint32_t *spikebits = nullptr, *counts = nullptr, *offsets = nullptr, *idx = nullptr;
  uint64_t batch_cap = 0;  // steps the batch buffers hold
  float *outV = nullptr, *outIrep = nullptr;
  uint32_t *outNS = nullptr;
  uint32_t *gv_sel = nullptr;
  float *gv_st = nullptr, *gv_xt = nullptr;
  uint32_t gv_cap = 0, gv_sel_cap = 0;
  uint64_t out_cap_steps = 0;  // steps the V/Irep/NS buffers hold
  int *derr = nullptr;
  // production
  fsp::Prod *prod = nullptr;
  // stats
  uint64_t steps_done = 0, spikes_total = 0, launches = 0;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  double kernel_ms = 0.0;
  uint64_t kernel_launches = 0;
};

namespace {

thread_local std::string g_err;

int set_err(fs_handle *h, int code, const std::string &msg) {
  if (h) h->err = msg;
  g_err = msg;
  return code;
}
int cuda_err(fs_handle *h, cudaError_t e, const char *where) {
  return set_err(h, FS_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}
#define CK(call)                                             \
  do {                                                       \
    cudaError_t _e = (call);                                 \
    if (_e != cudaSuccess) return cuda_err(h, _e, #call);    \
  } while (0)

template <class T>
int dalloc(fs_handle *h, T **p, size_t count) {
  *p = nullptr;
  if (count == 0) return FS_OK;
  void *q = nullptr;
  cudaError_t e = cudaMalloc(&q, count * sizeof(T));
  if (e != cudaSuccess) return set_err(h, FS_ERR_NOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
  h->allocs.push_back(q);
  *p = (T *)q;
  return FS_OK;
}
template <class T>
int upload(fs_handle *h, T **p, const T *src, size_t count) {
  int rc = dalloc(h, p, count);
  if (rc || count == 0) return rc;
  if (src) CK(cudaMemcpyAsync(*p, src, count * sizeof(T), cudaMemcpyHostToDevice, h->st));
  else CK(cudaMemsetAsync(*p, 0, count * sizeof(T), h->st));
  return FS_OK;
}
template <class T>
int zeros(fs_handle *h, T **p, size_t count) {
  return upload<T>(h, p, nullptr, count);
}

std::string lib_dir() {
  Dl_info info;
  if (dladdr((void *)&fs_abi_version, &info) && info.dli_fname) {
    std::string p = info.dli_fname;
    size_t s = p.rfind('/');
    if (s != std::string::npos) return p.substr(0, s);
  }
  return ".";
}

// Ziggurat tables (Burkardt's r4_nor_setup, code/StiExt.h:321-351) and the
// powers of the congruential map used by the injection noise.
void host_tables(uint32_t kn[128], float fn[128], float wn[128], uint32_t ja[32], uint32_t jc[32]) {
  double dn = 3.442619855899, tn = dn;
  const double m1 = 2147483648.0, vn = 9.91256303526217E-03;
  double q = vn / std::exp(-0.5 * dn * dn);
  kn[0] = (uint32_t)((dn / q) * m1);
  kn[1] = 0;
  wn[0] = (float)(q / m1);
  wn[127] = (float)(dn / m1);
  fn[0] = 1.0f;
  fn[127] = (float)std::exp(-0.5 * dn * dn);
  for (int i = 126; 1 <= i; i--) {
    dn = std::sqrt(-2.0 * std::log(vn / dn + std::exp(-0.5 * dn * dn)));
    kn[i + 1] = (uint32_t)((dn / tn) * m1);
    tn = dn;
    fn[i] = (float)std::exp(-0.5 * dn * dn);
    wn[i] = (float)(dn / m1);
  }
  uint32_t a = 69069u, c = 1234567u;
  for (int i = 0; i < 32; i++) {
    ja[i] = a;
    jc[i] = c;
    // square the map: x -> a(ax+c)+c
    c = a * c + c;
    a = a * a;
  }
}
uint32_t jcong_advance(uint32_t x, uint64_t k) {
  uint32_t a = 69069u, c = 1234567u;
  while (k) {
    if (k & 1) x = a * x + c;
    c = a * c + c;
    a = a * a;
    k >>= 1;
  }
  return x;
}

int ensure_batch(fs_handle *h, uint64_t steps) {
  if (steps <= h->batch_cap) return FS_OK;
  const uint32_t words = (h->n + 31) / 32;
  // buffers are not freed individually: a few regrowths at most
  int rc;
  if ((rc = dalloc(h, &h->spikebits, (size_t)steps * words))) return rc;
  if ((rc = dalloc(h, &h->counts, (size_t)steps))) return rc;
  if ((rc = dalloc(h, &h->offsets, (size_t)steps + 1))) return rc;
  if ((rc = dalloc(h, &h->idx, (size_t)steps * h->n))) return rc;
  h->batch_cap = steps;
  return FS_OK;
}

int upload_params(fs_handle *h) {
  if (!h->dirty) return FS_OK;
  const uint32_t n = h->n;
  std::vector<uint32_t> doff(n), ioff(n);
  uint32_t D = 0, J = 0;
  for (uint32_t i = 0; i < n; i++) {
    doff[i] = D;
    ioff[i] = J;
    const uint32_t a = h->act[i];
    D += ((a & FS_ACT_AMPA) != 0) + ((a & FS_ACT_GABA) != 0) + ((a & FS_ACT_ACH) != 0) +
         ((a & FS_ACT_GCL) != 0) + ((a & FS_ACT_NMDA) != 0);
    J += (a & FS_ACT_INJ) != 0;
  }
  if (h->mode == FS_MODE_COMPAT) {
    CK(cudaMemcpyAsync(h->drawoff, doff.data(), n * 4, cudaMemcpyHostToDevice, h->st));
    CK(cudaMemcpyAsync(h->injoff, ioff.data(), n * 4, cudaMemcpyHostToDevice, h->st));
    CK(cudaMemcpyAsync((void *)h->cd.pb, h->pb.data(), (size_t)FS_NREC * n * 4, cudaMemcpyHostToDevice, h->st));
    CK(cudaMemcpyAsync((void *)h->cd.act, h->act.data(), (size_t)n * 4, cudaMemcpyHostToDevice, h->st));
    CK(cudaMemcpyAsync((void *)h->cd.inj_mean, h->inj_mean.data(), (size_t)n * 4, cudaMemcpyHostToDevice, h->st));
    CK(cudaMemcpyAsync((void *)h->cd.inj_std, h->inj_std.data(), (size_t)n * 4, cudaMemcpyHostToDevice, h->st));
    h->cd.draws_per_step = D;
    h->cd.inj_per_step = J;
  } else {
    int rc = fsp::prod_upload_params(h->prod, h->pb.data(), h->act.data(), h->inj_mean.data(),
                                     h->inj_std.data(), h->st, h->err);
    if (rc) return set_err(h, rc, h->err);
  }
  h->dirty = false;
  return FS_OK;
}

int create_compat(fs_handle *h, const fs_net_desc *d) {
  const fs_neurons &v = d->neurons;
  const uint32_t n = v.n;
  const size_t nr = (size_t)FS_NREC * n;
  fsd::CompatDev &c = h->cd;
  c.n = n;
  c.glob = d->act_ctr;
  int rc = 0;
#define UP(field, src, cnt) \
  if ((rc = upload(h, (std::remove_const<std::remove_pointer<decltype(c.field)>::type>::type **)&c.field, src, cnt))) return rc
  UP(Vth, v.Vth, n); UP(El, v.El, n); UP(gl, v.gl, n); UP(Cm, v.Cm, n); UP(Vreset, v.Vreset, n);
  UP(df, v.df, n); UP(ef, v.ef, n); UP(dVmax, v.dVmax, n); UP(RfPed, v.RfPed, n); UP(SpiDy, v.SpiDy, n);
  UP(Vrev, v.Vrev, nr); UP(dfst, v.dfst, nr); UP(nmda_dfxt, v.nmda_dfxt, n); UP(nmda_efst, v.nmda_efst, n);
  UP(nmda_as, v.nmda_as, n); UP(nmda_mg, v.nmda_mg, n); UP(ext_g, v.ext_g, nr);
  UP(pb, h->pb.data(), nr); UP(act, h->act.data(), n);
  UP(inj_mean, h->inj_mean.data(), n); UP(inj_std, h->inj_std.data(), n);
  UP(stp_pv, v.stp_pv, n); UP(stp_dfD, v.stp_dfD, n); UP(stp_efD, v.stp_efD, n); UP(stp_aF, v.stp_aF, n);
  UP(stp_dfF, v.stp_dfF, n); UP(stp_efF, v.stp_efF, n); UP(stp_aCap, v.stp_aCap, n);
  UP(stp_dfCap, v.stp_dfCap, n); UP(stp_aCar, v.stp_aCar, n); UP(stp_dfCar, v.stp_dfCar, n);
  UP(stp_efCar, v.stp_efCar, n);
  UP(ltp_dfLP, v.ltp_dfLP, n); UP(ltp_Pos, v.ltp_PosISI, n); UP(ltp_Neg, v.ltp_NegISI, n);
  UP(ltp_SpiLPDy, v.ltp_SpiLPDy, n);
#undef UP
  if ((rc = zeros(h, &c.V, n)) || (rc = zeros(h, &c.Isyn, n)) || (rc = zeros(h, &c.G, nr)) ||
      (rc = zeros(h, &c.ext_st, (size_t)4 * n)) || (rc = zeros(h, &c.ext_xt_n, n)) ||
      (rc = zeros(h, &c.ext_st_n, n)) || (rc = zeros(h, &c.Irep, nr)) || (rc = zeros(h, &c.D, n)) ||
      (rc = zeros(h, &c.F, n)) || (rc = zeros(h, &c.Cap, n)) || (rc = zeros(h, &c.Car, n)) ||
      (rc = zeros(h, &c.LP, n)) || (rc = zeros(h, &c.Count, n)) || (rc = zeros(h, &c.CountLP, n)) ||
      (rc = zeros(h, &c.NS, n)))
    return rc;
  c.gate_off[0] = 0;
  c.rec_off[0] = 0;
  for (int r = 0; r < FS_NREC; r++) {
    const fs_rec_layout &L = d->compat->rec[r];
    fsd::RecDev &R = c.R[r];
    R.n_gates = L.n_gates;
    R.n_recs = L.n_recs;
    if ((rc = upload(h, (uint32_t **)&R.gate_pre, L.gate_pre, L.n_gates)) ||
        (rc = upload(h, (uint32_t **)&R.gate_post0, L.gate_post0, L.n_gates)) ||
        (rc = upload(h, (float **)&R.gate_g, L.gate_g, L.n_gates)) ||
        (rc = zeros(h, &R.gate_st, L.n_gates)) || (rc = zeros(h, &R.gate_xt, L.n_gates)))
      return rc;
    R.grow = nullptr;
    R.ggate = nullptr;
    if (L.gather_rowptr) {
      const uint32_t ne = L.gather_rowptr[n];
      if (ne) {
        if ((rc = upload(h, (uint32_t **)&R.grow, L.gather_rowptr, (size_t)n + 1)) ||
            (rc = upload(h, (uint32_t **)&R.ggate, L.gather_gate, ne)))
          return rc;
        for (uint32_t e = 0; e < ne; e++)
          if (L.gather_gate[e] >= L.n_gates) return set_err(h, FS_ERR_ARG, "gather_gate index out of range");
      }
    }
    for (uint32_t k = 0; k < L.n_gates; k++)
      if (L.gate_pre[k] >= n || L.gate_post0[k] >= n) return set_err(h, FS_ERR_ARG, "gate neuron index out of range");
    R.rrow = nullptr;
    if ((rc = upload(h, (uint32_t **)&R.rpre, L.rec_pre, L.n_recs)) ||
        (rc = upload(h, (uint32_t **)&R.rpost, L.rec_post, L.n_recs)) ||
        (rc = upload(h, &R.rg, L.rec_g, L.n_recs)) || (rc = zeros(h, &R.rst, L.n_recs)) ||
        (rc = zeros(h, &R.rxt, L.n_recs)))
      return rc;
    if (L.n_recs) {
      if (!L.rec_rowptr || L.rec_rowptr[n] != L.n_recs)
        return set_err(h, FS_ERR_ARG, "rec_rowptr missing or inconsistent");
      if ((rc = upload(h, (uint32_t **)&R.rrow, L.rec_rowptr, (size_t)n + 1))) return rc;
      for (uint32_t e = 0; e < L.n_recs; e++)
        if (L.rec_pre[e] >= n || L.rec_post[e] >= n) return set_err(h, FS_ERR_ARG, "record neuron index out of range");
    }
    c.gate_off[r + 1] = c.gate_off[r] + L.n_gates;
    c.rec_off[r + 1] = c.rec_off[r] + L.n_recs;
  }
  c.gap_row = nullptr;
  if (d->compat->gap_rowptr && d->compat->gap_rowptr[n]) {
    const uint32_t ne = d->compat->gap_rowptr[n];
    for (uint32_t e = 0; e < ne; e++)
      if (d->compat->gap_other[e] >= n) return set_err(h, FS_ERR_ARG, "gap index out of range");
    if ((rc = upload(h, (uint32_t **)&c.gap_row, d->compat->gap_rowptr, (size_t)n + 1)) ||
        (rc = upload(h, (uint32_t **)&c.gap_other, d->compat->gap_other, ne)) ||
        (rc = upload(h, (float **)&c.gap_g, d->compat->gap_g, ne)))
      return rc;
  }
  // random streams
  if ((rc = zeros(h, &h->drawoff, n)) || (rc = zeros(h, &h->injoff, n))) return rc;
  c.drawoff = h->drawoff;
  c.injoff = h->injoff;
  if ((rc = zeros(h, &h->mt_state, 624)) || (rc = zeros(h, &h->mt_pos, 1))) return rc;
  // exception tables
  std::vector<uint32_t> ek, lk;
  std::vector<float> ev, lv;
  const std::string dir = lib_dir();
  if (!fsh::read_table(dir + "/expf_glibc.bin", ek, ev) || !fsh::read_table(dir + "/logf_glibc.bin", lk, lv))
    return set_err(h, FS_ERR_IO, "missing " + dir + "/expf_glibc.bin or logf_glibc.bin (run the build)");
  if ((rc = upload(h, (uint32_t **)&c.expf_keys, ek.data(), ek.size())) ||
      (rc = upload(h, (float **)&c.expf_vals, ev.data(), ev.size())) ||
      (rc = upload(h, (uint32_t **)&c.logf_keys, lk.data(), lk.size())) ||
      (rc = upload(h, (float **)&c.logf_vals, lv.data(), lv.size())))
    return rc;
  c.expf_n = (uint32_t)ek.size();
  c.logf_n = (uint32_t)lk.size();
  uint32_t kn[128], ja[32], jc[32];
  float fn[128], wn[128];
  host_tables(kn, fn, wn, ja, jc);
  fsd::compat_set_tables(kn, fn, wn, ja, jc, h->st);
  CK(cudaGetLastError());
  if ((rc = zeros(h, &h->derr, 1))) return rc;
  c.err = h->derr;
  CK(cudaStreamSynchronize(h->st));  // host sources of the uploads are released after this call
  return FS_OK;
}

int compat_batch(fs_handle *h, uint32_t nsteps, fs_step_out *out, uint64_t *written, uint32_t done) {
  fsd::CompatDev &c = h->cd;
  const uint32_t n = h->n, words = (n + 31) / 32;
  int rc;
  if ((rc = ensure_batch(h, nsteps))) return rc;
  // draw buffer
  const uint64_t need = (uint64_t)nsteps * c.draws_per_step;
  if (need > h->draws_cap) {
    if ((rc = dalloc(h, &h->draws, (size_t)need))) return rc;
    h->draws_cap = need;
  }
  CK(fsd::mt_generate(h->mt_state, h->mt_pos, h->draws, need, h->st));
  h->launches += need ? 1 : 0;
  c.draws = h->draws;
  c.jcong_base = h->jcong;
  c.spikebits = h->spikebits;
  c.words = words;
  // optional per-step outputs
  const bool wantV = out && out->V, wantI = out && out->Irep, wantN = out && out->nstate;
  if ((wantV || wantI || wantN) && nsteps > h->out_cap_steps) {
    if ((rc = dalloc(h, &h->outV, (size_t)nsteps * n)) || (rc = dalloc(h, &h->outIrep, (size_t)nsteps * FS_NREC * n)) ||
        (rc = dalloc(h, &h->outNS, (size_t)nsteps * n)))
      return rc;
    h->out_cap_steps = nsteps;
  }
  c.outV = wantV ? h->outV : nullptr;
  c.outIrep = wantI ? h->outIrep : nullptr;
  c.outNS = wantN ? h->outNS : nullptr;
  c.gv_n = 0;
  if (out && out->gv_n && out->gv_sel) {
    const uint64_t need_gv = (uint64_t)nsteps * out->gv_n;
    if (need_gv > h->gv_cap) {
      if ((rc = dalloc(h, &h->gv_st, (size_t)need_gv)) || (rc = dalloc(h, &h->gv_xt, (size_t)need_gv))) return rc;
      h->gv_cap = (uint32_t)need_gv;
    }
    for (uint32_t q = 0; q < out->gv_n; q++) {
      const uint32_t r = out->gv_sel[q] >> 28, e = out->gv_sel[q] & 0x0fffffffu;
      if (r >= FS_NREC || e >= c.R[r].n_recs) return set_err(h, FS_ERR_ARG, "gv_sel entry out of range");
    }
    if (out->gv_n > h->gv_sel_cap) {
      if ((rc = dalloc(h, &h->gv_sel, out->gv_n))) return rc;
      h->gv_sel_cap = out->gv_n;
    }
    CK(cudaMemcpyAsync(h->gv_sel, out->gv_sel, (size_t)out->gv_n * 4, cudaMemcpyHostToDevice, h->st));
    c.gv_sel = h->gv_sel;
    c.gv_n = out->gv_n;
    c.gv_st = h->gv_st;
    c.gv_xt = h->gv_xt;
  }
  for (uint32_t s = 0; s < nsteps; s++) CK(fsd::compat_step(c, s, h->sm_count, h->st, &h->launches));
  CK(fsd::spikes_compact(h->spikebits, nsteps, words, h->counts, h->offsets, h->idx, h->st, &h->launches));
  h->jcong = jcong_advance(h->jcong, (uint64_t)nsteps * c.inj_per_step);
  uint32_t total = 0;
  CK(cudaMemcpyAsync(&total, h->offsets + nsteps, 4, cudaMemcpyDeviceToHost, h->st));
  if (out && out->spike_count)
    CK(cudaMemcpyAsync(out->spike_count + done, h->counts, (size_t)nsteps * 4, cudaMemcpyDeviceToHost, h->st));
  CK(cudaStreamSynchronize(h->st));
  int derr = 0;
  CK(cudaMemcpy(&derr, h->derr, 4, cudaMemcpyDeviceToHost));
  if (derr) return set_err(h, FS_ERR_TIMEOUT, "ziggurat rejection loop exceeded its bound");
  h->spikes_total += total;
  if (out && out->spike_idx) {
    if (*written + total > out->spike_cap) return set_err(h, FS_ERR_CAPACITY, "spike_idx buffer too small");
    CK(cudaMemcpy(out->spike_idx + *written, h->idx, (size_t)total * 4, cudaMemcpyDeviceToHost));
  }
  *written += total;
  if (wantV) CK(cudaMemcpy(out->V + (size_t)done * n, h->outV, (size_t)nsteps * n * 4, cudaMemcpyDeviceToHost));
  if (wantI)
    CK(cudaMemcpy(out->Irep + (size_t)done * FS_NREC * n, h->outIrep, (size_t)nsteps * FS_NREC * n * 4,
                  cudaMemcpyDeviceToHost));
  if (wantN) CK(cudaMemcpy(out->nstate + (size_t)done * n, h->outNS, (size_t)nsteps * n * 4, cudaMemcpyDeviceToHost));
  if (c.gv_n) {
    if (out->gv_st)
      CK(cudaMemcpy(out->gv_st + (size_t)done * c.gv_n, h->gv_st, (size_t)nsteps * c.gv_n * 4, cudaMemcpyDeviceToHost));
    if (out->gv_xt)
      CK(cudaMemcpy(out->gv_xt + (size_t)done * c.gv_n, h->gv_xt, (size_t)nsteps * c.gv_n * 4, cudaMemcpyDeviceToHost));
  }
  return FS_OK;
}

// steps per batch for compat: bounded by the draw buffer (<= 256 MB) and the
// spike buffers
uint32_t compat_batch_steps(fs_handle *h, uint32_t left) {
  uint64_t lim = h->chunk;
  const uint64_t D = std::max<uint32_t>(1, h->cd.draws_per_step);
  lim = std::min<uint64_t>(lim, std::max<uint64_t>(1, (64ull << 20) / D));
  lim = std::min<uint64_t>(lim, std::max<uint64_t>(1, (64ull << 20) / std::max<uint32_t>(1, h->n)));
  return (uint32_t)std::min<uint64_t>(lim, left);
}

}  // namespace

extern "C" {

int fs_abi_version(void) { return FS_ABI_VERSION; }

const char *fs_last_error(const fs_handle *h) { return h ? h->err.c_str() : g_err.c_str(); }

int fs_device_count(int *count) {
  int c = 0;
  cudaError_t e = cudaGetDeviceCount(&c);
  if (count) *count = (e == cudaSuccess) ? c : 0;
  if (e != cudaSuccess) return set_err(nullptr, FS_ERR_NODEVICE, cudaGetErrorString(e));
  return FS_OK;
}

int fs_create(const fs_net_desc *desc, const fs_run_opts *opts, fs_handle **out) {
  if (!out) return set_err(nullptr, FS_ERR_ARG, "fs_create: out is NULL");
  *out = nullptr;
  if (!desc || desc->neurons.n == 0) return set_err(nullptr, FS_ERR_ARG, "fs_create: empty network");
  fs_run_opts o{};
  if (opts) o = *opts;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    return set_err(nullptr, FS_ERR_NODEVICE, "fs_create: no CUDA device visible");
  if (o.device < 0 || o.device >= ndev) return set_err(nullptr, FS_ERR_ARG, "fs_create: bad device ordinal");
  if (o.mode == FS_MODE_COMPAT && !desc->compat)
    return set_err(nullptr, FS_ERR_ARG, "fs_create: FS_MODE_COMPAT needs desc->compat");
  if ((o.mode == FS_MODE_FP32 || o.mode == FS_MODE_FP64) && !desc->syn)
    return set_err(nullptr, FS_ERR_ARG, "fs_create: production modes need desc->syn");
  if (o.mode < FS_MODE_COMPAT || o.mode > FS_MODE_FP64) return set_err(nullptr, FS_ERR_ARG, "fs_create: bad mode");
  fs_handle *h = new fs_handle();
  h->mode = o.mode;
  h->device = o.device;
  h->n = desc->neurons.n;
  h->dt = desc->dt;
  h->glob = desc->act_ctr;
  h->chunk = o.chunk_steps ? o.chunk_steps : 1000;
  const uint32_t n = h->n;
  const size_t nr = (size_t)FS_NREC * n;
  auto cp = [](std::vector<float> &dst, const float *src, size_t k) {
    dst.assign(k, 0.0f);
    if (src) std::memcpy(dst.data(), src, k * 4);
  };
  cp(h->pb, desc->neurons.pb, nr);
  cp(h->inj_mean, desc->neurons.inj_mean, n);
  cp(h->inj_std, desc->neurons.inj_std, n);
  h->act.assign(n, desc->act_ctr);
  if (desc->neurons.act) std::memcpy(h->act.data(), desc->neurons.act, (size_t)n * 4);
  int rc = FS_OK;
  cudaError_t e = cudaSetDevice(o.device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&h->st, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreate(&h->ev0);
  if (e == cudaSuccess) e = cudaEventCreate(&h->ev1);
  if (e != cudaSuccess) {
    rc = cuda_err(h, e, "fs_create");
  } else {
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, o.device);
    h->sm_count = (uint32_t)sms;
    if (o.mode == FS_MODE_COMPAT) rc = create_compat(h, desc);
    else rc = fsp::prod_create(&h->prod, desc, o, h->sm_count, h->st, h->err);
    if (rc && h->err.empty()) h->err = "fs_create failed";
  }
  if (rc) {
    g_err = h->err;
    fs_destroy(h);
    return rc;
  }
  *out = h;
  return FS_OK;
}

int fs_destroy(fs_handle *h) {
  if (!h) return FS_OK;
  cudaSetDevice(h->device);
  if (h->st) cudaStreamSynchronize(h->st);
  if (h->prod) fsp::prod_destroy(h->prod);
  for (void *p : h->allocs) cudaFree(p);
  if (h->ev0) cudaEventDestroy(h->ev0);
  if (h->ev1) cudaEventDestroy(h->ev1);
  if (h->st) cudaStreamDestroy(h->st);
  delete h;
  return FS_OK;
}

int fs_reset(fs_handle *h, uint32_t mt_seed, uint32_t jcong_seed) {
  if (!h) return set_err(nullptr, FS_ERR_ARG, "fs_reset: null handle");
  CK(cudaSetDevice(h->device));
  int rc = upload_params(h);
  if (rc) return rc;
  if (h->mode == FS_MODE_COMPAT) {
    CK(fsd::compat_varinit(h->cd, h->st));
    // std::mt19937::seed (the standard's initialisation recurrence)
    uint32_t x[624];
    x[0] = mt_seed;
    for (uint32_t i = 1; i < 624; i++) x[i] = 1812433253u * (x[i - 1] ^ (x[i - 1] >> 30)) + i;
    const uint32_t pos = 624;
    CK(cudaMemcpyAsync(h->mt_state, x, sizeof x, cudaMemcpyHostToDevice, h->st));
    CK(cudaMemcpyAsync(h->mt_pos, &pos, 4, cudaMemcpyHostToDevice, h->st));
    h->jcong = jcong_seed;
    CK(cudaStreamSynchronize(h->st));
  } else {
    rc = fsp::prod_reset(h->prod, mt_seed, h->st, h->err);
    if (rc) return set_err(h, rc, h->err);
  }
  h->steps_done = 0;
  h->spikes_total = 0;
  return FS_OK;
}

int fs_set_drive(fs_handle *h, uint32_t first, uint32_t count, int rec, float pb) {
  if (!h) return set_err(nullptr, FS_ERR_ARG, "null handle");
  if (rec < 0 || rec >= FS_NREC || (uint64_t)first + count > h->n) return set_err(h, FS_ERR_ARG, "fs_set_drive: bad range");
  std::fill(h->pb.begin() + (size_t)rec * h->n + first, h->pb.begin() + (size_t)rec * h->n + first + count, pb);
  h->dirty = true;
  return FS_OK;
}

int fs_set_act(fs_handle *h, uint32_t first, uint32_t count, uint32_t clear_mask, uint32_t set_mask) {
  if (!h) return set_err(nullptr, FS_ERR_ARG, "null handle");
  if ((uint64_t)first + count > h->n) return set_err(h, FS_ERR_ARG, "fs_set_act: bad range");
  for (uint32_t i = first; i < first + count; i++) h->act[i] = (h->act[i] & ~clear_mask) | set_mask;
  h->dirty = true;
  return FS_OK;
}

int fs_set_injection(fs_handle *h, uint32_t first, uint32_t count, float mean, float sd) {
  if (!h) return set_err(nullptr, FS_ERR_ARG, "null handle");
  if ((uint64_t)first + count > h->n) return set_err(h, FS_ERR_ARG, "fs_set_injection: bad range");
  std::fill(h->inj_mean.begin() + first, h->inj_mean.begin() + first + count, mean);
  std::fill(h->inj_std.begin() + first, h->inj_std.begin() + first + count, sd);
  h->dirty = true;
  return FS_OK;
}

int fs_step(fs_handle *h, uint32_t nsteps, fs_step_out *out) {
  if (!h) return set_err(nullptr, FS_ERR_ARG, "null handle");
  CK(cudaSetDevice(h->device));
  int rc = upload_params(h);
  if (rc) return rc;
  uint64_t written = 0;
  const uint64_t l0 = h->launches;
  CK(cudaEventRecord(h->ev0, h->st));
  if (h->mode == FS_MODE_COMPAT) {
    uint32_t done = 0;
    while (done < nsteps) {
      const uint32_t b = compat_batch_steps(h, nsteps - done);
      rc = compat_batch(h, b, out, &written, done);
      if (rc) return rc;
      done += b;
    }
  } else {
    rc = fsp::prod_step(h->prod, nsteps, out, &written, h->st, &h->launches, &h->spikes_total, h->err);
    if (rc) return set_err(h, rc, h->err);
  }
  CK(cudaEventRecord(h->ev1, h->st));
  CK(cudaEventSynchronize(h->ev1));
  float ms = 0;
  CK(cudaEventElapsedTime(&ms, h->ev0, h->ev1));
  h->kernel_ms = ms;
  h->kernel_launches = h->launches - l0;
  if (out) out->spike_total = written;
  h->steps_done += nsteps;
  return FS_OK;
}

int fs_run(fs_handle *h, uint32_t nsteps) {
  if (!h) return set_err(nullptr, FS_ERR_ARG, "null handle");
  CK(cudaSetDevice(h->device));
  int rc = upload_params(h);
  if (rc) return rc;
  const uint64_t l0 = h->launches;
  if (h->mode == FS_MODE_COMPAT) {
    uint32_t done = 0;
    uint64_t written = 0;
    while (done < nsteps) {
      const uint32_t b = compat_batch_steps(h, nsteps - done);
      rc = compat_batch(h, b, nullptr, &written, done);
      if (rc) return rc;
      done += b;
    }
  } else {
    rc = fsp::prod_run(h->prod, nsteps, h->st, &h->launches, h->err);
    if (rc) return set_err(h, rc, h->err);
  }
  h->kernel_launches = h->launches - l0;
  h->steps_done += nsteps;
  return FS_OK;
}

int fs_run_timed(fs_handle *h, uint32_t nsteps, double *device_ms) {
  if (!h) return set_err(nullptr, FS_ERR_ARG, "null handle");
  CK(cudaSetDevice(h->device));
  int rc = upload_params(h);
  if (rc) return rc;
  CK(cudaEventRecord(h->ev0, h->st));
  rc = fs_run(h, nsteps);
  if (rc) return rc;
  CK(cudaEventRecord(h->ev1, h->st));
  CK(cudaEventSynchronize(h->ev1));
  float ms = 0;
  CK(cudaEventElapsedTime(&ms, h->ev0, h->ev1));
  if (device_ms) *device_ms = ms;
  return fs_sync(h);
}

int fs_sync(fs_handle *h) {
  if (!h) return set_err(nullptr, FS_ERR_ARG, "null handle");
  CK(cudaStreamSynchronize(h->st));
  if (h->prod) {
    int rc = fsp::prod_check(h->prod, h->st, &h->spikes_total, h->err);
    if (rc) return set_err(h, rc, h->err);
  }
  return FS_OK;
}

int fs_stats(fs_handle *h, uint64_t *steps_done, uint64_t *spikes_total, uint64_t *kernel_launches) {
  if (!h) return set_err(nullptr, FS_ERR_ARG, "null handle");
  if (steps_done) *steps_done = h->steps_done;
  if (spikes_total) *spikes_total = h->spikes_total;
  if (kernel_launches) *kernel_launches = h->launches;
  return FS_OK;
}

int fs_kernel_time(fs_handle *h, double *ms_per_launch, uint64_t *launches) {
  if (!h) return set_err(nullptr, FS_ERR_ARG, "null handle");
  if (h->prod) {
    double ms = 0;
    uint64_t l = 0;
    fsp::prod_kernel_time(h->prod, &ms, &l);
    if (ms_per_launch) *ms_per_launch = ms;
    if (launches) *launches = l;
    return FS_OK;
  }
  if (ms_per_launch) *ms_per_launch = h->kernel_launches ? h->kernel_ms / (double)h->kernel_launches : 0.0;
  if (launches) *launches = h->kernel_launches;
  return FS_OK;
}

int fs_get_state(fs_handle *h, float *V, int32_t *Count, uint32_t *NState) {
  if (!h) return set_err(nullptr, FS_ERR_ARG, "null handle");
  CK(cudaStreamSynchronize(h->st));
  if (h->mode != FS_MODE_COMPAT) {
    int rc = fsp::prod_get_state(h->prod, V, Count, NState, h->st, h->err);
    if (rc) return set_err(h, rc, h->err);
    return FS_OK;
  }
  const size_t n = h->n;
  if (V) CK(cudaMemcpy(V, h->cd.V, n * 4, cudaMemcpyDeviceToHost));
  if (Count) CK(cudaMemcpy(Count, h->cd.Count, n * 4, cudaMemcpyDeviceToHost));
  if (NState) CK(cudaMemcpy(NState, h->cd.NS, n * 4, cudaMemcpyDeviceToHost));
  return FS_OK;
}

int fs_get_weights(fs_handle *h, float *g, uint64_t n) {
  if (!h) return set_err(nullptr, FS_ERR_ARG, "null handle");
  if (h->mode == FS_MODE_COMPAT || !h->prod)
    return set_err(h, FS_ERR_UNSUPPORTED, "fs_get_weights: production modes only");
  if (n && !g) return set_err(h, FS_ERR_ARG, "fs_get_weights: null output");
  int rc = fsp::prod_get_weights(h->prod, g, n, h->st, h->err);
  return rc ? set_err(h, rc, h->err) : FS_OK;
}

int fs_debug_barrier_timeout(uint32_t poll_limit) {
  if (poll_limit == 0 || poll_limit > (1u << 24))
    return set_err(nullptr, FS_ERR_ARG, "fs_debug_barrier_timeout: poll limit must be 1 .. 2^24");
  std::string err;
  int word = 0;
  int rc = fsp::prod_barrier_probe(poll_limit, &word, err);
  if (rc) return set_err(nullptr, rc, err);
  if (word) return set_err(nullptr, FS_ERR_TIMEOUT, "barrier wait gave up (device error word set)");
  return FS_OK;
}

int fs_engine_layout(fs_handle *h, uint32_t *blocks, uint32_t *threads, uint32_t *interval, int *kernel) {
  if (!h) return set_err(nullptr, FS_ERR_ARG, "null handle");
  if (h->mode == FS_MODE_COMPAT || !h->prod)
    return set_err(h, FS_ERR_UNSUPPORTED, "fs_engine_layout: production modes only");
  fsp::ProdInfo pi{};
  fsp::prod_info(h->prod, &pi);
  if (blocks) *blocks = pi.blocks;
  if (threads) *threads = pi.threads;
  if (interval) *interval = pi.interval;
  if (kernel) *kernel = pi.single_step ? 1 : pi.tiles ? 2 : pi.ltp ? 3 : 0;
  return FS_OK;
}

int fs_debug_single_step_plan(const fs_net_desc *desc, uint32_t sm_count, uint64_t *stats) {
  if (!desc || !desc->syn || !stats || sm_count == 0)
    return set_err(nullptr, FS_ERR_ARG, "fs_debug_single_step_plan: null argument");
  std::string err;
  int rc = fsp::prod_check_single_plan(desc, sm_count, stats, err);
  if (!rc && !stats[0]) set_err(nullptr, FS_OK, err.empty() ? "not taken (delays or mode)" : err);
  return rc ? set_err(nullptr, rc, err) : FS_OK;
}

int fs_debug_philox(const uint32_t *ctr, const uint32_t *key, uint64_t k, uint32_t *out) {
  if (k == 0) return FS_OK;
  if (!ctr || !key || !out) return set_err(nullptr, FS_ERR_ARG, "fs_debug_philox: null argument");
  if (k > (1ull << 26)) return set_err(nullptr, FS_ERR_ARG, "fs_debug_philox: at most 2^26 blocks per call");
  std::string err;
  int rc = fsp::prod_debug_philox(ctr, key, k, out, err);
  return rc ? set_err(nullptr, rc, err) : FS_OK;
}

int fs_debug_drive(fs_handle *h, uint64_t t0, uint32_t nsteps, uint32_t first, uint32_t count, uint8_t *hits,
                   double *gauss) {
  if (!h) return set_err(nullptr, FS_ERR_ARG, "null handle");
  if (h->mode == FS_MODE_COMPAT || !h->prod)
    return set_err(h, FS_ERR_UNSUPPORTED, "fs_debug_drive: the Philox drive belongs to the production modes");
  if (!hits || !gauss) return set_err(h, FS_ERR_ARG, "fs_debug_drive: null output");
  if ((uint64_t)first + count > h->n) return set_err(h, FS_ERR_ARG, "fs_debug_drive: neuron range out of bounds");
  if ((uint64_t)nsteps * count > (1ull << 28)) return set_err(h, FS_ERR_ARG, "fs_debug_drive: at most 2^28 draws per call");
  if (nsteps == 0 || count == 0) return FS_OK;
  CK(cudaSetDevice(h->device));
  int rc = upload_params(h);
  if (rc) return rc;
  rc = fsp::prod_debug_drive(h->prod, t0, nsteps, first, count, hits, gauss, h->st, h->err);
  return rc ? set_err(h, rc, h->err) : FS_OK;
}

int fs_debug_phase_clock(fs_handle *h, int enable) {
  if (!h) return set_err(nullptr, FS_ERR_ARG, "null handle");
  if (h->mode == FS_MODE_COMPAT || !h->prod)
    return set_err(h, FS_ERR_UNSUPPORTED, "fs_debug_phase_clock: production modes only");
  CK(cudaSetDevice(h->device));
  int rc = fsp::prod_phase_clock(h->prod, enable, h->st, h->err);
  return rc ? set_err(h, rc, h->err) : FS_OK;
}

int fs_debug_phase_times(fs_handle *h, uint64_t *out, uint32_t cap, uint32_t *blocks) {
  if (!h) return set_err(nullptr, FS_ERR_ARG, "null handle");
  if (h->mode == FS_MODE_COMPAT || !h->prod)
    return set_err(h, FS_ERR_UNSUPPORTED, "fs_debug_phase_times: production modes only");
  CK(cudaSetDevice(h->device));
  int rc = fsp::prod_phase_times(h->prod, out, cap, blocks, h->st, h->err);
  return rc ? set_err(h, rc, h->err) : FS_OK;
}

int fs_debug_inject_wait_failure(fs_handle *h) {
  if (!h) return set_err(nullptr, FS_ERR_ARG, "null handle");
  if (h->mode == FS_MODE_COMPAT || !h->prod)
    return set_err(h, FS_ERR_UNSUPPORTED, "fs_debug_inject_wait_failure: production modes only");
  CK(cudaSetDevice(h->device));
  int rc = fsp::prod_inject_wait_failure(h->prod, h->st, h->err);
  return rc ? set_err(h, rc, h->err) : FS_OK;
}

// ---- checkpoints (production modes) ----------------------------------------
// Layout: CkptHead, the event-set parameters (pb [FS_NREC][n], act [n],
// inj_mean [n], inj_std [n]), then the engine's state blob.
namespace {
struct CkptHead {
  char magic[8];
  uint32_t version, mode, n, fp64, slots, interval, lin_receptors, pad;
  uint64_t lin_edges, nmda_edges, state_bytes, total_bytes;
};
constexpr char kCkptMagic[8] = {'F', 'S', 'B', '2', 'C', 'K', 'P', '\0'};

int ckpt_head(fs_handle *h, CkptHead &c) {
  if (!h) return set_err(nullptr, FS_ERR_ARG, "null handle");
  if (h->mode == FS_MODE_COMPAT || !h->prod)
    return set_err(h, FS_ERR_UNSUPPORTED, "checkpoints need a production mode (FS_MODE_FP32 or FS_MODE_FP64)");
  fsp::ProdInfo pi{};
  fsp::prod_info(h->prod, &pi);
  std::memset(&c, 0, sizeof c);
  std::memcpy(c.magic, kCkptMagic, 8);
  c.version = 1;
  c.mode = (uint32_t)h->mode;
  c.n = h->n;
  c.fp64 = (uint32_t)pi.fp64;
  c.slots = pi.slots;
  c.interval = pi.interval;
  c.lin_receptors = pi.lin_receptors;
  c.lin_edges = pi.lin_edges;
  c.nmda_edges = pi.nmda_edges;
  c.state_bytes = fsp::prod_state_bytes(h->prod);
  c.total_bytes = sizeof(CkptHead) + (uint64_t)h->n * 4 * (FS_NREC + 3) + c.state_bytes;
  return FS_OK;
}
}  // namespace

int fs_checkpoint_size(fs_handle *h, uint64_t *bytes) {
  CkptHead c;
  int rc = ckpt_head(h, c);
  if (rc) return rc;
  if (!bytes) return set_err(h, FS_ERR_ARG, "fs_checkpoint_size: null bytes");
  *bytes = c.total_bytes;
  return FS_OK;
}

int fs_checkpoint_save(fs_handle *h, void *buf, uint64_t cap, uint64_t *bytes) {
  CkptHead c;
  int rc = ckpt_head(h, c);
  if (rc) return rc;
  if (bytes) *bytes = c.total_bytes;
  if (!buf) return set_err(h, FS_ERR_ARG, "fs_checkpoint_save: null buffer");
  if (cap < c.total_bytes) return set_err(h, FS_ERR_CAPACITY, "fs_checkpoint_save: buffer smaller than fs_checkpoint_size");
  CK(cudaSetDevice(h->device));
  // the work in flight must have ended cleanly: a state whose barrier wait
  // gave up is half an interval and is never saved
  rc = fsp::prod_check(h->prod, h->st, &h->spikes_total, h->err);
  if (rc) return set_err(h, rc, "fs_checkpoint_save: " + h->err);
  uint8_t *o = (uint8_t *)buf;
  const size_t n = h->n;
  std::memcpy(o, &c, sizeof c);
  o += sizeof c;
  std::memcpy(o, h->pb.data(), (size_t)FS_NREC * n * 4);
  o += (size_t)FS_NREC * n * 4;
  std::memcpy(o, h->act.data(), n * 4);
  o += n * 4;
  std::memcpy(o, h->inj_mean.data(), n * 4);
  o += n * 4;
  std::memcpy(o, h->inj_std.data(), n * 4);
  o += n * 4;
  rc = fsp::prod_state_save(h->prod, o, h->st, h->err);
  if (rc) return set_err(h, rc, h->err);
  return FS_OK;
}

int fs_checkpoint_load(fs_handle *h, const void *buf, uint64_t bytes) {
  CkptHead c;
  int rc = ckpt_head(h, c);
  if (rc) return rc;
  if (!buf || bytes < sizeof(CkptHead)) return set_err(h, FS_ERR_ARG, "fs_checkpoint_load: no checkpoint");
  CkptHead f;
  std::memcpy(&f, buf, sizeof f);
  if (std::memcmp(f.magic, kCkptMagic, 8) != 0 || f.version != c.version)
    return set_err(h, FS_ERR_ARG, "fs_checkpoint_load: not a checkpoint of this library version");
  if (f.mode != c.mode || f.n != c.n || f.fp64 != c.fp64 || f.slots != c.slots || f.interval != c.interval ||
      f.lin_receptors != c.lin_receptors || f.lin_edges != c.lin_edges || f.nmda_edges != c.nmda_edges ||
      f.state_bytes != c.state_bytes || f.total_bytes != c.total_bytes)
    return set_err(h, FS_ERR_ARG, "fs_checkpoint_load: checkpoint of another network or mode");
  if (bytes < c.total_bytes) return set_err(h, FS_ERR_ARG, "fs_checkpoint_load: checkpoint truncated");
  CK(cudaSetDevice(h->device));
  const uint8_t *i = (const uint8_t *)buf + sizeof f;
  const size_t n = h->n;
  std::memcpy(h->pb.data(), i, (size_t)FS_NREC * n * 4);
  i += (size_t)FS_NREC * n * 4;
  std::memcpy(h->act.data(), i, n * 4);
  i += n * 4;
  std::memcpy(h->inj_mean.data(), i, n * 4);
  i += n * 4;
  std::memcpy(h->inj_std.data(), i, n * 4);
  i += n * 4;
  h->dirty = true;
  rc = fsp::prod_state_load(h->prod, i, h->st, h->err);
  if (rc) return set_err(h, rc, h->err);
  uint64_t t = 0, spk = 0;
  std::memcpy(&t, i, 8);
  std::memcpy(&spk, i + c.state_bytes - 8, 8);
  h->steps_done = t;
  h->spikes_total = spk;
  return upload_params(h);
}

int fs_get_syn_state(fs_handle *h, float *g, float *Isyn) {
  if (!h) return set_err(nullptr, FS_ERR_ARG, "null handle");
  CK(cudaStreamSynchronize(h->st));
  if (h->mode != FS_MODE_COMPAT) return set_err(h, FS_ERR_UNSUPPORTED, "fs_get_syn_state: compat mode only");
  const size_t n = h->n;
  if (g) CK(cudaMemcpy(g, h->cd.G, (size_t)FS_NREC * n * 4, cudaMemcpyDeviceToHost));
  if (Isyn) CK(cudaMemcpy(Isyn, h->cd.Isyn, n * 4, cudaMemcpyDeviceToHost));
  return FS_OK;
}

// engine table over the C ABI (ctx = fs_handle*)
static int e_reset(void *c, uint32_t a, uint32_t b) { return fs_reset((fs_handle *)c, a, b); }
static int e_drive(void *c, uint32_t f, uint32_t k, int r, float p) { return fs_set_drive((fs_handle *)c, f, k, r, p); }
static int e_act(void *c, uint32_t f, uint32_t k, uint32_t cl, uint32_t s) { return fs_set_act((fs_handle *)c, f, k, cl, s); }
static int e_inj(void *c, uint32_t f, uint32_t k, float m, float s) { return fs_set_injection((fs_handle *)c, f, k, m, s); }
static int e_step(void *c, uint32_t k, fs_step_out *o) { return fs_step((fs_handle *)c, k, o); }
static const char *e_err(void *c) { return fs_last_error((fs_handle *)c); }
static const fs_engine_vtbl kDeviceEngine = {e_reset, e_drive, e_act, e_inj, e_step, e_err};
const fs_engine_vtbl *fs_device_engine(void) { return &kDeviceEngine; }

// device expf used by the NMDA Mg block, for checks against glibc; every
// exit path frees the four staging buffers
int fs_debug_expf(const float *x, float *y, uint64_t k) {
  std::vector<uint32_t> ek;
  std::vector<float> ev;
  if (k && (!x || !y)) return set_err(nullptr, FS_ERR_ARG, "fs_debug_expf: null x or y");
  if (!fsh::read_table(lib_dir() + "/expf_glibc.bin", ek, ev)) return set_err(nullptr, FS_ERR_IO, "missing expf table");
  if (k == 0) return FS_OK;
  struct Bufs {
    float *dx = nullptr, *dy = nullptr, *dv = nullptr;
    uint32_t *dk = nullptr;
    ~Bufs() {
      if (dx) cudaFree(dx);
      if (dy) cudaFree(dy);
      if (dk) cudaFree(dk);
      if (dv) cudaFree(dv);
    }
  } b;
  fs_handle tmp;
  fs_handle *h = &tmp;
  CK(cudaMalloc(&b.dx, k * 4));
  CK(cudaMalloc(&b.dy, k * 4));
  CK(cudaMalloc(&b.dk, ek.size() * 4));
  CK(cudaMalloc(&b.dv, ev.size() * 4));
  CK(cudaMemcpy(b.dx, x, k * 4, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(b.dk, ek.data(), ek.size() * 4, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(b.dv, ev.data(), ev.size() * 4, cudaMemcpyHostToDevice));
  CK(fsd::expf_ref_eval(b.dx, b.dy, k, b.dk, b.dv, (uint32_t)ek.size(), nullptr));
  CK(cudaMemcpy(y, b.dy, k * 4, cudaMemcpyDeviceToHost));
  return FS_OK;
}

}  // extern "C"

// ---- allocation-free device expf check ------------------------------------
// fs_debug_expf_noalloc runs the same kernel as fs_debug_expf, with its
// exception table and its staging buffers in one fixed device array instead
// of four cudaMalloc'd ones.  Layout of the array (4 MiB):
//   keys[kNaTable] u32 | vals[kNaTable] f32 | x[kNaMaxK] f32 | y[kNaMaxK] f32
// Nothing in it must start at zero: the table is written once at set-up and
// every x / y element a call reads is written earlier in the same call.
namespace {
constexpr uint64_t kNaMaxK = FS_NOALLOC_MAX_K;  // values per call
constexpr uint32_t kNaTable = 1u << 18;         // exception entries (glibc expf has 140,931)
constexpr size_t kNaBytes = (size_t)kNaTable * 8 + (size_t)kNaMaxK * 8;
static __device__ __align__(256) unsigned char g_na_scratch[kNaBytes];

constexpr int kNaDevices = 64;
struct NaDevice {
  bool ready;
  uint32_t nk;
  unsigned char *base;  // device address of g_na_scratch on this device
};
NaDevice g_na[kNaDevices];
std::mutex g_na_mu;
uint32_t g_na_keys[kNaTable];  // host staging of the table at set-up
float g_na_vals[kNaTable];

// One-time set-up on the current device `dev` (g_na_mu held): resolve the
// scratch address and upload the expf exception table.
int na_setup(int dev) {
  fs_handle *h = nullptr;
  unsigned char *base = nullptr;
  CK(cudaGetSymbolAddress((void **)&base, g_na_scratch));
  const std::string path = lib_dir() + "/expf_glibc.bin";
  FILE *f = std::fopen(path.c_str(), "rb");
  if (!f) return set_err(nullptr, FS_ERR_IO, "fs_debug_expf_noalloc: missing expf table " + path);
  uint32_t magic = 0, n = 0;
  bool ok = std::fread(&magic, 4, 1, f) == 1 && std::fread(&n, 4, 1, f) == 1 && magic == 0x46534554u &&
            n <= kNaTable && std::fread(g_na_keys, 4, n, f) == n && std::fread(g_na_vals, 4, n, f) == n;
  std::fclose(f);
  if (!ok) return set_err(nullptr, FS_ERR_IO, "fs_debug_expf_noalloc: unreadable expf table " + path);
  cudaStream_t st = cudaStreamPerThread;
  CK(cudaMemcpyAsync(base, g_na_keys, (size_t)n * 4, cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(base + (size_t)kNaTable * 4, g_na_vals, (size_t)n * 4, cudaMemcpyHostToDevice, st));
  CK(cudaStreamSynchronize(st));
  g_na[dev].base = base;
  g_na[dev].nk = n;
  g_na[dev].ready = true;
  return FS_OK;
}
}  // namespace

extern "C" int fs_debug_expf_noalloc(const float *x, float *y, uint64_t k) {
  fs_handle *h = nullptr;
  if (k > kNaMaxK)
    return set_err(nullptr, FS_ERR_ARG,
                   "fs_debug_expf_noalloc: k = " + std::to_string(k) + " exceeds the fixed scratch of " +
                       std::to_string(kNaMaxK) + " values per call; split the input or use fs_debug_expf");
  if (k && (!x || !y)) return set_err(nullptr, FS_ERR_ARG, "fs_debug_expf_noalloc: null x or y");
  int dev = 0;
  CK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kNaDevices) return set_err(nullptr, FS_ERR_ARG, "fs_debug_expf_noalloc: device ordinal >= 64");
  NaDevice s;
  {
    std::lock_guard<std::mutex> lock(g_na_mu);
    if (!g_na[dev].ready) {
      const int rc = na_setup(dev);
      if (rc) return rc;
    }
    s = g_na[dev];
  }
  if (k == 0) return FS_OK;
  const uint32_t *dk = (const uint32_t *)s.base;
  const float *dv = (const float *)(s.base + (size_t)kNaTable * 4);
  float *dx = (float *)(s.base + (size_t)kNaTable * 8);
  float *dy = dx + kNaMaxK;
  cudaStream_t st = cudaStreamPerThread;
  CK(cudaMemcpyAsync(dx, x, k * 4, cudaMemcpyHostToDevice, st));
  CK(fsd::expf_ref_eval(dx, dy, k, dk, dv, s.nk, st));
  CK(cudaMemcpyAsync(y, dy, k * 4, cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  return FS_OK;
}

// ---- batches of independent production networks -----------------------------
struct fs_batch {
  int device = 0;
  cudaStream_t st = nullptr;
  fsp::Batch *b = nullptr;
  fsp::BatchPlan tuned{};
  std::string err;
};

namespace {
int batch_err(fs_batch *b, int code, const std::string &msg) {
  if (b) b->err = msg;
  g_err = msg;
  return code;
}
}  // namespace

extern "C" {

int fs_batch_create(uint32_t count, const fs_net_desc *const *descs, const fs_run_opts *opts, fs_batch **out) {
  if (!out) return set_err(nullptr, FS_ERR_ARG, "fs_batch_create: out is NULL");
  *out = nullptr;
  fs_run_opts o{};
  if (opts) o = *opts;
  if (o.mode == FS_MODE_COMPAT) o.mode = FS_MODE_FP32;
  if (o.mode != FS_MODE_FP32 && o.mode != FS_MODE_FP64)
    return set_err(nullptr, FS_ERR_ARG, "fs_batch_create: batches run FS_MODE_FP32 or FS_MODE_FP64");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    return set_err(nullptr, FS_ERR_NODEVICE, "fs_batch_create: no CUDA device visible");
  if (o.device < 0 || o.device >= ndev) return set_err(nullptr, FS_ERR_ARG, "fs_batch_create: bad device ordinal");
  for (uint32_t i = 0; i < count; i++)
    if (!descs || !descs[i] || !descs[i]->syn || descs[i]->neurons.n == 0)
      return set_err(nullptr, FS_ERR_ARG, "fs_batch_create: instance " + std::to_string(i) + " has no synapse list");
  fs_batch *b = new fs_batch();
  b->device = o.device;
  cudaError_t e = cudaSetDevice(o.device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->st, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    const int rc = set_err(nullptr, FS_ERR_CUDA, std::string("fs_batch_create: ") + cudaGetErrorString(e));
    delete b;
    return rc;
  }
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, o.device);
  std::string err;
  int rc = fsp::batch_create(&b->b, count, descs, o, (uint32_t)sms, b->st, err);
  if (rc) {
    set_err(nullptr, rc, "fs_batch_create: " + err);
    cudaStreamDestroy(b->st);
    delete b;
    return rc;
  }
  *out = b;
  return FS_OK;
}

int fs_batch_destroy(fs_batch *b) {
  if (!b) return FS_OK;
  cudaSetDevice(b->device);
  if (b->st) cudaStreamSynchronize(b->st);
  fsp::batch_destroy(b->b);
  if (b->st) cudaStreamDestroy(b->st);
  delete b;
  return FS_OK;
}

const char *fs_batch_error(const fs_batch *b) { return b ? b->err.c_str() : g_err.c_str(); }

int fs_batch_reset(fs_batch *b, const uint32_t *seeds) {
  if (!b) return set_err(nullptr, FS_ERR_ARG, "fs_batch_reset: null batch");
  cudaSetDevice(b->device);
  int rc = fsp::batch_reset(b->b, seeds, b->st, b->err);
  return rc ? batch_err(b, rc, b->err) : FS_OK;
}

int fs_batch_tune(fs_batch *b, uint32_t sample_steps, fs_batch_plan *plan) {
  if (!b) return set_err(nullptr, FS_ERR_ARG, "fs_batch_tune: null batch");
  cudaSetDevice(b->device);
  fsp::BatchPlan p{};
  int rc = fsp::batch_tune(b->b, sample_steps, b->st, &p, b->err);
  if (rc) return batch_err(b, rc, b->err);
  if (plan) {
    plan->blocks = p.blocks;
    plan->blocks_per_sm = p.blocks_per_sm;
    plan->candidates = p.candidates;
    plan->tile_posts = p.tile_posts;
    plan->edges_in_flight = p.edges_in_flight;
    plan->sample_ms = p.sample_ms;
  }
  return FS_OK;
}

int fs_batch_run(fs_batch *b, uint32_t nsteps, double *device_ms) {
  if (!b) return set_err(nullptr, FS_ERR_ARG, "fs_batch_run: null batch");
  cudaSetDevice(b->device);
  int rc = fsp::batch_run(b->b, nsteps, b->st, device_ms, b->err);
  return rc ? batch_err(b, rc, b->err) : FS_OK;
}

int fs_batch_info(fs_batch *b, uint32_t *count, uint32_t *blocks, uint32_t *blocks_per_sm, int *graph,
                  uint64_t *launches) {
  if (!b) return set_err(nullptr, FS_ERR_ARG, "fs_batch_info: null batch");
  fsp::BatchPlan p{};
  fsp::batch_info(b->b, &p);
  if (count) *count = fsp::batch_size(b->b);
  if (blocks) *blocks = p.blocks;
  if (blocks_per_sm) *blocks_per_sm = p.blocks_per_sm;
  if (graph) *graph = p.graph;
  if (launches) *launches = p.launches;
  return FS_OK;
}

int fs_batch_spike_counts(fs_batch *b, uint32_t inst, uint32_t *counts) {
  if (!b || !counts) return set_err(nullptr, FS_ERR_ARG, "fs_batch_spike_counts: null argument");
  cudaSetDevice(b->device);
  int rc = fsp::batch_spike_counts(b->b, inst, counts, b->st, b->err);
  return rc ? batch_err(b, rc, b->err) : FS_OK;
}

int fs_batch_spike_totals(fs_batch *b, uint64_t *totals) {
  if (!b || !totals) return set_err(nullptr, FS_ERR_ARG, "fs_batch_spike_totals: null argument");
  cudaSetDevice(b->device);
  int rc = fsp::batch_spike_totals(b->b, totals, b->st, b->err);
  return rc ? batch_err(b, rc, b->err) : FS_OK;
}

int fs_set_gains(fs_handle *h, const float *gains) {
  if (!h || !gains) return set_err(nullptr, FS_ERR_ARG, "fs_set_gains: null argument");
  if (h->mode == FS_MODE_COMPAT) return set_err(h, FS_ERR_UNSUPPORTED, "fs_set_gains: production modes only");
  fsp::prod_set_gains(h->prod, gains);
  return FS_OK;
}

int fs_batch_set_gains(fs_batch *b, uint32_t inst, const float *gains) {
  if (!b || !gains) return set_err(nullptr, FS_ERR_ARG, "fs_batch_set_gains: null argument");
  int rc = fsp::batch_set_gains(b->b, inst, gains, b->err);
  return rc ? batch_err(b, rc, b->err) : FS_OK;
}

int fs_batch_set_drive(fs_batch *b, uint32_t inst, const float *pb) {
  if (!b || !pb) return set_err(nullptr, FS_ERR_ARG, "fs_batch_set_drive: null argument");
  cudaSetDevice(b->device);
  int rc = fsp::batch_set_drive(b->b, inst, pb, b->st, b->err);
  return rc ? batch_err(b, rc, b->err) : FS_OK;
}

int fs_spike_counts(fs_handle *h, uint32_t *counts) {
  if (!h || !counts) return set_err(nullptr, FS_ERR_ARG, "fs_spike_counts: null argument");
  if (h->mode == FS_MODE_COMPAT) return set_err(h, FS_ERR_UNSUPPORTED, "fs_spike_counts: production modes only");
  cudaSetDevice(h->device);
  int rc = fsp::prod_spike_counts(h->prod, counts, h->st, h->err);
  return rc ? set_err(h, rc, h->err) : FS_OK;
}

}  // extern "C"
