// C-ABI of the B200 FDTD engine: device buffers, launches, CUDA-graph replay
// of the step loop, read-back and checkpointing.
//
// The reference's run() (src/simulation/simulation_hd.cu:106-257) builds ~47
// launches per step from per-object agencies and runs them on the default
// stream.  Here one step is 2-5 launches on the handle's own stream, captured
// into a CUDA graph of `graph_steps` steps and replayed; the step index lives
// in device memory (bumped once per captured chunk) so a captured chunk is
// valid for any starting step.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <new>
#include <string>
#include <vector>

#include "kernels.cuh"
#include "xfb_internal.h"

using namespace xfb;

namespace {
thread_local std::string g_err;
}

struct Buf {
  void* p = nullptr;
  size_t bytes = 0;
  bool state = false;  // part of the checkpoint state
};

struct xfb_handle {
  Compiled c;
  std::string err;
  int device = -1;
  cudaStream_t stream = nullptr;
  bool inited = false;
  long long step = 0;
  unsigned hint_grid[3] = {1, 1, 1}, hint_block[3] = {1, 1, 1};
  int tk = 32, tj = 8;
  int graph_on = 1, graph_steps = 64;
  std::map<int, cudaGraphExec_t> graphs;
  std::vector<Buf> bufs;
  size_t bytes = 0;
  int esize = 4;
  // field layout
  long long sx = 0, sy = 0, nzp = 0, elems = 0, guard = 0;
  void* f[6] = {};
  uint8_t* mid = nullptr;
  void* lut = nullptr;
  // CPML
  void* prof[12] = {};  // ae0 ae1 ae2 be0 be1 be2 ah0 ah1 ah2 bh0 bh1 bh2
  void* psi[12] = {};   // ey_x ez_x ez_y ex_y ex_z ey_z hy_x hz_x hz_y hx_y hx_z hy_z
  long long ysx = 0, zsx = 0, zsy = 0;
  // TFSF
  double* proj[6] = {};
  double* e_aux = nullptr;
  double* h_aux = nullptr;
  double* src = nullptr;
  // ADE
  void* ade_mat = nullptr;
  void* ade_pole = nullptr;
  void* J = nullptr;
  void* Jp = nullptr;
  void* Ep = nullptr;
  long long bsx = 0, bsy = 0, bn = 0;
  // NF2FF
  double2* nf_acc = nullptr;
  double2* te = nullptr;
  double2* th = nullptr;
  int nf_off[7] = {};
  long long nf_npts = 0;
  // monitors
  long long* probe_idx = nullptr;
  int* probe_field = nullptr;
  double* probe_out = nullptr;
  std::vector<double*> movie_out;
  std::vector<long long> movie_frames;
  long long* t_dev = nullptr;
  unsigned long long* scratch_u64 = nullptr;
};

namespace {

int set_err(xfb_handle* h, int code, const std::string& m) {
  if (h) h->err = m;
  g_err = m;
  return code;
}

int cuda_err(xfb_handle* h, cudaError_t e, const char* what) {
  return set_err(h, XFB_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

#define XFB_CUDA(h, call)                                   \
  do {                                                      \
    cudaError_t e_ = (call);                                \
    if (e_ != cudaSuccess) return cuda_err((h), e_, #call); \
  } while (0)

template <typename T>
T* as(void* p) { return static_cast<T*>(p); }

void free_device(xfb_handle* h) {
  for (auto& kv : h->graphs) cudaGraphExecDestroy(kv.second);
  h->graphs.clear();
  for (auto& b : h->bufs) cudaFree(b.p);
  h->bufs.clear();
  h->bytes = 0;
  h->movie_out.clear();
  h->movie_frames.clear();
  h->inited = false;
}

int alloc(xfb_handle* h, void** out, size_t bytes, bool state) {
  *out = nullptr;
  if (bytes == 0) return XFB_OK;
  void* p = nullptr;
  cudaError_t e = cudaMalloc(&p, bytes);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return set_err(h, XFB_ERR_OOM, "cudaMalloc of " + std::to_string(bytes) + " bytes failed: " + cudaGetErrorString(e));
  }
  e = cudaMemsetAsync(p, 0, bytes, h->stream);
  if (e != cudaSuccess) { cudaFree(p); return cuda_err(h, e, "cudaMemsetAsync"); }
  h->bufs.push_back({p, bytes, state});
  h->bytes += bytes;
  *out = p;
  return XFB_OK;
}

template <typename T>
int upload(xfb_handle* h, void** out, const std::vector<double>& v, bool state = false) {
  std::vector<T> tmp(v.begin(), v.end());
  int rc = alloc(h, out, tmp.size() * sizeof(T), state);
  if (rc) return rc;
  if (!tmp.empty()) XFB_CUDA(h, cudaMemcpy(*out, tmp.data(), tmp.size() * sizeof(T), cudaMemcpyHostToDevice));
  return XFB_OK;
}

long long roundup(long long v, long long m) { return (v + m - 1) / m * m; }

// element offset of component index (i, j, k) in the padded layout
long long off3(const xfb_handle* h, int i, int j, int k) { return i * h->sx + j * h->sy + k; }

void comp_shape(const Compiled& c, int f, int s[3]) {
  s[0] = c.nx + (f == XFB_EY || f == XFB_EZ || f == XFB_HX ? 1 : 0);
  s[1] = c.ny + (f == XFB_EX || f == XFB_EZ || f == XFB_HY ? 1 : 0);
  s[2] = c.nz + (f == XFB_EX || f == XFB_EY || f == XFB_HZ ? 1 : 0);
  if (c.dim == 2) s[2] = 1;
}

int nf_face_points(const Compiled& c, int face) {
  const FaceGeom g = face_geom(c, face);
  return g.ni * g.nj * g.nk;
}

// ---------------------------------------------------------------------------
template <typename T>
int init_device(xfb_handle* h) {
  Compiled& c = h->c;
  const int nx = c.nx, ny = c.ny, nz = c.nz;
  if (c.dim == 3) {
    h->nzp = roundup(nz + 1, 32);
    h->sy = h->nzp;
    h->sx = (ny + 1) * h->nzp;
  } else {
    h->nzp = 1;
    h->sy = 1;
    h->sx = roundup(ny + 1, 32);
  }
  h->elems = (nx + 1) * h->sx;
  h->guard = roundup(h->sx + h->sy + 64, 64);
  const size_t fbytes = (h->elems + 2 * h->guard) * sizeof(T);
  int rc;
  for (int q = 0; q < 6; ++q) {
    if (c.dim == 2 && !(q == XFB_EZ || q == XFB_HX || q == XFB_HY)) continue;
    void* p;
    if ((rc = alloc(h, &p, fbytes, true))) return rc;
    h->f[q] = as<T>(p) + h->guard;
  }
  // material ids in the padded layout
  {
    std::vector<uint8_t> m(static_cast<size_t>(h->elems), 0);
    for (int i = 0; i < nx; ++i)
      for (int j = 0; j < ny; ++j)
        for (int k = 0; k < nz; ++k) m[off3(h, i, j, k)] = c.mat_id[(static_cast<size_t>(i) * ny + j) * nz + k];
    void* p;
    if ((rc = alloc(h, &p, m.size(), false))) return rc;
    XFB_CUDA(h, cudaMemcpy(p, m.data(), m.size(), cudaMemcpyHostToDevice));
    h->mid = static_cast<uint8_t*>(p);
  }
  if ((rc = upload<T>(h, &h->lut, c.coeff))) return rc;
  // CPML
  const int L[6] = {c.pml[0], c.pml[1], c.pml[2], c.pml[3], c.pml[4], c.pml[5]};
  for (int a = 0; a < 3; ++a) {
    if ((rc = upload<T>(h, &h->prof[a], c.pml_ae[a]))) return rc;
    if ((rc = upload<T>(h, &h->prof[3 + a], c.pml_be[a]))) return rc;
    if ((rc = upload<T>(h, &h->prof[6 + a], c.pml_ah[a]))) return rc;
    if ((rc = upload<T>(h, &h->prof[9 + a], c.pml_bh[a]))) return rc;
  }
  const long long Lx = L[0] + L[1], Ly = L[2] + L[3], Lz = L[4] + L[5];
  if (c.dim == 3) {
    h->ysx = Ly * h->nzp;
    h->zsy = Lz;
    h->zsx = (ny + 1) * Lz;
    const size_t bx = Lx * h->sx * sizeof(T), by = (nx + 1) * h->ysx * sizeof(T), bz = (nx + 1) * h->zsx * sizeof(T);
    const size_t sz[12] = {bx, bx, by, by, bz, bz, bx, bx, by, by, bz, bz};
    for (int q = 0; q < 12; ++q)
      if ((rc = alloc(h, &h->psi[q], sz[q], true))) return rc;
  } else {
    h->ysx = Ly;
    const size_t bx = Lx * h->sx * sizeof(T), by = (nx + 1) * Ly * sizeof(T);
    if ((rc = alloc(h, &h->psi[1], bx, true))) return rc;   // ez_x
    if ((rc = alloc(h, &h->psi[2], by, true))) return rc;   // ez_y
    if ((rc = alloc(h, &h->psi[6], bx, true))) return rc;   // hy_x
    if ((rc = alloc(h, &h->psi[9], by, true))) return rc;   // hx_y
  }
  // TFSF
  if (c.tfsf_on) {
    for (int a = 0; a < 3; ++a) {
      void* p;
      if ((rc = upload<double>(h, &p, c.proj_int[a]))) return rc;
      h->proj[a] = static_cast<double*>(p);
      if ((rc = upload<double>(h, &p, c.proj_half[a]))) return rc;
      h->proj[3 + a] = static_cast<double*>(p);
    }
    void* p;
    if ((rc = alloc(h, &p, (c.aux_nl + 1) * sizeof(double), true))) return rc;
    h->e_aux = static_cast<double*>(p);
    if ((rc = alloc(h, &p, c.aux_nl * sizeof(double), true))) return rc;
    h->h_aux = static_cast<double*>(p);
    if ((rc = upload<double>(h, &p, c.aux_source))) return rc;
    h->src = static_cast<double*>(p);
  }
  // ADE
  if (c.ade_kind != XFB_ADE_NONE) {
    if ((rc = upload<T>(h, &h->ade_mat, c.ade_mat))) return rc;
    if ((rc = upload<T>(h, &h->ade_pole, c.ade_pole))) return rc;
    const int* b = c.ade_box;
    const long long bk = roundup(std::max(1, b[5] - b[4]), 32);
    h->bsy = bk;
    h->bsx = std::max(1, b[3] - b[2]) * bk;
    h->bn = std::max(1, b[1] - b[0]) * h->bsx;
    const int P = std::max(1, c.ade_poles);
    if ((rc = alloc(h, &h->J, 3 * P * h->bn * sizeof(T), true))) return rc;
    if (c.ade_kind == XFB_ADE_MLORENTZ) {
      if ((rc = alloc(h, &h->Jp, 3 * P * h->bn * sizeof(T), true))) return rc;
      if ((rc = alloc(h, &h->Ep, 3 * h->bn * sizeof(T), true))) return rc;
    }
  }
  // NF2FF
  if (c.nf_on) {
    h->nf_off[0] = 0;
    for (int f = 0; f < 6; ++f) h->nf_off[f + 1] = h->nf_off[f] + nf_face_points(c, f);
    h->nf_npts = h->nf_off[6];
    const size_t nfq = c.freqs.size();
    void* p;
    if ((rc = alloc(h, &p, nfq * 4 * h->nf_npts * sizeof(double2), true))) return rc;
    h->nf_acc = static_cast<double2*>(p);
    if ((rc = upload<double>(h, &p, c.te))) return rc;
    h->te = static_cast<double2*>(p);
    if ((rc = upload<double>(h, &p, c.th))) return rc;
    h->th = static_cast<double2*>(p);
  }
  // probes
  if (!c.probes.empty()) {
    const size_t n = c.probes.size();
    std::vector<long long> idx(n);
    std::vector<int> fld(n);
    for (size_t p = 0; p < n; ++p) {
      idx[p] = off3(h, c.probes[p].index[0], c.probes[p].index[1], c.dim == 3 ? c.probes[p].index[2] : 0);
      fld[p] = c.probes[p].field;
    }
    void* p;
    if ((rc = alloc(h, &p, n * sizeof(long long), false))) return rc;
    h->probe_idx = static_cast<long long*>(p);
    XFB_CUDA(h, cudaMemcpy(p, idx.data(), n * sizeof(long long), cudaMemcpyHostToDevice));
    if ((rc = alloc(h, &p, n * sizeof(int), false))) return rc;
    h->probe_field = static_cast<int*>(p);
    XFB_CUDA(h, cudaMemcpy(p, fld.data(), n * sizeof(int), cudaMemcpyHostToDevice));
    if ((rc = alloc(h, &p, n * std::max(1LL, c.total_steps) * sizeof(double), true))) return rc;
    h->probe_out = static_cast<double*>(p);
  }
  // movies
  for (const xfb_movie& mv : c.movies) {
    const long long frames = (c.total_steps + mv.interval - 1) / mv.interval;
    const long long per = static_cast<long long>(mv.hi[0] - mv.lo[0]) * (mv.hi[1] - mv.lo[1]) * (mv.hi[2] - mv.lo[2]);
    void* p;
    if ((rc = alloc(h, &p, std::max(1LL, frames) * per * sizeof(double), true))) return rc;
    h->movie_out.push_back(static_cast<double*>(p));
    h->movie_frames.push_back(frames);
  }
  void* p;
  if ((rc = alloc(h, &p, sizeof(long long), true))) return rc;
  h->t_dev = static_cast<long long*>(p);
  if ((rc = alloc(h, &p, sizeof(unsigned long long), false))) return rc;
  h->scratch_u64 = static_cast<unsigned long long*>(p);
  XFB_CUDA(h, cudaStreamSynchronize(h->stream));
  return XFB_OK;
}

// ---------------------------------------------------------------------------
template <typename T>
GridP<T> grid_params(xfb_handle* h) {
  GridP<T> g;
  g.nx = h->c.nx; g.ny = h->c.ny; g.nz = h->c.nz;
  g.sx = h->sx; g.sy = h->sy;
  g.ex = as<T>(h->f[0]); g.ey = as<T>(h->f[1]); g.ez = as<T>(h->f[2]);
  g.hx = as<T>(h->f[3]); g.hy = as<T>(h->f[4]); g.hz = as<T>(h->f[5]);
  g.mid = h->mid;
  g.lut = as<const T>(h->lut);
  return g;
}

template <typename T>
PmlP<T> pml_params(xfb_handle* h) {
  PmlP<T> p;
  for (int q = 0; q < 6; ++q) p.L[q] = h->c.pml[q];
  for (int a = 0; a < 3; ++a) {
    p.ae[a] = as<const T>(h->prof[a]); p.be[a] = as<const T>(h->prof[3 + a]);
    p.ah[a] = as<const T>(h->prof[6 + a]); p.bh[a] = as<const T>(h->prof[9 + a]);
  }
  T** ps[12] = {&p.ey_x, &p.ez_x, &p.ez_y, &p.ex_y, &p.ex_z, &p.ey_z, &p.hy_x, &p.hz_x, &p.hz_y, &p.hx_y, &p.hx_z, &p.hy_z};
  for (int q = 0; q < 12; ++q) *ps[q] = as<T>(h->psi[q]);
  p.ysx = h->ysx; p.zsx = h->zsx; p.zsy = h->zsy;
  return p;
}

TfsfP tfsf_params(xfb_handle* h) {
  TfsfP t{};
  const Compiled& c = h->c;
  t.on = c.tfsf_on;
  if (!t.on) return t;
  t.is = c.tf[0]; t.ie = c.tf[1]; t.js = c.tf[2]; t.je = c.tf[3]; t.ks = c.tf[4]; t.ke = c.tf[5];
  t.pi0 = h->proj[0]; t.pi1 = h->proj[1]; t.pi2 = h->proj[2];
  t.ph0 = h->proj[3]; t.ph1 = h->proj[4]; t.ph2 = h->proj[5];
  for (int a = 0; a < 3; ++a) { t.tre[a] = c.tr_e[a]; t.trh[a] = c.tr_h[a]; t.ca[a] = c.ca[a]; t.cb[a] = c.cb[a]; }
  t.e_aux = h->e_aux; t.h_aux = h->h_aux;
  return t;
}

template <typename T>
AdeP<T> ade_params(xfb_handle* h) {
  AdeP<T> a{};
  const Compiled& c = h->c;
  a.kind = c.ade_kind;
  if (a.kind == XFB_ADE_NONE) return a;
  a.P = c.ade_poles;
  a.b0 = c.ade_box[0]; a.b1 = c.ade_box[1]; a.b2 = c.ade_box[2]; a.b3 = c.ade_box[3]; a.b4 = c.ade_box[4]; a.b5 = c.ade_box[5];
  a.bsx = h->bsx; a.bsy = h->bsy; a.bn = h->bn;
  a.mat = as<const T>(h->ade_mat); a.pole = as<const T>(h->ade_pole);
  a.J = as<T>(h->J); a.Jp = as<T>(h->Jp); a.Ep = as<T>(h->Ep);
  return a;
}

int chunks_for(int tiles, int n_march, int threads) {
  const int resident = 148 * std::max(1, 2048 / threads);
  int ch = (4 * resident + tiles - 1) / std::max(1, tiles);
  ch = std::min(ch, std::max(1, n_march / 8));
  return std::max(1, ch);
}

// Optional per-launch CUDA-event bracketing (profile mode only).
struct Prof {
  cudaEvent_t ev[2 * 16];
  int cls[16];
  int n = 0;
};

inline void prof_begin(xfb_handle* h, Prof* p, int cls) {
  if (!p) return;
  p->cls[p->n] = cls;
  cudaEventRecord(p->ev[2 * p->n], h->stream);
}
inline void prof_end(xfb_handle* h, Prof* p) {
  if (!p) return;
  cudaEventRecord(p->ev[2 * p->n + 1], h->stream);
  ++p->n;
}

// Largest j-row count of a (32 x tj) tile that every bulk kernel of type T
// can launch with (register budget of the compiled kernels).
template <typename T>
int tile_rows(xfb_handle* h) {
  int lim = 1024;
  cudaFuncAttributes a;
  if (h->c.dim == 3) {
    if (cudaFuncGetAttributes(&a, k_h3<T>) == cudaSuccess) lim = std::min(lim, a.maxThreadsPerBlock);
    if (cudaFuncGetAttributes(&a, k_e3<T>) == cudaSuccess) lim = std::min(lim, a.maxThreadsPerBlock);
  }
  int tj = std::max(1, std::min(h->tj, lim / h->tk));
  int p = 1;
  while (p * 2 <= tj) p *= 2;
  return p;
}

template <typename T>
void enqueue_step(xfb_handle* h, int off, Prof* pf = nullptr) {
  const Compiled& c = h->c;
  TimeP tp{h->t_dev, off};
  GridP<T> g = grid_params<T>(h);
  PmlP<T> pm = pml_params<T>(h);
  TfsfP tf = tfsf_params(h);
  cudaStream_t s = h->stream;
  if (c.dim == 3) {
    const int tj = tile_rows<T>(h);
    dim3 blk(h->tk, tj);
    const int gx = (c.nz + h->tk - 1) / h->tk, gy = (c.ny + tj - 1) / tj;
    const int nch = chunks_for(gx * gy, c.nx, h->tk * tj);
    const int ich = (c.nx + nch - 1) / nch;
    dim3 grd(gx, gy, (c.nx + ich - 1) / ich);
    prof_begin(h, pf, XFB_K_UPDATE_H);
    k_h3<T><<<grd, blk, 0, s>>>(g, pm, tf, tp, ich);
    prof_end(h, pf);
    if (c.tfsf_on) {
      prof_begin(h, pf, XFB_K_AUX);
      k_aux<<<1, 1024, 0, s>>>(h->e_aux, h->h_aux, c.aux_nl, c.aux_ceih, c.aux_chie, c.aux_abc, h->src, tp);
      prof_end(h, pf);
    }
    prof_begin(h, pf, XFB_K_UPDATE_E);
    k_e3<T><<<grd, blk, 0, s>>>(g, pm, tf, ade_params<T>(h), tp, ich);
    prof_end(h, pf);
  } else {
    const int bx = 128;
    const int gx = (c.ny + bx - 1) / bx;
    const int nch = chunks_for(gx, c.nx, bx);
    const int ich = (c.nx + nch - 1) / nch;
    dim3 grd(gx, (c.nx + ich - 1) / ich);
    prof_begin(h, pf, XFB_K_UPDATE_H);
    k_h2<T><<<grd, bx, 0, s>>>(g, pm, tf, tp, ich);
    prof_end(h, pf);
    if (c.tfsf_on) {
      prof_begin(h, pf, XFB_K_AUX);
      k_aux<<<1, 1024, 0, s>>>(h->e_aux, h->h_aux, c.aux_nl, c.aux_ceih, c.aux_chie, c.aux_abc, h->src, tp);
      prof_end(h, pf);
    }
    prof_begin(h, pf, XFB_K_UPDATE_E);
    k_e2<T><<<grd, bx, 0, s>>>(g, pm, tf, tp, ich);
    prof_end(h, pf);
  }
  if (c.nf_on) {
    NfP nf{};
    nf.nfreq = static_cast<int>(c.freqs.size());
    for (int q = 0; q < 6; ++q) nf.box[q] = c.nf[q];
    for (int q = 0; q < 7; ++q) nf.off[q] = h->nf_off[q];
    nf.npts = h->nf_npts;
    nf.acc = h->nf_acc; nf.te = h->te; nf.th = h->th;
    nf.total_steps = c.total_steps;
    prof_begin(h, pf, XFB_K_NF2FF);
    k_nf2ff<T><<<static_cast<unsigned>((h->nf_npts + 255) / 256), 256, 0, s>>>(g, nf, tp);
    prof_end(h, pf);
  }
  if (!c.probes.empty()) {
    ProbeP pr{static_cast<int>(c.probes.size()), h->probe_idx, h->probe_field, h->probe_out, c.total_steps};
    prof_begin(h, pf, XFB_K_PROBE);
    k_probe<T><<<(pr.n + 127) / 128, 128, 0, s>>>(g, pr, tp);
    prof_end(h, pf);
  }
  for (size_t m = 0; m < c.movies.size(); ++m) {
    const xfb_movie& mv = c.movies[m];
    const int n0 = mv.hi[0] - mv.lo[0], n1 = mv.hi[1] - mv.lo[1], n2 = mv.hi[2] - mv.lo[2];
    const long long per = static_cast<long long>(n0) * n1 * n2;
    const int blocks = static_cast<int>(std::min<long long>((per + 255) / 256, 1024));
    prof_begin(h, pf, XFB_K_MOVIE);
    k_movie<T><<<blocks, 256, 0, s>>>(as<const T>(h->f[mv.field]), h->sx, h->sy, mv.lo[0], mv.lo[1], mv.lo[2], n0, n1, n2,
                                      mv.interval, h->movie_out[m], h->movie_frames[m], tp);
    prof_end(h, pf);
  }
}

template <typename T>
void enqueue_chunk(xfb_handle* h, int n) {
  for (int s = 0; s < n; ++s) enqueue_step<T>(h, s);
  k_bump<<<1, 1, 0, h->stream>>>(h->t_dev, n);
}

template <typename T>
int run_steps(xfb_handle* h, long long n) {
  long long left = n;
  while (left > 0) {
    const int chunk = static_cast<int>(std::min<long long>(left, h->graph_steps));
    if (h->graph_on) {
      auto it = h->graphs.find(chunk);
      if (it == h->graphs.end()) {
        cudaGraph_t graph;
        XFB_CUDA(h, cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
        enqueue_chunk<T>(h, chunk);
        XFB_CUDA(h, cudaStreamEndCapture(h->stream, &graph));
        cudaGraphExec_t ex;
        cudaError_t e = cudaGraphInstantiate(&ex, graph, 0);
        cudaGraphDestroy(graph);
        if (e != cudaSuccess) return cuda_err(h, e, "cudaGraphInstantiate");
        it = h->graphs.emplace(chunk, ex).first;
      }
      XFB_CUDA(h, cudaGraphLaunch(it->second, h->stream));
    } else {
      enqueue_chunk<T>(h, chunk);
      XFB_CUDA(h, cudaGetLastError());
    }
    left -= chunk;
    h->step += chunk;
  }
  return XFB_OK;
}

template <typename T>
int profile_steps(xfb_handle* h, long long n, double* ms, long long* launches) {
  for (int q = 0; q < XFB_K_COUNT; ++q) { ms[q] = 0; launches[q] = 0; }
  Prof pf;
  for (int e = 0; e < 32; ++e) XFB_CUDA(h, cudaEventCreate(&pf.ev[e]));
  int rc = XFB_OK;
  for (long long q = 0; q < n && rc == XFB_OK; ++q) {
    pf.n = 0;
    enqueue_step<T>(h, 0, &pf);
    k_bump<<<1, 1, 0, h->stream>>>(h->t_dev, 1);
    cudaError_t e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) { rc = cuda_err(h, e, "profile step"); break; }
    for (int k = 0; k < pf.n; ++k) {
      float t = 0;
      cudaEventElapsedTime(&t, pf.ev[2 * k], pf.ev[2 * k + 1]);
      ms[pf.cls[k]] += t;
      launches[pf.cls[k]] += 1;
    }
    h->step += 1;
  }
  for (int e = 0; e < 32; ++e) cudaEventDestroy(pf.ev[e]);
  return rc;
}

int launches_per_step(const Compiled& c) {
  return 2 + (c.tfsf_on ? 1 : 0) + (c.nf_on ? 1 : 0) + (c.probes.empty() ? 0 : 1) + static_cast<int>(c.movies.size());
}

int check_handle(xfb_handle* h, bool need_init) {
  if (!h) return set_err(nullptr, XFB_ERR_INVALID, "null handle");
  if (need_init && !h->inited) return set_err(h, XFB_ERR_STATE, "handle not initialised (call xfb_init or xfb_run)");
  if (h->inited) {
    cudaError_t e = cudaSetDevice(h->device);
    if (e != cudaSuccess) return cuda_err(h, e, "cudaSetDevice");
  }
  return XFB_OK;
}

template <typename T>
int read_field_t(xfb_handle* h, int f, double* dst) {
  std::vector<T> tmp(static_cast<size_t>(h->elems));
  XFB_CUDA(h, cudaStreamSynchronize(h->stream));
  XFB_CUDA(h, cudaMemcpy(tmp.data(), h->f[f], tmp.size() * sizeof(T), cudaMemcpyDeviceToHost));
  int s[3];
  comp_shape(h->c, f, s);
  size_t o = 0;
  for (int i = 0; i < s[0]; ++i)
    for (int j = 0; j < s[1]; ++j)
      for (int k = 0; k < s[2]; ++k) dst[o++] = static_cast<double>(tmp[off3(h, i, j, k)]);
  return XFB_OK;
}

template <typename T>
int write_field_t(xfb_handle* h, int f, const double* src) {
  std::vector<T> tmp(static_cast<size_t>(h->elems));
  XFB_CUDA(h, cudaStreamSynchronize(h->stream));
  XFB_CUDA(h, cudaMemcpy(tmp.data(), h->f[f], tmp.size() * sizeof(T), cudaMemcpyDeviceToHost));
  int s[3];
  comp_shape(h->c, f, s);
  size_t o = 0;
  for (int i = 0; i < s[0]; ++i)
    for (int j = 0; j < s[1]; ++j)
      for (int k = 0; k < s[2]; ++k) tmp[off3(h, i, j, k)] = static_cast<T>(src[o++]);
  XFB_CUDA(h, cudaMemcpy(h->f[f], tmp.data(), tmp.size() * sizeof(T), cudaMemcpyHostToDevice));
  return XFB_OK;
}

}  // namespace

// ===========================================================================
extern "C" {

int xfb_abi_version(void) { return XFB_ABI_VERSION; }

const char* xfb_status_string(int s) {
  switch (s) {
    case XFB_OK: return "ok";
    case XFB_ERR_INVALID: return "invalid argument";
    case XFB_ERR_CUDA: return "CUDA error";
    case XFB_ERR_OOM: return "out of memory";
    case XFB_ERR_STATE: return "invalid state";
    case XFB_ERR_RANGE: return "out of range";
    case XFB_ERR_NUMERIC: return "non-finite values";
    case XFB_ERR_TIMEOUT: return "device wait timed out";
    case XFB_ERR_NO_DEVICE: return "no CUDA device";
  }
  return "unknown status";
}

const char* xfb_last_error(const xfb_handle* h) { return h ? h->err.c_str() : g_err.c_str(); }

int xfb_create(const xfb_scene* scene, xfb_handle** out) {
  if (!scene || !out) return set_err(nullptr, XFB_ERR_INVALID, "null scene or output pointer");
  *out = nullptr;
  std::unique_ptr<xfb_handle> h(new (std::nothrow) xfb_handle());
  if (!h) return set_err(nullptr, XFB_ERR_OOM, "host allocation failed");
  std::string err;
  int rc;
  try {
    rc = compile_scene(*scene, h->c, &err);
  } catch (const std::bad_alloc&) {
    return set_err(nullptr, XFB_ERR_OOM, "host allocation failed while compiling the scene");
  }
  if (rc) return set_err(nullptr, rc, err);
  h->esize = h->c.prec == XFB_FP64 ? 8 : 4;
  *out = h.release();
  g_err.clear();
  return XFB_OK;
}

int xfb_destroy(xfb_handle* h) {
  if (!h) return XFB_OK;
  if (h->device >= 0) {
    cudaSetDevice(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    free_device(h);
    if (h->stream) cudaStreamDestroy(h->stream);
  }
  delete h;
  return XFB_OK;
}

int xfb_set_launch_hint(xfb_handle* h, const unsigned grid[3], const unsigned block[3]) {
  if (!h || !grid || !block) return set_err(h, XFB_ERR_INVALID, "null argument");
  for (int a = 0; a < 3; ++a) {
    h->hint_grid[a] = grid[a] ? grid[a] : 1;
    h->hint_block[a] = block[a] ? block[a] : 1;
  }
  const unsigned threads = h->hint_block[0] * h->hint_block[1] * h->hint_block[2];
  if (threads % 32 == 0 && threads <= 1024 && threads >= 32) {
    h->tk = 32;
    h->tj = static_cast<int>(threads / 32);
  }
  for (auto& kv : h->graphs) cudaGraphExecDestroy(kv.second);
  h->graphs.clear();
  return XFB_OK;
}

int xfb_set_device(xfb_handle* h, int ordinal) {
  if (!h) return set_err(nullptr, XFB_ERR_INVALID, "null handle");
  if (h->device >= 0) return set_err(h, XFB_ERR_STATE, "device already chosen (set it before the first xfb_init)");
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
    cudaGetLastError();
    return set_err(h, XFB_ERR_NO_DEVICE, "no CUDA device available");
  }
  if (ordinal < 0 || ordinal >= n) return set_err(h, XFB_ERR_RANGE, "device ordinal out of range");
  XFB_CUDA(h, cudaSetDevice(ordinal));
  h->device = ordinal;
  XFB_CUDA(h, cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
  return XFB_OK;
}

int xfb_set_graph(xfb_handle* h, int enabled, int steps_per_graph) {
  if (!h) return set_err(nullptr, XFB_ERR_INVALID, "null handle");
  if (steps_per_graph < 1 || steps_per_graph > 4096) return set_err(h, XFB_ERR_INVALID, "steps_per_graph must be in [1, 4096]");
  h->graph_on = enabled ? 1 : 0;
  h->graph_steps = steps_per_graph;
  return XFB_OK;
}

int xfb_prepare_tables(xfb_handle* h, long long total_steps) {
  if (!h) return set_err(nullptr, XFB_ERR_INVALID, "null handle");
  if (total_steps < 0 || total_steps > (1LL << 31)) return set_err(h, XFB_ERR_INVALID, "total_steps out of range");
  size_tables(h->c, total_steps);
  return XFB_OK;
}

int xfb_init(xfb_handle* h, long long total_steps) {
  if (!h) return set_err(nullptr, XFB_ERR_INVALID, "null handle");
  if (total_steps < 0 || total_steps > (1LL << 31)) return set_err(h, XFB_ERR_INVALID, "total_steps out of range");
  if (h->device < 0) {
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0) {
      cudaGetLastError();
      return set_err(h, XFB_ERR_NO_DEVICE, "no CUDA device available");
    }
    XFB_CUDA(h, cudaGetDevice(&h->device));
    XFB_CUDA(h, cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
  }
  XFB_CUDA(h, cudaSetDevice(h->device));
  XFB_CUDA(h, cudaStreamSynchronize(h->stream));
  free_device(h);
  size_tables(h->c, total_steps);
  int rc;
  try {
    rc = h->c.prec == XFB_FP64 ? init_device<double>(h) : init_device<float>(h);
  } catch (const std::bad_alloc&) {
    rc = set_err(h, XFB_ERR_OOM, "host allocation failed during init");
  }
  if (rc) {
    free_device(h);
    return rc;
  }
  h->step = 0;
  h->inited = true;
  return XFB_OK;
}

int xfb_step(xfb_handle* h, long long n) {
  int rc = check_handle(h, true);
  if (rc) return rc;
  if (n < 0) return set_err(h, XFB_ERR_INVALID, "negative step count");
  if (h->step + n > h->c.total_steps)
    return set_err(h, XFB_ERR_RANGE, "steps beyond the count xfb_init sized the run for");
  return h->c.prec == XFB_FP64 ? run_steps<double>(h, n) : run_steps<float>(h, n);
}

int xfb_sync(xfb_handle* h) {
  int rc = check_handle(h, true);
  if (rc) return rc;
  XFB_CUDA(h, cudaStreamSynchronize(h->stream));
  XFB_CUDA(h, cudaGetLastError());
  return XFB_OK;
}

int xfb_timed_step(xfb_handle* h, long long n, double* ms) {
  int rc = check_handle(h, true);
  if (rc) return rc;
  if (!ms) return set_err(h, XFB_ERR_INVALID, "null output");
  cudaEvent_t a, b;
  XFB_CUDA(h, cudaEventCreate(&a));
  XFB_CUDA(h, cudaEventCreate(&b));
  XFB_CUDA(h, cudaStreamSynchronize(h->stream));
  cudaEventRecord(a, h->stream);
  rc = xfb_step(h, n);
  cudaEventRecord(b, h->stream);
  cudaError_t e = cudaEventSynchronize(b);
  float t = 0;
  if (e == cudaSuccess) e = cudaEventElapsedTime(&t, a, b);
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  if (rc) return rc;
  if (e != cudaSuccess) return cuda_err(h, e, "timed step");
  *ms = t;
  return XFB_OK;
}

int xfb_profile_kernels(xfb_handle* h, long long n, double* ms, long long* launches) {
  int rc = check_handle(h, true);
  if (rc) return rc;
  if (!ms || !launches || n < 0) return set_err(h, XFB_ERR_INVALID, "bad arguments");
  if (h->step + n > h->c.total_steps) return set_err(h, XFB_ERR_RANGE, "steps beyond the count xfb_init sized the run for");
  XFB_CUDA(h, cudaStreamSynchronize(h->stream));
  return h->c.prec == XFB_FP64 ? profile_steps<double>(h, n, ms, launches) : profile_steps<float>(h, n, ms, launches);
}

int xfb_run(xfb_handle* h, long long n) {
  int rc = xfb_init(h, n);
  if (rc) return rc;
  if ((rc = xfb_step(h, n))) return rc;
  return xfb_sync(h);
}

int xfb_get_grid_info(const xfb_handle* h, xfb_grid_info* o) {
  if (!h || !o) return set_err(nullptr, XFB_ERR_INVALID, "null argument");
  const Compiled& c = h->c;
  std::memset(o, 0, sizeof(*o));
  o->dim = c.dim; o->precision = c.prec;
  o->nx = c.nx; o->ny = c.ny; o->nz = c.nz;
  o->dx = c.dx; o->dy = c.dy; o->dz = c.dz; o->dt = c.dt;
  for (int a = 0; a < 3; ++a) o->origin[a] = c.origin[a];
  o->n_materials = c.n_mat;
  o->ade_kind = c.ade_kind; o->ade_poles = c.ade_poles;
  if (c.tfsf_on) for (int q = 0; q < 6; ++q) o->tfsf_box[q] = c.tf[q];
  if (c.nf_on) for (int q = 0; q < 6; ++q) o->nf2ff_box[q] = c.nf[q];
  o->n_freqs = static_cast<int>(c.freqs.size());
  o->current_step = h->step;
  o->total_steps = c.total_steps;
  o->device_bytes = h->bytes;
  long long nd = 0;
  if (c.ade_kind != XFB_ADE_NONE)
    for (uint8_t m : c.mat_id) nd += c.ade_mat[static_cast<size_t>(m) * kAdeMat] != 0;
  o->n_dispersive_cells = nd;
  o->launches_per_step = launches_per_step(c);
  return XFB_OK;
}

int xfb_read_field(xfb_handle* h, int f, double* dst, size_t len) {
  int rc = check_handle(h, true);
  if (rc) return rc;
  if (f < 0 || f > 5 || !dst) return set_err(h, XFB_ERR_INVALID, "bad field or buffer");
  if (!h->f[f]) return set_err(h, XFB_ERR_INVALID, "component not present in a 2-D (TMz) scene");
  int s[3];
  comp_shape(h->c, f, s);
  if (len < static_cast<size_t>(s[0]) * s[1] * s[2]) return set_err(h, XFB_ERR_RANGE, "destination too small");
  return h->c.prec == XFB_FP64 ? read_field_t<double>(h, f, dst) : read_field_t<float>(h, f, dst);
}

int xfb_write_field(xfb_handle* h, int f, const double* src, size_t len) {
  int rc = check_handle(h, true);
  if (rc) return rc;
  if (f < 0 || f > 5 || !src) return set_err(h, XFB_ERR_INVALID, "bad field or buffer");
  if (!h->f[f]) return set_err(h, XFB_ERR_INVALID, "component not present in a 2-D (TMz) scene");
  int s[3];
  comp_shape(h->c, f, s);
  if (len < static_cast<size_t>(s[0]) * s[1] * s[2]) return set_err(h, XFB_ERR_RANGE, "source too small");
  return h->c.prec == XFB_FP64 ? write_field_t<double>(h, f, src) : write_field_t<float>(h, f, src);
}

int xfb_read_probe(xfb_handle* h, int id, double* dst, size_t len, long long* n_written) {
  int rc = check_handle(h, true);
  if (rc) return rc;
  if (id < 0 || id >= static_cast<int>(h->c.probes.size())) return set_err(h, XFB_ERR_RANGE, "probe id out of range");
  const long long n = h->step;
  if (len < static_cast<size_t>(n)) return set_err(h, XFB_ERR_RANGE, "destination too small");
  XFB_CUDA(h, cudaStreamSynchronize(h->stream));
  if (n > 0) XFB_CUDA(h, cudaMemcpy(dst, h->probe_out + id * h->c.total_steps, n * sizeof(double), cudaMemcpyDeviceToHost));
  if (n_written) *n_written = n;
  return XFB_OK;
}

int xfb_movie_shape(const xfb_handle* h, int id, int s[4]) {
  if (!h || !s) return set_err(nullptr, XFB_ERR_INVALID, "null argument");
  if (id < 0 || id >= static_cast<int>(h->c.movies.size())) return set_err(const_cast<xfb_handle*>(h), XFB_ERR_RANGE, "movie id out of range");
  const xfb_movie& mv = h->c.movies[id];
  s[0] = static_cast<int>((h->c.total_steps + mv.interval - 1) / mv.interval);
  for (int a = 0; a < 3; ++a) s[1 + a] = mv.hi[a] - mv.lo[a];
  return XFB_OK;
}

int xfb_read_movie(xfb_handle* h, int id, double* dst, size_t len) {
  int rc = check_handle(h, true);
  if (rc) return rc;
  int s[4];
  if ((rc = xfb_movie_shape(h, id, s))) return rc;
  const size_t n = static_cast<size_t>(s[0]) * s[1] * s[2] * s[3];
  if (len < n) return set_err(h, XFB_ERR_RANGE, "destination too small");
  XFB_CUDA(h, cudaStreamSynchronize(h->stream));
  if (n) XFB_CUDA(h, cudaMemcpy(dst, h->movie_out[id], n * sizeof(double), cudaMemcpyDeviceToHost));
  return XFB_OK;
}

int xfb_nf2ff_face_shape(const xfb_handle* h, int face, int s[3]) {
  if (!h || !s) return set_err(nullptr, XFB_ERR_INVALID, "null argument");
  if (!h->c.nf_on) return set_err(const_cast<xfb_handle*>(h), XFB_ERR_STATE, "scene has no NF2FF box");
  if (face < 0 || face > 5) return set_err(const_cast<xfb_handle*>(h), XFB_ERR_RANGE, "face out of range");
  const FaceGeom g = face_geom(h->c, face);
  s[0] = g.ni; s[1] = g.nj; s[2] = g.nk;
  return XFB_OK;
}

int xfb_read_nf2ff(xfb_handle* h, int freq, int face, int which, double* dst, size_t len) {
  int rc = check_handle(h, true);
  if (rc) return rc;
  int s[3];
  if ((rc = xfb_nf2ff_face_shape(h, face, s))) return rc;
  if (freq < 0 || freq >= static_cast<int>(h->c.freqs.size()) || which < 0 || which > 3)
    return set_err(h, XFB_ERR_RANGE, "frequency or current index out of range");
  const size_t n = static_cast<size_t>(s[0]) * s[1] * s[2];
  if (len < 2 * n) return set_err(h, XFB_ERR_RANGE, "destination too small (complex interleaved)");
  XFB_CUDA(h, cudaStreamSynchronize(h->stream));
  const double2* src = h->nf_acc + (static_cast<long long>(freq) * 4 + which) * h->nf_npts + h->nf_off[face];
  XFB_CUDA(h, cudaMemcpy(dst, src, n * sizeof(double2), cudaMemcpyDeviceToHost));
  return XFB_OK;
}

int xfb_far_field(xfb_handle* h, int freq, int n, const double* theta, const double* phi, double* out) {
  int rc = check_handle(h, true);
  if (rc) return rc;
  if (!h->c.nf_on) return set_err(h, XFB_ERR_STATE, "scene has no NF2FF box");
  if (freq < 0 || freq >= static_cast<int>(h->c.freqs.size())) return set_err(h, XFB_ERR_RANGE, "frequency index out of range");
  if (n < 0 || (n > 0 && (!theta || !phi || !out))) return set_err(h, XFB_ERR_INVALID, "bad angle arrays");
  if (n == 0) return XFB_OK;
  double *d_th = nullptr, *d_ph = nullptr, *d_out = nullptr;
  XFB_CUDA(h, cudaMalloc(&d_th, n * sizeof(double)));
  XFB_CUDA(h, cudaMalloc(&d_ph, n * sizeof(double)));
  XFB_CUDA(h, cudaMalloc(&d_out, 4 * n * sizeof(double)));
  cudaMemcpyAsync(d_th, theta, n * sizeof(double), cudaMemcpyHostToDevice, h->stream);
  cudaMemcpyAsync(d_ph, phi, n * sizeof(double), cudaMemcpyHostToDevice, h->stream);
  FarP fp{};
  const Compiled& c = h->c;
  for (int q = 0; q < 6; ++q) fp.box[q] = c.nf[q];
  for (int q = 0; q < 7; ++q) fp.off[q] = h->nf_off[q];
  fp.npts = h->nf_npts;
  fp.acc = h->nf_acc + static_cast<long long>(freq) * 4 * h->nf_npts;
  for (int a = 0; a < 3; ++a) fp.origin[a] = c.origin[a];
  fp.d[0] = c.dx; fp.d[1] = c.dy; fp.d[2] = c.dz;
  fp.k = 2 * kPi * c.freqs[freq] / c0();
  fp.eta = std::sqrt(kMu0 / kEps0);
  fp.theta = d_th; fp.phi = d_ph; fp.out = d_out;
  k_far<<<n, 256, 0, h->stream>>>(fp);
  cudaError_t e = cudaMemcpyAsync(out, d_out, 4 * n * sizeof(double), cudaMemcpyDeviceToHost, h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  cudaFree(d_th); cudaFree(d_ph); cudaFree(d_out);
  if (e != cudaSuccess) return cuda_err(h, e, "far-field kernel");
  return XFB_OK;
}

int xfb_state_size(const xfb_handle* h, size_t* bytes) {
  if (!h || !bytes) return set_err(nullptr, XFB_ERR_INVALID, "null argument");
  if (!h->inited) return set_err(const_cast<xfb_handle*>(h), XFB_ERR_STATE, "handle not initialised");
  size_t s = sizeof(long long);
  for (const Buf& b : h->bufs)
    if (b.state) s += b.bytes;
  *bytes = s;
  return XFB_OK;
}

int xfb_get_state(xfb_handle* h, void* dst, size_t len) {
  int rc = check_handle(h, true);
  if (rc) return rc;
  size_t need;
  if ((rc = xfb_state_size(h, &need))) return rc;
  if (!dst || len < need) return set_err(h, XFB_ERR_RANGE, "state buffer too small");
  XFB_CUDA(h, cudaStreamSynchronize(h->stream));
  char* o = static_cast<char*>(dst);
  std::memcpy(o, &h->step, sizeof(long long));
  o += sizeof(long long);
  for (const Buf& b : h->bufs)
    if (b.state) {
      XFB_CUDA(h, cudaMemcpy(o, b.p, b.bytes, cudaMemcpyDeviceToHost));
      o += b.bytes;
    }
  return XFB_OK;
}

int xfb_set_state(xfb_handle* h, const void* src, size_t len) {
  int rc = check_handle(h, true);
  if (rc) return rc;
  size_t need;
  if ((rc = xfb_state_size(h, &need))) return rc;
  if (!src || len < need) return set_err(h, XFB_ERR_RANGE, "state buffer too small");
  XFB_CUDA(h, cudaStreamSynchronize(h->stream));
  const char* o = static_cast<const char*>(src);
  long long step;
  std::memcpy(&step, o, sizeof(long long));
  if (step < 0 || step > h->c.total_steps) return set_err(h, XFB_ERR_INVALID, "state step outside this run");
  o += sizeof(long long);
  for (const Buf& b : h->bufs)
    if (b.state) {
      XFB_CUDA(h, cudaMemcpy(b.p, o, b.bytes, cudaMemcpyHostToDevice));
      o += b.bytes;
    }
  h->step = step;
  return XFB_OK;
}

int xfb_check_finite(xfb_handle* h, long long* bad) {
  int rc = check_handle(h, true);
  if (rc) return rc;
  XFB_CUDA(h, cudaMemsetAsync(h->scratch_u64, 0, sizeof(unsigned long long), h->stream));
  for (int q = 0; q < 6; ++q) {
    if (!h->f[q]) continue;
    if (h->c.prec == XFB_FP64)
      k_nonfinite<double><<<592, 256, 0, h->stream>>>(as<const double>(h->f[q]), h->elems, h->scratch_u64);
    else
      k_nonfinite<float><<<592, 256, 0, h->stream>>>(as<const float>(h->f[q]), h->elems, h->scratch_u64);
  }
  unsigned long long n = 0;
  XFB_CUDA(h, cudaMemcpyAsync(&n, h->scratch_u64, sizeof(n), cudaMemcpyDeviceToHost, h->stream));
  XFB_CUDA(h, cudaStreamSynchronize(h->stream));
  if (bad) *bad = static_cast<long long>(n);
  if (n) return set_err(h, XFB_ERR_NUMERIC, std::to_string(n) + " non-finite field values");
  return XFB_OK;
}

int xfb_compiled_view_get(const xfb_handle* h, xfb_compiled_view* v) {
  if (!h || !v) return set_err(nullptr, XFB_ERR_INVALID, "null argument");
  const Compiled& c = h->c;
  std::memset(v, 0, sizeof(*v));
  v->dim = c.dim; v->nx = c.nx; v->ny = c.ny; v->nz = c.nz;
  v->dx = c.dx; v->dy = c.dy; v->dz = c.dz; v->dt = c.dt;
  v->material_id = c.mat_id.data();
  v->n_materials = c.n_mat;
  v->coeff = c.coeff.data();
  v->ade_kind = c.ade_kind; v->ade_poles = c.ade_poles;
  v->ade_mat = c.ade_mat.data();
  v->ade_pole = c.ade_pole.data();
  for (int q = 0; q < 6; ++q) v->pml_cells[q] = c.pml[q];
  for (int a = 0; a < 3; ++a) {
    v->pml_ae[a] = c.pml_ae[a].data(); v->pml_be[a] = c.pml_be[a].data();
    v->pml_ah[a] = c.pml_ah[a].data(); v->pml_bh[a] = c.pml_bh[a].data();
  }
  v->tfsf_enabled = c.tfsf_on;
  for (int q = 0; q < 6; ++q) v->tfsf_box[q] = c.tf[q];
  for (int a = 0; a < 3; ++a) {
    v->tfsf_proj_int[a] = c.proj_int[a].data();
    v->tfsf_proj_half[a] = c.proj_half[a].data();
    v->tfsf_transform_e[a] = c.tr_e[a]; v->tfsf_transform_h[a] = c.tr_h[a];
    v->tfsf_ca[a] = c.ca[a]; v->tfsf_cb[a] = c.cb[a];
  }
  v->aux_nl = c.aux_nl;
  v->aux_ceih = c.aux_ceih; v->aux_chie = c.aux_chie; v->aux_abc = c.aux_abc;
  v->aux_source = c.aux_source.data();
  v->total_steps = c.total_steps;
  v->nf2ff_enabled = c.nf_on;
  for (int q = 0; q < 6; ++q) v->nf2ff_box[q] = c.nf[q];
  v->n_freqs = static_cast<int>(c.freqs.size());
  v->freqs = c.freqs.data();
  v->nf2ff_te = c.te.data();
  v->nf2ff_th = c.th.data();
  return XFB_OK;
}

}  // extern "C"
