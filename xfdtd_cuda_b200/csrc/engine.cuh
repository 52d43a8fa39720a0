// Per-precision engine: device buffers, launch sequencing, CUDA-graph replay,
// read-back.  Included by engine_f32.cu (compiled with FMA contraction) and
// engine_f64.cu (compiled with --fmad=false, so FP64 reproduces the CPU
// restatement bit for bit).
#pragma once

#include <cudaTypedefs.h>  // PFN_cuTensorMapEncodeTiled
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <omp.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>

#include "fused3d.cuh"
#include "handle.h"
#include "kernels.cuh"
#include "labc.cuh"
#include "plain.cuh"
#include "tb2d.cuh"

namespace xfb {

inline int upload_step_items(xfb_handle* h);
inline int upload_ade_runs(xfb_handle* h);
inline int upload_td(xfb_handle* h);
template <typename T>
int encode_stage_maps(xfb_handle* h);

// Tile of the blocked 2-D step: TJ + 2 S + 1 columns fill a shared row of
// kTbPitch, TI rows keep the tile count within two CTAs per SM when it can
// and the tile's shared memory within a CTA's 227 KB.
// False (one launch per step) when blocking is off, the scene has movie
// monitors (recorded between steps), or a tile's region would hold more CPML
// rows or columns than its psi tables.
template <typename T>
bool tb2d_plan(xfb_handle* h) {
  const Compiled& c = h->c;
  const int S = h->tb_steps;
  if (c.dim != 2 || S <= 0 || !c.movies.empty()) return false;
  const int TJ = kTbPitch - 1 - 2 * S;
  if (TJ < 16) return false;
  const int ntj = (c.ny + TJ - 1) / TJ;
  int TI = (c.nx + std::max(1, 296 / ntj) - 1) / std::max(1, 296 / ntj);
  TI = std::min(64, std::max(16, TI));
  // the tile's shared memory within the 227 KB a CTA may use
  while (TI > 16 && TbLayout<T>(TI + 2 * S + 1, c.n_mat).bytes > 227u * 1024u) --TI;
  if (TbLayout<T>(TI + 2 * S + 1, c.n_mat).bytes > 227u * 1024u) return false;
  auto fits = [&](int n, int tile, int lo, int hi) {  // slab cells of every tile's region along one axis
    for (int a0 = 0; a0 < n; a0 += tile) {
      int cnt = 0;
      for (int q = std::max(0, a0 - S); q <= std::min(n - 1, a0 + tile + S); ++q) cnt += (q < lo || q >= n - hi) ? 1 : 0;
      if (cnt > kTbSlab) return false;
    }
    return true;
  };
  if (!fits(c.nx, TI, c.pml[0], c.pml[1]) || !fits(c.ny, TJ, c.pml[2], c.pml[3])) return false;
  h->tb_ti = TI;
  h->tb_tj = TJ;
  return true;
}

// Update coefficients rounded to a 16-bit storage format (round to nearest
// even) and widened back: what a LUT stored in that format would hold.
inline std::vector<double> round_coefficients(const std::vector<double>& v, int storage) {
  std::vector<double> out(v.size());
  for (size_t q = 0; q < v.size(); ++q) {
    const float f = static_cast<float>(v[q]);
    out[q] = storage == XFB_COEFF_FP16 ? static_cast<double>(__half2float(__float2half_rn(f)))
                                       : static_cast<double>(__bfloat162float(__float2bfloat16_rn(f)));
  }
  return out;
}

// Material ids, dense [nx][ny][nz] -> padded (plane stride sx, row stride
// sy); a warp per (i, j) row.  (A template, like every kernel of this
// header, so that each engine unit keeps its own instance.)
template <typename U>
__global__ void k_spread_ids(const U* __restrict__ src, U* __restrict__ dst, int ny, int nz, long long sx,
                             long long sy, long long rows) {
  const int lane = threadIdx.x & 31;
  const long long w0 = (static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const long long nw = (static_cast<long long>(gridDim.x) * blockDim.x) >> 5;
  for (long long r = w0; r < rows; r += nw) {
    const long long i = r / ny, j = r - i * ny;
    const U* s = src + r * nz;
    U* d = dst + i * sx + j * sy;
    for (int k = lane; k < nz; k += 32) d[k] = s[k];
  }
}

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
  h->guard = roundup(h->sx + 40 * h->sy + 256, 64);
  const size_t fbytes = (h->elems + 2 * h->guard) * sizeof(T);
  int rc;
  {  // every component of both field sets in one block, in checkpoint order
    int comps[6], nc = 0;
    for (int q = 0; q < 6; ++q)
      if (c.dim == 3 || q == XFB_EZ || q == XFB_HX || q == XFB_HY) comps[nc++] = q;
    const int per = fused(h) ? 2 : 1;
    void* ps[12];
    if ((rc = alloc_block(h, ps, nc * per, fbytes, true))) return rc;
    for (int u = 0; u < nc; ++u) {
      h->f[comps[u]] = as<T>(ps[u * per]) + h->guard;
      if (fused(h)) h->f1[comps[u]] = as<T>(ps[u * per + 1]) + h->guard;
    }
  }
  // material ids in the padded layout: the dense array is copied as it is and
  // spread into the (zeroed) padded one on the device
  {
    void* p;  // same guard as the fields (the one-sweep kernel stages halo windows)
    if ((rc = alloc(h, &p, static_cast<size_t>(h->elems) + 2 * h->guard, false))) return rc;
    h->mid = static_cast<uint8_t*>(p) + h->guard;
    const size_t dense = c.mat_id.size();
    void* tmp = nullptr;
    if (cudaMalloc(&tmp, dense) != cudaSuccess) {
      cudaGetLastError();
      return set_err(h, XFB_ERR_OOM, "cudaMalloc of the material-id staging buffer failed");
    }
    rc = copy(h, tmp, c.mat_id.data(), dense, cudaMemcpyHostToDevice);
    if (rc == XFB_OK) {
      const long long rows = static_cast<long long>(nx) * ny;
      k_spread_ids<uint8_t><<<static_cast<unsigned>(std::min<long long>((rows + 7) / 8, 148LL * 64)), 256, 0, h->stream>>>(
          static_cast<const uint8_t*>(tmp), h->mid, ny, nz, h->sx, h->sy, rows);
      const cudaError_t e = cudaGetLastError();
      if (e != cudaSuccess) rc = cuda_err(h, e, "material-id spread");
      const cudaError_t e2 = cudaStreamSynchronize(h->stream);  // before the staging buffer is freed
      if (rc == XFB_OK && e2 != cudaSuccess) rc = cuda_err(h, e2, "material-id spread");
    }
    cudaFree(tmp);
    if (rc) return rc;
  }
  if (h->coeff_storage == XFB_COEFF_NATIVE) {
    if ((rc = upload<T>(h, &h->lut, c.coeff))) return rc;
    if ((rc = upload<T>(h, &h->lut8, c.coeff8))) return rc;
  } else {  // the storage trial: every coefficient rounded to FP16 or BF16 first
    if ((rc = upload<T>(h, &h->lut, round_coefficients(c.coeff, h->coeff_storage)))) return rc;
    if ((rc = upload<T>(h, &h->lut8, round_coefficients(c.coeff8, h->coeff_storage)))) return rc;
  }
  h->lines_on = fused(h) && c.dim == 3 && c.tfsf_on;
  if (h->lines_on) {  // TFSF line tables: [face][plane][component][k or j]
    // (rows at least as long as the widest box: 34 k values, TJ + 2 <= 18 j values)
    h->line_ykp = std::max<long long>(h->nzp, 64);
    h->line_zjp = std::max<long long>(roundup(c.ny, 2), 32);
    const size_t ny_el = 2ull * (c.nx + 1) * 2 * h->line_ykp, nz_el = 2ull * (c.nx + 1) * 2 * h->line_zjp;
    for (int q = 0; q < 4; ++q)
      if ((rc = alloc(h, &h->line_tab[q], (q < 2 ? ny_el : nz_el) * sizeof(double), false))) return rc;
  }
  if (fused(h) && c.dim == 3 && (rc = upload_step_items(h))) return rc;
  if (fused(h) && c.dim == 3 && h->ade_deferred && (rc = upload_ade_runs(h))) return rc;
  if (fused(h) && c.dim == 3) {
    if ((rc = encode_stage_maps<T>(h))) return rc;
    void* p;  // error word pair: flag, poll limit of the staging waits
    if ((rc = alloc(h, &p, 2 * sizeof(int), false))) return rc;
    h->step_err = static_cast<int*>(p);
    const int words[2] = {0, kWaitPolls};
    if ((rc = copy(h, p, words, sizeof(words), cudaMemcpyHostToDevice))) return rc;
  }
  if (plain(h)) {  // per-cell coefficient arrays, expanded from the LUT on the device
    PlainCoef<T> pc;
    for (int q = 0; q < 18; ++q) {
      if ((rc = alloc(h, &h->plain_c[q], h->elems * sizeof(T), false))) return rc;
      pc.c[q] = as<T>(h->plain_c[q]);
    }
    k_plain_expand<T><<<4 * 148, 256, 0, h->stream>>>(pc, h->mid, as<const T>(h->lut), h->elems);
    XFB_CUDA(h, cudaGetLastError());
  }
  {
    void* p;
    if ((rc = alloc(h, &p, c.mat_disp.size(), false))) return rc;
    if ((rc = copy(h, p, c.mat_disp.data(), c.mat_disp.size(), cudaMemcpyHostToDevice))) return rc;
    h->mat_disp = static_cast<uint8_t*>(p);
  }
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
    if (fused(h))
      for (int q = 0; q < 6; ++q)
        if ((rc = alloc(h, &h->psi_h1[q], sz[6 + q], true))) return rc;
  } else {
    h->ysx = Ly;
    const size_t bx = Lx * h->sx * sizeof(T), by = (nx + 1) * Ly * sizeof(T);
    if ((rc = alloc(h, &h->psi[1], bx, true))) return rc;   // ez_x
    if ((rc = alloc(h, &h->psi[2], by, true))) return rc;   // ez_y
    if ((rc = alloc(h, &h->psi[6], bx, true))) return rc;   // hy_x
    if ((rc = alloc(h, &h->psi[9], by, true))) return rc;   // hx_y
    if (fused(h)) {  // H-side psi of field set 1 (one-sweep path)
      if ((rc = alloc(h, &h->psi_h1[0], bx, true))) return rc;
      if ((rc = alloc(h, &h->psi_h1[3], by, true))) return rc;
    }
    h->tb_on = fused(h) && tb2d_plan<T>(h);
    if (h->tb_on) {  // the E-side psi alternates too on the blocked path
      if ((rc = alloc(h, &h->psi_e1[0], bx, true))) return rc;
      if ((rc = alloc(h, &h->psi_e1[1], by, true))) return rc;
      // the kernel's shared-memory limit, set (and the kernel loaded) here,
      // outside any stream capture of the step loop
      const TbLayout<T> lay(h->tb_ti + 2 * h->tb_steps + 1, c.n_mat);
      XFB_CUDA(h, cudaFuncSetAttribute(k_step2_tb<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(lay.bytes)));
    }
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
    // incident-field tables of every step of the run (k_aux_table)
    void* p;
    const size_t steps = static_cast<size_t>(c.total_steps);
    if ((rc = alloc(h, &p, (steps + 1) * (c.aux_nl + 1) * sizeof(double), false))) return rc;
    h->e_aux = static_cast<double*>(p);
    if ((rc = alloc(h, &p, std::max<size_t>(1, steps) * c.aux_nl * sizeof(double), false))) return rc;
    h->h_aux = static_cast<double*>(p);
    if (c.inc_given) {  // the caller's tables (rows of every step of the run)
      if ((rc = copy(h, h->e_aux, c.e_inc.data(), (steps + 1) * (c.aux_nl + 1) * sizeof(double), cudaMemcpyHostToDevice)))
        return rc;
      if (steps > 0 && (rc = copy(h, h->h_aux, c.h_inc.data(), steps * c.aux_nl * sizeof(double), cudaMemcpyHostToDevice)))
        return rc;
    } else {
      if ((rc = upload<double>(h, &p, c.aux_source))) return rc;
      h->src = static_cast<double*>(p);
      k_aux_table<<<1, 1024, 0, h->stream>>>(h->e_aux, h->h_aux, c.aux_nl, c.aux_ceih, c.aux_chie, c.aux_abc, h->src,
                                              c.total_steps);
      XFB_CUDA(h, cudaGetLastError());
    }
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
    if ((rc = alloc(h, &p, static_cast<size_t>(kNfRing) * 4 * h->nf_npts * sizeof(double), false))) return rc;
    h->nf_ring = static_cast<double*>(p);
    if ((rc = alloc(h, &p, sizeof(long long), true))) return rc;
    h->nf_done = static_cast<long long*>(p);
    if ((rc = upload<double>(h, &p, c.te))) return rc;
    h->te = static_cast<double2*>(p);
    if ((rc = upload<double>(h, &p, c.th))) return rc;
    h->th = static_cast<double2*>(p);
  }
  if (c.td_on && (rc = upload_td(h))) return rc;
  // probes
  if (!c.probes.empty()) {
    const size_t n = c.probes.size();
    std::vector<long long> idx(n);
    std::vector<int> fld(n);
    for (size_t p = 0; p < n; ++p) {
      idx[p] = off3(h, c.probes[p].index[0], c.probes[p].index[1], c.dim == 3 ? c.probes[p].index[2] : 0);
      const int pi = c.probes[p].index[0];
      fld[p] = pi >= own_lo(h) && pi < own_hi(h) ? c.probes[p].field : -1;  // -1: another x slab's probe
    }
    void* p;
    if ((rc = alloc(h, &p, n * sizeof(long long), false))) return rc;
    h->probe_idx = static_cast<long long*>(p);
    if ((rc = copy(h, p, idx.data(), n * sizeof(long long), cudaMemcpyHostToDevice))) return rc;
    if ((rc = alloc(h, &p, n * sizeof(int), false))) return rc;
    h->probe_field = static_cast<int*>(p);
    if ((rc = copy(h, p, fld.data(), n * sizeof(int), cudaMemcpyHostToDevice))) return rc;
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
  if ((rc = alloc(h, &p, sizeof(int), false))) return rc;
  h->scratch_err = static_cast<int*>(p);
  XFB_CUDA(h, cudaStreamSynchronize(h->stream));
  return XFB_OK;
}

// ---------------------------------------------------------------------------
template <typename T>
GridP<T> grid_params(xfb_handle* h, int set = 0) {
  GridP<T> g;
  g.nx = h->c.nx; g.ny = h->c.ny; g.nz = h->c.nz;
  g.sx = h->sx; g.sy = h->sy;
  void* const* f = set ? h->f1 : h->f;
  g.ex = as<T>(f[0]); g.ey = as<T>(f[1]); g.ez = as<T>(f[2]);
  g.hx = as<T>(f[3]); g.hy = as<T>(f[4]); g.hz = as<T>(f[5]);
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

inline TfsfP tfsf_params(xfb_handle* h) {
  TfsfP t{};
  const Compiled& c = h->c;
  t.on = c.tfsf_on;
  if (!t.on) return t;
  t.is = c.tf[0]; t.ie = c.tf[1]; t.js = c.tf[2]; t.je = c.tf[3]; t.ks = c.tf[4]; t.ke = c.tf[5];
  t.pi0 = h->proj[0]; t.pi1 = h->proj[1]; t.pi2 = h->proj[2];
  t.ph0 = h->proj[3]; t.ph1 = h->proj[4]; t.ph2 = h->proj[5];
  for (int a = 0; a < 3; ++a) { t.tre[a] = c.tr_e[a]; t.trh[a] = c.tr_h[a]; t.ca[a] = c.ca[a]; t.cb[a] = c.cb[a]; }
  t.e_tab = h->e_aux; t.h_tab = h->h_aux; t.nl = c.aux_nl; t.e_aux = nullptr; t.h_aux = nullptr;
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

inline int chunks_for(int tiles, int n_march, int threads) {
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
PsiH<T> psi_h_set(xfb_handle* h, int set) {
  void* const* q = set ? h->psi_h1 : h->psi + 6;
  return PsiH<T>{as<T>(q[0]), as<T>(q[1]), as<T>(q[2]), as<T>(q[3]), as<T>(q[4]), as<T>(q[5])};
}

// Tile configurations of the one-sweep kernel: rows per thread R, row warps
// NWM (tile rows TJ = R * NWM).  A single scene picks 8 or 16 rows by the
// launch hint's row count; a batch also tries 14 rows (an 8-warp CTA, whose
// register budget at two CTAs per SM is 128 instead of 96).
struct StepTile { int r, nwm; };
constexpr StepTile kStepTiles[kStepTileCount] = {{2, 4}, {2, 8}, {2, 7}};
// region kinds (kStepKinds, bits: 1 x-slab planes, 2 y-slab columns, 8
// z-slab columns, 4 ADE box, 16 TFSF): lean, x planes, ADE box, y columns,
// z columns, y+z corner columns, anything with ADE next to a slab (all
// without TFSF code), lean with TFSF corrections, lean interior (the
// bulk-copy path of single scenes), kinds 1..6 with TFSF corrections for the
// items that meet the TFSF surface, lean interior with TFSF corrections, the
// y-, z- and corner-column kinds on the bulk-copy path, and those three with
// TFSF corrections
constexpr int kStepKindCount = 22;

// True when a work item over planes [p, q) of the tile at (j0, k0) may meet a
// TFSF correction: the cells it updates (H at planes p-1 .. q-1, rows j0-1 ..
// j0+TJ-1, columns k0-1 .. k0+31, which contain its E cells) meet a face
// layer of the TFSF box (H at the plane, row or column before a face and on
// the far face, E on both faces).
inline bool tfsf_touch(const Compiled& c, int p, int q, int j0, int TJ, int k0) {
  if (!c.tfsf_on) return false;
  const int lo[3] = {p - 1, j0 - 1, k0 - 1}, hi[3] = {q - 1, j0 + TJ - 1, k0 + 31};
  auto meets = [&](int a, int l, int h) { return l <= hi[a] && h >= lo[a]; };
  for (int a = 0; a < 3; ++a) {
    const int s0 = c.tf[2 * a], s1 = c.tf[2 * a + 1];
    const bool layer = meets(a, s0 - 1, s0) || meets(a, s1, s1);
    bool across = true;
    for (int b = 0; b < 3; ++b)
      if (b != a) across = across && meets(b, c.tf[2 * b], c.tf[2 * b + 1]);
    if (layer && across) return true;
  }
  return false;
}

// Work items of the one-sweep kernel for tiles of TJ x 32 cells: every tile
// column is cut along i into plane ranges whose cells (with the H halo plane
// below the range and the halo row and column of the tile) need no more than
// the range's kind handles.  Ranges are at most `ich` planes long.
inline void build_step_items(const Compiled& c, int TJ, int NT, bool ade_deferred, std::vector<int4> (&out)[kStepKindCount],
                             int plane_chunk = 0, bool lean_interior = false, int p0 = 0, int p1 = -1,
                             bool lines = false) {
  const int nx = c.nx, ny = c.ny, nz = c.nz;
  if (p1 < 0) p1 = nx;  // planes [p0, p1): the whole grid, or an x slab
  const int* L = c.pml;
  const int gx = (nz + 31) / 32, gy = (ny + TJ - 1) / TJ;
  const int nch = chunks_for(gx * gy, p1 - p0, NT);
  const int ich = plane_chunk > 0 ? plane_chunk : std::max(8, (p1 - p0 + nch - 1) / nch);
  auto xs = [&](int p) { return p < L[0] || p >= nx - L[1]; };
  const int* b = c.ade_box;
  const bool ade = !ade_deferred && c.ade_kind != XFB_ADE_NONE && b[1] > b[0];
  auto kind_of = [](int bits) {
    switch (bits) {
      case 0: return 0;
      case 1: return 1;
      case 4: return 2;
      case 3: return 3;
      case 9: return 4;
      case 11: return 5;
      default: return 6;
    }
  };
  for (int by = 0; by < gy; ++by)
    for (int bx = 0; bx < gx; ++bx) {
      const int j0 = by * TJ, k0 = bx * 32;
      const int rlo = std::max(j0 - 1, 0), rhi = std::min(j0 + TJ - 1, ny - 1);
      const int clo = std::max(k0 - 1, 0), chi = std::min(k0 + 31, nz - 1);
      const bool ycol = rlo < L[2] || rhi >= ny - L[3], zcol = clo < L[4] || chi >= nz - L[5];
      const bool yz = ycol || zcol;
      const bool adecol = ade && j0 < b[3] && j0 + TJ > b[2] && k0 < b[5] && k0 + 32 > b[4];
      auto need = [&](int p) { return (xs(p) ? 1 : 0) | (adecol && p >= b[0] && p < b[1] ? 4 : 0); };
      int p = p0;
      while (p < p1) {
        int q = p + 1, bits;
        if (yz) {
          bits = 1 | (ycol ? 2 : 0) | (zcol ? 8 : 0) | (adecol ? 4 : 0);
          q = std::min(p1, p + ich);
        } else {
          const int nd = need(p), halo = p > 0 && xs(p - 1) ? 1 : 0;
          bits = nd | halo;
          if (!(halo & ~nd))  // the halo plane adds nothing: extend over equal needs
            while (q < p1 && need(q) == nd && q - p < ich) ++q;
        }
        int kind = kind_of(bits);
        if (tfsf_touch(c, p, q, j0, TJ, k0)) kind = kind == 0 ? 7 : kind + 8;
        // lean and fully inside: the tile, its halo row and column, first plane >= 1
        if ((kind == 0 || kind == 7) && lean_interior && p >= 1 && j0 >= 1 && k0 >= 1 && j0 + TJ <= ny &&
            k0 + 32 <= nz)
          kind = kind == 0 ? kLeanInterior : kLeanInteriorTf;
        if (lean_interior && (kind == 3 || kind == 4 || kind == 5)) kind = kind == 3 ? kFastY : kind == 4 ? kFastZ : kFastYZ;
        if (lean_interior && (kind == 11 || kind == 12 || kind == 13))
          kind = kind == 11 ? kFastYTf : kind == 12 ? kFastZTf : kFastYZTf;
        // with staged TFSF lines the bulk-copy TFSF bodies hold one face of
        // the box per axis; a tile that meets both (a box thinner than a
        // tile) runs the general body, which computes every incident value
        if (lines && (kind == kLeanInteriorTf || kind == kFastYTf || kind == kFastZTf || kind == kFastYZTf) &&
            (tfsf_line_face(c.tf[2], c.tf[3], j0, TJ) == 2 || tfsf_line_face(c.tf[4], c.tf[5], k0, 32) == 2))
          kind = kind == kLeanInteriorTf ? 7 : kind == kFastYTf ? 11 : kind == kFastZTf ? 12 : 13;
        out[kind].push_back(make_int4(bx, by, p, q));
        p = q;
      }
    }
}

// True when the ADE update of the one-sweep path can run as a separate pass
// (k_ade_box): the box of dispersive cells lies outside the CPML slabs and
// contains no TFSF face plane, so no dispersive cell takes a correction that
// the reference applies after the ADE update.
inline bool ade_can_defer(const Compiled& c) {
  const int* b = c.ade_box;
  if (c.ade_kind == XFB_ADE_NONE || b[1] <= b[0] || b[3] <= b[2] || b[5] <= b[4]) return false;
  const int n[3] = {c.nx, c.ny, c.nz};
  for (int a = 0; a < 3; ++a) {
    if (b[2 * a] < c.pml[2 * a] || b[2 * a + 1] > n[a] - c.pml[2 * a + 1]) return false;
    if (c.tfsf_on)
      for (int e = 0; e < 2; ++e) {
        const int f = c.tf[2 * a + e];
        if (f >= b[2 * a] - 1 && f <= b[2 * a + 1]) return false;
      }
  }
  return true;
}

// The driver's tensor-map encoder, through the runtime's entry-point query
// (no link to the driver library).
inline PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }
  return fn;
}

// Staging tensor maps of k_step3 for both tile configurations and field sets:
// each component (and the material ids) as a (k, j, i) tensor of extents
// (nzp, ny+1, nx+1) over the padded layout, box = one plane's staged window
// (RW x RH, resp. MW x RH), zero fill outside the extents.  Box origins are
// k0 - HP (resp. k0 - 16) with k0 a multiple of 32: 16-byte aligned.  The
// bulk-store maps of step_item_fast cover the cells of the same arrays
// (extents nz, ny, nx: an edge tile's cells outside the grid are clipped)
// with a box of one tile (32 x TJ), stored at (k0, j0) >= 0 only.
template <typename T>
int encode_stage_maps(xfb_handle* h) {
  auto enc = tensor_map_encoder();
  if (!enc) return set_err(h, XFB_ERR_CUDA, "cuTensorMapEncodeTiled is not available from the driver");
  const Compiled& c = h->c;
  const cuuint64_t dims[3] = {static_cast<cuuint64_t>(h->nzp), static_cast<cuuint64_t>(c.ny + 1),
                              static_cast<cuuint64_t>(c.nx + 1)};
  // bulk stores write cells only: extents (nz, ny, nx) clip an edge tile
  const cuuint64_t sdims[3] = {static_cast<cuuint64_t>(c.nz), static_cast<cuuint64_t>(c.ny),
                               static_cast<cuuint64_t>(c.nx)};
  const cuuint32_t estr[3] = {1, 1, 1};
  const CUtensorMapDataType ft = sizeof(T) == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
  for (int t = 0; t < kStepTileCount; ++t) {
    const int TJ = kStepTiles[t].r * kStepTiles[t].nwm;
    const cuuint32_t rh = static_cast<cuuint32_t>(TJ + 2);
    const cuuint32_t fbox[3] = {static_cast<cuuint32_t>(32 + 2 * (16 / sizeof(T))), rh, 1};
    const cuuint32_t mbox[3] = {64, rh, 1};
    const cuuint32_t sbox[3] = {32, static_cast<cuuint32_t>(TJ), 1};
    for (int set = 0; set < 2; ++set) {
      void* const* f = set ? h->f1 : h->f;
      const cuuint64_t fstr[2] = {static_cast<cuuint64_t>(h->sy) * sizeof(T), static_cast<cuuint64_t>(h->sx) * sizeof(T)};
      for (int q = 0; q < 6; ++q) {
        CUresult r = enc(&h->stage_maps[t][set][q], ft, 3, f[q], dims, fstr, fbox, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                         CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        if (r != CUDA_SUCCESS) return set_err(h, XFB_ERR_CUDA, "cuTensorMapEncodeTiled (field) failed: " + std::to_string(r));
        r = enc(&h->store_maps[t][set][q], ft, 3, f[q], sdims, fstr, sbox, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_NONE, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        if (r != CUDA_SUCCESS) return set_err(h, XFB_ERR_CUDA, "cuTensorMapEncodeTiled (store) failed: " + std::to_string(r));
      }
      const cuuint64_t mstr[2] = {static_cast<cuuint64_t>(h->sy), static_cast<cuuint64_t>(h->sx)};
      CUresult r = enc(&h->stage_maps[t][set][6], CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, h->mid, dims, mstr, mbox, estr,
                       CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                       CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
      if (r != CUDA_SUCCESS) return set_err(h, XFB_ERR_CUDA, "cuTensorMapEncodeTiled (ids) failed: " + std::to_string(r));
    }
    if (h->lines_on) {  // TFSF line tables as (k or j, component, plane, face), boxes of one plane's line pair
      for (int q = 0; q < 4; ++q) {
        const cuuint64_t w = static_cast<cuuint64_t>(q < 2 ? h->line_ykp : h->line_zjp);
        const cuuint64_t ldims[4] = {w, 2, static_cast<cuuint64_t>(c.nx + 1), 2};
        const cuuint64_t lstr[3] = {w * 8, 2 * w * 8, static_cast<cuuint64_t>(c.nx + 1) * 2 * w * 8};
        const cuuint32_t lbox[4] = {static_cast<cuuint32_t>(q < 2 ? 34 : TJ + 2), 2, 1, 1};
        const cuuint32_t lestr[4] = {1, 1, 1, 1};
        CUresult r = enc(&h->line_maps[t][q], CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4, h->line_tab[q], ldims, lstr, lbox,
                         lestr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                         CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        if (r != CUDA_SUCCESS) return set_err(h, XFB_ERR_CUDA, "cuTensorMapEncodeTiled (TFSF lines) failed: " + std::to_string(r));
      }
    }
  }
  return XFB_OK;
}

inline LineP line_params(const xfb_handle* h) {
  LineP lp{};
  lp.yh = static_cast<double*>(h->line_tab[0]); lp.ye = static_cast<double*>(h->line_tab[1]);
  lp.zh = static_cast<double*>(h->line_tab[2]); lp.ze = static_cast<double*>(h->line_tab[3]);
  lp.ykp = h->line_ykp; lp.zjp = h->line_zjp;
  lp.ysl = 2 * h->line_ykp; lp.zsl = 2 * h->line_zjp;
  lp.yfs = static_cast<long long>(h->c.nx + 1) * lp.ysl; lp.zfs = static_cast<long long>(h->c.nx + 1) * lp.zsl;
  return lp;
}

// The TFSF line values of one step (before the step kernel that reads them).
template <typename T>
void launch_lines(xfb_handle* h, TimeP tp, cudaStream_t st) {
  const Compiled& c = h->c;
  const long long ni = c.tf[1] - c.tf[0] + 1, nj = c.tf[3] - c.tf[2] + 1, nk = c.tf[5] - c.tf[4] + 1;
  const long long work = 2 * ni * (nj + nk);
  const int blocks = static_cast<int>(std::min<long long>((work + 255) / 256, 148LL * 8));
  k_tfsf_lines<T><<<blocks, 256, 0, st>>>(tfsf_params(h), tp, line_params(h));
}

// Tables of the time-domain NF2FF: the sample points of every (face, field
// kind), sorted by bin offset d0 = floor(delay + off) (off = 1/2 for E, 0
// for H) and cut into chunks of at most kTdChunk points with one d0; for
// every (component, bin offset w) of a step's window, the chunk slots that
// land there (CSR, chunk order).  Component of a chunk's slot s: W (kind H)
// or U (kind E) along the face's tangential axis a (s < 3) or b (s >= 3), at
// bin offset d0 + s % 3.
struct TdTables {
  std::vector<int4> ent, chunk;
  std::vector<double> tsd;
  std::vector<int> offs, list;
};

inline void build_td_tables(const Compiled& c, TdTables& tb, int own_lo = 0, int own_hi = 1 << 30) {
  tb = TdTables{};
  for (int face = 0; face < 6; ++face)
    for (int kind = 0; kind < 2; ++kind) {
      const FaceGeom g = td_face_geom(c, face);
      const double off = kind ? 0.0 : 0.5;
      std::map<int, std::vector<std::pair<int4, double>>> by_d0;
      for (int i = std::max(g.i0, own_lo); i < std::min(g.i0 + g.ni, own_hi); ++i)
        for (int j = g.j0; j < g.j0 + g.nj; ++j)
          for (int k = g.k0; k < g.k0 + g.nk; ++k) {
            const double tsd = td_delay_steps(c, face, i, j, k);
            by_d0[static_cast<int>(std::floor(tsd + off))].push_back({make_int4(i, j, k, face * 2 + kind), tsd});
          }
      for (auto& kv : by_d0)
        for (size_t q0 = 0; q0 < kv.second.size(); q0 += kTdChunk) {
          const size_t q1 = std::min(kv.second.size(), q0 + kTdChunk);
          tb.chunk.push_back(make_int4(static_cast<int>(tb.ent.size()), static_cast<int>(q1 - q0), face * 2 + kind, kv.first));
          for (size_t q = q0; q < q1; ++q) {
            tb.ent.push_back(kv.second[q].first);
            tb.tsd.push_back(kv.second[q].second);
          }
        }
    }
  const int span = c.td_span;
  std::vector<std::vector<int>> cells(static_cast<size_t>(6) * span);
  for (size_t q = 0; q < tb.chunk.size(); ++q) {
    const int4 ch = tb.chunk[q];
    const int face = ch.z >> 1, kind = ch.z & 1, ax = face >> 1;
    const int base = kind ? 0 : 3, ca = (ax + 1) % 3, cb = (ax + 2) % 3;
    for (int slot = 0; slot < 6; ++slot) {
      const int comp = base + (slot < 3 ? ca : cb), w = ch.w + slot % 3;
      cells[static_cast<size_t>(comp) * span + w].push_back(static_cast<int>(q) * 6 + slot);
    }
  }
  tb.offs.assign(1, 0);
  for (const auto& v : cells) {
    tb.list.insert(tb.list.end(), v.begin(), v.end());
    tb.offs.push_back(static_cast<int>(tb.list.size()));
  }
}

inline int upload_td(xfb_handle* h) {
  TdTables tb;
  build_td_tables(h->c, tb, own_lo(h), own_hi(h));
  h->td_n = static_cast<long long>(tb.ent.size());
  h->td_nchunks = static_cast<int>(tb.chunk.size());
  void* p;
  int rc;
  if ((rc = alloc(h, &h->td_ent, tb.ent.size() * sizeof(int4), false))) return rc;
  if ((rc = copy(h, h->td_ent, tb.ent.data(), tb.ent.size() * sizeof(int4), cudaMemcpyHostToDevice))) return rc;
  if ((rc = upload<double>(h, &p, tb.tsd))) return rc;
  h->td_tsd = static_cast<double*>(p);
  if ((rc = alloc(h, &p, 2 * tb.ent.size() * sizeof(double), true))) return rc;
  h->td_prev = static_cast<double*>(p);
  if ((rc = alloc(h, &h->td_chunk, tb.chunk.size() * sizeof(int4), false))) return rc;
  if ((rc = copy(h, h->td_chunk, tb.chunk.data(), tb.chunk.size() * sizeof(int4), cudaMemcpyHostToDevice))) return rc;
  if ((rc = alloc(h, &p, tb.chunk.size() * 6 * sizeof(double), false))) return rc;
  h->td_part = static_cast<double*>(p);
  if ((rc = alloc(h, &p, tb.offs.size() * sizeof(int), false))) return rc;
  h->td_offs = static_cast<int*>(p);
  if ((rc = copy(h, p, tb.offs.data(), tb.offs.size() * sizeof(int), cudaMemcpyHostToDevice))) return rc;
  if ((rc = alloc(h, &p, std::max<size_t>(1, tb.list.size()) * sizeof(int), false))) return rc;
  h->td_list = static_cast<int*>(p);
  if ((rc = copy(h, p, tb.list.data(), tb.list.size() * sizeof(int), cudaMemcpyHostToDevice))) return rc;
  if ((rc = alloc(h, &p, 6 * static_cast<size_t>(std::max(1LL, h->c.td_bins)) * sizeof(double), true))) return rc;
  h->td_pot = static_cast<double*>(p);
  return XFB_OK;
}

inline TdP td_params(const xfb_handle* h) {
  TdP td{};
  td.ent = static_cast<const int4*>(h->td_ent);
  td.tsd = h->td_tsd;
  td.prev = h->td_prev;
  td.n = h->td_n;
  td.chunk = static_cast<const int4*>(h->td_chunk);
  td.part = h->td_part;
  td.offs = h->td_offs;
  td.list = h->td_list;
  td.span = h->c.td_span;
  td.pot = h->td_pot;
  td.bins = h->c.td_bins;
  td.ds[0] = h->c.dy * h->c.dz;
  td.ds[1] = h->c.dz * h->c.dx;
  td.ds[2] = h->c.dx * h->c.dy;
  return td;
}

inline int upload_step_items(xfb_handle* h) {
  h->ade_deferred = ade_can_defer(h->c);
  for (int t = 0; t < 2; ++t) {
    std::vector<int4> items[kStepKindCount];
    const int nt = (kStepTiles[t].nwm + 1) * 32;
    build_step_items(h->c, kStepTiles[t].r * kStepTiles[t].nwm, nt, h->ade_deferred, items, 0, true,
                     is_slab(h) ? h->slab_i0 : 0, is_slab(h) ? h->slab_i1 : -1, h->lines_on);
    // one list, the kind in the high half of .x: first the costly kinds (y/z
    // CPML columns, in-kernel ADE), costliest first, so the long items start
    // early; then the lean and x-slab items ordered by first plane, then row
    // and column tile, so CTAs resident together cover neighbouring tiles of
    // the same plane range and the halo rows and columns one CTA stages are
    // the ones its neighbours read moments before (L2 hits)
    static const int costly[] = {14, 6, 13, 5, kFastYZTf, kFastYZ, 12, 4, kFastZTf, kFastZ, 11, 3, kFastYTf, kFastY, 10, 2};
    std::vector<int4> all, rest;
    for (int q : costly)
      for (int4 v : items[q]) all.push_back(make_int4(v.x | (q << 16), v.y, v.z, v.w));
    for (int q : {0, 1, 7, kLeanInterior, 9, kLeanInteriorTf})
      for (int4 v : items[q]) rest.push_back(make_int4(v.x | (q << 16), v.y, v.z, v.w));
    std::stable_sort(rest.begin(), rest.end(), [](const int4& a, const int4& b) {
      if (a.z != b.z) return a.z < b.z;
      if (a.y != b.y) return a.y < b.y;
      return (a.x & 0xffff) < (b.x & 0xffff);
    });
    all.insert(all.end(), rest.begin(), rest.end());
    h->n_step_items[t] = static_cast<int>(all.size());
    if (all.empty()) continue;
    int rc = alloc(h, &h->step_items[t], all.size() * sizeof(int4), false);
    if (rc) return rc;
    if ((rc = copy(h, h->step_items[t], all.data(), all.size() * sizeof(int4), cudaMemcpyHostToDevice))) return rc;
  }
  return XFB_OK;
}

// Work list of the deferred ADE pass: the dispersive cells of the ADE box as
// runs along k, cut at multiples of 32 (k_ade_runs), in (i, j, k) order.
// False (no list: k_ade_box) for grids with a side of 2^16 cells or more.
inline bool build_ade_runs(const Compiled& c, std::vector<int2>& runs, int p0 = 0, int p1 = -1) {
  const int* b = c.ade_box;
  runs.clear();
  if (c.nx >= 65536 || c.ny >= 65536 || c.nz >= 65536) return false;
  if (p1 < 0) p1 = c.nx;  // planes [p0, p1) (an x slab)
  const int i0 = std::max(b[0], p0), i1 = std::min(b[1], p1);
  if (i1 <= i0) return true;
  // the planes' runs are listed by plane-parallel threads, then joined in plane order
  std::vector<std::vector<int2>> per(static_cast<size_t>(i1 - i0));
#pragma omp parallel for schedule(dynamic, 4)
  for (int i = i0; i < i1; ++i) {
    std::vector<int2>& out = per[static_cast<size_t>(i - i0)];
    for (int j = b[2]; j < b[3]; ++j) {
      const uint8_t* row = c.mat_id.data() + (static_cast<size_t>(i) * c.ny + j) * c.nz;
      int k = b[4];
      while (k < b[5]) {
        if (!c.mat_disp[row[k]]) { ++k; continue; }
        const int kb = k & ~31;
        int e = k;
        while (e < b[5] && e < kb + 32 && c.mat_disp[row[e]]) ++e;
        out.push_back(make_int2(static_cast<int>(static_cast<unsigned>(i) | (static_cast<unsigned>(j) << 16)),
                                kb | ((k - kb) << 16) | ((e - kb) << 24)));
        k = e;
      }
    }
  }
  size_t n = 0;
  for (const auto& v : per) n += v.size();
  runs.reserve(n);
  for (const auto& v : per) runs.insert(runs.end(), v.begin(), v.end());
  return true;
}

inline int upload_ade_runs(xfb_handle* h) {
  std::vector<int2> runs;
  if (!build_ade_runs(h->c, runs, is_slab(h) ? h->slab_i0 : 0, is_slab(h) ? h->slab_i1 : -1)) return XFB_OK;
  h->n_ade_runs = static_cast<int>(runs.size());
  if (runs.empty()) return XFB_OK;
  int rc = alloc(h, &h->ade_runs, runs.size() * sizeof(int2), false);
  if (rc) return rc;
  return copy(h, h->ade_runs, runs.data(), runs.size() * sizeof(int2), cudaMemcpyHostToDevice);
}

// The deferred ADE pass of one step (E^n in field set `parity`, the plain
// eNext values in the other).
template <typename T>
void launch_ade(xfb_handle* h, int parity, cudaStream_t st) {
  if (h->n_ade_runs >= 0) {
    if (h->n_ade_runs > 0)
      k_ade_runs<T><<<(h->n_ade_runs + 3) / 4, 128, 0, st>>>(grid_params<T>(h, parity), grid_params<T>(h, 1 - parity),
                                                             ade_params<T>(h), static_cast<const int2*>(h->ade_runs),
                                                             h->n_ade_runs);
    return;
  }
  const int* b = h->c.ade_box;
  dim3 grd((b[5] - b[4] + 127) / 128, b[3] - b[2], b[1] - b[0]);
  k_ade_box<T><<<grd, 128, 0, st>>>(grid_params<T>(h, parity), grid_params<T>(h, 1 - parity), ade_params<T>(h),
                                    h->mat_disp);
}

template <typename T, int R, int NWM>
void launch_step3(xfb_handle* h, int t, int parity, TimeP tp, cudaStream_t st) {
  constexpr int NS = 4;
  using S = StepCfg<T, R, NWM, NS>;
  if (!h->n_step_items[t]) return;
  static bool attr_set[64] = {};  // per instantiation and device
  const int dev = h->device & 63;
  if (!attr_set[dev]) {
    cudaFuncSetAttribute(k_step3<T, R, NWM, NS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         static_cast<int>(S::bytes));
    attr_set[dev] = true;
  }
  // with the ADE update deferred to k_ade_box the step kernel does none
  AdeP<T> step_ade = ade_params<T>(h);
  if (h->ade_deferred) step_ade.kind = kAdeNone;
  StageMaps maps;
  std::memcpy(maps.f, h->stage_maps[t][parity], sizeof(maps.f));
  maps.mid = h->stage_maps[t][parity][6];
  StoreMaps outs;
  std::memcpy(outs.f, h->store_maps[t][1 - parity], sizeof(outs.f));
  LineMaps lines;
  if (h->lines_on) std::memcpy(&lines, h->line_maps[t], sizeof(lines));
  else std::memset(&lines, 0, sizeof(lines));
  k_step3<T, R, NWM, NS><<<h->n_step_items[t], S::NT, S::bytes, st>>>(
      grid_params<T>(h, parity), grid_params<T>(h, 1 - parity), pml_params<T>(h), psi_h_set<T>(h, parity),
      psi_h_set<T>(h, 1 - parity), tfsf_params(h), step_ade, tp, static_cast<const int4*>(h->step_items[t]),
      as<const T>(h->lut8), h->mat_disp, h->c.n_mat, maps, outs, lines, h->step_err);
}

// One-sweep step: one launch over all work items, for the tile the launch
// hint's row count picks (up to 8 rows: 8-row tiles, else 16 rows).
template <typename T>
void launch_fused(xfb_handle* h, int parity, TimeP tp, cudaStream_t st) {
  const int t = step_tile_index(h->tj);
  if (t == 0) launch_step3<T, kStepTiles[0].r, kStepTiles[0].nwm>(h, 0, parity, tp, st);
  else launch_step3<T, kStepTiles[1].r, kStepTiles[1].nwm>(h, 1, parity, tp, st);
}

// ---- learned absorbing boundary ---------------------------------------------
inline LabcP labc_params(const xfb_handle* h) {
  LabcP p = labc_layout(h->c.nx, h->c.ny, h->c.nz);
  const double cdt = c0() * h->c.dt, d[3] = {h->c.dx, h->c.dy, h->c.dz};
  for (int a = 0; a < 3; ++a) p.mur_k[a] = static_cast<float>((cdt - d[a]) / (cdt + d[a]));
  p.w = static_cast<const __nv_bfloat16*>(h->labc_w);
  p.hist = h->labc_hist;
  return p;
}

// ---- plain path (reference kernel structure) ------------------------------
constexpr int kPlainBlocks = 148 * 8, kPlainThreads = 256;

template <typename T, bool IS_E>
void plain_update(xfb_handle* h, const GridP<T>& g) {
  cudaStream_t s = h->stream;
  auto cf = [&](int q) { return as<const T>(h->plain_c[q]); };
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  if (IS_E) {
    k_plain_comp<T, true, 0><<<kPlainBlocks, kPlainThreads, 0, s>>>(g.ex, g.hy, g.hz, cf(CEXE), cf(CEXHY), cf(CEXHZ), nx, ny, nz, g.sx, g.sy);
    k_plain_comp<T, true, 1><<<kPlainBlocks, kPlainThreads, 0, s>>>(g.ey, g.hz, g.hx, cf(CEYE), cf(CEYHZ), cf(CEYHX), nx, ny, nz, g.sx, g.sy);
    k_plain_comp<T, true, 2><<<kPlainBlocks, kPlainThreads, 0, s>>>(g.ez, g.hx, g.hy, cf(CEZE), cf(CEZHX), cf(CEZHY), nx, ny, nz, g.sx, g.sy);
  } else {
    k_plain_comp<T, false, 0><<<kPlainBlocks, kPlainThreads, 0, s>>>(g.hx, g.ey, g.ez, cf(CHXH), cf(CHXEY), cf(CHXEZ), nx, ny, nz, g.sx, g.sy);
    k_plain_comp<T, false, 1><<<kPlainBlocks, kPlainThreads, 0, s>>>(g.hy, g.ez, g.ex, cf(CHYH), cf(CHYEZ), cf(CHYEX), nx, ny, nz, g.sx, g.sy);
    k_plain_comp<T, false, 2><<<kPlainBlocks, kPlainThreads, 0, s>>>(g.hz, g.ex, g.ey, cf(CHZH), cf(CHZEX), cf(CHZEY), nx, ny, nz, g.sx, g.sy);
  }
}

// TFSF agencies of one half step in the reference order (3-D agency,
// src/waveform_source/tfsf/tfsf_corrector.cu:201-271): face, field component.
template <typename T>
void plain_tfsf(xfb_handle* h, const GridP<T>& g, TimeP tp, int attr_h) {
  const Compiled& c = h->c;
  static const int order[12][2] = {{0, 2}, {1, 2}, {2, 2}, {3, 2}, {4, 0}, {5, 0},
                                   {2, 0}, {3, 0}, {4, 1}, {5, 1}, {0, 1}, {1, 1}};
  const TfsfP tf = tfsf_params(h);
  const int lo[3] = {c.tf[0], c.tf[2], c.tf[4]}, hi[3] = {c.tf[1], c.tf[3], c.tf[5]};
  for (int q = 0; q < 12; ++q) {
    const int face = order[q][0], fxyz = order[q][1];
    const int ax = face / 2, neg = (face % 2) == 0, a = (ax + 1) % 3, b = (ax + 2) % 3;
    PlainTfsfFace fc{};
    fc.neg = neg; fc.attr_h = attr_h; fc.fxyz = fxyz;
    fc.as = lo[a]; fc.ae = hi[a]; fc.bs = lo[b]; fc.be = hi[b];
    fc.cs = neg ? lo[ax] : hi[ax];
    const bool offset_a = (!attr_h && fxyz == b) || (attr_h && fxyz == a);
    if (offset_a) fc.ae += 1; else fc.be += 1;
    fc.dual = fxyz == a ? b : a;
    const int flag = (attr_h ? -1 : 1) * (fxyz == a ? -1 : 1) * (neg ? -1 : 1);
    fc.coef = (attr_h ? c.cb[ax] : c.ca[ax]) * flag;
    const long long n = static_cast<long long>(fc.ae - fc.as) * (fc.be - fc.bs);
    const int blocks = static_cast<int>(std::min<long long>((n + 255) / 256, kPlainBlocks));
    if (ax == 0) k_plain_tfsf<T, 0><<<blocks, 256, 0, h->stream>>>(g, tf, tp, fc);
    else if (ax == 1) k_plain_tfsf<T, 1><<<blocks, 256, 0, h->stream>>>(g, tf, tp, fc);
    else k_plain_tfsf<T, 2><<<blocks, 256, 0, h->stream>>>(g, tf, tp, fc);
  }
}

// CPML faces XN..ZP of one half step (pml_corrector.cu:273-291 task ranges).
template <typename T, bool IS_E>
void plain_pml(xfb_handle* h, const GridP<T>& g) {
  const Compiled& c = h->c;
  const PmlP<T> pm = pml_params<T>(h);
  const int n[3] = {c.nx, c.ny, c.nz};
  for (int face = 0; face < 6; ++face) {
    const int L = c.pml[face];
    if (!L) continue;
    const int ax = face / 2, side = face % 2, a = (ax + 1) % 3, b = (ax + 2) % 3;
    PlainPmlFace fc{};
    // E of a low face: planes 1 .. L-1 (plane L adds a zero correction); else the L slab planes
    const int planes = (IS_E && side == 0) ? L - 1 : L;
    fc.c0 = side ? n[ax] - L : (IS_E ? 1 : 0);
    if (planes <= 0) continue;
    // w = 0: component along a; w = 1: along b.  The +1 tangential extension
    // follows the reference ranges (pml_corrector.cu:121-133, 160-172).
    fc.a_end[0] = n[a] + (IS_E ? 0 : 1); fc.b_end[0] = n[b] + (IS_E ? 1 : 0);
    fc.a_end[1] = n[a] + (IS_E ? 1 : 0); fc.b_end[1] = n[b] + (IS_E ? 0 : 1);
    for (int w = 0; w < 2; ++w) fc.span[w] = static_cast<long long>(planes) * fc.a_end[w] * fc.b_end[w];
    // c_psi: coefficient of component a w.r.t. dual b (b = a+1: slot 3a+1),
    // of component b w.r.t. dual a (a = b+2: slot 3b+2)
    const int base = IS_E ? 0 : 9;
    const T* cps0 = as<const T>(h->plain_c[base + 3 * a + 1]);
    const T* cps1 = as<const T>(h->plain_c[base + 3 * b + 2]);
    const long long tot = fc.span[0] + fc.span[1];
    const int blocks = static_cast<int>(std::min<long long>((tot + 255) / 256, kPlainBlocks));
    if (ax == 0) k_plain_pml<T, IS_E, 0><<<blocks, 256, 0, h->stream>>>(g, pm, cps0, cps1, fc);
    else if (ax == 1) k_plain_pml<T, IS_E, 1><<<blocks, 256, 0, h->stream>>>(g, pm, cps0, cps1, fc);
    else k_plain_pml<T, IS_E, 2><<<blocks, 256, 0, h->stream>>>(g, pm, cps0, cps1, fc);
  }
}

// Monitors of one step (NF2FF accumulation, probes, movie frames) on the
// fields after the step, enqueued on stream s.
template <typename T>
void enqueue_records(xfb_handle* h, int parity, TimeP tp, cudaStream_t s, Prof* pf) {
  const Compiled& c = h->c;
  GridP<T> g = grid_params<T>(h, fused(h) ? 1 - parity : 0);
  if (c.nf_on) {
    NfP nf{};
    nf.nfreq = static_cast<int>(c.freqs.size());
    for (int q = 0; q < 6; ++q) nf.box[q] = c.nf[q];
    for (int q = 0; q < 7; ++q) nf.off[q] = h->nf_off[q];
    nf.npts = h->nf_npts;
    nf.acc = h->nf_acc; nf.te = h->te; nf.th = h->th;
    nf.total_steps = c.total_steps;
    nf.ring = h->nf_ring;
    nf.done = h->nf_done;
    nf.own_lo = own_lo(h);
    nf.own_hi = own_hi(h);
    prof_begin(h, pf, XFB_K_NF2FF);
    k_nf2ff<T><<<static_cast<unsigned>((h->nf_npts + 255) / 256), 256, 0, s>>>(g, nf, tp);
    prof_end(h, pf);
  }
  if (c.td_on && h->td_nchunks > 0) {
    const TdP td = td_params(h);
    prof_begin(h, pf, XFB_K_NF2FF);
    k_nftd_chunks<T><<<h->td_nchunks, kTdChunk, 0, s>>>(g, td, tp);
    k_nftd_bins<<<(6 * td.span + 127) / 128, 128, 0, s>>>(td, tp);
    prof_end(h, pf);
  }
  if (!c.probes.empty() && !h->tb_on) {  // the blocked 2-D kernel records its own
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
    k_movie<T><<<blocks, 256, 0, s>>>(as<const T>(field_ptr(h, fused(h) ? 1 - parity : 0, mv.field)), h->sx, h->sy, mv.lo[0], mv.lo[1], mv.lo[2], n0, n1, n2,
                                      mv.interval, h->movie_out[m], h->movie_frames[m], tp, own_lo(h), own_hi(h));
    prof_end(h, pf);
  }
}

template <typename T>
void enqueue_update(xfb_handle* h, int off, Prof* pf);
template <typename T>
void launch_tb2d(xfb_handle* h, int off, int S);

template <typename T>
void enqueue_step(xfb_handle* h, int off, Prof* pf = nullptr) {
  enqueue_update<T>(h, off, pf);
  TimeP tp{h->t_dev, off};
  enqueue_records<T>(h, static_cast<int>((h->step + off) & 1), tp, h->stream, pf);
}

// The update of one step (the field kernels, no monitors).
template <typename T>
void enqueue_update(xfb_handle* h, int off, Prof* pf) {
  const Compiled& c = h->c;
  TimeP tp{h->t_dev, off};
  const int parity = static_cast<int>((h->step + off) & 1);
  // fields after this step: the written set (one-sweep) or the only set (split)
  GridP<T> g = grid_params<T>(h, fused(h) ? 1 - parity : 0);
  PmlP<T> pm = pml_params<T>(h);
  TfsfP tf = tfsf_params(h);
  cudaStream_t s = h->stream;
  if (plain(h)) {
    prof_begin(h, pf, XFB_K_UPDATE_H);
    plain_update<T, false>(h, g);
    prof_end(h, pf);
    prof_begin(h, pf, XFB_K_CORRECT);
    if (c.tfsf_on) plain_tfsf<T>(h, g, tp, 1);
    plain_pml<T, false>(h, g);
    prof_end(h, pf);
    prof_begin(h, pf, XFB_K_UPDATE_E);
    plain_update<T, true>(h, g);
    prof_end(h, pf);
    prof_begin(h, pf, XFB_K_CORRECT);
    if (c.tfsf_on) plain_tfsf<T>(h, g, tp, 0);
    plain_pml<T, true>(h, g);
    prof_end(h, pf);
  } else if (fused(h)) {
    if (c.dim == 3 && h->lines_on) {  // the TFSF line values this step's kernel stages
      prof_begin(h, pf, XFB_K_AUX);
      launch_lines<T>(h, tp, s);
      prof_end(h, pf);
    }
    prof_begin(h, pf, XFB_K_STEP);
    if (c.dim == 2 && h->tb_on) {
      launch_tb2d<T>(h, off, 1);  // a single step (profiling): the blocked kernel with S = 1
    } else if (c.dim == 2) {
      // one-sweep 2-D step: 128-column blocks over plane chunks
      const int gx = (c.ny + 127) / 128;
      const int nch = chunks_for(gx, c.nx, 160);
      const int ich = (c.nx + nch - 1) / nch;
      k_step2<T><<<dim3(gx, (c.nx + ich - 1) / ich), 160, static_cast<size_t>(c.n_mat) * 18 * sizeof(T), s>>>(
          grid_params<T>(h, parity), grid_params<T>(h, 1 - parity), pml_params<T>(h), psi_h_set<T>(h, parity),
          psi_h_set<T>(h, 1 - parity), tfsf_params(h), tp, ich, h->c.n_mat);
    } else {
      launch_fused<T>(h, parity, tp, s);
    }
    if (h->ade_deferred) launch_ade<T>(h, parity, s);
    prof_end(h, pf);
    if (h->labc_on) {
      const LabcP lp = labc_params(h);
      prof_begin(h, pf, XFB_K_CORRECT);
      k_labc_apply<T><<<static_cast<unsigned>((lp.off[12] + 127) / 128), 128, 0, s>>>(
          grid_params<T>(h, parity), grid_params<T>(h, 1 - parity), lp);
      prof_end(h, pf);
    }
  } else if (c.dim == 3) {
    const int tj = tile_rows<T>(h);
    dim3 blk(h->tk, tj);
    const int gx = (c.nz + h->tk - 1) / h->tk, gy = (c.ny + tj - 1) / tj;
    const int nch = chunks_for(gx * gy, c.nx, h->tk * tj);
    const int ich = (c.nx + nch - 1) / nch;
    dim3 grd(gx, gy, (c.nx + ich - 1) / ich);
    prof_begin(h, pf, XFB_K_UPDATE_H);
    k_h3<T><<<grd, blk, 0, s>>>(g, pm, tf, tp, ich);
    prof_end(h, pf);
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
    prof_begin(h, pf, XFB_K_UPDATE_E);
    k_e2<T><<<grd, bx, 0, s>>>(g, pm, tf, tp, ich);
    prof_end(h, pf);
  }
}

// One step of an x slab, in two parts around the halo exchange: the update
// writes the owned planes of the new field set; the record samples the
// monitors on the owned planes (whose interpolations read the refilled halo
// planes) and advances the step counter.
template <typename T>
int slab_update(xfb_handle* h) {
  enqueue_update<T>(h, 0, nullptr);
  XFB_CUDA(h, cudaGetLastError());
  h->slab_pending = true;
  return XFB_OK;
}

template <typename T>
int slab_record(xfb_handle* h) {
  enqueue_records<T>(h, static_cast<int>(h->step & 1), TimeP{h->t_dev, 0}, h->stream, nullptr);
  k_bump<<<1, 1, 0, h->stream>>>(h->t_dev, 1);
  XFB_CUDA(h, cudaGetLastError());
  h->slab_pending = false;
  h->step += 1;
  return XFB_OK;
}

// One blocked 2-D launch: steps [off, off + S) of the chunk (S odd), read
// set and E-side psi buffer (step & 1), write the others.
template <typename T>
void launch_tb2d(xfb_handle* h, int off, int S) {
  const Compiled& c = h->c;
  const int parity = static_cast<int>((h->step + off) & 1);
  const TbLayout<T> lay(h->tb_ti + 2 * S + 1, c.n_mat);
  T* ez_x[2] = {as<T>(h->psi[1]), as<T>(h->psi_e1[0])};
  T* ez_y[2] = {as<T>(h->psi[2]), as<T>(h->psi_e1[1])};
  ProbeP pr{static_cast<int>(c.probes.size()), h->probe_idx, h->probe_field, h->probe_out, c.total_steps};
  const dim3 grid((c.ny + h->tb_tj - 1) / h->tb_tj, (c.nx + h->tb_ti - 1) / h->tb_ti);
  k_step2_tb<T><<<grid, kTbThreads, lay.bytes, h->stream>>>(
      grid_params<T>(h, parity), grid_params<T>(h, 1 - parity), pml_params<T>(h), psi_h_set<T>(h, parity),
      psi_h_set<T>(h, 1 - parity), ez_x[parity], ez_y[parity], ez_x[1 - parity], ez_y[1 - parity], tfsf_params(h),
      TimeP{h->t_dev, off}, pr, S, h->tb_ti, h->tb_tj, c.n_mat, h->scratch_err);
}

template <typename T>
void enqueue_chunk(xfb_handle* h, int n) {
  if (h->tb_on) {  // blocked 2-D: launches of odd step counts (each flips the sets once)
    for (int off = 0; off < n;) {
      int S = std::min(h->tb_steps, n - off);
      if (S % 2 == 0) --S;
      launch_tb2d<T>(h, off, S);
      off += S;
    }
  } else {
    for (int s = 0; s < n; ++s) enqueue_step<T>(h, s);
  }
  k_bump<<<1, 1, 0, h->stream>>>(h->t_dev, n);
}

template <typename T>
bool readback_buffers(xfb_handle* h);

template <typename T>
int run_steps(xfb_handle* h, long long n) {
  long long left = n;
  while (left > 0) {
    const int chunk = static_cast<int>(std::min<long long>(left, h->graph_steps));
    if (h->graph_on) {
      const int key = chunk * 2 + static_cast<int>(h->step & 1);
      auto it = h->graphs.find(key);
      if (it == h->graphs.end()) {
        cudaGraph_t graph;
        XFB_CUDA(h, cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
        enqueue_chunk<T>(h, chunk);
        XFB_CUDA(h, cudaStreamEndCapture(h->stream, &graph));
        cudaGraphExec_t ex;
        cudaError_t e = cudaGraphInstantiate(&ex, graph, 0);
        cudaGraphDestroy(graph);
        if (e != cudaSuccess) return cuda_err(h, e, "cudaGraphInstantiate");
        it = h->graphs.emplace(key, ex).first;
      }
      XFB_CUDA(h, cudaGraphLaunch(it->second, h->stream));
    } else {
      enqueue_chunk<T>(h, chunk);
      XFB_CUDA(h, cudaGetLastError());
    }
    left -= chunk;
    h->step += chunk;
  }
  // the read-back's staging buffers, allocated while the device steps (a
  // failure leaves the read-back to its unstaged form)
  if (n > 0 && !h->rb_host[1] && !readback_buffers<T>(h)) h->err.clear();
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



// Component f in the reference's dense layout, in the compute type: the
// component elements [q0, q0 + n) of the dense (i, j, k) order (s1 x s2
// elements per plane) gathered out of the padded layout, one thread per
// element.
template <typename T>
__global__ void k_gather_field(const T* src, T* dst, long long sx, long long sy, int s1, int s2, long long q0,
                               long long n) {
  for (long long q = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; q < n;
       q += static_cast<long long>(gridDim.x) * blockDim.x) {
    const long long e = q0 + q;
    const long long ij = e / s2;
    const long long i = ij / s1;
    const long long j = ij - i * s1, k = e - ij * s2;
    dst[q] = src[i * sx + j * sy + k];
  }
}

// Elements of one read-back chunk (device gather buffer and each pinned host
// buffer hold this many elements of the compute type).
constexpr long long kReadChunk = 4LL << 20;


// Read-back buffers of the handle (device gather buffer, two pinned host
// buffers, their events), allocated on first use and kept until the next
// init or destroy.  False when any allocation fails.
template <typename T>
bool readback_buffers(xfb_handle* h) {
  if (h->rb_dev && h->rb_host[0] && h->rb_host[1]) return true;
  const size_t bytes = static_cast<size_t>(kReadChunk) * sizeof(T);
  if (!h->rb_dev && alloc(h, &h->rb_dev, bytes, false) != XFB_OK) return false;
  for (int q = 0; q < 2; ++q) {
    if (!h->rb_host[q] && cudaHostAlloc(&h->rb_host[q], bytes, cudaHostAllocDefault) != cudaSuccess) {
      h->rb_host[q] = nullptr;
      cudaGetLastError();
      return false;
    }
    if (!h->rb_ev[q] && cudaEventCreateWithFlags(&h->rb_ev[q], cudaEventDisableTiming) != cudaSuccess) {
      h->rb_ev[q] = nullptr;
      cudaGetLastError();
      return false;
    }
  }
  return true;
}

// Read-back of component f into the caller's double array.  Chunks of
// kReadChunk elements are gathered on the device in the compute type, copied
// into pinned host buffer c & 1, and widened to double by host threads while
// the device gathers and copies the next chunk.  The host-side gather below
// runs when the read-back buffers cannot be allocated.
template <typename T>
int read_field_t(xfb_handle* h, int f, double* dst) {
  int s[3];
  comp_shape(h->c, f, s);
  const long long total = static_cast<long long>(s[0]) * s[1] * s[2];
  if (total == 0) return XFB_OK;
  if (readback_buffers<T>(h)) {
    const T* src = static_cast<const T*>(field_ptr(h, cur_set(h), f));
    T* stage = static_cast<T*>(h->rb_dev);
    const long long nch = (total + kReadChunk - 1) / kReadChunk;
    auto enqueue = [&](long long c) -> cudaError_t {
      const long long q0 = c * kReadChunk, n = std::min(kReadChunk, total - q0);
      const unsigned blocks = static_cast<unsigned>(std::min<long long>((n + 255) / 256, 148LL * 16));
      k_gather_field<T><<<blocks, 256, 0, h->stream>>>(src, stage, h->sx, h->sy, s[1], s[2], q0, n);
      cudaError_t e = cudaGetLastError();
      if (e == cudaSuccess) e = cudaMemcpyAsync(h->rb_host[c & 1], stage, n * sizeof(T), cudaMemcpyDeviceToHost, h->stream);
      if (e == cudaSuccess) e = cudaEventRecord(h->rb_ev[c & 1], h->stream);
      return e;
    };
    cudaError_t e = enqueue(0);
    for (long long c = 0; c < nch && e == cudaSuccess; ++c) {
      // host buffer (c + 1) & 1 was last read when chunk c - 1 was widened
      if (c + 1 < nch) e = enqueue(c + 1);
      if (e == cudaSuccess) e = cudaEventSynchronize(h->rb_ev[c & 1]);
      if (e != cudaSuccess) break;
      const long long q0 = c * kReadChunk, n = std::min(kReadChunk, total - q0);
      host_widen(static_cast<const T*>(h->rb_host[c & 1]), dst + q0, n);
      h->d2h_bytes += n * static_cast<long long>(sizeof(T));
    }
    if (e != cudaSuccess) {
      cudaStreamSynchronize(h->stream);  // no copy into the host buffers stays in flight
      return cuda_err(h, e, "field read-back");
    }
    return XFB_OK;
  }
  h->err.clear();  // no read-back buffers: gather on the host
  std::vector<T> tmp(static_cast<size_t>(h->elems));
  int rc;
  if ((rc = copy(h, tmp.data(), field_ptr(h, cur_set(h), f), tmp.size() * sizeof(T), cudaMemcpyDeviceToHost))) return rc;
  size_t o = 0;
  for (int i = 0; i < s[0]; ++i)
    for (int j = 0; j < s[1]; ++j)
      for (int k = 0; k < s[2]; ++k) dst[o++] = static_cast<double>(tmp[off3(h, i, j, k)]);
  return XFB_OK;
}

// dst <- src (device), bytes long, through the pinned read-back buffers:
// chunk c is copied into host buffer c & 1 while host threads copy chunk c - 1
// into dst.  Falls back to one pageable copy when the buffers cannot be had.
template <typename T>
int read_bytes_t(xfb_handle* h, void* dst, const void* src, size_t bytes) {
  if (bytes == 0) return XFB_OK;
  if (!readback_buffers<T>(h)) {
    h->err.clear();
    XFB_CUDA(h, cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, h->stream));
    XFB_CUDA(h, cudaStreamSynchronize(h->stream));
    h->d2h_bytes += static_cast<long long>(bytes);
    return XFB_OK;
  }
  const size_t chunk = static_cast<size_t>(kReadChunk) * sizeof(T);
  const size_t nch = (bytes + chunk - 1) / chunk;
  auto enqueue = [&](size_t c) -> cudaError_t {
    const size_t o = c * chunk, n = std::min(chunk, bytes - o);
    cudaError_t e = cudaMemcpyAsync(h->rb_host[c & 1], static_cast<const char*>(src) + o, n, cudaMemcpyDeviceToHost,
                                    h->stream);
    if (e == cudaSuccess) e = cudaEventRecord(h->rb_ev[c & 1], h->stream);
    return e;
  };
  cudaError_t e = enqueue(0);
  for (size_t c = 0; c < nch && e == cudaSuccess; ++c) {
    if (c + 1 < nch) e = enqueue(c + 1);
    if (e == cudaSuccess) e = cudaEventSynchronize(h->rb_ev[c & 1]);
    if (e != cudaSuccess) break;
    const size_t o = c * chunk, n = std::min(chunk, bytes - o);
    host_copy(h->rb_host[c & 1], static_cast<char*>(dst) + o, n);
    h->d2h_bytes += static_cast<long long>(n);
  }
  if (e != cudaSuccess) {
    cudaStreamSynchronize(h->stream);
    return cuda_err(h, e, "read-back");
  }
  return XFB_OK;
}

template <typename T>
int write_field_t(xfb_handle* h, int f, const double* src) {
  std::vector<T> tmp(static_cast<size_t>(h->elems));
  int rc;
  if ((rc = copy(h, tmp.data(), field_ptr(h, cur_set(h), f), tmp.size() * sizeof(T), cudaMemcpyDeviceToHost))) return rc;
  int s[3];
  comp_shape(h->c, f, s);
  size_t o = 0;
  for (int i = 0; i < s[0]; ++i)
    for (int j = 0; j < s[1]; ++j)
      for (int k = 0; k < s[2]; ++k) tmp[off3(h, i, j, k)] = static_cast<T>(src[o++]);
  // both sets: entries the update never writes (PEC walls, unused slots) must
  // agree in the two ping-pong buffers
  if ((rc = copy(h, h->f[f], tmp.data(), tmp.size() * sizeof(T), cudaMemcpyHostToDevice))) return rc;
  if (fused(h) && (rc = copy(h, h->f1[f], tmp.data(), tmp.size() * sizeof(T), cudaMemcpyHostToDevice))) return rc;
  return XFB_OK;
}

template <typename T>
void launch_nonfinite(xfb_handle* h) {
  for (int q = 0; q < 6; ++q) {
    if (!h->f[q]) continue;
    const T* fp = static_cast<const T*>(field_ptr(h, cur_set(h), q));
    k_nonfinite<T><<<592, 256, 0, h->stream>>>(fp, h->elems, h->scratch_u64);
  }
}

// ---- batches of scenes -----------------------------------------------------
template <typename T>
BatchScene<T> batch_scene(xfb_handle* h) {
  BatchScene<T> b{};
  b.g[0] = grid_params<T>(h, 0);
  b.g[1] = grid_params<T>(h, 1);
  b.psh[0] = psi_h_set<T>(h, 0);
  b.psh[1] = psi_h_set<T>(h, 1);
  b.pm = pml_params<T>(h);
  b.tf = tfsf_params(h);
  b.ad = ade_params<T>(h);
  if (h->ade_deferred) b.ad.kind = kAdeNone;
  b.lut8 = as<const T>(h->lut8);
  b.disp = h->mat_disp;
  b.n_mat = h->c.n_mat;
  if (h->lines_on) b.lines = line_params(h);
  return b;
}

inline int batch_upload(xfb_batch* b, void** dst, const void* src, size_t bytes) {
  cudaError_t e = cudaMalloc(dst, bytes);
  if (e != cudaSuccess) return batch_err(b, XFB_ERR_OOM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
  e = cudaMemcpyAsync(*dst, src, bytes, cudaMemcpyHostToDevice, b->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
  if (e != cudaSuccess) return batch_err(b, XFB_ERR_CUDA, std::string("batch upload: ") + cudaGetErrorString(e));
  return XFB_OK;
}

// Device tables of an initialised batch: scene parameters, the scenes'
// tensor maps, and for both tile configurations one work list over all scenes
// (costliest region kinds first; whole columns per item when the batch has
// enough columns to fill the GPU several times over).
template <typename T>
int batch_init(xfb_batch* b) {
  for (xfb_handle* h : b->hs)  // work items pack the k tile into 11 bits
    if ((h->c.nz + 31) / 32 > 2048) return batch_err(b, XFB_ERR_INVALID, "a batched scene has more than 65536 cells along z");
  std::vector<BatchScene<T>> sc;
  std::vector<BatchMaps> mp(b->hs.size());
  for (size_t q = 0; q < b->hs.size(); ++q) {
    xfb_handle* h = b->hs[q];
    sc.push_back(batch_scene<T>(h));
    for (int t = 0; t < kStepTileCount; ++t)
      for (int set = 0; set < 2; ++set) {
        std::memcpy(mp[q].stage[t][set].f, h->stage_maps[t][set], sizeof(mp[q].stage[t][set].f));
        mp[q].stage[t][set].mid = h->stage_maps[t][set][6];
        std::memcpy(mp[q].store[t][set].f, h->store_maps[t][set], sizeof(mp[q].store[t][set].f));
      }
    for (int t = 0; t < kStepTileCount; ++t)
      if (h->lines_on) std::memcpy(&mp[q].line[t], h->line_maps[t], sizeof(mp[q].line[t]));
  }
  int rc;
  b->lines_work = 0;  // largest line-table work of a scene (k_tfsf_lines_batch)
  for (xfb_handle* h : b->hs)
    if (h->lines_on) {
      const Compiled& c = h->c;
      const long long ni = c.tf[1] - c.tf[0] + 1, nj = c.tf[3] - c.tf[2] + 1, nk = c.tf[5] - c.tf[4] + 1;
      b->lines_work = std::max(b->lines_work, 2 * ni * (nj + nk));
    }
  if ((rc = batch_upload(b, &b->scenes, sc.data(), sc.size() * sizeof(BatchScene<T>)))) return rc;
  if ((rc = batch_upload(b, &b->maps, mp.data(), mp.size() * sizeof(BatchMaps)))) return rc;
  {  // error word pair: flag, poll limit of the staging waits
    static const int words[2] = {0, kWaitPolls};
    if ((rc = batch_upload(b, reinterpret_cast<void**>(&b->err_dev), words, sizeof(words)))) return rc;
  }
  for (int t = 0; t < kStepTileCount; ++t) {
    const int TJ = kStepTiles[t].r * kStepTiles[t].nwm, NT = (kStepTiles[t].nwm + 1) * 32;
    long long columns = 0;
    for (xfb_handle* h : b->hs) columns += static_cast<long long>((h->c.nz + 31) / 32) * ((h->c.ny + TJ - 1) / TJ);
    const bool whole = columns >= 8LL * 148 * 2;
    std::vector<int4> per_kind[kStepKindCount];
    for (size_t q = 0; q < b->hs.size(); ++q) {
      const xfb_handle* h = b->hs[q];
      std::vector<int4> items[kStepKindCount];
      build_step_items(h->c, TJ, NT, h->ade_deferred, items, whole ? h->c.nx : 0, true, 0, -1, h->lines_on);
      for (int k = 0; k < kStepKindCount; ++k)
        for (int4 v : items[k]) per_kind[k].push_back(make_int4(v.x | (k << 11) | (static_cast<int>(q) << 16), v.y, v.z, v.w));
    }
    std::vector<int4> all;
    for (int k = kStepKindCount - 1; k >= 0; --k) {
      // within a kind, longer plane ranges first
      std::stable_sort(per_kind[k].begin(), per_kind[k].end(), [](const int4& a, const int4& c) { return a.w - a.z > c.w - c.z; });
      all.insert(all.end(), per_kind[k].begin(), per_kind[k].end());
    }
    b->n_items[t] = static_cast<int>(all.size());
    if (!all.empty() && (rc = batch_upload(b, &b->items[t], all.data(), all.size() * sizeof(int4)))) return rc;
    // the persistent form takes the same list (costliest kinds of all scenes
    // first): listing the items scene by scene, which would let a scene's
    // next step start early, measured 1.6x slower on the 64-scene sweep even
    // for a single step; and the number of items of every scene
    std::vector<int> count(b->hs.size(), 0);
    for (const int4& v : all) ++count[static_cast<unsigned>(v.x) >> 16];
    if ((rc = batch_upload(b, &b->pscene_items[t], count.data(), count.size() * sizeof(int)))) return rc;
    b->pitems[t] = b->items[t];  // shared, freed once
  }
  {
    std::vector<unsigned> zero(1 + b->hs.size(), 0u);
    if ((rc = batch_upload(b, reinterpret_cast<void**>(&b->queue), zero.data(), zero.size() * sizeof(unsigned)))) return rc;
  }
  b->persist_ok = true;
  for (xfb_handle* h : b->hs) {
    const Compiled& c = h->c;
    if (h->ade_deferred || c.nf_on || c.td_on || !c.probes.empty() || !c.movies.empty()) b->persist_ok = false;
  }
  if (b->launch_req == XFB_BATCH_PERSISTENT && !b->persist_ok)
    return batch_err(b, XFB_ERR_INVALID, "persistent batch launches need scenes without monitors or a separate ADE pass");
  cudaError_t e = cudaMalloc(&b->t_dev, sizeof(long long));
  if (e != cudaSuccess) return batch_err(b, XFB_ERR_OOM, "cudaMalloc (batch step counter)");
  e = cudaMemsetAsync(b->t_dev, 0, sizeof(long long), b->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
  if (e != cudaSuccess) return batch_err(b, XFB_ERR_CUDA, cudaGetErrorString(e));
  return XFB_OK;
}

template <typename T, int R, int NWM>
void batch_step3(xfb_batch* b, int t, TimeP tp, int parity) {
  constexpr int NS = 4;
  using S = StepCfg<T, R, NWM, NS>;
  static bool attr_set[64] = {};
  if (!attr_set[b->device & 63]) {
    cudaFuncSetAttribute(k_step3_batch<T, R, NWM, NS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         static_cast<int>(S::bytes));
    attr_set[b->device & 63] = true;
  }
  k_step3_batch<T, R, NWM, NS><<<b->n_items[t], S::NT, S::bytes, b->stream>>>(
      static_cast<const BatchScene<T>*>(b->scenes), static_cast<const BatchMaps*>(b->maps),
      static_cast<const int4*>(b->items[t]), tp, parity, t, b->err_dev);
}

// n steps of every scene in one persistent launch (k_step3_persist): as many
// CTAs as fit on the device at once, each taking items from the queue.
template <typename T, int R, int NWM>
void batch_persist3(xfb_batch* b, int t, TimeP tp, int parity, int n) {
  constexpr int NS = 4;
  using S = StepCfg<T, R, NWM, NS>;
  static bool attr_set[64] = {};
  static int per_sm[64] = {};
  const int dev = b->device & 63;
  if (!attr_set[dev]) {
    cudaFuncSetAttribute(k_step3_persist<T, R, NWM, NS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         static_cast<int>(S::bytes));
    int blocks = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, k_step3_persist<T, R, NWM, NS>, S::NT, S::bytes);
    per_sm[dev] = std::max(1, blocks);
    attr_set[dev] = true;
  }
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device);
  const long long tickets = static_cast<long long>(n) * b->n_items[t];
  const int grid = static_cast<int>(std::min<long long>(tickets, static_cast<long long>(sms) * per_sm[dev]));
  cudaMemsetAsync(b->queue, 0, (1 + b->hs.size()) * sizeof(unsigned), b->stream);
  k_step3_persist<T, R, NWM, NS><<<grid, S::NT, S::bytes, b->stream>>>(
      static_cast<const BatchScene<T>*>(b->scenes), static_cast<const BatchMaps*>(b->maps),
      static_cast<const int4*>(b->pitems[t]), b->n_items[t], static_cast<const int*>(b->pscene_items[t]), tp, parity, n,
      t, b->queue, b->err_dev);
}

// One step of every scene: the one-sweep kernel over all work items,
// deferred ADE passes, monitors (the TFSF incident tables were computed when
// each handle was initialised).
template <typename T>
void batch_enqueue_step(xfb_batch* b, int off, int t) {
  TimeP tp{b->t_dev, off};
  const int parity = static_cast<int>((b->step + off) & 1);
  if (b->lines_work > 0) {  // the TFSF line values of every scene for this step
    const int bx = static_cast<int>(std::min<long long>((b->lines_work + 255) / 256, 64));
    k_tfsf_lines_batch<T><<<dim3(bx, static_cast<unsigned>(b->hs.size())), 256, 0, b->stream>>>(
        static_cast<const BatchScene<T>*>(b->scenes), tp);
  }
  if (b->n_items[t]) {
    if (t == 0) batch_step3<T, kStepTiles[0].r, kStepTiles[0].nwm>(b, 0, tp, parity);
    else if (t == 1) batch_step3<T, kStepTiles[1].r, kStepTiles[1].nwm>(b, 1, tp, parity);
    else batch_step3<T, kStepTiles[2].r, kStepTiles[2].nwm>(b, 2, tp, parity);
  }
  for (xfb_handle* h : b->hs) {
    const Compiled& c = h->c;
    if (h->ade_deferred) launch_ade<T>(h, parity, b->stream);
    if (c.nf_on || c.td_on || !c.probes.empty() || !c.movies.empty()) enqueue_records<T>(h, parity, tp, b->stream, nullptr);
  }
}

template <typename T>
int batch_chunk(xfb_batch* b, int n, int t, bool graph, int launch) {
  auto enqueue = [&]() {
    if (launch == XFB_BATCH_PERSISTENT) {
      if (b->n_items[t]) {
        TimeP tp{b->t_dev, 0};
        const int parity = static_cast<int>(b->step & 1);
        if (t == 0) batch_persist3<T, kStepTiles[0].r, kStepTiles[0].nwm>(b, 0, tp, parity, n);
        else if (t == 1) batch_persist3<T, kStepTiles[1].r, kStepTiles[1].nwm>(b, 1, tp, parity, n);
        else batch_persist3<T, kStepTiles[2].r, kStepTiles[2].nwm>(b, 2, tp, parity, n);
      }
    } else {
      for (int q = 0; q < n; ++q) batch_enqueue_step<T>(b, q, t);
    }
    k_bump<<<1, 1, 0, b->stream>>>(b->t_dev, n);
  };
  cudaError_t e = cudaSuccess;
  if (graph) {
    const int key = ((n * 2 + static_cast<int>(b->step & 1)) * 3 + launch) * kStepTileCount + t;
    auto it = b->graphs.find(key);
    if (it == b->graphs.end()) {
      cudaGraph_t g;
      e = cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal);
      if (e != cudaSuccess) return batch_err(b, XFB_ERR_CUDA, std::string("capture: ") + cudaGetErrorString(e));
      enqueue();
      e = cudaStreamEndCapture(b->stream, &g);
      if (e != cudaSuccess) return batch_err(b, XFB_ERR_CUDA, std::string("capture: ") + cudaGetErrorString(e));
      cudaGraphExec_t ex;
      e = cudaGraphInstantiate(&ex, g, 0);
      cudaGraphDestroy(g);
      if (e != cudaSuccess) return batch_err(b, XFB_ERR_CUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e));
      it = b->graphs.emplace(key, ex).first;
    }
    e = cudaGraphLaunch(it->second, b->stream);
  } else {
    enqueue();
    e = cudaGetLastError();
  }
  if (e != cudaSuccess) return batch_err(b, XFB_ERR_CUDA, cudaGetErrorString(e));
  b->step += n;
  for (xfb_handle* h : b->hs) h->step += n;
  return XFB_OK;
}

// Advance every scene n steps.  With tile autotuning on, the first call
// steps once with each tile configuration (untimed: the first launch of a
// kernel loads its module), then times a few steps with each (results do
// not depend on the tile) and keeps the fastest for the rest of the run.
// Autotuned tile configurations of batches, per (device name, precision,
// scene sizes), for the life of the process and, when the environment names
// a file in XFB_AUTOTUNE_CACHE, across processes (one "key tile" line each).
inline std::string tile_cache_key(const xfb_batch* b) {
  cudaDeviceProp prop{};
  cudaGetDeviceProperties(&prop, b->device);
  std::string k = std::string(prop.name) + "|" + (b->prec == XFB_FP64 ? "fp64" : "fp32");
  for (const xfb_handle* h : b->hs)
    k += "|" + std::to_string(h->c.nx) + "x" + std::to_string(h->c.ny) + "x" + std::to_string(h->c.nz);
  for (char& ch : k)
    if (ch == ' ') ch = '_';
  return k;
}

inline std::map<std::string, int>& tile_cache() {
  static std::map<std::string, int> m;
  return m;
}
inline std::mutex& tile_cache_mutex() {
  static std::mutex mu;
  return mu;
}

inline int tile_cache_get(const std::string& key) {
  std::lock_guard<std::mutex> lock(tile_cache_mutex());
  auto& m = tile_cache();
  if (m.count(key)) return m[key];
  if (const char* path = std::getenv("XFB_AUTOTUNE_CACHE")) {
    std::FILE* f = std::fopen(path, "r");
    if (f) {
      char line[4096];
      while (std::fgets(line, sizeof(line), f)) {
        std::string s(line);
        const size_t sp = s.rfind(' ');
        if (sp != std::string::npos && s.substr(0, sp) == key) m[key] = std::atoi(s.c_str() + sp + 1);
      }
      std::fclose(f);
    }
  }
  return m.count(key) ? m[key] : -1;
}

inline void tile_cache_put(const std::string& key, int tile) {
  std::lock_guard<std::mutex> lock(tile_cache_mutex());
  tile_cache()[key] = tile;
  if (const char* path = std::getenv("XFB_AUTOTUNE_CACHE")) {
    std::FILE* f = std::fopen(path, "a");
    if (f) {
      std::fprintf(f, "%s %d\n", key.c_str(), tile);
      std::fclose(f);
    }
  }
}

template <typename T>
int batch_run(xfb_batch* b, long long n) {
  int rc;
  // candidate launch forms: per step always, persistent when the scenes allow
  std::vector<int> forms;
  if (b->launch_req != XFB_BATCH_PERSISTENT) forms.push_back(XFB_BATCH_PER_STEP);
  if (b->launch_req != XFB_BATCH_PER_STEP && b->persist_ok) forms.push_back(XFB_BATCH_PERSISTENT);
  if (b->tile < 0 && b->tile_req == 0 && b->launch_req == XFB_BATCH_AUTO) {  // an earlier autotune of the same scenes
    const int v = tile_cache_get(tile_cache_key(b));
    const int t = v % kStepTileCount, f = v / kStepTileCount;
    if (v >= 0 && (f == XFB_BATCH_PER_STEP || (f == XFB_BATCH_PERSISTENT && b->persist_ok))) {
      b->tile = t;
      b->launch = f;
    }
  }
  if (b->tile < 0) {
    std::vector<int> tiles;
    for (int t = 0; t < kStepTileCount; ++t)
      if (b->tile_req == 0 || kStepTileRows[t] == b->tile_req) tiles.push_back(t);
    // too few steps to time every (tile, form): the tiles alone in the first form
    if (forms.size() > 1 && n < 2 * static_cast<long long>(tiles.size() * forms.size())) forms.resize(1);
    const long long cands = static_cast<long long>(tiles.size() * forms.size());
    if (cands == 1 || n < 2 * cands) {  // nothing to choose, or too few steps to time: 16-row tiles, first form
      b->tile = tiles.size() == 1 ? tiles[0] : 1;
      b->launch = forms[0];
    } else {
      // one untimed step per (tile, form) (the first launch of a kernel
      // loads its module), then a few timed steps per (tile, form); keep the
      // fastest
      for (int f : forms)
        for (int t : tiles)
          if ((rc = batch_chunk<T>(b, 1, t, false, f))) return rc;
      n -= cands;
      const int probe = static_cast<int>(std::min<long long>(4, n / cands));
      cudaEvent_t ev[2];
      cudaEventCreate(&ev[0]);
      cudaEventCreate(&ev[1]);
      rc = XFB_OK;
      float best = 0.0f;
      for (int f : forms)
        for (int t : tiles) {
          if (rc) break;
          float ms = 0.0f;
          cudaEventRecord(ev[0], b->stream);
          if ((rc = batch_chunk<T>(b, probe, t, false, f))) break;
          cudaEventRecord(ev[1], b->stream);
          cudaError_t e = cudaEventSynchronize(ev[1]);
          if (e != cudaSuccess) rc = batch_err(b, XFB_ERR_CUDA, cudaGetErrorString(e));
          else cudaEventElapsedTime(&ms, ev[0], ev[1]);
          n -= probe;
          if (!rc && (b->tile < 0 || ms < best)) {
            best = ms;
            b->tile = t;
            b->launch = f;
          }
        }
      cudaEventDestroy(ev[0]);
      cudaEventDestroy(ev[1]);
      if (rc) return rc;
      if (b->launch_req == XFB_BATCH_AUTO && b->tile_req == 0)
        tile_cache_put(tile_cache_key(b), b->tile + kStepTileCount * b->launch);
    }
  }
  if (b->launch < 0) b->launch = forms[0];
  while (n > 0) {
    const int chunk = static_cast<int>(std::min<long long>(n, b->graph_steps));
    if ((rc = batch_chunk<T>(b, chunk, b->tile, true, b->launch))) return rc;
    n -= chunk;
  }
  return XFB_OK;
}

}  // namespace xfb

#define XFB_INSTANTIATE_ENGINE(T)                                                          \
  namespace xfb {                                                                          \
  template int init_device<T>(xfb_handle*);                                                \
  template int run_steps<T>(xfb_handle*, long long);                                       \
  template int slab_update<T>(xfb_handle*);                                                \
  template int slab_record<T>(xfb_handle*);                                                \
  template int profile_steps<T>(xfb_handle*, long long, double*, long long*);              \
  template int read_field_t<T>(xfb_handle*, int, double*);                                 \
  template int read_bytes_t<T>(xfb_handle*, void*, const void*, size_t);                   \
  template int write_field_t<T>(xfb_handle*, int, const double*);                          \
  template void launch_nonfinite<T>(xfb_handle*);                                          \
  template int batch_init<T>(xfb_batch*);                                                  \
  template int batch_run<T>(xfb_batch*, long long);                                        \
  }
