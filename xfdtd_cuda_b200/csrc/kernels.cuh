// Device kernels of the B200 FDTD engine.
//
// One time step on the device (3-D):
//   k_h3   H half-step: Yee update of Hx,Hy,Hz + TFSF H correction + CPML psi
//          (reference: BasicUpdator::updateH, src/include/updator/basic_updator/
//          basic_updator.cuh:16-32; TFSFCorrector3DAgency::correctH,
//          src/waveform_source/tfsf/tfsf_corrector.cu:237-271; PMLCorrector<xyz>::
//          correctH, src/boundary/pml_corrector.cu:180-270)
//   (TFSF 1-D auxiliary grid: k_aux_table computes the incident E/H of every
//          step once at set-up, in FP64, as the reference's host set-up inside
//          XFDTD_CORE precomputes its incident tables)
//   k_e3   E half-step: Yee / ADE update + TFSF E correction + CPML psi
//          (BasicUpdator3D::updateE, src/updator/basic_updator/basic_updator_3d.cu:10-34;
//          TemplateADEUpdateScheme::updateE, src/include/updator/ade_updator/
//          template_ade_update_scheme.cuh:17-85; correctE of the TFSF/PML correctors)
//   k_nf2ff running DFT of the NF2FF surface currents
//          (src/nf2ff/frequency_domain/nf2ff_frequency_domain.data.cu:80-232)
//   k_probe / k_movie monitors (src/monitor/movie_monitor.cu:17-46)
//
// Arithmetic order.  Every update, correction and accumulation evaluates its
// terms in the reference's order (eNext/hNext, update_scheme.cuh:27-63; the
// corrector list TFSF -> PML x -> PML y -> PML z, src/simulation/simulation_hd.cu:
// 124-160; TFSF faces in agency launch order) and the library is compiled with
// --fmad=false, so the FP64 build reproduces the CPU restatement bit for bit.
#pragma once

#include <cstdint>

namespace xfb {

enum { kAdeNone = 0, kAdeDebye = 1, kAdeDrude = 2, kAdeMLorentz = 3 };

template <typename T>
struct GridP {
  int nx, ny, nz;
  long long sx, sy;  // element strides of i and j (k stride 1)
  T* ex; T* ey; T* ez; T* hx; T* hy; T* hz;
  const uint8_t* mid;  // material id, same strides as the fields
  const T* lut;        // [n_mat][18]
};

template <typename T>
struct PmlP {
  int L[6];           // thickness XN XP YN YP ZN ZP
  const T* ae[3]; const T* be[3]; const T* ah[3]; const T* bh[3];
  // psi slabs.  x: [Lx][ny+1][nzp] (strides sx, sy); y: [nx+1][Ly][nzp]
  // (strides ysx, sy); z: [nx+1][ny+1][Lz] (strides zsx, zsy).
  T* ey_x; T* ez_x; T* ez_y; T* ex_y; T* ex_z; T* ey_z;
  T* hy_x; T* hz_x; T* hz_y; T* hx_y; T* hx_z; T* hy_z;
  long long ysx, zsx, zsy;
};

struct TfsfP {
  int on;
  int is, ie, js, je, ks, ke;
  const double* pi0; const double* pi1; const double* pi2;  // projections at nodes
  const double* ph0; const double* ph1; const double* ph2;  // projections at half nodes
  double tre[3], trh[3], ca[3], cb[3];
  const double* e_tab;  // [total_steps + 1][nl + 1]: row t = E incident at t*dt
  const double* h_tab;  // [total_steps][nl]: row t = H incident at (t+1/2)*dt
  int nl;
  const double* e_aux;  // resolved by tfsf_at_step: the rows of the current step
  const double* h_aux;
};

// Resolve the rows of the auxiliary-grid tables of step t.
__device__ __forceinline__ TfsfP tfsf_at_step(TfsfP s, long long t) {
  s.e_aux = s.e_tab + t * (s.nl + 1);
  s.h_aux = s.h_tab + t * s.nl;
  return s;
}

template <typename T>
struct AdeP {
  int kind, P;
  int b0, b1, b2, b3, b4, b5;  // box i0 i1 j0 j1 k0 k1 (cells)
  long long bsx, bsy, bn;      // box strides and elements per (component, pole)
  const T* mat;   // [n_mat][3] dispersive, ceep, cejsum
  const T* pole;  // [n_mat][P][7] cjj cjjp cjen cje cjep cjsj cjsjp
  T* J; T* Jp; T* Ep;  // [3][P][bn], [3][P][bn], [3][bn]
};

struct TimeP {
  const long long* t;  // device step counter at the start of the captured chunk
  int off;             // step offset inside the chunk
};

__device__ __forceinline__ long long cur_step(const TimeP& tp) { return *tp.t + tp.off; }

// ---------------------------------------------------------------------------
// TFSF incident field (FP64), the reference TFSFCorrector::{e,h}{x,y,z}Inc
// (src/waveform_source/tfsf/tfsf_corrector.cu:18-130).
__device__ __forceinline__ double aux_lerp(const double* a, double proj) {
  const long long idx = static_cast<long long>(proj);
  const double w = proj - static_cast<double>(idx);
  return (1 - w) * a[idx] + w * a[idx + 1];
}
__device__ __forceinline__ double ex_inc(const TfsfP& s, int i, int j, int k) {
  const double p = s.ph0[i - s.is + 1] + s.pi1[j - s.js] + s.pi2[k - s.ks];
  return s.tre[0] * aux_lerp(s.e_aux, p);
}
__device__ __forceinline__ double ey_inc(const TfsfP& s, int i, int j, int k) {
  const double p = s.pi0[i - s.is] + s.ph1[j - s.js + 1] + s.pi2[k - s.ks];
  return s.tre[1] * aux_lerp(s.e_aux, p);
}
__device__ __forceinline__ double ez_inc(const TfsfP& s, int i, int j, int k) {
  const double p = s.pi0[i - s.is] + s.pi1[j - s.js] + s.ph2[k - s.ks + 1];
  return s.tre[2] * aux_lerp(s.e_aux, p);
}
__device__ __forceinline__ double hx_inc(const TfsfP& s, int i, int j, int k) {
  const double p = s.pi0[i - s.is] + s.ph1[j - s.js + 1] + s.ph2[k - s.ks + 1] - 0.5;
  return s.trh[0] * aux_lerp(s.h_aux, p);
}
__device__ __forceinline__ double hy_inc(const TfsfP& s, int i, int j, int k) {
  const double p = s.ph0[i - s.is + 1] + s.pi1[j - s.js] + s.ph2[k - s.ks + 1] - 0.5;
  return s.trh[1] * aux_lerp(s.h_aux, p);
}
__device__ __forceinline__ double hz_inc(const TfsfP& s, int i, int j, int k) {
  const double p = s.ph0[i - s.is + 1] + s.ph1[j - s.js + 1] + s.pi2[k - s.ks] - 0.5;
  return s.trh[2] * aux_lerp(s.h_aux, p);
}

// The incident fields of a step's tables (projection arrays, the step's
// auxiliary rows) behind one interface for the correction routines.
struct IncTables {
  const TfsfP& s;
  __device__ __forceinline__ double ex(int i, int j, int k) const { return ex_inc(s, i, j, k); }
  __device__ __forceinline__ double ey(int i, int j, int k) const { return ey_inc(s, i, j, k); }
  __device__ __forceinline__ double ez(int i, int j, int k) const { return ez_inc(s, i, j, k); }
  __device__ __forceinline__ double hx(int i, int j, int k) const { return hx_inc(s, i, j, k); }
  __device__ __forceinline__ double hy(int i, int j, int k) const { return hy_inc(s, i, j, k); }
  __device__ __forceinline__ double hz(int i, int j, int k) const { return hz_inc(s, i, j, k); }
};

// field += inc * coefficient (tfsf_corrector.cuh:137,151,166), in double.
template <typename T>
__device__ __forceinline__ void add_inc(T& f, double inc, double coef) {
  f = static_cast<T>(static_cast<double>(f) + inc * coef);
}

// ---------------------------------------------------------------------------
// CPML slab lookup: slab plane index of coordinate q on an axis with N/P
// layers Ln/Lp and n cells, or -1.
__device__ __forceinline__ int slab(int q, int n, int Ln, int Lp) {
  if (q < Ln) return q;
  if (q >= n - Lp) return Ln + q - (n - Lp);
  return -1;
}

// ---------------------------------------------------------------------------
// H half-step, 3-D.  Block (TK, TJ) threads own a (j, k) tile and march along i
// (the slowest-stride axis) over [i0, i1): E values of plane i+1 are carried in
// registers to the next plane, so every E element is fetched from memory once
// per plane; k and j neighbours come from lines the block already holds in L1.
template <typename T>
__global__ void k_h3(GridP<T> g, PmlP<T> pm, TfsfP tf_in, TimeP tp, int i_chunk) {
  const TfsfP tf = tfsf_at_step(tf_in, cur_step(tp));
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (k >= g.nz || j >= g.ny) return;
  const int i0 = blockIdx.z * i_chunk;
  const int i1 = min(g.nx, i0 + i_chunk);
  if (i0 >= i1) return;
  const long long sx = g.sx, sy = g.sy;
  long long idx = static_cast<long long>(i0) * sx + static_cast<long long>(j) * sy + k;
  T ey_c = g.ey[idx], ez_c = g.ez[idx];
  const int sy_pml = slab(j, g.ny, pm.L[2], pm.L[3]);
  const int sz_pml = slab(k, g.nz, pm.L[4], pm.L[5]);
  for (int i = i0; i < i1; ++i, idx += sx) {
    const T ey_n = g.ey[idx + sx];
    const T ez_n = g.ez[idx + sx];
    const T ex_c = g.ex[idx];
    const T ex_k1 = g.ex[idx + 1];
    const T ex_j1 = g.ex[idx + sy];
    const T ey_k1 = g.ey[idx + 1];
    const T ez_j1 = g.ez[idx + sy];
    const T* c = g.lut + 18 * static_cast<int>(g.mid[idx]);
    // hNext: chch*hc + chcea*(ea_q - ea_p) + chceb*(eb_q - eb_p)
    const T d_hx_a = ey_k1 - ey_c;  // Hx: Ea = Ey along z
    const T d_hx_b = ez_j1 - ez_c;  // Hx: Eb = Ez along y
    const T d_hy_a = ez_n - ez_c;   // Hy: Ea = Ez along x
    const T d_hy_b = ex_k1 - ex_c;  // Hy: Eb = Ex along z
    const T d_hz_a = ex_j1 - ex_c;  // Hz: Ea = Ex along y
    const T d_hz_b = ey_n - ey_c;   // Hz: Eb = Ey along x
    T hxv = c[9] * g.hx[idx] + c[10] * d_hx_a + c[11] * d_hx_b;
    T hyv = c[12] * g.hy[idx] + c[13] * d_hy_a + c[14] * d_hy_b;
    T hzv = c[15] * g.hz[idx] + c[16] * d_hz_a + c[17] * d_hz_b;

    if (tf.on) {
      // Corrections on the scattered-field side of the TF box, in the agency
      // order XN-Z XP-Z YN-Z YP-Z ZN-X ZP-X YN-X YP-X ZN-Y ZP-Y XN-Y XP-Y.
      const bool iin = i >= tf.is && i <= tf.ie, jin = j >= tf.js && j <= tf.je, kin = k >= tf.ks && k <= tf.ke;
      // Hz: XN (i = is-1), XP (i = ie): j in [js,je), k in [ks,ke]
      if (jin && j < tf.je && kin) {
        if (i == tf.is - 1) add_inc(hzv, ey_inc(tf, tf.is, j, k), tf.cb[0]);
        if (i == tf.ie) add_inc(hzv, ey_inc(tf, tf.ie, j, k), -tf.cb[0]);
      }
      // Hz: YN (j = js-1), YP (j = je): i in [is,ie), k in [ks,ke]
      if (iin && i < tf.ie && kin) {
        if (j == tf.js - 1) add_inc(hzv, ex_inc(tf, i, tf.js, k), -tf.cb[1]);
        if (j == tf.je) add_inc(hzv, ex_inc(tf, i, tf.je, k), tf.cb[1]);
      }
      // Hx: ZN (k = ks-1), ZP (k = ke): i in [is,ie], j in [js,je)
      if (iin && jin && j < tf.je) {
        if (k == tf.ks - 1) add_inc(hxv, ey_inc(tf, i, j, tf.ks), -tf.cb[2]);
        if (k == tf.ke) add_inc(hxv, ey_inc(tf, i, j, tf.ke), tf.cb[2]);
      }
      // Hx: YN, YP: i in [is,ie], k in [ks,ke)
      if (iin && kin && k < tf.ke) {
        if (j == tf.js - 1) add_inc(hxv, ez_inc(tf, i, tf.js, k), tf.cb[1]);
        if (j == tf.je) add_inc(hxv, ez_inc(tf, i, tf.je, k), -tf.cb[1]);
      }
      // Hy: ZN, ZP: i in [is,ie), j in [js,je]
      if (iin && i < tf.ie && jin) {
        if (k == tf.ks - 1) add_inc(hyv, ex_inc(tf, i, j, tf.ks), tf.cb[2]);
        if (k == tf.ke) add_inc(hyv, ex_inc(tf, i, j, tf.ke), -tf.cb[2]);
      }
      // Hy: XN, XP: j in [js,je], k in [ks,ke)
      if (jin && kin && k < tf.ke) {
        if (i == tf.is - 1) add_inc(hyv, ez_inc(tf, tf.is, j, k), -tf.cb[0]);
        if (i == tf.ie) add_inc(hyv, ez_inc(tf, tf.ie, j, k), tf.cb[0]);
      }
    }
    // CPML: psi = b psi + a (E(c+1) - E(c)); H += c_psi psi  (pml_corrector.cu:9-48)
    const int sx_pml = slab(i, g.nx, pm.L[0], pm.L[1]);
    if (sx_pml >= 0) {
      const long long p = sx_pml * sx + static_cast<long long>(j) * sy + k;
      const T a = pm.ah[0][i], b = pm.bh[0][i];
      T py = b * pm.hy_x[p] + a * d_hy_a;  // Hy (H_a of X) from Ez
      pm.hy_x[p] = py;
      hyv = hyv + c[13] * py;
      T pz = b * pm.hz_x[p] + a * d_hz_b;  // Hz (H_b of X) from Ey
      pm.hz_x[p] = pz;
      hzv = hzv + c[17] * pz;
    }
    if (sy_pml >= 0) {
      const long long p = static_cast<long long>(i) * pm.ysx + sy_pml * sy + k;
      const T a = pm.ah[1][j], b = pm.bh[1][j];
      T pz = b * pm.hz_y[p] + a * d_hz_a;  // Hz (H_a of Y) from Ex
      pm.hz_y[p] = pz;
      hzv = hzv + c[16] * pz;
      T px = b * pm.hx_y[p] + a * d_hx_b;  // Hx (H_b of Y) from Ez
      pm.hx_y[p] = px;
      hxv = hxv + c[11] * px;
    }
    if (sz_pml >= 0) {
      const long long p = static_cast<long long>(i) * pm.zsx + static_cast<long long>(j) * pm.zsy + sz_pml;
      const T a = pm.ah[2][k], b = pm.bh[2][k];
      T px = b * pm.hx_z[p] + a * d_hx_a;  // Hx (H_a of Z) from Ey
      pm.hx_z[p] = px;
      hxv = hxv + c[10] * px;
      T py = b * pm.hy_z[p] + a * d_hy_b;  // Hy (H_b of Z) from Ex
      pm.hy_z[p] = py;
      hyv = hyv + c[14] * py;
    }
    g.hx[idx] = hxv;
    g.hy[idx] = hyv;
    g.hz[idx] = hzv;
    ey_c = ey_n;
    ez_c = ez_n;
  }
}

// ADE update of one E component at a dispersive cell (template_ade_update_scheme.cuh:70-83
// with the Debye / Drude / M-Lorentz recursions of src/updator/ade_updator/*.cu).
// `plain` = eNext(...); returns E^{n+1}.  The J recursion sees E before the
// TFSF/CPML corrections, as in the reference (correctE runs after updateE).
template <typename T>
__device__ __forceinline__ T ade_e(const AdeP<T>& a, int comp, long long bi, int m, T e_cur, T plain) {
  const T* am = a.mat + 3 * m;
  const T* ap = a.pole + static_cast<long long>(m) * a.P * 7;
  T* J = a.J + static_cast<long long>(comp) * a.P * a.bn + bi;
  if (a.kind == kAdeMLorentz) {
    T* Jp = a.Jp + static_cast<long long>(comp) * a.P * a.bn + bi;
    T* Ep = a.Ep + static_cast<long long>(comp) * a.bn + bi;
    T jsum = 0;
    for (int p = 0; p < a.P; ++p) jsum = jsum + (ap[7 * p + 5] * J[p * a.bn] + ap[7 * p + 6] * Jp[p * a.bn]);
    const T e_prev = *Ep;
    const T e_new = am[1] * e_prev + plain + am[2] * jsum;
    for (int p = 0; p < a.P; ++p) {
      const T* q = ap + 7 * p;
      const T jv = J[p * a.bn], jpv = Jp[p * a.bn];
      const T jn = q[2] * e_new + q[3] * e_cur + q[4] * e_prev + q[0] * jv + q[1] * jpv;
      Jp[p * a.bn] = jv;
      J[p * a.bn] = jn;
    }
    *Ep = e_cur;
    return e_new;
  }
  T jsum = 0;
  for (int p = 0; p < a.P; ++p) jsum = jsum + ap[7 * p + 5] * J[p * a.bn];
  const T e_new = plain + am[2] * jsum;
  for (int p = 0; p < a.P; ++p) {
    const T* q = ap + 7 * p;
    const T jv = J[p * a.bn];
    J[p * a.bn] = (a.kind == kAdeDrude) ? q[0] * jv + q[3] * (e_new + e_cur) : q[0] * jv + q[3] * (e_new - e_cur);
  }
  return e_new;
}

// Deferred ADE update of one dispersive cell of the box after a one-sweep
// step.  The step kernel stored the plain eNext value of every cell in `d`;
// this applies the TemplateADEUpdateScheme::updateE recursion with E^n from
// `s` (k_ade_box: one thread per box cell, k fastest; k_ade_runs: one thread
// per dispersive cell).  All inputs of a cell (E^n, plain values, J, J_prev,
// E_prev of the three components) are loaded before any update, so the loads
// overlap; the arithmetic and its order are those of ade_e.  Valid only when
// no dispersive cell also takes a TFSF or CPML correction, which the
// reference applies after the ADE update.
template <typename T>
__device__ __forceinline__ void ade_box_cell(const GridP<T>& s, const GridP<T>& d, const AdeP<T>& ad, int i, int j,
                                             int k, long long idx, int m) {
  constexpr int MP = 4;  // XFB_MAX_POLES
  const long long bi = static_cast<long long>(i - ad.b0) * ad.bsx + static_cast<long long>(j - ad.b2) * ad.bsy + (k - ad.b4);
  const bool upd[3] = {j > 0 && k > 0, i > 0 && k > 0, i > 0 && j > 0};
  T* dd[3] = {d.ex, d.ey, d.ez};
  const T* ss[3] = {s.ex, s.ey, s.ez};
  const bool ml = ad.kind == kAdeMLorentz;
  const int P = ad.P;
  T ec[3], pl[3], J[3][MP], Jp[3][MP], Ep[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    ec[c] = ss[c][idx];
    pl[c] = dd[c][idx];
    Ep[c] = ml ? ad.Ep[c * ad.bn + bi] : T(0);
#pragma unroll
    for (int p = 0; p < MP; ++p) {
      const long long o = (static_cast<long long>(c) * P + p) * ad.bn + bi;
      J[c][p] = p < P ? ad.J[o] : T(0);
      Jp[c][p] = (p < P && ml) ? ad.Jp[o] : T(0);
    }
  }
  const T* am = ad.mat + 3 * m;
  const T* ap = ad.pole + static_cast<long long>(m) * P * 7;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    if (!upd[c]) continue;
    T e_new;
    if (ml) {
      T jsum = 0;
#pragma unroll
      for (int p = 0; p < MP; ++p)
        if (p < P) jsum = jsum + (ap[7 * p + 5] * J[c][p] + ap[7 * p + 6] * Jp[c][p]);
      e_new = am[1] * Ep[c] + pl[c] + am[2] * jsum;
#pragma unroll
      for (int p = 0; p < MP; ++p)
        if (p < P) {
          const T* q = ap + 7 * p;
          const long long o = (static_cast<long long>(c) * P + p) * ad.bn + bi;
          const T jn = q[2] * e_new + q[3] * ec[c] + q[4] * Ep[c] + q[0] * J[c][p] + q[1] * Jp[c][p];
          ad.Jp[o] = J[c][p];
          ad.J[o] = jn;
        }
      ad.Ep[c * ad.bn + bi] = ec[c];
    } else {
      T jsum = 0;
#pragma unroll
      for (int p = 0; p < MP; ++p)
        if (p < P) jsum = jsum + ap[7 * p + 5] * J[c][p];
      e_new = pl[c] + am[2] * jsum;
#pragma unroll
      for (int p = 0; p < MP; ++p)
        if (p < P) {
          const T* q = ap + 7 * p;
          const long long o = (static_cast<long long>(c) * P + p) * ad.bn + bi;
          ad.J[o] = (ad.kind == kAdeDrude) ? q[0] * J[c][p] + q[3] * (e_new + ec[c]) : q[0] * J[c][p] + q[3] * (e_new - ec[c]);
        }
    }
    dd[c][idx] = e_new;
  }
}

template <typename T>
__global__ void k_ade_box(GridP<T> s, GridP<T> d, AdeP<T> ad, const uint8_t* disp) {
  const int k = ad.b4 + blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= ad.b5) return;
  const int j = ad.b2 + blockIdx.y, i = ad.b0 + blockIdx.z;
  const long long idx = static_cast<long long>(i) * s.sx + static_cast<long long>(j) * s.sy + k;
  const int m = s.mid[idx];
  if (!disp[m]) return;
  ade_box_cell(s, d, ad, i, j, k, idx, m);
}

// The same update over a list of runs of dispersive cells (one warp per run
// of at most 32 cells inside one 32-aligned k segment, so each warp's field
// accesses stay inside one 128-byte line per array): run q = {i | j << 16,
// kb | lo << 16 | hi << 24}, cells k = kb + lane for lo <= lane < hi.  FP32:
// 64 registers, so 8 CTAs (32 warps) fit an SM (the pass is load-latency
// bound); FP64 keeps its own register count (it would spill at 64).
template <typename T>
__global__ void __launch_bounds__(128, sizeof(T) == 4 ? 8 : 1) k_ade_runs(GridP<T> s, GridP<T> d, AdeP<T> ad, const int2* runs, int n_runs) {
  const int q = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (q >= n_runs) return;
  const int lane = threadIdx.x & 31;
  const int2 r = runs[q];
  const int lo = (r.y >> 16) & 0xff, hi = static_cast<int>(static_cast<unsigned>(r.y) >> 24);
  if (lane < lo || lane >= hi) return;
  const int i = r.x & 0xffff, j = static_cast<int>(static_cast<unsigned>(r.x) >> 16), k = (r.y & 0xffff) + lane;
  const long long idx = static_cast<long long>(i) * s.sx + static_cast<long long>(j) * s.sy + k;
  ade_box_cell(s, d, ad, i, j, k, idx, s.mid[idx]);
}

// E half-step, 3-D.  Same tiling as k_h3; H values of plane i are carried to
// plane i+1 as its i-1 neighbours.
template <typename T>
__global__ void k_e3(GridP<T> g, PmlP<T> pm, TfsfP tf_in, AdeP<T> ad, TimeP tp, int i_chunk) {
  const TfsfP tf = tfsf_at_step(tf_in, cur_step(tp));
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (k >= g.nz || j >= g.ny) return;
  const int i0 = blockIdx.z * i_chunk;
  const int i1 = min(g.nx, i0 + i_chunk);
  if (i0 >= i1) return;
  const long long sx = g.sx, sy = g.sy;
  long long idx = static_cast<long long>(i0) * sx + static_cast<long long>(j) * sy + k;
  T hy_p = g.hy[idx - sx], hz_p = g.hz[idx - sx];
  const int sy_pml = slab(j, g.ny, pm.L[2], pm.L[3]);
  const int sz_pml = slab(k, g.nz, pm.L[4], pm.L[5]);
  const bool jpos = j > 0, kpos = k > 0;
  for (int i = i0; i < i1; ++i, idx += sx) {
    const T hx_c = g.hx[idx], hy_c = g.hy[idx], hz_c = g.hz[idx];
    const T hx_km = g.hx[idx - 1], hx_jm = g.hx[idx - sy];
    const T hy_km = g.hy[idx - 1];
    const T hz_jm = g.hz[idx - sy];
    const int m = g.mid[idx];
    const T* c = g.lut + 18 * m;
    // eNext: cece*ec + cecha*(ha_p - ha_q) + cechb*(hb_p - hb_q)
    const T d_ex_a = hy_c - hy_km;  // Ex: Ha = Hy along z
    const T d_ex_b = hz_c - hz_jm;  // Ex: Hb = Hz along y
    const T d_ey_a = hz_c - hz_p;   // Ey: Ha = Hz along x
    const T d_ey_b = hx_c - hx_km;  // Ey: Hb = Hx along z
    const T d_ez_a = hx_c - hx_jm;  // Ez: Ha = Hx along y
    const T d_ez_b = hy_c - hy_p;   // Ez: Hb = Hy along x
    const bool ipos = i > 0;
    const bool upd_x = jpos && kpos, upd_y = ipos && kpos, upd_z = ipos && jpos;
    const T ex_o = g.ex[idx], ey_o = g.ey[idx], ez_o = g.ez[idx];
    T exv = c[0] * ex_o + c[1] * d_ex_a + c[2] * d_ex_b;
    T eyv = c[3] * ey_o + c[4] * d_ey_a + c[5] * d_ey_b;
    T ezv = c[6] * ez_o + c[7] * d_ez_a + c[8] * d_ez_b;
    if (ad.kind != kAdeNone && ad.mat[3 * m] != T(0)) {
      const long long bi = static_cast<long long>(i - ad.b0) * ad.bsx + static_cast<long long>(j - ad.b2) * ad.bsy + (k - ad.b4);
      if (upd_x) exv = ade_e(ad, 0, bi, m, ex_o, exv);
      if (upd_y) eyv = ade_e(ad, 1, bi, m, ey_o, eyv);
      if (upd_z) ezv = ade_e(ad, 2, bi, m, ez_o, ezv);
    }
    if (tf.on) {
      const bool iin = i >= tf.is && i <= tf.ie, jin = j >= tf.js && j <= tf.je, kin = k >= tf.ks && k <= tf.ke;
      // agency order: XN-Z XP-Z YN-Z YP-Z ZN-X ZP-X YN-X YP-X ZN-Y ZP-Y XN-Y XP-Y
      // Ez: XN (i = is), XP (i = ie): j in [js,je], k in [ks,ke)
      if (jin && kin && k < tf.ke) {
        if (i == tf.is) add_inc(ezv, hy_inc(tf, tf.is - 1, j, k), -tf.ca[0]);
        if (i == tf.ie) add_inc(ezv, hy_inc(tf, tf.ie, j, k), tf.ca[0]);
      }
      // Ez: YN (j = js), YP (j = je): i in [is,ie], k in [ks,ke)
      if (iin && kin && k < tf.ke) {
        if (j == tf.js) add_inc(ezv, hx_inc(tf, i, tf.js - 1, k), tf.ca[1]);
        if (j == tf.je) add_inc(ezv, hx_inc(tf, i, tf.je, k), -tf.ca[1]);
      }
      // Ex: ZN (k = ks), ZP (k = ke): i in [is,ie), j in [js,je]
      if (iin && i < tf.ie && jin) {
        if (k == tf.ks) add_inc(exv, hy_inc(tf, i, j, tf.ks - 1), tf.ca[2]);
        if (k == tf.ke) add_inc(exv, hy_inc(tf, i, j, tf.ke), -tf.ca[2]);
      }
      // Ex: YN, YP: i in [is,ie), k in [ks,ke]
      if (iin && i < tf.ie && kin) {
        if (j == tf.js) add_inc(exv, hz_inc(tf, i, tf.js - 1, k), -tf.ca[1]);
        if (j == tf.je) add_inc(exv, hz_inc(tf, i, tf.je, k), tf.ca[1]);
      }
      // Ey: ZN, ZP: i in [is,ie], j in [js,je)
      if (iin && jin && j < tf.je) {
        if (k == tf.ks) add_inc(eyv, hx_inc(tf, i, j, tf.ks - 1), -tf.ca[2]);
        if (k == tf.ke) add_inc(eyv, hx_inc(tf, i, j, tf.ke), tf.ca[2]);
      }
      // Ey: XN, XP: j in [js,je), k in [ks,ke]
      if (jin && j < tf.je && kin) {
        if (i == tf.is) add_inc(eyv, hz_inc(tf, tf.is - 1, j, k), tf.ca[0]);
        if (i == tf.ie) add_inc(eyv, hz_inc(tf, tf.ie, j, k), -tf.ca[0]);
      }
    }
    // CPML: psi = b psi + a (H(c) - H(c-1)); E += c_psi psi
    const int sx_pml = slab(i, g.nx, pm.L[0], pm.L[1]);
    if (sx_pml >= 0) {
      const long long p = sx_pml * sx + static_cast<long long>(j) * sy + k;
      const T a = pm.ae[0][i], b = pm.be[0][i];
      if (upd_y) {  // Ey (E_a of X) from Hz
        T ps = b * pm.ey_x[p] + a * d_ey_a;
        pm.ey_x[p] = ps;
        eyv = eyv + c[4] * ps;
      }
      if (upd_z) {  // Ez (E_b of X) from Hy
        T ps = b * pm.ez_x[p] + a * d_ez_b;
        pm.ez_x[p] = ps;
        ezv = ezv + c[8] * ps;
      }
    }
    if (sy_pml >= 0) {
      const long long p = static_cast<long long>(i) * pm.ysx + sy_pml * sy + k;
      const T a = pm.ae[1][j], b = pm.be[1][j];
      if (upd_z) {  // Ez (E_a of Y) from Hx
        T ps = b * pm.ez_y[p] + a * d_ez_a;
        pm.ez_y[p] = ps;
        ezv = ezv + c[7] * ps;
      }
      if (upd_x) {  // Ex (E_b of Y) from Hz
        T ps = b * pm.ex_y[p] + a * d_ex_b;
        pm.ex_y[p] = ps;
        exv = exv + c[2] * ps;
      }
    }
    if (sz_pml >= 0) {
      const long long p = static_cast<long long>(i) * pm.zsx + static_cast<long long>(j) * pm.zsy + sz_pml;
      const T a = pm.ae[2][k], b = pm.be[2][k];
      if (upd_x) {  // Ex (E_a of Z) from Hy
        T ps = b * pm.ex_z[p] + a * d_ex_a;
        pm.ex_z[p] = ps;
        exv = exv + c[1] * ps;
      }
      if (upd_y) {  // Ey (E_b of Z) from Hx
        T ps = b * pm.ey_z[p] + a * d_ey_b;
        pm.ey_z[p] = ps;
        eyv = eyv + c[5] * ps;
      }
    }
    if (upd_x) g.ex[idx] = exv;
    if (upd_y) g.ey[idx] = eyv;
    if (upd_z) g.ez[idx] = ezv;
    hy_p = hy_c;
    hz_p = hz_c;
  }
}

// ---------------------------------------------------------------------------
// 2-D TMz half-steps (reference BasicUpdatorTE, src/updator/basic_updator/
// basic_updator_te.cu:9-20 with the 2-D TFSF agency, tfsf_corrector.cu:155-189).
// Fields: Ez (nx+1, ny+1), Hx (nx+1, ny), Hy (nx, ny+1); idx = i*sx + j.
template <typename T>
__global__ void k_h2(GridP<T> g, PmlP<T> pm, TfsfP tf_in, TimeP tp, int i_chunk) {
  const TfsfP tf = tfsf_at_step(tf_in, cur_step(tp));
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= g.ny) return;
  const int i0 = blockIdx.y * i_chunk;
  const int i1 = min(g.nx, i0 + i_chunk);
  if (i0 >= i1) return;
  const long long sx = g.sx;
  long long idx = static_cast<long long>(i0) * sx + j;
  T ez_c = g.ez[idx];
  const int sy_pml = slab(j, g.ny, pm.L[2], pm.L[3]);
  for (int i = i0; i < i1; ++i, idx += sx) {
    const T ez_n = g.ez[idx + sx];
    const T ez_j1 = g.ez[idx + 1];
    const T* c = g.lut + 18 * static_cast<int>(g.mid[idx]);
    const T d_hx_b = ez_j1 - ez_c;  // Hx from Ez along y
    const T d_hy_a = ez_n - ez_c;   // Hy from Ez along x
    T hxv = c[9] * g.hx[idx] + c[11] * d_hx_b;
    T hyv = c[12] * g.hy[idx] + c[13] * d_hy_a;
    if (tf.on) {
      // XN-Y, XP-Y: Hy at i = is-1 / ie, j in [js, je]
      if (j >= tf.js && j <= tf.je) {
        if (i == tf.is - 1) add_inc(hyv, ez_inc(tf, tf.is, j, 0), -tf.cb[0]);
        if (i == tf.ie) add_inc(hyv, ez_inc(tf, tf.ie, j, 0), tf.cb[0]);
      }
      // YN-X, YP-X: Hx at j = js-1 / je, i in [is, ie]
      if (i >= tf.is && i <= tf.ie) {
        if (j == tf.js - 1) add_inc(hxv, ez_inc(tf, i, tf.js, 0), tf.cb[1]);
        if (j == tf.je) add_inc(hxv, ez_inc(tf, i, tf.je, 0), -tf.cb[1]);
      }
    }
    const int sx_pml = slab(i, g.nx, pm.L[0], pm.L[1]);
    if (sx_pml >= 0) {
      const long long p = sx_pml * sx + j;
      T py = pm.bh[0][i] * pm.hy_x[p] + pm.ah[0][i] * d_hy_a;
      pm.hy_x[p] = py;
      hyv = hyv + c[13] * py;
    }
    if (sy_pml >= 0) {
      const long long p = static_cast<long long>(i) * pm.ysx + sy_pml;
      T px = pm.bh[1][j] * pm.hx_y[p] + pm.ah[1][j] * d_hx_b;
      pm.hx_y[p] = px;
      hxv = hxv + c[11] * px;
    }
    g.hx[idx] = hxv;
    g.hy[idx] = hyv;
    ez_c = ez_n;
  }
}

template <typename T>
__global__ void k_e2(GridP<T> g, PmlP<T> pm, TfsfP tf_in, TimeP tp, int i_chunk) {
  const TfsfP tf = tfsf_at_step(tf_in, cur_step(tp));
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= g.ny) return;
  const int i0 = blockIdx.y * i_chunk;
  const int i1 = min(g.nx, i0 + i_chunk);
  if (i0 >= i1) return;
  const long long sx = g.sx;
  long long idx = static_cast<long long>(i0) * sx + j;
  T hy_p = g.hy[idx - sx];
  const int sy_pml = slab(j, g.ny, pm.L[2], pm.L[3]);
  for (int i = i0; i < i1; ++i, idx += sx) {
    const T hx_c = g.hx[idx], hx_jm = g.hx[idx - 1];
    const T hy_c = g.hy[idx];
    if (i > 0 && j > 0) {
      const T* c = g.lut + 18 * static_cast<int>(g.mid[idx]);
      const T d_ez_a = hx_c - hx_jm;
      const T d_ez_b = hy_c - hy_p;
      T ezv = c[6] * g.ez[idx] + c[7] * d_ez_a + c[8] * d_ez_b;
      if (tf.on) {
        if (j >= tf.js && j <= tf.je) {
          if (i == tf.is) add_inc(ezv, hy_inc(tf, tf.is - 1, j, 0), -tf.ca[0]);
          if (i == tf.ie) add_inc(ezv, hy_inc(tf, tf.ie, j, 0), tf.ca[0]);
        }
        if (i >= tf.is && i <= tf.ie) {
          if (j == tf.js) add_inc(ezv, hx_inc(tf, i, tf.js - 1, 0), tf.ca[1]);
          if (j == tf.je) add_inc(ezv, hx_inc(tf, i, tf.je, 0), -tf.ca[1]);
        }
      }
      const int sx_pml = slab(i, g.nx, pm.L[0], pm.L[1]);
      if (sx_pml >= 0) {
        const long long p = sx_pml * sx + j;
        T ps = pm.be[0][i] * pm.ez_x[p] + pm.ae[0][i] * d_ez_b;
        pm.ez_x[p] = ps;
        ezv = ezv + c[8] * ps;
      }
      if (sy_pml >= 0) {
        const long long p = static_cast<long long>(i) * pm.ysx + sy_pml;
        T ps = pm.be[1][j] * pm.ez_y[p] + pm.ae[1][j] * d_ez_a;
        pm.ez_y[p] = ps;
        ezv = ezv + c[7] * ps;
      }
      g.ez[idx] = ezv;
    }
    hy_p = hy_c;
  }
}

// ---------------------------------------------------------------------------
// TFSF 1-D auxiliary grid: its whole history, computed once when the run is
// set up (the grid depends on the source only, not on the 3-D fields), so no
// time step waits on it.  Row t of e_tab holds E^t, row t of h_tab H^{t+1/2};
// step t: h = h_prev + chie (e[l+1] - e[l]), then E^{t+1} with the source at
// node 0 and a first-order Mur boundary at node nl.  One block walks the
// steps (one barrier per half-step); e_tab row 0 is zero.
static __global__ void k_aux_table(double* e_tab, double* h_tab, int nl, double ceih, double chie, double abc,
                                   const double* src, long long steps) {
  for (long long t = 0; t < steps; ++t) {
    const double* e = e_tab + t * (nl + 1);
    const double* hp = t > 0 ? h_tab + (t - 1) * nl : nullptr;
    double* h = h_tab + t * nl;
    double* en = e_tab + (t + 1) * (nl + 1);
    for (int l = threadIdx.x; l < nl; l += blockDim.x) h[l] = (hp ? hp[l] : 0.0) + chie * (e[l + 1] - e[l]);
    __syncthreads();
    for (int l = threadIdx.x + 1; l < nl; l += blockDim.x) en[l] = e[l] + ceih * (h[l] - h[l - 1]);
    if (threadIdx.x == 0) en[0] = src[t + 1];
    __syncthreads();
    if (threadIdx.x == 0) en[nl] = e[nl - 1] + abc * (en[nl - 1] - e[nl]);
    __syncthreads();
  }
}

static __global__ void k_bump(long long* t, int n) { *t += n; }

// ---------------------------------------------------------------------------
// TFSF line tables of one step.  Every cell on a y or z face line of the TFSF
// surface (the rows js-1, js, je; the columns ks-1, ks, ke) takes its
// corrections from two incident-field components at a fixed node of the line;
// the step kernel stages those values per plane with its bulk copies, next to
// the fields, instead of computing each from the projections and the
// auxiliary row (two dependent loads per corrected cell).  Tables, all FP64:
//   yh[f][i][c][k]: H pass, row js-1 (f = 0: values at j = js) or je (f = 1):
//                   c = 0 ex_inc, c = 1 ez_inc
//   ye[f][i][c][k]: E pass, row js (f = 0: values at j = js-1) or je:
//                   c = 0 hx_inc, c = 1 hz_inc
//   zh[f][i][c][j]: H pass, column ks-1 (f = 0: values at k = ks) or ke:
//                   c = 0 ey_inc, c = 1 ex_inc
//   ze[f][i][c][j]: E pass, column ks (f = 0: values at k = ks-1) or ke:
//                   c = 0 hy_inc, c = 1 hx_inc
// over i in [is, ie] and k (j) in [ks, ke] ([js, je]), each entry only where
// a correction reads it (the others stay zero); rows of k pitch ykp, rows of
// j pitch zjp.  The values are those ex_inc .. hz_inc return, so the
// corrections are unchanged bit for bit.
struct LineP {
  double* yh; double* ye; double* zh; double* ze;
  long long ykp, zjp;  // row pitch (elements) of the y and z tables
  long long ysl, zsl;  // elements per plane i (2 components)
  long long yfs, zfs;  // elements per face
};

// Entries w0, w0 + stride, ... of the line tables of the step whose rows tf
// holds (the y tables first, then the z tables).
__device__ __forceinline__ void tfsf_lines_fill(const TfsfP& tf, const LineP& lp, long long w0, long long stride) {
  const int ni = tf.ie - tf.is + 1, nk = tf.ke - tf.ks + 1, nj = tf.je - tf.js + 1;
  const long long ny_work = 2LL * ni * nk, nz_work = 2LL * ni * nj;
  for (long long w = w0; w < ny_work + nz_work; w += stride) {
    if (w < ny_work) {
      const int f = static_cast<int>(w / (static_cast<long long>(ni) * nk));
      const long long r = w - static_cast<long long>(f) * ni * nk;
      const int i = tf.is + static_cast<int>(r / nk), k = tf.ks + static_cast<int>(r % nk);
      const long long o = f * lp.yfs + i * lp.ysl + k;
      const int jh = f ? tf.je : tf.js, je = f ? tf.je : tf.js - 1;
      // only the entries a correction reads (the others stay zero)
      if (i < tf.ie) lp.yh[o] = ex_inc(tf, i, jh, k);
      if (k < tf.ke) lp.yh[o + lp.ykp] = ez_inc(tf, i, jh, k);
      if (k < tf.ke) lp.ye[o] = hx_inc(tf, i, je, k);
      if (i < tf.ie) lp.ye[o + lp.ykp] = hz_inc(tf, i, je, k);
    } else {
      const long long v = w - ny_work;
      const int f = static_cast<int>(v / (static_cast<long long>(ni) * nj));
      const long long r = v - static_cast<long long>(f) * ni * nj;
      const int i = tf.is + static_cast<int>(r / nj), j = tf.js + static_cast<int>(r % nj);
      const long long o = f * lp.zfs + i * lp.zsl + j;
      const int kh = f ? tf.ke : tf.ks, ke = f ? tf.ke : tf.ks - 1;
      if (j < tf.je) lp.zh[o] = ey_inc(tf, i, j, kh);
      if (i < tf.ie) lp.zh[o + lp.zjp] = ex_inc(tf, i, j, kh);
      if (i < tf.ie) lp.ze[o] = hy_inc(tf, i, j, ke);
      if (j < tf.je) lp.ze[o + lp.zjp] = hx_inc(tf, i, j, ke);
    }
  }
}

// (kernels instantiated per engine precision, so the FP64 engine's copies are
// compiled with that engine's no-contraction rule)
template <typename T>
__global__ void k_tfsf_lines(TfsfP tf_in, TimeP tp, LineP lp) {
  tfsf_lines_fill(tfsf_at_step(tf_in, cur_step(tp)), lp, blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x,
                  static_cast<long long>(gridDim.x) * blockDim.x);
}

// ---------------------------------------------------------------------------
// NF2FF frequency-domain accumulation: one thread per face point, all faces and
// frequencies in one launch.  The four surface samples of a point (the
// interpolated tangential H and E with the current signs) are kept for
// kNfRing steps in a ring; every kNfRing-th step the point's accumulators are
// read once, advanced over the buffered steps in step order, and written
// back, so the running DFT costs one accumulator round trip per kNfRing steps
// instead of one per step.  A host read first runs k_nf2ff_flush over the
// steps still in the ring; `done` (steps already in the accumulators beyond
// the last full ring) keeps a flushed step from being added twice.
constexpr int kNfRing = 8;

struct NfP {
  int nfreq;
  int box[6];                 // is ie js je ks ke
  int off[7];                 // point offsets of the six faces (prefix sums)
  long long npts;             // total points
  double2* acc;               // [nfreq][4][npts]  ja jb ma mb
  const double2* te; const double2* th;  // [nfreq][total_steps]
  long long total_steps;
  double* ring;               // [kNfRing][4][npts] samples of the buffered steps
  long long* done;            // steps accumulated by the last flush
  int own_lo, own_hi;         // planes i this handle samples (an x slab: the planes it owns)
};

// Advance the accumulators of point pt over steps lo .. hi-1 taken from the
// ring, then (cur) over step hi with the samples s[4]; frequencies in groups
// of four so the accumulators of a group stay in registers.  Every
// accumulator sees its steps in increasing order, as in a per-step update.
__device__ __forceinline__ void nf_advance(const NfP& nf, long long pt, long long lo, long long hi, bool cur,
                                           const double s[4]) {
  for (int f0 = 0; f0 < nf.nfreq; f0 += 4) {
    const int nfg = min(4, nf.nfreq - f0);
    double2 a[4][4];
#pragma unroll
    for (int g = 0; g < 4; ++g)
      if (g < nfg)
#pragma unroll
        for (int w = 0; w < 4; ++w) a[g][w] = nf.acc[(static_cast<long long>(f0 + g) * 4 + w) * nf.npts + pt];
    for (long long t = lo; t <= hi; ++t) {
      if (t == hi && !cur) break;
      double v[4];
      if (t == hi) {
#pragma unroll
        for (int w = 0; w < 4; ++w) v[w] = s[w];
      } else {
        const double* r = nf.ring + static_cast<long long>(t % kNfRing) * 4 * nf.npts + pt;
#pragma unroll
        for (int w = 0; w < 4; ++w) v[w] = r[w * nf.npts];
      }
#pragma unroll
      for (int g = 0; g < 4; ++g)
        if (g < nfg) {
          const double2 th = nf.th[(f0 + g) * nf.total_steps + t], te = nf.te[(f0 + g) * nf.total_steps + t];
          a[g][0].x = a[g][0].x + v[0] * th.x; a[g][0].y = a[g][0].y + v[0] * th.y;
          a[g][1].x = a[g][1].x + v[1] * th.x; a[g][1].y = a[g][1].y + v[1] * th.y;
          a[g][2].x = a[g][2].x + v[2] * te.x; a[g][2].y = a[g][2].y + v[2] * te.y;
          a[g][3].x = a[g][3].x + v[3] * te.x; a[g][3].y = a[g][3].y + v[3] * te.y;
        }
    }
#pragma unroll
    for (int g = 0; g < 4; ++g)
      if (g < nfg)
#pragma unroll
        for (int w = 0; w < 4; ++w) nf.acc[(static_cast<long long>(f0 + g) * 4 + w) * nf.npts + pt] = a[g][w];
  }
}

// Steps [max(t_end - t_end % kNfRing, *done), t_end) still in the ring into
// the accumulators (t_end: steps taken).  *done is set afterwards by
// k_nf2ff_done, so every thread reads the value of before the flush.
static __global__ void k_nf2ff_flush(NfP nf, long long t_end) {
  const long long pt = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (pt >= nf.npts) return;
  const long long lo = max(t_end - t_end % kNfRing, *nf.done);
  if (lo >= t_end) return;
  const double none[4] = {0, 0, 0, 0};
  nf_advance(nf, pt, lo, t_end, false, none);
}

static __global__ void k_nf2ff_done(long long* done, long long v) { *done = v; }

template <typename T>
__device__ __forceinline__ double ld(const T* p, long long i) { return static_cast<double>(p[i]); }

// Tangential fields at the centre of the face-normal `axis` cell face whose
// node is element x: H_a, H_b, E_a, E_b of the face's tangential axes (a, b)
// = (y, z), (z, x), (x, y) (interpolateSurfaceCenter,
// src/include/nf2ff/interpolate_scheme.cuh:11-134).
template <typename T>
__device__ __forceinline__ void nf_face_samples(const GridP<T>& g, int axis, long long x, double& ha, double& hb,
                                                double& ea, double& eb) {
  const long long sx = g.sx, sy = g.sy;
  if (axis == 0) {
    hb = 0.25 * (ld(g.hz, x + 1) + ld(g.hz, x) + ld(g.hz, x - sx + 1) + ld(g.hz, x - sx));  // HzFaceX
    ha = 0.25 * (ld(g.hy, x + sy) + ld(g.hy, x) + ld(g.hy, x - sx + sy) + ld(g.hy, x - sx));  // HyFaceX
    eb = 0.5 * (ld(g.ez, x + sy) + ld(g.ez, x));  // EzFaceX
    ea = 0.5 * (ld(g.ey, x + 1) + ld(g.ey, x));   // EyFaceX
  } else if (axis == 1) {
    hb = 0.25 * (ld(g.hx, x + sx) + ld(g.hx, x) + ld(g.hx, x + sx - sy) + ld(g.hx, x - sy));  // HxFaceY
    ha = 0.25 * (ld(g.hz, x + 1) + ld(g.hz, x) + ld(g.hz, x - sy + 1) + ld(g.hz, x - sy));    // HzFaceY
    eb = 0.5 * (ld(g.ex, x + 1) + ld(g.ex, x));   // ExFaceY
    ea = 0.5 * (ld(g.ez, x + sx) + ld(g.ez, x));  // EzFaceY
  } else {
    hb = 0.25 * (ld(g.hy, x) + ld(g.hy, x + sy) + ld(g.hy, x - 1) + ld(g.hy, x + sy - 1));  // HyFaceZ
    ha = 0.25 * (ld(g.hx, x + sx) + ld(g.hx, x) + ld(g.hx, x - 1) + ld(g.hx, x + sx - 1));  // HxFaceZ
    eb = 0.5 * (ld(g.ey, x + sx) + ld(g.ey, x));  // EyFaceZ
    ea = 0.5 * (ld(g.ex, x + sy) + ld(g.ex, x));  // ExFaceZ
  }
}

template <typename T>
__global__ void k_nf2ff(GridP<T> g, NfP nf, TimeP tp) {
  const long long pt = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (pt >= nf.npts) return;
  const long long t = cur_step(tp);
  int face = 0;
  while (face < 5 && pt >= nf.off[face + 1]) ++face;
  const long long q = pt - nf.off[face];
  const int axis = face >> 1, pos = face & 1;
  const int* b = nf.box;
  int i, j, k;
  if (axis == 0) { const int nk = b[5] - b[4]; i = pos ? b[1] : b[0]; j = b[2] + static_cast<int>(q / nk); k = b[4] + static_cast<int>(q % nk); }
  else if (axis == 1) { const int nk = b[5] - b[4]; j = pos ? b[3] : b[2]; i = b[0] + static_cast<int>(q / nk); k = b[4] + static_cast<int>(q % nk); }
  else { const int nj = b[3] - b[2]; k = pos ? b[5] : b[4]; i = b[0] + static_cast<int>(q / nj); j = b[2] + static_cast<int>(q % nj); }
  if (i < nf.own_lo || i >= nf.own_hi) return;  // another slab's point: its ring and sums stay zero here
  const long long x = static_cast<long long>(i) * g.sx + static_cast<long long>(j) * g.sy + k;
  double hb, ha, eb, ea;  // interpolated H_b, H_a, E_b, E_a at the face centre
  nf_face_samples(g, axis, x, ha, hb, ea, eb);
  const double cja = pos ? -1.0 : 1.0, cjb = pos ? 1.0 : -1.0;
  const double cma = pos ? 1.0 : -1.0, cmb = pos ? -1.0 : 1.0;
  const double smp[4] = {cja * hb, cjb * ha, cma * eb, cmb * ea};  // J_a, J_b, M_a, M_b samples
  const int slot = static_cast<int>(t % kNfRing);
  if (slot != kNfRing - 1) {
    double* r = nf.ring + static_cast<long long>(slot) * 4 * nf.npts + pt;
#pragma unroll
    for (int w = 0; w < 4; ++w) r[w * nf.npts] = smp[w];
    return;
  }
  nf_advance(nf, pt, max(t - (kNfRing - 1), *nf.done), t, true, smp);
}

// ---------------------------------------------------------------------------
// Time-domain NF2FF (NF2FFTimeDomainData<D>::update,
// src/nf2ff/time_domain/nf2ff_time_domain_data.cu:113-175).  The reference
// runs the whole surface on one thread per face because several face points
// add into the same time bin ("Here need to reduce sum", :174, and the
// <<<1,1>>> launches at :213-223).  Here the sample points of each (face,
// field kind) are sorted at init by their bin offset d0 = floor(delay + off)
// and cut into chunks of at most kTdChunk points with one d0.  At step t a
// point's two bins are t + d0 + rel and t + d0 + rel + 1 with rel = 0 or 1
// (the rounding of delay + off + t can carry into the next integer), so a
// chunk's contributions fall into three bins per tangential component:
// k_nftd_chunks sums them per chunk (warp shuffles, then the warps in
// order), k_nftd_bins adds, for every (component, bin) of the step's window,
// the chunk sums that land there, in chunk order.  Both levels have a fixed
// order: the potentials are reproducible run to run.
constexpr int kTdChunk = 256;

struct TdP {
  const int4* ent;      // per point (chunk order): i, j, k, face * 2 + kind (0: E, 1: H)
  const double* tsd;    // per point: delay in steps, (ref - r . dir) / (c dt)
  double* prev;         // [2][n]: the a and b samples of the previous step
  long long n;          // points (both kinds)
  const int4* chunk;    // first point, count, face * 2 + kind, d0
  double* part;         // [chunks][6]: (a, b) x bins t + d0 + {0, 1, 2}
  const int* offs;      // [6 * span + 1] CSR over (component, bin offset)
  const int* list;      // chunk * 6 + slot entries
  int span;             // bin offsets 0 .. span - 1 of a step
  double* pot;          // [6][bins]: W_x W_y W_z U_x U_y U_z
  long long bins;
  double ds[3];         // face area per normal axis
};

template <typename T>
__global__ void __launch_bounds__(kTdChunk) k_nftd_chunks(GridP<T> g, TdP td, TimeP tp) {
  const int4 ch = td.chunk[blockIdx.x];
  const long long t = cur_step(tp);
  const int face = ch.z >> 1, kind = ch.z & 1, axis = face >> 1;
  const bool neg = (face & 1) == 0;
  double v[6] = {0, 0, 0, 0, 0, 0};
  if (static_cast<int>(threadIdx.x) < ch.y) {
    const long long id = ch.x + threadIdx.x;
    const int4 p = td.ent[id];
    const long long x = static_cast<long long>(p.x) * g.sx + static_cast<long long>(p.y) * g.sy + p.z;
    double ha, hb, ea, eb;
    nf_face_samples(g, axis, x, ha, hb, ea, eb);
    const double a = kind ? ha : ea, b = kind ? hb : eb;
    const double da = a - td.prev[id], db = b - td.prev[td.n + id];
    td.prev[id] = a;
    td.prev[td.n + id] = b;
    // coefficients and time offset of the field kind (nf2ff_time_domain_data.cu:121-131)
    const double off = kind ? 0.0 : 0.5;
    double ca = kind ? -1.0 : 1.0, cb = kind ? 1.0 : -1.0;
    if (neg) { ca *= -1.0; cb *= -1.0; }
    const double u = td.tsd[id] + off + static_cast<double>(t);
    const double nn = floor(u);
    const double f = u - nn;
    const int rel = static_cast<int>(static_cast<long long>(nn) - t - ch.w);  // 0 or 1
    const double ds = td.ds[axis];
    v[rel] = ca * (1 - f) * ds * db;
    v[rel + 1] = ca * f * ds * db;
    v[3 + rel] = cb * (1 - f) * ds * da;
    v[3 + rel + 1] = cb * f * ds * da;
  }
  __shared__ double red[kTdChunk / 32][6];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < 6; ++q) {
    double s = v[q];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (lane == 0) red[wid][q] = s;
  }
  __syncthreads();
  if (threadIdx.x < 6) {
    double s = 0;
    for (int w = 0; w < static_cast<int>(blockDim.x >> 5); ++w) s += red[w][threadIdx.x];
    td.part[static_cast<long long>(blockIdx.x) * 6 + threadIdx.x] = s;
  }
}

static __global__ void k_nftd_bins(TdP td, TimeP tp) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= 6 * td.span) return;
  const int lo = td.offs[q], hi = td.offs[q + 1];
  if (lo == hi) return;
  const long long t = cur_step(tp);
  double s = 0;
  for (int e = lo; e < hi; ++e) s += td.part[td.list[e]];
  td.pot[(q / td.span) * td.bins + t + q % td.span] += s;
}

// ---------------------------------------------------------------------------
// Point probes: one value per step.
struct ProbeP {
  int n;
  const long long* idx;   // element index in the component array
  const int* field;       // component
  double* out;            // [n][total_steps]
  long long total_steps;
};

template <typename T>
__global__ void k_probe(GridP<T> g, ProbeP pr, TimeP tp) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= pr.n) return;
  const long long t = cur_step(tp);
  const int fld = pr.field[p];
  if (fld < 0) return;  // a probe of another x slab
  const T* f[6] = {g.ex, g.ey, g.ez, g.hx, g.hy, g.hz};
  pr.out[p * pr.total_steps + t] = static_cast<double>(f[fld][pr.idx[p]]);
}

// Movie frame: copies the component box every `interval` steps
// (MovieMonitor<F>::update, src/monitor/movie_monitor.cu:17-46).
template <typename T>
__global__ void k_movie(const T* fld, long long sx, long long sy, int lo0, int lo1, int lo2, int n0, int n1, int n2,
                        int interval, double* out, long long n_frames, TimeP tp, int own_lo, int own_hi) {
  const long long t = cur_step(tp);
  if (t % interval != 0) return;
  const long long frame = t / interval;
  if (frame >= n_frames) return;
  const long long per = static_cast<long long>(n0) * n1 * n2;
  for (long long e = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; e < per;
       e += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int c = static_cast<int>(e % n2);
    const int b = static_cast<int>((e / n2) % n1);
    const int a = static_cast<int>(e / (static_cast<long long>(n1) * n2));
    if (lo0 + a < own_lo || lo0 + a >= own_hi) continue;  // a plane of another x slab
    out[frame * per + e] = static_cast<double>(fld[static_cast<long long>(lo0 + a) * sx + static_cast<long long>(lo1 + b) * sy + lo2 + c]);
  }
}

// ---------------------------------------------------------------------------
// Far field from the surface currents: one block per observation angle, a
// block-wide reduction (warp shuffles + shared memory) over all face points.
struct FarP {
  int box[6];
  int off[7];
  long long npts;
  const double2* acc;  // accumulators of one frequency: [4][npts]
  double origin[3], d[3];
  double k;            // wavenumber
  double eta;          // free-space impedance
  const double* theta; const double* phi;
  double* out;         // [n][4]
};

__device__ __forceinline__ double warp_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

static __global__ void k_far(FarP fp) {
  const int a = blockIdx.x;
  const double th = fp.theta[a], ph = fp.phi[a];
  const double st = sin(th), ct = cos(th), sp = sin(ph), cp = cos(ph);
  const double rx = st * cp, ry = st * sp, rz = ct;
  double acc[12];  // N (x,y,z re/im), L (x,y,z re/im)
  for (int q = 0; q < 12; ++q) acc[q] = 0;
  const int* b = fp.box;
  for (long long pt = threadIdx.x; pt < fp.npts; pt += blockDim.x) {
    int face = 0;
    while (face < 5 && pt >= fp.off[face + 1]) ++face;
    const long long q = pt - fp.off[face];
    const int axis = face >> 1, pos = face & 1;
    double x, y, z, ds;
    int ca, cb;  // components of (ja, jb) / (ma, mb)
    if (axis == 0) {
      const int nk = b[5] - b[4];
      x = fp.origin[0] + (pos ? b[1] : b[0]) * fp.d[0];
      y = fp.origin[1] + (b[2] + q / nk + 0.5) * fp.d[1];
      z = fp.origin[2] + (b[4] + q % nk + 0.5) * fp.d[2];
      ds = fp.d[1] * fp.d[2]; ca = 1; cb = 2;
    } else if (axis == 1) {
      const int nk = b[5] - b[4];
      y = fp.origin[1] + (pos ? b[3] : b[2]) * fp.d[1];
      x = fp.origin[0] + (b[0] + q / nk + 0.5) * fp.d[0];
      z = fp.origin[2] + (b[4] + q % nk + 0.5) * fp.d[2];
      ds = fp.d[0] * fp.d[2]; ca = 2; cb = 0;
    } else {
      const int nj = b[3] - b[2];
      z = fp.origin[2] + (pos ? b[5] : b[4]) * fp.d[2];
      x = fp.origin[0] + (b[0] + q / nj + 0.5) * fp.d[0];
      y = fp.origin[1] + (b[2] + q % nj + 0.5) * fp.d[1];
      ds = fp.d[0] * fp.d[1]; ca = 0; cb = 1;
    }
    double sn, cs;
    sincos(fp.k * (rx * x + ry * y + rz * z), &sn, &cs);
    const double2 ja = fp.acc[pt], jb = fp.acc[fp.npts + pt], ma = fp.acc[2 * fp.npts + pt], mb = fp.acc[3 * fp.npts + pt];
    // (re + j im) * (cs + j sn) * ds
    acc[2 * ca] += (ja.x * cs - ja.y * sn) * ds; acc[2 * ca + 1] += (ja.x * sn + ja.y * cs) * ds;
    acc[2 * cb] += (jb.x * cs - jb.y * sn) * ds; acc[2 * cb + 1] += (jb.x * sn + jb.y * cs) * ds;
    acc[6 + 2 * ca] += (ma.x * cs - ma.y * sn) * ds; acc[6 + 2 * ca + 1] += (ma.x * sn + ma.y * cs) * ds;
    acc[6 + 2 * cb] += (mb.x * cs - mb.y * sn) * ds; acc[6 + 2 * cb + 1] += (mb.x * sn + mb.y * cs) * ds;
  }
  __shared__ double red[32][12];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int q = 0; q < 12; ++q) {
    const double v = warp_sum(acc[q]);
    if (lane == 0) red[wid][q] = v;
  }
  __syncthreads();
  if (wid == 0) {
    const int nw = (blockDim.x + 31) >> 5;
    for (int q = 0; q < 12; ++q) {
      double v = lane < nw ? red[lane][q] : 0.0;
      v = warp_sum(v);
      if (lane == 0) red[0][q] = v;
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const double* s = red[0];
    // N_theta, N_phi, L_theta, L_phi (complex)
    const double nthr = s[0] * ct * cp + s[2] * ct * sp - s[4] * st, nthi = s[1] * ct * cp + s[3] * ct * sp - s[5] * st;
    const double nphr = -s[0] * sp + s[2] * cp, nphi = -s[1] * sp + s[3] * cp;
    const double lthr = s[6] * ct * cp + s[8] * ct * sp - s[10] * st, lthi = s[7] * ct * cp + s[9] * ct * sp - s[11] * st;
    const double lphr = -s[6] * sp + s[8] * cp, lphi = -s[7] * sp + s[9] * cp;
    const double eta = fp.eta;
    const double f = fp.k / (4 * 3.14159265358979323846);
    // E_theta = -j f (L_phi + eta N_theta); E_phi = j f (L_theta - eta N_phi)
    const double xr = lphr + eta * nthr, xi = lphi + eta * nthi;
    const double yr = lthr - eta * nphr, yi = lthi - eta * nphi;
    double* o = fp.out + 4 * a;
    o[0] = f * xi; o[1] = -f * xr;
    o[2] = -f * yi; o[3] = f * yr;
  }
}

// Count non-finite values of a field array (watchdog).
template <typename T>
__global__ void k_nonfinite(const T* f, long long n, unsigned long long* bad) {
  unsigned long long c = 0;
  for (long long e = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; e < n;
       e += static_cast<long long>(gridDim.x) * blockDim.x)
    if (!isfinite(static_cast<double>(f[e]))) ++c;
  if (c) atomicAdd(bad, c);
}

}  // namespace xfb
