// The "plain" GPU form of the time step: the reference's own kernel structure,
// kept as the baseline the fused paths are measured against.
//
//  * 18 per-cell coefficient arrays (the reference FDTDCoefficient arrays,
//    include/xfdtd_cuda/calculation_param/fdtd_coefficient.cuh:15-168), here in
//    the engine's padded field layout and filled once from the material LUT.
//  * One launch per field component, one thread per cell index of the flat
//    nx*ny*nz range with the row-major (i, j, k) decomposition by division and
//    modulo (src/include/updator/update_scheme.cuh:132-197).
//  * CPML corrections as one launch per face and half step over the face's
//    whole range including the +1 tangential extension
//    (src/boundary/pml_corrector.cu:9-291), TFSF corrections as one launch per
//    face/component agency (src/include/waveform_source/tfsf/tfsf_corrector.cuh:20-170,
//    src/waveform_source/tfsf/tfsf_corrector.cu:155-271), in the reference's
//    phase order: updateH, correctH (TFSF, CPML), updateE, correctE.
// Dispersive (ADE) scenes and 2-D scenes are not handled by this form.
#pragma once

#include "kernels.cuh"

namespace xfb {

template <typename T>
struct PlainCoef {
  T* c[18];  // slots in the order of enum Coef
};

template <typename T>
__global__ void k_plain_expand(PlainCoef<T> pc, const uint8_t* mid, const T* lut, long long n) {
  for (long long q = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; q < n;
       q += static_cast<long long>(gridDim.x) * blockDim.x) {
    const T* l = lut + 18 * static_cast<int>(mid[q]);
#pragma unroll
    for (int r = 0; r < 18; ++r) pc.c[r][q] = l[r];
  }
}

// Update of field component C (0..2 = x..z) of E (IS_E) or H over the cell
// range.  Tangential axes a = C+1, b = C+2 (mod 3); the E update skips the
// cells with a == 0 or b == 0 (PEC walls), as eNext/hNext do.
template <typename T, bool IS_E, int C>
__global__ void k_plain_comp(T* f, const T* fa, const T* fb, const T* cc, const T* ca, const T* cb, int nx, int ny,
                             int nz, long long sx, long long sy) {
  constexpr int A = (C + 1) % 3, B = (C + 2) % 3;
  const long long st_a = A == 0 ? sx : A == 1 ? sy : 1;
  const long long st_b = B == 0 ? sx : B == 1 ? sy : 1;
  const long long n = static_cast<long long>(nx) * ny * nz;
  const long long nyz = static_cast<long long>(ny) * nz;
  for (long long q = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; q < n;
       q += static_cast<long long>(gridDim.x) * blockDim.x) {
    const long long k = q % nz;
    const long long j = (q / nz) % ny;
    const long long i = q / nyz;
    const long long idx = i * sx + j * sy + k;
    if (IS_E) {
      const long long ca_ = A == 0 ? i : A == 1 ? j : k;
      const long long cb_ = B == 0 ? i : B == 1 ? j : k;
      if (ca_ == 0 || cb_ == 0) continue;
      // eNext: cece*E + cecha*(Ha - Ha[b-1]) + cechb*(Hb - Hb[a-1])
      f[idx] = cc[idx] * f[idx] + ca[idx] * (fa[idx] - fa[idx - st_b]) + cb[idx] * (fb[idx] - fb[idx - st_a]);
    } else {
      // hNext: chch*H + chcea*(Ea[b+1] - Ea) + chceb*(Eb[a+1] - Eb)
      f[idx] = cc[idx] * f[idx] + ca[idx] * (fa[idx + st_b] - fa[idx]) + cb[idx] * (fb[idx + st_a] - fb[idx]);
    }
  }
}

// CPML correction of one face of axis C for one half step: psi = b*psi +
// a*(dual difference along C), field += c_psi * psi for the two tangential
// components (cps0: component along a, cps1: along b).  c_psi is the per-cell
// update coefficient of the field with respect to that dual component.  The E
// range of a low face starts at plane 1 and stops before plane L, where the
// profile's a is zero and the correction adds nothing.
struct PlainPmlFace {
  int c0;                 // first plane along the face axis
  int a_end[2], b_end[2]; // tangential ranges of the two components
  long long span[2];      // planes * a_end * b_end per component
};

template <typename T, bool IS_E, int C>
__global__ void k_plain_pml(GridP<T> g, PmlP<T> pm, const T* cps0, const T* cps1, PlainPmlFace fc) {
  constexpr int A = (C + 1) % 3, B = (C + 2) % 3;
  const long long st_c = C == 0 ? g.sx : C == 1 ? g.sy : 1;
  const int n_c = C == 0 ? g.nx : C == 1 ? g.ny : g.nz;
  const T* pa = IS_E ? pm.ae[C] : pm.ah[C];
  const T* pb = IS_E ? pm.be[C] : pm.bh[C];
  const long long n_all = fc.span[0] + fc.span[1];
  for (long long q = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; q < n_all;
       q += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int w = q < fc.span[0] ? 0 : 1;
    const long long r = w == 0 ? q : q - fc.span[0];
    const int bn = w == 0 ? fc.b_end[0] : fc.b_end[1];
    const int an = w == 0 ? fc.a_end[0] : fc.a_end[1];
    const int vb = static_cast<int>(r % bn);
    const int va = static_cast<int>((r / bn) % an);
    const int cc = fc.c0 + static_cast<int>(r / (static_cast<long long>(bn) * an));
    const long long i = C == 0 ? cc : A == 0 ? va : vb;
    const long long j = C == 1 ? cc : A == 1 ? va : vb;
    const long long k = C == 2 ? cc : A == 2 ? va : vb;
    const long long idx = i * g.sx + j * g.sy + k;
    // w = 0: the component along a (dual along b); w = 1: along b (dual along a)
    T* F;
    const T* D;
    T* psi;
    if (w == 0) {
      F = IS_E ? (A == 0 ? g.ex : A == 1 ? g.ey : g.ez) : (A == 0 ? g.hx : A == 1 ? g.hy : g.hz);
      D = IS_E ? (B == 0 ? g.hx : B == 1 ? g.hy : g.hz) : (B == 0 ? g.ex : B == 1 ? g.ey : g.ez);
      psi = IS_E ? (C == 0 ? pm.ey_x : C == 1 ? pm.ez_y : pm.ex_z) : (C == 0 ? pm.hy_x : C == 1 ? pm.hz_y : pm.hx_z);
    } else {
      F = IS_E ? (B == 0 ? g.ex : B == 1 ? g.ey : g.ez) : (B == 0 ? g.hx : B == 1 ? g.hy : g.hz);
      D = IS_E ? (A == 0 ? g.hx : A == 1 ? g.hy : g.hz) : (A == 0 ? g.ex : A == 1 ? g.ey : g.ez);
      psi = IS_E ? (C == 0 ? pm.ez_x : C == 1 ? pm.ex_y : pm.ey_z) : (C == 0 ? pm.hz_x : C == 1 ? pm.hx_y : pm.hy_z);
    }
    const T* cps = w == 0 ? cps0 : cps1;
    const int s = slab(cc, n_c, pm.L[2 * C], pm.L[2 * C + 1]);
    long long p;
    if (C == 0) p = s * g.sx + j * g.sy + k;
    else if (C == 1) p = i * pm.ysx + s * g.sy + k;
    else p = i * pm.zsx + j * pm.zsy + s;
    const T dp = D[idx];
    T v;
    if (IS_E) v = pb[cc] * psi[p] + pa[cc] * (dp - D[idx - st_c]);
    else v = pb[cc] * psi[p] + pa[cc] * (D[idx + st_c] - dp);
    psi[p] = v;
    F[idx] = F[idx] + cps[idx] * v;
  }
}

// One TFSF correction agency: face (axis c, negative or positive side),
// attribute and field component, over the face rectangle.
struct PlainTfsfFace {
  int neg, attr_h, fxyz, dual;
  int as, ae, bs, be, cs;  // [as, ae) x [bs, be) along a, b; face plane cs along c
  double coef;
};

__device__ __forceinline__ double plain_inc(const TfsfP& tf, int attr_h, int comp, int i, int j, int k) {
  if (!attr_h) return comp == 0 ? ex_inc(tf, i, j, k) : comp == 1 ? ey_inc(tf, i, j, k) : ez_inc(tf, i, j, k);
  return comp == 0 ? hx_inc(tf, i, j, k) : comp == 1 ? hy_inc(tf, i, j, k) : hz_inc(tf, i, j, k);
}

template <typename T, int C>
__global__ void k_plain_tfsf(GridP<T> g, TfsfP tf_in, TimeP tp, PlainTfsfFace fc) {
  constexpr int A = (C + 1) % 3, B = (C + 2) % 3;
  const TfsfP tf = tfsf_at_step(tf_in, cur_step(tp));
  const int nb = fc.be - fc.bs;
  const long long n = static_cast<long long>(fc.ae - fc.as) * nb;
  T* F = fc.attr_h ? (fc.fxyz == 0 ? g.hx : fc.fxyz == 1 ? g.hy : g.hz) : (fc.fxyz == 0 ? g.ex : fc.fxyz == 1 ? g.ey : g.ez);
  for (long long q = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; q < n;
       q += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int va = fc.as + static_cast<int>(q / nb), vb = fc.bs + static_cast<int>(q % nb);
    // (i, j, k) on the face plane (p) and one plane outside it (m)
    const int pi = C == 0 ? fc.cs : A == 0 ? va : vb;
    const int pj = C == 1 ? fc.cs : A == 1 ? va : vb;
    const int pk = C == 2 ? fc.cs : A == 2 ? va : vb;
    const int mi = pi - (C == 0), mj = pj - (C == 1), mk = pk - (C == 2);
    long long idx;
    double inc;
    if (fc.neg) {
      if (!fc.attr_h) {  // E on the face plane, H incident one plane outside
        idx = pi * g.sx + pj * g.sy + pk;
        inc = plain_inc(tf, 1, fc.dual, mi, mj, mk);
      } else {           // H one plane outside, E incident on the face plane
        idx = mi * g.sx + mj * g.sy + mk;
        inc = plain_inc(tf, 0, fc.dual, pi, pj, pk);
      }
    } else {
      idx = pi * g.sx + pj * g.sy + pk;
      inc = plain_inc(tf, fc.attr_h ? 0 : 1, fc.dual, pi, pj, pk);
    }
    add_inc(F[idx], inc, fc.coef);
  }
}

}  // namespace xfb
