// Temporally blocked 2-D TMz step: S time steps per launch.
//
// The 2-D grid of the benchmarks is small enough to sit in L2 (1044^2 cells:
// 13 MB of FP32 fields), so a launch per step is bound by launch and memory
// latency, not bandwidth.  Here a CTA owns a tile of TI x TJ cells, loads the
// tile with a halo of S cells on every side into shared memory (Ez, Hx, Hy,
// material ids, the CPML psi of the tile's slab rows and columns, the
// coefficient LUT), advances it S steps there -- every step the region whose
// values are exact shrinks by one cell per side: H needs Ez one cell up, E
// needs H one cell down -- and writes back its interior.  Neighbouring tiles
// recompute each other's halo, so no CTA waits for another.  Probes inside
// the interior are recorded after every step of the block.
//
// Field and psi buffers alternate between launches: a launch reads set p and
// writes set 1-p (the E-side psi too, which the one-launch-per-step kernel
// keeps in place), so S is odd and the set holding step t is t & 1, as for
// the per-step kernels.  The per-cell arithmetic, the TFSF and CPML
// corrections and their order are those of k_step2 (and so of k_h2/k_e2 and
// the CPU restatement), FP64 results are bit-identical.
#pragma once

#include "fused3d.cuh"

namespace xfb {

// Asynchronous copy of one element into shared memory; zeros when !in (no
// byte is read then, and the source address given is the array's first).
template <typename T>
__device__ __forceinline__ void cp_async_zfill(T* smem, const T* gmem, bool in) {
  const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.ca.shared.global [%0], [%1], %2, %3;\n" ::"r"(d), "l"(gmem), "n"(sizeof(T)),
               "r"(in ? static_cast<int>(sizeof(T)) : 0)
               : "memory");
}

constexpr int kTbPitch = 96;   // columns of a shared tile row (j), TJ + 2 S + 1 <= 96
constexpr int kTbSlab = 16;    // CPML rows (columns) of a tile's region that fit its psi tables
constexpr int kTbThreads = 512;

// Shared-memory layout of one tile: fields [3][XI][kTbPitch], material ids
// [XI][kTbPitch], psi of the x-slab rows [2][kTbSlab][kTbPitch] (Hy, Ez), of
// the y-slab columns [2][XI][kTbSlab] (Hx, Ez), the LUT [n_mat][18], the
// slot maps (row -> x-slab slot, column -> y-slab slot) and the incident
// fields of one step on the TFSF lines the region holds: per column, E at
// is and ie and H at is-1 and ie; per row, E at js and je and H at js-1, je.
template <typename T>
struct TbLayout {
  int XI;
  size_t f, m, px, py, lut, slots, inc, bytes;
  __host__ __device__ TbLayout(int xi, int n_mat) : XI(xi) {
    f = 0;
    m = f + 3ull * xi * kTbPitch * sizeof(T);
    px = (m + static_cast<size_t>(xi) * kTbPitch + 15) / 16 * 16;
    py = px + 2ull * kTbSlab * kTbPitch * sizeof(T);
    lut = py + 2ull * xi * kTbSlab * sizeof(T);
    slots = lut + static_cast<size_t>(n_mat) * 18 * sizeof(T);
    inc = (slots + (static_cast<size_t>(xi) + kTbPitch) * sizeof(int) + 15) / 16 * 16;
    bytes = inc + (4ull * kTbPitch + 4ull * xi) * sizeof(double);
  }
};

template <typename T>
__global__ void __launch_bounds__(kTbThreads) k_step2_tb(GridP<T> s, GridP<T> d, PmlP<T> pm, PsiH<T> ps, PsiH<T> pd,
                                                         const T* ezx_r, const T* ezy_r, T* ezx_w, T* ezy_w,
                                                         TfsfP tf_in, TimeP tp, ProbeP pr, int S, int TI, int TJ,
                                                         int n_mat, int* err) {
  extern __shared__ __align__(16) unsigned char tb_smem[];
  const int XI = TI + 2 * S + 1, XJ = TJ + 2 * S + 1;
  const TbLayout<T> lay(XI, n_mat);
  T* __restrict__ E = reinterpret_cast<T*>(tb_smem + lay.f);
  T* __restrict__ HX = E + XI * kTbPitch;
  T* __restrict__ HY = HX + XI * kTbPitch;
  uint8_t* __restrict__ M = tb_smem + lay.m;
  T* __restrict__ PX = reinterpret_cast<T*>(tb_smem + lay.px);   // [2][kTbSlab][kTbPitch]: Hy_x, Ez_x
  T* __restrict__ PY = reinterpret_cast<T*>(tb_smem + lay.py);   // [2][XI][kTbSlab]: Hx_y, Ez_y
  T* __restrict__ lut = reinterpret_cast<T*>(tb_smem + lay.lut);
  int* xslot = reinterpret_cast<int*>(tb_smem + lay.slots);
  int* yslot = xslot + XI;
  double* incc = reinterpret_cast<double*>(tb_smem + lay.inc);  // [4][kTbPitch]: E(is), E(ie), H(is-1), H(ie)
  double* incr = incc + 4 * kTbPitch;                              // [4][XI]: E(js), E(je), H(js-1), H(je)

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, nw = kTbThreads / 32;
  const int I0 = blockIdx.y * TI, J0 = blockIdx.x * TJ;
  const int ib = I0 - S, jb = J0 - S;  // global index of row / column 0 of the region
  const int nx = s.nx, ny = s.ny;
  const long long sx = s.sx;
  const long long t0 = cur_step(tp);

  for (int q = tid; q < n_mat * 18; q += kTbThreads) lut[q] = s.lut[q];
  if (tid == 0) {  // slab slots of the region's rows and columns, in order
    // (the host plans tiles whose regions fit the tables; a row past them
    // would be left without psi and flagged)
    int n = 0, over = 0;
    for (int r = 0; r < XI; ++r) {
      const int i = ib + r;
      const int sl = i >= 0 && i < nx ? slab(i, nx, pm.L[0], pm.L[1]) : -1;
      xslot[r] = sl >= 0 && n < kTbSlab ? n++ : -1;
      over |= sl >= 0 && xslot[r] < 0;
    }
    int m = 0;
    for (int c = 0; c < kTbPitch; ++c) {
      const int j = jb + c;
      const int sl = c < XJ && j >= 0 && j < ny ? slab(j, ny, pm.L[2], pm.L[3]) : -1;
      yslot[c] = sl >= 0 && m < kTbSlab ? m++ : -1;
      over |= sl >= 0 && yslot[c] < 0;
    }
    if (over) atomicExch(err, 2);
  }
  __syncthreads();
  // ---- load the region: asynchronous copies, all in flight at once (zero
  // fill outside the arrays: such entries are never used by an update) -------
  for (int r = warp; r < XI; r += nw) {
    const int i = ib + r;
    const bool irow = i >= 0 && i <= nx;
    const int sxs = xslot[r];
    const int sxp = sxs >= 0 ? slab(i, nx, pm.L[0], pm.L[1]) : -1;
#pragma unroll
    for (int cc = 0; cc < kTbPitch / 32; ++cc) {
      const int c = lane + 32 * cc;
      const int j = jb + c;
      const bool in = irow && c < XJ && j >= 0 && j <= ny;
      const long long g = in ? static_cast<long long>(i) * sx + j : 0;
      const int o = r * kTbPitch + c;
      cp_async_zfill<T>(E + o, s.ez + g, in);
      cp_async_zfill<T>(HX + o, s.hx + g, in);
      cp_async_zfill<T>(HY + o, s.hy + g, in);
      if (sxs >= 0) {
        const bool jv = in && j < ny;
        const long long p = jv ? static_cast<long long>(sxp) * sx + j : 0;
        cp_async_zfill<T>(PX + sxs * kTbPitch + c, ps.hy_x + p, jv);
        cp_async_zfill<T>(PX + (kTbSlab + sxs) * kTbPitch + c, ezx_r + p, jv);
      }
      const int sys = yslot[c];
      if (sys >= 0) {
        const long long p = irow ? static_cast<long long>(i) * pm.ysx + slab(j, ny, pm.L[2], pm.L[3]) : 0;
        cp_async_zfill<T>(PY + r * kTbSlab + sys, ps.hx_y + p, irow);
        cp_async_zfill<T>(PY + (XI + r) * kTbSlab + sys, ezy_r + p, irow);
      }
    }
    cp_async_commit();
  }
  // material ids: plain loads, a row's three chunks issued together
  for (int r = warp; r < XI; r += nw) {
    const int i = ib + r;
    uint8_t m[kTbPitch / 32];
#pragma unroll
    for (int cc = 0; cc < kTbPitch / 32; ++cc) {
      const int j = jb + lane + 32 * cc;
      m[cc] = i >= 0 && i < nx && lane + 32 * cc < XJ && j >= 0 && j < ny ? s.mid[static_cast<long long>(i) * sx + j] : 0;
    }
#pragma unroll
    for (int cc = 0; cc < kTbPitch / 32; ++cc) M[r * kTbPitch + lane + 32 * cc] = m[cc];
  }
  cp_async_wait<0>();
  __syncthreads();

  // TFSF lines inside the region (row and column ranges of the box)
  const bool tf_cols = tf_in.on && ((tf_in.is - 1 >= ib && tf_in.is - 1 < ib + XI) || (tf_in.is >= ib && tf_in.is < ib + XI) ||
                                    (tf_in.ie >= ib && tf_in.ie < ib + XI));
  const bool tf_rows = tf_in.on && ((tf_in.js - 1 >= jb && tf_in.js - 1 < jb + XJ) || (tf_in.js >= jb && tf_in.js < jb + XJ) ||
                                    (tf_in.je >= jb && tf_in.je < jb + XJ));
  for (int st = 0; st < S; ++st) {
    const long long t = t0 + st;
    const TfsfP tf = tfsf_at_step(tf_in, t);
    // the step's incident values on the region's TFSF lines, one per thread
    // (the corrections below then read shared memory); the same expressions
    // as the per-cell corrections evaluate
    if (tf_cols || tf_rows) {
      for (int q = tid; q < 4 * kTbPitch + 4 * XI; q += kTbThreads) {
        double v = 0;
        if (q < 4 * kTbPitch) {
          const int w = q / kTbPitch, c = q - w * kTbPitch, j = jb + c;
          if (tf_cols && c < XJ && j >= tf.js && j <= tf.je)
            v = w == 0 ? ez_inc(tf, tf.is, j, 0) : w == 1 ? ez_inc(tf, tf.ie, j, 0)
                : w == 2 ? hy_inc(tf, tf.is - 1, j, 0) : hy_inc(tf, tf.ie, j, 0);
          incc[q] = v;
        } else {
          const int q2 = q - 4 * kTbPitch, w = q2 / XI, r = q2 - w * XI, i = ib + r;
          if (tf_rows && i >= tf.is && i <= tf.ie)
            v = w == 0 ? ez_inc(tf, i, tf.js, 0) : w == 1 ? ez_inc(tf, i, tf.je, 0)
                : w == 2 ? hx_inc(tf, i, tf.js - 1, 0) : hx_inc(tf, i, tf.je, 0);
          incr[q2] = v;
        }
      }
      __syncthreads();
    }
    // ---- H of rows st .. XI-2-st, columns st .. XJ-2-st (cells of the grid) --
    const int hr0 = max(st, -ib), hr1 = min(XI - 2 - st, nx - 1 - ib);
    const int hc0 = max(st, -jb), hc1 = min(XJ - 2 - st, ny - 1 - jb);
    for (int r = hr0 + warp; r <= hr1; r += nw) {
      const int i = ib + r;
      const int sxs = xslot[r];
      const bool tf_iin = tf.on && i >= tf.is && i <= tf.ie;
      const bool tf_hplane = tf.on && (i == tf.is - 1 || i == tf.ie);
      for (int c = hc0 + lane; c <= hc1; c += 32) {
        const int j = jb + c;
        const int o = r * kTbPitch + c;
        const T* cf = lut + 18 * M[o];
        const T ez_c = E[o];
        const T d_hx_b = E[o + 1] - ez_c;         // Hx from Ez along y
        const T d_hy_a = E[o + kTbPitch] - ez_c;  // Hy from Ez along x
        T hxv = cf[9] * HX[o] + cf[11] * d_hx_b;
        T hyv = cf[12] * HY[o] + cf[13] * d_hy_a;
        const bool tf_jin = tf.on && j >= tf.js && j <= tf.je;
        const bool tf_hline = tf.on && (j == tf.js - 1 || j == tf.je);
        if ((tf_hplane && tf_jin) || (tf_hline && tf_iin)) {
          if (tf_jin) {
            if (i == tf.is - 1) add_inc(hyv, incc[c], -tf.cb[0]);
            if (i == tf.ie) add_inc(hyv, incc[kTbPitch + c], tf.cb[0]);
          }
          if (tf_iin) {
            if (j == tf.js - 1) add_inc(hxv, incr[r], tf.cb[1]);
            if (j == tf.je) add_inc(hxv, incr[XI + r], -tf.cb[1]);
          }
        }
        if (sxs >= 0) {
          T& pp = PX[sxs * kTbPitch + c];
          const T py = pm.bh[0][i] * pp + pm.ah[0][i] * d_hy_a;
          pp = py;
          hyv = hyv + cf[13] * py;
        }
        const int sys = yslot[c];
        if (sys >= 0) {
          T& pp = PY[r * kTbSlab + sys];
          const T px = pm.bh[1][j] * pp + pm.ah[1][j] * d_hx_b;
          pp = px;
          hxv = hxv + cf[11] * px;
        }
        HX[o] = hxv;
        HY[o] = hyv;
      }
    }
    __syncthreads();
    // ---- E of rows st+1 .. XI-2-st, columns st+1 .. XJ-2-st (PEC walls kept) --
    const int er0 = max(st + 1, 1 - ib), er1 = min(XI - 2 - st, nx - 1 - ib);
    const int ec0 = max(st + 1, 1 - jb), ec1 = min(XJ - 2 - st, ny - 1 - jb);
    for (int r = er0 + warp; r <= er1; r += nw) {
      const int i = ib + r;
      const int sxs = xslot[r];
      const bool tf_iin = tf.on && i >= tf.is && i <= tf.ie;
      const bool tf_eplane = tf.on && (i == tf.is || i == tf.ie);
      for (int c = ec0 + lane; c <= ec1; c += 32) {
        const int j = jb + c;
        const int o = r * kTbPitch + c;
        const T* cf = lut + 18 * M[o];
        const T d_ez_a = HX[o] - HX[o - 1];
        const T d_ez_b = HY[o] - HY[o - kTbPitch];
        T ezv = cf[6] * E[o] + cf[7] * d_ez_a + cf[8] * d_ez_b;
        const bool tf_jin = tf.on && j >= tf.js && j <= tf.je;
        const bool tf_eline = tf.on && (j == tf.js || j == tf.je);
        if ((tf_eplane && tf_jin) || (tf_eline && tf_iin)) {
          if (tf_jin) {
            if (i == tf.is) add_inc(ezv, incc[2 * kTbPitch + c], -tf.ca[0]);
            if (i == tf.ie) add_inc(ezv, incc[3 * kTbPitch + c], tf.ca[0]);
          }
          if (tf_iin) {
            if (j == tf.js) add_inc(ezv, incr[2 * XI + r], tf.ca[1]);
            if (j == tf.je) add_inc(ezv, incr[3 * XI + r], -tf.ca[1]);
          }
        }
        if (sxs >= 0) {
          T& pp = PX[(kTbSlab + sxs) * kTbPitch + c];
          const T q = pm.be[0][i] * pp + pm.ae[0][i] * d_ez_b;
          pp = q;
          ezv = ezv + cf[8] * q;
        }
        const int sys = yslot[c];
        if (sys >= 0) {
          T& pp = PY[(XI + r) * kTbSlab + sys];
          const T q = pm.be[1][j] * pp + pm.ae[1][j] * d_ez_a;
          pp = q;
          ezv = ezv + cf[7] * q;
        }
        E[o] = ezv;
      }
    }
    __syncthreads();
    // ---- probes of the interior (and of the wall nodes past the last tiles) --
    for (int p = tid; p < pr.n; p += kTbThreads) {
      const int fld = pr.field[p];
      if (fld < 0) continue;
      const int i = static_cast<int>(pr.idx[p] / sx), j = static_cast<int>(pr.idx[p] - static_cast<long long>(i) * sx);
      const bool own_i = i >= I0 && (i < I0 + TI || I0 + TI >= nx);
      const bool own_j = j >= J0 && (j < J0 + TJ || J0 + TJ >= ny);
      if (!own_i || !own_j) continue;
      const int o = (i - ib) * kTbPitch + (j - jb);
      const T v = fld == XFB_EZ ? E[o] : fld == XFB_HX ? HX[o] : HY[o];
      pr.out[p * pr.total_steps + t] = static_cast<double>(v);
    }
  }
  // ---- write back the interior (what the per-step kernel writes) ------------
  for (int r = S + warp; r < S + TI; r += nw) {
    const int i = ib + r;
    if (i >= nx) continue;
    const int sxs = xslot[r];
    const int sxp = sxs >= 0 ? slab(i, nx, pm.L[0], pm.L[1]) : -1;
    for (int c = S + lane; c < S + TJ; c += 32) {
      const int j = jb + c;
      if (j >= ny) continue;
      const int o = r * kTbPitch + c;
      const long long g = static_cast<long long>(i) * sx + j;
      d.hx[g] = HX[o];
      d.hy[g] = HY[o];
      const bool e_upd = i >= 1 && j >= 1;
      if (e_upd) d.ez[g] = E[o];
      if (sxs >= 0) {
        const long long p = static_cast<long long>(sxp) * sx + j;
        pd.hy_x[p] = PX[sxs * kTbPitch + c];
        if (e_upd) ezx_w[p] = PX[(kTbSlab + sxs) * kTbPitch + c];
      }
      const int sys = yslot[c];
      if (sys >= 0) {
        const long long p = static_cast<long long>(i) * pm.ysx + slab(j, ny, pm.L[2], pm.L[3]);
        pd.hx_y[p] = PY[r * kTbSlab + sys];
        if (e_upd) ezy_w[p] = PY[(XI + r) * kTbSlab + sys];
      }
    }
  }
}

}  // namespace xfb
