// One-sweep 3-D time step: H half-step and E half-step of a whole Yee step in
// a single kernel (temporal fusion), so each field component crosses HBM once
// per step (read E^n, H^{n-1/2}; write H^{n+1/2}, E^{n+1}) instead of the
// 9 + 9 transfers of two separate half-step kernels.
//
// Tiling.  A CTA owns a (TJ x 32) tile of (j, k) and marches along i over a
// chunk of planes.  NWM "row" warps own the tile: lane = k, and every thread
// carries R consecutive rows of j, so the per-plane bookkeeping (barrier,
// staging, ring rotation, plane-uniform tests) is paid once per R cells and a
// thread's own H values of the two previous planes stay in registers.  One
// more "halo" warp recomputes the H values the tile's E update needs from the
// neighbouring tiles (row j0-1 and column k0-1), so no CTA waits for another.
// For every plane i:
//   * staging: the six components and the material ids of plane i+3 are copied
//     into a 4-deep shared-memory ring with cp.async (planes i, i+1 resident,
//     i+2, i+3 in flight), rows j0-1 .. j0+TJ and a 16-byte aligned k window.
//   * H pass (plane i): H^{n+1/2} of the tile and its low halos, into a
//     2-plane shared ring (for the neighbours' reads), into registers (for the
//     thread's own E update) and, for owned cells, to HBM.
//   * E pass (plane i-1, one plane behind): E^{n+1} of the owned cells from the
//     H planes i-1 and i-2 and E^n taken from the ring one iteration earlier.
//     With the skew, the H and E passes of an iteration touch disjoint shared
//     data: one barrier per plane.
// Fields and the H-side CPML psi are ping-pong buffered (read set s, write set
// d) so a neighbour's halo reads never see a half-updated value; E-side psi,
// ADE state and material ids are only touched by their owner.
//
// Work comes as a list of items (tile column, plane range), one CTA each, and
// the kernel is specialised by the kind of region its items cover: KIND bit 1
// = planes of the x CPML slabs, bit 2 = columns touching the y/z CPML slabs,
// bit 4 = the box of dispersive (ADE) cells.  The host classifies the grid so
// that every item (with its halo plane, row and column) needs no more than its
// kind compiles in; TFSF is handled by every kind.
//
// The per-cell arithmetic (hNext/eNext, TFSF, CPML, ADE and their order) is the
// one of k_h3/k_e3, so results are identical to the split path and, in FP64,
// to the CPU restatement bit for bit.
#pragma once

#include <cuda.h>  // CUtensorMap

#include "kernels.cuh"

namespace xfb {

// Tensor maps of the staging copies of one field set and tile shape: the six
// components and the material ids as 3-D tensors (k, j, i) over the padded
// layout, boxes of one plane's staged window (zero fill outside the grid).
struct StageMaps {
  CUtensorMap f[6];
  CUtensorMap mid;
};

// Tensor maps of the bulk stores of the lean interior body: the six
// components of the write set (Ex Ey Ez Hx Hy Hz), box 32 x TJ x 1.
struct StoreMaps {
  CUtensorMap f[6];
};

// Tensor maps of the TFSF line tables (k_tfsf_lines): yh, ye as 4-D tensors
// (k, component, i, face), box (34 x 2 x 1 x 1) from k0 - 2; zh, ze as
// (j, component, i, face), box (TJ + 2) x 2 x 1 x 1 from j0 - 2.
struct LineMaps {
  CUtensorMap yh, ye, zh, ze;
};

__device__ __forceinline__ unsigned smem_u32(const void* p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* b, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(b)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory"); }
// orders this thread's earlier shared-memory accesses before later bulk
// (async-proxy) copies into or out of the same memory
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(uint64_t* b, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(b)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* b, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(b)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Default poll limit of the bounded staging waits, far beyond the latency of
// any staging copy.  The step kernels read their limit from err[1] (the
// handle's error word pair: flag, poll limit), which the host sets to this
// value at init; a smaller limit (xfb_set_wait_limit) lets a test make the
// waits run out.
constexpr int kWaitPolls = 1 << 22;
// Bounded wait for phase `parity` of barrier b: false after `polls` polls
// (the copies then never completed).
__device__ __forceinline__ bool mbar_wait(uint64_t* b, unsigned parity, int polls = kWaitPolls) {
  for (int n = 0; n < polls; ++n)
    if (mbar_try_wait(b, parity)) return true;
  return false;
}
// Tiled bulk copy of one box of a 3-D tensor into shared memory, completing
// on barrier `bar`, into this CTA's shared memory only.
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int x, int y, int z, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
      "[%5];\n" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void tma_load_4d(void* dst, const CUtensorMap* map, int x, int y, int z, int w,
                                            uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
      "[%6];\n" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(w), "r"(smem_u32(bar))
      : "memory");
}
// Tiled bulk store of one box from shared memory (bulk-group completion).
__device__ __forceinline__ void tma_store_3d(const CUtensorMap* map, const void* src, int x, int y, int z) {
  asm volatile("cp.async.bulk.tensor.3d.global.shared::cta.bulk_group [%0, {%2, %3, %4}], [%1];\n" ::"l"(
                   reinterpret_cast<uint64_t>(map)),
               "r"(smem_u32(src)), "r"(x), "r"(y), "r"(z)
               : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;\n" ::: "memory"); }
// the committed bulk stores have read their shared-memory sources
__device__ __forceinline__ void bulk_wait_read() { asm volatile("cp.async.bulk.wait_group.read 0;\n" ::: "memory"); }
// ... and completed their global writes
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;\n" ::: "memory"); }

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

template <typename T>
struct PsiH {  // H-side CPML psi of one buffer set
  T* hy_x; T* hz_x; T* hz_y; T* hx_y; T* hx_z; T* hy_z;
};

// One-sweep 2-D TMz step: the H and E half-steps of a Yee step in one
// launch (the TFSF incident fields come from the precomputed tables).  A block owns 128
// columns j0 .. j0+127 over a chunk of planes [i0, i1) and marches along i;
// thread t holds column j0 - 1 + t, thread 0 the halo column whose Hx the
// first column's Ez update needs, so no block reads what another writes in
// the same launch: fields and H-side psi are ping-pong buffered (read s / ps,
// write d / pd; the E-side psi has one owner per cell).  At plane i a thread
// computes H of plane i (Hx from Ez(i, j+1) - Ez(i, j), Hy from Ez(i+1, j) -
// Ez(i, j), both from the read set) and then Ez of plane i from Hy(i) -
// Hy(i-1) (its own registers) and Hx(i, j) - Hx(i, j-1) (its left
// neighbour's, through shared memory): one barrier per plane.  The march
// starts a plane early (i0 - 1) for Hy(i0 - 1).  PEC wall entries (i = 0 or
// j = 0 for Ez) are never written, so both sets keep their value.  The
// arithmetic and its order are those of k_h2 and k_e2.
template <typename T>
__global__ void __launch_bounds__(160) k_step2(GridP<T> s, GridP<T> d, PmlP<T> pm, PsiH<T> ps, PsiH<T> pd,
                                               TfsfP tf_in, TimeP tp, int i_chunk, int n_mat) {
  const TfsfP tf = tfsf_at_step(tf_in, cur_step(tp));
  __shared__ T hxs[2][160];
  extern __shared__ __align__(16) unsigned char k2_smem[];
  T* lut = reinterpret_cast<T*>(k2_smem);  // [n_mat][18] coefficients
  const int t = threadIdx.x;
  const int j = blockIdx.x * 128 + t - 1;
  const int i0 = blockIdx.y * i_chunk;
  const int i1 = min(s.nx, i0 + i_chunk);
  if (i0 >= i1) return;  // the whole block
  for (int q = t; q < n_mat * 18; q += blockDim.x) lut[q] = s.lut[q];
  const bool hcol = t <= 128 && j >= 0 && j < s.ny;  // H of this column is computed
  const bool own = hcol && t >= 1;                    // and written, with its Ez
  const long long sx = s.sx;
  const int sy_pml = hcol ? slab(j, s.ny, pm.L[2], pm.L[3]) : -1;
  // TFSF lines through this column (the plane tests are made once per plane)
  const bool tf_jin = tf.on && j >= tf.js && j <= tf.je;
  const bool tf_hline = tf.on && (j == tf.js - 1 || j == tf.je);  // Hx corrections
  const bool tf_eline = tf.on && (j == tf.js || j == tf.je);      // Ez corrections
  const int ib = i0 > 0 ? i0 - 1 : 0;
  // plane i's inputs, loaded one iteration ahead: Ez(i, j), Ez(i+1, j),
  // Ez(i, j+1), Hx(i, j), Hy(i, j), material id
  T ez_c = T(0), ez_n = T(0), ez_j1 = T(0), hx_o = T(0), hy_o = T(0);
  int m = 0;
  if (hcol) {
    const long long x0 = static_cast<long long>(ib) * sx + j;
    ez_c = s.ez[x0]; ez_n = s.ez[x0 + sx]; ez_j1 = s.ez[x0 + 1]; hx_o = s.hx[x0]; hy_o = s.hy[x0];
    m = s.mid[x0];
  }
  __syncthreads();  // shared LUT ready
  T hy_prev = T(0);
  for (int i = ib; i < i1; ++i) {
    const long long idx = static_cast<long long>(i) * sx + j;
    const bool in_range = i >= i0;
    const bool wr = own && in_range;
    T nez_n = T(0), nez_j1 = T(0), nhx = T(0), nhy = T(0);
    int nm = 0;
    if (hcol && i + 1 < i1) {  // plane i+1
      const long long x1 = idx + sx;
      nez_n = s.ez[x1 + sx]; nez_j1 = s.ez[x1 + 1]; nhx = s.hx[x1]; nhy = s.hy[x1];
      nm = s.mid[x1];
    }
    const int sx_pml = slab(i, s.nx, pm.L[0], pm.L[1]);  // plane-uniform
    const bool tf_iin = tf.on && i >= tf.is && i <= tf.ie;
    const bool tf_hplane = tf.on && (i == tf.is - 1 || i == tf.ie);
    const bool tf_eplane = tf.on && (i == tf.is || i == tf.ie);
    T hxv = T(0), hyv = T(0);
    const T* c = lut + 18 * m;
    if (hcol) {
      const T d_hx_b = ez_j1 - ez_c;  // Hx from Ez along y
      const T d_hy_a = ez_n - ez_c;   // Hy from Ez along x
      hxv = c[9] * hx_o + c[11] * d_hx_b;
      hyv = c[12] * hy_o + c[13] * d_hy_a;
      if ((tf_hplane && tf_jin) || (tf_hline && tf_iin)) {
        if (tf_jin) {
          if (i == tf.is - 1) add_inc(hyv, ez_inc(tf, tf.is, j, 0), -tf.cb[0]);
          if (i == tf.ie) add_inc(hyv, ez_inc(tf, tf.ie, j, 0), tf.cb[0]);
        }
        if (tf_iin) {
          if (j == tf.js - 1) add_inc(hxv, ez_inc(tf, i, tf.js, 0), tf.cb[1]);
          if (j == tf.je) add_inc(hxv, ez_inc(tf, i, tf.je, 0), -tf.cb[1]);
        }
      }
      if (sx_pml >= 0) {
        const long long p = sx_pml * sx + j;
        T py = pm.bh[0][i] * ps.hy_x[p] + pm.ah[0][i] * d_hy_a;
        if (wr) pd.hy_x[p] = py;
        hyv = hyv + c[13] * py;
      }
      if (sy_pml >= 0) {
        const long long p = static_cast<long long>(i) * pm.ysx + sy_pml;
        T px = pm.bh[1][j] * ps.hx_y[p] + pm.ah[1][j] * d_hx_b;
        if (wr) pd.hx_y[p] = px;
        hxv = hxv + c[11] * px;
      }
      if (wr) {
        d.hx[idx] = hxv;
        d.hy[idx] = hyv;
      }
    }
    hxs[i & 1][t] = hxv;
    __syncthreads();
    if (wr && i > 0 && j > 0) {
      const T hx_c = hxv, hx_jm = hxs[i & 1][t - 1];
      const T hy_c = hyv, hy_p = hy_prev;
      const T d_ez_a = hx_c - hx_jm;
      const T d_ez_b = hy_c - hy_p;
      T ezv = c[6] * ez_c + c[7] * d_ez_a + c[8] * d_ez_b;
      if ((tf_eplane && tf_jin) || (tf_eline && tf_iin)) {
        if (tf_jin) {
          if (i == tf.is) add_inc(ezv, hy_inc(tf, tf.is - 1, j, 0), -tf.ca[0]);
          if (i == tf.ie) add_inc(ezv, hy_inc(tf, tf.ie, j, 0), tf.ca[0]);
        }
        if (tf_iin) {
          if (j == tf.js) add_inc(ezv, hx_inc(tf, i, tf.js - 1, 0), tf.ca[1]);
          if (j == tf.je) add_inc(ezv, hx_inc(tf, i, tf.je, 0), -tf.ca[1]);
        }
      }
      if (sx_pml >= 0) {
        const long long p = sx_pml * sx + j;
        T q = pm.be[0][i] * pm.ez_x[p] + pm.ae[0][i] * d_ez_b;
        pm.ez_x[p] = q;
        ezv = ezv + c[8] * q;
      }
      if (sy_pml >= 0) {
        const long long p = static_cast<long long>(i) * pm.ysx + sy_pml;
        T q = pm.be[1][j] * pm.ez_y[p] + pm.ae[1][j] * d_ez_a;
        pm.ez_y[p] = q;
        ezv = ezv + c[7] * q;
      }
      d.ez[idx] = ezv;
    }
    hy_prev = hyv;
    ez_c = ez_n; ez_n = nez_n; ez_j1 = nez_j1; hx_o = nhx; hy_o = nhy; m = nm;
  }
}

// Four coefficients of one half of the compact LUT (E: ce, cb/dx, cb/dy, cb/dz;
// H: ch, db/dx, db/dy, db/dz), read from shared memory with vector loads.
template <typename T>
struct C4 {
  T c, x, y, z;
};
__device__ __forceinline__ C4<float> ld_c4(const float* p) {
  const float4 v = *reinterpret_cast<const float4*>(p);
  return {v.x, v.y, v.z, v.w};
}
__device__ __forceinline__ C4<double> ld_c4(const double* p) {
  const double2 a = *reinterpret_cast<const double2*>(p);
  const double2 b = *reinterpret_cast<const double2*>(p + 2);
  return {a.x, a.y, b.x, b.y};
}

// Geometry and shared-memory layout of k_step3 (dynamic shared memory).
template <typename T, int R, int NWM, int NS_>
struct StepCfg {
  static constexpr int TK = 32, TJ = R * NWM;
  static constexpr int NS = NS_;             // staging ring depth (planes)
  static constexpr int HP = 16 / sizeof(T);  // elements per 16-byte copy
  static constexpr int RW = TK + 2 * HP;     // staged row width: k0-HP .. k0+TK+HP
  static constexpr int RH = TJ + 2;          // staged rows j0-1 .. j0+TJ
  static constexpr int MW = TK + 32;         // material-id row window [k0-16, k0+TK+16)
  static constexpr int HW = TK + 1, HH = TJ + 1;  // shared H plane: row 0 = j0-1, column 0 = k0-1
  static constexpr int HPL = HH * HW;
  static constexpr int LUTM = 16;            // materials whose coefficients sit in shared memory
  static constexpr int CW = RW / HP;         // 16-byte chunks per staged field row
  static constexpr int MC = MW / 16;         // 16-byte chunks per material row
  static constexpr int PLA = 128 / sizeof(T);
  // elements of one staged component plane, rounded up so every plane of the
  // ring starts on a 128-byte boundary (bulk-copy destinations)
  static constexpr int PL = (RH * RW + PLA - 1) / PLA * PLA;
  static constexpr int NT = (NWM + 1) * 32;  // row warps + halo warp
  // shared memory, from a 128-byte aligned base: field ring [NS][6][PL],
  // material ring [NS][MPL], NS staging barriers, H planes, E planes of
  // the lean interior body, LUT [LUTM][8], dispersive flags [LUTM]
  static constexpr size_t f_bytes = static_cast<size_t>(NS) * 6 * PL * sizeof(T);
  // material plane of the ring, rounded up so every plane starts on a
  // 128-byte boundary (bulk-copy destinations)
  static constexpr int MPL = (RH * MW + 127) / 128 * 128;
  static constexpr size_t m_bytes = static_cast<size_t>(NS) * MPL;
  static constexpr size_t h_bytes = (2ull * 3 * HPL * sizeof(T) + 15) / 16 * 16;
  static constexpr size_t l_bytes = LUTM * 8 * sizeof(T);
  static constexpr size_t d_bytes = LUTM;
  // lean interior body: H planes [2][3][LCS] (per component a dense TJ x 32
  // tile, then the halo row j0-1 and the halo column k0-1, 32 slots each) and
  // E planes [2][3][TJ][32], both the sources of bulk stores
  static constexpr int LCS = (TJ + 2) * 32;
  static constexpr size_t lh_bytes = 2ull * 3 * LCS * sizeof(T);
  static constexpr size_t le_bytes = 2ull * 3 * TJ * 32 * sizeof(T);
  static constexpr size_t hr_bytes = (h_bytes > lh_bytes ? h_bytes : lh_bytes);
  static constexpr size_t off_m = f_bytes, off_b = f_bytes + m_bytes;
  static constexpr size_t off_h = (off_b + 8 * NS + 127) / 128 * 128;
  static constexpr size_t off_e = off_h + (hr_bytes + 127) / 128 * 128;
  static constexpr size_t off_l = off_e + le_bytes, off_d = off_l + l_bytes;
  // CPML profile coefficients (ah, bh, ae, be) of the tile's rows or columns
  // with their halo, for the CPML column bodies of step_item_fast
  static constexpr int NC = 40;
  static constexpr size_t off_c = (off_d + d_bytes + 15) / 16 * 16;
  static constexpr size_t c_bytes = 8 * NC * sizeof(T);  // column axis, and z of a corner tile
  // TFSF line values of the items on the TFSF surface, a ring of NS slots
  // filled with the planes: per slot the y-line box (2 components x YW
  // doubles from k0 - 2) of the H pass at the slot's plane i and of the E pass
  // at plane i - 1, then the z-line boxes (2 x ZW from j0 - 2) likewise, each
  // box 128-byte aligned
  static constexpr int YW = TK + 2, ZW = TJ + 2;
  static constexpr int YB = (2 * YW * 8 + 127) / 128 * 128, ZB = (2 * ZW * 8 + 127) / 128 * 128;
  static constexpr int LSLOT = 2 * YB + 2 * ZB;
  static constexpr size_t off_t = (off_c + c_bytes + 127) / 128 * 128;
  static constexpr size_t bytes = off_t + static_cast<size_t>(NS) * LSLOT + 128;  // + alignment slack of the base
  static_assert((ZW * 8) % 16 == 0, "z-line boxes span whole 16-byte granules");
  static_assert(NC >= RH && NC >= TK + 1, "coefficient table covers the tile with its halo");
  // bytes one staged plane brings (six field boxes and the material box)
  static constexpr unsigned tx_bytes = static_cast<unsigned>(6 * RH * RW * sizeof(T) + RH * MW);
  // CTAs per SM that the 228 KB of shared memory per SM admits (1 KB reserved
  // per CTA), at most 4; the register budget is sized for that residency
  static constexpr int fit = static_cast<int>((228u * 1024u) / (bytes + 1024u));
  static constexpr int min_blocks = fit < 1 ? 1 : fit > 4 ? 4 : fit;
  static_assert(TJ <= 32, "the halo warp covers the k0-1 column with one lane per row");
  static_assert(R >= 2, "the halo warp computes two H cells per plane");
  static_assert(NS >= 3, "planes i and i+1 in use while one more is in flight");
};

// Everything an H-cell update reads (references to the launch's parameters,
// so nothing is copied to local memory).
template <typename T>
struct HCtx {
  const GridP<T>& s;
  const GridP<T>& d;
  const PmlP<T>& pm;
  const PsiH<T>& ps;
  const PsiH<T>& pd;
  const TfsfP& tf;
};

// Per-thread constants of one cell of the tile, computed once per CTA.
struct Cell {
  int wf;  // staged-ring offset of (j, k) inside a component plane
  int mo;  // material-ring offset inside a plane
  int hs;  // shared-H-plane offset
  int go;  // global offset inside a field plane (j * sy + k)
  int j, k;
  int py, pz;  // y / z CPML slab index of the cell, or -1
  int tfl;     // bit 0: on a TFSF H correction line (j = js-1, je or k = ks-1, ke); bit 1: E line (js, je, ks, ke)
};

// TFSF H corrections of cell (i, jj, kk), in the reference's agency order
// (TFSFCorrector3DAgency::correctH, src/waveform_source/tfsf/tfsf_corrector.cu:237-271);
// the incident fields come from `in`.
template <typename T, class Inc>
__device__ __forceinline__ void tfsf_h(const TfsfP& tf, const Inc& in, int i, int jj, int kk, T& hxv, T& hyv, T& hzv) {
  const bool iin = i >= tf.is && i <= tf.ie, jin = jj >= tf.js && jj <= tf.je, kin = kk >= tf.ks && kk <= tf.ke;
  if (jin && jj < tf.je && kin) {
    if (i == tf.is - 1) add_inc(hzv, in.ey(tf.is, jj, kk), tf.cb[0]);
    if (i == tf.ie) add_inc(hzv, in.ey(tf.ie, jj, kk), -tf.cb[0]);
  }
  if (iin && i < tf.ie && kin) {
    if (jj == tf.js - 1) add_inc(hzv, in.ex(i, tf.js, kk), -tf.cb[1]);
    if (jj == tf.je) add_inc(hzv, in.ex(i, tf.je, kk), tf.cb[1]);
  }
  if (iin && jin && jj < tf.je) {
    if (kk == tf.ks - 1) add_inc(hxv, in.ey(i, jj, tf.ks), -tf.cb[2]);
    if (kk == tf.ke) add_inc(hxv, in.ey(i, jj, tf.ke), tf.cb[2]);
  }
  if (iin && kin && kk < tf.ke) {
    if (jj == tf.js - 1) add_inc(hxv, in.ez(i, tf.js, kk), tf.cb[1]);
    if (jj == tf.je) add_inc(hxv, in.ez(i, tf.je, kk), -tf.cb[1]);
  }
  if (iin && i < tf.ie && jin) {
    if (kk == tf.ks - 1) add_inc(hyv, in.ex(i, jj, tf.ks), tf.cb[2]);
    if (kk == tf.ke) add_inc(hyv, in.ex(i, jj, tf.ke), -tf.cb[2]);
  }
  if (jin && kin && kk < tf.ke) {
    if (i == tf.is - 1) add_inc(hyv, in.ez(tf.is, jj, kk), -tf.cb[0]);
    if (i == tf.ie) add_inc(hyv, in.ez(tf.ie, jj, kk), tf.cb[0]);
  }
}

// TFSF E corrections of cell (i, j, k) (TFSFCorrector3DAgency::correctE,
// src/waveform_source/tfsf/tfsf_corrector.cu:201-236).
template <typename T, class Inc>
__device__ __forceinline__ void tfsf_e(const TfsfP& tf, const Inc& in, int i, int j, int k, T& exv, T& eyv, T& ezv) {
  const bool iin = i >= tf.is && i <= tf.ie, jin = j >= tf.js && j <= tf.je, kin = k >= tf.ks && k <= tf.ke;
  if (jin && kin && k < tf.ke) {
    if (i == tf.is) add_inc(ezv, in.hy(tf.is - 1, j, k), -tf.ca[0]);
    if (i == tf.ie) add_inc(ezv, in.hy(tf.ie, j, k), tf.ca[0]);
  }
  if (iin && kin && k < tf.ke) {
    if (j == tf.js) add_inc(ezv, in.hx(i, tf.js - 1, k), tf.ca[1]);
    if (j == tf.je) add_inc(ezv, in.hx(i, tf.je, k), -tf.ca[1]);
  }
  if (iin && i < tf.ie && jin) {
    if (k == tf.ks) add_inc(exv, in.hy(i, j, tf.ks - 1), tf.ca[2]);
    if (k == tf.ke) add_inc(exv, in.hy(i, j, tf.ke), -tf.ca[2]);
  }
  if (iin && i < tf.ie && kin) {
    if (j == tf.js) add_inc(exv, in.hz(i, tf.js - 1, k), -tf.ca[1]);
    if (j == tf.je) add_inc(exv, in.hz(i, tf.je, k), tf.ca[1]);
  }
  if (iin && jin && j < tf.je) {
    if (k == tf.ks) add_inc(eyv, in.hx(i, j, tf.ks - 1), -tf.ca[2]);
    if (k == tf.ke) add_inc(eyv, in.hx(i, j, tf.ke), tf.ca[2]);
  }
  if (jin && j < tf.je && kin) {
    if (i == tf.is) add_inc(eyv, in.hz(tf.is - 1, j, k), tf.ca[0]);
    if (i == tf.ie) add_inc(eyv, in.hz(tf.ie, j, k), -tf.ca[0]);
  }
}

// TFSF line values of one plane, staged in shared memory from the line
// tables: the two components of the tile's y line (from k0 - 2, pitch yw)
// and of its z line (from j0 - 2, pitch zw).
struct LineVals {
  const double* y;
  const double* z;
  int yw, zw, k0m2, j0m2;
};

// tfsf_h with the incident values of the y- and z-face lines taken from the
// staged lines (the x-face planes still from `in`): the same terms in the
// same order, so the result is unchanged.  yh holds (ex, ez) at the face row
// (js for the row js-1, je for je), zh (ey, ex) at the face column.
template <typename T, class Inc>
__device__ __forceinline__ void tfsf_h_lines(const TfsfP& tf, const Inc& in, const LineVals& lv, int i, int jj, int kk,
                                             T& hxv, T& hyv, T& hzv) {
  const bool iin = i >= tf.is && i <= tf.ie, jin = jj >= tf.js && jj <= tf.je, kin = kk >= tf.ks && kk <= tf.ke;
  if (jin && jj < tf.je && kin) {
    if (i == tf.is - 1) add_inc(hzv, in.ey(tf.is, jj, kk), tf.cb[0]);
    if (i == tf.ie) add_inc(hzv, in.ey(tf.ie, jj, kk), -tf.cb[0]);
  }
  if (iin && i < tf.ie && kin) {
    if (jj == tf.js - 1) add_inc(hzv, lv.y[kk - lv.k0m2], -tf.cb[1]);
    if (jj == tf.je) add_inc(hzv, lv.y[kk - lv.k0m2], tf.cb[1]);
  }
  if (iin && jin && jj < tf.je) {
    if (kk == tf.ks - 1) add_inc(hxv, lv.z[jj - lv.j0m2], -tf.cb[2]);
    if (kk == tf.ke) add_inc(hxv, lv.z[jj - lv.j0m2], tf.cb[2]);
  }
  if (iin && kin && kk < tf.ke) {
    if (jj == tf.js - 1) add_inc(hxv, lv.y[lv.yw + kk - lv.k0m2], tf.cb[1]);
    if (jj == tf.je) add_inc(hxv, lv.y[lv.yw + kk - lv.k0m2], -tf.cb[1]);
  }
  if (iin && i < tf.ie && jin) {
    if (kk == tf.ks - 1) add_inc(hyv, lv.z[lv.zw + jj - lv.j0m2], tf.cb[2]);
    if (kk == tf.ke) add_inc(hyv, lv.z[lv.zw + jj - lv.j0m2], -tf.cb[2]);
  }
  if (jin && kin && kk < tf.ke) {
    if (i == tf.is - 1) add_inc(hyv, in.ez(tf.is, jj, kk), -tf.cb[0]);
    if (i == tf.ie) add_inc(hyv, in.ez(tf.ie, jj, kk), tf.cb[0]);
  }
}

// tfsf_e likewise: ye holds (hx, hz) at the row js-1 (for the row js) or je,
// ze (hy, hx) at the column ks-1 (for ks) or ke.
template <typename T, class Inc>
__device__ __forceinline__ void tfsf_e_lines(const TfsfP& tf, const Inc& in, const LineVals& lv, int i, int j, int k,
                                             T& exv, T& eyv, T& ezv) {
  const bool iin = i >= tf.is && i <= tf.ie, jin = j >= tf.js && j <= tf.je, kin = k >= tf.ks && k <= tf.ke;
  if (jin && kin && k < tf.ke) {
    if (i == tf.is) add_inc(ezv, in.hy(tf.is - 1, j, k), -tf.ca[0]);
    if (i == tf.ie) add_inc(ezv, in.hy(tf.ie, j, k), tf.ca[0]);
  }
  if (iin && kin && k < tf.ke) {
    if (j == tf.js) add_inc(ezv, lv.y[k - lv.k0m2], tf.ca[1]);
    if (j == tf.je) add_inc(ezv, lv.y[k - lv.k0m2], -tf.ca[1]);
  }
  if (iin && i < tf.ie && jin) {
    if (k == tf.ks) add_inc(exv, lv.z[j - lv.j0m2], tf.ca[2]);
    if (k == tf.ke) add_inc(exv, lv.z[j - lv.j0m2], -tf.ca[2]);
  }
  if (iin && i < tf.ie && kin) {
    if (j == tf.js) add_inc(exv, lv.y[lv.yw + k - lv.k0m2], -tf.ca[1]);
    if (j == tf.je) add_inc(exv, lv.y[lv.yw + k - lv.k0m2], tf.ca[1]);
  }
  if (iin && jin && j < tf.je) {
    if (k == tf.ks) add_inc(eyv, lv.z[lv.zw + j - lv.j0m2], -tf.ca[2]);
    if (k == tf.ke) add_inc(eyv, lv.z[lv.zw + j - lv.j0m2], tf.ca[2]);
  }
  if (jin && j < tf.je && kin) {
    if (i == tf.is) add_inc(eyv, in.hz(tf.is - 1, j, k), tf.ca[0]);
    if (i == tf.ie) add_inc(eyv, in.hz(tf.ie, j, k), -tf.ca[0]);
  }
}

// Face of the TFSF box whose y (z) line a tile meets: 0 the low face (the H
// row js-1 among the tile's H rows j0-1 .. j0+TJ-1, or the E row js among its
// rows j0 .. j0+TJ-1), 1 the high face (je), -1 none; 2 both (tiles of boxes
// thinner than a tile, which the host gives the general body).
__device__ __host__ __forceinline__ int tfsf_line_face(int lo, int hi, int c0, int n) {
  const bool f0 = (lo - 1 >= c0 - 1 && lo - 1 <= c0 + n - 1) || (lo >= c0 && lo <= c0 + n - 1);
  const bool f1 = hi >= c0 - 1 && hi <= c0 + n - 1;
  return f0 && f1 ? 2 : f0 ? 0 : f1 ? 1 : -1;
}

// H^{n+1/2} of cell c at plane i: hNext from the staged E^n planes i and i+1
// and H^{n-1/2}, then the TFSF and CPML corrections of H.  Stores the result
// in the shared H plane; `own` also writes it (and the new H psi) to HBM
// through the plane pointers o{x,y,z}.
// (pa, p0, p1): the old H psi pair of one slab axis (0 x, 1 y, 2 z; -1 none),
// loaded one plane ahead; psi of any other slab axis is loaded here.
template <typename T, int KIND, class Cfg>
__device__ __forceinline__ void h_cell(const HCtx<T>& x, const T* Fc, const T* Fn, const uint8_t* Mc, const T* lut,
                                       T* Hc, int i, const Cell& c, bool own, T* ox, T* oy, T* oz, int sxp,
                                       bool tf_hplane, int pa, T p0, T p1, T& hxv, T& hyv, T& hzv, T& ex_c,
                                       T& ey_c, T& ez_c, int& m) {
  constexpr int PL = Cfg::PL, RW = Cfg::RW;
  m = Mc[c.mo];
  const C4<T> cf = ld_c4(lut + 8 * m + 4);  // ch, db/dx, db/dy, db/dz
  const T* f = Fc + c.wf;
  ex_c = f[0]; ey_c = f[PL]; ez_c = f[2 * PL];
  const T d_hx_a = f[PL + 1] - ey_c;          // Hx: Ey along z
  const T d_hx_b = f[2 * PL + RW] - ez_c;     // Hx: Ez along y
  const T d_hy_a = Fn[c.wf + 2 * PL] - ez_c;  // Hy: Ez along x
  const T d_hy_b = f[1] - ex_c;               // Hy: Ex along z
  const T d_hz_a = f[RW] - ex_c;              // Hz: Ex along y
  const T d_hz_b = Fn[c.wf + PL] - ey_c;      // Hz: Ey along x
  // hNext with chxey = db/dz, chxez = -db/dy, chyez = db/dx, chyex = -db/dz,
  // chzex = db/dy, chzey = -db/dx
  hxv = cf.c * f[3 * PL] + cf.z * d_hx_a - cf.y * d_hx_b;
  hyv = cf.c * f[4 * PL] + cf.x * d_hy_a - cf.z * d_hy_b;
  hzv = cf.c * f[5 * PL] + cf.y * d_hz_a - cf.x * d_hz_b;
  const TfsfP& tf = x.tf;
  const int j = c.j, k = c.k;
  if (((KIND & 16) != 0) && (tf_hplane || (c.tfl & 1))) tfsf_h(tf, IncTables{tf}, i, j, k, hxv, hyv, hzv);
  constexpr bool PX = (KIND & 1) != 0, PY = (KIND & 2) != 0, PZ = (KIND & 8) != 0;
  if (PX || PY || PZ) {
    const PmlP<T>& pm = x.pm;
    const long long sx = x.s.sx, sy = x.s.sy;
    const int hsy = PY ? c.py : -1;
    const int hsz = PZ ? c.pz : -1;
    if (!PX) sxp = -1;
    if (sxp >= 0 || hsy >= 0 || hsz >= 0) {
      if (sxp >= 0) {
        const long long p = sxp * sx + c.go;
        const T a = pm.ah[0][i], b = pm.bh[0][i];
        const T py = b * (pa == 0 ? p0 : x.ps.hy_x[p]) + a * d_hy_a;
        hyv = hyv + cf.x * py;   // c_psi = chyez
        const T pz = b * (pa == 0 ? p1 : x.ps.hz_x[p]) + a * d_hz_b;
        hzv = hzv - cf.x * pz;   // c_psi = chzey
        if (own) { x.pd.hy_x[p] = py; x.pd.hz_x[p] = pz; }
      }
      if (hsy >= 0) {
        const long long p = static_cast<long long>(i) * pm.ysx + hsy * sy + k;
        const T a = pm.ah[1][j], b = pm.bh[1][j];
        const T pz = b * (pa == 1 ? p0 : x.ps.hz_y[p]) + a * d_hz_a;
        hzv = hzv + cf.y * pz;   // chzex
        const T px = b * (pa == 1 ? p1 : x.ps.hx_y[p]) + a * d_hx_b;
        hxv = hxv - cf.y * px;   // chxez
        if (own) { x.pd.hz_y[p] = pz; x.pd.hx_y[p] = px; }
      }
      if (hsz >= 0) {
        const long long p = static_cast<long long>(i) * pm.zsx + static_cast<long long>(j) * pm.zsy + hsz;
        const T a = pm.ah[2][k], b = pm.bh[2][k];
        const T px = b * (pa == 2 ? p0 : x.ps.hx_z[p]) + a * d_hx_a;
        hxv = hxv + cf.z * px;   // chxey
        const T py = b * (pa == 2 ? p1 : x.ps.hy_z[p]) + a * d_hy_b;
        hyv = hyv - cf.z * py;   // chyex
        if (own) { x.pd.hx_z[p] = px; x.pd.hy_z[p] = py; }
      }
    }
  }
  Hc[c.hs] = hxv;
  Hc[Cfg::HPL + c.hs] = hyv;
  Hc[2 * Cfg::HPL + c.hs] = hzv;
  if (own) {
    ox[c.go] = hxv; oy[c.go] = hyv; oz[c.go] = hzv;
  }
}

// Old H psi pair of cell c at plane ip for one slab axis, preferring y, then
// z, then x (the axis whose slab holds the whole tile row, column or plane):
// returns the axis or -1.
template <typename T, int KIND>
__device__ __forceinline__ int prefetch_h_psi(const HCtx<T>& x, int ip, int sxp, const Cell& c, bool valid, T& v0, T& v1) {
  constexpr bool PX = (KIND & 1) != 0, PY = (KIND & 2) != 0, PZ = (KIND & 8) != 0;
  if (!valid) return -1;
  const PmlP<T>& pm = x.pm;
  if (PY && c.py >= 0) {
    const long long p = static_cast<long long>(ip) * pm.ysx + c.py * x.s.sy + c.k;
    v0 = x.ps.hz_y[p]; v1 = x.ps.hx_y[p];
    return 1;
  }
  if (PZ && c.pz >= 0) {
    const long long p = static_cast<long long>(ip) * pm.zsx + static_cast<long long>(c.j) * pm.zsy + c.pz;
    v0 = x.ps.hx_z[p]; v1 = x.ps.hy_z[p];
    return 2;
  }
  if (PX && sxp >= 0) {
    const long long p = sxp * x.s.sx + c.go;
    v0 = x.ps.hy_x[p]; v1 = x.ps.hz_x[p];
    return 0;
  }
  return -1;
}

// E psi pair of cell c at plane ip, same axis preference; the pair is the one
// the E update reads first for that axis (y: ez, ex; z: ex, ey; x: ey, ez).
template <typename T, int KIND>
__device__ __forceinline__ int prefetch_e_psi(const PmlP<T>& pm, const GridP<T>& s, int ip, int sxe, const Cell& c,
                                              bool valid, T& v0, T& v1) {
  constexpr bool PX = (KIND & 1) != 0, PY = (KIND & 2) != 0, PZ = (KIND & 8) != 0;
  if (!valid) return -1;
  if (PY && c.py >= 0) {
    const long long p = static_cast<long long>(ip) * pm.ysx + c.py * s.sy + c.k;
    v0 = pm.ez_y[p]; v1 = pm.ex_y[p];
    return 1;
  }
  if (PZ && c.pz >= 0) {
    const long long p = static_cast<long long>(ip) * pm.zsx + static_cast<long long>(c.j) * pm.zsy + c.pz;
    v0 = pm.ex_z[p]; v1 = pm.ey_z[p];
    return 2;
  }
  if (PX && sxe >= 0) {
    const long long p = sxe * s.sx + c.go;
    v0 = pm.ey_x[p]; v1 = pm.ez_x[p];
    return 0;
  }
  return -1;
}

// One work item of the one-sweep step, compiled for region kind KIND.
// TMA: staging by tiled bulk copies from `maps` (one thread issues a plane's
// seven boxes, a barrier per ring slot counts their bytes); otherwise every
// thread stages 16-byte chunks with cp.async.  A staging wait that runs out
// (after err[1] polls) sets err[0] = 1 and ends the item after the copies in
// flight have landed (those waits use the default limit).
template <typename T, int R, int NWM, int NS_, int KIND, bool TMA>
__device__ __forceinline__ void step_item(const GridP<T>& s, const GridP<T>& d, const PmlP<T>& pm, const PsiH<T>& ps,
                                          const PsiH<T>& pd, const TfsfP& tf, const AdeP<T>& ad, int4 item,
                                          const T* lut8, const uint8_t* disp, int n_mat, const StageMaps* maps,
                                          int* err) {
  constexpr bool PX = (KIND & 1) != 0, PY = (KIND & 2) != 0, PZ = (KIND & 8) != 0, PML = PX || PY || PZ;
  constexpr bool TFC = (KIND & 16) != 0;  // TFSF corrections compiled in
  using L = StepCfg<T, R, NWM, NS_>;
  constexpr int NS = L::NS, HP = L::HP, RW = L::RW, RH = L::RH, MW = L::MW, HW = L::HW, TK = L::TK, TJ = L::TJ;
  constexpr int CW = L::CW, MC = L::MC, NT = L::NT, PL = L::PL, HPL = L::HPL;
  constexpr int NFC = (RH * CW + NT - 1) / NT;  // staged field chunks per thread
  constexpr int NMC = (RH * MC + NT - 1) / NT;  // staged material chunks per thread
  extern __shared__ __align__(16) unsigned char smem_raw[];
  unsigned char* base = smem_raw + ((128u - (smem_u32(smem_raw) & 127u)) & 127u);
  T* sF = reinterpret_cast<T*>(base);                               // [NS][6][PL]
  uint8_t* sM = base + L::off_m;                                    // [NS][MPL]: RH rows of MW
  uint64_t* bar = reinterpret_cast<uint64_t*>(base + L::off_b);     // [NS]
  T* sH = reinterpret_cast<T*>(base + L::off_h);                    // [2][3][HH][HW]
  T* sL = reinterpret_cast<T*>(base + L::off_l);                    // [LUTM][8]
  uint8_t* sD = base + L::off_d;                                    // [LUTM]
  static_assert(L::off_h + L::h_bytes <= L::off_e, "H planes inside their region");

  const HCtx<T> x{s, d, pm, ps, pd, tf};
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int k0 = (item.x & 0xffff) * TK, j0 = item.y * TJ;
  const int i_start = item.z, i_end = item.w;
  const int i_first = i_start > 0 ? i_start - 1 : 0;
  const long long sx = s.sx;
  const int sy = static_cast<int>(s.sy);
  const bool lut_shared = n_mat <= L::LUTM;
  if (lut_shared) {
    for (int q = tid; q < n_mat * 8; q += NT) sL[q] = lut8[q];
    for (int q = tid; q < n_mat; q += NT) sD[q] = disp[q];
  }
  const T* lut = lut_shared ? sL : lut8;          // compact coefficients per material
  const uint8_t* dtab = lut_shared ? sD : disp;   // dispersive flag per material
  for (int q = tid; q < 2 * 3 * HPL; q += NT) sH[q] = T(0);

  // staging chunks of this thread (shared and global offsets inside a plane):
  // field chunks from the first threads, material chunks from the last ones
  int fso[NFC], fgo[NFC], mso[NMC], mgo[NMC];
  bool fok[NFC], mok[NMC];
#pragma unroll
  for (int c = 0; c < NFC; ++c) {
    const int q = tid + c * NT, r = q / CW, cc = q - (q / CW) * CW;
    fok[c] = q < RH * CW;
    fso[c] = r * RW + cc * HP;
    fgo[c] = (j0 - 1 + r) * sy + (k0 - HP) + cc * HP;
  }
#pragma unroll
  for (int c = 0; c < NMC; ++c) {
    const int q = NT - 1 - tid + c * NT, r = q / MC, cc = q - (q / MC) * MC;
    mok[c] = q < RH * MC;
    mso[c] = r * MW + cc * 16;
    mgo[c] = (j0 - 1 + r) * sy + (k0 - 16) + cc * 16;
  }
  // planes i_start-1 .. i_end are read (i_end <= nx); nothing past i_end is
  // staged, but every call commits a group so the wait counts stay fixed
  if (TMA && tid == 0) {
    for (int q = 0; q < NS; ++q) mbar_init(bar + q, 1);
    fence_mbar_init();
  }
  int staged = -1;  // last plane whose copies were issued (thread 0)
  auto stage = [&](int plane, int st) {
    if (TMA) {
      if (tid == 0 && plane <= i_end) {
        staged = plane;
        fence_proxy_async();
        mbar_expect_tx(bar + st, L::tx_bytes);
        T* dst = sF + st * 6 * PL;
#pragma unroll
        for (int f = 0; f < 6; ++f) tma_load_3d(dst + f * PL, &maps->f[f], k0 - HP, j0 - 1, plane, bar + st);
        tma_load_3d(sM + st * L::MPL, &maps->mid, k0 - 16, j0 - 1, plane, bar + st);
      }
      return;
    }
    if (plane <= i_end) {
      const long long pb = static_cast<long long>(plane) * sx;
      const T* gex = s.ex + pb; const T* gey = s.ey + pb; const T* gez = s.ez + pb;
      const T* ghx = s.hx + pb; const T* ghy = s.hy + pb; const T* ghz = s.hz + pb;
      T* dst0 = sF + st * 6 * PL;
#pragma unroll
      for (int c = 0; c < NFC; ++c)
        if (fok[c]) {
          T* dst = dst0 + fso[c];
          cp_async16(dst, gex + fgo[c]);
          cp_async16(dst + PL, gey + fgo[c]);
          cp_async16(dst + 2 * PL, gez + fgo[c]);
          cp_async16(dst + 3 * PL, ghx + fgo[c]);
          cp_async16(dst + 4 * PL, ghy + fgo[c]);
          cp_async16(dst + 5 * PL, ghz + fgo[c]);
        }
      const uint8_t* gm = s.mid + pb;
#pragma unroll
      for (int c = 0; c < NMC; ++c)
        if (mok[c]) cp_async16(sM + st * L::MPL + mso[c], gm + mgo[c]);
    }
    cp_async_commit();
  };
  if (TMA) __syncthreads();  // barriers initialised before any copy or wait
  for (int q = 0; q < NS - 1; ++q) stage(i_first + q, (i_first + q) % NS);
  int slot = i_first % NS;  // ring slot of plane i
  // phase of the ring barrier of plane p (the slots are used in plane order)
  auto phase = [&](int p) { return static_cast<unsigned>(((p - i_first) / NS) & 1); };
  int waited = i_first - 1;  // last plane whose staging barrier was passed
  bool ok = true;
  const int polls = TMA ? err[1] : 0;  // poll limit of the staging waits
  if (TMA) {
    ok = mbar_wait(bar + slot, phase(i_first), polls);
    if (ok) waited = i_first;
  }

  // H cells of this thread: a row warp's R rows at column `lane`; the halo
  // warp's row j0-1 at column `lane` (u = 0) and column k0-1 at row `lane`
  // (u = 1).  Row warps also own the E update of their cells.
  const bool row_warp = warp < NWM;
  Cell cell[R];
  unsigned valid = 0;
#pragma unroll
  for (int u = 0; u < R; ++u) {
    const int rr = row_warp ? warp * R + u : (u == 0 ? -1 : lane);
    const int cc = row_warp ? lane : (u == 0 ? lane : -1);
    const int j = j0 + rr, k = k0 + cc;
    bool ok;
    if (row_warp) ok = j < s.ny && k < s.nz;
    else if (u == 0) ok = j0 > 0 && k < s.nz;
    else ok = u == 1 && lane < TJ && k0 > 0 && j < s.ny;
    valid |= ok ? 1u << u : 0u;
    cell[u].wf = (rr + 1) * RW + cc + HP;
    cell[u].mo = (rr + 1) * MW + cc + 16;
    cell[u].hs = (rr + 1) * HW + cc + 1;
    cell[u].go = j * sy + k;
    cell[u].j = j;
    cell[u].k = k;
    cell[u].py = PY ? slab(j, s.ny, pm.L[2], pm.L[3]) : -1;
    cell[u].pz = PZ ? slab(k, s.nz, pm.L[4], pm.L[5]) : -1;
    cell[u].tfl = TFC && tf.on ? ((j == tf.js - 1 || j == tf.je || k == tf.ks - 1 || k == tf.ke) ? 1 : 0) |
                              ((j == tf.js || j == tf.je || k == tf.ks || k == tf.ke) ? 2 : 0)
                        : 0;
  }
  // registers: H of the thread's own cells at planes i (new), i-1, i-2 (y, z only)
  T hnx[R], hny[R], hnz[R], hpx[R], hpy[R], hpz[R], hqy[R], hqz[R];
  T eox[R], eoy[R], eoz[R];  // E^n of plane i-1, taken from the ring one iteration earlier
  int em[R];                 // material of those cells
  T enx[R], eny[R], enz[R];  // E^n of plane i, read by the H pass
  int enm[R];
  // CPML psi pairs loaded one plane ahead (axis -1: none)
  T ph0[R], ph1[R], pe0[R], pe1[R];
  int pha[R], pea[R];
#pragma unroll
  for (int u = 0; u < R; ++u) {
    hnx[u] = hny[u] = hnz[u] = hpx[u] = hpy[u] = hpz[u] = hqy[u] = hqz[u] = T(0);
    eox[u] = eoy[u] = eoz[u] = T(0);
    enx[u] = eny[u] = enz[u] = T(0);
    enm[u] = 0;
    ph0[u] = ph1[u] = pe0[u] = pe1[u] = T(0);
    pha[u] = pea[u] = -1;
    em[u] = 0;
  }
  const bool has_ade = (KIND & 4) != 0 && ad.kind != kAdeNone;
  if (PML) {
    const int sxp = PX ? slab(i_first, s.nx, pm.L[0], pm.L[1]) : -1;
#pragma unroll
    for (int u = 0; u < R; ++u)
      pha[u] = prefetch_h_psi<T, KIND>(x, i_first, sxp, cell[u], (valid >> u) & 1u, ph0[u], ph1[u]);
  }

  // Iteration i computes H of plane i and E of plane i-1 (skewed by one plane,
  // so the E pass only reads H planes finished before the iteration's barrier).
  for (int i = i_first; i <= i_end; ++i) {
    const int ie = i - 1;
    const bool do_h = i < i_end;
    const bool write_h = do_h && i >= i_start && row_warp;
    const int slot_n = slot + 1 == NS ? 0 : slot + 1;      // plane i+1
    const int slot_p = slot == 0 ? NS - 1 : slot - 1;      // plane i-1, refilled with plane i+NS-1
    if (TMA) {
      if (i + 1 <= i_end && ok) {  // plane i+1 has landed (plane i did one iteration earlier)
        ok = mbar_wait(bar + slot_n, phase(i + 1), polls);
        if (ok) waited = i + 1;
      }
      // every thread saw its planes land; iteration i-1 is complete everywhere
      if (__syncthreads_or(!ok)) {
        ok = false;
        break;
      }
    } else {
      cp_async_wait<NS - 3>();  // planes i and i+1 have landed (this thread's copies)
      __syncthreads();          // ... everyone's copies; iteration i-1 is complete everywhere
    }
    stage(i + NS - 1, slot_p);  // whose last readers finished iteration i-1
    const T* Fc = sF + slot * 6 * PL;
    const T* Fn = sF + slot_n * 6 * PL;
    const uint8_t* Mc = sM + slot * L::MPL;
    slot = slot_n;
    T* Hc = sH + (i & 1) * 3 * HPL;              // H plane i (written here)
    const T* Hq = sH + ((i + 1) & 1) * 3 * HPL;  // H plane i-1
    // ---- H pass, plane i ----------------------------------------------------
    if (do_h) {
      const int sxp = PX ? slab(i, s.nx, pm.L[0], pm.L[1]) : -1;
      const bool tf_hplane = TFC && tf.on && (i == tf.is - 1 || i == tf.ie);
      const long long pb = static_cast<long long>(i) * sx;
      T* ox = d.hx + pb; T* oy = d.hy + pb; T* oz = d.hz + pb;
#pragma unroll
      for (int u = 0; u < R; ++u)
        if ((valid >> u) & 1u)
          h_cell<T, KIND, L>(x, Fc, Fn, Mc, lut, Hc, i, cell[u], write_h, ox, oy, oz, sxp, tf_hplane, pha[u], ph0[u],
                             ph1[u], hnx[u], hny[u], hnz[u], enx[u], eny[u], enz[u], enm[u]);
    }
    // H psi of plane i+1, issued now that plane i's is consumed
    if (PML && i + 1 < i_end) {
      const int sxp = PX ? slab(i + 1, s.nx, pm.L[0], pm.L[1]) : -1;
#pragma unroll
      for (int u = 0; u < R; ++u)
        pha[u] = prefetch_h_psi<T, KIND>(x, i + 1, sxp, cell[u], (valid >> u) & 1u, ph0[u], ph1[u]);
    }
    // ---- E pass, plane ie = i-1 ----------------------------------------------
    if (row_warp && ie >= i_start) {
      const int sxe = PX ? slab(ie, s.nx, pm.L[0], pm.L[1]) : -1;
      const bool tf_eplane = TFC && tf.on && (ie == tf.is || ie == tf.ie);
      const long long pb = static_cast<long long>(ie) * sx;
      T* oex = d.ex + pb; T* oey = d.ey + pb; T* oez = d.ez + pb;
      const bool ipos = ie > 0;
#pragma unroll
      for (int u = 0; u < R; ++u) {
        if (!((valid >> u) & 1u)) continue;
        const Cell& c = cell[u];
        const int j = c.j, k = c.k;
        const bool jpos = j > 0, kpos = k > 0;
        const bool upd_x = jpos && kpos, upd_y = ipos && kpos, upd_z = ipos && jpos;
        const int m = em[u];
        const C4<T> cf = ld_c4(lut + 8 * m);  // ce, cb/dx, cb/dy, cb/dz
        const int hs = c.hs;
        // H^{n+1/2} of plane ie: own value from registers, k-1 from the shared
        // plane, j-1 from the previous row of this thread or the shared plane
        const T hx_c = hpx[u], hy_c = hpy[u], hz_c = hpz[u];
        const T hx_km = Hq[hs - 1], hy_km = Hq[HPL + hs - 1];
        const T hx_jm = u > 0 ? hpx[u > 0 ? u - 1 : 0] : Hq[hs - HW];
        const T hz_jm = u > 0 ? hpz[u > 0 ? u - 1 : 0] : Hq[2 * HPL + hs - HW];
        const T hy_p = hqy[u], hz_p = hqz[u];  // plane ie-1
        const T d_ex_a = hy_c - hy_km;
        const T d_ex_b = hz_c - hz_jm;
        const T d_ey_a = hz_c - hz_p;
        const T d_ey_b = hx_c - hx_km;
        const T d_ez_a = hx_c - hx_jm;
        const T d_ez_b = hy_c - hy_p;
        const T ex_o = eox[u], ey_o = eoy[u], ez_o = eoz[u];
        // eNext with cexhy = -cb/dz, cexhz = cb/dy, ceyhz = -cb/dx, ceyhx = cb/dz,
        // cezhx = -cb/dy, cezhy = cb/dx
        T exv = cf.c * ex_o - cf.z * d_ex_a + cf.y * d_ex_b;
        T eyv = cf.c * ey_o - cf.x * d_ey_a + cf.z * d_ey_b;
        T ezv = cf.c * ez_o - cf.y * d_ez_a + cf.x * d_ez_b;
        if (has_ade && dtab[m]) {
          const long long abi = static_cast<long long>(ie - ad.b0) * ad.bsx + static_cast<long long>(j - ad.b2) * ad.bsy + (k - ad.b4);
          if (upd_x) exv = ade_e(ad, 0, abi, m, ex_o, exv);
          if (upd_y) eyv = ade_e(ad, 1, abi, m, ey_o, eyv);
          if (upd_z) ezv = ade_e(ad, 2, abi, m, ez_o, ezv);
        }
        if (TFC && (tf_eplane || (c.tfl & 2))) tfsf_e(tf, IncTables{tf}, ie, j, k, exv, eyv, ezv);
        if (PML) {
          const int sy_pml = c.py, sz_pml = c.pz;
          if (sxe >= 0 || sy_pml >= 0 || sz_pml >= 0) {
            const int pa = pea[u];
            if (sxe >= 0) {
              const long long p = sxe * sx + c.go;
              const T a = pm.ae[0][ie], b = pm.be[0][ie];
              if (upd_y) { T q = b * (pa == 0 ? pe0[u] : pm.ey_x[p]) + a * d_ey_a; pm.ey_x[p] = q; eyv = eyv - cf.x * q; }  // ceyhz
              if (upd_z) { T q = b * (pa == 0 ? pe1[u] : pm.ez_x[p]) + a * d_ez_b; pm.ez_x[p] = q; ezv = ezv + cf.x * q; }  // cezhy
            }
            if (sy_pml >= 0) {
              const long long p = static_cast<long long>(ie) * pm.ysx + sy_pml * sy + k;
              const T a = pm.ae[1][j], b = pm.be[1][j];
              if (upd_z) { T q = b * (pa == 1 ? pe0[u] : pm.ez_y[p]) + a * d_ez_a; pm.ez_y[p] = q; ezv = ezv - cf.y * q; }  // cezhx
              if (upd_x) { T q = b * (pa == 1 ? pe1[u] : pm.ex_y[p]) + a * d_ex_b; pm.ex_y[p] = q; exv = exv + cf.y * q; }  // cexhz
            }
            if (sz_pml >= 0) {
              const long long p = static_cast<long long>(ie) * pm.zsx + static_cast<long long>(j) * pm.zsy + sz_pml;
              const T a = pm.ae[2][k], b = pm.be[2][k];
              if (upd_x) { T q = b * (pa == 2 ? pe0[u] : pm.ex_z[p]) + a * d_ex_a; pm.ex_z[p] = q; exv = exv - cf.z * q; }  // cexhy
              if (upd_y) { T q = b * (pa == 2 ? pe1[u] : pm.ey_z[p]) + a * d_ey_b; pm.ey_z[p] = q; eyv = eyv + cf.z * q; }  // ceyhx
            }
          }
        }
        // E components on PEC walls keep their value in the new buffer
        oex[c.go] = upd_x ? exv : ex_o;
        oey[c.go] = upd_y ? eyv : ey_o;
        oez[c.go] = upd_z ? ezv : ez_o;
      }
    }
    // rotate the register planes; E-pass inputs of plane i for the next iteration
    if (row_warp && do_h) {
#pragma unroll
      for (int u = 0; u < R; ++u) {
        hqy[u] = hpy[u]; hqz[u] = hpz[u];
        hpx[u] = hnx[u]; hpy[u] = hny[u]; hpz[u] = hnz[u];
        em[u] = enm[u];
        eox[u] = enx[u]; eoy[u] = eny[u]; eoz[u] = enz[u];
      }
    }
    // CPML psi of the next iteration: E of plane i
    if (PML) {
      if (row_warp && do_h && i >= i_start) {
        const int sxe = PX ? slab(i, s.nx, pm.L[0], pm.L[1]) : -1;
#pragma unroll
        for (int u = 0; u < R; ++u)
          pea[u] = prefetch_e_psi<T, KIND>(pm, s, i, sxe, cell[u], (valid >> u) & 1u, pe0[u], pe1[u]);
      }
    }
  }
  if (!TMA) {
    cp_async_wait<0>();
  } else if (!ok && tid == 0) {
    // a staging wait ran out: flag it, then let the copies still in flight
    // (planes waited+1 .. the last staged one) land before the CTA exits
    atomicExch(err, 1);
    for (int p = waited + 1; p <= staged; ++p) mbar_wait(bar + p % NS, phase(p));
  }
}

// Bulk-copy body of a work item: the lean interior items (PK = 0: no CPML or
// ADE cell and no PEC wall within reach, the tile with its halo row and
// column inside the grid, first plane >= 1) and the y- or z-slab CPML columns
// (PK = 3 or 9: x+y or x+z slab kinds, at the grid's edges).  The arithmetic
// is step_item's (hNext, TFSF, CPML x, y, z corrections; eNext, TFSF, CPML),
// term for term and in the same order; what differs is the data movement.
// The H planes live in dense shared tiles (with the halo row j0-1 and halo
// column k0-1 after them): the E update reads its j-1 and k-1 neighbours
// there at per-thread constant offsets, and the tiles are also the sources
// of bulk tensor stores, whose tensor extents (nz, ny, nx) clip an edge
// tile's cells outside the grid (the k extent only to 16-byte granules, so
// those cells carry their old values into the tiles: a store that reaches the
// wall column k = nz writes back what is there).  E^{n+1} goes to dense tiles
// too, with the PEC walls' components keeping their old value.  At iteration i one
// thread issues the stores of H plane i-1 and E plane i-2 (both finished
// before the iteration's barrier) and waits, before the next barrier, until
// they have read their tiles.  CPML: per-thread psi offsets and y/z profile
// coefficients are computed once per item; the psi pair of the slab axis of
// each cell (H of the next plane, E of the current one) is loaded a plane
// ahead; x-slab psi (planes near the x faces) inline.  TF: with the TFSF
// corrections of the cells on the TFSF surface; LN: the incident values of
// the tile's y and z face lines arrive with each staged plane (one bulk copy
// per line window and pass from the tables of k_tfsf_lines, on the plane's
// barrier), the x-face planes compute theirs in place.
template <typename T, int R, int NWM, int NS_, bool TF, int PK, bool LN>
__device__ __forceinline__ void step_item_fast(const GridP<T>& s, const PmlP<T>& pm, const PsiH<T>& ps,
                                               const PsiH<T>& pd, int4 item, const T* lut8, int n_mat,
                                               const TfsfP& tf, const StageMaps* maps, const StoreMaps* outs,
                                               const LineMaps* lines, int* err) {
  using L = StepCfg<T, R, NWM, NS_>;
  constexpr int NS = L::NS, HP = L::HP, RW = L::RW, MW = L::MW, TJ = L::TJ, PL = L::PL, NT = L::NT;
  constexpr int CS = L::LCS, ET = TJ * 32;
  constexpr bool PX = (PK & 1) != 0, PY = (PK & 2) != 0, PZ = (PK & 8) != 0, PML = PK != 0;
  // column axis whose psi pair is loaded a plane ahead (y when both are
  // present), and z as a second column axis (corner columns, loaded inline)
  constexpr bool CZ = PZ && !PY, Z2 = PY && PZ;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  unsigned char* base = smem_raw + ((128u - (smem_u32(smem_raw) & 127u)) & 127u);
  T* sF = reinterpret_cast<T*>(base);                            // [NS][6][PL]
  uint8_t* sM = base + L::off_m;                                 // [NS][MPL]: RH rows of MW
  uint64_t* bar = reinterpret_cast<uint64_t*>(base + L::off_b);  // [NS]
  T* sH = reinterpret_cast<T*>(base + L::off_h);                 // [2][3][CS]
  T* sE = reinterpret_cast<T*>(base + L::off_e);                 // [2][3][TJ * 32]
  T* sL = reinterpret_cast<T*>(base + L::off_l);                 // [LUTM][8]
  T* sC = reinterpret_cast<T*>(base + L::off_c);                 // [2][4][NC] CPML coefficients

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int k0 = (item.x & 0xffff) * 32, j0 = item.y * TJ;
  const int i_start = item.z, i_end = item.w, i_first = i_start > 0 ? i_start - 1 : 0;
  const bool lut_shared = n_mat <= L::LUTM;
  if (lut_shared)
    for (int q = tid; q < n_mat * 8; q += NT) sL[q] = lut8[q];
  const T* lut = lut_shared ? sL : lut8;
  if ((PY || PZ) && tid < L::NC) {  // profile coefficients of the tile's rows / columns
    const int q = PY ? j0 - 1 + tid : k0 - 1 + tid;
    const int n = PY ? s.ny : s.nz, ax = PY ? 1 : 2;
    const bool in = q >= 0 && q < n && slab(q, n, pm.L[2 * ax], pm.L[2 * ax + 1]) >= 0;
    sC[tid] = in ? pm.ah[ax][q] : T(0);
    sC[L::NC + tid] = in ? pm.bh[ax][q] : T(0);
    sC[2 * L::NC + tid] = in ? pm.ae[ax][q] : T(0);
    sC[3 * L::NC + tid] = in ? pm.be[ax][q] : T(0);
    if (Z2) {  // the z columns of a corner tile
      const int qk = k0 - 1 + tid;
      const bool inz = qk >= 0 && qk < s.nz && slab(qk, s.nz, pm.L[4], pm.L[5]) >= 0;
      T* z = sC + 4 * L::NC;
      z[tid] = inz ? pm.ah[2][qk] : T(0);
      z[L::NC + tid] = inz ? pm.bh[2][qk] : T(0);
      z[2 * L::NC + tid] = inz ? pm.ae[2][qk] : T(0);
      z[3 * L::NC + tid] = inz ? pm.be[2][qk] : T(0);
    }
  }
  if (tid == 0) {
    for (int q = 0; q < NS; ++q) mbar_init(bar + q, 1);
    fence_mbar_init();
  }
  __syncthreads();
  // TFSF line values (LN): the face of the y and z lines the tile meets (the
  // host gives tiles that meet both faces of an axis the general body)
  const int fy = TF && LN && tf.on ? tfsf_line_face(tf.js, tf.je, j0, TJ) : -1;
  const int fz = TF && LN && tf.on ? tfsf_line_face(tf.ks, tf.ke, k0, 32) : -1;
  unsigned char* sT = base + L::off_t;  // [NS][LSLOT]: y boxes (H, E), z boxes (H, E)
  const unsigned line_tx = (fy >= 0 ? 2u * 2u * L::YW * 8u : 0u) + (fz >= 0 ? 2u * 2u * L::ZW * 8u : 0u);
  int staged = -1;  // last plane whose copies were issued (thread 0)
  auto stage = [&](int plane, int st) {
    if (tid == 0 && plane <= i_end) {
      staged = plane;
      fence_proxy_async();
      mbar_expect_tx(bar + st, L::tx_bytes + line_tx);
      T* dst = sF + st * 6 * PL;
#pragma unroll
      for (int f = 0; f < 6; ++f) tma_load_3d(dst + f * PL, &maps->f[f], k0 - HP, j0 - 1, plane, bar + st);
      tma_load_3d(sM + st * L::MPL, &maps->mid, k0 - 16, j0 - 1, plane, bar + st);
      if (LN) {
        // the H-pass lines of this plane, the E-pass lines of the plane before
        unsigned char* t = sT + st * L::LSLOT;
        if (fy >= 0) {
          tma_load_4d(t, &lines->yh, k0 - 2, 0, plane, fy, bar + st);
          tma_load_4d(t + L::YB, &lines->ye, k0 - 2, 0, plane - 1, fy, bar + st);
        }
        if (fz >= 0) {
          tma_load_4d(t + 2 * L::YB, &lines->zh, j0 - 2, 0, plane, fz, bar + st);
          tma_load_4d(t + 2 * L::YB + L::ZB, &lines->ze, j0 - 2, 0, plane - 1, fz, bar + st);
        }
      }
    }
  };
  for (int q = 0; q < NS - 1; ++q) stage(i_first + q, (i_first + q) % NS);
  auto phase = [&](int p) { return static_cast<unsigned>(((p - i_first) / NS) & 1); };

  // cells of this thread: a row warp's R rows at column `lane`; the halo
  // warp's row j0-1 at column `lane` (u = 0) and column k0-1 at row `lane`
  // (u = 1, lane < TJ).  wf: staged offset, mo: material offset, hs: slot in
  // the H tile, km: the k-1 neighbour's slot (row warps).
  const bool row_warp = warp < NWM;
  int wf[R], mo[R], hs[R], km[R];
  int cj[R], ck[R], tfl[R];  // cell indices, TFSF line flags (TF only)
  bool act[R];
#pragma unroll
  for (int u = 0; u < R; ++u) {
    cj[u] = row_warp ? j0 + warp * R + u : (u == 0 ? j0 - 1 : j0 + lane);
    ck[u] = row_warp ? k0 + lane : (u == 0 ? k0 + lane : k0 - 1);
    tfl[u] = TF && tf.on ? ((cj[u] == tf.js - 1 || cj[u] == tf.je || ck[u] == tf.ks - 1 || ck[u] == tf.ke) ? 1 : 0) |
                               ((cj[u] == tf.js || cj[u] == tf.je || ck[u] == tf.ks || ck[u] == tf.ke) ? 2 : 0)
                         : 0;
    if (row_warp) {
      const int r = warp * R + u;
      wf[u] = (r + 1) * RW + HP + lane;
      mo[u] = (r + 1) * MW + 16 + lane;
      hs[u] = r * 32 + lane;
      km[u] = lane ? r * 32 + lane - 1 : (TJ + 1) * 32 + r;
      act[u] = true;
    } else if (u == 0) {
      wf[u] = HP + lane;
      mo[u] = 16 + lane;
      hs[u] = TJ * 32 + lane;
      km[u] = 0;
      act[u] = true;
    } else {
      wf[u] = (lane + 1) * RW + HP - 1;
      mo[u] = (lane + 1) * MW + 15;
      hs[u] = (TJ + 1) * 32 + lane;
      km[u] = 0;
      act[u] = u == 1 && lane < TJ;
    }
  }
  const int jm0 = warp * R > 0 ? (warp * R - 1) * 32 + lane : TJ * 32 + lane;  // j-1 of row u = 0

  // CPML: per cell the slab index of the column axis (-1: outside the slab or
  // outside the grid), its psi offset inside a plane and its profile
  // coefficients; the x-slab offset inside a plane; the PEC wall flags
  int sp[R], so[R], go[R];
  // (the coefficients themselves sit in the shared table sC at index ci,
  // filled before the first barrier of the item)
  int ci[R];
  int spz[R], soz[R], ciz[R];  // second column axis (z of a corner tile)
  bool in_grid[R];
#pragma unroll
  for (int u = 0; u < R; ++u) {
    const int j = cj[u], k = ck[u];
    in_grid[u] = act[u] && j >= 0 && k >= 0 && j < s.ny && k < s.nz;
    go[u] = j * static_cast<int>(s.sy) + k;
    sp[u] = -1;
    so[u] = 0;
    ci[u] = PY ? j - j0 + 1 : k - k0 + 1;
    spz[u] = -1;
    soz[u] = 0;
    ciz[u] = k - k0 + 1;
    if (PY && in_grid[u]) {
      sp[u] = slab(j, s.ny, pm.L[2], pm.L[3]);
      if (sp[u] >= 0) so[u] = sp[u] * static_cast<int>(s.sy) + k;
    }
    if (CZ && in_grid[u]) {
      sp[u] = slab(k, s.nz, pm.L[4], pm.L[5]);
      if (sp[u] >= 0) so[u] = j * static_cast<int>(pm.zsy) + sp[u];
    }
    if (Z2 && in_grid[u]) {
      spz[u] = slab(k, s.nz, pm.L[4], pm.L[5]);
      if (spz[u] >= 0) soz[u] = j * static_cast<int>(pm.zsy) + spz[u];
    }
  }
  const T* cah = sC;
  const T* cbh = sC + L::NC;
  const T* cae = sC + 2 * L::NC;
  const T* cbe = sC + 3 * L::NC;
  const T* zah = sC + 4 * L::NC;  // z coefficients of a corner tile
  const T* zbh = sC + 5 * L::NC;
  const T* zae = sC + 6 * L::NC;
  const T* zbe = sC + 7 * L::NC;
  const long long psx = PY ? pm.ysx : pm.zsx;  // psi plane stride of the column axis
  // psi arrays of the column axis, in the order the updates read them
  // (H: y: hz, hx; z: hx, hy; E: y: ez, ex; z: ex, ey)
  const T* hr0 = PY ? ps.hz_y : ps.hx_z;
  const T* hr1 = PY ? ps.hx_y : ps.hy_z;
  T* hw0 = PY ? pd.hz_y : pd.hx_z;
  T* hw1 = PY ? pd.hx_y : pd.hy_z;
  T* er0 = PY ? pm.ez_y : pm.ex_z;
  T* er1 = PY ? pm.ex_y : pm.ey_z;

  T hnx[R], hny[R], hnz[R], hpx[R], hpy[R], hpz[R], hqy[R], hqz[R];
  T eox[R], eoy[R], eoz[R], enx[R], eny[R], enz[R];
  T ph0[R], ph1[R], pe0[R], pe1[R];  // column-axis psi pairs loaded a plane ahead
  int em[R], enm[R];
#pragma unroll
  for (int u = 0; u < R; ++u) {
    hnx[u] = hny[u] = hnz[u] = hpx[u] = hpy[u] = hpz[u] = hqy[u] = hqz[u] = T(0);
    eox[u] = eoy[u] = eoz[u] = enx[u] = eny[u] = enz[u] = T(0);
    ph0[u] = ph1[u] = pe0[u] = pe1[u] = T(0);
    em[u] = enm[u] = 0;
  }
  if (PML && (PY || PZ)) {
    const T* a0 = hr0 + static_cast<long long>(i_first) * psx;
    const T* a1 = hr1 + static_cast<long long>(i_first) * psx;
#pragma unroll
    for (int u = 0; u < R; ++u)
      if (sp[u] >= 0) { ph0[u] = a0[so[u]]; ph1[u] = a1[so[u]]; }
  }
  int slot = i_first % NS;
  int waited = i_first - 1;
  const int polls = err[1];  // poll limit of the staging waits
  bool ok = mbar_wait(bar + slot, phase(i_first), polls);
  if (ok) waited = i_first;
  for (int i = i_first; i <= i_end; ++i) {
    const int ie = i - 1;
    const bool do_h = i < i_end;
    const int slot_n = slot + 1 == NS ? 0 : slot + 1;
    const int slot_p = slot == 0 ? NS - 1 : slot - 1;
    if (i + 1 <= i_end && ok) {
      ok = mbar_wait(bar + slot_n, phase(i + 1), polls);
      if (ok) waited = i + 1;
    }
    if (__syncthreads_or(!ok)) {
      ok = false;
      break;
    }
    stage(i + NS - 1, slot_p);
    if (tid == 0) {  // planes finished by iteration i-1 (fenced by their writers)
      if (i - 1 >= i_start) {
        const T* src = sH + ((i - 1) & 1) * 3 * CS;
#pragma unroll
        for (int c = 0; c < 3; ++c) tma_store_3d(&outs->f[3 + c], src + c * CS, k0, j0, i - 1);
      }
      if (i - 2 >= i_start) {
        const T* src = sE + ((i - 2) & 1) * 3 * ET;
#pragma unroll
        for (int c = 0; c < 3; ++c) tma_store_3d(&outs->f[c], src + c * ET, k0, j0, i - 2);
      }
      bulk_commit();
    }
    const T* Fc = sF + slot * 6 * PL;
    const T* Fn = sF + slot_n * 6 * PL;
    const uint8_t* Mc = sM + slot * L::MPL;
    // staged TFSF lines of this slot: H pass of plane i, E pass of plane i-1
    const unsigned char* tl = sT + slot * L::LSLOT;
    const LineVals lvh{reinterpret_cast<const double*>(tl), reinterpret_cast<const double*>(tl + 2 * L::YB), L::YW,
                       L::ZW, k0 - 2, j0 - 2};
    const LineVals lve{reinterpret_cast<const double*>(tl + L::YB),
                       reinterpret_cast<const double*>(tl + 2 * L::YB + L::ZB), L::YW, L::ZW, k0 - 2, j0 - 2};
    slot = slot_n;
    T* Hc = sH + (i & 1) * 3 * CS;              // H plane i (written here)
    const T* Hq = sH + ((i + 1) & 1) * 3 * CS;  // H plane i-1
    // ---- H pass, plane i ------------------------------------------------------
    const bool tf_hplane = TF && tf.on && (i == tf.is - 1 || i == tf.ie);
    const int sxp = PX ? slab(i, s.nx, pm.L[0], pm.L[1]) : -1;
    const bool own_h = row_warp && i >= i_start;
    if (do_h) {
      // psi planes of the column axis at plane i (H written to the other set)
      T* w0 = hw0 + static_cast<long long>(i) * psx;
      T* w1 = hw1 + static_cast<long long>(i) * psx;
#pragma unroll
      for (int u = 0; u < R; ++u) {
        if (!act[u]) continue;
        const int m = Mc[mo[u]];
        const C4<T> cf = ld_c4(lut + 8 * m + 4);  // ch, db/dx, db/dy, db/dz
        const T* f = Fc + wf[u];
        const T ex_c = f[0], ey_c = f[PL], ez_c = f[2 * PL];
        const T d_hx_a = f[PL + 1] - ey_c;
        const T d_hx_b = f[2 * PL + RW] - ez_c;
        const T d_hy_a = Fn[wf[u] + 2 * PL] - ez_c;
        const T d_hy_b = f[1] - ex_c;
        const T d_hz_a = f[RW] - ex_c;
        const T d_hz_b = Fn[wf[u] + PL] - ey_c;
        T hxv = cf.c * f[3 * PL] + cf.z * d_hx_a - cf.y * d_hx_b;
        T hyv = cf.c * f[4 * PL] + cf.x * d_hy_a - cf.z * d_hy_b;
        T hzv = cf.c * f[5 * PL] + cf.y * d_hz_a - cf.x * d_hz_b;
        if (TF && (tf_hplane || (tfl[u] & 1))) {
          if (LN) tfsf_h_lines(tf, IncTables{tf}, lvh, i, cj[u], ck[u], hxv, hyv, hzv);
          else tfsf_h(tf, IncTables{tf}, i, cj[u], ck[u], hxv, hyv, hzv);
        }
        if (PX && sxp >= 0 && in_grid[u]) {
          const long long p = static_cast<long long>(sxp) * s.sx + go[u];
          const T a = pm.ah[0][i], b = pm.bh[0][i];
          const T qy = b * ps.hy_x[p] + a * d_hy_a;
          hyv = hyv + cf.x * qy;   // chyez
          const T qz = b * ps.hz_x[p] + a * d_hz_b;
          hzv = hzv - cf.x * qz;   // chzey
          if (own_h) { pd.hy_x[p] = qy; pd.hz_x[p] = qz; }
        }
        if (PY && sp[u] >= 0) {
          const T qz = cbh[ci[u]] * ph0[u] + cah[ci[u]] * d_hz_a;
          hzv = hzv + cf.y * qz;   // chzex
          const T qx = cbh[ci[u]] * ph1[u] + cah[ci[u]] * d_hx_b;
          hxv = hxv - cf.y * qx;   // chxez
          if (own_h) { w0[so[u]] = qz; w1[so[u]] = qx; }
        }
        if (CZ && sp[u] >= 0) {
          const T qx = cbh[ci[u]] * ph0[u] + cah[ci[u]] * d_hx_a;
          hxv = hxv + cf.z * qx;   // chxey
          const T qy = cbh[ci[u]] * ph1[u] + cah[ci[u]] * d_hy_b;
          hyv = hyv - cf.z * qy;   // chyex
          if (own_h) { w0[so[u]] = qx; w1[so[u]] = qy; }
        }
        if (Z2 && spz[u] >= 0) {
          const long long p = static_cast<long long>(i) * pm.zsx + soz[u];
          const T qx = zbh[ciz[u]] * ps.hx_z[p] + zah[ciz[u]] * d_hx_a;
          hxv = hxv + cf.z * qx;   // chxey
          const T qy = zbh[ciz[u]] * ps.hy_z[p] + zah[ciz[u]] * d_hy_b;
          hyv = hyv - cf.z * qy;   // chyex
          if (own_h) { pd.hx_z[p] = qx; pd.hy_z[p] = qy; }
        }
        if (PML && !in_grid[u]) {  // outside the grid: the bulk store writes back the old value
          hxv = f[3 * PL]; hyv = f[4 * PL]; hzv = f[5 * PL];
        }
        Hc[hs[u]] = hxv;
        Hc[CS + hs[u]] = hyv;
        Hc[2 * CS + hs[u]] = hzv;
        hnx[u] = hxv; hny[u] = hyv; hnz[u] = hzv;
        enx[u] = ex_c; eny[u] = ey_c; enz[u] = ez_c;
        enm[u] = m;
      }
    }
    // column-axis H psi of plane i+1, issued now that plane i's is consumed:
    // the E pass, the stores and the barrier cover its latency
    if (PML && (PY || PZ) && i + 1 < i_end) {
      const T* a0 = hr0 + static_cast<long long>(i + 1) * psx;
      const T* a1 = hr1 + static_cast<long long>(i + 1) * psx;
#pragma unroll
      for (int u = 0; u < R; ++u)
        if (sp[u] >= 0) { ph0[u] = a0[so[u]]; ph1[u] = a1[so[u]]; }
    }
    // ---- E pass, plane ie = i-1 ------------------------------------------------
    const bool tf_eplane = TF && tf.on && (ie == tf.is || ie == tf.ie);
    if (row_warp && ie >= i_start) {
      T* Eo = sE + (ie & 1) * 3 * ET;
      const int sxe = PX ? slab(ie, s.nx, pm.L[0], pm.L[1]) : -1;
      T* e0p = er0 + static_cast<long long>(ie) * psx;
      T* e1p = er1 + static_cast<long long>(ie) * psx;
      const bool ipos = ie > 0;
#pragma unroll
      for (int u = 0; u < R; ++u) {
        const C4<T> cf = ld_c4(lut + 8 * em[u]);  // ce, cb/dx, cb/dy, cb/dz
        const T hx_c = hpx[u], hy_c = hpy[u], hz_c = hpz[u];
        const T hx_km = Hq[km[u]], hy_km = Hq[CS + km[u]];
        const T hx_jm = u > 0 ? hpx[u > 0 ? u - 1 : 0] : Hq[jm0];
        const T hz_jm = u > 0 ? hpz[u > 0 ? u - 1 : 0] : Hq[2 * CS + jm0];
        const T hy_p = hqy[u], hz_p = hqz[u];
        const T d_ex_a = hy_c - hy_km;
        const T d_ex_b = hz_c - hz_jm;
        const T d_ey_a = hz_c - hz_p;
        const T d_ey_b = hx_c - hx_km;
        const T d_ez_a = hx_c - hx_jm;
        const T d_ez_b = hy_c - hy_p;
        const int o = (warp * R + u) * 32 + lane;
        T exv = cf.c * eox[u] - cf.z * d_ex_a + cf.y * d_ex_b;
        T eyv = cf.c * eoy[u] - cf.x * d_ey_a + cf.z * d_ey_b;
        T ezv = cf.c * eoz[u] - cf.y * d_ez_a + cf.x * d_ez_b;
        if (TF && (tf_eplane || (tfl[u] & 2))) {
          if (LN) tfsf_e_lines(tf, IncTables{tf}, lve, ie, cj[u], ck[u], exv, eyv, ezv);
          else tfsf_e(tf, IncTables{tf}, ie, cj[u], ck[u], exv, eyv, ezv);
        }
        if (PML) {
          const bool jpos = cj[u] > 0, kpos = ck[u] > 0;
          const bool upd_x = jpos && kpos, upd_y = ipos && kpos, upd_z = ipos && jpos;
          if (PX && sxe >= 0 && in_grid[u]) {
            const long long p = static_cast<long long>(sxe) * s.sx + go[u];
            const T a = pm.ae[0][ie], b = pm.be[0][ie];
            if (upd_y) { T q = b * pm.ey_x[p] + a * d_ey_a; pm.ey_x[p] = q; eyv = eyv - cf.x * q; }  // ceyhz
            if (upd_z) { T q = b * pm.ez_x[p] + a * d_ez_b; pm.ez_x[p] = q; ezv = ezv + cf.x * q; }  // cezhy
          }
          if (PY && sp[u] >= 0) {
            if (upd_z) { T q = cbe[ci[u]] * pe0[u] + cae[ci[u]] * d_ez_a; e0p[so[u]] = q; ezv = ezv - cf.y * q; }  // cezhx
            if (upd_x) { T q = cbe[ci[u]] * pe1[u] + cae[ci[u]] * d_ex_b; e1p[so[u]] = q; exv = exv + cf.y * q; }  // cexhz
          }
          if (CZ && sp[u] >= 0) {
            if (upd_x) { T q = cbe[ci[u]] * pe0[u] + cae[ci[u]] * d_ex_a; e0p[so[u]] = q; exv = exv - cf.z * q; }  // cexhy
            if (upd_y) { T q = cbe[ci[u]] * pe1[u] + cae[ci[u]] * d_ey_b; e1p[so[u]] = q; eyv = eyv + cf.z * q; }  // ceyhx
          }
          if (Z2 && spz[u] >= 0) {
            const long long p = static_cast<long long>(ie) * pm.zsx + soz[u];
            if (upd_x) { T q = zbe[ciz[u]] * pm.ex_z[p] + zae[ciz[u]] * d_ex_a; pm.ex_z[p] = q; exv = exv - cf.z * q; }  // cexhy
            if (upd_y) { T q = zbe[ciz[u]] * pm.ey_z[p] + zae[ciz[u]] * d_ey_b; pm.ey_z[p] = q; eyv = eyv + cf.z * q; }  // ceyhx
          }
          // E components on PEC walls keep their value, and so do the cells
          // of an edge tile outside the grid (a bulk store clips the k extent
          // only to 16-byte granules, so it may write the wall column k = nz)
          if (!upd_x || !in_grid[u]) exv = eox[u];
          if (!upd_y || !in_grid[u]) eyv = eoy[u];
          if (!upd_z || !in_grid[u]) ezv = eoz[u];
        }
        Eo[o] = exv;
        Eo[ET + o] = eyv;
        Eo[2 * ET + o] = ezv;
      }
    }
    if (row_warp && do_h) {
#pragma unroll
      for (int u = 0; u < R; ++u) {
        hqy[u] = hpy[u]; hqz[u] = hpz[u];
        hpx[u] = hnx[u]; hpy[u] = hny[u]; hpz[u] = hnz[u];
        em[u] = enm[u];
        eox[u] = enx[u]; eoy[u] = eny[u]; eoz[u] = enz[u];
      }
    }
    // column-axis E psi of the next iteration (plane i)
    if (PML && (PY || PZ) && row_warp && do_h && i >= i_start) {
      const T* b0 = er0 + static_cast<long long>(i) * psx;
      const T* b1 = er1 + static_cast<long long>(i) * psx;
#pragma unroll
      for (int u = 0; u < R; ++u)
        if (sp[u] >= 0) { pe0[u] = b0[so[u]]; pe1[u] = b1[so[u]]; }
    }
    fence_proxy_async();             // this thread's tile writes before the next iteration's bulk stores
    if (tid == 0) bulk_wait_read();  // this iteration's stores have read their tiles
  }
  if (ok) {
    __syncthreads();  // E plane i_end-1 is complete
    if (tid == 0) {
      if (i_end - 1 >= i_start) {
        const T* src = sE + ((i_end - 1) & 1) * 3 * ET;
#pragma unroll
        for (int c = 0; c < 3; ++c) tma_store_3d(&outs->f[c], src + c * ET, k0, j0, i_end - 1);
      }
      bulk_commit();
      bulk_wait_all();
    }
  } else if (tid == 0) {
    // a staging wait ran out: flag it, let the copies in flight land and the
    // issued stores finish before the CTA exits
    atomicExch(err, 1);
    for (int p = waited + 1; p <= staged; ++p) mbar_wait(bar + p % NS, phase(p));
    bulk_wait_all();
  }
}

// The one-sweep step kernel: one CTA per work item (x: k tile | kind << 16,
// y: j tile, z: first plane, w: end plane); every kind runs its own
// specialised body, so one launch covers the whole grid.  Region bits of a
// kind: 1 x-slab planes, 2 y-slab columns, 8 z-slab columns, 4 ADE box, 16
// TFSF corrections.  Kind indices 0..6: lean, x planes, ADE box, y columns,
// z columns, y+z corner columns, ADE next to a slab, all without TFSF code;
// 7: lean with TFSF; 8: lean interior; 9..14: kinds 1..6 with TFSF; 15: lean
// interior with TFSF; 16..18: y, z and corner columns on the bulk-copy body;
// 19..21: those with TFSF.  kStepKinds gives the bits of indices 0..15.
constexpr int kStepKinds[16] = {0, 1, 4, 3, 9, 11, 15, 16, 0, 1 | 16, 4 | 16, 3 | 16, 9 | 16, 11 | 16, 15 | 16, 16};

// kind indices of the lean interior items (step_item_fast, bulk-copy path
// only), without and with TFSF corrections
constexpr int kLeanInterior = 8, kLeanInteriorTf = 15;
// kind indices of the y- and z-slab CPML columns run by step_item_fast (the
// bulk-copy path only; without TFSF cells)
constexpr int kFastY = 16, kFastZ = 17;
// ... and of the y+z corner columns
constexpr int kFastYZ = 18;
// ... and of the same three column kinds with TFSF corrections (a tile
// column whose 32 columns or TJ rows hold both CPML cells and a TFSF face)
constexpr int kFastYTf = 19, kFastZTf = 20, kFastYZTf = 21;

// LN: the TFSF bodies take the y- and z-line incident values from the line
// tables (single scenes, which compute them every step); batches compute
// them from the projections and the auxiliary rows.
template <typename T, int R, int NWM, int NS_, bool TMA, bool LN = false>
__device__ __forceinline__ void step_dispatch(const GridP<T>& s, const GridP<T>& d, const PmlP<T>& pm,
                                              const PsiH<T>& ps, const PsiH<T>& pd, const TfsfP& tf,
                                              const AdeP<T>& ad, int4 item, const T* lut8, const uint8_t* disp,
                                              int n_mat, const StageMaps* maps, const StoreMaps* outs, int* err,
                                              const LineMaps* lines = nullptr) {
  if (TMA) {
#define XFB_FAST(tfc, pk) step_item_fast<T, R, NWM, NS_, tfc, pk, LN>(s, pm, ps, pd, item, lut8, n_mat, tf, maps, outs, lines, err)
    switch (item.x >> 16) {
      case kLeanInterior: XFB_FAST(false, 0); return;
      case kLeanInteriorTf: XFB_FAST(true, 0); return;
      case kFastY: XFB_FAST(false, 3); return;
      case kFastZ: XFB_FAST(false, 9); return;
      case kFastYZ: XFB_FAST(false, 11); return;
      case kFastYTf: XFB_FAST(true, 3); return;
      case kFastZTf: XFB_FAST(true, 9); return;
      case kFastYZTf: XFB_FAST(true, 11); return;
      default: break;
    }
#undef XFB_FAST
  }
#define XFB_ITEM(q) step_item<T, R, NWM, NS_, kStepKinds[q], TMA>(s, d, pm, ps, pd, tf, ad, item, lut8, disp, n_mat, maps, err)
  switch (item.x >> 16) {
    case 0: XFB_ITEM(0); break;
    case 1: XFB_ITEM(1); break;
    case 2: XFB_ITEM(2); break;
    case 3: XFB_ITEM(3); break;
    case 4: XFB_ITEM(4); break;
    case 5: XFB_ITEM(5); break;
    case 6: XFB_ITEM(6); break;
    case 7: XFB_ITEM(7); break;
    case 9: XFB_ITEM(9); break;
    case 10: XFB_ITEM(10); break;
    case 11: XFB_ITEM(11); break;
    case 12: XFB_ITEM(12); break;
    case 13: XFB_ITEM(13); break;
    default: XFB_ITEM(14); break;
  }
#undef XFB_ITEM
}

// The single-scene step stages with tiled bulk copies from the tensor maps of
// its read set (`maps`, a grid constant), together with the TFSF line values
// of the items on the TFSF surface (`lines`, tables k_tfsf_lines filled for
// this step); its lean interior and CPML column items store through the maps
// of the write set (`outs`); a staging wait that runs out sets *err.
template <typename T, int R, int NWM, int NS_>
__global__ void __launch_bounds__(StepCfg<T, R, NWM, NS_>::NT, StepCfg<T, R, NWM, NS_>::min_blocks)
    k_step3(GridP<T> s, GridP<T> d, PmlP<T> pm, PsiH<T> ps, PsiH<T> pd, TfsfP tf_in, AdeP<T> ad, TimeP tp,
            const int4* items, const T* lut8, const uint8_t* disp, int n_mat, const __grid_constant__ StageMaps maps,
            const __grid_constant__ StoreMaps outs, const __grid_constant__ LineMaps lines, int* err) {
  const TfsfP tf = tfsf_at_step(tf_in, cur_step(tp));
  step_dispatch<T, R, NWM, NS_, true, true>(s, d, pm, ps, pd, tf, ad, items[blockIdx.x], lut8, disp, n_mat, &maps,
                                            &outs, err, &lines);
}

// Everything the one-sweep step reads of one scene of a batch.  Both field
// and H-psi buffer sets are listed; the launch's parity picks read and write.
template <typename T>
struct BatchScene {
  GridP<T> g[2];
  PsiH<T> psh[2];
  PmlP<T> pm;
  TfsfP tf;
  AdeP<T> ad;
  const T* lut8;
  const uint8_t* disp;
  int n_mat;
  int pad;
  LineP lines;  // TFSF line tables (per-step form)
};

// Tensor maps of one scene of a batch, in global memory: staging maps per tile
// configuration and read set, bulk-store maps per tile configuration and
// write set, TFSF line maps per tile configuration.
struct BatchMaps {
  StageMaps stage[3][2];
  StoreMaps store[3][2];
  LineMaps line[3];
};

// The TFSF line tables of one step of every scene of a batch (blockIdx.y:
// the scene), ahead of the batch's step kernel.
template <typename T>
__global__ void k_tfsf_lines_batch(const BatchScene<T>* scenes, TimeP tp) {
  const BatchScene<T>& sc = scenes[blockIdx.y];
  if (!sc.tf.on) return;
  tfsf_lines_fill(tfsf_at_step(sc.tf, cur_step(tp)), sc.lines,
                  blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x,
                  static_cast<long long>(gridDim.x) * blockDim.x);
}

// The one-sweep step of a batch of scenes in one launch: one CTA per work
// item (x: k tile | kind << 11 | scene << 16, y: j tile, z/w: plane range).
// The CTA copies its scene's parameters into shared memory and runs the same
// region-specialised bodies as k_step3 (bulk copies through the scene's
// tensor maps in `maps`, tile configuration `tile`, TFSF line values from the
// tables k_tfsf_lines_batch filled for this step); a staging wait that runs
// out sets *err.
template <typename T, int R, int NWM, int NS_>
__global__ void __launch_bounds__(StepCfg<T, R, NWM, NS_>::NT, StepCfg<T, R, NWM, NS_>::min_blocks)
    k_step3_batch(const BatchScene<T>* scenes, const BatchMaps* maps, const int4* items, TimeP tp, int parity,
                  int tile, int* err) {
  __shared__ BatchScene<T> sp;
  const int4 it = items[blockIdx.x];
  const int scene = static_cast<int>(static_cast<unsigned>(it.x) >> 16);
  {
    const int* src = reinterpret_cast<const int*>(scenes + scene);
    int* dst = reinterpret_cast<int*>(&sp);
    for (int q = threadIdx.x; q < static_cast<int>(sizeof(BatchScene<T>) / 4); q += blockDim.x) dst[q] = src[q];
  }
  __syncthreads();
  if (threadIdx.x == 0) sp.tf = tfsf_at_step(sp.tf, cur_step(tp));  // incident-table rows of this step
  __syncthreads();
  const int4 item = make_int4((it.x & 0x7ff) | (((it.x >> 11) & 0x1f) << 16), it.y, it.z, it.w);
  const BatchMaps& bm = maps[scene];
  step_dispatch<T, R, NWM, NS_, true, true>(sp.g[parity], sp.g[1 - parity], sp.pm, sp.psh[parity],
                                            sp.psh[1 - parity], sp.tf, sp.ad, item, sp.lut8, sp.disp, sp.n_mat,
                                            &bm.stage[tile][parity], &bm.store[tile][1 - parity], err, &bm.line[tile]);
}

__device__ __forceinline__ unsigned ld_acquire_gpu(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];\n" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void red_release_gpu_add(unsigned* p, unsigned v) {
  asm volatile("red.release.gpu.global.add.u32 [%0], %1;\n" ::"l"(p), "r"(v) : "memory");
}
// orders generic-proxy accesses to global memory with later (or, on the
// writing side, earlier) async-proxy accesses: bulk tensor copies of data
// other CTAs wrote with plain stores, and plain reads of data bulk stores wrote
__device__ __forceinline__ void fence_proxy_async_global() { asm volatile("fence.proxy.async.global;\n" ::: "memory"); }
__device__ __forceinline__ void mbar_inval(uint64_t* b) {
  asm volatile("mbarrier.inval.shared::cta.b64 [%0];\n" ::"r"(smem_u32(b)) : "memory");
}

// One work item of the persistent batch step.  Kept out of line: the item
// bodies get the kernel's whole register budget, and the queue loop around
// them keeps (almost) nothing live across the call.
template <typename T, int R, int NWM, int NS_>
__device__ __noinline__ void persist_item(const BatchScene<T>& sp, const TfsfP& tf, const BatchMaps* maps, int4 it,
                                          int parity, int tile, int* err) {
  const int scene = static_cast<int>(static_cast<unsigned>(it.x) >> 16);
  const int4 item = make_int4((it.x & 0x7ff) | (((it.x >> 11) & 0x1f) << 16), it.y, it.z, it.w);
  const BatchMaps& bm = maps[scene];
  step_dispatch<T, R, NWM, NS_, true>(sp.g[parity], sp.g[1 - parity], sp.pm, sp.psh[parity], sp.psh[1 - parity], tf,
                                      sp.ad, item, sp.lut8, sp.disp, sp.n_mat, &bm.stage[tile][parity],
                                      &bm.store[tile][1 - parity], err);
}

// Persistent form of the batch step: n_steps steps of every scene in one
// launch.  A grid of resident CTAs draws tickets from a device queue
// (queue[0]); ticket q is item q % n_items of step q / n_items, so all items
// of a step are handed out before any of the next.  An item of step s > 0
// starts once every item of step s - 1 of its scene has finished: each CTA
// counts its finished items per scene (queue[1 + scene], release), the
// next step's items of that scene wait for the count s * scene_items[scene]
// (acquire).  That is the whole step-to-step dependency of a scene: the step
// reads the field set its previous step wrote and writes the set that step
// read.  A scene's next step can start while other scenes still finish the
// current one; no CTA ever waits for an item that has not been handed out,
// so the queue cannot deadlock.  The waits are bounded (err[1] polls, as the
// staging waits); a wait that runs out, or any earlier error, sets err[0] and
// every CTA stops at its next ticket.  queue[] is zeroed before each launch.
template <typename T, int R, int NWM, int NS_>
__global__ void __launch_bounds__(StepCfg<T, R, NWM, NS_>::NT, StepCfg<T, R, NWM, NS_>::min_blocks)
    k_step3_persist(const BatchScene<T>* scenes, const BatchMaps* maps, const int4* items, int n_items,
                    const int* scene_items, TimeP tp, int parity0, int n_steps, int tile, unsigned* queue, int* err) {
  using L = StepCfg<T, R, NWM, NS_>;
  __shared__ BatchScene<T> sp;
  __shared__ TfsfP s_tf;
  __shared__ unsigned s_ticket;
  __shared__ int s_go, s_cur;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  if (threadIdx.x == 0) s_cur = -1;  // scene whose parameters sit in sp
  for (;;) {
    if (threadIdx.x == 0) {
      const unsigned q = atomicAdd(queue, 1u);
      int go = q < static_cast<unsigned>(n_steps) * static_cast<unsigned>(n_items) &&
               *reinterpret_cast<volatile int*>(err) == 0;
      if (go && q >= static_cast<unsigned>(n_items)) {
        const unsigned s = q / static_cast<unsigned>(n_items);
        const int scene = static_cast<int>(static_cast<unsigned>(items[q - s * n_items].x) >> 16);
        const unsigned need = s * static_cast<unsigned>(scene_items[scene]);
        const int polls = err[1];
        int n = 0;
        while (ld_acquire_gpu(queue + 1 + scene) < need) {
          if (*reinterpret_cast<volatile int*>(err) != 0) { go = 0; break; }
          if (++n > polls) {
            atomicExch(err, 1);
            go = 0;
            break;
          }
          __nanosleep(128);
        }
        fence_proxy_async_global();  // the previous step's writes, before this CTA's bulk copies read them
      }
      s_ticket = q;
      s_go = go;
    }
    __syncthreads();
    if (!s_go) break;
    const unsigned s = s_ticket / static_cast<unsigned>(n_items);
    const int4 it = items[s_ticket - s * n_items];
    const int scene = static_cast<int>(static_cast<unsigned>(it.x) >> 16);
    if (scene != s_cur) {
      const int* src = reinterpret_cast<const int*>(scenes + scene);
      int* dst = reinterpret_cast<int*>(&sp);
      for (int w = threadIdx.x; w < static_cast<int>(sizeof(BatchScene<T>) / 4); w += blockDim.x) dst[w] = src[w];
      __syncthreads();
      if (threadIdx.x == 0) s_cur = scene;
    }
    if (threadIdx.x == 0) s_tf = tfsf_at_step(sp.tf, cur_step(tp) + s);  // incident-table rows of this item's step
    __syncthreads();
    persist_item<T, R, NWM, NS_>(sp, s_tf, maps, it, (parity0 + static_cast<int>(s)) & 1, tile, err);
    __threadfence();  // this thread's plain stores of the item, before the count below
    __syncthreads();  // every thread is done with the item and its shared memory
    if (threadIdx.x == 0) {
      uint64_t* bar = reinterpret_cast<uint64_t*>(smem_raw + ((128u - (smem_u32(smem_raw) & 127u)) & 127u) + L::off_b);
      for (int b = 0; b < NS_; ++b) mbar_inval(bar + b);  // the next item initialises them again
      fence_proxy_async_global();  // the item's bulk stores (completed by this thread), before the count
      red_release_gpu_add(queue + 1 + scene, 1u);
    }
  }
}

}  // namespace xfb
