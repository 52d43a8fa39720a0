// One-sweep 3-D time step: H half-step and E half-step of a whole Yee step in
// a single kernel (temporal fusion), so each field component crosses HBM once
// per step (read E^n, H^{n-1/2}; write H^{n+1/2}, E^{n+1}) instead of the
// 9 + 9 transfers of two separate half-step kernels.
//
// Tiling.  A CTA owns a (TJ x TK) tile of (j, k) and marches along i over a
// chunk of planes.  For every plane i:
//   * staging: all six components and the material id of plane i+3 are copied
//     into a 4-deep shared-memory ring with cp.async (planes i and i+1 are
//     resident, i+2, i+3 in flight), rows j0-1 .. j0+TJ and a 16-byte aligned
//     k window [k0-HP, k0+TK+HP).  No global load sits on the critical path of
//     the bulk update.
//   * H pass (plane i): one thread per cell of the (TJ+1) x (TK+1) tile that
//     includes a one-cell halo on the low j and k sides (the E update needs H
//     at j-1 and k-1).  Halo cells are recomputed here instead of being read
//     from the neighbouring CTA, so no CTA ever waits for another.  H^{n+1/2}
//     goes to a 3-plane shared ring and, for owned cells, to HBM.
//   * E pass (plane i-1, one plane behind): one thread per owned cell, from the
//     shared H planes i-1 and i-2 and the E^n values the thread took from the
//     ring one iteration earlier.  With the skew the H and E passes of an
//     iteration touch disjoint shared data: one barrier per plane.
// Fields and the H-side CPML psi are ping-pong buffered (read set s, write set
// d) so a neighbour's halo reads never see a half-updated value; E-side psi,
// ADE state and material ids are only touched by their owner.
//
// The per-cell arithmetic (hNext/eNext, TFSF, CPML, ADE and their order) is the
// one of k_h3/k_e3, so results are identical to the split path and, in FP64,
// to the CPU restatement bit for bit.
#pragma once

#include "kernels.cuh"

namespace xfb {

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

// Shared-memory layout of k_step3 (dynamic).
template <typename T, int TK, int TJ>
struct StepSmem {
  static constexpr int NS = 4;               // staging ring depth: planes i, i+1 in use, i+2, i+3 in flight
  static constexpr int HP = 16 / sizeof(T);  // elements per 16-byte copy
  static constexpr int RW = TK + 2 * HP;     // staged row width
  static constexpr int RH = TJ + 2;          // staged rows j0-1 .. j0+TJ
  static constexpr int MW = TK + 32;         // material-id row window [k0-16, k0+TK+16)
  static constexpr int HW = TK + 1, HH = TJ + 1;  // H tile with the low halos
  static constexpr int LUTM = 256;           // every material fits (ids are bytes)
  static constexpr int CW = RW / HP;         // 16-byte chunks per staged field row
  static constexpr int MC = MW / 16;         // 16-byte chunks per material row
  static constexpr size_t plane = static_cast<size_t>(RH) * RW;  // elements of one staged component plane
  static constexpr size_t f_bytes = NS * 6 * plane * sizeof(T);
  static constexpr size_t h_bytes = (3ull * 3 * HH * HW * sizeof(T) + 15) / 16 * 16;  // H planes i, i-1, i-2
  static constexpr size_t l_bytes = LUTM * 8 * sizeof(T);
  static constexpr size_t d_bytes = LUTM;
  static constexpr size_t bytes = f_bytes + h_bytes + l_bytes + d_bytes + NS * RH * MW;
  static constexpr int threads = ((TK + 1) * (TJ + 1) + 31) / 32 * 32;
  // resident CTAs per SM the register budget is sized for
  static constexpr int min_blocks = TJ <= 4 ? 4 : TJ <= 8 ? 3 : 2;
  static_assert(RH * CW <= threads && RH * MC <= threads, "one staging chunk per thread and component");
};

template <typename T, int TK, int TJ>
__global__ void __launch_bounds__(StepSmem<T, TK, TJ>::threads, StepSmem<T, TK, TJ>::min_blocks)
    k_step3(GridP<T> s, GridP<T> d, PmlP<T> pm, PsiH<T> ps, PsiH<T> pd, TfsfP tf_in, AdeP<T> ad, TimeP tp,
            int i_chunk, const T* lut8, const uint8_t* disp, int n_mat) {
  using L = StepSmem<T, TK, TJ>;
  constexpr int NS = L::NS, HP = L::HP, RW = L::RW, RH = L::RH, MW = L::MW, HW = L::HW, HH = L::HH;
  constexpr int CW = L::CW, MC = L::MC, NT = L::threads;
  constexpr int PL = static_cast<int>(L::plane);
  constexpr int HPL = HH * HW;  // elements of one shared H component plane
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* sF = reinterpret_cast<T*>(smem_raw);                                       // [NS][6][RH][RW]
  T* sH = reinterpret_cast<T*>(smem_raw + L::f_bytes);                          // [2][3][HH][HW]
  T* sL = reinterpret_cast<T*>(smem_raw + L::f_bytes + L::h_bytes);             // [LUTM][8]
  uint8_t* sD = smem_raw + L::f_bytes + L::h_bytes + L::l_bytes;                // [LUTM]
  uint8_t* sM = smem_raw + L::f_bytes + L::h_bytes + L::l_bytes + L::d_bytes;   // [NS][RH][MW]

  const TfsfP tf = tfsf_at_step(tf_in, cur_step(tp));
  const int tid = threadIdx.x;
  const int k0 = blockIdx.x * TK, j0 = blockIdx.y * TJ;
  const int i_start = blockIdx.z * i_chunk;
  const int i_end = min(s.nx, i_start + i_chunk);
  if (i_start >= i_end) return;  // uniform per CTA
  const int i_first = i_start > 0 ? i_start - 1 : 0;
  const long long sx = s.sx, sy = s.sy;
  for (int q = tid; q < n_mat * 8; q += NT) sL[q] = lut8[q];
  for (int q = tid; q < n_mat; q += NT) sD[q] = disp[q];

  // staging: thread tid copies chunk (r, cc) = (tid / CW, tid % CW) of every
  // component row window, and chunk tid of the material window
  const bool st_f = tid < RH * CW, st_m = tid < RH * MC;
  const int f_r = tid / CW, f_c = tid - (tid / CW) * CW;
  const int m_r = tid / MC, m_c = tid - (tid / MC) * MC;
  const int f_soff = f_r * RW + f_c * HP;
  const long long f_goff = static_cast<long long>(j0 - 1 + f_r) * sy + (k0 - HP) + f_c * HP;
  const int m_soff = m_r * MW + m_c * 16;
  const long long m_goff = static_cast<long long>(j0 - 1 + m_r) * sy + (k0 - 16) + m_c * 16;
  auto stage = [&](int plane) {
    if (plane <= s.nx) {
      const int st = plane % NS;
      const long long pb = static_cast<long long>(plane) * sx;
      if (st_f) {
        T* dst = sF + st * 6 * PL + f_soff;
        const long long go = pb + f_goff;
        cp_async16(dst, s.ex + go);
        cp_async16(dst + PL, s.ey + go);
        cp_async16(dst + 2 * PL, s.ez + go);
        cp_async16(dst + 3 * PL, s.hx + go);
        cp_async16(dst + 4 * PL, s.hy + go);
        cp_async16(dst + 5 * PL, s.hz + go);
      }
      if (st_m) cp_async16(sM + st * RH * MW + m_soff, s.mid + pb + m_goff);
    }
    cp_async_commit();
  };

  for (int q = tid; q < 3 * 3 * HPL; q += NT) sH[q] = T(0);
  for (int q = 0; q < NS - 1; ++q) stage(i_first + q);

  // ---- per-thread constants ------------------------------------------------
  // H-pass cell: tile + low halos, (hr, hc) in [0,HH) x [0,HW)
  const bool hcell = tid < HPL;
  const int hr = tid / HW, hc = tid - (tid / HW) * HW;
  const int hj = j0 - 1 + hr, hk = k0 - 1 + hc;
  const bool hvalid = hcell && hj >= 0 && hk >= 0 && hj < s.ny && hk < s.nz;
  const bool hown = hvalid && hr > 0 && hc > 0;
  const int hsy = slab(hj, s.ny, pm.L[2], pm.L[3]);
  const int hsz = slab(hk, s.nz, pm.L[4], pm.L[5]);
  const int hF = hr * RW + hc - 1 + HP;   // staged offset of (hj, hk)
  const int hM = hr * MW + hc - 1 + 16;   // material offset
  const int hS = hr * HW + hc;            // sH offset
  const long long hG = static_cast<long long>(hj) * sy + hk;  // global offset inside a plane
  const bool h_tf_line = tf.on && ((hj == tf.js - 1 || hj == tf.je) || (hk == tf.ks - 1 || hk == tf.ke));
  // E-pass cell
  const bool ecell = tid < TJ * TK;
  const int er = tid / TK, ec = tid - (tid / TK) * TK;
  const int j = j0 + er, k = k0 + ec;
  const bool eown = ecell && j < s.ny && k < s.nz;
  const bool jpos = j > 0, kpos = k > 0;
  const int sy_pml = slab(j, s.ny, pm.L[2], pm.L[3]);
  const int sz_pml = slab(k, s.nz, pm.L[4], pm.L[5]);
  const int eF = (er + 1) * RW + ec + HP;
  const int eM = (er + 1) * MW + ec + 16;
  const int eS = (er + 1) * HW + ec + 1;
  const long long eG = static_cast<long long>(j) * sy + k;
  const bool e_tf_line = tf.on && ((j == tf.js || j == tf.je) || (k == tf.ks || k == tf.ke));
  const bool has_ade = ad.kind != kAdeNone;
  // E^n and material of the owned cell, taken from the staging ring while the
  // plane is current (one iteration before its E pass)
  T ex_o = 0, ey_o = 0, ez_o = 0;
  int em = 0;

  // Iteration i computes H of plane i and E of plane i-1 (skewed by one plane,
  // so the E pass only reads H planes finished before the iteration's barrier).
  for (int i = i_first; i <= i_end; ++i) {
    const int ie = i - 1;
    const bool do_h = i < i_end;
    const bool write_h = do_h && i >= i_start;
    const bool h_active = do_h && hvalid && (write_h || hown);
    const bool e_active = eown && ie >= i_start;
    const bool upd_x = jpos && kpos, upd_y = ie > 0 && kpos, upd_z = ie > 0 && jpos;
    cp_async_wait<NS - 3>();  // planes i and i+1 have landed (this thread's copies)
    __syncthreads();          // ... everyone's copies; iteration i-1 is complete everywhere
    stage(i + NS - 1);        // into the slot of plane i-1, whose last readers finished iteration i-1
    const int cur = i % NS, nxt = (i + 1) % NS;
    const T* Fc = sF + cur * 6 * PL;
    const T* Fn = sF + nxt * 6 * PL;
    const uint8_t* Mc = sM + cur * RH * MW;
    T* Hc = sH + (i % 3) * 3 * HPL;              // H plane i (written here)
    const T* He = sH + ((i + 2) % 3) * 3 * HPL;  // H plane i-1
    const T* Hp = sH + ((i + 1) % 3) * 3 * HPL;  // H plane i-2
    // ---- H pass, plane i ----------------------------------------------------
    if (h_active) {
      const int sxp = slab(i, s.nx, pm.L[0], pm.L[1]);
      const bool tf_hplane = tf.on && (i == tf.is - 1 || i == tf.ie);
      const int m = Mc[hM];
      const C4<T> cf = ld_c4(sL + 8 * m + 4);  // ch, db/dx, db/dy, db/dz
      const T* f = Fc + hF;
      const T ex_c = f[0], ey_c = f[PL], ez_c = f[2 * PL];
      const T d_hx_a = f[PL + 1] - ey_c;         // Hx: Ey along z
      const T d_hx_b = f[2 * PL + RW] - ez_c;    // Hx: Ez along y
      const T d_hy_a = Fn[hF + 2 * PL] - ez_c;   // Hy: Ez along x
      const T d_hy_b = f[1] - ex_c;              // Hy: Ex along z
      const T d_hz_a = f[RW] - ex_c;             // Hz: Ex along y
      const T d_hz_b = Fn[hF + PL] - ey_c;       // Hz: Ey along x
      // hNext with chxey = db/dz, chxez = -db/dy, chyez = db/dx, chyex = -db/dz,
      // chzex = db/dy, chzey = -db/dx
      T hxv = cf.c * f[3 * PL] + cf.z * d_hx_a - cf.y * d_hx_b;
      T hyv = cf.c * f[4 * PL] + cf.x * d_hy_a - cf.z * d_hy_b;
      T hzv = cf.c * f[5 * PL] + cf.y * d_hz_a - cf.x * d_hz_b;
      if (h_tf_line || tf_hplane) {
        const int jj = hj, kk = hk;
        const bool iin = i >= tf.is && i <= tf.ie, jin = jj >= tf.js && jj <= tf.je, kin = kk >= tf.ks && kk <= tf.ke;
        if (jin && jj < tf.je && kin) {
          if (i == tf.is - 1) add_inc(hzv, ey_inc(tf, tf.is, jj, kk), tf.cb[0]);
          if (i == tf.ie) add_inc(hzv, ey_inc(tf, tf.ie, jj, kk), -tf.cb[0]);
        }
        if (iin && i < tf.ie && kin) {
          if (jj == tf.js - 1) add_inc(hzv, ex_inc(tf, i, tf.js, kk), -tf.cb[1]);
          if (jj == tf.je) add_inc(hzv, ex_inc(tf, i, tf.je, kk), tf.cb[1]);
        }
        if (iin && jin && jj < tf.je) {
          if (kk == tf.ks - 1) add_inc(hxv, ey_inc(tf, i, jj, tf.ks), -tf.cb[2]);
          if (kk == tf.ke) add_inc(hxv, ey_inc(tf, i, jj, tf.ke), tf.cb[2]);
        }
        if (iin && kin && kk < tf.ke) {
          if (jj == tf.js - 1) add_inc(hxv, ez_inc(tf, i, tf.js, kk), tf.cb[1]);
          if (jj == tf.je) add_inc(hxv, ez_inc(tf, i, tf.je, kk), -tf.cb[1]);
        }
        if (iin && i < tf.ie && jin) {
          if (kk == tf.ks - 1) add_inc(hyv, ex_inc(tf, i, jj, tf.ks), tf.cb[2]);
          if (kk == tf.ke) add_inc(hyv, ex_inc(tf, i, jj, tf.ke), -tf.cb[2]);
        }
        if (jin && kin && kk < tf.ke) {
          if (i == tf.is - 1) add_inc(hyv, ez_inc(tf, tf.is, jj, kk), -tf.cb[0]);
          if (i == tf.ie) add_inc(hyv, ez_inc(tf, tf.ie, jj, kk), tf.cb[0]);
        }
      }
      const bool wpsi = write_h && hown;
      if (sxp >= 0 || hsy >= 0 || hsz >= 0) {
        if (sxp >= 0) {
          const long long p = sxp * sx + hG;
          const T a = pm.ah[0][i], b = pm.bh[0][i];
          const T py = b * ps.hy_x[p] + a * d_hy_a;
          hyv = hyv + cf.x * py;   // c_psi = chyez
          const T pz = b * ps.hz_x[p] + a * d_hz_b;
          hzv = hzv - cf.x * pz;   // c_psi = chzey
          if (wpsi) { pd.hy_x[p] = py; pd.hz_x[p] = pz; }
        }
        if (hsy >= 0) {
          const long long p = static_cast<long long>(i) * pm.ysx + hsy * sy + hk;
          const T a = pm.ah[1][hj], b = pm.bh[1][hj];
          const T pz = b * ps.hz_y[p] + a * d_hz_a;
          hzv = hzv + cf.y * pz;   // chzex
          const T px = b * ps.hx_y[p] + a * d_hx_b;
          hxv = hxv - cf.y * px;   // chxez
          if (wpsi) { pd.hz_y[p] = pz; pd.hx_y[p] = px; }
        }
        if (hsz >= 0) {
          const long long p = static_cast<long long>(i) * pm.zsx + static_cast<long long>(hj) * pm.zsy + hsz;
          const T a = pm.ah[2][hk], b = pm.bh[2][hk];
          const T px = b * ps.hx_z[p] + a * d_hx_a;
          hxv = hxv + cf.z * px;   // chxey
          const T py = b * ps.hy_z[p] + a * d_hy_b;
          hyv = hyv - cf.z * py;   // chyex
          if (wpsi) { pd.hx_z[p] = px; pd.hy_z[p] = py; }
        }
      }
      Hc[hS] = hxv;
      Hc[HPL + hS] = hyv;
      Hc[2 * HPL + hS] = hzv;
      if (wpsi) {
        const long long idx = static_cast<long long>(i) * sx + hG;
        d.hx[idx] = hxv; d.hy[idx] = hyv; d.hz[idx] = hzv;
      }
    }
    // ---- E pass, plane ie = i-1 ----------------------------------------------
    if (e_active) {
      const long long idx = static_cast<long long>(ie) * sx + eG;
      const int m = em;
      const C4<T> cf = ld_c4(sL + 8 * m);  // ce, cb/dx, cb/dy, cb/dz
      const T hx_c = He[eS], hy_c = He[HPL + eS], hz_c = He[2 * HPL + eS];
      const T hx_km = He[eS - 1], hx_jm = He[eS - HW];
      const T hy_km = He[HPL + eS - 1];
      const T hz_jm = He[2 * HPL + eS - HW];
      const T hy_p = Hp[HPL + eS], hz_p = Hp[2 * HPL + eS];  // plane ie-1
      const T d_ex_a = hy_c - hy_km;
      const T d_ex_b = hz_c - hz_jm;
      const T d_ey_a = hz_c - hz_p;
      const T d_ey_b = hx_c - hx_km;
      const T d_ez_a = hx_c - hx_jm;
      const T d_ez_b = hy_c - hy_p;
      // eNext with cexhy = -cb/dz, cexhz = cb/dy, ceyhz = -cb/dx, ceyhx = cb/dz,
      // cezhx = -cb/dy, cezhy = cb/dx
      T exv = cf.c * ex_o - cf.z * d_ex_a + cf.y * d_ex_b;
      T eyv = cf.c * ey_o - cf.x * d_ey_a + cf.z * d_ey_b;
      T ezv = cf.c * ez_o - cf.y * d_ez_a + cf.x * d_ez_b;
      if (has_ade && sD[m]) {
        const long long abi = static_cast<long long>(ie - ad.b0) * ad.bsx + static_cast<long long>(j - ad.b2) * ad.bsy + (k - ad.b4);
        if (upd_x) exv = ade_e(ad, 0, abi, m, ex_o, exv);
        if (upd_y) eyv = ade_e(ad, 1, abi, m, ey_o, eyv);
        if (upd_z) ezv = ade_e(ad, 2, abi, m, ez_o, ezv);
      }
      const bool tf_eplane = tf.on && (ie == tf.is || ie == tf.ie);
      if (e_tf_line || tf_eplane) {
        const int i = ie;
        const bool iin = i >= tf.is && i <= tf.ie, jin = j >= tf.js && j <= tf.je, kin = k >= tf.ks && k <= tf.ke;
        if (jin && kin && k < tf.ke) {
          if (i == tf.is) add_inc(ezv, hy_inc(tf, tf.is - 1, j, k), -tf.ca[0]);
          if (i == tf.ie) add_inc(ezv, hy_inc(tf, tf.ie, j, k), tf.ca[0]);
        }
        if (iin && kin && k < tf.ke) {
          if (j == tf.js) add_inc(ezv, hx_inc(tf, i, tf.js - 1, k), tf.ca[1]);
          if (j == tf.je) add_inc(ezv, hx_inc(tf, i, tf.je, k), -tf.ca[1]);
        }
        if (iin && i < tf.ie && jin) {
          if (k == tf.ks) add_inc(exv, hy_inc(tf, i, j, tf.ks - 1), tf.ca[2]);
          if (k == tf.ke) add_inc(exv, hy_inc(tf, i, j, tf.ke), -tf.ca[2]);
        }
        if (iin && i < tf.ie && kin) {
          if (j == tf.js) add_inc(exv, hz_inc(tf, i, tf.js - 1, k), -tf.ca[1]);
          if (j == tf.je) add_inc(exv, hz_inc(tf, i, tf.je, k), tf.ca[1]);
        }
        if (iin && jin && j < tf.je) {
          if (k == tf.ks) add_inc(eyv, hx_inc(tf, i, j, tf.ks - 1), -tf.ca[2]);
          if (k == tf.ke) add_inc(eyv, hx_inc(tf, i, j, tf.ke), tf.ca[2]);
        }
        if (jin && j < tf.je && kin) {
          if (i == tf.is) add_inc(eyv, hz_inc(tf, tf.is - 1, j, k), tf.ca[0]);
          if (i == tf.ie) add_inc(eyv, hz_inc(tf, tf.ie, j, k), -tf.ca[0]);
        }
      }
      const int sxe = slab(ie, s.nx, pm.L[0], pm.L[1]);
      if (sxe >= 0 || sy_pml >= 0 || sz_pml >= 0) {
        if (sxe >= 0) {
          const long long p = sxe * sx + eG;
          const T a = pm.ae[0][ie], b = pm.be[0][ie];
          if (upd_y) { T q = b * pm.ey_x[p] + a * d_ey_a; pm.ey_x[p] = q; eyv = eyv - cf.x * q; }  // ceyhz
          if (upd_z) { T q = b * pm.ez_x[p] + a * d_ez_b; pm.ez_x[p] = q; ezv = ezv + cf.x * q; }  // cezhy
        }
        if (sy_pml >= 0) {
          const long long p = static_cast<long long>(ie) * pm.ysx + sy_pml * sy + k;
          const T a = pm.ae[1][j], b = pm.be[1][j];
          if (upd_z) { T q = b * pm.ez_y[p] + a * d_ez_a; pm.ez_y[p] = q; ezv = ezv - cf.y * q; }  // cezhx
          if (upd_x) { T q = b * pm.ex_y[p] + a * d_ex_b; pm.ex_y[p] = q; exv = exv + cf.y * q; }  // cexhz
        }
        if (sz_pml >= 0) {
          const long long p = static_cast<long long>(ie) * pm.zsx + static_cast<long long>(j) * pm.zsy + sz_pml;
          const T a = pm.ae[2][k], b = pm.be[2][k];
          if (upd_x) { T q = b * pm.ex_z[p] + a * d_ex_a; pm.ex_z[p] = q; exv = exv - cf.z * q; }  // cexhy
          if (upd_y) { T q = b * pm.ey_z[p] + a * d_ey_b; pm.ey_z[p] = q; eyv = eyv + cf.z * q; }  // ceyhx
        }
      }
      // E components on PEC walls keep their value in the new buffer
      d.ex[idx] = upd_x ? exv : ex_o;
      d.ey[idx] = upd_y ? eyv : ey_o;
      d.ez[idx] = upd_z ? ezv : ez_o;
    }
    // E-pass inputs of plane i for the next iteration
    if (eown && do_h) {
      em = Mc[eM];
      ex_o = Fc[eF]; ey_o = Fc[PL + eF]; ez_o = Fc[2 * PL + eF];
    }
  }
  cp_async_wait<0>();
}

}  // namespace xfb
