// Scenes compiled by XFDTD_CORE, read from the arrays its Simulation::init
// produces (the data the reference's *HD wrappers copy to the device:
// FDTDCoefficientHD, src/calculation_param/fdtd_coefficient_hd.cu:9-51;
// PMLCorrectorHD, src/boundary/pml_corrector_hd.cu:8-34; TFSFCorrectorHD,
// src/waveform_source/tfsf/tfsf_corrector_hd.cu:9-73; ADEMethodStorageHD,
// src/material/ade_method/ade_method_hd.cu:5-24).
//
// The engine keeps one material id per cell and a table of coefficient sets,
// so the 18 per-cell coefficient arrays (and the per-cell ADE coefficients)
// are compressed: the coefficients every update reads at cell (i, j, k) form
// the cell's key, and cells with bitwise-equal keys share a material.  A
// material must have the isotropic form the one-sweep update uses (one ce for
// the three E components, cexhy = -ceyhx, ..., the H side alike); otherwise
// the arrays are refused.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <unordered_map>
#include <vector>

#include "xfb_internal.h"

namespace xfb {

namespace {

// element index of (i, j, k) in a row-major array of shape (s0, s1, s2)
inline size_t at3(int s1, int s2, int i, int j, int k) {
  return (static_cast<size_t>(i) * s1 + j) * s2 + k;
}

// shape of the field coefficient q belongs to (q / 3: Ex Ey Ez Hx Hy Hz)
void coeff_shape(const xfb_core_arrays& a, int q, int s[3]) {
  const int f = q / 3;
  s[0] = a.nx + (f == XFB_EY || f == XFB_EZ || f == XFB_HX ? 1 : 0);
  s[1] = a.ny + (f == XFB_EX || f == XFB_EZ || f == XFB_HY ? 1 : 0);
  s[2] = a.nz + (f == XFB_EX || f == XFB_EY || f == XFB_HZ ? 1 : 0);
}

}  // namespace

int compile_arrays(const xfb_core_arrays& a, Compiled& c, std::string* err) {
  auto fail = [&](const std::string& m) {
    if (err) *err = m;
    return XFB_ERR_INVALID;
  };
  if (a.precision != XFB_FP32 && a.precision != XFB_FP64) return fail("precision must be XFB_FP32 or XFB_FP64");
  if (a.nx < 1 || a.ny < 1 || a.nz < 1) return fail("grid must have at least one cell per axis");
  if (!(a.dx > 0 && a.dy > 0 && a.dz > 0 && a.dt > 0)) return fail("cell sizes and dt must be positive");
  for (int q = 0; q < kCoeffs; ++q)
    if (!a.coeff[q]) return fail("every one of the 18 coefficient arrays is required");
  const int P = a.ade_kind == XFB_ADE_NONE ? 0 : a.ade_poles;
  if (a.ade_kind < XFB_ADE_NONE || a.ade_kind > XFB_ADE_MLORENTZ) return fail("unknown ADE kind");
  if (a.ade_kind != XFB_ADE_NONE) {
    if (P < 1 || P > XFB_MAX_POLES) return fail("ADE needs 1..XFB_MAX_POLES poles");
    for (int q = 0; q < kAdeMat; ++q)
      if (!a.ade_cell[q]) return fail("ADE cell arrays missing");
    for (int q = 0; q < kAdePole; ++q)
      if (!a.ade_pole[q]) return fail("ADE pole arrays missing");
  }
  c = Compiled{};
  c.dim = 3;
  c.prec = a.precision;
  c.nx = a.nx; c.ny = a.ny; c.nz = a.nz;
  c.dx = a.dx; c.dy = a.dy; c.dz = a.dz; c.dt = a.dt;
  for (int q = 0; q < 3; ++q) c.origin[q] = a.origin[q];

  // ---- materials: one key per cell --------------------------------------
  int shp[kCoeffs][3];
  for (int q = 0; q < kCoeffs; ++q) coeff_shape(a, q, shp[q]);
  const int nkey = kCoeffs + (P ? kAdeMat + P * kAdePole : 0);
  std::unordered_map<std::string, int> ids;
  std::vector<double> keys;  // [n_mat][nkey]
  c.mat_id.assign(static_cast<size_t>(a.nx) * a.ny * a.nz, 0);
  std::vector<double> key(nkey), prev(nkey);
  int prev_id = -1;
  for (int i = 0; i < a.nx; ++i)
    for (int j = 0; j < a.ny; ++j)
      for (int k = 0; k < a.nz; ++k) {
        for (int q = 0; q < kCoeffs; ++q) key[q] = a.coeff[q][at3(shp[q][1], shp[q][2], i, j, k)];
        if (P) {
          const size_t cell = at3(a.ny, a.nz, i, j, k);
          for (int q = 0; q < kAdeMat; ++q) key[kCoeffs + q] = a.ade_cell[q][cell];
          for (int p = 0; p < P; ++p)
            for (int q = 0; q < kAdePole; ++q) key[kCoeffs + kAdeMat + p * kAdePole + q] = a.ade_pole[q][cell * P + p];
        }
        int id;
        if (prev_id >= 0 && std::memcmp(key.data(), prev.data(), nkey * sizeof(double)) == 0) {
          id = prev_id;  // runs along k usually share a material
        } else {
          std::string kb(reinterpret_cast<const char*>(key.data()), nkey * sizeof(double));
          auto it = ids.find(kb);
          if (it == ids.end()) {
            if (ids.size() >= XFB_MAX_MATERIALS)
              return fail("more than " + std::to_string(XFB_MAX_MATERIALS) + " distinct coefficient sets");
            it = ids.emplace(kb, static_cast<int>(ids.size())).first;
            keys.insert(keys.end(), key.begin(), key.end());
          }
          id = it->second;
          prev = key;
          prev_id = id;
        }
        c.mat_id[at3(a.ny, a.nz, i, j, k)] = static_cast<uint8_t>(id);
      }
  c.n_mat = static_cast<int>(ids.size());
  c.coeff.assign(static_cast<size_t>(c.n_mat) * kCoeffs, 0.0);
  c.coeff8.assign(static_cast<size_t>(c.n_mat) * 8, 0.0);
  c.mat_disp.assign(c.n_mat, 0);
  c.mat_is_pec.assign(c.n_mat, 0);
  c.ade_kind = P ? a.ade_kind : XFB_ADE_NONE;
  c.ade_poles = P;
  c.ade_mat.assign(static_cast<size_t>(c.n_mat) * kAdeMat, 0.0);
  c.ade_pole.assign(static_cast<size_t>(c.n_mat) * std::max(1, P) * kAdePole, 0.0);
  for (int m = 0; m < c.n_mat; ++m) {
    const double* kk = &keys[static_cast<size_t>(m) * nkey];
    double* k18 = &c.coeff[static_cast<size_t>(m) * kCoeffs];
    std::memcpy(k18, kk, kCoeffs * sizeof(double));
    // the compact form: ce, cb/dx, cb/dy, cb/dz, ch, db/dx, db/dy, db/dz,
    // with every other entry its copy or its negation (bitwise)
    const double ce = k18[CEXE], bx = k18[CEZHY], by = k18[CEXHZ], bz = k18[CEYHX];
    const double ch = k18[CHXH], dx = k18[CHYEZ], dy = k18[CHZEX], dz = k18[CHXEY];
    const bool iso = k18[CEYE] == ce && k18[CEZE] == ce && k18[CEYHZ] == -bx && k18[CEZHX] == -by &&
                     k18[CEXHY] == -bz && k18[CHYH] == ch && k18[CHZH] == ch && k18[CHZEY] == -dx &&
                     k18[CHXEZ] == -dy && k18[CHYEX] == -dz;
    if (!iso) return fail("material " + std::to_string(m) + ": coefficients not of the isotropic form the update uses");
    double* k8 = &c.coeff8[static_cast<size_t>(m) * 8];
    k8[0] = ce; k8[1] = bx; k8[2] = by; k8[3] = bz; k8[4] = ch; k8[5] = dx; k8[6] = dy; k8[7] = dz;
    c.mat_is_pec[m] = ce == 0 && bx == 0 && by == 0 && bz == 0;
    if (P) {
      std::memcpy(&c.ade_mat[static_cast<size_t>(m) * kAdeMat], kk + kCoeffs, kAdeMat * sizeof(double));
      std::memcpy(&c.ade_pole[static_cast<size_t>(m) * P * kAdePole], kk + kCoeffs + kAdeMat,
                  static_cast<size_t>(P) * kAdePole * sizeof(double));
      c.mat_disp[m] = kk[kCoeffs] != 0 ? 1 : 0;
    }
  }
  if (P) {  // the box of dispersive cells
    int b[6] = {c.nx, 0, c.ny, 0, c.nz, 0};
    for (int i = 0; i < c.nx; ++i)
      for (int j = 0; j < c.ny; ++j)
        for (int k = 0; k < c.nz; ++k)
          if (c.mat_disp[c.mat_id[at3(c.ny, c.nz, i, j, k)]]) {
            b[0] = std::min(b[0], i); b[1] = std::max(b[1], i + 1);
            b[2] = std::min(b[2], j); b[3] = std::max(b[3], j + 1);
            b[4] = std::min(b[4], k); b[5] = std::max(b[5], k + 1);
          }
    if (b[0] >= b[1])
      for (int& v : b) v = 0;
    std::memcpy(c.ade_box, b, sizeof(b));
  }

  // ---- CPML -------------------------------------------------------------
  const int n[3] = {c.nx, c.ny, c.nz};
  for (int f = 0; f < 6; ++f) {
    if (a.pml[f] < 0 || 2 * a.pml[f] > n[f / 2]) return fail("CPML thickness out of range");
    c.pml[f] = a.pml[f];
  }
  for (int ax = 0; ax < 3; ++ax) {
    const bool any = c.pml[2 * ax] + c.pml[2 * ax + 1] > 0;
    if (any && (!a.pml_ae[ax] || !a.pml_be[ax] || !a.pml_ah[ax] || !a.pml_bh[ax])) return fail("CPML profiles missing");
    c.pml_ae[ax].assign(n[ax] + 1, 0.0);
    c.pml_be[ax].assign(n[ax] + 1, 0.0);
    c.pml_ah[ax].assign(n[ax], 0.0);
    c.pml_bh[ax].assign(n[ax], 0.0);
    if (any) {
      std::memcpy(c.pml_ae[ax].data(), a.pml_ae[ax], (n[ax] + 1) * sizeof(double));
      std::memcpy(c.pml_be[ax].data(), a.pml_be[ax], (n[ax] + 1) * sizeof(double));
      std::memcpy(c.pml_ah[ax].data(), a.pml_ah[ax], n[ax] * sizeof(double));
      std::memcpy(c.pml_bh[ax].data(), a.pml_bh[ax], n[ax] * sizeof(double));
    }
  }

  // ---- TFSF -------------------------------------------------------------
  if (a.tfsf_enabled) {
    const int* t = a.tfsf_box;
    for (int ax = 0; ax < 3; ++ax)
      if (t[2 * ax] < 1 || t[2 * ax + 1] >= n[ax] || t[2 * ax + 1] <= t[2 * ax]) return fail("TFSF box does not fit");
    if (a.aux_nl < 2 || a.inc_steps < 0 || !a.e_inc || (a.inc_steps > 0 && !a.h_inc))
      return fail("TFSF incident tables missing");
    c.tfsf_on = 1;
    std::memcpy(c.tf, t, sizeof(c.tf));
    for (int ax = 0; ax < 3; ++ax) {
      if (!a.tfsf_proj_int[ax] || !a.tfsf_proj_half[ax]) return fail("TFSF projections missing");
      const int nb = t[2 * ax + 1] - t[2 * ax];
      c.proj_int[ax].assign(a.tfsf_proj_int[ax], a.tfsf_proj_int[ax] + nb + 1);
      c.proj_half[ax].assign(a.tfsf_proj_half[ax], a.tfsf_proj_half[ax] + nb + 2);
      c.tr_e[ax] = a.tfsf_transform_e[ax];
      c.tr_h[ax] = a.tfsf_transform_h[ax];
      c.ca[ax] = a.tfsf_ca[ax];
      c.cb[ax] = a.tfsf_cb[ax];
    }
    c.aux_nl = a.aux_nl;
    c.inc_given = true;
    c.inc_steps = a.inc_steps;
    c.e_inc.assign(a.e_inc, a.e_inc + static_cast<size_t>(a.inc_steps + 1) * (a.aux_nl + 1));
    c.h_inc.assign(a.h_inc ? a.h_inc : a.e_inc, (a.h_inc ? a.h_inc : a.e_inc) + static_cast<size_t>(a.inc_steps) * a.aux_nl);
  }

  // ---- NF2FF, monitors ----------------------------------------------------
  if (a.nf2ff_enabled) {
    const int* b = a.nf2ff_box;
    for (int ax = 0; ax < 3; ++ax)
      if (b[2 * ax] < 1 || b[2 * ax + 1] >= n[ax] || b[2 * ax + 1] <= b[2 * ax]) return fail("NF2FF box does not fit");
    if (a.n_freqs < 1 || !a.freqs) return fail("NF2FF needs at least one frequency");
    c.nf_on = 1;
    std::memcpy(c.nf, b, sizeof(c.nf));
    c.freqs.assign(a.freqs, a.freqs + a.n_freqs);
  }
  if (a.nf2ff_td_enabled) {
    const int* b = a.nf2ff_td_box;
    for (int ax = 0; ax < 3; ++ax)
      if (b[2 * ax] < 1 || b[2 * ax + 1] >= n[ax] || b[2 * ax + 1] <= b[2 * ax])
        return fail("time-domain NF2FF box does not fit");
    if (!std::isfinite(a.nf2ff_td_theta) || !std::isfinite(a.nf2ff_td_phi))
      return fail("time-domain NF2FF direction must be finite");
    c.td_on = 1;
    std::memcpy(c.td, b, sizeof(c.td));
    compile_td(c, a.nf2ff_td_theta, a.nf2ff_td_phi);
  }
  for (int p = 0; p < a.n_probes; ++p) {
    const xfb_probe& pr = a.probes[p];
    if (pr.field < 0 || pr.field > 5) return fail("probe field out of range");
    int s[3];
    coeff_shape(a, 3 * pr.field, s);
    for (int ax = 0; ax < 3; ++ax)
      if (pr.index[ax] < 0 || pr.index[ax] >= s[ax]) return fail("probe index outside the component");
    c.probes.push_back(pr);
  }
  for (int m = 0; m < a.n_movies; ++m) {
    const xfb_movie& mv = a.movies[m];
    if (mv.field < 0 || mv.field > 5 || mv.interval < 1) return fail("bad movie monitor");
    int s[3];
    coeff_shape(a, 3 * mv.field, s);
    for (int ax = 0; ax < 3; ++ax)
      if (mv.lo[ax] < 0 || mv.hi[ax] > s[ax] || mv.hi[ax] <= mv.lo[ax]) return fail("movie box outside the component");
    c.movies.push_back(mv);
  }
  return XFB_OK;
}

}  // namespace xfb
