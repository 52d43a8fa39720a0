// Host scene compiler: xfb_scene -> Compiled.
//
// This is the work XFDTD_CORE's Simulation::init does before the reference
// copies arrays to the device (src/simulation/simulation_hd.cu:259-267):
// voxelisation, Yee update coefficients, CPML profiles, TFSF geometry and the
// NF2FF surfaces.  XFDTD_CORE's source is not part of the reference, so every
// formula here is restated from the published literature and named:
//   * Yee coefficients with conductivity: Taflove & Hagness, Computational
//     Electrodynamics, 3rd ed. (T&H), eqs. 3.29-3.34 (the same form as the
//     reference prototype test/2d.cu:692-735).
//   * CPML (CFS, kappa = 1): Roden & Gedney 2000; T&H section 7.9, eqs.
//     7.102-7.114, sigma_opt from T&H eq. 7.67.
//   * ADE dispersive media: T&H section 9.4 (Debye, Drude: trapezoidal
//     two-level recursions; Lorentz / modified Lorentz: the three-level
//     central-difference recursion of T&H 9.4.3 generalised to a first-order
//     numerator).
//   * TFSF plane-wave geometry: the projection / auxiliary-grid construction of
//     the reference prototype test/2d.cu:760-890 extended to three axes.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <sstream>

#include "xfb_internal.h"

namespace xfb {

namespace {

bool inside(const xfb_object& o, double x, double y, double z) {
  const double* p = o.p;
  switch (o.shape) {
    case XFB_SHAPE_CUBE: {
      const double c[3] = {x, y, z};
      for (int a = 0; a < 3; ++a) {
        const double lo = p[a];
        const double hi = std::isinf(p[3 + a]) ? std::numeric_limits<double>::infinity() : p[a] + p[3 + a];
        if (!(c[a] >= lo && c[a] < hi)) return false;
      }
      return true;
    }
    case XFB_SHAPE_SPHERE: {
      const double ddx = x - p[0], ddy = y - p[1], ddz = z - p[2];
      return ddx * ddx + ddy * ddy + ddz * ddz <= p[3] * p[3];
    }
    case XFB_SHAPE_CYLINDER: {
      const int ax = static_cast<int>(p[4]);
      const double c[3] = {x, y, z};
      double r2 = 0;
      for (int a = 0; a < 3; ++a) {
        if (a == ax) continue;
        const double d = c[a] - (std::isinf(p[a]) ? 0.0 : p[a]);
        r2 += d * d;
      }
      if (r2 > p[3] * p[3]) return false;
      if (std::isinf(p[5])) return true;
      const double ca = std::isinf(p[ax]) ? 0.0 : p[ax];
      return std::fabs(c[ax] - ca) <= 0.5 * p[5];
    }
  }
  return false;
}

// Convert one pole to the general (a0, a1, b0, b1, b2) form.
void pole_to_mlorentz(const xfb_pole& p, double out[5]) {
  switch (p.kind) {
    case XFB_POLE_DEBYE:  // d_eps / (1 + jw tau)
      out[0] = p.p[0]; out[1] = 0; out[2] = 1; out[3] = p.p[1]; out[4] = 0;
      break;
    case XFB_POLE_DRUDE:  // wp^2 / (jw gamma + (jw)^2)
      out[0] = p.p[0] * p.p[0]; out[1] = 0; out[2] = 0; out[3] = p.p[1]; out[4] = 1;
      break;
    case XFB_POLE_LORENTZ:  // d_eps w0^2 / (w0^2 + 2 delta jw + (jw)^2)
      out[0] = p.p[0] * p.p[1] * p.p[1]; out[1] = 0; out[2] = p.p[1] * p.p[1];
      out[3] = 2 * p.p[2]; out[4] = 1;
      break;
    default:
      for (int i = 0; i < 5; ++i) out[i] = p.p[i];
  }
}

}  // namespace

double waveform(const Compiled& c, double t) {
  const double u = (t - c.wave_t0) / c.wave_tau;
  const double g = std::exp(-u * u);
  if (c.wave_kind == XFB_WAVE_COS_GAUSSIAN) return g * std::cos(2 * kPi * c.wave_freq * (t - c.wave_t0));
  return g;
}

void size_tables(Compiled& c, long long total_steps) {
  c.total_steps = total_steps;
  c.td_bins = c.td_on ? total_steps + c.td_span : 0;
  c.aux_source.assign(static_cast<size_t>(total_steps + 1), 0.0);
  if (c.tfsf_on && !c.inc_given)
    for (long long t = 0; t <= total_steps; ++t) c.aux_source[t] = waveform(c, t * c.dt);
  const size_t nf = c.freqs.size();
  c.te.assign(nf * static_cast<size_t>(total_steps) * 2, 0.0);
  c.th.assign(nf * static_cast<size_t>(total_steps) * 2, 0.0);
  // DFT kernels of the running transform: E after step t lives at (t+1) dt,
  // H after step t at (t+1/2) dt (the reference eTime/hTime convention,
  // include/xfdtd_cuda/calculation_param/time_param.cuh:42-50).
  for (size_t f = 0; f < nf; ++f) {
    const double w = 2 * kPi * c.freqs[f];
    for (long long t = 0; t < total_steps; ++t) {
      const double pe = w * (t + 1.0) * c.dt, ph = w * (t + 0.5) * c.dt;
      const size_t o = (f * total_steps + t) * 2;
      c.te[o] = c.dt * std::cos(pe);
      c.te[o + 1] = -c.dt * std::sin(pe);
      c.th[o] = c.dt * std::cos(ph);
      c.th[o + 1] = -c.dt * std::sin(ph);
    }
  }
}

static FaceGeom box_face(const int* b, int face) {
  FaceGeom g{};
  g.axis = face / 2;
  g.positive = face % 2;
  g.i0 = b[0]; g.j0 = b[2]; g.k0 = b[4];
  g.ni = b[1] - b[0]; g.nj = b[3] - b[2]; g.nk = b[5] - b[4];
  if (g.axis == 0) { g.i0 = g.positive ? b[1] : b[0]; g.ni = 1; }
  if (g.axis == 1) { g.j0 = g.positive ? b[3] : b[2]; g.nj = 1; }
  if (g.axis == 2) { g.k0 = g.positive ? b[5] : b[4]; g.nk = 1; }
  return g;
}

FaceGeom face_geom(const Compiled& c, int face) { return box_face(c.nf, face); }
FaceGeom td_face_geom(const Compiled& c, int face) { return box_face(c.td, face); }

static void td_position(const Compiled& c, int face, int i, int j, int k, double r[3]) {
  const int ax = face / 2;
  const double d[3] = {c.dx, c.dy, c.dz};
  const int n[3] = {i, j, k};
  for (int a = 0; a < 3; ++a) r[a] = c.origin[a] + (n[a] + (a == ax ? 0.0 : 0.5)) * d[a];
}

double td_delay_steps(const Compiled& c, int face, int i, int j, int k) {
  double r[3];
  td_position(c, face, i, j, k, r);
  // timeDelay / (C_0 dt) in the reference's operation order
  // (nf2ff_time_domain_data.cuh:64-71, nf2ff_time_domain_data.cu:145-147)
  const double delay = c.td_ref - (r[0] * c.td_dir[0] + r[1] * c.td_dir[1] + r[2] * c.td_dir[2]);
  return delay / (kTdC0 * c.dt);
}

// Direction, reference distance and bin span of a time-domain NF2FF whose
// box c.td is set.
void compile_td(Compiled& c, double theta, double phi) {
  c.td_theta = theta;
  c.td_phi = phi;
  c.td_dir[0] = std::sin(theta) * std::cos(phi);
  c.td_dir[1] = std::sin(theta) * std::sin(phi);
  c.td_dir[2] = std::cos(theta);
  // reference distance: the largest r . dir over the sample points, so every
  // delay is >= 0; then the largest bin offset a step reaches
  double best = -std::numeric_limits<double>::infinity();
  for (int f = 0; f < 6; ++f) {
    const FaceGeom g = td_face_geom(c, f);
    for (int i = g.i0; i < g.i0 + g.ni; ++i)
      for (int j = g.j0; j < g.j0 + g.nj; ++j)
        for (int k = g.k0; k < g.k0 + g.nk; ++k) {
          double r[3];
          td_position(c, f, i, j, k, r);
          best = std::max(best, r[0] * c.td_dir[0] + r[1] * c.td_dir[1] + r[2] * c.td_dir[2]);
        }
  }
  c.td_ref = best;
  double dmax = 0;
  for (int f = 0; f < 6; ++f) {
    const FaceGeom g = td_face_geom(c, f);
    for (int i = g.i0; i < g.i0 + g.ni; ++i)
      for (int j = g.j0; j < g.j0 + g.nj; ++j)
        for (int k = g.k0; k < g.k0 + g.nk; ++k) dmax = std::max(dmax, td_delay_steps(c, f, i, j, k));
  }
  // bins t + floor(delay + 1/2) + {0, 1, 2} (the rounding of the sum with t
  // can add one)
  c.td_span = static_cast<int>(std::floor(dmax + 0.5)) + 3;
}

int compile_scene(const xfb_scene& s, Compiled& c, std::string* err) {
  auto fail = [&](const std::string& m) {
    if (err) *err = m;
    return XFB_ERR_INVALID;
  };
  if (s.dim != 2 && s.dim != 3) return fail("scene.dim must be 2 or 3");
  if (s.precision != XFB_FP32 && s.precision != XFB_FP64) return fail("scene.precision must be XFB_FP32 or XFB_FP64");
  if (!(s.dx > 0 && s.dy > 0 && s.dz > 0)) return fail("cell sizes must be positive");
  if (!(s.courant > 0 && s.courant <= 1.0)) return fail("courant number must be in (0, 1]");
  if (s.n_materials < 1 || s.n_materials > XFB_MAX_MATERIALS || s.materials == nullptr)
    return fail("need 1..255 materials (materials[0] is the background)");
  if (s.n_objects < 0 || (s.n_objects > 0 && s.objects == nullptr)) return fail("bad object list");
  for (int a = 0; a < 3; ++a)
    if (s.domain_cells[a] < 1) return fail("domain_cells must be >= 1");
  if (s.dim == 2 && s.domain_cells[2] != 1) return fail("2-D scenes need domain_cells[2] == 1");
  for (int f = 0; f < 6; ++f)
    if (s.pml.cells[f] < 0 || s.pml.cells[f] > 64) return fail("pml cells must be in [0, 64]");
  if (s.dim == 2 && (s.pml.cells[4] || s.pml.cells[5])) return fail("2-D scenes have no z CPML");

  c = Compiled{};
  c.dim = s.dim;
  c.prec = s.precision;
  c.dx = s.dx; c.dy = s.dy; c.dz = s.dz;
  for (int f = 0; f < 6; ++f) c.pml[f] = s.pml.cells[f];
  c.nx = s.domain_cells[0] + c.pml[0] + c.pml[1];
  c.ny = s.domain_cells[1] + c.pml[2] + c.pml[3];
  c.nz = s.domain_cells[2] + c.pml[4] + c.pml[5];
  if (c.nx < 2 || c.ny < 2 || (s.dim == 3 && c.nz < 2)) return fail("grid too small");
  if ((double)c.nx * c.ny * c.nz > 4.0e9) return fail("grid too large");
  const double inv2 = 1.0 / (s.dx * s.dx) + 1.0 / (s.dy * s.dy) + (s.dim == 3 ? 1.0 / (s.dz * s.dz) : 0.0);
  c.dt = s.courant / (c0() * std::sqrt(inv2));
  c.origin[0] = s.domain_min[0] - c.pml[0] * s.dx;
  c.origin[1] = s.domain_min[1] - c.pml[2] * s.dy;
  c.origin[2] = s.dim == 3 ? s.domain_min[2] - c.pml[4] * s.dz : 0.0;
  const double dt = c.dt;

  // ---- materials: Yee coefficients + ADE ---------------------------------
  c.n_mat = s.n_materials;
  c.coeff.assign(static_cast<size_t>(c.n_mat) * kCoeffs, 0.0);
  c.coeff8.assign(static_cast<size_t>(c.n_mat) * 8, 0.0);
  c.mat_disp.assign(c.n_mat, 0);
  c.mat_is_pec.assign(c.n_mat, 0);
  // ADE kind of the whole scene (the reference selects one updator for the
  // whole grid by the storage type: src/simulation/simulation_hd.cu:464-503).
  bool any_disp = false, all_debye = true, all_drude = true;
  int max_poles = 0;
  for (int m = 0; m < c.n_mat; ++m) {
    const xfb_material& mt = s.materials[m];
    if (mt.n_poles < 0 || mt.n_poles > XFB_MAX_POLES) return fail("material n_poles out of range");
    if (!(mt.eps_r > 0 && mt.mu_r > 0 && mt.sigma_e >= 0 && mt.sigma_m >= 0)) return fail("bad material constants");
    if (mt.n_poles > 0 && !mt.is_pec) {
      any_disp = true;
      max_poles = std::max(max_poles, mt.n_poles);
      for (int p = 0; p < mt.n_poles; ++p) {
        if (mt.poles[p].kind != XFB_POLE_DEBYE) all_debye = false;
        if (mt.poles[p].kind != XFB_POLE_DRUDE) all_drude = false;
      }
    }
  }
  c.ade_kind = !any_disp ? XFB_ADE_NONE : all_drude ? XFB_ADE_DRUDE : all_debye ? XFB_ADE_DEBYE : XFB_ADE_MLORENTZ;
  c.ade_poles = max_poles;
  c.ade_mat.assign(static_cast<size_t>(c.n_mat) * kAdeMat, 0.0);
  c.ade_pole.assign(static_cast<size_t>(c.n_mat) * std::max(1, max_poles) * kAdePole, 0.0);

  for (int m = 0; m < c.n_mat; ++m) {
    const xfb_material& mt = s.materials[m];
    double* k = &c.coeff[static_cast<size_t>(m) * kCoeffs];
    const double eps = kEps0 * mt.eps_r, mu = kMu0 * mt.mu_r;
    double ce, cbv;
    if (mt.is_pec) {
      ce = 0; cbv = 0;
      c.mat_is_pec[m] = 1;
    } else if (mt.n_poles == 0) {
      ce = (2 * eps - mt.sigma_e * dt) / (2 * eps + mt.sigma_e * dt);
      cbv = 2 * dt / (2 * eps + mt.sigma_e * dt);
    } else {
      // Ampere at n+1/2 with the polarisation current averaged in time:
      // eps0 eps_inf (E+ - E)/dt + sigma (E+ + E)/2 + sum_p (J_p+ + J_p)/2 = curl H
      double* am = &c.ade_mat[static_cast<size_t>(m) * kAdeMat];
      double sum_en = 0, sum_e = 0, sum_ep = 0;
      for (int p = 0; p < mt.n_poles; ++p) {
        double* q = &c.ade_pole[(static_cast<size_t>(m) * max_poles + p) * kAdePole];
        double cjj = 0, cjjp = 0, cjen = 0, cje = 0, cjep = 0;
        if (c.ade_kind == XFB_ADE_DRUDE) {
          // dJ/dt + gamma J = eps0 wp^2 E, trapezoidal (T&H 9.4.2):
          // J+ = kj J + bd (E+ + E)
          const double wp = mt.poles[p].p[0], g = mt.poles[p].p[1];
          cjj = (1 - g * dt / 2) / (1 + g * dt / 2);
          cje = (kEps0 * wp * wp * dt / 2) / (1 + g * dt / 2);
          cjen = cje;
          sum_en += cje;
          sum_e += cje;
        } else if (c.ade_kind == XFB_ADE_DEBYE) {
          // tau dJ/dt + J = eps0 d_eps dE/dt, trapezoidal (T&H 9.4.1):
          // J+ = kd J + bb (E+ - E)
          const double de = mt.poles[p].p[0], tau = mt.poles[p].p[1];
          if (!(tau > 0)) return fail("Debye tau must be > 0");
          cjj = (tau / dt - 0.5) / (tau / dt + 0.5);
          cje = (kEps0 * de / dt) / (tau / dt + 0.5);
          cjen = cje;
          sum_en += cje;
          sum_e -= cje;
        } else {
          // b2 J'' + b1 J' + b0 J = eps0 (a0 E' + a1 E''), centred at n
          // (T&H 9.4.3, eq. for Lorentz media, with a first-order numerator).
          double a[5];
          pole_to_mlorentz(mt.poles[p], a);
          const double A = a[4] + a[3] * dt / 2;
          if (!(std::fabs(A) > 0)) return fail("modified-Lorentz pole needs b2 + b1 dt/2 != 0");
          cjj = (2 * a[4] - a[2] * dt * dt) / A;
          cjjp = (a[3] * dt / 2 - a[4]) / A;
          cjen = kEps0 * (a[0] * dt / 2 + a[1]) / A;
          cje = -2 * kEps0 * a[1] / A;
          cjep = kEps0 * (a[1] - a[0] * dt / 2) / A;
          sum_en += cjen;
          sum_e += cje;
          sum_ep += cjep;
        }
        q[0] = cjj; q[1] = cjjp; q[2] = cjen; q[3] = cje; q[4] = cjep;
        q[5] = 1 + cjj;  // cjsj: weight of J^n in sum (J+ + J)
        q[6] = cjjp;     // cjsjp
        if (c.ade_kind != XFB_ADE_MLORENTZ) { q[1] = 0; q[4] = 0; q[6] = 0; }
      }
      const double epsinf = kEps0 * mt.eps_r;
      const double D = epsinf / dt + mt.sigma_e / 2 + sum_en / 2;
      ce = (epsinf / dt - mt.sigma_e / 2 - sum_e / 2) / D;
      cbv = 1 / D;
      am[0] = 1;                  // dispersive
      am[1] = -sum_ep / (2 * D);  // ceep
      am[2] = -1 / (2 * D);       // cejsum
    }
    // E_c = cece E_c + cecha (Ha_p - Ha_q) + cechb (Hb_p - Hb_q), with
    // (a, b) the cyclic tangential axes of c
    // (src/include/updator/update_scheme.cuh:27-32):
    k[CEXE] = ce; k[CEXHY] = -cbv / s.dz; k[CEXHZ] = cbv / s.dy;
    k[CEYE] = ce; k[CEYHZ] = -cbv / s.dx; k[CEYHX] = cbv / s.dz;
    k[CEZE] = ce; k[CEZHX] = -cbv / s.dy; k[CEZHY] = cbv / s.dx;
    // H_c = chch H_c + chcea (Ea_q - Ea_p) + chceb (Eb_q - Eb_p)
    // (update_scheme.cuh:59-63):
    const double ch = (2 * mu - mt.sigma_m * dt) / (2 * mu + mt.sigma_m * dt);
    const double db = 2 * dt / (2 * mu + mt.sigma_m * dt);
    k[CHXH] = ch; k[CHXEY] = db / s.dz; k[CHXEZ] = -db / s.dy;
    k[CHYH] = ch; k[CHYEZ] = db / s.dx; k[CHYEX] = -db / s.dz;
    k[CHZH] = ch; k[CHZEX] = db / s.dy; k[CHZEY] = -db / s.dx;
    double* k8 = &c.coeff8[static_cast<size_t>(m) * 8];
    k8[0] = ce; k8[1] = cbv / s.dx; k8[2] = cbv / s.dy; k8[3] = cbv / s.dz;
    k8[4] = ch; k8[5] = db / s.dx; k8[6] = db / s.dy; k8[7] = db / s.dz;
    c.mat_disp[m] = c.ade_mat[static_cast<size_t>(m) * kAdeMat] != 0 ? 1 : 0;
  }

  // ---- voxelisation: material of the last object holding the cell centre --
  const size_t ncell = static_cast<size_t>(c.nx) * c.ny * c.nz;
  c.mat_id.resize(ncell);  // zeroed plane by plane below (first touch spread over the threads)
  {
    const size_t plane = static_cast<size_t>(c.ny) * c.nz;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < c.nx; ++i) std::memset(c.mat_id.data() + i * plane, 0, plane);
  }
  // union of the cell boxes of the objects with a dispersive material: the
  // only cells that can hold one (unless material 0, the fill, is dispersive)
  int dlo[3] = {c.nx, c.ny, c.nz}, dhi[3] = {0, 0, 0};
  if (c.n_mat > 0 && c.mat_disp[0]) {
    dlo[0] = dlo[1] = dlo[2] = 0;
    dhi[0] = c.nx; dhi[1] = c.ny; dhi[2] = c.nz;
  }
  for (int o = 0; o < s.n_objects; ++o) {
    const xfb_object& ob = s.objects[o];
    if (ob.material < 0 || ob.material >= c.n_mat) return fail("object material index out of range");
    if (ob.shape < XFB_SHAPE_CUBE || ob.shape > XFB_SHAPE_CYLINDER) return fail("unknown shape");
    if (ob.shape == XFB_SHAPE_CYLINDER && (ob.p[4] < 0 || ob.p[4] > 2)) return fail("cylinder axis must be 0, 1 or 2");
    // bounding box in cell indices to keep big grids fast
    int lo[3] = {0, 0, 0}, hi[3] = {c.nx, c.ny, c.nz};
    const double d[3] = {s.dx, s.dy, s.dz};
    const int n[3] = {c.nx, c.ny, c.nz};
    if (ob.shape == XFB_SHAPE_SPHERE) {
      for (int a = 0; a < 3; ++a) {
        if (a == 2 && s.dim == 2) continue;
        lo[a] = std::max(0, static_cast<int>(std::floor((ob.p[a] - ob.p[3] - c.origin[a]) / d[a])) - 1);
        hi[a] = std::min(n[a], static_cast<int>(std::ceil((ob.p[a] + ob.p[3] - c.origin[a]) / d[a])) + 1);
      }
    }
    if (c.mat_disp[ob.material])
      for (int a = 0; a < 3; ++a) {
        dlo[a] = std::min(dlo[a], lo[a]);
        dhi[a] = std::max(dhi[a], hi[a]);
      }
    // planes are independent (each cell is written by one plane's thread)
#pragma omp parallel for schedule(static)
    for (int i = lo[0]; i < hi[0]; ++i) {
      const double x = c.origin[0] + (i + 0.5) * s.dx;
      for (int j = lo[1]; j < hi[1]; ++j) {
        const double y = c.origin[1] + (j + 0.5) * s.dy;
        for (int kk = lo[2]; kk < hi[2]; ++kk) {
          const double z = s.dim == 3 ? c.origin[2] + (kk + 0.5) * s.dz : 0.0;
          if (inside(ob, x, y, z)) c.mat_id[(static_cast<size_t>(i) * c.ny + j) * c.nz + kk] = static_cast<uint8_t>(ob.material);
        }
      }
    }
  }
  // ADE box: bounding box of cells holding a dispersive material.
  if (c.ade_kind != XFB_ADE_NONE) {
    int b0 = c.nx, b1 = 0, b2 = c.ny, b3 = 0, b4 = c.nz, b5 = 0;
#pragma omp parallel for schedule(static) reduction(min : b0, b2, b4) reduction(max : b1, b3, b5)
    for (int i = dlo[0]; i < dhi[0]; ++i)
      for (int j = dlo[1]; j < dhi[1]; ++j)
        for (int kk = dlo[2]; kk < dhi[2]; ++kk) {
          const int m = c.mat_id[(static_cast<size_t>(i) * c.ny + j) * c.nz + kk];
          if (c.ade_mat[static_cast<size_t>(m) * kAdeMat] != 0) {
            b0 = std::min(b0, i); b1 = std::max(b1, i + 1);
            b2 = std::min(b2, j); b3 = std::max(b3, j + 1);
            b4 = std::min(b4, kk); b5 = std::max(b5, kk + 1);
          }
        }
    int b[6] = {b0, b1, b2, b3, b4, b5};
    if (b[0] >= b[1]) {
      // dispersive materials exist but occupy no cell
      for (int q = 0; q < 6; ++q) b[q] = 0;
    }
    std::memcpy(c.ade_box, b, sizeof(b));
  }

  // ---- CPML profiles (per axis, E at nodes c, H at half nodes c+1/2) -----
  const double m_ord = s.pml.order_m > 0 ? s.pml.order_m : 3.0;
  const double s_ratio = s.pml.sigma_ratio > 0 ? s.pml.sigma_ratio : 1.0;
  const double a_max = s.pml.alpha_max >= 0 ? s.pml.alpha_max : 0.05;
  const double eta0 = std::sqrt(kMu0 / kEps0);
  const int nax[3] = {c.nx, c.ny, c.nz};
  const double dax[3] = {s.dx, s.dy, s.dz};
  for (int a = 0; a < 3; ++a) {
    const int n = nax[a], Ln = c.pml[2 * a], Lp = c.pml[2 * a + 1];
    if (Ln + Lp >= n) return fail("CPML layers leave no interior");
    const double smax = s_ratio * 0.8 * (m_ord + 1) / (eta0 * dax[a]);
    c.pml_ae[a].assign(n + 1, 0.0); c.pml_be[a].assign(n + 1, 0.0);
    c.pml_ah[a].assign(n, 0.0); c.pml_bh[a].assign(n, 0.0);
    auto prof = [&](double rho, double& av, double& bv) {
      const double sg = smax * std::pow(rho, m_ord);
      const double al = a_max * (1 - rho);
      bv = std::exp(-(sg + al) * dt / kEps0);
      av = (sg + al) > 0 ? sg / (sg + al) * (bv - 1) : 0.0;
    };
    for (int q = 0; q <= n; ++q) {
      double rho = -1;
      if (Ln > 0 && q < Ln) rho = double(Ln - q) / Ln;
      if (Lp > 0 && q >= n - Lp) rho = double(q - (n - Lp)) / Lp;
      if (rho >= 0) prof(rho, c.pml_ae[a][q], c.pml_be[a][q]);
    }
    for (int q = 0; q < n; ++q) {
      double rho = -1;
      if (Ln > 0 && q < Ln) rho = (Ln - q - 0.5) / Ln;
      if (Lp > 0 && q >= n - Lp) rho = (q + 0.5 - (n - Lp)) / Lp;
      if (rho >= 0) prof(rho, c.pml_ah[a][q], c.pml_bh[a][q]);
    }
  }

  // ---- TFSF ----------------------------------------------------------------
  if (s.tfsf.enabled) {
    const xfb_tfsf& t = s.tfsf;
    if (!(t.tau > 0)) return fail("TFSF waveform tau must be > 0");
    c.tfsf_on = 1;
    c.wave_kind = t.waveform;
    c.wave_tau = t.tau; c.wave_t0 = t.t0; c.wave_freq = t.freq;
    const int is = c.pml[0] + t.inset[0], ie = c.nx - c.pml[1] - t.inset[0];
    const int js = c.pml[2] + t.inset[1], je = c.ny - c.pml[3] - t.inset[1];
    int ks = 0, ke = 1;
    if (s.dim == 3) { ks = c.pml[4] + t.inset[2]; ke = c.nz - c.pml[5] - t.inset[2]; }
    if (is < 1 || js < 1 || ie >= c.nx || je >= c.ny || ie <= is || je <= js)
      return fail("TFSF box does not fit inside the grid");
    if (s.dim == 3 && (ks < 1 || ke >= c.nz || ke <= ks)) return fail("TFSF box does not fit inside the grid (z)");
    c.tf[0] = is; c.tf[1] = ie; c.tf[2] = js; c.tf[3] = je; c.tf[4] = ks; c.tf[5] = ke;
    double th = t.theta, ph = t.phi, ps = t.psi;
    if (s.dim == 2) th = kPi / 2;  // in-plane incidence for TMz
    double kv[3] = {std::sin(th) * std::cos(ph), std::sin(th) * std::sin(ph), std::cos(th)};
    for (double& v : kv)
      if (std::fabs(v) < 1e-6) v = 0;
    const double s4 = std::pow(std::sin(th), 4), c4p = std::pow(std::cos(ph), 4), s4p = std::pow(std::sin(ph), 4);
    const double ratio = 1.0 / std::sqrt(s4 * (c4p + s4p) + std::pow(std::cos(th), 4));
    const int start[3] = {kv[0] >= 0 ? is : ie, kv[1] >= 0 ? js : je, kv[2] >= 0 ? ks : ke};
    const int box0[3] = {is, js, ks};
    const int nbox[3] = {ie - is, je - js, ke - ks};
    for (int a = 0; a < 3; ++a) {
      const double inc = start[a] - 2 * kv[a] / ratio;
      c.proj_int[a].resize(nbox[a] + 1);
      c.proj_half[a].resize(nbox[a] + 2);
      for (int q = 0; q <= nbox[a]; ++q) c.proj_int[a][q] = (q + box0[a] - inc) * kv[a] * ratio;
      for (int q = 0; q <= nbox[a] + 1; ++q) c.proj_half[a][q] = (q + box0[a] - inc - 0.5) * kv[a] * ratio;
    }
    const double diag = std::sqrt(double(nbox[0]) * nbox[0] + double(nbox[1]) * nbox[1] + double(nbox[2]) * nbox[2]);
    c.aux_nl = static_cast<int>(std::ceil(ratio * diag)) + 4 + 1;
    c.aux_dl = s.dx / ratio;
    c.aux_ceih = -dt / (kEps0 * c.aux_dl);
    c.aux_chie = -dt / (kMu0 * c.aux_dl);
    c.aux_abc = (c0() * dt - c.aux_dl) / (c0() * dt + c.aux_dl);
    // polarisation (theta-hat / phi-hat basis, test/2d.cu:910-921) and H = k x E
    const double ct = std::cos(th), st = std::sin(th), cp = std::cos(ph), sp = std::sin(ph);
    const double cs = std::cos(ps), ss = std::sin(ps);
    c.tr_e[0] = ss * (-sp) + cs * (cp * ct);
    c.tr_e[1] = ss * cp + cs * (sp * ct);
    c.tr_e[2] = cs * (-st);
    c.tr_h[0] = kv[1] * c.tr_e[2] - kv[2] * c.tr_e[1];
    c.tr_h[1] = kv[2] * c.tr_e[0] - kv[0] * c.tr_e[2];
    c.tr_h[2] = kv[0] * c.tr_e[1] - kv[1] * c.tr_e[0];
    for (int a = 0; a < 3; ++a) {
      c.ca[a] = dt / (kEps0 * dax[a]);
      c.cb[a] = dt / (kMu0 * dax[a]);
    }
    // every interpolation stencil must stay inside the auxiliary grid
    // (sum over axes of the per-axis extremes bounds every stencil)
    double pmin = 0, pmax = 0;
    for (int a = 0; a < 3; ++a) {
      double lo = 1e300, hi = -1e300;
      for (double v : c.proj_int[a]) { lo = std::min(lo, v); hi = std::max(hi, v); }
      for (double v : c.proj_half[a]) { lo = std::min(lo, v); hi = std::max(hi, v); }
      pmin += lo;
      pmax += hi;
    }
    if (pmin - 0.5 < -1e-9 || pmax + 1 > c.aux_nl - 1) return fail("TFSF auxiliary grid does not cover the box (internal)");
  }

  // ---- NF2FF ---------------------------------------------------------------
  if (s.nf2ff.enabled) {
    if (s.dim != 3) return fail("NF2FF is supported on 3-D scenes");
    if (s.nf2ff.n_freqs < 1 || s.nf2ff.freqs == nullptr) return fail("NF2FF needs at least one frequency");
    c.nf_on = 1;
    const xfb_nf2ff& n = s.nf2ff;
    c.nf[0] = c.pml[0] + n.inset[0]; c.nf[1] = c.nx - c.pml[1] - n.inset[0];
    c.nf[2] = c.pml[2] + n.inset[1]; c.nf[3] = c.ny - c.pml[3] - n.inset[1];
    c.nf[4] = c.pml[4] + n.inset[2]; c.nf[5] = c.nz - c.pml[5] - n.inset[2];
    for (int a = 0; a < 3; ++a)
      if (c.nf[2 * a] < 1 || c.nf[2 * a + 1] >= nax[a] || c.nf[2 * a + 1] <= c.nf[2 * a])
        return fail("NF2FF box does not fit inside the grid");
    c.freqs.assign(n.freqs, n.freqs + n.n_freqs);
  }
  if (s.nf2ff_td.enabled) {
    if (s.dim != 3) return fail("time-domain NF2FF is supported on 3-D scenes");
    const xfb_nf2ff_td& n = s.nf2ff_td;
    if (!std::isfinite(n.theta) || !std::isfinite(n.phi)) return fail("time-domain NF2FF direction must be finite");
    c.td_on = 1;
    c.td[0] = c.pml[0] + n.inset[0]; c.td[1] = c.nx - c.pml[1] - n.inset[0];
    c.td[2] = c.pml[2] + n.inset[1]; c.td[3] = c.ny - c.pml[3] - n.inset[1];
    c.td[4] = c.pml[4] + n.inset[2]; c.td[5] = c.nz - c.pml[5] - n.inset[2];
    for (int a = 0; a < 3; ++a)
      if (c.td[2 * a] < 1 || c.td[2 * a + 1] >= nax[a] || c.td[2 * a + 1] <= c.td[2 * a])
        return fail("time-domain NF2FF box does not fit inside the grid");
    compile_td(c, n.theta, n.phi);
  }

  // ---- monitors ------------------------------------------------------------
  auto comp_shape = [&](int f, int shp[3]) {
    shp[0] = c.nx + (f == XFB_EY || f == XFB_EZ || f == XFB_HX ? 1 : 0);
    shp[1] = c.ny + (f == XFB_EX || f == XFB_EZ || f == XFB_HY ? 1 : 0);
    shp[2] = c.nz + (f == XFB_EX || f == XFB_EY || f == XFB_HZ ? 1 : 0);
    if (c.dim == 2) shp[2] = 1;
  };
  for (int p = 0; p < s.n_probes; ++p) {
    const xfb_probe& pr = s.probes[p];
    if (pr.field < 0 || pr.field > 5) return fail("probe field out of range");
    if (c.dim == 2 && !(pr.field == XFB_EZ || pr.field == XFB_HX || pr.field == XFB_HY))
      return fail("2-D probes must watch Ez, Hx or Hy");
    int shp[3];
    comp_shape(pr.field, shp);
    for (int a = 0; a < 3; ++a)
      if (pr.index[a] < 0 || pr.index[a] >= shp[a]) return fail("probe index outside the component");
    c.probes.push_back(pr);
  }
  for (int m = 0; m < s.n_movies; ++m) {
    const xfb_movie& mv = s.movies[m];
    if (mv.field < 0 || mv.field > 5) return fail("movie field out of range");
    if (c.dim == 2 && !(mv.field == XFB_EZ || mv.field == XFB_HX || mv.field == XFB_HY))
      return fail("2-D movies must watch Ez, Hx or Hy");
    if (mv.interval < 1) return fail("movie interval must be >= 1");
    int shp[3];
    comp_shape(mv.field, shp);
    for (int a = 0; a < 3; ++a)
      if (mv.lo[a] < 0 || mv.hi[a] > shp[a] || mv.hi[a] <= mv.lo[a]) return fail("movie box outside the component");
    c.movies.push_back(mv);
  }
  return XFB_OK;
}

}  // namespace xfb
