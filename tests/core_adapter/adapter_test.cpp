// The XFDTD_CORE adapter (include/xfdtd_b200/xfdtd_core_adapter.hpp) run
// against the stand-in accessor surface in fake/: a 10x9x8 scene with a Drude
// block, x CPML whose c_psi is the curl coefficient times dx, a TFSF box, a
// frequency- and a time-domain NF2FF box and an Ez movie.  The packed arrays
// go through xfb_create_from_arrays (host only, no device) and the compiled
// scene is checked entry by entry.  Prints "ok" and exits 0 on success.
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>

#include "xfdtd_b200/xfdtd_core_adapter.hpp"

using namespace xfdtd;

#define CHECK(c)                                                    \
  do {                                                              \
    if (!(c)) {                                                     \
      std::fprintf(stderr, "%s:%d: check failed: %s\n", __FILE__, __LINE__, #c); \
      std::exit(1);                                                 \
    }                                                               \
  } while (0)

static bool near(double a, double b, double rel = 1e-12) { return std::fabs(a - b) <= rel * std::fabs(b) + 1e-300; }

static const int NX = 10, NY = 9, NZ = 8;
static const double DL = 1e-3, DT = 1e-12;

struct Mat {
  double ce, bx, by, bz, ch, dx, dy, dz;
  // cexe cexhy cexhz ceye ceyhz ceyhx ceze cezhx cezhy chxh chxey chxez chyh chyez chyex chzh chzex chzey
  void fill(double k[18]) const {
    const double v[18] = {ce, -bz, by, ce, -bx, bz, ce, -by, bx, ch, dz, -dy, ch, dx, -dz, ch, dy, -dx};
    std::memcpy(k, v, sizeof(v));
  }
};
static const Mat kVac{1.0, 0.51, 0.52, 0.53, 1.0, 0.31, 0.32, 0.33};
static const Mat kBlock{0.9, 0.25, 0.26, 0.27, 1.0, 0.31, 0.32, 0.33};

static bool in_block(int i, int j, int k) { return i >= 4 && i < 6 && j >= 3 && j < 6 && k >= 3 && k < 5; }

static IndexTask task(int x0, int x1, int y0, int y1, int z0, int z1) {
  IndexTask t;
  t.x = {std::size_t(x0), std::size_t(x1)};
  t.y = {std::size_t(y0), std::size_t(y1)};
  t.z = {std::size_t(z0), std::size_t(z1)};
  return t;
}

// curl coefficient index (0..17) of field f from dual field d
static int curl_index(int f, int d) { return 3 * f + ((d % 3) == (f % 3 + 1) % 3 ? 1 : 2); }

static std::shared_ptr<PML> make_pml(const Simulation& sim, bool high) {
  auto p = std::make_shared<PML>();
  p->axis = Axis::XYZ::X;
  const int L = 2;
  p->t = high ? task(NX - L, NX, 0, NY, 0, NZ) : task(0, L, 0, NY, 0, NZ);
  p->e_start = high ? NX - L : 0;
  p->h_start = high ? NX - L : 0;
  p->ae = Array<double>({3}, 0.0);
  p->be = Array<double>({3}, 0.0);
  p->ah = Array<double>({2}, 0.0);
  p->bh = Array<double>({2}, 0.0);
  for (int q = 0; q < 3; ++q) {
    p->ae(q) = (high ? 0.04 : 0.02) + 0.001 * q;
    p->be(q) = 0.9 + 0.01 * q;
  }
  for (int q = 0; q < 2; ++q) {
    p->ah(q) = (high ? 0.05 : 0.03) + 0.001 * q;
    p->bh(q) = 0.8 + 0.01 * q;
  }
  const auto& cf = *sim.param->coeff;
  // c_psi = curl coefficient * dx over the layer: Ey<-Hz, Ez<-Hy, Hy<-Ez, Hz<-Ey
  const struct { Array<double>* dst; int f, d; } layers[4] = {
      {&p->c_ea, XFB_EY, XFB_HZ}, {&p->c_eb, XFB_EZ, XFB_HY}, {&p->c_ha, XFB_HY, XFB_EZ}, {&p->c_hb, XFB_HZ, XFB_EY}};
  for (const auto& l : layers) {
    const std::size_t ext = l.f < 3 ? 3 : 2;
    *l.dst = Array<double>({ext, NY + 1, NZ + 1}, 0.0);
    const auto& c = cf.c[curl_index(l.f, l.d)];
    for (std::size_t q = 0; q < ext; ++q)
      for (int j = 0; j <= NY; ++j)
        for (int k = 0; k <= NZ; ++k) {
          const std::size_t i = q + p->e_start;
          if (i > NX) continue;
          (*l.dst)(q, j, k) = c.v[(i * (NY + 1) + j) * (NZ + 1) + k] * DL;
        }
  }
  return p;
}

static void build(Simulation& sim) {
  auto& g = *sim.grid;
  g.n[0] = NX; g.n[1] = NY; g.n[2] = NZ;
  const int n[3] = {NX, NY, NZ};
  for (int ax = 0; ax < 3; ++ax) {
    g.e[ax] = Array<double>({std::size_t(n[ax] + 1)}, 0.0);
    for (int q = 0; q <= n[ax]; ++q) g.e[ax](q) = -5e-3 + q * DL;
  }
  sim.param->time->step = DT;
  auto& cf = *sim.param->coeff;
  for (int q = 0; q < 18; ++q) cf.c[q] = Array<double>({NX + 1, NY + 1, NZ + 1}, 0.0);
  for (int i = 0; i <= NX; ++i)
    for (int j = 0; j <= NY; ++j)
      for (int k = 0; k <= NZ; ++k) {
        double v[18];
        (in_block(i, j, k) ? kBlock : kVac).fill(v);
        for (int q = 0; q < 18; ++q) cf.c[q](i, j, k) = v[q];
      }
  auto ade = std::make_shared<DrudeADEMethodStorage>();
  for (int q = 0; q < 7; ++q) ade->pole[q] = Array<double>({NX, NY, NZ, 1}, 0.0);
  ade->eep = Array<double>({NX, NY, NZ}, 0.0);
  ade->ejs = Array<double>({NX, NY, NZ}, 0.0);
  for (int i = 0; i < NX; ++i)
    for (int j = 0; j < NY; ++j)
      for (int k = 0; k < NZ; ++k)
        if (in_block(i, j, k)) {
          ade->pole[0](i, j, k, 0) = 0.7;
          ade->pole[3](i, j, k, 0) = 0.1;
          ade->pole[5](i, j, k, 0) = 0.2;
          ade->ejs(i, j, k) = 0.05;
        }
  sim.ade = ade;
  sim.bounds.push_back(make_pml(sim, false));
  sim.bounds.push_back(make_pml(sim, true));

  auto tf = std::make_shared<TFSF>();
  tf->box = task(3, 7, 2, 6, 2, 6);
  const int nb[3] = {4, 4, 4};
  for (int ax = 0; ax < 3; ++ax) {
    tf->pi[ax] = Array<double>({std::size_t(nb[ax] + 1)}, 0.0);
    tf->ph[ax] = Array<double>({std::size_t(nb[ax] + 2)}, 0.0);
    for (int q = 0; q <= nb[ax]; ++q) tf->pi[ax](q) = 1.0 + 0.3 * q + 0.01 * ax;
    for (int q = 0; q <= nb[ax] + 1; ++q) tf->ph[ax](q) = 0.85 + 0.3 * q + 0.01 * ax;
  }
  tf->e_inc = Array<double>({12, 20}, 0.0);
  tf->h_inc = Array<double>({12, 19}, 0.0);
  for (int t = 0; t < 12; ++t) {
    for (int q = 0; q < 20; ++q) tf->e_inc(t, q) = std::sin(0.1 * t + 0.2 * q);
    for (int q = 0; q < 19; ++q) tf->h_inc(t, q) = std::cos(0.1 * t + 0.2 * q);
  }
  tf->te = {0.1, -0.2, 0.97};
  tf->th = {0.3, 0.9, 0.1};
  for (int ax = 0; ax < 3; ++ax) {
    tf->ca[ax] = 0.4 + 0.1 * ax;
    tf->cb[ax] = 0.7 + 0.1 * ax;
  }
  sim.sources.push_back(tf);

  auto fd = std::make_shared<NFFFTFrequencyDomain>();
  const int fb[6] = {2, 8, 2, 7, 2, 6};
  auto faces = [&](NFFFT& nf, const int b[6]) {
    nf.face[0] = task(b[0], b[0] + 1, b[2], b[3], b[4], b[5]);
    nf.face[1] = task(b[1], b[1] + 1, b[2], b[3], b[4], b[5]);
    nf.face[2] = task(b[0], b[1], b[2], b[2] + 1, b[4], b[5]);
    nf.face[3] = task(b[0], b[1], b[3], b[3] + 1, b[4], b[5]);
    nf.face[4] = task(b[0], b[1], b[2], b[3], b[4], b[4] + 1);
    nf.face[5] = task(b[0], b[1], b[2], b[3], b[5], b[5] + 1);
  };
  faces(*fd, fb);
  for (double f : {3e9, 7.5e9}) {
    Array<std::complex<double>> tr({12}, {0, 0});
    for (int t = 0; t < 12; ++t) tr(t) = DT * std::exp(std::complex<double>(0, -2 * M_PI * f * (t + 0.5) * DT));
    fd->te.push_back(tr);
  }
  sim.nf.push_back(fd);
  auto td = std::make_shared<NFFFTTimeDomain>();
  const int tb[6] = {3, 7, 3, 6, 3, 5};
  faces(*td, tb);
  td->dir = {2 * std::sin(0.7) * std::cos(1.9), 2 * std::sin(0.7) * std::sin(1.9), 2 * std::cos(0.7)};
  sim.nf.push_back(td);

  auto fm = std::make_shared<FieldMonitor>();
  fm->f = EMF::Field::EZ;
  fm->t = task(1, 9, 2, 7, 4, 5);
  auto mv = std::make_shared<MovieMonitor>();
  mv->fr = fm;
  mv->interval = 3;
  sim.mons.push_back(mv);
}

int main() {
  Simulation sim;
  build(sim);
  xfb_core::CoreScene cs(sim, 12, XFB_FP64);
  CHECK(sim.inited == 12);
  const xfb_core_arrays& a = cs.arrays();
  CHECK(a.nx == NX && a.ny == NY && a.nz == NZ && near(a.dx, DL) && a.dt == DT);
  CHECK(near(a.origin[0], -5e-3) && a.n_movies == 1);
  CHECK(a.movies[0].field == XFB_EZ && a.movies[0].lo[0] == 1 && a.movies[0].hi[1] == 7 && a.movies[0].interval == 3);
  CHECK(a.inc_steps == 12 && a.aux_nl == 19);

  xfb_handle* h = cs.create();
  xfb_compiled_view v;
  CHECK(xfb_compiled_view_get(h, &v) == XFB_OK);
  CHECK(v.nx == NX && v.ny == NY && v.nz == NZ && v.n_materials == 2);
  const int mv = v.material_id[0], mb = v.material_id[(4 * NY + 3) * NZ + 3];
  CHECK(mv != mb);
  double kv[18], kb[18];
  kVac.fill(kv);
  kBlock.fill(kb);
  for (int q = 0; q < 18; ++q) CHECK(v.coeff[mv * 18 + q] == kv[q] && v.coeff[mb * 18 + q] == kb[q]);
  for (int i = 0; i < NX; ++i)
    for (int j = 0; j < NY; ++j)
      for (int k = 0; k < NZ; ++k) CHECK(v.material_id[(i * NY + j) * NZ + k] == (in_block(i, j, k) ? mb : mv));
  CHECK(v.ade_kind == XFB_ADE_DRUDE && v.ade_poles == 1);
  CHECK(v.ade_mat[mb * 3 + 0] == 1.0 && v.ade_mat[mb * 3 + 2] == 0.05 && v.ade_mat[mv * 3 + 0] == 0.0);
  CHECK(v.ade_pole[mb * 7 + 0] == 0.7 && v.ade_pole[mb * 7 + 3] == 0.1 && v.ade_pole[mb * 7 + 5] == 0.2);

  CHECK(v.pml_cells[0] == 2 && v.pml_cells[1] == 2 && v.pml_cells[2] == 0);
  for (int q = 0; q < 3; ++q) {
    CHECK(near(v.pml_ae[0][q], (0.02 + 0.001 * q) * DL, 1e-14));
    CHECK(near(v.pml_ae[0][NX - 2 + q], (0.04 + 0.001 * q) * DL, 1e-14));
    CHECK(v.pml_be[0][NX - 2 + q] == 0.9 + 0.01 * q);
  }
  for (int q = 0; q < 2; ++q) {
    CHECK(near(v.pml_ah[0][q], (0.03 + 0.001 * q) * DL, 1e-14));
    CHECK(near(v.pml_ah[0][NX - 2 + q], (0.05 + 0.001 * q) * DL, 1e-14));
    CHECK(v.pml_bh[0][q] == 0.8 + 0.01 * q);
  }
  CHECK(v.pml_ae[0][4] == 0 && v.pml_be[0][4] == 0 && v.pml_ah[0][5] == 0);

  CHECK(v.tfsf_enabled && v.tfsf_box[0] == 3 && v.tfsf_box[1] == 7 && v.tfsf_box[3] == 6);
  CHECK(v.tfsf_proj_int[1][2] == 1.0 + 0.3 * 2 + 0.01 && v.tfsf_proj_half[2][5] == 0.85 + 0.3 * 5 + 0.02);
  CHECK(v.tfsf_transform_e[2] == 0.97 && v.tfsf_transform_h[1] == 0.9 && v.tfsf_ca[1] == 0.4 + 0.1 && v.tfsf_cb[2] == 0.7 + 0.1 * 2);
  CHECK(v.aux_nl == 19);

  CHECK(v.nf2ff_enabled && v.nf2ff_box[0] == 2 && v.nf2ff_box[1] == 8 && v.nf2ff_box[3] == 7 && v.nf2ff_box[5] == 6);
  CHECK(v.n_freqs == 2 && near(v.freqs[0], 3e9, 1e-9) && near(v.freqs[1], 7.5e9, 1e-9));
  CHECK(v.nf2ff_td_enabled && v.nf2ff_td_box[0] == 3 && v.nf2ff_td_box[1] == 7 && v.nf2ff_td_box[5] == 5);
  CHECK(near(v.nf2ff_td_theta, 0.7, 1e-12) && near(v.nf2ff_td_phi, 1.9, 1e-12));
  xfb_destroy(h);

  // c_psi that is not one multiple of the curl coefficient is refused
  {
    Simulation bad;
    build(bad);
    auto* p = dynamic_cast<PML*>(bad.bounds[0].get());
    p->c_ea(1, 2, 2) *= 1.5;
    bool threw = false;
    try {
      xfb_core::CoreScene c2(bad, 12);
    } catch (const std::runtime_error& e) {
      threw = std::strstr(e.what(), "multiple") != nullptr;
    }
    CHECK(threw);
  }
  // a coefficient set that is not of the isotropic form is refused by the library
  {
    Simulation bad;
    build(bad);
    bad.param->coeff->c[1](0, 0, 0) *= 2;  // cexhy of cell 0 no longer -ceyhx
    xfb_core::CoreScene c3(bad, 12);
    bool threw = false;
    try {
      xfb_destroy(c3.create());
    } catch (const std::runtime_error& e) {
      threw = std::strstr(e.what(), "isotropic") != nullptr;
    }
    CHECK(threw);
  }
  std::puts("ok");
  return 0;
}
