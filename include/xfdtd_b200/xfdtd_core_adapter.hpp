// XFDTD_CORE -> xfb_core_arrays: the drop-in for SimulationHD's host side.
//
// The reference's SimulationHD (src/simulation/simulation_hd.cu:105-267) calls
// host()->init(steps) and then wraps XFDTD_CORE's host arrays one by one for
// the device:
//   FDTDCoefficientHD  cexe() ... chzey()          calculation_param/fdtd_coefficient_hd.cu:9-51
//   PMLCorrectorHD     task(), global{E,H}NodeStartIndexMainAxis(),
//                      coeff{AE,BE,AH,BH}(), coeff{EAPsiHB,EBPsiHA,HAPsiEB,HBPsiEA}()
//                                                  boundary/pml_corrector_hd.cu:8-34
//   TFSFCorrectorHD    projection{X,Y,Z}{Int,Half}(), eInc(), hInc(), globalTask(),
//                      ca{x,y,z}(), cb{x,y,z}(), transformE(), transformH()
//                                                  waveform_source/tfsf/tfsf_corrector_hd.cu:9-73
//   ADEMethodStorageHD coeffJJ() ... coeffEEPrev() material/ade_method/ade_method_hd.cu:5-24
//   NF2FF FD / TD      globalTaskSurface{XN..ZP}(), freqCount(), transformE(i);
//                      nodeTaskSurface{XN..ZP}(), observationDirection()
//                                                  nf2ff/frequency_domain/nf2ff_frequency_domain_hd.cu:137-178,
//                                                  nf2ff/time_domain/nf2ff_time_domain_hd.cu:43,129-146
//   MovieMonitorHD     frame() -> FieldMonitor field(), globalTask(); frameInterval()
//                                                  include/monitor/movie_monitor_hd.cuh:30-45
// CoreScene reads the same accessors once and packs them into the plain
// arrays of xfb_core_arrays; xfb_create_from_arrays compresses the per-cell
// coefficients into the engine's material table.  Only the element
// accessors shape(), size() and data() of XFDTD_CORE's arrays are used, so
// single- and double-precision builds of XFDTD_CORE both work (values are
// widened to double).
//
// The CPML correction of XFDTD_CORE multiplies psi by its own per-cell
// coefficient c_psi; the engine multiplies by the cell's curl coefficient.
// CoreScene measures c_psi / curl over each layer (it must be one constant r
// per layer and field kind, else std::runtime_error) and scales that layer's
// a-profile by r: identical arithmetic when r == 1, equal up to rounding
// otherwise.  The NF2FF frequencies are read back from the phase advance of
// transformE(i) between steps 0 and 1.
//
// Compiled only where XFDTD_CORE's headers are on the include path.
#ifndef XFDTD_B200_XFDTD_CORE_ADAPTER_HPP_
#define XFDTD_B200_XFDTD_CORE_ADAPTER_HPP_

#include "../xfdtd_b200.h"

#if __has_include(<xfdtd/simulation/simulation.h>)

#include <xfdtd/boundary/pml.h>
#include <xfdtd/calculation_param/calculation_param.h>
#include <xfdtd/grid_space/grid_space.h>
#include <xfdtd/material/ade_method/debye_ade_method.h>
#include <xfdtd/material/ade_method/drude_ade_method.h>
#include <xfdtd/material/ade_method/m_lor_ade_method.h>
#include <xfdtd/monitor/field_monitor.h>
#include <xfdtd/monitor/movie_monitor.h>
#include <xfdtd/nffft/nffft_frequency_domain.h>
#include <xfdtd/nffft/nffft_time_domain.h>
#include <xfdtd/simulation/simulation.h>
#include <xfdtd/waveform_source/tfsf.h>

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstddef>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace xfb_core {

class CoreScene {
 public:
  // Calls sim.init(steps) (what SimulationHD::init does) and packs the scene.
  CoreScene(xfdtd::Simulation& sim, long long steps, int precision = XFB_FP64) {
    sim.init(steps);
    a_ = xfb_core_arrays{};
    a_.precision = precision;
    grid(sim);
    coefficients(sim);
    ade(sim);
    pml(sim);
    tfsf(sim);
    nf2ff(sim);
    movies(sim);
  }

  CoreScene(const CoreScene&) = delete;
  CoreScene& operator=(const CoreScene&) = delete;

  const xfb_core_arrays& arrays() const { return a_; }

  // A device handle of the scene; throws with the library's message on failure.
  xfb_handle* create() const {
    xfb_handle* h = nullptr;
    const int st = xfb_create_from_arrays(&a_, &h);
    if (st != XFB_OK) throw std::runtime_error(std::string("xfb_create_from_arrays: ") + xfb_last_error(nullptr));
    return h;
  }

 private:
  xfb_core_arrays a_;
  std::vector<std::vector<double>> store_;  // every array a_ points into
  std::vector<xfb_movie> movies_;

  double* keep(std::vector<double> v) {
    store_.push_back(std::move(v));
    return store_.back().data();
  }

  // element (i, j, k[, p]) of a row-major XFDTD_CORE array, as double
  template <typename Arr>
  static double at(const Arr& arr, std::size_t i, std::size_t j, std::size_t k) {
    const auto& s = arr.shape();
    return static_cast<double>(arr.data()[(i * s[1] + j) * s[2] + k]);
  }

  template <typename Arr>
  static std::vector<double> flat(const Arr& arr) {
    std::vector<double> v(arr.size());
    for (std::size_t q = 0; q < v.size(); ++q) v[q] = static_cast<double>(arr.data()[q]);
    return v;
  }

  template <typename Arr>
  static void need_shape(const Arr& arr, std::size_t s0, std::size_t s1, std::size_t s2, const char* what) {
    const auto& s = arr.shape();
    if (arr.dimension() < 3 || s[0] < s0 || s[1] < s1 || s[2] < s2)
      throw std::runtime_error(std::string("XFDTD_CORE array too small: ") + what);
  }

  void field_shape(int f, int s[3]) const {
    s[0] = a_.nx + (f == XFB_EY || f == XFB_EZ || f == XFB_HX ? 1 : 0);
    s[1] = a_.ny + (f == XFB_EX || f == XFB_EZ || f == XFB_HY ? 1 : 0);
    s[2] = a_.nz + (f == XFB_EX || f == XFB_EY || f == XFB_HZ ? 1 : 0);
  }

  static int axis_index(xfdtd::Axis::XYZ x) {
    return x == xfdtd::Axis::XYZ::X ? 0 : x == xfdtd::Axis::XYZ::Y ? 1 : 2;
  }

  template <typename Task>
  static void box_of(const Task& t, int b[6]) {
    b[0] = static_cast<int>(t.xRange().start());
    b[1] = static_cast<int>(t.xRange().end());
    b[2] = static_cast<int>(t.yRange().start());
    b[3] = static_cast<int>(t.yRange().end());
    b[4] = static_cast<int>(t.zRange().start());
    b[5] = static_cast<int>(t.zRange().end());
  }

  void grid(xfdtd::Simulation& sim) {
    const auto gs = sim.gridSpace();
    if (gs->dimension() != xfdtd::GridSpace::Dimension::THREE)
      throw std::runtime_error("xfb_create_from_arrays takes 3-D scenes");
    a_.nx = static_cast<int>(gs->sizeX());
    a_.ny = static_cast<int>(gs->sizeY());
    a_.nz = static_cast<int>(gs->sizeZ());
    const auto* nodes_x = &gs->eNodeX();
    const auto* nodes_y = &gs->eNodeY();
    const auto* nodes_z = &gs->eNodeZ();
    double d[3];
    const decltype(nodes_x) nodes[3] = {nodes_x, nodes_y, nodes_z};
    for (int ax = 0; ax < 3; ++ax) {
      const auto& e = *nodes[ax];
      if (e.size() < 2) throw std::runtime_error("grid axis without cells");
      d[ax] = static_cast<double>(e.data()[1]) - static_cast<double>(e.data()[0]);
      for (std::size_t q = 1; q < e.size(); ++q) {
        const double dq = static_cast<double>(e.data()[q]) - static_cast<double>(e.data()[q - 1]);
        if (std::fabs(dq - d[ax]) > 1e-9 * std::fabs(d[ax])) throw std::runtime_error("the engine needs a uniform grid");
      }
      a_.origin[ax] = static_cast<double>(e.data()[0]);
    }
    a_.dx = d[0];
    a_.dy = d[1];
    a_.dz = d[2];
    a_.dt = static_cast<double>(sim.calculationParam()->timeParam()->dt());
  }

  void coefficients(xfdtd::Simulation& sim) {
    const auto cf = sim.calculationParam()->fdtdCoefficient();
    // xfb order: cexe cexhy cexhz ceye ceyhz ceyhx ceze cezhx cezhy
    //            chxh chxey chxez chyh chyez chyex chzh chzex chzey
    const decltype(&cf->cexe()) src[18] = {
        &cf->cexe(), &cf->cexhy(), &cf->cexhz(), &cf->ceye(), &cf->ceyhz(), &cf->ceyhx(),
        &cf->ceze(), &cf->cezhx(), &cf->cezhy(), &cf->chxh(), &cf->chxey(), &cf->chxez(),
        &cf->chyh(), &cf->chyez(), &cf->chyex(), &cf->chzh(), &cf->chzex(), &cf->chzey()};
    for (int q = 0; q < 18; ++q) {
      const auto& s = *src[q];
      int shp[3];
      field_shape(q / 3, shp);
      need_shape(s, a_.nx, a_.ny, a_.nz, "coefficient");
      std::vector<double> v(static_cast<std::size_t>(shp[0]) * shp[1] * shp[2], 0.0);
      for (int i = 0; i < a_.nx; ++i)
        for (int j = 0; j < a_.ny; ++j)
          for (int k = 0; k < a_.nz; ++k)
            v[(static_cast<std::size_t>(i) * shp[1] + j) * shp[2] + k] = at(s, i, j, k);
      a_.coeff[q] = keep(std::move(v));
    }
  }

  void ade(xfdtd::Simulation& sim) {
    const auto st = sim.aDEMethodStorage();
    if (st == nullptr) return;
    if (std::dynamic_pointer_cast<xfdtd::DrudeADEMethodStorage>(st)) a_.ade_kind = XFB_ADE_DRUDE;
    else if (std::dynamic_pointer_cast<xfdtd::DebyeADEMethodStorage>(st)) a_.ade_kind = XFB_ADE_DEBYE;
    else if (std::dynamic_pointer_cast<xfdtd::MLorentzADEMethodStorage>(st)) a_.ade_kind = XFB_ADE_MLORENTZ;
    else throw std::runtime_error("unknown ADE storage");
    const auto& cjj = st->coeffJJ();
    if (cjj.dimension() != 4) throw std::runtime_error("ADE pole coefficients must be (x, y, z, pole)");
    const int P = static_cast<int>(cjj.shape()[3]);
    a_.ade_poles = P;
    const std::size_t cells = static_cast<std::size_t>(a_.nx) * a_.ny * a_.nz;
    const decltype(&st->coeffJJ()) poles[7] = {&st->coeffJJ(), &st->coeffJJPrev(), &st->coeffJENext(),
                                               &st->coeffJE(), &st->coeffJEPrev(), &st->coeffJSumJ(),
                                               &st->coeffJSumJPrev()};
    std::vector<double> flag(cells, 0.0), ceep(cells), cejsum(cells);
    std::vector<std::vector<double>> pv(7, std::vector<double>(cells * P));
    const auto& eep = st->coeffEEPrev();
    const auto& ejs = st->coeffEJSum();
    need_shape(eep, a_.nx, a_.ny, a_.nz, "coeffEEPrev");
    need_shape(ejs, a_.nx, a_.ny, a_.nz, "coeffEJSum");
    for (int i = 0; i < a_.nx; ++i)
      for (int j = 0; j < a_.ny; ++j)
        for (int k = 0; k < a_.nz; ++k) {
          const std::size_t c = (static_cast<std::size_t>(i) * a_.ny + j) * a_.nz + k;
          ceep[c] = at(eep, i, j, k);
          cejsum[c] = at(ejs, i, j, k);
          bool any = ceep[c] != 0 || cejsum[c] != 0;
          for (int q = 0; q < 7; ++q) {
            const auto& s = *poles[q];
            const auto& sh = s.shape();
            for (int p = 0; p < P; ++p) {
              const double v = static_cast<double>(s.data()[((i * sh[1] + j) * sh[2] + k) * sh[3] + p]);
              pv[q][c * P + p] = v;
              any = any || v != 0;
            }
          }
          flag[c] = any ? 1.0 : 0.0;  // the reference updates every cell; zero sets reduce to the plain update
        }
    a_.ade_cell[0] = keep(std::move(flag));
    a_.ade_cell[1] = keep(std::move(ceep));
    a_.ade_cell[2] = keep(std::move(cejsum));
    for (int q = 0; q < 7; ++q) a_.ade_pole[q] = keep(std::move(pv[q]));
  }

  // c_psi / curl coefficient over a layer: one constant, or throw
  template <typename Arr>
  double psi_ratio(const Arr& cpsi, int field, int dual, int main_ax, int node_start) const {
    const int pos = dual % 3 == (field % 3 + 1) % 3 ? 1 : 2;
    const double* curl = a_.coeff[3 * field + pos];
    int shp[3];
    field_shape(field, shp);
    const auto& s = cpsi.shape();
    double r = 0;
    bool have = false;
    for (std::size_t i = 0; i < s[0]; ++i)
      for (std::size_t j = 0; j < s[1]; ++j)
        for (std::size_t k = 0; k < s[2]; ++k) {
          int g[3] = {static_cast<int>(i), static_cast<int>(j), static_cast<int>(k)};
          g[main_ax] += node_start;
          if (g[0] >= a_.nx || g[1] >= a_.ny || g[2] >= a_.nz) continue;
          const double cv = curl[(static_cast<std::size_t>(g[0]) * shp[1] + g[1]) * shp[2] + g[2]];
          const double pv = at(cpsi, i, j, k);
          if (cv == 0) {
            if (pv != 0) throw std::runtime_error("CPML c_psi nonzero where the curl coefficient is zero");
            continue;
          }
          const double q = pv / cv;
          if (!have) {
            r = q;
            have = true;
          } else if (std::fabs(q - r) > 1e-12 * std::fabs(r)) {
            throw std::runtime_error("CPML c_psi is not one multiple of the curl coefficient over its layer");
          }
        }
    return have ? r : 1.0;
  }

  void pml(xfdtd::Simulation& sim) {
    const int n[3] = {a_.nx, a_.ny, a_.nz};
    std::vector<double> ae[3], be[3], ah[3], bh[3];
    for (int ax = 0; ax < 3; ++ax) {
      ae[ax].assign(n[ax] + 1, 0.0);
      be[ax].assign(n[ax] + 1, 0.0);
      ah[ax].assign(n[ax], 0.0);
      bh[ax].assign(n[ax], 0.0);
    }
    for (const auto& b : sim.boundaries()) {
      auto* p = dynamic_cast<xfdtd::PML*>(b.get());
      if (p == nullptr) continue;
      const int ax = axis_index(p->mainAxis());
      const int fa = (ax + 1) % 3, fb = (ax + 2) % 3;  // tangential axes a, b
      int tb[6];
      box_of(p->task(), tb);
      const int lo = tb[2 * ax], hi = tb[2 * ax + 1];
      const int face = 2 * ax + (lo == 0 ? 0 : 1);
      a_.pml[face] = hi - lo;
      const int es = static_cast<int>(p->globalENodeStartIndexMainAxis());
      const int hs = static_cast<int>(p->globalHNodeStartIndexMainAxis());
      const double re_a = psi_ratio(p->coeffEAPsiHB(), fa, 3 + fb, ax, static_cast<int>(p->nodeENodeStartIndexMainAxis()));
      const double re_b = psi_ratio(p->coeffEBPsiHA(), fb, 3 + fa, ax, static_cast<int>(p->nodeENodeStartIndexMainAxis()));
      const double rh_a = psi_ratio(p->coeffHAPsiEB(), 3 + fa, fb, ax, static_cast<int>(p->nodeHNodeStartIndexMainAxis()));
      const double rh_b = psi_ratio(p->coeffHBPsiEA(), 3 + fb, fa, ax, static_cast<int>(p->nodeHNodeStartIndexMainAxis()));
      if (std::fabs(re_a - re_b) > 1e-12 * std::fabs(re_a) || std::fabs(rh_a - rh_b) > 1e-12 * std::fabs(rh_a))
        throw std::runtime_error("CPML c_psi ratios differ between the two tangential fields");
      const auto& cae = p->coeffAE();
      const auto& cbe = p->coeffBE();
      const auto& cah = p->coeffAH();
      const auto& cbh = p->coeffBH();
      for (std::size_t q = 0; q < cae.size(); ++q) {
        const std::size_t g = es + q;
        if (g > static_cast<std::size_t>(n[ax])) throw std::runtime_error("CPML E profile outside the grid");
        ae[ax][g] = static_cast<double>(cae.data()[q]) * re_a;
        be[ax][g] = static_cast<double>(cbe.data()[q]);
      }
      for (std::size_t q = 0; q < cah.size(); ++q) {
        const std::size_t g = hs + q;
        if (g >= static_cast<std::size_t>(n[ax])) throw std::runtime_error("CPML H profile outside the grid");
        ah[ax][g] = static_cast<double>(cah.data()[q]) * rh_a;
        bh[ax][g] = static_cast<double>(cbh.data()[q]);
      }
    }
    for (int ax = 0; ax < 3; ++ax) {
      a_.pml_ae[ax] = keep(std::move(ae[ax]));
      a_.pml_be[ax] = keep(std::move(be[ax]));
      a_.pml_ah[ax] = keep(std::move(ah[ax]));
      a_.pml_bh[ax] = keep(std::move(bh[ax]));
    }
  }

  void tfsf(xfdtd::Simulation& sim) {
    for (const auto& w : sim.waveformSources()) {
      auto* t = dynamic_cast<xfdtd::TFSF*>(w.get());
      if (t == nullptr) continue;
      if (a_.tfsf_enabled) throw std::runtime_error("the engine takes one TFSF source");
      a_.tfsf_enabled = 1;
      box_of(t->globalTask(), a_.tfsf_box);
      a_.tfsf_proj_int[0] = keep(flat(t->projectionXInt()));
      a_.tfsf_proj_int[1] = keep(flat(t->projectionYInt()));
      a_.tfsf_proj_int[2] = keep(flat(t->projectionZInt()));
      a_.tfsf_proj_half[0] = keep(flat(t->projectionXHalf()));
      a_.tfsf_proj_half[1] = keep(flat(t->projectionYHalf()));
      a_.tfsf_proj_half[2] = keep(flat(t->projectionZHalf()));
      for (int ax = 0; ax < 3; ++ax) {
        const int nb = a_.tfsf_box[2 * ax + 1] - a_.tfsf_box[2 * ax];
        const std::size_t ni = store_[store_.size() - 6 + ax].size(), nh = store_[store_.size() - 3 + ax].size();
        if (ni < static_cast<std::size_t>(nb + 1) || nh < static_cast<std::size_t>(nb + 2))
          throw std::runtime_error("TFSF projections shorter than the box");
      }
      const auto te = t->transformE();
      const auto th = t->transformH();
      a_.tfsf_transform_e[0] = te.x(); a_.tfsf_transform_e[1] = te.y(); a_.tfsf_transform_e[2] = te.z();
      a_.tfsf_transform_h[0] = th.x(); a_.tfsf_transform_h[1] = th.y(); a_.tfsf_transform_h[2] = th.z();
      a_.tfsf_ca[0] = t->cax(); a_.tfsf_ca[1] = t->cay(); a_.tfsf_ca[2] = t->caz();
      a_.tfsf_cb[0] = t->cbx(); a_.tfsf_cb[1] = t->cby(); a_.tfsf_cb[2] = t->cbz();
      // e_inc (rows, le), h_inc (rows, lh): the engine reads E rows of aux_nl + 1
      // and H rows of aux_nl entries, inc_steps rows of H and one more of E
      const auto& ei = t->eInc();
      const auto& hi = t->hInc();
      const std::size_t er = ei.shape()[0], el = ei.shape()[1], hr = hi.shape()[0], hl = hi.shape()[1];
      const std::size_t nl = std::min(el - 1, hl);
      if (el < 2 || hl < 1 || nl < 2) throw std::runtime_error("TFSF incident tables too short");
      const std::size_t rows = std::min(er, hr);
      std::vector<double> e((rows + 1) * (nl + 1), 0.0), h(rows * nl);
      for (std::size_t r = 0; r < rows + 1 && r < er; ++r)
        for (std::size_t q = 0; q <= nl; ++q) e[r * (nl + 1) + q] = static_cast<double>(ei.data()[r * el + q]);
      for (std::size_t r = 0; r < rows; ++r)
        for (std::size_t q = 0; q < nl; ++q) h[r * nl + q] = static_cast<double>(hi.data()[r * hl + q]);
      a_.aux_nl = static_cast<int>(nl);
      a_.inc_steps = static_cast<long long>(rows);
      a_.e_inc = keep(std::move(e));
      a_.h_inc = keep(std::move(h));
    }
  }

  void nf2ff(xfdtd::Simulation& sim) {
    for (const auto& n : sim.nf2ffs()) {
      if (auto* fd = dynamic_cast<xfdtd::NFFFTFrequencyDomain*>(n.get())) {
        if (a_.nf2ff_enabled) throw std::runtime_error("the engine takes one frequency-domain NF2FF box");
        a_.nf2ff_enabled = 1;
        int xn[6], xp[6], yn[6], yp[6], zn[6], zp[6];
        box_of(fd->globalTaskSurfaceXN(), xn);
        box_of(fd->globalTaskSurfaceXP(), xp);
        box_of(fd->globalTaskSurfaceYN(), yn);
        box_of(fd->globalTaskSurfaceYP(), yp);
        box_of(fd->globalTaskSurfaceZN(), zn);
        box_of(fd->globalTaskSurfaceZP(), zp);
        const int b[6] = {xn[0], xp[0], yn[2], yp[2], zn[4], zp[4]};
        std::copy(b, b + 6, a_.nf2ff_box);
        std::vector<double> f;
        for (int q = 0; q < static_cast<int>(fd->freqCount()); ++q) {
          const auto& tr = fd->transformE(q);
          if (tr.size() < 2) throw std::runtime_error("NF2FF transform needs two steps");
          const std::complex<double> t0(tr.data()[0]), t1(tr.data()[1]);
          f.push_back(-std::arg(t1 / t0) / (2 * 3.14159265358979323846 * a_.dt));
        }
        a_.n_freqs = static_cast<int>(f.size());
        a_.freqs = keep(std::move(f));
      } else if (auto* td = dynamic_cast<xfdtd::NFFFTTimeDomain*>(n.get())) {
        if (a_.nf2ff_td_enabled) throw std::runtime_error("the engine takes one time-domain NF2FF box");
        a_.nf2ff_td_enabled = 1;
        int xn[6], xp[6], yn[6], yp[6], zn[6], zp[6];
        box_of(td->nodeTaskSurfaceXN(), xn);
        box_of(td->nodeTaskSurfaceXP(), xp);
        box_of(td->nodeTaskSurfaceYN(), yn);
        box_of(td->nodeTaskSurfaceYP(), yp);
        box_of(td->nodeTaskSurfaceZN(), zn);
        box_of(td->nodeTaskSurfaceZP(), zp);
        const int b[6] = {xn[0], xp[0], yn[2], yp[2], zn[4], zp[4]};
        std::copy(b, b + 6, a_.nf2ff_td_box);
        const auto r = td->observationDirection();
        const double x = r.x(), y = r.y(), z = r.z();
        const double len = std::sqrt(x * x + y * y + z * z);
        a_.nf2ff_td_theta = std::acos(z / len);
        a_.nf2ff_td_phi = std::atan2(y, x);
      }
    }
  }

  void movies(xfdtd::Simulation& sim) {
    for (const auto& m : sim.monitors()) {
      auto* mv = dynamic_cast<xfdtd::MovieMonitor*>(m.get());
      if (mv == nullptr) continue;
      auto* fm = dynamic_cast<xfdtd::FieldMonitor*>(mv->frame().get());
      if (fm == nullptr) continue;
      xfb_movie x{};
      switch (fm->field()) {
        case xfdtd::EMF::Field::EX: x.field = XFB_EX; break;
        case xfdtd::EMF::Field::EY: x.field = XFB_EY; break;
        case xfdtd::EMF::Field::EZ: x.field = XFB_EZ; break;
        case xfdtd::EMF::Field::HX: x.field = XFB_HX; break;
        case xfdtd::EMF::Field::HY: x.field = XFB_HY; break;
        case xfdtd::EMF::Field::HZ: x.field = XFB_HZ; break;
        default: continue;
      }
      int b[6];
      box_of(fm->globalTask(), b);
      for (int ax = 0; ax < 3; ++ax) {
        x.lo[ax] = b[2 * ax];
        x.hi[ax] = b[2 * ax + 1];
      }
      x.interval = static_cast<int>(mv->frameInterval());
      movies_.push_back(x);
    }
    a_.n_movies = static_cast<int>(movies_.size());
    a_.movies = movies_.empty() ? nullptr : movies_.data();
  }
};

}  // namespace xfb_core

#endif  // __has_include(<xfdtd/simulation/simulation.h>)
#endif  // XFDTD_B200_XFDTD_CORE_ADAPTER_HPP_
