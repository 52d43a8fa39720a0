// C++ host side of the B200 engine: the reference's xfdtd::cuda::SimulationHD
// surface (include/xfdtd_cuda/simulation/simulation_hd.cuh:37-88) over the
// C-ABI of xfdtd_b200.h, and a scene builder standing in for the XFDTD_CORE
// xfdtd::Simulation the reference is constructed from.  Header-only; link
// with -lxfdtd_b200.
//
// Errors are reported as in the reference, by exceptions
// (std::runtime_error carrying the library's message), not status codes.
#pragma once

#include <array>
#include <cmath>
#include <cstddef>
#include <stdexcept>
#include <string>
#include <thread>
#include <utility>
#include <vector>

#include "../xfdtd_b200.h"

namespace xfdtd {
namespace b200 {

inline void check(int status, const xfb_handle* h = nullptr) {
  if (status != XFB_OK) {
    const char* m = xfb_last_error(h);
    throw std::runtime_error(std::string("xfdtd_b200: ") + (m && *m ? m : xfb_status_string(status)));
  }
}

// Scene description with the vocabulary of XFDTD_CORE (Simulation(dx, dy,
// dz, courant), addObject, addWaveformSource, addBoundary, addMonitor,
// addNF2FF), producing the xfb_scene the engine compiles.  The first object
// added is the domain; later objects win where they overlap.
class Scene {
 public:
  Scene(double dx, double dy, double dz, double courant, int precision = XFB_FP64, int dim = 3)
      : dx_(dx), dy_(dy), dz_(dz), courant_(courant), precision_(precision), dim_(dim) {}

  // material index for use by addObject
  int addMaterial(double eps_r, double mu_r = 1.0, double sigma_e = 0.0, double sigma_m = 0.0, bool pec = false) {
    xfb_material m{};
    m.eps_r = eps_r;
    m.mu_r = mu_r;
    m.sigma_e = sigma_e;
    m.sigma_m = sigma_m;
    m.is_pec = pec ? 1 : 0;
    materials_.push_back(m);
    return static_cast<int>(materials_.size()) - 1;
  }
  int addDispersiveMaterial(double eps_inf, const std::vector<xfb_pole>& poles, double mu_r = 1.0) {
    if (poles.size() > XFB_MAX_POLES) throw std::runtime_error("xfdtd_b200: too many poles");
    int id = addMaterial(eps_inf, mu_r);
    materials_[id].n_poles = static_cast<int>(poles.size());
    for (size_t q = 0; q < poles.size(); ++q) materials_[id].poles[q] = poles[q];
    return id;
  }
  // the domain: an axis-aligned box [origin, origin + size) of `material`
  Scene& addDomain(std::array<double, 3> origin, std::array<double, 3> size, int material) {
    domain_origin_ = origin;
    domain_size_ = size;
    domain_material_ = material;
    return *this;
  }
  Scene& addCube(std::array<double, 3> origin, std::array<double, 3> size, int material) {
    xfb_object o{};
    o.shape = XFB_SHAPE_CUBE;
    o.material = material;
    for (int a = 0; a < 3; ++a) {
      o.p[a] = origin[a];
      o.p[3 + a] = size[a];
    }
    objects_.push_back(o);
    return *this;
  }
  Scene& addSphere(std::array<double, 3> centre, double radius, int material) {
    xfb_object o{};
    o.shape = XFB_SHAPE_SPHERE;
    o.material = material;
    for (int a = 0; a < 3; ++a) o.p[a] = centre[a];
    o.p[3] = radius;
    objects_.push_back(o);
    return *this;
  }
  // CPML of `cells` cells on face `face` (enum xfb_face)
  Scene& addBoundary(int face, int cells) {
    pml_.cells[face] = cells;
    return *this;
  }
  // TFSF plane wave, Gaussian pulse exp(-((t - t0) / tau)^2)
  Scene& addWaveformSource(std::array<int, 3> inset, double theta, double phi, double psi, double tau, double t0) {
    tfsf_.enabled = 1;
    for (int a = 0; a < 3; ++a) tfsf_.inset[a] = inset[a];
    tfsf_.theta = theta;
    tfsf_.phi = phi;
    tfsf_.psi = psi;
    tfsf_.waveform = XFB_WAVE_GAUSSIAN;
    tfsf_.tau = tau;
    tfsf_.t0 = t0;
    return *this;
  }
  Scene& addNF2FF(std::array<int, 3> inset, std::vector<double> freqs) {
    nf_freqs_ = std::move(freqs);
    nf2ff_.enabled = 1;
    for (int a = 0; a < 3; ++a) nf2ff_.inset[a] = inset[a];
    return *this;
  }
  // point probe of field `field` at component index (i, j, k)
  Scene& addPointMonitor(int field, int i, int j, int k) {
    xfb_probe p{};
    p.field = field;
    p.index[0] = i;
    p.index[1] = j;
    p.index[2] = k;
    probes_.push_back(p);
    return *this;
  }

  // the C description; valid while this Scene lives and is not modified
  const xfb_scene& lower() {
    sc_ = xfb_scene{};
    sc_.dim = dim_;
    sc_.precision = precision_;
    sc_.dx = dx_;
    sc_.dy = dy_;
    sc_.dz = dz_;
    sc_.courant = courant_;
    const double d[3] = {dx_, dy_, dz_};
    for (int a = 0; a < 3; ++a) {
      sc_.domain_min[a] = domain_origin_[a];
      sc_.domain_cells[a] = static_cast<int>(std::lround(domain_size_[a] / d[a]));
    }
    if (dim_ == 2) sc_.domain_cells[2] = 1;
    lowered_materials_ = materials_;
    if (domain_material_ != 0)  // the engine takes materials[0] as the background
      std::swap(lowered_materials_[0], lowered_materials_[domain_material_]);
    lowered_objects_ = objects_;
    for (auto& o : lowered_objects_) {
      if (o.material == 0) o.material = domain_material_;
      else if (o.material == domain_material_) o.material = 0;
    }
    sc_.n_materials = static_cast<int>(lowered_materials_.size());
    sc_.materials = lowered_materials_.data();
    sc_.n_objects = static_cast<int>(lowered_objects_.size());
    sc_.objects = lowered_objects_.data();
    sc_.pml = pml_;
    if (sc_.pml.order_m == 0) {
      sc_.pml.order_m = 3.0;
      sc_.pml.sigma_ratio = 1.0;
      sc_.pml.alpha_max = 0.05;
    }
    sc_.tfsf = tfsf_;
    sc_.nf2ff = nf2ff_;
    sc_.nf2ff.n_freqs = static_cast<int>(nf_freqs_.size());
    sc_.nf2ff.freqs = nf_freqs_.data();
    sc_.n_probes = static_cast<int>(probes_.size());
    sc_.probes = probes_.data();
    return sc_;
  }

 private:
  double dx_, dy_, dz_, courant_;
  int precision_, dim_;
  std::array<double, 3> domain_origin_{}, domain_size_{};
  int domain_material_ = 0;
  std::vector<xfb_material> materials_, lowered_materials_;
  std::vector<xfb_object> objects_, lowered_objects_;
  xfb_pml pml_{};
  xfb_tfsf tfsf_{};
  xfb_nf2ff nf2ff_{};
  std::vector<double> nf_freqs_;
  std::vector<xfb_probe> probes_;
  xfb_scene sc_{};
};

}  // namespace b200

namespace cuda {

using Index = std::size_t;

struct Dim3 {
  unsigned x = 1, y = 1, z = 1;
};

// The reference's SimulationHD (include/xfdtd_cuda/simulation/simulation_hd.cuh:37-88):
// built from the host scene, setGridDim / setBlockDim, run(n).  After run()
// or copyDeviceToHost() the fields are available from field(), in the
// reference's component shapes (row-major i, j, k), as double.
class SimulationHD {
 public:
  explicit SimulationHD(b200::Scene& host) { b200::check(xfb_create(&host.lower(), &h_)); }
  ~SimulationHD() { releaseDevice(); }
  SimulationHD(const SimulationHD&) = delete;
  SimulationHD& operator=(const SimulationHD&) = delete;

  // device buffers for n steps (reference init + copyHostToDevice); the host
  // result arrays are allocated meanwhile
  void init(Index time_step) {
    start_results();
    b200::check(xfb_init(h_, static_cast<long long>(time_step)), h_);
    total_ = time_step;
  }
  void copyHostToDevice() { init(total_); }
  // re-initialise for n steps, advance them, pull the results
  void run(Index time_step) {
    start_results();
    b200::check(xfb_run(h_, static_cast<long long>(time_step)), h_);
    total_ = time_step;
    copyDeviceToHost();
  }
  void copyDeviceToHost() {
    join_results();
    xfb_grid_info gi{};
    b200::check(xfb_get_grid_info(h_, &gi), h_);
    for (int f = 0; f < 6; ++f) {
      if (gi.dim == 2 && !(f == XFB_EZ || f == XFB_HX || f == XFB_HY)) {
        fields_[f].clear();
        continue;
      }
      const size_t n = field_size(gi, f);
      if (fields_[f].size() != n) fields_[f].assign(n, 0.0);
      b200::check(xfb_read_field(h_, f, fields_[f].data(), n), h_);
    }
  }
  void releaseDevice() {
    join_results();
    if (h_) xfb_destroy(h_);
    h_ = nullptr;
  }
  void setGridDim(Dim3 g) {
    grid_ = g;
    hint();
  }
  void setBlockDim(Dim3 b) {
    block_ = b;
    hint();
  }

  const std::vector<double>& field(int f) const { return fields_[f]; }
  std::vector<double> probe(int id) {
    std::vector<double> v(total_);
    long long n = 0;
    b200::check(xfb_read_probe(h_, id, v.data(), v.size(), &n), h_);
    v.resize(static_cast<size_t>(n));
    return v;
  }
  // far field (E_theta, E_phi, complex interleaved per angle) of frequency `freq`
  std::vector<double> farField(int freq, const std::vector<double>& theta, const std::vector<double>& phi) {
    std::vector<double> out(4 * theta.size());
    b200::check(xfb_far_field(h_, freq, static_cast<int>(theta.size()), theta.data(), phi.data(), out.data()), h_);
    return out;
  }
  xfb_handle* handle() const { return h_; }

 private:
  static size_t field_size(const xfb_grid_info& gi, int f) {
    const long long nx = gi.nx, ny = gi.ny, nz = gi.nz;
    long long s[3] = {nx + (f == XFB_EY || f == XFB_EZ || f == XFB_HX), ny + (f == XFB_EX || f == XFB_EZ || f == XFB_HY),
                      nz + (f == XFB_EX || f == XFB_EY || f == XFB_HZ)};
    if (gi.dim == 2) s[2] = 1;
    return static_cast<size_t>(s[0] * s[1] * s[2]);
  }
  // The result arrays of the components (zero-filled, so every page is
  // faulted in) are allocated by one host thread each while the device
  // initialises and steps; copyDeviceToHost joins them first.  A thread that
  // cannot allocate leaves its array empty for copyDeviceToHost to size.
  void start_results() {
    join_results();
    xfb_grid_info gi{};
    b200::check(xfb_get_grid_info(h_, &gi), h_);
    for (int f = 0; f < 6; ++f) {
      if (gi.dim == 2 && !(f == XFB_EZ || f == XFB_HX || f == XFB_HY)) continue;
      const size_t n = field_size(gi, f);
      if (fields_[f].size() == n) continue;
      std::vector<double>* v = &fields_[f];
      alloc_.emplace_back([v, n] {
        try {
          v->assign(n, 0.0);
        } catch (...) {
          v->clear();
        }
      });
    }
  }
  void join_results() {
    for (std::thread& t : alloc_) t.join();
    alloc_.clear();
  }
  void hint() {
    const unsigned g[3] = {grid_.x, grid_.y, grid_.z}, b[3] = {block_.x, block_.y, block_.z};
    b200::check(xfb_set_launch_hint(h_, g, b), h_);
  }

  xfb_handle* h_ = nullptr;
  Index total_ = 0;
  Dim3 grid_, block_;
  std::array<std::vector<double>, 6> fields_;
  std::vector<std::thread> alloc_;  // result-array allocation threads
};

}  // namespace cuda
}  // namespace xfdtd
