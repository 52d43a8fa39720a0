// Internal types shared by the host scene compiler, the kernels and the C-ABI.
#pragma once

#include <cstdint>
#include <memory>
#include <new>
#include <string>
#include <vector>

#include "../../include/xfdtd_b200.h"

namespace xfb {

// Physical constants (CODATA values used throughout the engine).
constexpr double kEps0 = 8.854187817e-12;
constexpr double kMu0 = 4.0 * 3.14159265358979323846 * 1e-7;
constexpr double kPi = 3.14159265358979323846;
inline double c0() { return 1.0 / __builtin_sqrt(kEps0 * kMu0); }

constexpr int kCoeffs = 18;     // per-material Yee coefficients
constexpr int kAdeMat = 3;      // is_dispersive, ceep, cejsum
constexpr int kAdePole = 7;     // cjj cjjp cjen cje cjep cjsj cjsjp

// LUT slots (the reference's 18 FDTDCoefficient arrays,
// include/xfdtd_cuda/calculation_param/fdtd_coefficient.cuh:15-168).
enum Coef {
  CEXE = 0, CEXHY, CEXHZ, CEYE, CEYHZ, CEYHX, CEZE, CEZHX, CEZHY,
  CHXH, CHXEY, CHXEZ, CHYH, CHYEZ, CHYEX, CHZH, CHZEX, CHZEY
};

// Allocator whose resize() leaves new elements uninitialised, so that a large
// array is first touched (its pages faulted in) by the threads that fill it.
template <typename T>
struct DefaultInit : std::allocator<T> {
  template <typename U>
  struct rebind {
    using other = DefaultInit<U>;
  };
  DefaultInit() = default;
  template <typename U>
  DefaultInit(const DefaultInit<U>&) noexcept {}
  template <typename U>
  void construct(U* p) noexcept {
    ::new (static_cast<void*>(p)) U;
  }
  template <typename U, typename... A>
  void construct(U* p, A&&... a) {
    ::new (static_cast<void*>(p)) U(static_cast<A&&>(a)...);
  }
};

// Result of compiling an xfb_scene on the host: the data XFDTD_CORE would hand
// to the reference's *HD wrappers, in engine form (material index + LUT
// instead of 18 per-cell coefficient arrays).
struct Compiled {
  int dim = 3, prec = XFB_FP32;
  int nx = 0, ny = 0, nz = 0;
  double dx = 0, dy = 0, dz = 0, dt = 0;
  double origin[3] = {0, 0, 0};
  std::vector<uint8_t, DefaultInit<uint8_t>> mat_id;   // [nx][ny][nz]
  int n_mat = 0;
  std::vector<double> coeff;     // [n_mat][18]
  // Compact form of the same coefficients: [n_mat][8] = ce, cb/dx, cb/dy, cb/dz,
  // ch, db/dx, db/dy, db/dz.  Every entry of `coeff` is +- one of these values
  // exactly (e.g. cexhy = -cb/dz), so kernels reading this form with the sign
  // applied reproduce the 18-coefficient update bit for bit.
  std::vector<double> coeff8;
  std::vector<uint8_t> mat_disp; // [n_mat] 1 if the material has ADE poles
  std::vector<int> mat_is_pec;
  // ADE (dispersive media)
  int ade_kind = XFB_ADE_NONE, ade_poles = 0;
  std::vector<double> ade_mat;   // [n_mat][3]
  std::vector<double> ade_pole;  // [n_mat][ade_poles][7]
  int ade_box[6] = {0, 0, 0, 0, 0, 0};  // i0 i1 j0 j1 k0 k1 (cells), empty if i0==i1
  // CPML
  int pml[6] = {0, 0, 0, 0, 0, 0};
  std::vector<double> pml_ae[3], pml_be[3], pml_ah[3], pml_bh[3];
  // TFSF
  int tfsf_on = 0;
  int tf[6] = {0, 0, 0, 0, 0, 0};  // is ie js je ks ke (nodes)
  std::vector<double> proj_int[3], proj_half[3];
  double tr_e[3] = {0, 0, 0}, tr_h[3] = {0, 0, 0};
  double ca[3] = {0, 0, 0}, cb[3] = {0, 0, 0};
  int aux_nl = 0;
  double aux_dl = 0, aux_ceih = 0, aux_chie = 0, aux_abc = 0;
  // incident tables handed over by the caller (xfb_create_from_arrays)
  // instead of the 1-D auxiliary grid's: rows of E (nl + 1) and H (nl)
  bool inc_given = false;
  long long inc_steps = 0;
  std::vector<double> e_inc, h_inc;
  int wave_kind = XFB_WAVE_GAUSSIAN;
  double wave_tau = 0, wave_t0 = 0, wave_freq = 0;
  // NF2FF
  int nf_on = 0;
  int nf[6] = {0, 0, 0, 0, 0, 0};  // is ie js je ks ke (nodes)
  std::vector<double> freqs;
  // time-domain NF2FF: box, observation direction, reference distance (the
  // largest r . dir over the sample points) and the bins one step can reach
  int td_on = 0;
  int td[6] = {0, 0, 0, 0, 0, 0};  // is ie js je ks ke (nodes)
  double td_theta = 0, td_phi = 0;
  double td_dir[3] = {0, 0, 0};
  double td_ref = 0;
  int td_span = 0;
  long long td_bins = 0;           // total_steps + td_span (size_tables)
  // monitors
  std::vector<xfb_probe> probes;
  std::vector<xfb_movie> movies;
  // tables sized by init(total_steps)
  long long total_steps = 0;
  std::vector<double> aux_source;  // [total_steps + 1]
  std::vector<double> te, th;      // [n_freqs][total_steps][2]
};

// Host scene compiler (scene_compile.cpp).  Returns XFB_OK or an error with
// a message in *err.
int compile_scene(const xfb_scene& s, Compiled& out, std::string* err);
// The same from arrays XFDTD_CORE compiled (core_ingest.cpp).
int compile_arrays(const xfb_core_arrays& a, Compiled& out, std::string* err);
// Sizes the step-count dependent tables (TFSF source samples, NF2FF DFT
// kernels) for a run of total_steps steps.
void size_tables(Compiled& c, long long total_steps);
// Incident waveform value at time t.
double waveform(const Compiled& c, double t);

// NF2FF face geometry: extents (n0, n1) along the face's two tangential axes
// (a, b) and the first node of the face in (i, j, k).
struct FaceGeom {
  int axis;        // normal axis 0/1/2
  int positive;    // 1 for XP/YP/ZP
  int i0, j0, k0;  // first face point
  int ni, nj, nk;  // extents in i, j, k (normal extent 1)
};
FaceGeom face_geom(const Compiled& c, int face);
// The same geometry for the time-domain NF2FF box.
FaceGeom td_face_geom(const Compiled& c, int face);
// Speed of light of the reference's time-domain NF2FF
// (src/nf2ff/time_domain/nf2ff_time_domain_data.cu:16).
constexpr double kTdC0 = 299792458.0;
// Time-domain NF2FF sample point (i, j, k) of `face`: its position (the face
// node along the normal, cell centres along the tangential axes,
// nf2ff_time_domain_data.cu:53-66) and its delay in steps,
// (ref - r . dir) / (c dt).
double td_delay_steps(const Compiled& c, int face, int i, int j, int k);
void compile_td(Compiled& c, double theta, double phi);

// Read-back copies into large host result arrays, split over host threads
// (host_copy.cpp): dst[q] = double(src[q]) for q < n, and a byte copy.
void host_widen(const float* src, double* dst, long long n);
void host_widen(const double* src, double* dst, long long n);
void host_copy(const void* src, void* dst, size_t bytes);

}  // namespace xfb
