// A stand-in for the XFDTD_CORE accessor surface that the reference's *HD
// wrappers call (src/simulation/simulation_hd.cu:105-398 and the wrappers it
// builds).  Test infrastructure: it holds plain arrays the test fills, so the
// adapter header compiles and runs where XFDTD_CORE is absent.  Arrays follow
// the xtensor calls the adapter uses: shape(), size(), dimension(), data().
#pragma once

#include <complex>
#include <cstddef>
#include <memory>
#include <vector>

namespace xfdtd {

template <typename T>
struct Array {
  std::vector<std::size_t> s;
  std::vector<T> v;
  Array() = default;
  Array(std::vector<std::size_t> shape, T fill) : s(std::move(shape)) {
    std::size_t n = 1;
    for (auto d : s) n *= d;
    v.assign(n, fill);
  }
  const std::vector<std::size_t>& shape() const { return s; }
  std::size_t size() const { return v.size(); }
  std::size_t dimension() const { return s.size(); }
  const T* data() const { return v.data(); }
  T& operator()(std::size_t i) { return v[i]; }
  T& operator()(std::size_t i, std::size_t j) { return v[i * s[1] + j]; }
  T& operator()(std::size_t i, std::size_t j, std::size_t k) { return v[(i * s[1] + j) * s[2] + k]; }
  T& operator()(std::size_t i, std::size_t j, std::size_t k, std::size_t p) {
    return v[((i * s[1] + j) * s[2] + k) * s[3] + p];
  }
};

struct Range {
  std::size_t a = 0, b = 0;
  std::size_t start() const { return a; }
  std::size_t end() const { return b; }
};

struct IndexTask {
  Range x, y, z;
  const Range& xRange() const { return x; }
  const Range& yRange() const { return y; }
  const Range& zRange() const { return z; }
};

struct Vector {
  double vx = 0, vy = 0, vz = 0;
  double x() const { return vx; }
  double y() const { return vy; }
  double z() const { return vz; }
};

namespace Axis {
enum class XYZ { X, Y, Z };
}
namespace EMF {
enum class Field { EX, EY, EZ, HX, HY, HZ, EM, HM };
}

struct GridSpace {
  enum class Dimension { ONE, TWO, THREE };
  Dimension dim = Dimension::THREE;
  std::size_t n[3] = {0, 0, 0};
  Array<double> e[3];
  Dimension dimension() const { return dim; }
  std::size_t sizeX() const { return n[0]; }
  std::size_t sizeY() const { return n[1]; }
  std::size_t sizeZ() const { return n[2]; }
  const Array<double>& eNodeX() const { return e[0]; }
  const Array<double>& eNodeY() const { return e[1]; }
  const Array<double>& eNodeZ() const { return e[2]; }
};

struct TimeParam {
  double step = 0;
  double dt() const { return step; }
};

struct FDTDCoefficient {
  Array<double> c[18];  // cexe cexhy cexhz ceye ceyhz ceyhx ceze cezhx cezhy chxh chxey chxez chyh chyez chyex chzh chzex chzey
  const Array<double>& cexe() const { return c[0]; }
  const Array<double>& cexhy() const { return c[1]; }
  const Array<double>& cexhz() const { return c[2]; }
  const Array<double>& ceye() const { return c[3]; }
  const Array<double>& ceyhz() const { return c[4]; }
  const Array<double>& ceyhx() const { return c[5]; }
  const Array<double>& ceze() const { return c[6]; }
  const Array<double>& cezhx() const { return c[7]; }
  const Array<double>& cezhy() const { return c[8]; }
  const Array<double>& chxh() const { return c[9]; }
  const Array<double>& chxey() const { return c[10]; }
  const Array<double>& chxez() const { return c[11]; }
  const Array<double>& chyh() const { return c[12]; }
  const Array<double>& chyez() const { return c[13]; }
  const Array<double>& chyex() const { return c[14]; }
  const Array<double>& chzh() const { return c[15]; }
  const Array<double>& chzex() const { return c[16]; }
  const Array<double>& chzey() const { return c[17]; }
};

struct CalculationParam {
  std::shared_ptr<TimeParam> time = std::make_shared<TimeParam>();
  std::shared_ptr<FDTDCoefficient> coeff = std::make_shared<FDTDCoefficient>();
  std::shared_ptr<TimeParam> timeParam() const { return time; }
  std::shared_ptr<FDTDCoefficient> fdtdCoefficient() const { return coeff; }
};

struct Boundary {
  virtual ~Boundary() = default;
};

struct PML : Boundary {
  Axis::XYZ axis = Axis::XYZ::X;
  IndexTask t;
  std::size_t e_start = 0, h_start = 0;
  Array<double> ae, be, ah, bh, c_ea, c_eb, c_ha, c_hb;
  Axis::XYZ mainAxis() const { return axis; }
  const IndexTask& task() const { return t; }
  std::size_t globalENodeStartIndexMainAxis() const { return e_start; }
  std::size_t globalHNodeStartIndexMainAxis() const { return h_start; }
  std::size_t nodeENodeStartIndexMainAxis() const { return e_start; }
  std::size_t nodeHNodeStartIndexMainAxis() const { return h_start; }
  const Array<double>& coeffAE() const { return ae; }
  const Array<double>& coeffBE() const { return be; }
  const Array<double>& coeffAH() const { return ah; }
  const Array<double>& coeffBH() const { return bh; }
  const Array<double>& coeffEAPsiHB() const { return c_ea; }
  const Array<double>& coeffEBPsiHA() const { return c_eb; }
  const Array<double>& coeffHAPsiEB() const { return c_ha; }
  const Array<double>& coeffHBPsiEA() const { return c_hb; }
};

struct WaveformSource {
  virtual ~WaveformSource() = default;
};

struct TFSF : WaveformSource {
  IndexTask box;
  Array<double> pi[3], ph[3], e_inc, h_inc;
  Vector te, th;
  double ca[3] = {0, 0, 0}, cb[3] = {0, 0, 0};
  const IndexTask& globalTask() const { return box; }
  const Array<double>& projectionXInt() const { return pi[0]; }
  const Array<double>& projectionYInt() const { return pi[1]; }
  const Array<double>& projectionZInt() const { return pi[2]; }
  const Array<double>& projectionXHalf() const { return ph[0]; }
  const Array<double>& projectionYHalf() const { return ph[1]; }
  const Array<double>& projectionZHalf() const { return ph[2]; }
  const Array<double>& eInc() const { return e_inc; }
  const Array<double>& hInc() const { return h_inc; }
  Vector transformE() const { return te; }
  Vector transformH() const { return th; }
  double cax() const { return ca[0]; }
  double cay() const { return ca[1]; }
  double caz() const { return ca[2]; }
  double cbx() const { return cb[0]; }
  double cby() const { return cb[1]; }
  double cbz() const { return cb[2]; }
};

struct NFFFT {
  virtual ~NFFFT() = default;
  IndexTask face[6];  // XN XP YN YP ZN ZP
};

struct NFFFTFrequencyDomain : NFFFT {
  std::vector<Array<std::complex<double>>> te;
  std::size_t freqCount() const { return te.size(); }
  const Array<std::complex<double>>& transformE(std::size_t i) const { return te[i]; }
  const IndexTask& globalTaskSurfaceXN() const { return face[0]; }
  const IndexTask& globalTaskSurfaceXP() const { return face[1]; }
  const IndexTask& globalTaskSurfaceYN() const { return face[2]; }
  const IndexTask& globalTaskSurfaceYP() const { return face[3]; }
  const IndexTask& globalTaskSurfaceZN() const { return face[4]; }
  const IndexTask& globalTaskSurfaceZP() const { return face[5]; }
};

struct NFFFTTimeDomain : NFFFT {
  Vector dir;
  Vector observationDirection() const { return dir; }
  const IndexTask& nodeTaskSurfaceXN() const { return face[0]; }
  const IndexTask& nodeTaskSurfaceXP() const { return face[1]; }
  const IndexTask& nodeTaskSurfaceYN() const { return face[2]; }
  const IndexTask& nodeTaskSurfaceYP() const { return face[3]; }
  const IndexTask& nodeTaskSurfaceZN() const { return face[4]; }
  const IndexTask& nodeTaskSurfaceZP() const { return face[5]; }
};

struct Monitor {
  virtual ~Monitor() = default;
};

struct FieldMonitor : Monitor {
  EMF::Field f = EMF::Field::EZ;
  IndexTask t;
  EMF::Field field() const { return f; }
  const IndexTask& globalTask() const { return t; }
};

struct MovieMonitor : Monitor {
  std::shared_ptr<Monitor> fr;
  std::size_t interval = 1;
  const std::shared_ptr<Monitor>& frame() const { return fr; }
  std::size_t frameInterval() const { return interval; }
};

struct ADEMethodStorage {
  virtual ~ADEMethodStorage() = default;
  Array<double> pole[7];  // jj jjp jen je jep jsj jsjp, (nx, ny, nz, poles)
  Array<double> eep, ejs;
  const Array<double>& coeffJJ() const { return pole[0]; }
  const Array<double>& coeffJJPrev() const { return pole[1]; }
  const Array<double>& coeffJENext() const { return pole[2]; }
  const Array<double>& coeffJE() const { return pole[3]; }
  const Array<double>& coeffJEPrev() const { return pole[4]; }
  const Array<double>& coeffJSumJ() const { return pole[5]; }
  const Array<double>& coeffJSumJPrev() const { return pole[6]; }
  const Array<double>& coeffEEPrev() const { return eep; }
  const Array<double>& coeffEJSum() const { return ejs; }
};
struct DrudeADEMethodStorage : ADEMethodStorage {};
struct DebyeADEMethodStorage : ADEMethodStorage {};
struct MLorentzADEMethodStorage : ADEMethodStorage {};

struct Simulation {
  long long inited = -1;
  std::shared_ptr<GridSpace> grid = std::make_shared<GridSpace>();
  std::shared_ptr<CalculationParam> param = std::make_shared<CalculationParam>();
  std::shared_ptr<ADEMethodStorage> ade;
  std::vector<std::shared_ptr<Boundary>> bounds;
  std::vector<std::shared_ptr<WaveformSource>> sources;
  std::vector<std::shared_ptr<NFFFT>> nf;
  std::vector<std::shared_ptr<Monitor>> mons;
  void init(long long steps) { inited = steps; }
  std::shared_ptr<GridSpace> gridSpace() const { return grid; }
  std::shared_ptr<CalculationParam> calculationParam() const { return param; }
  std::shared_ptr<ADEMethodStorage> aDEMethodStorage() const { return ade; }
  const std::vector<std::shared_ptr<Boundary>>& boundaries() const { return bounds; }
  const std::vector<std::shared_ptr<WaveformSource>>& waveformSources() const { return sources; }
  const std::vector<std::shared_ptr<NFFFT>>& nf2ffs() const { return nf; }
  const std::vector<std::shared_ptr<Monitor>>& monitors() const { return mons; }
};

}  // namespace xfdtd
