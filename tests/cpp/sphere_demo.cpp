// The reference's usage pattern (build a Simulation, wrap it in SimulationHD,
// set launch dims, run) through the C++ host header, on the FP64 dielectric
// sphere of the parity tests.  Prints one line:
//   ok <sum Ez> <sum |Hx|> <probe value at the last step> <|E_theta| at theta = pi/2>
// or, when the library reports an error, "error: <message>" and exit code 3.
#include <cmath>
#include <cstdio>
#include <numeric>
#include <stdexcept>

#include "xfdtd_b200/simulation_hd.hpp"

int main(int argc, char** argv) {
  const int steps = argc > 1 ? std::atoi(argv[1]) : 60;
  try {
    const double dl = 5e-3, side = 28 * dl, h = side / 2;
    xfdtd::b200::Scene sim(dl, dl, dl, 0.9, XFB_FP64);
    const int air = sim.addMaterial(1.0);
    const int diel = sim.addMaterial(3.0, 2.0);
    sim.addDomain({-h, -h, -h}, {side, side, side}, air);
    sim.addSphere({0.0, 0.0, 0.0}, 0.03, diel);
    for (int f = 0; f < 6; ++f) sim.addBoundary(f, 6);
    const double tau = 20 * dl / 6e8;
    sim.addWaveformSource({5, 5, 5}, M_PI / 2, 0.0, 0.0, tau, 4.5 * tau);
    sim.addNF2FF({3, 3, 3}, {1.5e9});
    sim.addPointMonitor(XFB_EZ, 20, 20, 20);
    xfdtd::cuda::SimulationHD hd(sim);
    hd.setGridDim({4, 4, 4});
    hd.setBlockDim({32, 8, 1});
    hd.run(static_cast<xfdtd::cuda::Index>(steps));
    const auto& ez = hd.field(XFB_EZ);
    const auto& hx = hd.field(XFB_HX);
    const double sez = std::accumulate(ez.begin(), ez.end(), 0.0);
    double shx = 0;
    for (double v : hx) shx += std::fabs(v);
    const auto pr = hd.probe(0);
    const auto ff = hd.farField(0, {M_PI / 2}, {0.0});
    std::printf("ok %.17g %.17g %.17g %.17g\n", sez, shx, pr.back(), std::hypot(ff[0], ff[1]));
  } catch (const std::runtime_error& e) {
    std::printf("error: %s\n", e.what());
    return 3;
  }
  return 0;
}
