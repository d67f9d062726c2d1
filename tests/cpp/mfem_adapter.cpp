// The MFEM-side adapter of include/theseus_b200/RHSOperator.hpp
// (MFEMRHSOperator, an mfem::TimeDependentOperator), compiled against the
// test-only MFEM stand-in in tests/cpp/mfem_stub and driven by its
// RK3SSPSolver as the reference's Simulation drives its operator
// (src/Simulation.cpp:256-285,1255): Navier-Stokes Taylor-Green vortex,
// 3^3 hexes, p=4, Ranocha / HLL, two steps of dt = 1e-3.  Writes the initial
// and the final state (doubles, byNODES) and the stability rates of the
// initial state to the file named by argv[1].  Exit code 3 reports an
// operator error (for example "no CUDA device") on stderr.
#define THESEUS_B200_WITH_MFEM
#include "theseus_b200/RHSOperator.hpp"

#include <cmath>
#include <cstdio>
#include <memory>
#include <vector>

int main(int argc, char **argv) {
  if (argc < 2) return 2;
  const double pi = 3.14159265358979323846;
  auto g = theseus_b200::Geometry::PeriodicBox(3, 4, {3, 3, 3}, {0, 0, 0}, {2 * pi, 2 * pi, 2 * pi}, true);
  const long long L = (long long)g.num_elements * g.nodes_per_element();
  std::vector<double> u0(5 * L), u1(5 * L);
  const double gamma = 1.4, Ma = 0.1, p0 = 1.0 / (gamma * Ma * Ma);
  for (long long i = 0; i < L; ++i) {
    const double x = g.coords[i], y = g.coords[L + i], z = g.coords[2 * L + i];
    const double vx = std::sin(x) * std::cos(y) * std::cos(z), vy = -std::cos(x) * std::sin(y) * std::cos(z);
    const double p = p0 + 1.0 / 16.0 * (std::cos(2 * x) + std::cos(2 * y)) * (std::cos(2 * z) + 2.0);
    u0[i] = 1.0;
    u0[L + i] = vx;
    u0[2 * L + i] = vy;
    u0[3 * L + i] = 0.0;
    u0[4 * L + i] = p / (gamma - 1.0) + 0.5 * (vx * vx + vy * vy);
  }
  double rates[3] = {0, 0, 0};
  try {
    thx_config phys = theseus_b200::DefaultPhysics();
    phys.mu = 1.0 / 1600;
    phys.Pr = 0.71;
    auto op = std::make_shared<theseus_b200::NSOperator>(g, theseus_b200::Selection{"ranocha", "hll", "llf"},
                                                         phys);
    theseus_b200::MFEMRHSOperator f(op);
    if (f.Height() != (int)(5 * L)) return 8;
    mfem::Vector x(f.Height());
    double *xp = x.HostWrite();
    for (long long i = 0; i < 5 * L; ++i) xp[i] = u0[i];
    const auto est = f.EstimateStability(x);
    rates[0] = est.advective_rate;
    rates[1] = est.surface_rate;
    rates[2] = est.diffusive_rate;
    mfem::RK3SSPSolver ode;
    ode.Init(f);
    double t = 0.0, dt = 1e-3;
    for (int step = 0; step < 2; ++step) ode.Step(x, t, dt);
    const double *xr = x.HostRead();
    for (long long i = 0; i < 5 * L; ++i) u1[i] = xr[i];
    if (std::fabs(t - 2e-3) > 1e-15) return 7;
  } catch (const std::exception &e) {
    std::fprintf(stderr, "error: %s\n", e.what());
    return 3;
  }
  FILE *fo = std::fopen(argv[1], "wb");
  if (!fo) return 5;
  std::fwrite(u0.data(), sizeof(double), u0.size(), fo);
  std::fwrite(u1.data(), sizeof(double), u1.size(), fo);
  std::fwrite(rates, sizeof(double), 3, fo);
  std::fclose(fo);
  return 0;
}
