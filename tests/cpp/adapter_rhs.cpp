// C++ caller of the library through include/theseus_b200/RHSOperator.hpp:
// Navier-Stokes Taylor-Green vortex (3^3 hexes, p=4, Ranocha volume / HLL
// surface flux), one Mult on device memory (checked against the same rate
// through host buffers, exit code 6, and followed by a three-cycle clocked
// time loop, exit code 7).  Writes u and dudt (doubles, byNODES) to the file
// named by argv[1].  Exit code 3 reports an operator
// error (for example "no CUDA device") on stderr.
#include "theseus_b200/RHSOperator.hpp"

#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <vector>

int main(int argc, char **argv) {
  if (argc < 2) return 2;
  const double pi = 3.14159265358979323846;
  auto g = theseus_b200::Geometry::PeriodicBox(3, 4, {3, 3, 3}, {0, 0, 0}, {2 * pi, 2 * pi, 2 * pi}, true);
  const long long L = (long long)g.num_elements * g.nodes_per_element();
  std::vector<double> u(5 * L), du(5 * L);
  const double gamma = 1.4, Ma = 0.1, p0 = 1.0 / (gamma * Ma * Ma);
  for (long long i = 0; i < L; ++i) {
    const double x = g.coords[i], y = g.coords[L + i], z = g.coords[2 * L + i];
    const double vx = std::sin(x) * std::cos(y) * std::cos(z), vy = -std::cos(x) * std::sin(y) * std::cos(z);
    const double p = p0 + 1.0 / 16.0 * (std::cos(2 * x) + std::cos(2 * y)) * (std::cos(2 * z) + 2.0);
    u[i] = 1.0;
    u[L + i] = vx;
    u[2 * L + i] = vy;
    u[3 * L + i] = 0.0;
    u[4 * L + i] = p / (gamma - 1.0) + 0.5 * (vx * vx + vy * vy);
  }
  try {
    thx_config phys = theseus_b200::DefaultPhysics();
    phys.mu = 1.0 / 1600;
    phys.Pr = 0.71;
    theseus_b200::NSOperator op(g, theseus_b200::Selection{"ranocha", "hll", "llf"}, phys);
    double *ud = nullptr, *dd = nullptr;
    if (cudaMalloc(&ud, sizeof(double) * u.size()) != cudaSuccess ||
        cudaMalloc(&dd, sizeof(double) * u.size()) != cudaSuccess)
      return 4;
    cudaMemcpy(ud, u.data(), sizeof(double) * u.size(), cudaMemcpyHostToDevice);
    op.Mult(ud, dd);
    cudaMemcpy(du.data(), dd, sizeof(double) * du.size(), cudaMemcpyDeviceToHost);
    // the same rate through host buffers, twice in one call
    std::vector<double> h0(du.size()), h1(du.size());
    const double *ins[2] = {u.data(), u.data()};
    double *outs[2] = {h0.data(), h1.data()};
    op.MultHost(2, ins, outs);
    cudaDeviceSynchronize();
    if (h0 != du || h1 != du) return 6;
    // three fixed steps of the clocked loop, then a finished loop leaves u alone
    thx_time_loop loop = theseus_b200::TimeLoopDefaults(1.0, 1e-3, 3, -1.0), *loop_dev = nullptr;
    if (cudaMalloc(&loop_dev, sizeof(loop)) != cudaSuccess) return 4;
    cudaMemcpy(loop_dev, &loop, sizeof(loop), cudaMemcpyHostToDevice);
    op.RunTimeLoop(ud, 0.0, 5, loop_dev);
    cudaMemcpy(&loop, loop_dev, sizeof(loop), cudaMemcpyDeviceToHost);
    cudaFree(loop_dev);
    if (loop.cycle != 3 || !loop.done || std::fabs(loop.t - 3e-3) > 1e-15) return 7;
    cudaFree(ud);
    cudaFree(dd);
    std::printf("%s\n", op.Describe().c_str());
  } catch (const std::exception &e) {
    std::fprintf(stderr, "error: %s\n", e.what());
    return 3;
  }
  FILE *f = std::fopen(argv[1], "wb");
  if (!f) return 5;
  std::fwrite(u.data(), sizeof(double), u.size(), f);
  std::fwrite(du.data(), sizeof(double), du.size(), f);
  std::fclose(f);
  return 0;
}
