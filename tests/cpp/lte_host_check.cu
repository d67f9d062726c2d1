// Host-side check of the library's LTE Helmholtz arithmetic (theseus_b200/csrc/
// thx_lte.cuh, the same __host__ __device__ functions the kernels run) against
// the CPU oracle (oracle/lte_oracle.h): temperature recovery and the LTEEC
// volume and face fluxes must agree bit for bit on seeded states, including
// equal and nearly equal endpoints and endpoints in different table cells.
// Build: nvcc -std=c++17 -Xcompiler -ffp-contract=off (no GPU needed to run).
#include "thx_lte.cuh"
#include "lte_oracle.h"
#include "theseus_b200.h"

#include <cstdio>
#include <cstring>
#include <random>
#include <vector>

int main() {
  const int nx = 96, ny = 160;
  std::vector<double> rho(nx), T(ny), planes(6 * nx * ny), e(ny), inv(nx * ny);
  thx_idg_params g{8.314462618 / 0.0319988, 1.5e5, 59500.0, 1.9e-5, 273.15, 0.71};
  if (thx_lte_idg_table(&g, nx, ny, -6, 1, 2.3, 4.3, rho.data(), T.data(), planes.data()) ||
      thx_lte_inverse_table(nx, ny, rho.data(), T.data(), planes.data(), e.data(), inv.data()))
    return 2;
  thx::LteDev t;
  t.nx = nx; t.ny = ny; t.rho = rho.data(); t.T = T.data(); t.e = e.data();
  t.planes = planes.data(); t.inv = inv.data();
  orc::lte::Table o;
  o.nx = nx; o.ny = ny; o.rho = rho.data(); o.T = T.data(); o.e = e.data();
  o.planes = planes.data(); o.inv = inv.data();
  std::mt19937_64 r(1);
  std::uniform_real_distribution<double> U(0, 1);
  int bad = 0, n = 0;
  for (int k = 0; k < 20000; ++k) {
    auto make = [&](double *q) {
      const double rh = 0.01 * (1 + (k % 3 == 0 ? 1e-9 : 0.3) * U(r));
      const double Tt = 3000 * (1 + (k % 5 == 0 ? 1e-10 : 0.5) * U(r));
      const double ei = orc::lte::at(o, rh, Tt).energy();
      const double u[3] = {300 * (2 * U(r) - 1), 300 * (2 * U(r) - 1), 300 * (2 * U(r) - 1)};
      q[0] = rh; q[1] = rh * u[0]; q[2] = rh * u[1]; q[3] = rh * u[2];
      q[4] = rh * ei + 0.5 * rh * (u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
    };
    double q1[5], q2[5], d1[3], d2[3];
    make(q1);
    if (k % 7 == 0) std::memcpy(q2, q1, sizeof(q1));
    else make(q2);
    for (int i = 0; i < 3; ++i) { d1[i] = 2 * U(r) - 1; d2[i] = 2 * U(r) - 1; }
    // temperature recovery
    bool bp = false;
    const thx::LteEval s1 = thx::lte_state<3>(t, q1, &bp), s2 = thx::lte_state<3>(t, q2, &bp);
    bool bo = false;
    const orc::lte::Eval o1 = orc::lte::evaluate_state(o, 3, q1, &bo);
    if (bp || bo || std::memcmp(&s1.T, &o1.T, sizeof(double)) != 0) ++bad;
    const thx::LteJet j1 = thx::lte_jet(t, s1), j2 = thx::lte_jet(t, s2);
    for (int face = 0; face < 2; ++face) {
      double Fo[5], Fp[5], m[3];
      bool b = false;
      orc::lte::lteec(o, 3, face, q1, q2, d1, face ? d1 : d2, Fo, &b);
      if (face) {
        // the face kernel's jets carry the traces' squared sound speeds
        thx::lte_ec_flux<3, true>(t, q1, q2, s1, s2, thx::lte_face_jet(t, s1), thx::lte_face_jet(t, s2),
                                  d1, d1, Fp);
      } else {
        // the volume kernel passes the averaged metric as both rows
        for (int i = 0; i < 3; ++i) m[i] = 0.5 * (d1[i] + d2[i]);
        thx::lte_ec_flux<3, false>(t, q1, q2, s1, s2, j1, j2, m, m, Fp);
      }
      ++n;
      if (b || std::memcmp(Fo, Fp, sizeof(Fo)) != 0) {
        if (bad < 5) std::printf("mismatch k=%d face=%d\n", k, face);
        ++bad;
      }
    }
  }
  std::printf("%d fluxes, %d mismatches\n", n, bad);
  return bad != 0;
}
