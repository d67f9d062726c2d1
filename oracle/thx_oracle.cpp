// thx_oracle.cpp -- TEST INFRASTRUCTURE ONLY.
//
// CPU, FP64 restatement of Theseus's DGSEM right-hand-side evaluation, used as
// the correctness oracle for the CUDA path and as the timed CPU baseline.  It
// is never linked into, loaded by, or called from the product library.
//
// Every routine names the reference file:line whose arithmetic it restates
// (paths relative to the reference project root).  The MFEM-owned pieces the
// reference relies on (LGL rule, periodic Cartesian mesh, geometric factors,
// face restriction and its transpose, SSP-RK3) are restated from their
// published definitions.
//
// Parity pin: the pointwise fluxes, the volume/face/FV/gradient/viscous point
// kernels and the full RHS of this file are compared against the reference's
// own headers compiled here (oracle/ref_harness.cpp -> oracle/_ref/) and
// against fixtures generated from it (tests/golden/).
#include "../include/theseus_b200.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "lte_oracle.h"
#ifdef _OPENMP
#include <omp.h>
#endif

namespace orc {

constexpr int MAXEQ = 5;
constexpr int MAXDIM = 3;

// ---------------------------------------------------------------------------
// Ideal-gas model: include/Physics.hpp:22-35 (PhysicsConstants), include/EOS.hpp
// (IdealSingleGasEOS), include/Transport.hpp (constant or Sutherland viscosity).
struct Gas {
  int dim;
  double gamma, gm1, gm1_inv, R, cp, Pr_inv, mu, mu0, mu_bulk, T0, Ts;
  bool sutherland;
  const lte::Table *lte = nullptr;       // LTE Helmholtz gas when set
  std::atomic<int> *bad = nullptr;       // failed temperature recoveries
};

static inline lte::Eval lte_state(const Gas &g, const double *q) {
  bool bad = false;
  lte::Eval s = lte::evaluate_state(*g.lte, g.dim, q, &bad);
  if (bad && g.bad) g.bad->fetch_add(1);
  return s;
}

static Gas make_gas(const thx_config &c, int dim) {
  Gas g;
  g.dim = dim;
  g.gamma = c.gamma;
  g.gm1 = c.gamma - 1.0;
  g.gm1_inv = 1.0 / g.gm1;
  const double gamma_gm1_inv = c.gamma * g.gm1_inv;
  g.R = c.R_gas;
  g.cp = gamma_gm1_inv * c.R_gas;
  g.Pr_inv = 1.0 / c.Pr;
  g.mu = c.mu;
  g.mu0 = c.mu0;
  g.mu_bulk = c.mu_bulk;
  g.T0 = c.T0;
  g.Ts = c.Ts;
  g.sutherland = c.sutherland != 0;
  return g;
}

static inline double vel(const double *q, int d) { return q[1 + d] / q[0]; }
// include/EOS.hpp:88-97
static inline double ke_density(const Gas &g, const double *q) {
  double m2 = 0.0;
  for (int d = 0; d < g.dim; ++d) m2 += q[1 + d] * q[1 + d];
  return 0.5 * m2 / q[0];
}
// include/EOS.hpp:130-138
static inline double pressure(const Gas &g, const double *q) {
  return g.gm1 * (q[g.dim + 1] - ke_density(g, q));
}
// include/EOS.hpp:119-126
static inline double spec_internal_energy(const Gas &g, const double *q) {
  return (q[g.dim + 1] - ke_density(g, q)) / q[0];
}
// include/EOS.hpp:177-184
static inline double sound_speed(const Gas &g, const double *q) {
  return std::sqrt(g.gamma * pressure(g, q) / q[0]);
}
// include/EOS.hpp:150-157
static inline double temperature(const Gas &g, const double *q) {
  return pressure(g, q) / (q[0] * g.R);
}
// include/Transport.hpp:26-40; LTE: include/LTETransport.hpp:33-65 (table planes)
static inline double viscosity(const Gas &g, const double *q) {
  if (g.lte) return lte_state(g, q).transport(*g.lte, 4);
  if (g.sutherland) {
    const double T = temperature(g, q);
    const double Trel = T / g.T0;
    const double T0pTs = g.T0 + g.Ts;
    return g.mu0 * T0pTs * Trel * std::sqrt(Trel) / (T + g.Ts);
  }
  return g.mu;
}
// include/Transport.hpp:50-57
static inline double conductivity(const Gas &g, const double *q) {
  if (g.lte) return lte_state(g, q).transport(*g.lte, 5);
  return viscosity(g, q) * g.cp * g.Pr_inv;
}
// include/EOS.hpp:159-173
static inline void grad_temperature(const Gas &g, const double *q,
                                    const double *grho, const double *gp,
                                    double *gT) {
  if (g.lte) {  // include/LTEHelmholtzGasEOS.hpp:133-142
    for (int i = 0; i < g.dim; ++i) gT[i] = gp[i];
    return;
  }
  const double rho = q[0];
  const double pressor = pressure(g, q) / rho;
  const double cv = g.cp / g.gamma;
  const double fac = g.gm1_inv / (cv * rho);
  for (int i = 0; i < g.dim; ++i) gT[i] = fac * (gp[i] - pressor * grho[i]);
}
// include/EOS.hpp:206-234; LTE: include/LTEHelmholtzGasEOS.hpp:144-157
static inline void entropy_vars(const Gas &g, const double *q, double *w) {
  if (g.lte) {
    const lte::Eval s = lte_state(g, q);
    const double beta = 1 / s.T;
    double m2 = 0.0;
    for (int d = 0; d < g.dim; ++d) m2 += q[1 + d] * q[1 + d];
    const double kinetic = (0.5 * m2 / q[0]) / q[0];
    w[0] = beta * (s.gibbs() - kinetic);
    for (int d = 0; d < g.dim; ++d) w[1 + d] = beta * (q[1 + d] / q[0]);
    w[g.dim + 1] = -beta;
    return;
  }
  const double p = pressure(g, q);
  const double rho = q[0];
  const double s = std::log(p) - g.gamma * std::log(rho);
  const double beta = rho / p;
  const double v2o2 = ke_density(g, q) / rho;
  const double s_rho = (g.gamma - s) / (g.gamma - 1) - beta * v2o2;
  w[0] = s_rho;
  for (int d = 0; d < g.dim; ++d) w[1 + d] = beta * vel(q, d);
  w[g.dim + 1] = -beta;
}
// include/EOS.hpp:236-263 (gradient of entropy variables -> gradient of
// (rho, u, p) in one physical direction)
static inline void grad_entropy_to_prim(const Gas &g, const double *q,
                                        const double *dE, double *dP) {
  const int dim = g.dim, E = dim + 1;
  if (g.lte) {
    // include/LTEHelmholtzGasEOS.hpp:159-172: the energy slot holds grad T
    const double t = lte_state(g, q).T;
    dP[0] = 0.0;
    for (int d = 0; d < dim; ++d) dP[1 + d] = t * dE[1 + d] + t * (q[1 + d] / q[0]) * dE[E];
    dP[E] = t * t * dE[E];
    return;
  }
  const double ke = ke_density(g, q);
  const double p = pressure(g, q);
  const double rho = q[0];
  const double ie = q[E] - ke;
  double drho = 0.0;
  for (int d = 0; d < dim; ++d) {
    dP[1 + d] = p / rho * (dE[1 + d] + vel(q, d) * dE[E]);
    drho += q[1 + d] * dP[1 + d];
  }
  drho = rho * dE[0] - dE[E] * (ke - ie) + rho * drho / p;
  dP[0] = drho;
  dP[E] = p / rho * (dP[0] + p * dE[E]);
}

// include/theseus_kernels.hpp:106-123
static inline double log_mean(double x, double y) {
  const double eps = 1e-4;
  const double xi = y / x;
  const double u = (xi * (xi - 2.0) + 1.0) / (xi * (xi + 2.0) + 1.0);
  if (u < eps) {
    const double denom = 105.0 + u * (35.0 + u * (21.0 + 15.0 * u));
    return (x + y) * 52.5 / denom;
  }
  return (y - x) / std::log(xi);
}

// ---------------------------------------------------------------------------
// Two-point volume fluxes.
// include/ChandrashekarFlux.hpp:20-89
static void vol_chandrashekar(const Gas &g, const double *q1, const double *q2,
                              const double *m1, const double *m2, double *F) {
  const int dim = g.dim;
  double met[3] = {0, 0, 0};
  for (int d = 0; d < dim; ++d) met[d] = 0.5 * (m1[d] + m2[d]);
  const double rho1 = q1[0], rho2 = q2[0];
  const double rho_ln = log_mean(rho1, rho2);
  double mom_hat[3] = {0, 0, 0};
  double h_hat = 0.0, vn = 0.0;
  for (int d = 0; d < dim; ++d) {
    const double v1 = vel(q1, d), v2 = vel(q2, d);
    const double vbar = 0.5 * (v1 + v2);
    vn += vbar * met[d];
    mom_hat[d] = rho_ln * vbar;
    h_hat += -0.25 * (v1 * v1 + v2 * v2) + vbar * vbar;
  }
  const double p1 = pressure(g, q1), p2 = pressure(g, q2);
  const double beta1 = 0.5 * rho1 / p1, beta2 = 0.5 * rho2 / p2;
  const double beta_ln = log_mean(beta1, beta2);
  const double p_hat = 0.5 * (rho1 + rho2) / (beta1 + beta2);
  const double gm1_av_inv = 2.0 / (g.gamma + g.gamma - 2.0);
  h_hat += 0.5 / beta_ln * gm1_av_inv + p_hat / rho_ln;
  F[0] = rho_ln * vn;
  for (int d = 0; d < dim; ++d) F[1 + d] = vn * mom_hat[d] + p_hat * met[d];
  F[dim + 1] = rho_ln * vn * h_hat;
}

// include/RanochaFlux.hpp:20-79
static void vol_ranocha(const Gas &g, const double *q1, const double *q2,
                        const double *m1, const double *m2, double *F) {
  const int dim = g.dim;
  double met[3] = {0, 0, 0};
  for (int d = 0; d < dim; ++d) met[d] = 0.5 * (m1[d] + m2[d]);
  const double rho1 = q1[0], rho2 = q2[0];
  const double rho_ln = log_mean(rho1, rho2);
  double vbar[3] = {0, 0, 0}, ppm[3] = {0, 0, 0};
  double ke = 0.0, vn = 0.0;
  const double p1 = pressure(g, q1), p2 = pressure(g, q2);
  const double pbar = 0.5 * (p1 + p2);
  for (int d = 0; d < dim; ++d) {
    const double v1 = vel(q1, d), v2 = vel(q2, d);
    vbar[d] = 0.5 * (v1 + v2);
    vn += vbar[d] * met[d];
    ke += 0.5 * (v1 * v2);
    ppm[d] = 0.5 * (p1 * v2 + p2 * v1);
  }
  const double inv_beta_ln = (p1 * p2) / log_mean(rho1 * p2, rho2 * p1);
  const double inv_gm1 = 1.0 / (g.gamma - 1.0);
  const double ie = inv_beta_ln * inv_gm1;
  F[0] = rho_ln * vn;
  double fe = 0.0;
  for (int d = 0; d < dim; ++d) {
    F[1 + d] = rho_ln * vn * vbar[d] + pbar * met[d];
    fe += ppm[d] * met[d];
  }
  fe += rho_ln * (ie + ke) * vn;
  F[dim + 1] = fe;
}

// include/PirozzoliFlux.hpp:19-71
static void vol_pirozzoli(const Gas &g, const double *q1, const double *q2,
                          const double *m1, const double *m2, double *F) {
  const int dim = g.dim;
  double met[3] = {0, 0, 0};
  for (int d = 0; d < dim; ++d) met[d] = 0.5 * (m1[d] + m2[d]);
  const double rho1 = q1[0], rho2 = q2[0];
  const double rho_mean = 0.5 * (rho1 + rho2);
  double vbar[3] = {0, 0, 0};
  double ke_mean = 0.0, vn = 0.0;
  const double p1 = pressure(g, q1), p2 = pressure(g, q2);
  const double pbar = 0.5 * (p1 + p2);
  for (int d = 0; d < dim; ++d) {
    const double v1 = vel(q1, d), v2 = vel(q2, d);
    vbar[d] = 0.5 * (v1 + v2);
    vn += vbar[d] * met[d];
    ke_mean += 0.25 * ((v1 * v1) + (v2 * v2));
  }
  const double h_mean = 0.5 * (spec_internal_energy(g, q1) + p1 / rho1 +
                               spec_internal_energy(g, q2) + p2 / rho2);
  F[0] = rho_mean * vn;
  for (int d = 0; d < dim; ++d) F[1 + d] = rho_mean * vn * vbar[d] + pbar * met[d];
  F[dim + 1] = rho_mean * (h_mean + ke_mean) * vn;
}

// Physical Euler flux tensor: include/NavierStokesFlux.hpp:110-158
static void inviscid_flux(const Gas &g, const double *q, double f[MAXEQ][MAXDIM]) {
  const int dim = g.dim;
  const double spec_vol = 1.0 / q[0];
  const double energy = q[dim + 1];
  const double p = pressure(g, q);
  const double H = (energy + p) * spec_vol;
  for (int d = 0; d < dim; ++d) {
    f[0][d] = q[1 + d];
    for (int i = 0; i < dim; ++i) f[1 + i][d] = q[1 + i] * q[1 + d] * spec_vol;
    f[1 + d][d] += p;
    f[dim + 1][d] = q[1 + d] * H;
  }
}

// Central volume flux of HLL/LLF/Roe: include/HLLFlux.hpp:21-51,
// include/LaxFriedrichsFlux.hpp:156-186, include/RoeFlux.hpp:12-37
static void vol_central(const Gas &g, const double *q1, const double *q2,
                        const double *m1, const double *m2, double *F) {
  const int dim = g.dim;
  double met[3] = {0, 0, 0};
  for (int d = 0; d < dim; ++d) met[d] = 0.5 * (m1[d] + m2[d]);
  double f1[MAXEQ][MAXDIM], f2[MAXEQ][MAXDIM];
  inviscid_flux(g, q1, f1);
  inviscid_flux(g, q2, f2);
  for (int e = 0; e < dim + 2; ++e) {
    double acc = 0.0;
    for (int d = 0; d < dim; ++d) acc += 0.5 * (f1[e][d] + f2[e][d]) * met[d];
    F[e] = acc;
  }
}

// ---------------------------------------------------------------------------
// Normal Euler flux by equation: include/NavierStokesFlux.hpp:43-103
struct NState { const double *q; double inv_rho, p, H; };
static inline NState nstate(const Gas &g, const double *q) {
  NState s;
  s.q = q;
  s.inv_rho = 1.0 / q[0];
  s.p = pressure(g, q);
  s.H = (q[g.dim + 1] + s.p) * s.inv_rho;
  return s;
}
static inline double normal_flux(const Gas &g, const NState &s, const double *n, int eq) {
  double r = 0.0;
  for (int dir = 0; dir < g.dim; ++dir) {
    const double m = s.q[1 + dir];
    double pf;
    if (eq == 0) pf = m;
    else if (eq <= g.dim) {
      const int c = eq - 1;
      pf = s.q[1 + c] * m * s.inv_rho;
      if (c == dir) pf += s.p;
    } else pf = m * s.H;
    r += pf * n[dir];
  }
  return r;
}
// include/NavierStokesFlux.hpp:16-41
static inline double max_normal_speed(const Gas &g, const double *q1, const double *q2,
                                      const double *n) {
  double vn1 = 0, vn2 = 0, nn = 0;
  for (int d = 0; d < g.dim; ++d) {
    vn1 += vel(q1, d) * n[d];
    vn2 += vel(q2, d) * n[d];
    nn += n[d] * n[d];
  }
  const double nm = std::sqrt(nn);
  return std::max(std::fabs(vn1) + sound_speed(g, q1) * nm,
                  std::fabs(vn2) + sound_speed(g, q2) * nm);
}

// include/DissipationOperator.hpp:57-172 (Roe dissipation with Harten-Hyman fix)
static void roe_dissipation(const Gas &g, const double *q1, const double *q2,
                            const double *n, double *diss) {
  const int dim = g.dim, E = dim + 1;
  double vn1 = 0, vn2 = 0, vn_roe = 0, nor_mag = 0;
  const double rho1 = q1[0], rho2 = q2[0];
  const double H1 = (q1[E] + pressure(g, q1)) / rho1;
  const double H2 = (q2[E] + pressure(g, q2)) / rho2;
  double roe[MAXEQ] = {0, 0, 0, 0, 0};
  const double ratio = std::sqrt(rho2 / rho1);
  const double a = 1.0 / (ratio + 1.0);
  const double b = a * ratio;
  roe[0] = ratio * rho1;
  roe[E] = a * H1 + b * H2;
  double del_mom[3] = {0, 0, 0};
  double ke = 0.0;
  for (int d = 0; d < dim; ++d) {
    nor_mag += n[d] * n[d];
    const double v1 = vel(q1, d), v2 = vel(q2, d);
    del_mom[d] = v2 - v1;
    roe[1 + d] = a * v1 + b * v2;
    ke += 0.5 * roe[1 + d] * roe[1 + d];
    vn1 += v1 * n[d];
    vn2 += v2 * n[d];
    vn_roe += roe[1 + d] * n[d];
  }
  nor_mag = std::sqrt(nor_mag);
  const double inv_nor_mag = 1.0 / nor_mag;
  vn1 *= inv_nor_mag;
  vn2 *= inv_nor_mag;
  vn_roe *= inv_nor_mag;
  const double c_roe = std::sqrt((g.gamma - 1) * (roe[E] - ke));
  double eig[3] = {0.0, std::fabs(vn_roe), 0.0};
  const double c1 = sound_speed(g, q1), c2 = sound_speed(g, q2);
  {
    const double er = vn_roe - c_roe;
    const double eps = std::max(0.0, std::max(er - (vn1 - c1), (vn2 - c2) - er));
    eig[0] = (std::fabs(er) < eps) ? 0.5 * (eps + (er * er) / eps) : std::fabs(er);
  }
  {
    const double er = vn_roe + c_roe;
    const double eps = std::max(0.0, std::max(er - (vn1 + c1), (vn2 + c2) - er));
    eig[2] = (std::fabs(er) < eps) ? 0.5 * (eps + (er * er) / eps) : std::fabs(er);
  }
  const double del_rho = rho2 - rho1;
  const double del_vn = vn2 - vn1;
  const double del_p = pressure(g, q2) - pressure(g, q1);
  const double ov_csq = 1.0 / (c_roe * c_roe);
  const double pov_csq = del_p * ov_csq;
  const double rhoc_del_vn = roe[0] * del_vn * c_roe * ov_csq;
  const double alpha_Vn = eig[1] * (del_rho - pov_csq);
  const double alpha_Vn_rho = eig[1] * roe[0];
  const double alpha_left = 0.5 * (eig[0] * (pov_csq - rhoc_del_vn));
  const double alpha_right = 0.5 * (eig[2] * (pov_csq + rhoc_del_vn));
  diss[0] = 0.5 * (alpha_Vn + alpha_left + alpha_right);
  double de = 0.0;
  for (int d = 0; d < dim; ++d) {
    double dm = 0.5 * (alpha_Vn * roe[1 + d] +
                       alpha_Vn_rho * (del_mom[d] - n[d] * inv_nor_mag * del_vn));
    dm += 0.5 * (alpha_left * (roe[1 + d] - n[d] * inv_nor_mag * c_roe) +
                 alpha_right * (roe[1 + d] + n[d] * inv_nor_mag * c_roe));
    diss[1 + d] = dm;
    de += 0.5 * alpha_Vn_rho * (roe[1 + d] * del_mom[d]);
  }
  de -= 0.5 * alpha_Vn_rho * vn_roe * del_vn;
  de += 0.5 * alpha_Vn * ke + 0.5 * alpha_left * (roe[E] - vn_roe * c_roe) +
        0.5 * alpha_right * (roe[E] + vn_roe * c_roe);
  diss[E] = de;
  for (int e = 0; e < dim + 2; ++e) diss[e] *= nor_mag;
}

// include/DissipationOperator.hpp:174-232
static void scalar_dissipation(const Gas &g, const double *q1, const double *q2,
                               const double *n, double *diss) {
  const int dim = g.dim, E = dim + 1;
  const double rho1 = q1[0], rho2 = q2[0];
  const double rho_mean = 0.5 * (rho1 + rho2);
  const double drho = rho2 - rho1;
  const double p1 = pressure(g, q1), p2 = pressure(g, q2);
  double vn1 = 0, vn2 = 0, nor_mag = 0, de = 0.0;
  for (int d = 0; d < dim; ++d) {
    nor_mag += n[d] * n[d];
    const double v1 = vel(q1, d), v2 = vel(q2, d);
    const double dv = v2 - v1;
    const double vbar = 0.5 * (v1 + v2);
    vn1 += v1 * n[d];
    vn2 += v2 * n[d];
    de += 0.5 * drho * v1 * v2 + rho_mean * dv * vbar;
  }
  nor_mag = std::sqrt(nor_mag);
  const double lambda_max = std::max(std::fabs(vn1) + sound_speed(g, q1) * nor_mag,
                                     std::fabs(vn2) + sound_speed(g, q2) * nor_mag);
  const double gm1_av_inv = 1.0 / (g.gamma - 1.0);
  const double beta1 = 0.5 * rho1 / p1, beta2 = 0.5 * rho2 / p2;
  const double beta_ln = log_mean(beta1, beta2);
  de += 0.5 * drho * gm1_av_inv / beta_ln +
        0.5 * rho_mean * gm1_av_inv * (1.0 / beta2 - 1.0 / beta1);
  diss[0] = 0.5 * lambda_max * drho;
  for (int d = 0; d < dim; ++d) diss[1 + d] = 0.5 * lambda_max * (q2[1 + d] - q1[1 + d]);
  diss[E] = de * (0.5 * lambda_max);
}

// ---------------------------------------------------------------------------
// Surface fluxes.
// include/ChandrashekarFlux.hpp:91-155
static void face_chandrashekar(const Gas &g, const double *q1, const double *q2,
                               const double *n, double *F) {
  const int dim = g.dim, E = dim + 1;
  const double rho1 = q1[0], rho2 = q2[0];
  const double rho_ln = log_mean(rho1, rho2);
  double mom[3] = {0, 0, 0};
  double hhat = 0.0, vn = 0.0;
  double diss[MAXEQ] = {0, 0, 0, 0, 0};
  for (int d = 0; d < dim; ++d) {
    const double v1 = vel(q1, d), v2 = vel(q2, d);
    const double vbar = 0.5 * (v1 + v2);
    vn += vbar * n[d];
    mom[d] = rho_ln * vbar;
    hhat += -0.25 * (v1 * v1 + v2 * v2) + vbar * vbar;
  }
  const double p1 = pressure(g, q1), p2 = pressure(g, q2);
  const double beta1 = 0.5 * rho1 / p1, beta2 = 0.5 * rho2 / p2;
  const double beta_ln = log_mean(beta1, beta2);
  const double p_hat = 0.5 * (rho1 + rho2) / (beta1 + beta2);
  const double gm1_av_inv = 2.0 / (g.gamma + g.gamma - 2.0);
  hhat += 0.5 / beta_ln * gm1_av_inv + p_hat / rho_ln;
  scalar_dissipation(g, q1, q2, n, diss);
  F[0] = rho_ln * vn - diss[0];
  for (int d = 0; d < dim; ++d) F[1 + d] = vn * mom[d] + p_hat * n[d] - diss[1 + d];
  F[E] = rho_ln * vn * hhat - diss[E];
}

// include/RanochaFlux.hpp:81-134
static void face_ranocha(const Gas &g, const double *q1, const double *q2,
                         const double *n, double *F) {
  const int dim = g.dim, E = dim + 1;
  const double rho1 = q1[0], rho2 = q2[0];
  const double rho_ln = log_mean(rho1, rho2);
  double vbar[3] = {0, 0, 0}, ppm[3] = {0, 0, 0};
  double diss[MAXEQ] = {0, 0, 0, 0, 0};
  double ke = 0.0, vn = 0.0;
  const double p1 = pressure(g, q1), p2 = pressure(g, q2);
  const double pbar = 0.5 * (p1 + p2);
  for (int d = 0; d < dim; ++d) {
    const double v1 = vel(q1, d), v2 = vel(q2, d);
    vbar[d] = 0.5 * (v1 + v2);
    vn += vbar[d] * n[d];
    ke += 0.5 * (v1 * v2);
    ppm[d] = 0.5 * (p1 * v2 + p2 * v1);
  }
  const double inv_beta_ln = (p1 * p2) / log_mean(rho1 * p2, rho2 * p1);
  const double inv_gm1 = 1.0 / (g.gamma - 1.0);
  const double ie = inv_beta_ln * inv_gm1;
  roe_dissipation(g, q1, q2, n, diss);
  F[0] = rho_ln * vn - diss[0];
  double fe = 0.0;
  for (int d = 0; d < dim; ++d) {
    F[1 + d] = rho_ln * vn * vbar[d] + pbar * n[d] - diss[1 + d];
    fe += ppm[d] * n[d];
  }
  fe += rho_ln * (ie + ke) * vn - diss[E];
  F[E] = fe;
}

// include/PirozzoliFlux.hpp:73-120
static void face_pirozzoli(const Gas &g, const double *q1, const double *q2,
                           const double *n, double *F) {
  const int dim = g.dim, E = dim + 1;
  const double rho1 = q1[0], rho2 = q2[0];
  const double rho_mean = 0.5 * (rho1 + rho2);
  double vbar[3] = {0, 0, 0};
  double diss[MAXEQ] = {0, 0, 0, 0, 0};
  double ke_mean = 0.0, vn = 0.0;
  const double p1 = pressure(g, q1), p2 = pressure(g, q2);
  const double pbar = 0.5 * (p1 + p2);
  for (int d = 0; d < dim; ++d) {
    const double v1 = vel(q1, d), v2 = vel(q2, d);
    vbar[d] = 0.5 * (v1 + v2);
    vn += vbar[d] * n[d];
    ke_mean += 0.25 * ((v1 * v1) + (v2 * v2));
  }
  const double h_mean = 0.5 * (spec_internal_energy(g, q1) + p1 / rho1 +
                               spec_internal_energy(g, q2) + p2 / rho2);
  roe_dissipation(g, q1, q2, n, diss);
  F[0] = rho_mean * vn - diss[0];
  for (int d = 0; d < dim; ++d) F[1 + d] = rho_mean * vn * vbar[d] + pbar * n[d] - diss[1 + d];
  F[E] = 0.0 + (rho_mean * (h_mean + ke_mean) * vn - diss[E]);
}

// include/HLLFlux.hpp:53-116
static void face_hll(const Gas &g, const double *q1, const double *q2,
                     const double *n, double *F) {
  const int dim = g.dim;
  const NState L = nstate(g, q1), R = nstate(g, q2);
  double un1 = 0, un2 = 0, nn = 0;
  for (int d = 0; d < dim; ++d) {
    un1 += vel(q1, d) * n[d];
    un2 += vel(q2, d) * n[d];
    nn += n[d] * n[d];
  }
  const double nm = std::sqrt(nn);
  const double c1 = sound_speed(g, q1) * nm, c2 = sound_speed(g, q2) * nm;
  const double sL1 = un1 - c1, sL2 = un2 - c2, sR1 = un1 + c1, sR2 = un2 + c2;
  const double sL = (sL1 < sL2) ? sL1 : sL2;
  const double sR = (sR1 > sR2) ? sR1 : sR2;
  for (int e = 0; e < dim + 2; ++e) {
    const double fn1 = normal_flux(g, L, n, e), fn2 = normal_flux(g, R, n, e);
    if (sL >= 0.0) F[e] = fn1;
    else if (sR <= 0.0) F[e] = fn2;
    else F[e] = (sR * fn1 - sL * fn2 + sL * sR * (q2[e] - q1[e])) / (sR - sL);
  }
}

// include/LaxFriedrichsFlux.hpp:188-211
static void face_llf(const Gas &g, const double *q1, const double *q2,
                     const double *n, double *F) {
  const NState L = nstate(g, q1), R = nstate(g, q2);
  const double lmax = max_normal_speed(g, q1, q2, n);
  for (int e = 0; e < g.dim + 2; ++e) {
    const double nl = normal_flux(g, L, n, e), nr = normal_flux(g, R, n, e);
    F[e] = 0.5 * (nl + nr) - 0.5 * lmax * (q2[e] - q1[e]);
  }
}

// include/RoeFlux.hpp:42-149
static void face_roe(const Gas &g, const double *qL, const double *qR,
                     const double *n, double *F) {
  const int dim = g.dim, E = dim + 1;
  const NState left = nstate(g, qL), right = nstate(g, qR);
  double nm2 = 0.0;
  for (int d = 0; d < dim; ++d) nm2 += n[d] * n[d];
  const double nm = std::sqrt(nm2);
  const double inv_nm = 1.0 / nm;
  const double rhoL = qL[0], rhoR = qR[0];
  const double pL = left.p, pR = right.p;
  const double rootL = std::sqrt(rhoL), rootR = std::sqrt(rhoR);
  const double rsi = 1.0 / (rootL + rootR);
  const double rho_roe = rootL * rootR;
  const double HL = (qL[E] + pL) / rhoL, HR = (qR[E] + pR) / rhoR;
  const double H = (rootL * HL + rootR * HR) * rsi;
  double u[3] = {0, 0, 0}, du[3] = {0, 0, 0}, du_t[3] = {0, 0, 0}, nh[3] = {0, 0, 0};
  double u2 = 0, un = 0, dun = 0;
  for (int d = 0; d < dim; ++d) {
    const double uL = vel(qL, d), uR = vel(qR, d);
    nh[d] = n[d] * inv_nm;
    u[d] = (rootL * uL + rootR * uR) * rsi;
    du[d] = uR - uL;
    u2 += u[d] * u[d];
    un += u[d] * nh[d];
    dun += du[d] * nh[d];
  }
  const double gamma = g.gamma;
  const double a2 = (gamma - 1.0) * (H - 0.5 * u2);
  const double a = std::sqrt(a2);
  const double dp = pR - pL, drho = rhoR - rhoL;
  const double am = 0.5 * (dp - rho_roe * a * dun) / a2;
  const double ap = 0.5 * (dp + rho_roe * a * dun) / a2;
  const double az = drho - dp / a2;
  const double lm = std::fabs(un - a) * nm;
  const double lz = std::fabs(un) * nm;
  const double lp = std::fabs(un + a) * nm;
  for (int d = 0; d < dim; ++d) du_t[d] = du[d] - dun * nh[d];
  const double dmass = lm * am + lz * az + lp * ap;
  double diss[MAXEQ] = {0, 0, 0, 0, 0};
  diss[0] = dmass;
  for (int d = 0; d < dim; ++d)
    diss[1 + d] = lm * am * (u[d] - a * nh[d]) + lz * (az * u[d] + rho_roe * du_t[d]) +
                  lp * ap * (u[d] + a * nh[d]);
  double udt = 0.0;
  for (int d = 0; d < dim; ++d) udt += u[d] * du_t[d];
  diss[E] = lm * am * (H - a * un) + lz * (0.5 * az * u2 + rho_roe * udt) + lp * ap * (H + a * un);
  for (int e = 0; e < dim + 2; ++e) {
    const double central = 0.5 * (normal_flux(g, left, n, e) + normal_flux(g, right, n, e));
    F[e] = central - 0.5 * diss[e];
  }
}

typedef void (*VolFn)(const Gas &, const double *, const double *, const double *,
                      const double *, double *);
typedef void (*FaceFn)(const Gas &, const double *, const double *, const double *, double *);

// LTEEC (include/LTEECFlux.hpp:86-99): volume form with the averaged metric,
// face form with the Lax dissipation; needs the LTE Helmholtz gas.
static void vol_lteec(const Gas &g, const double *q1, const double *q2, const double *m1,
                      const double *m2, double *F) {
  bool bad = false;
  lte::lteec(*g.lte, g.dim, false, q1, q2, m1, m2, F, &bad);
  if (bad && g.bad) g.bad->fetch_add(1);
}
static void face_lteec(const Gas &g, const double *q1, const double *q2, const double *n,
                       double *F) {
  bool bad = false;
  lte::lteec(*g.lte, g.dim, true, q1, q2, n, n, F, &bad);
  if (bad && g.bad) g.bad->fetch_add(1);
}

static VolFn vol_fn(int f) {
  switch (f) {
    case THX_FLUX_LTEEC: return vol_lteec;
    case THX_FLUX_CHANDRASHEKAR: return vol_chandrashekar;
    case THX_FLUX_RANOCHA: return vol_ranocha;
    case THX_FLUX_PIROZZOLI: return vol_pirozzoli;
    case THX_FLUX_HLL: case THX_FLUX_LLF: case THX_FLUX_ROE: return vol_central;
  }
  return nullptr;
}
static FaceFn face_fn(int f) {
  switch (f) {
    case THX_FLUX_LTEEC: return face_lteec;
    case THX_FLUX_CHANDRASHEKAR: return face_chandrashekar;
    case THX_FLUX_RANOCHA: return face_ranocha;
    case THX_FLUX_PIROZZOLI: return face_pirozzoli;
    case THX_FLUX_HLL: return face_hll;
    case THX_FLUX_LLF: return face_llf;
    case THX_FLUX_ROE: return face_roe;
  }
  return nullptr;
}

// include/NavierStokesFlux.hpp:160-290 (Cartesian, no axisymmetric source)
static void viscous_flux(const Gas &g, const double *q, const double *const dprim[3],
                         double vf[MAXEQ][MAXDIM]) {
  const int dim = g.dim, E = dim + 1;
  for (int e = 0; e < MAXEQ; ++e)
    for (int d = 0; d < dim; ++d) vf[e][d] = 0.0;
  const double mu = viscosity(g, q);
  const double kappa = conductivity(g, q);
  const double mub = g.mu_bulk;
  double grho[3] = {0, 0, 0}, gp[3] = {0, 0, 0}, gT[3] = {0, 0, 0};
  for (int d = 0; d < dim; ++d) {
    grho[d] = dprim[d][0];
    gp[d] = dprim[d][E];
  }
  grad_temperature(g, q, grho, gp, gT);
  double v[3] = {0, 0, 0};
  double div = 0.0;
  for (int i = 0; i < dim; ++i) {
    v[i] = vel(q, i);
    div += dprim[i][1 + i];
  }
  for (int dir = 0; dir < dim; ++dir) {
    const double *dg = dprim[dir];
    for (int mom = 0; mom < dim; ++mom) {
      double tau;
      if (mom == dir) tau = mu * (2.0 * dg[1 + mom] - mub * div);
      else tau = mu * (dg[1 + mom] + dprim[mom][1 + dir]);
      vf[1 + mom][dir] = tau;
    }
    double ef = kappa * gT[dir];
    for (int mom = 0; mom < dim; ++mom) ef += v[mom] * vf[1 + mom][dir];
    vf[E][dir] = ef;
  }
}

// ---------------------------------------------------------------------------
// LGL rule on [0,1]: nodes are the endpoints and the roots of P'_{n-1}
// (Newton iteration on the Legendre recurrence), weights 2/(n(n-1)P_{n-1}^2)
// mapped to the unit interval.
static void lgl(int np, double *x, double *w) {
  const int N = np - 1;
  for (int i = 0; i < np; ++i) {
    double z = -std::cos(M_PI * i / N);
    for (int it = 0; it < 100; ++it) {
      double p0 = 1.0, p1 = z;
      for (int k = 2; k <= N; ++k) {
        const double p2 = ((2.0 * k - 1.0) * z * p1 - (k - 1.0) * p0) / k;
        p0 = p1;
        p1 = p2;
      }
      // p1 = P_N(z), p0 = P_{N-1}(z)
      const double dz = (z * p1 - p0) / (np * p1);
      z -= dz;
      if (std::fabs(dz) < 1e-16) break;
    }
    double p0 = 1.0, p1 = z;
    for (int k = 2; k <= N; ++k) {
      const double p2 = ((2.0 * k - 1.0) * z * p1 - (k - 1.0) * p0) / k;
      p0 = p1;
      p1 = p2;
    }
    x[i] = 0.5 * (z + 1.0);
    w[i] = 1.0 / (N * np * p1 * p1);
  }
  if (np > 1) { x[0] = 0.0; x[np - 1] = 1.0; }
}

// Shifted Legendre P_n(2x-1), n = 0..order (MFEM Poly_1D::CalcLegendre as used
// by src/ModalBasis.cpp:115-140).
static void shifted_legendre(int order, double x, double *L) {
  const double z = 2.0 * x - 1.0;
  L[0] = 1.0;
  if (order >= 1) L[1] = z;
  for (int n = 1; n < order; ++n) L[n + 1] = ((2.0 * n + 1.0) * z * L[n] - n * L[n - 1]) / (n + 1.0);
}

// Gauss-Jordan inverse with partial pivoting (dense, row-major).
static bool invert(int n, std::vector<double> &A) {
  std::vector<double> I(n * n, 0.0);
  for (int i = 0; i < n; ++i) I[i * n + i] = 1.0;
  for (int c = 0; c < n; ++c) {
    int piv = c;
    for (int r = c + 1; r < n; ++r)
      if (std::fabs(A[r * n + c]) > std::fabs(A[piv * n + c])) piv = r;
    if (A[piv * n + c] == 0.0) return false;
    if (piv != c)
      for (int k = 0; k < n; ++k) { std::swap(A[c * n + k], A[piv * n + k]); std::swap(I[c * n + k], I[piv * n + k]); }
    const double inv = 1.0 / A[c * n + c];
    for (int k = 0; k < n; ++k) { A[c * n + k] *= inv; I[c * n + k] *= inv; }
    for (int r = 0; r < n; ++r) {
      if (r == c) continue;
      const double f = A[r * n + c];
      if (f == 0.0) continue;
      for (int k = 0; k < n; ++k) { A[r * n + k] -= f * A[c * n + k]; I[r * n + k] -= f * I[c * n + k]; }
    }
  }
  A.swap(I);
  return true;
}

// ---------------------------------------------------------------------------
// Discretisation: operators on [0,1] (include/dgsem_cache_utilities.hpp:123-181).
struct Disc {
  int dim, p, Np, Nx, Ny, Nz, nd, nfp, neq, ne, nf;
  std::vector<double> x, w, D, Dhat, Dhat2;  // D[i*Np+l] = l'_l(x_i)
  std::vector<double> modal;                // [m][q] = Vinv(m,q)
  std::vector<double> keep1, keep2;
  const thx_geometry *geom;
  Gas gas;
  thx_config cfg;
  // elem -> (face, side) per local face; -1 if none
  std::vector<int> elem_face;
  std::vector<double> sub_xi, sub_eta, sub_zeta;  // subcell metrics
  double threshold;
};

static int trace_node(const Disc &c, int lf, int fp) {
  const int N = c.Np;
  const int dir = lf / 2;
  const int pos = (lf % 2) ? N - 1 : 0;
  if (c.dim == 2) {
    return dir == 0 ? pos + N * fp : fp + N * pos;
  }
  const int a = fp % N, b = fp / N;
  if (dir == 0) return pos + N * (a + N * b);
  if (dir == 1) return a + N * (pos + N * b);
  return a + N * (b + N * pos);
}

static int setup(Disc &c, const thx_geometry *g, const thx_config *cfg) {
  if (!g || !cfg) return THX_ERR_INVALID_ARGUMENT;
  if (g->dim < 2 || g->dim > 3 || g->order < 1 || g->order > 8) return THX_ERR_UNSUPPORTED;
  c.geom = g;
  c.cfg = *cfg;
  c.dim = g->dim;
  c.p = g->order;
  c.Np = c.p + 1;
  c.Nx = c.Np;
  c.Ny = c.Np;
  c.Nz = c.dim > 2 ? c.Np : 1;
  c.nd = c.Nx * c.Ny * c.Nz;
  c.nfp = c.dim == 2 ? c.Np : c.Np * c.Np;
  c.neq = c.dim + 2;
  c.ne = g->num_elements;
  c.nf = g->num_faces;
  c.gas = make_gas(*cfg, c.dim);
  const int N = c.Np;
  c.x.resize(N);
  c.w.resize(N);
  lgl(N, c.x.data(), c.w.data());
  // barycentric weights and D (include/dgsem_cache_utilities.hpp:129-153)
  std::vector<double> wb(N, 1.0);
  for (int i = 1; i < N; ++i)
    for (int j = 0; j < i; ++j) {
      wb[j] *= (c.x[j] - c.x[i]);
      wb[i] *= (c.x[i] - c.x[j]);
    }
  for (int i = 0; i < N; ++i) wb[i] = 1.0 / wb[i];
  c.D.assign(N * N, 0.0);
  for (int l = 0; l < N; ++l)
    for (int i = 0; i < N; ++i)
      if (l != i) {
        c.D[i * N + l] = wb[l] / wb[i] / (c.x[i] - c.x[l]);
        c.D[i * N + i] -= c.D[i * N + l];
      }
  // Dhat(i,l) = D(i,l) with boundary terms (weak-form derivative), Dhat2 = 2D + boundary
  c.Dhat = c.D;
  c.Dhat[0] += 1.0 / c.w[0];
  c.Dhat[N * N - 1] -= 1.0 / c.w[N - 1];
  c.Dhat2.resize(N * N);
  for (int k = 0; k < N * N; ++k) c.Dhat2[k] = 2.0 * c.D[k];
  c.Dhat2[0] += 1.0 / c.w[0];
  c.Dhat2[N * N - 1] -= 1.0 / c.w[N - 1];
  // element -> face table
  c.elem_face.assign(c.ne * 2 * c.dim, -1);
  for (int f = 0; f < c.nf; ++f)
    for (int s = 0; s < 2; ++s) {
      const int e = g->face_elem[2 * f + s];
      const int lf = g->face_lface[2 * f + s];
      if (e < 0 || e >= c.ne || lf < 0 || lf >= 2 * c.dim) return THX_ERR_INVALID_ARGUMENT;
      c.elem_face[e * 2 * c.dim + lf] = 2 * f + s;
    }
  c.threshold = cfg->modal_threshold > 0 ? cfg->modal_threshold
                                         : 0.5 * std::pow(10.0, -1.8 * std::pow((double)c.p, 0.25));
  if (cfg->blending) {
    // Persson modal transform (src/ModalBasis.cpp:42-140;
    // include/dgsem_cache_utilities.hpp:867-943)
    const int nd = c.nd;
    std::vector<int> degs(nd * 3, 0);
    {
      int n = 0;
      if (c.dim == 2) {
        for (int i = 0; i < N; ++i)
          for (int j = 0; j < N; ++j) { degs[n * 3] = i; degs[n * 3 + 1] = j; ++n; }
      } else {
        for (int i = 0; i < N; ++i)
          for (int j = 0; j < N; ++j)
            for (int k = 0; k < N; ++k) { degs[n * 3] = i; degs[n * 3 + 1] = j; degs[n * 3 + 2] = k; ++n; }
      }
    }
    std::vector<double> V(nd * nd), L(N);
    for (int i = 0; i < nd; ++i) {
      const int ix[3] = {i % N, (i / N) % N, i / (N * N)};
      for (int j = 0; j < c.dim; ++j) {
        shifted_legendre(c.p, c.x[ix[j]], L.data());
        for (int k = 0; k < nd; ++k) {
          const double v = L[degs[k * 3 + j]];
          V[i * nd + k] = (j == 0) ? v : V[i * nd + k] * v;
        }
      }
    }
    if (!invert(nd, V)) return THX_ERR_NUMERICS;
    c.modal = V;  // modal[m*nd + q] = Vinv(m,q)
    c.keep1.resize(nd);
    c.keep2.resize(nd);
    for (int m = 0; m < nd; ++m) {
      bool k1 = true, k2 = true;
      for (int d = 0; d < c.dim; ++d) {
        if (degs[m * 3 + d] > c.p - 2) k2 = false;
        if (degs[m * 3 + d] > c.p - 1) k1 = false;
      }
      c.keep1[m] = k1 ? 1.0 : 0.0;
      c.keep2[m] = k2 ? 1.0 : 0.0;
    }
    // subcell metrics (include/dgsem_cache_utilities.hpp:641-763)
    const int dim = c.dim, Nx = c.Nx, Ny = c.Ny, Nz = c.Nz;
    const int nxi = (Nx + 1) * Ny * Nz, neta = Nx * (Ny + 1) * Nz, nzeta = Nx * Ny * (Nz + 1);
    c.sub_xi.assign((size_t)nxi * dim * c.ne, 0.0);
    if (dim > 1) c.sub_eta.assign((size_t)neta * dim * c.ne, 0.0);
    if (dim > 2) c.sub_zeta.assign((size_t)nzeta * dim * c.ne, 0.0);
    const double *metric = g->metric;
    const int nq = nd;
    for (int el = 0; el < c.ne; ++el)
      for (int k = 0; k < Nz; ++k)
        for (int j = 0; j < Ny; ++j)
          for (int i = 1; i < Nx; ++i)
            for (int d = 0; d < dim; ++d) {
              const int line = k * Ny * Nx + j * Nx;
              double nrm = metric[((size_t)(el * nq + line) * dim) * dim + d];
              for (int l = 0; l < i; ++l) {
                double sum = 0.0;
                for (int m = 0; m < Nx; ++m) sum += metric[((size_t)(el * nq + line + m) * dim) * dim + d] * c.D[l * Nx + m];
                sum *= c.w[l];
                nrm += sum;
              }
              c.sub_xi[((size_t)el * nxi + line + i) * dim + d] = nrm;
            }
    if (dim > 1)
      for (int el = 0; el < c.ne; ++el)
        for (int k = 0; k < Nz; ++k)
          for (int i = 0; i < Nx; ++i)
            for (int j = 1; j < Ny; ++j)
              for (int d = 0; d < dim; ++d) {
                const int line = k * Ny * Nx + i;
                double nrm = metric[((size_t)(el * nq + line) * dim + 1) * dim + d];
                for (int l = 0; l < j; ++l) {
                  double sum = 0.0;
                  for (int m = 0; m < Ny; ++m) sum += metric[((size_t)(el * nq + line + m * Nx) * dim + 1) * dim + d] * c.D[l * Nx + m];
                  sum *= c.w[l];
                  nrm += sum;
                }
                c.sub_eta[((size_t)el * neta + k * Ny * Nx + j * Nx + i) * dim + d] = nrm;
              }
    if (dim > 2)
      for (int el = 0; el < c.ne; ++el)
        for (int j = 0; j < Ny; ++j)
          for (int i = 0; i < Nx; ++i)
            for (int k = 1; k < Nz; ++k)
              for (int d = 0; d < dim; ++d) {
                const int line = j * Nx + i;
                double nrm = metric[((size_t)(el * nq + line) * dim + 2) * dim + d];
                for (int l = 0; l < k; ++l) {
                  double sum = 0.0;
                  for (int m = 0; m < Nz; ++m) sum += metric[((size_t)(el * nq + line + m * Ny * Nx) * dim + 2) * dim + d] * c.D[l * Nx + m];
                  sum *= c.w[l];
                  nrm += sum;
                }
                c.sub_zeta[((size_t)el * nzeta + k * Ny * Nx + line) * dim + d] = nrm;
              }
  }
  return THX_OK;
}

// Gather element state [eq][node] from the byNODES L-vector.
static inline void gather_elem(const Disc &c, const double *u, int e, double *ue) {
  const size_t stride = (size_t)c.ne * c.nd;
  for (int q = 0; q < c.neq; ++q)
    std::memcpy(ue + q * c.nd, u + q * stride + (size_t)e * c.nd, sizeof(double) * c.nd);
}

// Persson-Peraire indicator and blending coefficient
// (include/RHSOperator_impl.hpp:355-527)
static void blending(const Disc &c, const double *u, double *alpha, double *eta, int nthreads) {
  const int nd = c.nd;
#pragma omp parallel for num_threads(nthreads) schedule(static)
  for (int e = 0; e < c.ne; ++e) {
    std::vector<double> ue(c.neq * nd), field(nd);
    gather_elem(c, u, e, ue.data());
    for (int i = 0; i < nd; ++i) {
      double q[MAXEQ];
      for (int k = 0; k < c.neq; ++k) q[k] = ue[k * nd + i];
      field[i] = pressure(c.gas, q) * q[0];
    }
    double mm = 0, m1 = 0, m2 = 0;
    for (int m = 0; m < nd; ++m) {
      double mode = 0.0;
      for (int q = 0; q < nd; ++q) mode += c.modal[m * nd + q] * field[q];
      const double mode2 = mode * mode;
      mm += mode2;
      m1 += c.keep1[m] * mode2;
      m2 += c.keep2[m] * mode2;
    }
    const double eps = 1.0e-30;
    double val = 0.0;
    if (mm > eps) {
      val = 1.0 - m1 / mm;
      if (m1 > eps) val = std::max(val, 1.0 - m2 / m1);
      else val = 1.0;
    }
    const double et = std::min(std::max(val, 0.0), 1.0);
    if (eta) eta[e] = et;
    const double th = c.threshold;
    double a = 1.0 / (1.0 + std::exp(-c.cfg.sharpness * (et - th) / th));
    if (a < c.cfg.alpha_min) a = 0.0;
    else if (a > (1.0 - c.cfg.alpha_min)) a = 1.0;
    alpha[e] = std::min(a, c.cfg.alpha_max);
  }
}

// Subcell first-order FV (include/DGSEMIntegrator.hpp:338-483)
static void fv_element(const Disc &c, FaceFn ff, const double *ue, const double *jac,
                       const double *mxi, const double *meta, const double *mzeta, double *du) {
  const int dim = c.dim, Nx = c.Nx, Ny = c.Ny, Nz = c.Nz, neq = c.neq, npe = c.nd;
  const double *w = c.w.data();
  double fnum[MAXEQ], dus[MAXEQ], s1[MAXEQ], s2[MAXEQ];
  for (int i = 0; i < npe * neq; ++i) du[i] = 0.0;
  auto gather = [&](int id, double *s) { for (int q = 0; q < neq; ++q) s[q] = ue[q * npe + id]; };
  for (int k = 0; k < Nz; ++k)
    for (int j = 0; j < Ny; ++j) {
      for (int q = 0; q < neq; ++q) dus[q] = 0.0;
      int id1 = k * Ny * Nx + j * Nx;
      gather(id1, s1);
      for (int i = 0; i < Nx - 1; ++i) {
        const int id2 = id1 + 1;
        gather(id2, s2);
        ff(c.gas, s1, s2, mxi + id2 * dim, fnum);
        for (int q = 0; q < neq; ++q) dus[q] -= fnum[q];
        for (int q = 0; q < neq; ++q) dus[q] /= (jac[id1] * w[i]);
        for (int q = 0; q < neq; ++q) du[id1 + q * npe] = dus[q];
        for (int q = 0; q < neq; ++q) { dus[q] = fnum[q]; s1[q] = s2[q]; }
        id1 = id2;
      }
      for (int q = 0; q < neq; ++q) dus[q] /= (jac[id1] * w[Nx - 1]);
      for (int q = 0; q < neq; ++q) du[id1 + q * npe] = dus[q];
    }
  if (dim > 1) {
    for (int k = 0; k < Nz; ++k)
      for (int i = 0; i < Nx; ++i) {
        for (int q = 0; q < neq; ++q) dus[q] = 0.0;
        int id1 = k * Ny * Nx + i;
        gather(id1, s1);
        for (int j = 0; j < Ny - 1; ++j) {
          const int id2 = k * Ny * Nx + (j + 1) * Nx + i;
          gather(id2, s2);
          ff(c.gas, s1, s2, meta + id2 * dim, fnum);
          for (int q = 0; q < neq; ++q) dus[q] -= fnum[q];
          for (int q = 0; q < neq; ++q) dus[q] /= (jac[id1] * w[j]);
          for (int q = 0; q < neq; ++q) du[id1 + q * npe] += dus[q];
          for (int q = 0; q < neq; ++q) { dus[q] = fnum[q]; s1[q] = s2[q]; }
          id1 = id2;
        }
        for (int q = 0; q < neq; ++q) dus[q] /= (jac[id1] * w[Ny - 1]);
        for (int q = 0; q < neq; ++q) du[id1 + q * npe] += dus[q];
      }
    if (dim > 2) {
      for (int j = 0; j < Ny; ++j)
        for (int i = 0; i < Nx; ++i) {
          for (int q = 0; q < neq; ++q) dus[q] = 0.0;
          int id1 = j * Nx + i;
          gather(id1, s1);
          for (int k = 0; k < Nz - 1; ++k) {
            const int id2 = (k + 1) * Ny * Nx + j * Nx + i;
            gather(id2, s2);
            ff(c.gas, s1, s2, mzeta + id2 * dim, fnum);
            for (int q = 0; q < neq; ++q) dus[q] -= fnum[q];
            for (int q = 0; q < neq; ++q) dus[q] /= (jac[id1] * w[k]);
            for (int q = 0; q < neq; ++q) du[id1 + q * npe] += dus[q];
            for (int q = 0; q < neq; ++q) { dus[q] = fnum[q]; s1[q] = s2[q]; }
            id1 = id2;
          }
          for (int q = 0; q < neq; ++q) dus[q] /= (jac[id1] * w[Nz - 1]);
          for (int q = 0; q < neq; ++q) du[id1 + q * npe] += dus[q];
        }
    }
  }
}

// Flux-differencing volume term of one element, point form
// (include/DGSEMIntegrator.hpp:124-218).  du is assigned.
static void volume_element(const Disc &c, VolFn vf, const double *ue, const double *jac,
                           const double *met, double *du) {
  const int dim = c.dim, N = c.Np, nd = c.nd, neq = c.neq;
  const double *Dh2 = c.Dhat2.data();
  double sl[MAXEQ], su[MAXEQ], fl[MAXEQ];
  for (int point = 0; point < nd; ++point) {
    const int i = point % N, j = (point / N) % c.Ny, k = point / (N * c.Ny);
    double rate[MAXEQ] = {0, 0, 0, 0, 0};
    for (int dir = 0; dir < dim; ++dir) {
      const int me = dir == 0 ? i : (dir == 1 ? j : k);
      for (int m = 0; m < N; ++m) {
        if (m == me) continue;
        const int lo = m < me ? m : me, hi = m < me ? me : m;
        int lp, up;
        if (dir == 0) { lp = k * c.Ny * N + j * N + lo; up = k * c.Ny * N + j * N + hi; }
        else if (dir == 1) { lp = k * c.Ny * N + lo * N + i; up = k * c.Ny * N + hi * N + i; }
        else { lp = lo * c.Ny * N + j * N + i; up = hi * c.Ny * N + j * N + i; }
        for (int q = 0; q < neq; ++q) { sl[q] = ue[q * nd + lp]; su[q] = ue[q * nd + up]; }
        vf(c.gas, sl, su, met + lp * dim * dim + dir * dim, met + up * dim * dim + dir * dim, fl);
        const double coef = Dh2[me * N + m];
        for (int q = 0; q < neq; ++q) rate[q] += coef * fl[q];
      }
    }
    const double s = -1.0 / jac[point];
    for (int q = 0; q < neq; ++q) du[point + q * nd] = s * rate[q];
  }
}

// BR1 gradient of entropy variables, then conversion to primitive gradients
// (include/NSOperator_impl.hpp:11-159, include/DGSEMIntegrator.hpp:764-850,1011-1044).
// grad[c][eq][e][node] (byNODES per direction).
// Boundary jump of the entropy variables w for the BR1 lift
// (include/bc_kernels.hpp:32-135, ComputeBdrFaceGradFlux): exterior minus
// interior entropy state; zero for the conditions without one.
static void bc_grad_flux(const Gas &g, const thx_bc &bc, const double *data, const double *w,
                         double *F) {
  const int dim = g.dim, neq = dim + 2;
  for (int q = 0; q < neq; ++q) F[q] = 0.0;
  switch (bc.type) {
    case THX_BC_PRESCRIBED_STATE: {
      double e[MAXEQ];
      entropy_vars(g, data + bc.data_index, e);
      for (int q = 0; q < neq; ++q) F[q] = e[q] - w[q];
      return;
    }
    case THX_BC_NOSLIP_ADIABATIC: {
      const double *vwall = data + bc.data_index;
      const double v = -w[dim + 1];
      F[0] = w[0];
      for (int d = 0; d < dim; ++d) F[1 + d] = vwall[d] * v;
      F[dim + 1] = -v;
      for (int q = 0; q < neq; ++q) F[q] -= w[q];
      return;
    }
    case THX_BC_NOSLIP_ISOTHERMAL: {
      const double *bd = data + bc.data_index;
      const double beta = 1.0 / (g.R * bd[dim]);   // include/EOS.hpp:41-46
      F[0] = w[0];
      for (int d = 0; d < dim; ++d) F[1 + d] = bd[d] * beta;
      F[dim + 1] = -beta;
      for (int q = 0; q < neq; ++q) F[q] -= w[q];
      return;
    }
    default:
      return;
  }
}

static void gradient(const Disc &c, const double *u, double *grad, int nthreads) {
  const int dim = c.dim, N = c.Np, nd = c.nd, neq = c.neq, ne = c.ne;
  const size_t L = (size_t)ne * nd;
  std::vector<double> S((size_t)neq * L);
  // entropy state (L-vector)
#pragma omp parallel for num_threads(nthreads) schedule(static)
  for (long pt = 0; pt < (long)L; ++pt) {
    double q[MAXEQ], w[MAXEQ];
    for (int k = 0; k < neq; ++k) q[k] = u[k * L + pt];
    entropy_vars(c.gas, q, w);
    for (int k = 0; k < neq; ++k) S[k * L + pt] = w[k];
  }
  // volume part
#pragma omp parallel for num_threads(nthreads) schedule(static)
  for (int e = 0; e < ne; ++e) {
    const double *J = c.geom->jac + (size_t)e * nd;
    const double *M = c.geom->metric + (size_t)e * nd * dim * dim;
    for (int point = 0; point < nd; ++point) {
      const int i = point % N, j = (point / N) % c.Ny, k = point / (N * c.Ny);
      double dxi[MAXEQ] = {0}, deta[MAXEQ] = {0}, dzeta[MAXEQ] = {0};
      for (int l = 0; l < N; ++l) {
        const int s = k * c.Ny * N + j * N + l;
        const double co = c.D[i * N + l];
        for (int q = 0; q < neq; ++q) dxi[q] += S[q * L + (size_t)e * nd + s] * co;
      }
      for (int l = 0; l < N; ++l) {
        const int s = k * c.Ny * N + l * N + i;
        const double co = c.D[j * N + l];
        for (int q = 0; q < neq; ++q) deta[q] += S[q * L + (size_t)e * nd + s] * co;
      }
      if (dim > 2)
        for (int l = 0; l < N; ++l) {
          const int s = l * c.Ny * N + j * N + i;
          const double co = c.D[k * N + l];
          for (int q = 0; q < neq; ++q) dzeta[q] += S[q * L + (size_t)e * nd + s] * co;
        }
      const double invJ = 1.0 / J[point];
      const double *adj = M + point * dim * dim;
      for (int q = 0; q < neq; ++q) {
        const size_t o = q * L + (size_t)e * nd + point;
        if (dim == 2) {
          grad[0 * neq * L + o] = invJ * (dxi[q] * adj[0] + deta[q] * adj[2]);
          grad[1 * neq * L + o] = invJ * (dxi[q] * adj[1] + deta[q] * adj[3]);
        } else {
          grad[0 * neq * L + o] = invJ * (dxi[q] * adj[0] + deta[q] * adj[3] + dzeta[q] * adj[6]);
          grad[1 * neq * L + o] = invJ * (dxi[q] * adj[1] + deta[q] * adj[4] + dzeta[q] * adj[7]);
          grad[2 * neq * L + o] = invJ * (dxi[q] * adj[2] + deta[q] * adj[5] + dzeta[q] * adj[8]);
        }
      }
    }
  }
  // face lift, summed per direction then added (restr_f->MultTranspose; +=)
  std::vector<double> acc((size_t)neq * L);
  for (int cdir = 0; cdir < dim; ++cdir) {
    std::fill(acc.begin(), acc.end(), 0.0);
    for (int f = 0; f < c.nf; ++f) {
      const int em = c.geom->face_elem[2 * f], ep = c.geom->face_elem[2 * f + 1];
      const int lm = c.geom->face_lface[2 * f], lpf = c.geom->face_lface[2 * f + 1];
      for (int fp = 0; fp < c.nfp; ++fp) {
        const size_t nm = (size_t)em * nd + trace_node(c, lm, fp);
        const size_t np = (size_t)ep * nd + trace_node(c, lpf, fp);
        const double wm = c.geom->face_wminus[(size_t)f * c.nfp + fp];
        const double wp = c.geom->face_wplus[(size_t)f * c.nfp + fp];
        const double nd_ = c.geom->face_normal[((size_t)f * c.nfp + fp) * dim + cdir];
        for (int q = 0; q < neq; ++q) {
          const double jump = 0.5 * (S[q * L + np] - S[q * L + nm]);
          const double fd = jump * nd_;
          acc[q * L + nm] += wm * fd;
          acc[q * L + np] += wp * fd;
        }
      }
    }
    double *gc = grad + (size_t)cdir * neq * L;
    for (size_t i = 0; i < (size_t)neq * L; ++i) gc[i] += acc[i];
  }
  // boundary faces (include/NSOperator_impl.hpp:285-404,
  // include/DGSEMIntegrator.hpp:1068-1094): scale * jump * n per point, in
  // boundary-face order, then added per direction
  const thx_geometry *gg = c.geom;
  if (gg->num_bdr_faces > 0) {
    for (int cdir = 0; cdir < dim; ++cdir) {
      std::fill(acc.begin(), acc.end(), 0.0);
      for (int b = 0; b < gg->num_bdr_faces; ++b) {
        const int e = gg->bdr_elem[b], lf = gg->bdr_lface[b];
        const thx_bc &bc = gg->bcs[gg->bdr_bc[b]];
        for (int fp = 0; fp < c.nfp; ++fp) {
          const size_t nm = (size_t)e * nd + trace_node(c, lf, fp);
          double w[MAXEQ], fl[MAXEQ];
          for (int q = 0; q < neq; ++q) w[q] = S[q * L + nm];
          bc_grad_flux(c.gas, bc, gg->bc_data, w, fl);
          const double scale = gg->bdr_weight[(size_t)b * c.nfp + fp];
          const double nd_ = gg->bdr_normal[((size_t)b * c.nfp + fp) * dim + cdir];
          for (int q = 0; q < neq; ++q) acc[q * L + nm] += scale * (fl[q] * nd_);
        }
      }
      double *gc = grad + (size_t)cdir * neq * L;
      for (size_t i = 0; i < (size_t)neq * L; ++i) gc[i] += acc[i];
    }
  }
  // entropy gradient -> primitive gradient, per direction
  for (int cdir = 0; cdir < dim; ++cdir) {
    double *gc = grad + (size_t)cdir * neq * L;
#pragma omp parallel for num_threads(nthreads) schedule(static)
    for (long pt = 0; pt < (long)L; ++pt) {
      double q[MAXEQ], dE[MAXEQ], dP[MAXEQ];
      for (int k = 0; k < neq; ++k) { q[k] = u[k * L + pt]; dE[k] = gc[k * L + pt]; }
      grad_entropy_to_prim(c.gas, q, dE, dP);
      for (int k = 0; k < neq; ++k) gc[k * L + pt] = dP[k];
    }
  }
}

// Full RHS: include/RHSOperator_impl.hpp:719-793 with EulerOperator::FlowMult
// (include/EulerOperator_impl.hpp:28-421) or NSOperator::FlowMult
// (include/NSOperator_impl.hpp:161-1105).
// ---------------------------------------------------------------------------
// Boundary conditions.
// Momentum component c of the wall-rotated state (include/Flow.hpp:77-150):
// along the unit normal, then the tangent picked by the smallest normal
// component, then normal x tangent.
static double wall_momentum(int dim, const double *q, const double *n, double inv, int c) {
  const double nx = n[0] * inv, ny = n[1] * inv, nz = dim > 2 ? n[2] * inv : 0.0;
  double x = nx, y = ny, z = nz;
  if (c > 0) {
    double tx, ty, tz;
    if (dim == 2) {
      tx = -ny; ty = nx; tz = 0.0;
    } else if (std::abs(nx) <= std::abs(ny) && std::abs(nx) <= std::abs(nz)) {
      tx = 0.0; ty = nz; tz = -ny;
    } else if (std::abs(ny) <= std::abs(nx) && std::abs(ny) <= std::abs(nz)) {
      tx = -nz; ty = 0.0; tz = nx;
    } else {
      tx = ny; ty = -nx; tz = 0.0;
    }
    if (c == 1) {
      x = tx; y = ty; z = tz;
    } else {
      x = ny * tz - nz * ty;
      y = nz * tx - nx * tz;
      z = nx * ty - ny * tx;
    }
  }
  double r = 0.0;
  r += q[1] * x;
  r += q[2] * y;
  if (dim == 3) r += q[3] * z;
  return r;
}

// Slip-wall pressure p* on the face-rotated state (include/Flow.hpp:54-75,
// 155-170).
static double slipwall_pstar_normal(const Gas &g, const double *q, const double *n) {
  const int dim = g.dim;
  double mag2 = 0.0;
  for (int d = 0; d < dim; ++d) mag2 += n[d] * n[d];
  if (mag2 == 0.0) return 0.0;
  const double inv = 1.0 / std::sqrt(mag2);
  double qr[MAXEQ];
  qr[0] = q[0];
  for (int c = 0; c < dim; ++c) qr[1 + c] = wall_momentum(dim, q, n, inv, c);
  qr[dim + 1] = q[dim + 1];
  const double rho = qr[0];
  const double c = sound_speed(g, qr);
  const double p = pressure(g, qr);
  const double v = qr[1] / qr[0];
  const double gamma = g.gamma;
  const double gammaP1 = gamma + 1.;
  const double gammaM1 = gamma - 1.;
  const double gammaP1Inverse = 1.0 / gammaP1;
  const double gammaM1Inverse = 1.0 / gammaM1;
  if (v > 0.0)
    return (p + 0.25 * v * gammaP1 * rho *
                    (v + std::sqrt(v * v + 8.0 * gammaP1Inverse * p * (gammaM1 * gammaP1Inverse + 1.0) / rho)));
  return p * std::pow(std::max(1.0 + 0.5 * gammaM1 * v / c, 0.0001), 2.0 * gamma * gammaM1Inverse);
}

// Inviscid boundary flux of one boundary face point (include/bc_kernels.hpp:138-152,
// 219-279); sf is the configured surface flux.
static void bc_inviscid(const Gas &g, FaceFn sf, const thx_bc &bc, const double *data, const double *q,
                        const double *n, double *F) {
  const int dim = g.dim, neq = dim + 2;
  switch (bc.type) {
    case THX_BC_SLIP_WALL: {
      const double ps = slipwall_pstar_normal(g, q, n);
      for (int k = 0; k < neq; ++k) F[k] = 0.0;
      for (int d = 0; d < dim; ++d) F[1 + d] = ps * n[d];
      return;
    }
    case THX_BC_SUPERSONIC_OUTFLOW:
      sf(g, q, q, n, F);
      return;
    case THX_BC_PRESCRIBED_STATE:
    case THX_BC_SUPERSONIC_INFLOW:
      sf(g, q, data + bc.data_index, n, F);
      return;
    case THX_BC_SYMMETRY: {
      double qb[MAXEQ], un[MAXDIM], mom[MAXDIM];
      for (int k = 0; k < neq; ++k) qb[k] = q[k];
      for (int d = 0; d < dim; ++d) { un[d] = n[d]; mom[d] = q[1 + d]; }
      double fac = 0.0;
      for (int d = 0; d < dim; ++d) fac += (un[d] * un[d]);
      fac = 1.0 / std::sqrt(fac);
      for (int d = 0; d < dim; ++d) un[d] *= fac;
      double nv = 0.0;
      for (int d = 0; d < dim; ++d) nv += mom[d] * un[d];
      for (int d = 0; d < dim; ++d) qb[1 + d] = -2.0 * nv * un[d] + mom[d];
      sf(g, q, qb, n, F);
      return;
    }
    default:
      for (int k = 0; k < neq; ++k) F[k] = 0.0;
      return;
  }
}

// Normal viscous flux n . F_v from the primitive gradients
// (include/NavierStokesFlux.hpp:296-355, Cartesian).
static void viscous_normal_flux(const Gas &g, const double *q, const double *const dp[3],
                                const double *n, double *flux) {
  const int dim = g.dim, neq = dim + 2, E = dim + 1;
  const double mu = viscosity(g, q);
  const double kappa = conductivity(g, q);
  const double mu_bulk = g.mu_bulk;
  double grho[MAXDIM] = {}, gth[MAXDIM] = {}, gT[MAXDIM] = {};
  double divergence = 0.0;
  for (int d = 0; d < dim; ++d) {
    grho[d] = dp[d][0];
    gth[d] = dp[d][E];
    divergence += dp[d][1 + d];
  }
  grad_temperature(g, q, grho, gth, gT);
  for (int k = 0; k < neq; ++k) flux[k] = 0.0;
  double energy_flux = 0.0;
  for (int comp = 0; comp < dim; ++comp) {
    double traction = 0.0;
    for (int dir = 0; dir < dim; ++dir) {
      const double stress = comp == dir ? mu * (2.0 * dp[dir][1 + comp] - mu_bulk * divergence)
                                        : mu * (dp[dir][1 + comp] + dp[comp][1 + dir]);
      traction += n[dir] * stress;
    }
    flux[1 + comp] = traction;
    energy_flux += vel(q, comp) * traction;
  }
  for (int dir = 0; dir < dim; ++dir) energy_flux += n[dir] * kappa * gT[dir];
  flux[E] = energy_flux;
}

// Viscous boundary flux of one boundary face point (include/bc_kernels.hpp:154-217,
// 281-374): inviscid conditions as above; the exterior state minus the
// interior viscous flux; the no-slip walls from the wall pressure p* and the
// normal viscous flux with the wall's heat flux or temperature.
static void bc_viscous(const Gas &g, FaceFn sf, const thx_bc &bc, const double *data, const double *q,
                       const double *const dp[3], const double *n, double *F) {
  const int dim = g.dim, neq = dim + 2, E = dim + 1;
  switch (bc.type) {
    case THX_BC_PRESCRIBED_STATE: {
      bc_inviscid(g, sf, bc, data, q, n, F);
      double vfl[MAXEQ][MAXDIM];
      viscous_flux(g, q, dp, vfl);
      for (int k = 0; k < neq; ++k)
        for (int d = 0; d < dim; ++d) F[k] -= vfl[k][d] * n[d];
      return;
    }
    case THX_BC_NOSLIP_ADIABATIC: {
      const double *vwall = data + bc.data_index;
      const double qwall = vwall[dim];
      const double ps = slipwall_pstar_normal(g, q, n);
      viscous_normal_flux(g, q, dp, n, F);
      double mag2 = 0.0;
      for (int d = 0; d < dim; ++d) mag2 += n[d] * n[d];
      double ef = qwall * std::sqrt(mag2);
      for (int d = 0; d < dim; ++d) ef += vwall[d] * F[1 + d];
      F[E] = ef;
      for (int k = 0; k < neq; ++k) F[k] = -F[k];
      for (int d = 0; d < dim; ++d) F[1 + d] += ps * n[d];
      return;
    }
    case THX_BC_NOSLIP_ISOTHERMAL: {
      const double *vwall = data + bc.data_index;
      const double ps = slipwall_pstar_normal(g, q, n);
      viscous_normal_flux(g, q, dp, n, F);
      for (int d = 0; d < dim; ++d) F[E] -= vel(q, d) * F[1 + d];
      for (int d = 0; d < dim; ++d) F[E] += vwall[d] * F[1 + d];
      for (int k = 0; k < neq; ++k) F[k] = -F[k];
      for (int d = 0; d < dim; ++d) F[1 + d] += ps * n[d];
      return;
    }
    case THX_BC_SLIP_WALL:
    case THX_BC_SUPERSONIC_INFLOW:
    case THX_BC_SUPERSONIC_OUTFLOW:
    case THX_BC_SYMMETRY:
      bc_inviscid(g, sf, bc, data, q, n, F);
      return;
    default:
      for (int k = 0; k < neq; ++k) F[k] = 0.0;
      return;
  }
}

static int rhs(const Disc &c, const double *u, double *dudt, int nthreads,
               double *alpha_out, double *eta_out) {
  const int dim = c.dim, N = c.Np, nd = c.nd, neq = c.neq, ne = c.ne;
  const size_t L = (size_t)ne * nd;
  VolFn vf = vol_fn(c.cfg.volume_flux);
  FaceFn sf = face_fn(c.cfg.surface_flux);
  FaceFn fvf = face_fn(c.cfg.fv_flux);
  if (!vf || !sf || (c.cfg.blending && !fvf)) return THX_ERR_INVALID_ARGUMENT;
  const bool ns = c.cfg.flow_model == THX_FLOW_NAVIER_STOKES;
  std::vector<double> alpha(ne, 0.0), eta(ne, 0.0);
  if (c.cfg.blending) blending(c, u, alpha.data(), eta.data(), nthreads);
  if (alpha_out) std::memcpy(alpha_out, alpha.data(), sizeof(double) * ne);
  if (eta_out) std::memcpy(eta_out, eta.data(), sizeof(double) * ne);
  std::vector<double> grad;
  if (ns) {
    grad.resize((size_t)dim * neq * L);
    gradient(c, u, grad.data(), nthreads);
  }
  const int nxi = (c.Nx + 1) * c.Ny * c.Nz, neta = c.Nx * (c.Ny + 1) * c.Nz,
            nzeta = c.Nx * c.Ny * (c.Nz + 1);
  // volume
#pragma omp parallel for num_threads(nthreads) schedule(static)
  for (int e = 0; e < ne; ++e) {
    std::vector<double> ue(neq * nd), du(neq * nd), dfv(neq * nd);
    gather_elem(c, u, e, ue.data());
    const double *J = c.geom->jac + (size_t)e * nd;
    const double *M = c.geom->metric + (size_t)e * nd * dim * dim;
    volume_element(c, vf, ue.data(), J, M, du.data());
    if (c.cfg.blending && alpha[e] > 1e-16) {
      const double adg = 1.0 - alpha[e];
      fv_element(c, fvf, ue.data(), J, c.sub_xi.data() + (size_t)e * nxi * dim,
                 dim > 1 ? c.sub_eta.data() + (size_t)e * neta * dim : nullptr,
                 dim > 2 ? c.sub_zeta.data() + (size_t)e * nzeta * dim : nullptr, dfv.data());
      for (int v = 0; v < neq * nd; ++v) du[v] = adg * du[v] + alpha[e] * dfv[v];
    }
    if (ns) {
      // viscous volume flux cache then weak-form divergence
      // (include/DGSEMIntegrator.hpp:486-622)
      std::vector<double> fl((size_t)dim * neq * nd);
      for (int point = 0; point < nd; ++point) {
        double q[MAXEQ], g0[MAXEQ], g1[MAXEQ], g2[MAXEQ] = {0};
        for (int k = 0; k < neq; ++k) {
          q[k] = ue[k * nd + point];
          const size_t o = k * L + (size_t)e * nd + point;
          g0[k] = grad[0 * neq * L + o];
          g1[k] = grad[1 * neq * L + o];
          if (dim > 2) g2[k] = grad[2 * neq * L + o];
        }
        const double *dp[3] = {g0, g1, g2};
        double vfl[MAXEQ][MAXDIM];
        viscous_flux(c.gas, q, dp, vfl);
        for (int dir = 0; dir < dim; ++dir) {
          const double *row = M + (point * dim + dir) * dim;
          for (int k = 0; k < neq; ++k) {
            double f = 0.0;
            for (int pd = 0; pd < dim; ++pd) f += row[pd] * vfl[k][pd];
            fl[(dir * neq + k) * nd + point] = f;
          }
        }
      }
      const double *Dh = c.Dhat.data();
      for (int point = 0; point < nd; ++point) {
        const int i = point % N, j = (point / N) % c.Ny, k = point / (N * c.Ny);
        double dv[MAXEQ] = {0, 0, 0, 0, 0};
        for (int l = 0; l < N; ++l) {
          const int s = k * c.Ny * N + j * N + l;
          const double co = Dh[i * N + l];
          for (int q = 0; q < neq; ++q) dv[q] += co * fl[(0 * neq + q) * nd + s];
        }
        for (int l = 0; l < N; ++l) {
          const int s = k * c.Ny * N + l * N + i;
          const double co = Dh[j * N + l];
          for (int q = 0; q < neq; ++q) dv[q] += co * fl[(1 * neq + q) * nd + s];
        }
        if (dim > 2)
          for (int l = 0; l < N; ++l) {
            const int s = l * c.Ny * N + j * N + i;
            const double co = Dh[k * N + l];
            for (int q = 0; q < neq; ++q) dv[q] += co * fl[(2 * neq + q) * nd + s];
          }
        const double sc = 1.0 / J[point];
        for (int q = 0; q < neq; ++q) du[point + q * nd] += sc * dv[q];
      }
    }
    for (int q = 0; q < neq; ++q)
      std::memcpy(dudt + q * L + (size_t)e * nd, du.data() + q * nd, sizeof(double) * nd);
  }
  // interior faces: flux per face point, then transpose-scatter and add
  std::vector<double> ff((size_t)c.nf * c.nfp * neq);
#pragma omp parallel for num_threads(nthreads) schedule(static)
  for (int f = 0; f < c.nf; ++f) {
    const int em = c.geom->face_elem[2 * f], ep = c.geom->face_elem[2 * f + 1];
    const int lm = c.geom->face_lface[2 * f], lpf = c.geom->face_lface[2 * f + 1];
    for (int fp = 0; fp < c.nfp; ++fp) {
      const size_t nm = (size_t)em * nd + trace_node(c, lm, fp);
      const size_t np = (size_t)ep * nd + trace_node(c, lpf, fp);
      double qm[MAXEQ], qp[MAXEQ], F[MAXEQ];
      for (int q = 0; q < neq; ++q) { qm[q] = u[q * L + nm]; qp[q] = u[q * L + np]; }
      const double *nrm = c.geom->face_normal + ((size_t)f * c.nfp + fp) * dim;
      sf(c.gas, qm, qp, nrm, F);
      if (ns) {
        // include/DGSEMIntegrator.hpp:261-316
        double gm[3][MAXEQ], gp[3][MAXEQ];
        for (int d = 0; d < dim; ++d)
          for (int q = 0; q < neq; ++q) {
            gm[d][q] = grad[(size_t)d * neq * L + q * L + nm];
            gp[d][q] = grad[(size_t)d * neq * L + q * L + np];
          }
        const double *dm[3] = {gm[0], gm[1], gm[2]};
        const double *dpp[3] = {gp[0], gp[1], gp[2]};
        double vm[MAXEQ][MAXDIM], vp[MAXEQ][MAXDIM];
        viscous_flux(c.gas, qm, dm, vm);
        viscous_flux(c.gas, qp, dpp, vp);
        for (int q = 0; q < neq; ++q)
          for (int d = 0; d < dim; ++d) F[q] -= nrm[d] * (0.5 * (vm[q][d] + vp[q][d]));
      }
      for (int q = 0; q < neq; ++q) ff[((size_t)f * c.nfp + fp) * neq + q] = F[q];
    }
  }
  std::vector<double> acc((size_t)neq * L, 0.0);
  for (int f = 0; f < c.nf; ++f) {
    const int em = c.geom->face_elem[2 * f], ep = c.geom->face_elem[2 * f + 1];
    const int lm = c.geom->face_lface[2 * f], lpf = c.geom->face_lface[2 * f + 1];
    for (int fp = 0; fp < c.nfp; ++fp) {
      const size_t nm = (size_t)em * nd + trace_node(c, lm, fp);
      const size_t np = (size_t)ep * nd + trace_node(c, lpf, fp);
      const double wm = c.geom->face_wminus[(size_t)f * c.nfp + fp];
      const double wp = c.geom->face_wplus[(size_t)f * c.nfp + fp];
      for (int q = 0; q < neq; ++q) {
        const double F = ff[((size_t)f * c.nfp + fp) * neq + q];
        acc[q * L + nm] += -wm * F;
        acc[q * L + np] += wp * F;
      }
    }
  }
  for (size_t i = 0; i < (size_t)neq * L; ++i) dudt[i] += acc[i];
  // boundary faces (include/EulerOperator_impl.hpp:292-392): flux per point,
  // -w * flux scattered in boundary-face order, then added
  const thx_geometry *g = c.geom;
  if (g->num_bdr_faces > 0) {
    std::vector<double> accb((size_t)neq * L, 0.0);
    for (int b = 0; b < g->num_bdr_faces; ++b) {
      const int e = g->bdr_elem[b], lf = g->bdr_lface[b];
      const thx_bc &bc = g->bcs[g->bdr_bc[b]];
      for (int fp = 0; fp < c.nfp; ++fp) {
        const size_t nm = (size_t)e * nd + trace_node(c, lf, fp);
        double q[MAXEQ], F[MAXEQ];
        for (int k = 0; k < neq; ++k) q[k] = u[k * L + nm];
        const double *nrm = g->bdr_normal + ((size_t)b * c.nfp + fp) * dim;
        if (ns) {
          double gd[3][MAXEQ] = {};
          for (int d = 0; d < dim; ++d)
            for (int k = 0; k < neq; ++k) gd[d][k] = grad[(size_t)d * neq * L + k * L + nm];
          const double *dp[3] = {gd[0], gd[1], gd[2]};
          bc_viscous(c.gas, sf, bc, g->bc_data, q, dp, nrm, F);
        } else {
          bc_inviscid(c.gas, sf, bc, g->bc_data, q, nrm, F);
        }
        const double scale = -g->bdr_weight[(size_t)b * c.nfp + fp];
        for (int k = 0; k < neq; ++k) accb[k * L + nm] += scale * F[k];
      }
    }
    for (size_t i = 0; i < (size_t)neq * L; ++i) dudt[i] += accb[i];
  }
  return THX_OK;
}

}  // namespace orc

using namespace orc;

extern "C" {

int orc_lgl(int np, double *x, double *w) {
  if (np < 2 || !x || !w) return THX_ERR_INVALID_ARGUMENT;
  orc::lgl(np, x, w);
  return THX_OK;
}

int orc_operators(int order, double *D, double *Dhat, double *Dhat2) {
  thx_geometry g{};
  g.dim = 2;
  g.order = order;
  thx_config cfg{};
  cfg.gamma = 1.4; cfg.Pr = 0.72; cfg.R_gas = 287.05;
  Disc c;
  const int st = setup(c, &g, &cfg);
  if (st) return st;
  const int n = c.Np * c.Np;
  std::memcpy(D, c.D.data(), sizeof(double) * n);
  std::memcpy(Dhat, c.Dhat.data(), sizeof(double) * n);
  std::memcpy(Dhat2, c.Dhat2.data(), sizeof(double) * n);
  return THX_OK;
}

// Periodic Cartesian box (MFEM MakeCartesian numbering, x fastest; CalcOrtho
// normals; w = 1/(w0 J)), restated independently of the product library.
int orc_box_geometry(int dim, int order, const int32_t *n, const double *lo, const double *hi,
                     double *jac, double *metric, int32_t *face_elem, int32_t *face_lface,
                     double *face_normal, double *face_wminus, double *face_wplus,
                     double *coords) {
  if (dim < 2 || dim > 3 || order < 1) return THX_ERR_INVALID_ARGUMENT;
  const int Np = order + 1;
  const int nd = dim == 2 ? Np * Np : Np * Np * Np;
  const int nfp = dim == 2 ? Np : Np * Np;
  int nn[3] = {n[0], n[1], dim > 2 ? n[2] : 1};
  const int ne = nn[0] * nn[1] * nn[2];
  double h[3];
  for (int d = 0; d < 3; ++d) h[d] = d < dim ? (hi[d] - lo[d]) / nn[d] : 1.0;
  std::vector<double> x(Np), w(Np);
  orc::lgl(Np, x.data(), w.data());
  const double J = dim == 2 ? h[0] * h[1] : h[0] * h[1] * h[2];
  for (int e = 0; e < ne; ++e) {
    const int ex = e % nn[0], ey = (e / nn[0]) % nn[1], ez = e / (nn[0] * nn[1]);
    for (int a = 0; a < nd; ++a) {
      jac[(size_t)e * nd + a] = J;
      double *M = metric + ((size_t)e * nd + a) * dim * dim;
      for (int r = 0; r < dim * dim; ++r) M[r] = 0.0;
      // adjugate of diag(h): row dir has entry prod_{d != dir} h_d
      for (int dir = 0; dir < dim; ++dir) {
        double v = 1.0;
        for (int d = 0; d < dim; ++d) if (d != dir) v *= h[d];
        M[dir * dim + dir] = v;
      }
      if (coords) {
        const int i = a % Np, j = (a / Np) % Np, k = a / (Np * Np);
        const size_t L = (size_t)ne * nd;
        coords[0 * L + (size_t)e * nd + a] = lo[0] + h[0] * (ex + x[i]);
        coords[1 * L + (size_t)e * nd + a] = lo[1] + h[1] * (ey + x[j]);
        if (dim > 2) coords[2 * L + (size_t)e * nd + a] = lo[2] + h[2] * (ez + x[k]);
      }
    }
  }
  int f = 0;
  for (int dir = 0; dir < dim; ++dir)
    for (int e = 0; e < ne; ++e) {
      int ix[3] = {e % nn[0], (e / nn[0]) % nn[1], e / (nn[0] * nn[1])};
      ix[dir] = (ix[dir] + 1) % nn[dir];
      const int ep = ix[0] + nn[0] * (ix[1] + nn[1] * ix[2]);
      face_elem[2 * f] = e;
      face_elem[2 * f + 1] = ep;
      face_lface[2 * f] = 2 * dir + 1;
      face_lface[2 * f + 1] = 2 * dir;
      double area = 1.0;
      for (int d = 0; d < dim; ++d) if (d != dir) area *= h[d];
      for (int fp = 0; fp < nfp; ++fp) {
        for (int d = 0; d < dim; ++d) face_normal[((size_t)f * nfp + fp) * dim + d] = d == dir ? area : 0.0;
        face_wminus[(size_t)f * nfp + fp] = 1.0 / (w[0] * J);
        face_wplus[(size_t)f * nfp + fp] = 1.0 / (w[0] * J);
      }
      ++f;
    }
  return THX_OK;
}

int orc_rhs(const thx_geometry *g, const thx_config *cfg, const double *u, double *dudt,
            int nthreads, double *alpha, double *eta) {
  Disc c;
  int st = setup(c, g, cfg);
  if (st) return st;
  if (nthreads < 1) nthreads = 1;
  return rhs(c, u, dudt, nthreads, alpha, eta);
}

// Primitive gradients as NSOperator stores them (byNODES per direction).
int orc_gradient(const thx_geometry *g, const thx_config *cfg, const double *u, double *grad,
                 int nthreads) {
  Disc c;
  int st = setup(c, g, cfg);
  if (st) return st;
  gradient(c, u, grad, nthreads < 1 ? 1 : nthreads);
  return THX_OK;
}

// SSP-RK3 in the arithmetic order of mfem::RK3SSPSolver::Step (Shu-Osher form).
int orc_rk3_steps(const thx_geometry *g, const thx_config *cfg, double *u, double dt, int nsteps,
                  int nthreads) {
  Disc c;
  int st = setup(c, g, cfg);
  if (st) return st;
  if (nthreads < 1) nthreads = 1;
  const size_t n = (size_t)c.neq * c.ne * c.nd;
  std::vector<double> k(n), y(n);
  for (int s = 0; s < nsteps; ++s) {
    st = rhs(c, u, k.data(), nthreads, nullptr, nullptr);
    if (st) return st;
    for (size_t i = 0; i < n; ++i) y[i] = u[i] + dt * k[i];
    st = rhs(c, y.data(), k.data(), nthreads, nullptr, nullptr);
    if (st) return st;
    for (size_t i = 0; i < n; ++i) { y[i] += dt * k[i]; y[i] = 0.75 * u[i] + 0.25 * y[i]; }
    st = rhs(c, y.data(), k.data(), nthreads, nullptr, nullptr);
    if (st) return st;
    for (size_t i = 0; i < n; ++i) { y[i] += dt * k[i]; u[i] = (1.0 / 3.0) * u[i] + (2.0 / 3.0) * y[i]; }
  }
  return THX_OK;
}

// Stability estimate (include/RHSOperator_impl.hpp:10-174,
// include/StabilityEstimate.hpp:12-92), with the boundary-point term.
int orc_estimate_dt(const thx_geometry *g, const thx_config *cfg, const double *u, double cfl,
                    double *dt, double *rates) {
  Disc c;
  int st = setup(c, g, cfg);
  if (st) return st;
  static const double adv_cal[] = {0.0, 2.19706891727, 5.41995189335, 9.64849524786,
                                   14.7297419321, 20.5984751391, 27.2141622680, 34.5459214016,
                                   42.5691944324, 51.2637780299, 60.6126232210, 70.6010566044,
                                   81.2162499718};
  static const double dif_cal[] = {0.0, 4.0, 25.5969429388, 82.9000427145, 203.470468982,
                                   426.230394541, 799.733889878, 1383.0975821, 2244.38177282,
                                   3461.2550528, 5121.29136549, 7321.77632194, 10169.7148876};
  const int p = c.p;
  const double adv_scale = (p > 0 && p < 13) ? 1.05 * adv_cal[p] : 0.65 * (p + 1) * (p + 1);
  const double dif_scale = (p > 0 && p < 13) ? 1.25 * dif_cal[p]
                                             : 0.5 * (p + 1.0) * (p + 1.0) * (p + 1.0) * (p + 1.0);
  const double surf_scale = adv_scale / (1.0 / c.w[0]);
  const bool visc = c.cfg.flow_model == THX_FLOW_NAVIER_STOKES;
  const int dim = c.dim, nd = c.nd, neq = c.neq;
  const size_t L = (size_t)c.ne * nd;
  double adv = 0.0, dif = 0.0, sur = 0.0;
  for (size_t pt = 0; pt < L; ++pt) {
    double q[MAXEQ];
    for (int k = 0; k < neq; ++k) q[k] = u[k * L + pt];
    const double ij = 1.0 / g->jac[pt];
    double ds = 0.0, mss = 0.0;
    const double a = sound_speed(c.gas, q);
    for (int rd = 0; rd < dim; ++rd) {
      double vdm = 0.0, mn2 = 0.0;
      for (int pd = 0; pd < dim; ++pd) {
        const double v = g->metric[(pt * dim + rd) * dim + pd];
        vdm += vel(q, pd) * v;
        mn2 += v * v;
      }
      ds += (std::fabs(vdm) + a * std::sqrt(mn2)) * ij;
      mss += mn2 * ij * ij;
    }
    adv = std::max(adv, adv_scale * ds);
    if (visc) {
      const double rho = q[0];
      const double mu = viscosity(c.gas, q);
      const double lon = (2.0 - c.gas.mu_bulk) * mu;
      const double md = std::max(mu, lon) / rho;
      const double td = conductivity(c.gas, q) * c.gas.gamma / (rho * c.gas.cp);
      dif = std::max(dif, dif_scale * std::max(md, td) * mss);
    }
  }
  for (int f = 0; f < c.nf; ++f) {
    const int em = g->face_elem[2 * f], ep = g->face_elem[2 * f + 1];
    const int lm = g->face_lface[2 * f], lp = g->face_lface[2 * f + 1];
    for (int fp = 0; fp < c.nfp; ++fp) {
      const size_t nm = (size_t)em * nd + trace_node(c, lm, fp);
      const size_t np = (size_t)ep * nd + trace_node(c, lp, fp);
      double qm[MAXEQ] = {0}, qp[MAXEQ] = {0};
      for (int k = 0; k < neq; ++k) { qm[k] = u[k * L + nm]; qp[k] = u[k * L + np]; }
      const double *nr = g->face_normal + ((size_t)f * c.nfp + fp) * dim;
      double n2 = 0, vm = 0, vp = 0;
      for (int d = 0; d < dim; ++d) { n2 += nr[d] * nr[d]; vm += vel(qm, d) * nr[d]; vp += vel(qp, d) * nr[d]; }
      const double nm_ = std::sqrt(n2);
      const double ws = std::max(std::fabs(vm) + sound_speed(c.gas, qm) * nm_,
                                 std::fabs(vp) + sound_speed(c.gas, qp) * nm_);
      const double wmx = std::max(std::fabs(g->face_wminus[(size_t)f * c.nfp + fp]),
                                  std::fabs(g->face_wplus[(size_t)f * c.nfp + fp]));
      sur = std::max(sur, ws * wmx * surf_scale);
    }
  }
  // boundary points (include/RHSOperator_impl.hpp:176-268): the interior
  // wave speed, for an exterior state also its speed and (viscous) its
  // effective diffusivity times the trace's metric square sum
  for (int b = 0; b < g->num_bdr_faces; ++b) {
    const int e = g->bdr_elem[b], lf = g->bdr_lface[b];
    const thx_bc &bc = g->bcs[g->bdr_bc[b]];
    for (int fp = 0; fp < c.nfp; ++fp) {
      const size_t nm = (size_t)e * nd + trace_node(c, lf, fp);
      double q[MAXEQ] = {0};
      for (int k = 0; k < neq; ++k) q[k] = u[k * L + nm];
      const double *nr = g->bdr_normal + ((size_t)b * c.nfp + fp) * dim;
      double n2 = 0.0, vn = 0.0;
      for (int d = 0; d < dim; ++d) { n2 += nr[d] * nr[d]; vn += vel(q, d) * nr[d]; }
      double ws = std::fabs(vn) + sound_speed(c.gas, q) * std::sqrt(n2);
      if (bc.type == THX_BC_PRESCRIBED_STATE || bc.type == THX_BC_SUPERSONIC_INFLOW) {
        const double *qe = g->bc_data + bc.data_index;
        if (visc) {
          const double ij = 1.0 / g->jac[nm];
          double mss = 0.0;
          for (int rd = 0; rd < dim; ++rd) {
            double mn2 = 0.0;
            for (int pd = 0; pd < dim; ++pd) {
              const double v = g->metric[(nm * dim + rd) * dim + pd];
              mn2 += v * v;
            }
            mss += mn2 * ij * ij;
          }
          const double rho = qe[0];
          const double mu = viscosity(c.gas, qe);
          const double lon = (2.0 - c.gas.mu_bulk) * mu;
          const double md = std::max(mu, lon) / rho;
          const double td = conductivity(c.gas, qe) * c.gas.gamma / (rho * c.gas.cp);
          dif = std::max(dif, dif_scale * std::max(md, td) * mss);
        }
        double ve = 0.0;
        for (int d = 0; d < dim; ++d) ve += vel(qe, d) * nr[d];
        ws = std::max(ws, std::fabs(ve) + sound_speed(c.gas, qe) * std::sqrt(n2));
      }
      sur = std::max(sur, ws * std::fabs(g->bdr_weight[(size_t)b * c.nfp + fp]) * surf_scale);
    }
  }
  if (rates) { rates[0] = adv; rates[1] = sur; rates[2] = dif; }
  const double total = std::max(adv, sur) + dif;
  if (!(total > 0.0)) return THX_ERR_NUMERICS;
  *dt = cfl / total;
  return THX_OK;
}

// Pointwise fluxes for known-answer tests.
int orc_volume_flux(int flux, const thx_config *cfg, int dim, const double *q1, const double *q2,
                    const double *m1, const double *m2, double *F) {
  VolFn f = vol_fn(flux);
  if (!f) return THX_ERR_INVALID_ARGUMENT;
  Gas g = make_gas(*cfg, dim);
  f(g, q1, q2, m1, m2, F);
  return THX_OK;
}
int orc_face_flux(int flux, const thx_config *cfg, int dim, const double *qm, const double *qp,
                  const double *n, double *F) {
  FaceFn f = face_fn(flux);
  if (!f) return THX_ERR_INVALID_ARGUMENT;
  Gas g = make_gas(*cfg, dim);
  f(g, qm, qp, n, F);
  return THX_OK;
}
int orc_entropy_vars(const thx_config *cfg, int dim, const double *q, double *w) {
  Gas g = make_gas(*cfg, dim);
  entropy_vars(g, q, w);
  return THX_OK;
}
int orc_viscous_flux(const thx_config *cfg, int dim, const double *q, const double *dprim,
                     double *vf_out /* [neq][dim] */) {
  Gas g = make_gas(*cfg, dim);
  const double *dp[3] = {dprim, dprim + (dim + 2), dprim + 2 * (dim + 2)};
  double vf[MAXEQ][MAXDIM];
  viscous_flux(g, q, dp, vf);
  for (int e = 0; e < dim + 2; ++e)
    for (int d = 0; d < dim; ++d) vf_out[e * dim + d] = vf[e][d];
  return THX_OK;
}

// Global entropy-production residual R_S = sum_e sum_i w_i J_i v(U_i).dU_i/dt
// (definition stated for the oracle; v from include/EOS.hpp:206-234).
int orc_entropy_residual(const thx_geometry *g, const thx_config *cfg, const double *u,
                         const double *dudt, double *out) {
  Disc c;
  int st = setup(c, g, cfg);
  if (st) return st;
  const int nd = c.nd, neq = c.neq, N = c.Np;
  const size_t L = (size_t)c.ne * nd;
  long double acc = 0.0L;
  for (size_t pt = 0; pt < L; ++pt) {
    const int a = (int)(pt % nd);
    const int i = a % N, j = (a / N) % N, k = a / (N * N);
    double wq = c.w[i] * c.w[j] * (c.dim > 2 ? c.w[k] : 1.0);
    double q[MAXEQ], v[MAXEQ];
    for (int kk = 0; kk < neq; ++kk) q[kk] = u[kk * L + pt];
    entropy_vars(c.gas, q, v);
    double dot = 0.0;
    for (int kk = 0; kk < neq; ++kk) dot += v[kk] * dudt[kk * L + pt];
    acc += (long double)(wq * g->jac[pt] * dot);
  }
  *out = (double)acc;
  return THX_OK;
}

int orc_blending(const thx_geometry *g, const thx_config *cfg, const double *u, double *alpha,
                 double *eta) {
  Disc c;
  int st = setup(c, g, cfg);
  if (st) return st;
  if (!cfg->blending) return THX_ERR_INVALID_ARGUMENT;
  blending(c, u, alpha, eta, 1);
  return THX_OK;
}

// Subcell FV metrics in the reference layout
// (include/dgsem_cache_utilities.hpp:641-763); any pointer may be NULL.
int orc_subcell_metrics(const thx_geometry *g, const thx_config *cfg, double *xi, double *eta,
                        double *zeta) {
  thx_config c2 = *cfg;
  c2.blending = 1;
  Disc c;
  int st = setup(c, g, &c2);
  if (st) return st;
  if (xi) std::memcpy(xi, c.sub_xi.data(), sizeof(double) * c.sub_xi.size());
  if (eta && !c.sub_eta.empty()) std::memcpy(eta, c.sub_eta.data(), sizeof(double) * c.sub_eta.size());
  if (zeta && !c.sub_zeta.empty()) std::memcpy(zeta, c.sub_zeta.data(), sizeof(double) * c.sub_zeta.size());
  return THX_OK;
}

// ---- LTE Helmholtz gas ------------------------------------------------------
static lte::Table lte_view(const thx_lte_table *t) {
  lte::Table v;
  v.nx = t->nx; v.ny = t->ny; v.rho = t->rho_grid; v.T = t->T_grid; v.e = t->e_grid;
  v.planes = t->planes; v.inv = t->inverse;
  return v;
}

int orc_lte_idg_table(const thx_idg_params *p, int nx, int ny, double lr0, double lr1, double lt0,
                      double lt1, double *rho, double *T, double *planes) {
  if (!p || nx < 2 || ny < 2 || !rho || !T || !planes) return THX_ERR_INVALID_ARGUMENT;
  lte::IDG g{p->R, p->rho_d, p->theta_d, p->mu0, p->T0, p->Pr};
  lte::idg_table(g, nx, ny, lr0, lr1, lt0, lt1, rho, T, planes);
  return THX_OK;
}

int orc_lte_inverse_table(int nx, int ny, const double *rho, const double *T, const double *planes,
                          double *egrid, double *inv) {
  if (nx < 2 || ny < 2) return THX_ERR_INVALID_ARGUMENT;
  return lte::inverse_table(nx, ny, rho, T, planes, egrid, inv) ? THX_OK : THX_ERR_NUMERICS;
}

// out: p, e, gibbs, cv, c^2, mu, lambda at (rho, T)
int orc_lte_point(const thx_lte_table *t, double rho, double T, double *out) {
  const lte::Table v = lte_view(t);
  const lte::Eval s = lte::at(v, rho, T);
  if (!s.valid) return THX_ERR_NUMERICS;
  out[0] = s.pressure(); out[1] = s.energy(); out[2] = s.gibbs(); out[3] = s.cv();
  out[4] = s.c2(); out[5] = s.transport(v, 4); out[6] = s.transport(v, 5);
  return THX_OK;
}

int orc_lte_temperature(const thx_lte_table *t, double rho, double e, double *T, int *status) {
  const lte::Table v = lte_view(t);
  *T = lte::temperature(v, rho, e, status);
  return THX_OK;
}

int orc_lte_flux(const thx_lte_table *t, int dim, int face, const double *q1, const double *q2,
                 const double *d1, const double *d2, double *F) {
  const lte::Table v = lte_view(t);
  bool bad = false;
  lte::lteec(v, dim, face != 0, q1, q2, d1, d2, F, &bad);
  return bad ? THX_ERR_NUMERICS : THX_OK;
}

int orc_rhs_lte(const thx_geometry *g, const thx_config *cfg, const thx_lte_table *t,
                const double *u, double *dudt, int nthreads) {
  Disc c;
  int st = setup(c, g, cfg);
  if (st) return st;
  const lte::Table v = lte_view(t);
  std::atomic<int> bad{0};
  c.gas.lte = &v;
  c.gas.bad = &bad;
  st = rhs(c, u, dudt, nthreads < 1 ? 1 : nthreads, nullptr, nullptr);
  if (st) return st;
  return bad.load() ? THX_ERR_NUMERICS : THX_OK;
}

// Integral measures (include/RHSOperator_impl.hpp:530-717): per element, in
// node order, the sums of rho, |m|^2/(2 rho) and rho E weighted by
// J * (w_a w_b w_c), and the extrema of pressure, temperature and density;
// then the element sums and extrema in element order.  out[9] = mass, ke,
// energy, min p, max p, min T, max T, min rho, max rho.  LTE gas when t.
static int integral_measures(Disc &c, const double *u, double *out) {
  const Gas &g = c.gas;
  const long long L = (long long)c.ne * c.nd;
  double mass = 0, ke = 0, en = 0, pmin = 1e32, pmax = 0, tmin = 1e32, tmax = 0, rmin = 1e32, rmax = 0;
  for (int e = 0; e < c.ne; ++e) {
    double m_i = 0, k_i = 0, e_i = 0, pn = 1e32, px = 0, tn = 1e32, tx = 0, dn = 1e32, dx = 0;
    for (int n = 0; n < c.nd; ++n) {
      double q[MAXEQ];
      for (int k = 0; k < c.neq; ++k) q[k] = u[k * L + (long long)e * c.nd + n];
      const int a = n % c.Np, b = (n / c.Np) % c.Np, cz = n / (c.Np * c.Np);
      double W = c.w[a] * c.w[b];
      if (c.dim == 3) W = W * c.w[cz];
      const double measure = c.geom->jac[(long long)e * c.nd + n] * W;
      const double rho = q[0];
      const double kin = ke_density(g, q);
      const double rhoE = q[c.dim + 1];
      double press, temper;
      if (g.lte) {
        const lte::Eval s = lte_state(g, q);
        press = s.pressure();
        temper = s.T;
      } else {
        press = pressure(g, q);
        temper = temperature(g, q);
      }
      m_i += rho * measure;
      k_i += kin * measure;
      e_i += rhoE * measure;
      tn = std::min(tn, temper); tx = std::max(tx, temper);
      dn = std::min(dn, rho); dx = std::max(dx, rho);
      pn = std::min(pn, press); px = std::max(px, press);
    }
    mass += m_i; ke += k_i; en += e_i;
    pmin = std::min(pmin, pn); pmax = std::max(pmax, px);
    tmin = std::min(tmin, tn); tmax = std::max(tmax, tx);
    rmin = std::min(rmin, dn); rmax = std::max(rmax, dx);
  }
  const double r[9] = {mass, ke, en, pmin, pmax, tmin, tmax, rmin, rmax};
  for (int k = 0; k < 9; ++k) out[k] = r[k];
  return THX_OK;
}

int orc_integral_measures(const thx_geometry *g, const thx_config *cfg, const thx_lte_table *t,
                          const double *u, double *out) {
  Disc c;
  int st = setup(c, g, cfg);
  if (st) return st;
  lte::Table v;
  std::atomic<int> bad{0};
  if (t) {
    v = lte_view(t);
    c.gas.lte = &v;
    c.gas.bad = &bad;
  }
  st = integral_measures(c, u, out);
  if (st) return st;
  return bad.load() ? THX_ERR_NUMERICS : THX_OK;
}

int orc_max_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

}  // extern "C"
