// thx_lte_host.cpp -- host-side set-up of the LTE Helmholtz gas table: the
// energy grid and inverse table that HelmholtzTable::Build derives from a
// forward table, and the synthetic ideal-dissociating-gas table that stands in
// for the reference's PLATO-built one.  No device work happens here.
#include "thx_lte.cuh"
#include "theseus_b200.h"

#include <algorithm>
#include <cfloat>
#include <cmath>

namespace {

using thx::LteDev;

// Equilibrium degree of dissociation alpha and 1 - alpha of Lighthill's gas,
// alpha^2 / (1 - alpha) = K = (rho_d / rho) exp(-theta_d / T); 1 - alpha is
// formed without cancellation as (4/K) / (s + 1)^2, s = sqrt(1 + 4/K).
void idg_alpha(const thx_idg_params &g, double rho, double T, double *a, double *oma) {
  const double K = (g.rho_d / rho) * std::exp(-g.theta_d / T);
  if (K <= 0.0) {
    *a = 0.0;
    *oma = 1.0;
    return;
  }
  const double s = std::sqrt(1.0 + 4.0 / K);
  *a = 2.0 / (1.0 + s);
  *oma = (4.0 / K) / ((s + 1.0) * (s + 1.0));
}

double x_log_y(double x, double y) { return x == 0.0 ? 0.0 : x * std::log(y); }

// Free energy per unit mass and its physical derivatives at one sample:
//   H = R T [(1-a) ln((1-a) rho) + 2a ln(a rho / rho_a) - 3 ln T] + a R theta_d,
//   rho_a = sqrt(e rho_d); dH/da = 0 at equilibrium, so
//   H_rho = R T (1+a) / rho,  H_T = R [bracket] - 3R,
//   H_rhoT = R (1+a) / rho + R T a_T / rho,  a_T = theta_d a (1-a) / (T^2 (2-a));
// mu = mu0 (T/T0)^0.7 and lambda = mu 4R(1+a)/Pr.
void idg_sample(const thx_idg_params &g, double rho, double T, double *out) {
  double a, oma;
  idg_alpha(g, rho, T, &a, &oma);
  const double rho_a = std::sqrt(std::exp(1.0) * g.rho_d);
  const double bracket = x_log_y(oma, oma * rho) + 2.0 * x_log_y(a, a * rho / rho_a) - 3.0 * std::log(T);
  out[0] = g.R * T * bracket + a * g.R * g.theta_d;
  out[1] = g.R * T * (1.0 + a) / rho;
  out[2] = g.R * bracket - 3.0 * g.R;
  const double a_T = g.theta_d * a * oma / (T * T * (2.0 - a));
  out[3] = g.R * (1.0 + a) / rho + g.R * T * a_T / rho;
  const double mu = g.mu0 * std::pow(T / g.T0, 0.7);
  out[4] = mu;
  out[5] = mu * 4.0 * g.R * (1.0 + a) / g.Pr;
}

}  // namespace

extern "C" {

int thx_lte_idg_table(const thx_idg_params *gas, int nx, int ny, double lr0, double lr1, double lt0,
                      double lt1, double *rho_grid, double *T_grid, double *planes) {
  if (!gas || nx < 2 || ny < 2 || !rho_grid || !T_grid || !planes || !(lr1 > lr0) || !(lt1 > lt0) ||
      !(gas->R > 0) || !(gas->rho_d > 0) || !(gas->theta_d > 0) || !(gas->T0 > 0) || !(gas->Pr > 0))
    return THX_ERR_INVALID_ARGUMENT;
  // log-spaced samples, base times a power (include/LTETable.hpp:95-103)
  const double sr = (lr1 - lr0) / (nx - 1), st = (lt1 - lt0) / (ny - 1);
  for (int i = 0; i < nx; ++i) rho_grid[i] = std::pow(10.0, lr0) * std::pow(10.0, i * sr);
  for (int j = 0; j < ny; ++j) T_grid[j] = std::pow(10.0, lt0) * std::pow(10.0, j * st);
  const long plane = (long)nx * ny;
  for (int j = 0; j < ny; ++j)
    for (int i = 0; i < nx; ++i) {
      double v[6];
      idg_sample(*gas, rho_grid[i], T_grid[j], v);
      for (int p = 0; p < 6; ++p) planes[p * plane + (long)j * nx + i] = v[p];
    }
  return THX_OK;
}

// include/LTEHelmholtzTableBuilder.hpp:148-170 (padded energy range) and
// :172-216 (60-step bisection of e(rho_i, T) = e_j between the grid's end
// temperatures, clamped outside the sampled energy range).
int thx_lte_inverse_table(int nx, int ny, const double *rho_grid, const double *T_grid,
                          const double *planes, double *e_grid, double *inverse) {
  if (nx < 2 || ny < 2 || !rho_grid || !T_grid || !planes || !e_grid || !inverse)
    return THX_ERR_INVALID_ARGUMENT;
  const long ps = (long)nx * ny;
  double emin = HUGE_VAL, emax = -HUGE_VAL, scale = 1.0;
  for (int j = 0; j < ny; ++j)
    for (int i = 0; i < nx; ++i) {
      const long k = (long)j * nx + i;
      const double h = planes[k], tht = T_grid[j] * planes[2 * ps + k];
      const double e = h - tht;
      emin = std::min(emin, e);
      emax = std::max(emax, e);
      scale = std::max(scale, std::fabs(h) + std::fabs(tht));
    }
  if (!std::isfinite(emin) || !std::isfinite(emax) || !(emax > emin)) return THX_ERR_NUMERICS;
  const double pad = 64 * DBL_EPSILON * scale;
  emin -= pad;
  emax += pad;
  const double step = (emax - emin) / (ny - 1);
  for (int j = 0; j < ny; ++j) e_grid[j] = emin + j * step;
  LteDev t;
  t.nx = nx;
  t.ny = ny;
  t.rho = rho_grid;
  t.T = T_grid;
  t.e = e_grid;
  t.planes = planes;
  t.inv = inverse;
  auto energy = [&](double rho, double T) { return thx::lte_energy(t, thx::lte_at(t, rho, T)); };
  for (int i = 0; i < nx; ++i) {
    const double lo_T = T_grid[0], hi_T = T_grid[ny - 1];
    const double lo_e = energy(rho_grid[i], lo_T), hi_e = energy(rho_grid[i], hi_T);
    if (!std::isfinite(lo_e) || !std::isfinite(hi_e) || hi_e <= lo_e) return THX_ERR_NUMERICS;
    for (int j = 0; j < ny; ++j) {
      const double e = e_grid[j];
      double lo = lo_T, hi = hi_T;
      if (e <= lo_e) hi = lo;
      else if (e >= hi_e) lo = hi;
      else
        for (int it = 0; it < 60; ++it) {
          const double mid = lo + (hi - lo) / 2;
          if (energy(rho_grid[i], mid) < e) lo = mid;
          else hi = mid;
        }
      inverse[(long)j * nx + i] = lo + (hi - lo) / 2;
    }
  }
  return THX_OK;
}

}  // extern "C"
