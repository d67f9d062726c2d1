// lte_oracle.h -- TEST INFRASTRUCTURE ONLY.
//
// CPU FP64 restatement of the reference's LTE Helmholtz equation of state and
// its entropy-conservative flux, used by oracle/thx_oracle.cpp:
//   table layout and cell search     include/LTEHelmholtzTable.hpp:13-35,83-105
//   bicubic Hermite evaluation       include/LTEHelmholtzInterpolation.hpp:15-212
//   state evaluation, T(rho,e) Newton include/LTEHelmholtzEOS.hpp:14-223
//   discrete gradients, means        include/LTEHelmholtzEOS.hpp:225-397
//   gas adapter                      include/LTEHelmholtzGasEOS.hpp:10-172
//   LTEEC flux                       include/LTEECFlux.hpp:11-91
//   inverse table (PLATO-free part)  include/LTEHelmholtzTableBuilder.hpp:131-218
//   grids                            include/LTETable.hpp:85-103
#pragma once
#include <cmath>
#include <limits>
#include <vector>

namespace orc {
namespace lte {

struct Table {
  int nx = 0, ny = 0;                      // density, temperature samples
  const double *rho = nullptr, *T = nullptr, *e = nullptr;
  const double *planes = nullptr;          // [6][ny][nx]: H, H_r, H_T, H_rT, mu, lambda
  const double *inv = nullptr;             // [ny][nx]
  int index(int prop, int i, int j) const { return prop * nx * ny + j * nx + i; }
};

inline int find_cell(const double *grid, int count, double v) {
  if (count < 2 || !std::isfinite(v) || v < grid[0] || v > grid[count - 1]) return -1;
  int lo = 0, hi = count - 1;
  while (hi - lo > 1) {
    const int mid = lo + (hi - lo) / 2;
    if (v < grid[mid]) hi = mid;
    else lo = mid;
  }
  return lo;
}

// Cubic Hermite bases on [0,1] and their derivatives (order 0..2).
inline double pos_basis(int d, int side, double x) {
  const double x2 = x * x;
  if (d == 0) { const double x3 = x2 * x; return side == 0 ? 2 * x3 - 3 * x2 + 1 : -2 * x3 + 3 * x2; }
  if (d == 1) return side == 0 ? 6 * x2 - 6 * x : -6 * x2 + 6 * x;
  return side == 0 ? 12 * x - 6 : -12 * x + 6;
}
inline double slope_basis(int d, int side, double x) {
  const double x2 = x * x;
  if (d == 0) { const double x3 = x2 * x; return side == 0 ? x3 - 2 * x2 + x : x3 - x2; }
  if (d == 1) return side == 0 ? 3 * x2 - 4 * x + 1 : 3 * x2 - 2 * x;
  return side == 0 ? 6 * x - 4 : 6 * x - 2;
}
// divided differences of the bases between x and y (coincident-safe)
inline double div_pos_basis(int d, int side, double x, double y) {
  double v;
  if (d == 0) v = 2 * (x * x + x * y + y * y) - 3 * (x + y);
  else if (d == 1) v = 6 * (x + y) - 6;
  else v = 12;
  return side == 0 ? v : -v;
}
inline double div_slope_basis(int d, int side, double x, double y) {
  if (d == 0) return x * x + x * y + y * y - (side == 0 ? 2 : 1) * (x + y) + (side == 0 ? 1 : 0);
  if (d == 1) return 3 * (x + y) - (side == 0 ? 4 : 2);
  return 6;
}
inline double coord_scale(int d, double w) { return d == 0 ? 1.0 : (d == 1 ? w : w * w); }

struct Cell {
  const double *H, *Hr, *HT, *HrT;   // lower corner in each plane
  int stride;                        // nx
  double dr, dt;                     // cell widths
};

inline double evaluate(const Cell &c, int dr_ord, int dt_ord, double xi, double eta) {
  double r = 0.0;
  for (int ds = 0; ds < 2; ++ds) {
    const double dv = pos_basis(dr_ord, ds, xi), dsl = slope_basis(dr_ord, ds, xi);
    for (int ts = 0; ts < 2; ++ts) {
      const int o = ds + ts * c.stride;
      const double tv = pos_basis(dt_ord, ts, eta), tsl = slope_basis(dt_ord, ts, eta);
      r += c.H[o] * dv * tv;
      r += (c.Hr[o] * c.dr) * dsl * tv;
      r += (c.HT[o] * c.dt) * dv * tsl;
      r += (c.HrT[o] * c.dr * c.dt) * dsl * tsl;
    }
  }
  return r / (coord_scale(dr_ord, c.dr) * coord_scale(dt_ord, c.dt));
}

// axis 0: density varies (eta2 unused); axis 1: temperature varies
inline double divided(const Cell &c, int axis, int dr_ord, int dt_ord, double xi1, double eta1,
                      double xi2, double eta2) {
  double r = 0.0;
  for (int i = 0; i < 2; ++i) {
    const double rv = axis == 0 ? div_pos_basis(dr_ord, i, xi1, xi2) : pos_basis(dr_ord, i, xi1);
    const double rs = axis == 0 ? div_slope_basis(dr_ord, i, xi1, xi2) : slope_basis(dr_ord, i, xi1);
    for (int j = 0; j < 2; ++j) {
      const double tv = axis == 1 ? div_pos_basis(dt_ord, j, eta1, eta2) : pos_basis(dt_ord, j, eta1);
      const double ts = axis == 1 ? div_slope_basis(dt_ord, j, eta1, eta2) : slope_basis(dt_ord, j, eta1);
      const int o = i + j * c.stride;
      r += c.H[o] * rv * tv;
      r += (c.Hr[o] * c.dr) * rs * tv;
      r += (c.HT[o] * c.dt) * rv * ts;
      r += (c.HrT[o] * c.dr * c.dt) * rs * ts;
    }
  }
  const double sc = coord_scale(dr_ord, c.dr) * coord_scale(dt_ord, c.dt) * (axis == 0 ? c.dr : c.dt);
  return r / sc;
}

struct Eval {
  Cell cell{};
  double xi = 0, eta = 0, rho = 0, T = 0;
  bool valid = false;
  double H(int a = 0, int b = 0) const { return evaluate(cell, a, b, xi, eta); }
  double pressure() const { return rho * rho * H(1, 0); }
  double energy() const { return H() - T * H(0, 1); }
  double gibbs() const { return H() + rho * H(1, 0); }
  double dp_drho() const { return 2 * rho * H(1, 0) + rho * rho * H(2, 0); }
  double dp_dT() const { return rho * rho * H(1, 1); }
  double dg_drho() const { return 2 * H(1, 0) + rho * H(2, 0); }
  double dg_dT() const { return H(0, 1) + rho * H(1, 1); }
  double cv() const { return -T * H(0, 2); }
  double c2() const {
    const double m = H(1, 1);
    return dp_drho() - rho * rho * m * m / H(0, 2);
  }
  double transport(const Table &t, int prop) const {
    const long off = cell.H - t.planes;
    const double *p = t.planes + (long)prop * t.nx * t.ny + off;
    return p[0] * (1 - xi) * (1 - eta) + p[1] * xi * (1 - eta) + p[t.nx] * (1 - xi) * eta +
           p[t.nx + 1] * xi * eta;
  }
};

inline Eval at(const Table &t, double rho, double T) {
  Eval r;
  const int i = find_cell(t.rho, t.nx, rho), j = find_cell(t.T, t.ny, T);
  if (i < 0 || j < 0) return r;
  const int off = j * t.nx + i, size = t.nx * t.ny;
  const double dr = t.rho[i + 1] - t.rho[i], dt = t.T[j + 1] - t.T[j];
  r.cell = {t.planes + off, t.planes + size + off, t.planes + 2 * size + off,
            t.planes + 3 * size + off, t.nx, dr, dt};
  r.xi = (rho - t.rho[i]) / dr;
  r.eta = (T - t.T[j]) / dt;
  r.rho = rho;
  r.T = T;
  r.valid = true;
  return r;
}

enum Status { CONVERGED = 0, OUTSIDE = 1, INVALID = 2, ITERATIONS = 3 };

// Inverse-table guess, then Newton on e(rho,T) with the analytic cv.
inline double temperature(const Table &t, double rho, double e, int *status) {
  *status = OUTSIDE;
  const int i = find_cell(t.rho, t.nx, rho), j = find_cell(t.e, t.ny, e);
  if (i < 0 || j < 0) return 0.0;
  const double x = (rho - t.rho[i]) / (t.rho[i + 1] - t.rho[i]);
  const double y = (e - t.e[j]) / (t.e[j + 1] - t.e[j]);
  const double *p = t.inv + j * t.nx + i;
  const double lower = p[0] + x * (p[1] - p[0]);
  const double upper = p[t.nx] + x * (p[t.nx + 1] - p[t.nx]);
  double T = lower + y * (upper - lower);
  for (int it = 0; it < 100; ++it) {
    const Eval s = at(t, rho, T);
    if (!s.valid) return T;
    const double cv = s.cv(), guess = s.energy();
    if (!std::isfinite(cv) || cv <= 0 || !std::isfinite(guess)) { *status = INVALID; return T; }
    const double step = (e - guess) / cv;
    const double next = T + step;
    const bool inside = std::isfinite(next) && next >= t.T[0] && next <= t.T[t.ny - 1];
    if (std::fabs(step) <= 1e-9 + 1e-12 * T) {
      if (next < t.T[0]) T = t.T[0];
      else if (next > t.T[t.ny - 1]) T = t.T[t.ny - 1];
      else T = next;
      *status = CONVERGED;
      return T;
    }
    T = next;
    if (!inside) return T;
  }
  *status = ITERATIONS;
  return T;
}

// Itoh-Abe discrete gradient of f/T in (rho, beta=1/T); f = p (prop 0) or g (prop 1)
inline double value(int prop, const Eval &s) { return prop == 0 ? s.pressure() : s.gibbs(); }

inline double density_secant(int prop, const Eval &a, const Eval &b, double eta) {
  const Cell &c = a.cell;
  const double r1 = a.rho, r2 = b.rho;
  const double mean_hr = 0.5 * (evaluate(c, 1, 0, a.xi, eta) + evaluate(c, 1, 0, b.xi, eta));
  const double div_hr = divided(c, 0, 1, 0, a.xi, eta, b.xi, eta);
  if (prop == 0) return 0.5 * (r1 * r1 + r2 * r2) * div_hr + (r1 + r2) * mean_hr;
  const double div_h = divided(c, 0, 0, 0, a.xi, eta, b.xi, eta);
  return div_h + 0.5 * (r1 + r2) * div_hr + mean_hr;
}

inline double beta_secant(int prop, const Eval &a, const Eval &b, double xi, double rho) {
  const Cell &c = a.cell;
  const double mean_t = 0.5 * (a.T + b.T);
  const double mean_hr = 0.5 * (evaluate(c, 1, 0, xi, a.eta) + evaluate(c, 1, 0, xi, b.eta));
  const double div_hr = divided(c, 1, 1, 0, xi, a.eta, xi, b.eta);
  const double hr_beta = mean_hr - mean_t * div_hr;
  if (prop == 0) return rho * rho * hr_beta;
  const double mean_h = 0.5 * (evaluate(c, 0, 0, xi, a.eta) + evaluate(c, 0, 0, xi, b.eta));
  const double div_h = divided(c, 1, 0, 0, xi, a.eta, xi, b.eta);
  return mean_h - mean_t * div_h + rho * hr_beta;
}

struct Grad { double rho, beta; };

inline Grad discrete_gradient(int prop, const Table &t, const Eval &left, const Eval &right) {
  const bool rev = left.rho > right.rho || (left.rho == right.rho && left.T > right.T);
  const Eval &A = rev ? right : left;
  const Eval &B = rev ? left : right;
  const double b1 = 1 / A.T, b2 = 1 / B.T;
  const double dr = B.rho - A.rho, db = b2 - b1;
  const double rmax = A.rho > B.rho ? A.rho : B.rho;
  const double bmax = b1 > b2 ? b1 : b2;
  const bool ddiff = std::fabs(dr) >= 2.22e-15 + 1.49e-8 * rmax;
  const bool bdiff = std::fabs(db) >= 2.22e-15 + 1.49e-8 * bmax;
  const double f11 = value(prop, A), f22 = value(prop, B);
  Grad g{0.0, 0.0};
  if (A.cell.H == B.cell.H) {
    if (ddiff) g.rho = 0.5 * (density_secant(prop, A, B, A.eta) * b1 + density_secant(prop, A, B, B.eta) * b2);
    if (bdiff) g.beta = 0.5 * (beta_secant(prop, A, B, A.xi, A.rho) + beta_secant(prop, A, B, B.xi, B.rho));
  } else if (ddiff || bdiff) {
    const double f12 = value(prop, at(t, A.rho, B.T));
    const double f21 = value(prop, at(t, B.rho, A.T));
    if (ddiff) g.rho = 0.5 * ((f21 * b1 - f11 * b1) + (f22 * b2 - f12 * b2)) / dr;
    if (bdiff) g.beta = 0.5 * ((f12 * b2 - f11 * b1) + (f22 * b2 - f21 * b1)) / db;
  }
  if (!ddiff)
    g.rho = prop == 0 ? 0.5 * (A.dp_drho() * b1 + B.dp_drho() * b2)
                      : 0.5 * (A.dg_drho() * b1 + B.dg_drho() * b2);
  if (!bdiff) {
    const double d1 = prop == 0 ? A.dp_dT() : A.dg_dT();
    const double d2 = prop == 0 ? B.dp_dT() : B.dg_dT();
    g.beta = 0.5 * ((f11 - A.T * d1) + (f22 - B.T * d2));
  }
  return g;
}

inline void means(const Table &t, const Eval &l, const Eval &r, double *rho_mean, double *e_mean) {
  const Grad p = discrete_gradient(0, t, l, r);
  const Grad g = discrete_gradient(1, t, l, r);
  *rho_mean = p.rho / g.rho;
  *e_mean = g.beta - p.beta / *rho_mean;
}

// Gas adapter: recover T from (rho, e) and evaluate there.  Failures set *bad.
inline Eval evaluate_state(const Table &t, int dim, const double *q, bool *bad) {
  double m2 = 0.0;
  for (int d = 0; d < dim; ++d) m2 += q[1 + d] * q[1 + d];
  const double ke = 0.5 * m2 / q[0];
  const double e = (q[dim + 1] - ke) / q[0];
  int st;
  const double T = temperature(t, q[0], e, &st);
  if (st != CONVERGED) { *bad = true; return Eval{}; }
  Eval s = at(t, q[0], T);
  if (!s.valid) *bad = true;
  return s;
}

// LTEEC flux: face (Lax dissipation, dir1 = normal) or volume (averaged metric)
inline void lteec(const Table &t, int dim, bool face, const double *q1, const double *q2,
                  const double *d1, const double *d2, double *F, bool *bad) {
  const Eval s1 = evaluate_state(t, dim, q1, bad);
  const Eval s2 = evaluate_state(t, dim, q2, bad);
  if (*bad) { for (int k = 0; k < dim + 2; ++k) F[k] = NAN; return; }
  double rho_mean, e_mean;
  means(t, s1, s2, &rho_mean, &e_mean);
  const double p1 = s1.pressure(), p2 = s2.pressure();
  double c1 = 0, c2 = 0;
  if (face) { c1 = std::sqrt(s1.c2()); c2 = std::sqrt(s2.c2()); }
  const double pm = 0.5 * (p1 + p2);
  double vn = 0, ck = 0, pw = 0, v1n = 0, v2n = 0, nn = 0;
  for (int d = 0; d < dim; ++d) {
    const double dir = face ? d1[d] : 0.5 * (d1[d] + d2[d]);
    const double u1 = q1[1 + d] / q1[0], u2 = q2[1 + d] / q2[0];
    vn += 0.5 * (u1 + u2) * dir;
    ck += 0.5 * u1 * u2;
    pw += 0.5 * (p1 * u2 + p2 * u1) * dir;
    if (face) { v1n += u1 * dir; v2n += u2 * dir; nn += dir * dir; }
  }
  double dis = 0.0;
  if (face) {
    const double nm = std::sqrt(nn);
    const double sp1 = std::fabs(v1n) + c1 * nm, sp2 = std::fabs(v2n) + c2 * nm;
    dis = 0.5 * (sp1 > sp2 ? sp1 : sp2);
  }
  const double mf = rho_mean * vn;
  F[0] = mf - dis * (q2[0] - q1[0]);
  for (int d = 0; d < dim; ++d) {
    const double dir = face ? d1[d] : 0.5 * (d1[d] + d2[d]);
    const double v = 0.5 * (q1[1 + d] / q1[0] + q2[1 + d] / q2[0]);
    F[1 + d] = mf * v + pm * dir - dis * (q2[1 + d] - q1[1 + d]);
  }
  F[dim + 1] = mf * (e_mean + ck) + pw - dis * (q2[dim + 1] - q1[dim + 1]);
}

}  // namespace lte
}  // namespace orc

namespace orc {
namespace lte {

// Synthetic ideal-dissociating gas (Lighthill), the table the project supplies
// in place of the reference's PLATO build.  Per unit mass, with R the
// molecular gas constant, rho_d the characteristic density, theta_d the
// dissociation temperature and alpha the equilibrium degree of dissociation
//   alpha^2/(1-alpha) = (rho_d/rho) exp(-theta_d/T),
//   H(rho,T) = R T [(1-alpha) ln((1-alpha) rho) + 2 alpha ln(alpha rho/rho_a) - 3 ln T]
//              + alpha R theta_d,          rho_a = sqrt(e rho_d),
// so that p = rho^2 H_rho = rho R T (1+alpha) and e = H - T H_T = 3 R T + alpha R theta_d.
// First derivatives follow from dH/dalpha = 0 at equilibrium; H_rhoT adds the
// alpha_T term.  Transport planes: mu = mu0 (T/T0)^0.7, lambda = mu * 4R(1+alpha)/Pr.
struct IDG { double R, rho_d, theta_d, mu0, T0, Pr; };

inline void idg_alpha(const IDG &g, double rho, double T, double *a, double *oma) {
  const double K = (g.rho_d / rho) * std::exp(-g.theta_d / T);
  if (K <= 0.0) { *a = 0.0; *oma = 1.0; return; }
  const double s = std::sqrt(1.0 + 4.0 / K);
  *a = 2.0 / (1.0 + s);
  *oma = (4.0 / K) / ((s + 1.0) * (s + 1.0));
}
inline double xlogy(double x, double y) { return x == 0.0 ? 0.0 : x * std::log(y); }

inline void idg_point(const IDG &g, double rho, double T, double *out /*[6]*/) {
  double a, oma;
  idg_alpha(g, rho, T, &a, &oma);
  const double rho_a = std::sqrt(std::exp(1.0) * g.rho_d);
  const double bracket = xlogy(oma, oma * rho) + 2.0 * xlogy(a, a * rho / rho_a) - 3.0 * std::log(T);
  out[0] = g.R * T * bracket + a * g.R * g.theta_d;                 // H
  out[1] = g.R * T * (1.0 + a) / rho;                               // H_rho
  out[2] = g.R * bracket - 3.0 * g.R;                               // H_T
  const double a_T = g.theta_d * a * oma / (T * T * (2.0 - a));
  out[3] = g.R * (1.0 + a) / rho + g.R * T * a_T / rho;             // H_rhoT
  const double mu = g.mu0 * std::pow(T / g.T0, 0.7);
  out[4] = mu;
  out[5] = mu * 4.0 * g.R * (1.0 + a) / g.Pr;
}

// log-spaced grid (include/LTETable.hpp:95-103) and the full forward planes
inline void idg_table(const IDG &g, int nx, int ny, double lr0, double lr1, double lt0, double lt1,
                      double *rho, double *T, double *planes) {
  const double sr = (lr1 - lr0) / (nx - 1), st = (lt1 - lt0) / (ny - 1);
  for (int i = 0; i < nx; ++i) rho[i] = std::pow(10.0, lr0) * std::pow(10.0, i * sr);
  for (int j = 0; j < ny; ++j) T[j] = std::pow(10.0, lt0) * std::pow(10.0, j * st);
  for (int j = 0; j < ny; ++j)
    for (int i = 0; i < nx; ++i) {
      double v[6];
      idg_point(g, rho[i], T[j], v);
      for (int p = 0; p < 6; ++p) planes[(long)p * nx * ny + (long)j * nx + i] = v[p];
    }
}

// Energy grid and inverse table (include/LTEHelmholtzTableBuilder.hpp:131-218)
inline bool inverse_table(int nx, int ny, const double *rho, const double *T, const double *planes,
                          double *egrid, double *inv) {
  double emin = HUGE_VAL, emax = -HUGE_VAL, scale = 1.0;
  const long ps = (long)nx * ny;
  for (int j = 0; j < ny; ++j)
    for (int i = 0; i < nx; ++i) {
      const long k = (long)j * nx + i;
      const double h = planes[k], tht = T[j] * planes[2 * ps + k];
      const double e = h - tht;
      emin = std::min(emin, e);
      emax = std::max(emax, e);
      scale = std::max(scale, std::fabs(h) + std::fabs(tht));
    }
  const double pad = 64 * std::numeric_limits<double>::epsilon() * scale;
  emin -= pad;
  emax += pad;
  const double step = (emax - emin) / (ny - 1);
  for (int j = 0; j < ny; ++j) egrid[j] = emin + j * step;
  Table t;
  t.nx = nx; t.ny = ny; t.rho = rho; t.T = T; t.e = egrid; t.planes = planes; t.inv = inv;
  for (int i = 0; i < nx; ++i) {
    const double lo_T = T[0], hi_T = T[ny - 1];
    const double lo_e = at(t, rho[i], lo_T).energy(), hi_e = at(t, rho[i], hi_T).energy();
    if (!std::isfinite(lo_e) || !std::isfinite(hi_e) || hi_e <= lo_e) return false;
    for (int j = 0; j < ny; ++j) {
      const double e = egrid[j];
      double lo = lo_T, hi = hi_T;
      if (e <= lo_e) hi = lo;
      else if (e >= hi_e) lo = hi;
      else
        for (int it = 0; it < 60; ++it) {
          const double mid = lo + (hi - lo) / 2;
          if (at(t, rho[i], mid).energy() < e) lo = mid;
          else hi = mid;
        }
      inv[(long)j * nx + i] = lo + (hi - lo) / 2;
    }
  }
  return true;
}

}  // namespace lte
}  // namespace orc
