// thx_lte.cuh -- LTE Helmholtz equation of state and the LTEEC flux, for host
// and device (FP64).
//
// Restates, in the reference's operation order:
//   table layout, cell search        include/LTEHelmholtzTable.hpp:13-35,83-105
//   bicubic Hermite evaluation       include/LTEHelmholtzInterpolation.hpp:15-212
//   state evaluation, Newton T(rho,e) include/LTEHelmholtzEOS.hpp:14-223
//   Itoh-Abe discrete gradients      include/LTEHelmholtzEOS.hpp:225-397
//   gas adapter (entropy variables,  include/LTEHelmholtzGasEOS.hpp:10-172,
//     gradient conversion, transport) include/LTETransport.hpp:19-66
//   LTEEC flux                       include/LTEECFlux.hpp:11-99
// Failed recoveries are reported through a status flag instead of the
// reference's device trap.
#pragma once
#include <cuda_runtime.h>
#include <cmath>

namespace thx {

#define THX_HD __host__ __device__ __forceinline__
// The Newton recovery is called, not inlined.  The discrete gradients are
// inlined: called, they kept a 1.6 KB stack frame per thread whose traffic
// cost more than the spills of the inlined form (LTEEC volume kernel 2.24 ->
// 1.68 ms at 24^3 p=4).
#define THX_HDC static __host__ __device__ __noinline__

struct LteDev {
  int nx = 0, ny = 0;
  const double *rho = nullptr, *T = nullptr, *e = nullptr;
  const double *planes = nullptr;  // [6][ny][nx]
  const double *inv = nullptr;     // [ny][nx]
};

THX_HD int lte_find_cell(const double *grid, int count, double v) {
  if (count < 2 || !isfinite(v) || v < grid[0] || v > grid[count - 1]) return -1;
  int lo = 0, hi = count - 1;
  while (hi - lo > 1) {
    const int mid = lo + (hi - lo) / 2;
    if (v < grid[mid]) hi = mid;
    else lo = mid;
  }
  return lo;
}

// lte_find_cell(grid, count, v) found by walking from the cell `from`
// (0 <= from <= count - 2): the same cell, in a step or two when v moved
// little since `from` was found.
THX_HD int lte_walk_cell(const double *grid, int count, double v, int from) {
  if (count < 2 || !isfinite(v) || v < grid[0] || v > grid[count - 1]) return -1;
  int lo = from;
  while (lo > 0 && v < grid[lo]) --lo;
  while (lo < count - 2 && v >= grid[lo + 1]) ++lo;
  return lo;
}

template <int D> THX_HD double hpos(int side, double x) {
  const double x2 = x * x;
  if (D == 0) { const double x3 = x2 * x; return side == 0 ? 2 * x3 - 3 * x2 + 1 : -2 * x3 + 3 * x2; }
  if (D == 1) return side == 0 ? 6 * x2 - 6 * x : -6 * x2 + 6 * x;
  return side == 0 ? 12 * x - 6 : -12 * x + 6;
}
template <int D> THX_HD double hslope(int side, double x) {
  const double x2 = x * x;
  if (D == 0) { const double x3 = x2 * x; return side == 0 ? x3 - 2 * x2 + x : x3 - x2; }
  if (D == 1) return side == 0 ? 3 * x2 - 4 * x + 1 : 3 * x2 - 2 * x;
  return side == 0 ? 6 * x - 4 : 6 * x - 2;
}
template <int D> THX_HD double hdivpos(int side, double x, double y) {
  double v;
  if (D == 0) v = 2 * (x * x + x * y + y * y) - 3 * (x + y);
  else if (D == 1) v = 6 * (x + y) - 6;
  else v = 12;
  return side == 0 ? v : -v;
}
template <int D> THX_HD double hdivslope(int side, double x, double y) {
  if (D == 0) return x * x + x * y + y * y - (side == 0 ? 2 : 1) * (x + y) + (side == 0 ? 1 : 0);
  if (D == 1) return 3 * (x + y) - (side == 0 ? 4 : 2);
  return 6;
}
template <int D> THX_HD double hscale(double w) { return D == 0 ? 1.0 : (D == 1 ? w : w * w); }

// One table cell: lower-corner index into a plane, widths, density count.
struct LteCell {
  int off;       // j*nx + i
  int nx;
  double dr, dt;
};

template <int DR, int DT>
THX_HD double lte_eval(const LteDev &t, const LteCell &c, double xi, double eta) {
  const long ps = (long)t.nx * t.ny;
  const double *H = t.planes + c.off, *Hr = H + ps, *HT = H + 2 * ps, *HrT = H + 3 * ps;
  double r = 0.0;
#pragma unroll
  for (int ds = 0; ds < 2; ++ds) {
    const double dv = hpos<DR>(ds, xi), dsl = hslope<DR>(ds, xi);
#pragma unroll
    for (int ts = 0; ts < 2; ++ts) {
      const int o = ds + ts * c.nx;
      const double tv = hpos<DT>(ts, eta), tsl = hslope<DT>(ts, eta);
      r += H[o] * dv * tv;
      r += (Hr[o] * c.dr) * dsl * tv;
      r += (HT[o] * c.dt) * dv * tsl;
      r += (HrT[o] * c.dr * c.dt) * dsl * tsl;
    }
  }
  return r / (hscale<DR>(c.dr) * hscale<DT>(c.dt));
}

// Divided difference along AXIS (0: density, 1: temperature) within one cell.
template <int AXIS, int DR, int DT>
THX_HD double lte_divided(const LteDev &t, const LteCell &c, double xi1, double eta1, double xi2,
                          double eta2) {
  const long ps = (long)t.nx * t.ny;
  const double *H = t.planes + c.off, *Hr = H + ps, *HT = H + 2 * ps, *HrT = H + 3 * ps;
  double r = 0.0;
#pragma unroll
  for (int i = 0; i < 2; ++i) {
    const double rv = AXIS == 0 ? hdivpos<DR>(i, xi1, xi2) : hpos<DR>(i, xi1);
    const double rs = AXIS == 0 ? hdivslope<DR>(i, xi1, xi2) : hslope<DR>(i, xi1);
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      const double tv = AXIS == 1 ? hdivpos<DT>(j, eta1, eta2) : hpos<DT>(j, eta1);
      const double ts = AXIS == 1 ? hdivslope<DT>(j, eta1, eta2) : hslope<DT>(j, eta1);
      const int o = i + j * c.nx;
      r += H[o] * rv * tv;
      r += (Hr[o] * c.dr) * rs * tv;
      r += (HT[o] * c.dt) * rv * ts;
      r += (HrT[o] * c.dr * c.dt) * rs * ts;
    }
  }
  const double sc = hscale<DR>(c.dr) * hscale<DT>(c.dt) * (AXIS == 0 ? c.dr : c.dt);
  return r / sc;
}

struct LteEval {
  LteCell cell;
  double xi, eta, rho, T;
  bool valid;
};

THX_HD LteEval lte_at(const LteDev &t, double rho, double T) {
  LteEval r;
  r.valid = false;
  r.cell = {0, t.nx, 0.0, 0.0};
  r.xi = r.eta = r.rho = r.T = 0.0;
  const int i = lte_find_cell(t.rho, t.nx, rho), j = lte_find_cell(t.T, t.ny, T);
  if (i < 0 || j < 0) return r;
  const double dr = t.rho[i + 1] - t.rho[i], dt = t.T[j + 1] - t.T[j];
  r.cell = {j * t.nx + i, t.nx, dr, dt};
  r.xi = (rho - t.rho[i]) / dr;
  r.eta = (T - t.T[j]) / dt;
  r.rho = rho;
  r.T = T;
  r.valid = true;
  return r;
}

// lte_at(t, a.rho, b.T) for two points that lte_at has already located: the
// density cell and position are a's, the temperature cell and position b's
// (the same searches on the same values give the same cells), so the cross
// state of a discrete gradient needs no table search.
THX_HD LteEval lte_cross(const LteEval &a, const LteEval &b) {
  LteEval r;
  const int nx = a.cell.nx;
  r.cell = {(b.cell.off / nx) * nx + a.cell.off % nx, nx, a.cell.dr, b.cell.dt};
  r.xi = a.xi;
  r.eta = b.eta;
  r.rho = a.rho;
  r.T = b.T;
  r.valid = a.valid && b.valid;
  return r;
}

// lte_at(t, rho, T) given the cell lte_at finds there (cell.off, as the
// temperature recovery stores it per node): the same evaluation without the
// two binary searches.  A cell that is not a valid lower corner (-1: none
// found) falls back to the search.
THX_HD LteEval lte_at_cell(const LteDev &t, double rho, double T, int cell) {
  if (cell < 0) return lte_at(t, rho, T);
  const int i = cell % t.nx, j = cell / t.nx;
  if (i > t.nx - 2 || j > t.ny - 2) return lte_at(t, rho, T);
  LteEval r;
  const double dr = t.rho[i + 1] - t.rho[i], dt = t.T[j + 1] - t.T[j];
  r.cell = {cell, t.nx, dr, dt};
  r.xi = (rho - t.rho[i]) / dr;
  r.eta = (T - t.T[j]) / dt;
  r.rho = rho;
  r.T = T;
  r.valid = true;
  return r;
}

THX_HD double lte_pressure(const LteDev &t, const LteEval &s) {
  return s.rho * s.rho * lte_eval<1, 0>(t, s.cell, s.xi, s.eta);
}
THX_HD double lte_energy(const LteDev &t, const LteEval &s) {
  return lte_eval<0, 0>(t, s.cell, s.xi, s.eta) - s.T * lte_eval<0, 1>(t, s.cell, s.xi, s.eta);
}
THX_HD double lte_gibbs(const LteDev &t, const LteEval &s) {
  return lte_eval<0, 0>(t, s.cell, s.xi, s.eta) + s.rho * lte_eval<1, 0>(t, s.cell, s.xi, s.eta);
}
THX_HD double lte_dp_drho(const LteDev &t, const LteEval &s) {
  return 2 * s.rho * lte_eval<1, 0>(t, s.cell, s.xi, s.eta) +
         s.rho * s.rho * lte_eval<2, 0>(t, s.cell, s.xi, s.eta);
}
THX_HD double lte_dp_dT(const LteDev &t, const LteEval &s) {
  return s.rho * s.rho * lte_eval<1, 1>(t, s.cell, s.xi, s.eta);
}
THX_HD double lte_dg_drho(const LteDev &t, const LteEval &s) {
  return 2 * lte_eval<1, 0>(t, s.cell, s.xi, s.eta) + s.rho * lte_eval<2, 0>(t, s.cell, s.xi, s.eta);
}
THX_HD double lte_dg_dT(const LteDev &t, const LteEval &s) {
  return lte_eval<0, 1>(t, s.cell, s.xi, s.eta) + s.rho * lte_eval<1, 1>(t, s.cell, s.xi, s.eta);
}
THX_HD double lte_cv(const LteDev &t, const LteEval &s) {
  return -s.T * lte_eval<0, 2>(t, s.cell, s.xi, s.eta);
}
THX_HD double lte_c2(const LteDev &t, const LteEval &s) {
  const double m = lte_eval<1, 1>(t, s.cell, s.xi, s.eta);
  return lte_dp_drho(t, s) - s.rho * s.rho * m * m / lte_eval<0, 2>(t, s.cell, s.xi, s.eta);
}
// bilinear transport plane (4: mu, 5: lambda)
THX_HD double lte_transport(const LteDev &t, const LteEval &s, int prop) {
  const double *p = t.planes + (long)prop * t.nx * t.ny + s.cell.off;
  return p[0] * (1 - s.xi) * (1 - s.eta) + p[1] * s.xi * (1 - s.eta) + p[t.nx] * (1 - s.xi) * s.eta +
         p[t.nx + 1] * s.xi * s.eta;
}

// One cell's sixteen corner values (H, H_rho, H_T, H_rhoT at its four
// corners), read once and evaluated at several points or orders:
// lte_eval_k does lte_eval's operations in lte_eval's order.
struct LteCorners {
  double H[4], Hr[4], HT[4], HrT[4];  // corner j = rho side + 2 * T side
  double dr, dt;
};

THX_HD LteCorners lte_corners(const LteDev &t, const LteCell &c) {
  const long ps = (long)t.nx * t.ny;
  const double *H = t.planes + c.off;
  LteCorners k;
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const int o = (j & 1) + (j >> 1) * c.nx;
    k.H[j] = H[o];
    k.Hr[j] = H[ps + o];
    k.HT[j] = H[2 * ps + o];
    k.HrT[j] = H[3 * ps + o];
  }
  k.dr = c.dr;
  k.dt = c.dt;
  return k;
}

template <int DR, int DT>
THX_HD double lte_eval_k(const LteCorners &k, double xi, double eta) {
  double r = 0.0;
#pragma unroll
  for (int ds = 0; ds < 2; ++ds) {
    const double dv = hpos<DR>(ds, xi), dsl = hslope<DR>(ds, xi);
#pragma unroll
    for (int ts = 0; ts < 2; ++ts) {
      const int o = ds + 2 * ts;
      const double tv = hpos<DT>(ts, eta), tsl = hslope<DT>(ts, eta);
      r += k.H[o] * dv * tv;
      r += (k.Hr[o] * k.dr) * dsl * tv;
      r += (k.HT[o] * k.dt) * dv * tsl;
      r += (k.HrT[o] * k.dr * k.dt) * dsl * tsl;
    }
  }
  return r / (hscale<DR>(k.dr) * hscale<DT>(k.dt));
}

enum LteStatus { LTE_CONVERGED = 0, LTE_OUTSIDE = 1, LTE_INVALID = 2, LTE_ITERATIONS = 3 };

// Inverse-table guess, then Newton on e(rho, T) with the analytic cv.
THX_HDC double lte_temperature(const LteDev &t, double rho, double e, int *status) {
  *status = LTE_OUTSIDE;
  const int i = lte_find_cell(t.rho, t.nx, rho), j = lte_find_cell(t.e, t.ny, e);
  if (i < 0 || j < 0) return 0.0;
  const double x = (rho - t.rho[i]) / (t.rho[i + 1] - t.rho[i]);
  const double y = (e - t.e[j]) / (t.e[j + 1] - t.e[j]);
  const double *p = t.inv + j * t.nx + i;
  const double lower = p[0] + x * (p[1] - p[0]);
  const double upper = p[t.nx] + x * (p[t.nx + 1] - p[t.nx]);
  double T = lower + y * (upper - lower);
  // lte_at(t, rho, T) every iteration, with the density cell (the search
  // above) and its position held, the temperature cell found by walking from
  // the previous iteration's, and the cell's corners read when it changes;
  // lte_cv and lte_energy are then lte_eval_k of those corners
  const double dr = t.rho[i + 1] - t.rho[i];
  const double xi = (rho - t.rho[i]) / dr;
  int jt = -1;
  LteCorners k;
  for (int it = 0; it < 100; ++it) {
    const int jn = jt < 0 ? lte_find_cell(t.T, t.ny, T) : lte_walk_cell(t.T, t.ny, T, jt);
    if (jn < 0) return T;
    if (jn != jt) {
      jt = jn;
      k = lte_corners(t, LteCell{jt * t.nx + i, t.nx, dr, t.T[jt + 1] - t.T[jt]});
    }
    const double eta = (T - t.T[jt]) / k.dt;
    const double cv = -T * lte_eval_k<0, 2>(k, xi, eta);
    const double guess = lte_eval_k<0, 0>(k, xi, eta) - T * lte_eval_k<0, 1>(k, xi, eta);
    if (!isfinite(cv) || cv <= 0 || !isfinite(guess)) { *status = LTE_INVALID; return T; }
    const double step = (e - guess) / cv;
    const double next = T + step;
    const bool inside = isfinite(next) && next >= t.T[0] && next <= t.T[t.ny - 1];
    if (fabs(step) <= 1e-9 + 1e-12 * T) {
      if (next < t.T[0]) T = t.T[0];
      else if (next > t.T[t.ny - 1]) T = t.T[t.ny - 1];
      else T = next;
      *status = LTE_CONVERGED;
      return T;
    }
    T = next;
    if (!inside) return T;
  }
  *status = LTE_ITERATIONS;
  return T;
}

// Recover T from a conserved state and evaluate there (adapter evaluate()).
template <int DIM>
THX_HD LteEval lte_state(const LteDev &t, const double *q, bool *bad) {
  double m2 = 0.0;
#pragma unroll
  for (int d = 0; d < DIM; ++d) m2 += q[1 + d] * q[1 + d];
  const double e = (q[DIM + 1] - 0.5 * m2 / q[0]) / q[0];
  int st;
  const double T = lte_temperature(t, q[0], e, &st);
  LteEval s = lte_at(t, q[0], T);
  if (st != LTE_CONVERGED || !s.valid) *bad = true;
  return s;
}

// ---- discrete gradients of f/T in (rho, beta=1/T); f = p (P=0) or g (P=1) ---
template <int P> THX_HD double lte_value(const LteDev &t, const LteEval &s) {
  return P == 0 ? lte_pressure(t, s) : lte_gibbs(t, s);
}

template <int P>
THX_HD double lte_density_secant(const LteDev &t, const LteEval &a, const LteEval &b, double eta) {
  const LteCell &c = a.cell;
  const double r1 = a.rho, r2 = b.rho;
  const double mean_hr = 0.5 * (lte_eval<1, 0>(t, c, a.xi, eta) + lte_eval<1, 0>(t, c, b.xi, eta));
  const double div_hr = lte_divided<0, 1, 0>(t, c, a.xi, eta, b.xi, eta);
  if (P == 0) return 0.5 * (r1 * r1 + r2 * r2) * div_hr + (r1 + r2) * mean_hr;
  const double div_h = lte_divided<0, 0, 0>(t, c, a.xi, eta, b.xi, eta);
  return div_h + 0.5 * (r1 + r2) * div_hr + mean_hr;
}

template <int P>
THX_HD double lte_beta_secant(const LteDev &t, const LteEval &a, const LteEval &b, double xi,
                              double rho) {
  const LteCell &c = a.cell;
  const double mean_t = 0.5 * (a.T + b.T);
  const double mean_hr = 0.5 * (lte_eval<1, 0>(t, c, xi, a.eta) + lte_eval<1, 0>(t, c, xi, b.eta));
  const double div_hr = lte_divided<1, 1, 0>(t, c, xi, a.eta, xi, b.eta);
  const double hr_beta = mean_hr - mean_t * div_hr;
  if (P == 0) return rho * rho * hr_beta;
  const double mean_h = 0.5 * (lte_eval<0, 0>(t, c, xi, a.eta) + lte_eval<0, 0>(t, c, xi, b.eta));
  const double div_h = lte_divided<1, 0, 0>(t, c, xi, a.eta, xi, b.eta);
  return mean_h - mean_t * div_h + rho * hr_beta;
}

template <int P>
THX_HDC void lte_discrete_gradient(const LteDev &t, const LteEval &left, const LteEval &right,
                                  double *grho, double *gbeta) {
  const bool rev = left.rho > right.rho || (left.rho == right.rho && left.T > right.T);
  const LteEval &A = rev ? right : left;
  const LteEval &B = rev ? left : right;
  const double b1 = 1 / A.T, b2 = 1 / B.T;
  const double dr = B.rho - A.rho, db = b2 - b1;
  const double rmx = A.rho > B.rho ? A.rho : B.rho;
  const double bmx = b1 > b2 ? b1 : b2;
  const bool ddiff = fabs(dr) >= 2.22e-15 + 1.49e-8 * rmx;
  const bool bdiff = fabs(db) >= 2.22e-15 + 1.49e-8 * bmx;
  const double f11 = lte_value<P>(t, A), f22 = lte_value<P>(t, B);
  double gr = 0.0, gb = 0.0;
  if (A.cell.off == B.cell.off) {
    if (ddiff) gr = 0.5 * (lte_density_secant<P>(t, A, B, A.eta) * b1 + lte_density_secant<P>(t, A, B, B.eta) * b2);
    if (bdiff) gb = 0.5 * (lte_beta_secant<P>(t, A, B, A.xi, A.rho) + lte_beta_secant<P>(t, A, B, B.xi, B.rho));
  } else if (ddiff || bdiff) {
    const double f12 = lte_value<P>(t, lte_cross(A, B));
    const double f21 = lte_value<P>(t, lte_cross(B, A));
    if (ddiff) gr = 0.5 * ((f21 * b1 - f11 * b1) + (f22 * b2 - f12 * b2)) / dr;
    if (bdiff) gb = 0.5 * ((f12 * b2 - f11 * b1) + (f22 * b2 - f21 * b1)) / db;
  }
  if (!ddiff)
    gr = P == 0 ? 0.5 * (lte_dp_drho(t, A) * b1 + lte_dp_drho(t, B) * b2)
                : 0.5 * (lte_dg_drho(t, A) * b1 + lte_dg_drho(t, B) * b2);
  if (!bdiff) {
    const double d1 = P == 0 ? lte_dp_dT(t, A) : lte_dg_dT(t, A);
    const double d2 = P == 0 ? lte_dp_dT(t, B) : lte_dg_dT(t, B);
    gb = 0.5 * ((f11 - A.T * d1) + (f22 - B.T * d2));
  }
  *grho = gr;
  *gbeta = gb;
}

// ---- both discrete gradients at once ------------------------------------
// The pressure (P=0) and Gibbs (P=1) gradients of the LTEEC means evaluate
// the same bicubic jets at the same points; lte_discrete_gradients forms each
// jet once and, when both endpoints share a table cell, reads that cell's
// sixteen corner values once.  Every output is computed with the operations,
// in the order, of lte_discrete_gradient<P>.
template <int AXIS, int DR, int DT>
THX_HD double lte_divided_k(const LteCorners &k, double xi1, double eta1, double xi2, double eta2) {
  double r = 0.0;
#pragma unroll
  for (int i = 0; i < 2; ++i) {
    const double rv = AXIS == 0 ? hdivpos<DR>(i, xi1, xi2) : hpos<DR>(i, xi1);
    const double rs = AXIS == 0 ? hdivslope<DR>(i, xi1, xi2) : hslope<DR>(i, xi1);
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      const double tv = AXIS == 1 ? hdivpos<DT>(j, eta1, eta2) : hpos<DT>(j, eta1);
      const double ts = AXIS == 1 ? hdivslope<DT>(j, eta1, eta2) : hslope<DT>(j, eta1);
      const int o = i + 2 * j;
      r += k.H[o] * rv * tv;
      r += (k.Hr[o] * k.dr) * rs * tv;
      r += (k.HT[o] * k.dt) * rv * ts;
      r += (k.HrT[o] * k.dr * k.dt) * rs * ts;
    }
  }
  const double sc = hscale<DR>(k.dr) * hscale<DT>(k.dt) * (AXIS == 0 ? k.dr : k.dt);
  return r / sc;
}

// Jets of one endpoint at its own point: H, H_rho, H_T, H_rhorho, H_rhoT.
struct LteJet {
  double H, Hr, HT, Hrr, HrT;
  double c2;  // squared sound speed (lte_face_jet only)
};

THX_HD LteJet lte_jet(const LteDev &t, const LteEval &s) {
  const LteCorners k = lte_corners(t, s.cell);
  LteJet j;
  j.H = lte_eval_k<0, 0>(k, s.xi, s.eta);
  j.Hr = lte_eval_k<1, 0>(k, s.xi, s.eta);
  j.HT = lte_eval_k<0, 1>(k, s.xi, s.eta);
  j.Hrr = lte_eval_k<2, 0>(k, s.xi, s.eta);
  j.HrT = lte_eval_k<1, 1>(k, s.xi, s.eta);
  j.c2 = 0.0;
  return j;
}

// lte_jet and lte_c2 of a face trace from one read of its cell's corners
// (lte_c2 alone reads them four times), with lte_c2's operations.
THX_HD LteJet lte_face_jet(const LteDev &t, const LteEval &s) {
  const LteCorners k = lte_corners(t, s.cell);
  LteJet j;
  j.H = lte_eval_k<0, 0>(k, s.xi, s.eta);
  j.Hr = lte_eval_k<1, 0>(k, s.xi, s.eta);
  j.HT = lte_eval_k<0, 1>(k, s.xi, s.eta);
  j.Hrr = lte_eval_k<2, 0>(k, s.xi, s.eta);
  j.HrT = lte_eval_k<1, 1>(k, s.xi, s.eta);
  const double m = j.HrT;
  j.c2 = 2 * s.rho * j.Hr + s.rho * s.rho * j.Hrr - s.rho * s.rho * m * m / lte_eval_k<0, 2>(k, s.xi, s.eta);
  return j;
}

// g[0..3] = (p: d/drho, d/dbeta; g: d/drho, d/dbeta); jl, jr: lte_jet of
// left and right
THX_HD void lte_discrete_gradients(const LteDev &t, const LteEval &left, const LteEval &right,
                                    const LteJet &jl, const LteJet &jr, double *g) {
  const bool rev = left.rho > right.rho || (left.rho == right.rho && left.T > right.T);
  const LteEval &A = rev ? right : left;
  const LteEval &B = rev ? left : right;
  const LteJet &JA = rev ? jr : jl;
  const LteJet &JB = rev ? jl : jr;
  const double b1 = 1 / A.T, b2 = 1 / B.T;
  const double dr = B.rho - A.rho, db = b2 - b1;
  const double rmx = A.rho > B.rho ? A.rho : B.rho;
  const double bmx = b1 > b2 ? b1 : b2;
  const bool ddiff = fabs(dr) >= 2.22e-15 + 1.49e-8 * rmx;
  const bool bdiff = fabs(db) >= 2.22e-15 + 1.49e-8 * bmx;
  // f11, f22: pressure and Gibbs energy at the endpoints
  const double p11 = A.rho * A.rho * JA.Hr, p22 = B.rho * B.rho * JB.Hr;
  const double g11 = JA.H + A.rho * JA.Hr, g22 = JB.H + B.rho * JB.Hr;
  double pr = 0.0, pb = 0.0, gr = 0.0, gb = 0.0;
  if (A.cell.off == B.cell.off) {
    const LteCorners k = lte_corners(t, A.cell);
    const double r1 = A.rho, r2 = B.rho;
    if (ddiff) {
      double ps[2], gs[2];
#pragma unroll
      for (int side = 0; side < 2; ++side) {
        const double eta = side == 0 ? A.eta : B.eta;
        const double mean_hr = 0.5 * (lte_eval_k<1, 0>(k, A.xi, eta) + lte_eval_k<1, 0>(k, B.xi, eta));
        const double div_hr = lte_divided_k<0, 1, 0>(k, A.xi, eta, B.xi, eta);
        const double div_h = lte_divided_k<0, 0, 0>(k, A.xi, eta, B.xi, eta);
        ps[side] = 0.5 * (r1 * r1 + r2 * r2) * div_hr + (r1 + r2) * mean_hr;
        gs[side] = div_h + 0.5 * (r1 + r2) * div_hr + mean_hr;
      }
      pr = 0.5 * (ps[0] * b1 + ps[1] * b2);
      gr = 0.5 * (gs[0] * b1 + gs[1] * b2);
    }
    if (bdiff) {
      const double mean_t = 0.5 * (A.T + B.T);
      double ps[2], gs[2];
#pragma unroll
      for (int side = 0; side < 2; ++side) {
        const double xi = side == 0 ? A.xi : B.xi;
        const double rho = side == 0 ? A.rho : B.rho;
        const double mean_hr = 0.5 * (lte_eval_k<1, 0>(k, xi, A.eta) + lte_eval_k<1, 0>(k, xi, B.eta));
        const double div_hr = lte_divided_k<1, 1, 0>(k, xi, A.eta, xi, B.eta);
        const double hr_beta = mean_hr - mean_t * div_hr;
        const double mean_h = 0.5 * (lte_eval_k<0, 0>(k, xi, A.eta) + lte_eval_k<0, 0>(k, xi, B.eta));
        const double div_h = lte_divided_k<1, 0, 0>(k, xi, A.eta, xi, B.eta);
        ps[side] = rho * rho * hr_beta;
        gs[side] = mean_h - mean_t * div_h + rho * hr_beta;
      }
      pb = 0.5 * (ps[0] + ps[1]);
      gb = 0.5 * (gs[0] + gs[1]);
    }
  } else if (ddiff || bdiff) {
    const LteEval s12 = lte_cross(A, B), s21 = lte_cross(B, A);
    const LteCorners k12 = lte_corners(t, s12.cell), k21 = lte_corners(t, s21.cell);
    const double hr12 = lte_eval_k<1, 0>(k12, s12.xi, s12.eta);
    const double hr21 = lte_eval_k<1, 0>(k21, s21.xi, s21.eta);
    const double p12 = s12.rho * s12.rho * hr12, p21 = s21.rho * s21.rho * hr21;
    const double g12 = lte_eval_k<0, 0>(k12, s12.xi, s12.eta) + s12.rho * hr12;
    const double g21 = lte_eval_k<0, 0>(k21, s21.xi, s21.eta) + s21.rho * hr21;
    if (ddiff) {
      pr = 0.5 * ((p21 * b1 - p11 * b1) + (p22 * b2 - p12 * b2)) / dr;
      gr = 0.5 * ((g21 * b1 - g11 * b1) + (g22 * b2 - g12 * b2)) / dr;
    }
    if (bdiff) {
      pb = 0.5 * ((p12 * b2 - p11 * b1) + (p22 * b2 - p21 * b1)) / db;
      gb = 0.5 * ((g12 * b2 - g11 * b1) + (g22 * b2 - g21 * b1)) / db;
    }
  }
  if (!ddiff) {
    const double dpA = 2 * A.rho * JA.Hr + A.rho * A.rho * JA.Hrr;
    const double dpB = 2 * B.rho * JB.Hr + B.rho * B.rho * JB.Hrr;
    const double dgA = 2 * JA.Hr + A.rho * JA.Hrr, dgB = 2 * JB.Hr + B.rho * JB.Hrr;
    pr = 0.5 * (dpA * b1 + dpB * b2);
    gr = 0.5 * (dgA * b1 + dgB * b2);
  }
  if (!bdiff) {
    const double dpA = A.rho * A.rho * JA.HrT, dpB = B.rho * B.rho * JB.HrT;
    const double dgA = JA.HT + A.rho * JA.HrT, dgB = JB.HT + B.rho * JB.HrT;
    pb = 0.5 * ((p11 - A.T * dpA) + (p22 - B.T * dpB));
    gb = 0.5 * ((g11 - A.T * dgA) + (g22 - B.T * dgB));
  }
  g[0] = pr;
  g[1] = pb;
  g[2] = gr;
  g[3] = gb;
}

// LTEEC flux from two evaluated endpoints with their jets (lte_jet): FACE
// uses the normal d1 and the Lax dissipation; the volume form averages the
// two metric rows.
template <int DIM, bool FACE>
THX_HD void lte_ec_flux(const LteDev &t, const double *q1, const double *q2, const LteEval &s1,
                        const LteEval &s2, const LteJet &j1, const LteJet &j2, const double *d1,
                        const double *d2, double *F) {
  double dg[4];
  lte_discrete_gradients(t, s1, s2, j1, j2, dg);
  const double pr = dg[0], pb = dg[1], gr = dg[2], gb = dg[3];
  // p = rho^2 H_rho
  const double p1 = s1.rho * s1.rho * j1.Hr, p2 = s2.rho * s2.rho * j2.Hr;
  const double rho_mean = pr / gr;
  const double e_mean = gb - pb / rho_mean;
  double c1 = 0, c2 = 0;
  if (FACE) { c1 = sqrt(j1.c2); c2 = sqrt(j2.c2); }  // j1, j2 from lte_face_jet
  const double pm = 0.5 * (p1 + p2);
  double vn = 0, ck = 0, pw = 0, v1n = 0, v2n = 0, nn = 0;
#pragma unroll
  for (int d = 0; d < DIM; ++d) {
    const double dir = FACE ? d1[d] : 0.5 * (d1[d] + d2[d]);
    const double u1 = q1[1 + d] / q1[0], u2 = q2[1 + d] / q2[0];
    vn += 0.5 * (u1 + u2) * dir;
    ck += 0.5 * u1 * u2;
    pw += 0.5 * (p1 * u2 + p2 * u1) * dir;
    if (FACE) { v1n += u1 * dir; v2n += u2 * dir; nn += dir * dir; }
  }
  double dis = 0.0;
  if (FACE) {
    const double nm = sqrt(nn);
    const double sp1 = fabs(v1n) + c1 * nm, sp2 = fabs(v2n) + c2 * nm;
    dis = 0.5 * (sp1 > sp2 ? sp1 : sp2);
  }
  const double mf = rho_mean * vn;
  F[0] = mf - dis * (q2[0] - q1[0]);
#pragma unroll
  for (int d = 0; d < DIM; ++d) {
    const double dir = FACE ? d1[d] : 0.5 * (d1[d] + d2[d]);
    const double v = 0.5 * (q1[1 + d] / q1[0] + q2[1 + d] / q2[0]);
    F[1 + d] = mf * v + pm * dir - dis * (q2[1 + d] - q1[1 + d]);
  }
  F[DIM + 1] = mf * (e_mean + ck) + pw - dis * (q2[DIM + 1] - q1[DIM + 1]);
}

#undef THX_HD
#undef THX_HDC

}  // namespace thx
