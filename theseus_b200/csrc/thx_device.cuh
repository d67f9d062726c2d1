// thx_device.cuh -- pointwise device arithmetic of the DGSEM right-hand side:
// ideal-gas model, logarithmic mean, two-point volume fluxes, Riemann
// (surface) fluxes and the Navier-Stokes viscous flux.  Templated on the
// arithmetic type R (double for the FP64 path, float for the FP32-mixed path).
//
// Formulas follow the reference's device functions (paths relative to the
// reference project root); the per-node quantities that the reference
// recomputes inside every pair (velocity, pressure, beta) are computed once per
// node by node_prims and passed to the pair fluxes, with identical arithmetic.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

#include "thx_lte.cuh"

namespace thx {

constexpr int MAXEQ = 5;

// include/Physics.hpp:22-35, include/Transport.hpp, include/EOS.hpp
template <typename R>
struct GasT {
  R gamma, gm1, gm1_inv, R_gas, cp, Pr_inv, mu, mu0, mu_bulk, T0, Ts;
  R gm1_av_inv;   // 2/(gamma+gamma-2): Chandrashekar's averaged 1/(gamma-1)
  R inv_gm1;      // 1/(gamma-1)
  R cv;           // cp/gamma
  int sutherland;
  // FP32 working copies hold u - qref (a caller-chosen constant state);
  // ke_ref and p_ref are its kinetic energy density and pressure.  Zero and
  // unused in FP64.
  R qref[5];
  R ke_ref, p_ref;
  // FP32 perturbation form (pert = 1): the fluxes are evaluated as
  // G = F - F(qref), from the deviations of the state from qref, whose
  // primitive values follow (rho_r, v_r, p_r, beta_r = rho_r/(2 p_r),
  // h_r = Chandrashekar's averaged enthalpy of qref with itself, Hr = E_r + p_r)
  int pert;
  R rho_r, v_r[3], p_r, beta_r, h_r, Hr;
  // LTE Helmholtz gas (FP64 only): the device table and the per-node
  // temperatures recovered once per right-hand side, [elem][node].
  LteDev lte{};
  const double *Tn = nullptr;
  // table cell (lte_at's cell.off) of (rho, Tn) per node, written with Tn;
  // -1 where lte_at finds none
  const int *Cn = nullptr;
};

// The FP32-mixed path carries the state as an offset from qref and the
// pressure as its fluctuation pp = p - p_ref; the FP64 path carries neither.
template <typename R> struct IsF32 { static constexpr bool value = false; };
template <> struct IsF32<float> { static constexpr bool value = true; };
template <typename R, int DIM> constexpr int nprim() { return DIM + 3 + (IsF32<R>::value ? 1 : 0); }

// FP32 division: the fast reciprocal form (2 ulp), one special-function
// instruction instead of the IEEE sequence, which shortens the
// instruction-issue-bound FP32 kernels.  FP64 keeps IEEE division, so the
// FP64 path is unchanged.
template <typename R> __device__ __forceinline__ R fdiv(R a, R b) { return a / b; }
template <> __device__ __forceinline__ float fdiv(float a, float b) { return __fdividef(a, b); }

template <typename R> __device__ __forceinline__ R rsqrt_(R x);
template <> __device__ __forceinline__ double rsqrt_(double x) { return sqrt(x); }
template <> __device__ __forceinline__ float rsqrt_(float x) { return sqrtf(x); }
__device__ __forceinline__ double rlog(double x) { return log(x); }
__device__ __forceinline__ float rlog(float x) { return logf(x); }
__device__ __forceinline__ double rexp(double x) { return exp(x); }
__device__ __forceinline__ float rexp(float x) { return expf(x); }
template <typename R> __device__ __forceinline__ R rabs(R x) { return x < R(0) ? -x : x; }
template <typename R> __device__ __forceinline__ R rmax(R a, R b) { return a > b ? a : b; }

// include/theseus_kernels.hpp:106-123.  In FP32 the series branch (equal
// arguments, where the closed form cancels) is evaluated in FP64.
__device__ __forceinline__ double log_mean(double x, double y) {
  const double xi = y / x;
  const double u = (xi * (xi - 2.0) + 1.0) / (xi * (xi + 2.0) + 1.0);
  if (u < 1e-4) {
    const double denom = 105.0 + u * (35.0 + u * (21.0 + 15.0 * u));
    return (x + y) * 52.5 / denom;
  }
  return (y - x) / log(xi);
}
// FP32 path: the same function with f = (xi-1)/(xi+1) = (y-x)/(y+x) formed
// directly (one division; y-x is exact for near-equal arguments) and
// u = f^2.  The near-equal series is evaluated in FP64: its argument u < 1e-4
// only scales corrections of relative size u/3, so it is formed in FP32; and
// with eps = u (35 + u (21 + 15 u)) / 105 <= 3.4e-5, 52.5 / (105 (1 + eps)) =
// (1 - eps + eps^2) / 2 to a relative 4e-14, far below the FP32 result's
// rounding, without an FP64 division.
__device__ __forceinline__ float log_mean(float x, float y) {
  const float s = x + y, d = y - x;
  const float f = fdiv(d, s);
  const float u = f * f;
  if (u < 1e-4f) {
    const double ud = u;
    const double eps = ud * (35.0 + ud * (21.0 + 15.0 * ud)) * (1.0 / 105.0);
    return s * (float)(0.5 * (1.0 - eps + eps * eps));
  }
  return fdiv(d, logf(fdiv(y, x)));
}

// ---- gas functions on a conserved state q[DIM+2] -------------------------
template <typename R, int DIM>
__device__ __forceinline__ R ke_density(const R *q) {
  R m2 = R(0);
#pragma unroll
  for (int d = 0; d < DIM; ++d) m2 += q[1 + d] * q[1 + d];
  return fdiv(R(0.5) * m2, q[0]);
}
template <typename R, int DIM>
__device__ __forceinline__ R pressure(const GasT<R> &g, const R *q) {
  return g.gm1 * (q[DIM + 1] - ke_density<R, DIM>(q));
}
template <typename R, int DIM>
__device__ __forceinline__ R sound_speed(const GasT<R> &g, const R *q) {
  return rsqrt_(g.gamma * pressure<R, DIM>(g, q) / q[0]);
}
template <typename R, int DIM>
__device__ __forceinline__ R viscosity(const GasT<R> &g, const R *q) {
  if (g.sutherland) {
    const R T = pressure<R, DIM>(g, q) / (q[0] * g.R_gas);
    const R Trel = T / g.T0;
    const R T0pTs = g.T0 + g.Ts;
    return g.mu0 * T0pTs * Trel * rsqrt_(Trel) / (T + g.Ts);
  }
  return g.mu;
}

// Per-node data used by the volume kernel (node_prims): density, velocity,
// pressure and one flux-specific auxiliary (beta = rho/(2p) for Chandrashekar,
// specific enthalpy e + p/rho for Pirozzoli, total enthalpy (rhoE+p)/rho for
// central), plus in FP32 the pressure fluctuation p - p_ref.

enum VolKind { VOL_CHANDRASHEKAR = 0, VOL_RANOCHA = 1, VOL_PIROZZOLI = 2, VOL_CENTRAL = 3,
               VOL_LTEEC = 4 };

template <typename R, int DIM, int VOL>
__device__ __forceinline__ void node_prims(const GasT<R> &g, const R *raw, R *out /*[nprim]*/) {
  if constexpr (IsF32<R>::value) {
    R q[DIM + 2];
#pragma unroll
    for (int k = 0; k < DIM + 2; ++k) q[k] = g.qref[k] + raw[k];
    const R rho = q[0];
    const R ke = ke_density<R, DIM>(q);
    const R pp = g.gm1 * (raw[DIM + 1] - (ke - g.ke_ref));
    const R p = g.p_ref + pp;
    if (VOL == VOL_CHANDRASHEKAR && g.pert) {
      // perturbation form: rho, dv = v - v_r, beta, dbeta = beta - beta_r,
      // drho; the pressure deviation from the kinetic-energy deviation
      // ke - ke_r = drho |v|^2/2 + rho_r (v_r.dv + |dv|^2/2), free of the
      // cancellation of ke - ke_r formed from the two
      R dv[DIM];
      R v2 = R(0), vrdv = R(0), dvdv = R(0);
#pragma unroll
      for (int d = 0; d < DIM; ++d) {
        dv[d] = fdiv(raw[1 + d] - raw[0] * g.v_r[d], rho);
        const R v = g.v_r[d] + dv[d];
        v2 += v * v;
        vrdv += g.v_r[d] * dv[d];
        dvdv += dv[d] * dv[d];
      }
      const R dke = R(0.5) * raw[0] * v2 + g.rho_r * (vrdv + R(0.5) * dvdv);
      const R ppp = g.gm1 * (raw[DIM + 1] - dke);
      const R pq = g.p_r + ppp;
      out[0] = rho;
#pragma unroll
      for (int d = 0; d < DIM; ++d) out[1 + d] = dv[d];
      out[DIM + 1] = fdiv(R(0.5) * rho, pq);
      out[DIM + 2] = fdiv(R(0.5) * (raw[0] * g.p_r - g.rho_r * ppp), pq * g.p_r);
      out[DIM + 3] = raw[0];
      return;
    }
    out[0] = rho;
#pragma unroll
    for (int d = 0; d < DIM; ++d) out[1 + d] = fdiv(q[1 + d], rho);
    out[DIM + 1] = p;
    if (VOL == VOL_CHANDRASHEKAR) out[DIM + 2] = fdiv(R(0.5) * rho, p);
    else if (VOL == VOL_PIROZZOLI) out[DIM + 2] = fdiv(p * g.gm1_inv, rho) + fdiv(p, rho);
    else if (VOL == VOL_CENTRAL) out[DIM + 2] = (q[DIM + 1] + p) * fdiv(R(1), rho);
    else out[DIM + 2] = R(0);
    out[DIM + 3] = pp;
  } else {
    const R *q = raw;
    const R rho = q[0];
    R v[DIM];
#pragma unroll
    for (int d = 0; d < DIM; ++d) v[d] = q[1 + d] / rho;
    const R ke = ke_density<R, DIM>(q);
    const R p = g.gm1 * (q[DIM + 1] - ke);
    out[0] = rho;
#pragma unroll
    for (int d = 0; d < DIM; ++d) out[1 + d] = v[d];
    out[DIM + 1] = p;
    if (VOL == VOL_CHANDRASHEKAR) out[DIM + 2] = R(0.5) * rho / p;
    else if (VOL == VOL_PIROZZOLI) out[DIM + 2] = (q[DIM + 1] - ke) / rho + p / rho;
    else if (VOL == VOL_CENTRAL) out[DIM + 2] = (q[DIM + 1] + p) * (R(1) / rho);
    else out[DIM + 2] = R(0);
  }
}

// Pressure that enters the momentum fluxes: the fluctuation in FP32, p in FP64.
template <typename R, int DIM>
__device__ __forceinline__ R mom_p(const R *a) {
  if constexpr (IsF32<R>::value) return a[DIM + 3];
  else return a[DIM + 1];
}

// ---- FP32 perturbation form ------------------------------------------------
// Log mean of x1 = xr + d1, x2 = xr + d2 and its deviation from xr, both to
// FP32 accuracy relative to their own size: for u = ((x2-x1)/(x2+x1))^2 <
// 1/16 the mean is ((x1+x2)/2) / S(u) with S(u) = artanh(f)/f = sum u^k/(2k+1)
// (f^2 = u; terms through u^6, truncation below 5e-9), so the deviation is
// (d1+d2)/2 - ((x1+x2)/2) (S-1)/S with no cancellation; beyond, the closed
// form, whose deviation is formed by difference.
__device__ __forceinline__ void log_mean_dev(float x1, float x2, float d1, float d2, float xr,
                                             float &val, float &dev) {
  const float s = x1 + x2, d = x2 - x1;
  const float f = fdiv(d, s);
  const float u = f * f;
  if (u < 0.0625f) {
    const float sm1 =
        u * (1.f / 3.f + u * (1.f / 5.f + u * (1.f / 7.f + u * (1.f / 9.f + u * (1.f / 11.f + u * (1.f / 13.f))))));
    const float mean = 0.5f * s;
    val = fdiv(mean, 1.f + sm1);
    dev = 0.5f * (d1 + d2) - val * sm1;
  } else {
    val = fdiv(d, logf(fdiv(x2, x1)));
    dev = val - xr;
  }
}

// Chandrashekar's two-point flux minus its value at the reference state,
// G = F(a, b) - F(ref, ref), from the per-node deviations (node_prims layout
// rho, dv, beta, dbeta, drho):
//   G_rho = drho_ln vn + rho_r dvn
//   G_m   = G_rho vbar + rho_r vn_r dvbar + dp_hat m
//   G_E   = G_rho h_hat + rho_r vn_r dh_hat
// with dp_hat = ((drho1+drho2)/2 - p_r (dbeta1+dbeta2)) / (beta1+beta2) and
// dh_hat = -dbeta_ln g1/(2 beta_ln beta_r) + v_r.dvbar + |dvbar|^2
//          - (|dv1|^2 + |dv2|^2)/4 + (dp_hat rho_r - p_r drho_ln)/(rho_ln rho_r).
template <int DIM>
__device__ __forceinline__ void vol_chandrashekar_pert(const GasT<float> &g, const float *a, const float *b,
                                                       const float *met, float *F) {
  float rho_ln, drho_ln, beta_ln, dbeta_ln;
  log_mean_dev(a[0], b[0], a[DIM + 3], b[DIM + 3], g.rho_r, rho_ln, drho_ln);
  log_mean_dev(a[DIM + 1], b[DIM + 1], a[DIM + 2], b[DIM + 2], g.beta_r, beta_ln, dbeta_ln);
  float dvb[DIM], vb[DIM];
  float dvn = 0.f, vnr = 0.f, vrdv = 0.f, dv2 = 0.f, dvs = 0.f;
#pragma unroll
  for (int d = 0; d < DIM; ++d) {
    const float d1 = a[1 + d], d2 = b[1 + d];
    dvb[d] = 0.5f * (d1 + d2);
    vb[d] = g.v_r[d] + dvb[d];
    dvn += dvb[d] * met[d];
    vnr += g.v_r[d] * met[d];
    vrdv += g.v_r[d] * dvb[d];
    dv2 += dvb[d] * dvb[d];
    dvs += d1 * d1 + d2 * d2;
  }
  const float vn = vnr + dvn;
  const float bsum = a[DIM + 1] + b[DIM + 1];
  const float dph = fdiv(0.5f * (a[DIM + 3] + b[DIM + 3]) - g.p_r * (a[DIM + 2] + b[DIM + 2]), bsum);
  const float Gr = drho_ln * vn + g.rho_r * dvn;
  const float dh = -fdiv(dbeta_ln * g.gm1_av_inv, 2.f * beta_ln * g.beta_r) + vrdv + dv2 - 0.25f * dvs +
                   fdiv(dph * g.rho_r - g.p_r * drho_ln, rho_ln * g.rho_r);
  F[0] = Gr;
#pragma unroll
  for (int d = 0; d < DIM; ++d) F[1 + d] = Gr * vb[d] + g.rho_r * vnr * dvb[d] + dph * met[d];
  F[DIM + 1] = Gr * (g.h_r + dh) + g.rho_r * vnr * dh;
}

// ---- two-point volume fluxes (metric rows already averaged) --------------
// include/ChandrashekarFlux.hpp:20-89
template <typename R, int DIM>
__device__ __forceinline__ void vol_chandrashekar(const GasT<R> &g, const R *a, const R *b,
                                                  const R *met, R *F) {
  if constexpr (IsF32<R>::value) {
    if (g.pert) {
      vol_chandrashekar_pert<DIM>(g, a, b, met, F);
      return;
    }
  }
  const R rho1 = a[0], rho2 = b[0];
  const R rho_ln = log_mean(rho1, rho2);
  R mom_hat[DIM];
  R h_hat = R(0), vn = R(0);
#pragma unroll
  for (int d = 0; d < DIM; ++d) {
    const R v1 = a[1 + d], v2 = b[1 + d];
    const R vbar = R(0.5) * (v1 + v2);
    vn += vbar * met[d];
    mom_hat[d] = rho_ln * vbar;
    h_hat += -R(0.25) * (v1 * v1 + v2 * v2) + vbar * vbar;
  }
  const R beta1 = a[DIM + 2], beta2 = b[DIM + 2];
  const R beta_ln = log_mean(beta1, beta2);
  const R p_hat = fdiv(R(0.5) * (rho1 + rho2), beta1 + beta2);
  h_hat += fdiv(R(0.5), beta_ln) * g.gm1_av_inv + fdiv(p_hat, rho_ln);
  // FP32: p_hat - p_ref = (beta1 pp1 + beta2 pp2)/(beta1 + beta2), exactly
  R p_mom = p_hat;
  if constexpr (IsF32<R>::value) p_mom = fdiv(beta1 * a[DIM + 3] + beta2 * b[DIM + 3], beta1 + beta2);
  F[0] = rho_ln * vn;
#pragma unroll
  for (int d = 0; d < DIM; ++d) F[1 + d] = vn * mom_hat[d] + p_mom * met[d];
  F[DIM + 1] = rho_ln * vn * h_hat;
}

// include/RanochaFlux.hpp:20-79
template <typename R, int DIM>
__device__ __forceinline__ void vol_ranocha(const GasT<R> &g, const R *a, const R *b,
                                            const R *met, R *F) {
  const R rho1 = a[0], rho2 = b[0];
  const R rho_ln = log_mean(rho1, rho2);
  const R p1 = a[DIM + 1], p2 = b[DIM + 1];
  const R pbar = R(0.5) * (p1 + p2);
  R vbar[DIM];
  R ke = R(0), vn = R(0), fe = R(0);
#pragma unroll
  for (int d = 0; d < DIM; ++d) {
    const R v1 = a[1 + d], v2 = b[1 + d];
    vbar[d] = R(0.5) * (v1 + v2);
    vn += vbar[d] * met[d];
    ke += R(0.5) * (v1 * v2);
    fe += (R(0.5) * (p1 * v2 + p2 * v1)) * met[d];
  }
  const R inv_beta_ln = fdiv(p1 * p2, log_mean(rho1 * p2, rho2 * p1));
  const R ie = inv_beta_ln * g.inv_gm1;
  const R p_mom = IsF32<R>::value ? R(0.5) * (mom_p<R, DIM>(a) + mom_p<R, DIM>(b)) : pbar;
  F[0] = rho_ln * vn;
#pragma unroll
  for (int d = 0; d < DIM; ++d) F[1 + d] = rho_ln * vn * vbar[d] + p_mom * met[d];
  F[DIM + 1] = fe + rho_ln * (ie + ke) * vn;
}

// include/PirozzoliFlux.hpp:19-71
template <typename R, int DIM>
__device__ __forceinline__ void vol_pirozzoli(const GasT<R> &g, const R *a, const R *b,
                                              const R *met, R *F) {
  const R rho_mean = R(0.5) * (a[0] + b[0]);
  const R pbar = R(0.5) * (a[DIM + 1] + b[DIM + 1]);
  R vbar[DIM];
  R ke_mean = R(0), vn = R(0);
#pragma unroll
  for (int d = 0; d < DIM; ++d) {
    const R v1 = a[1 + d], v2 = b[1 + d];
    vbar[d] = R(0.5) * (v1 + v2);
    vn += vbar[d] * met[d];
    ke_mean += R(0.25) * ((v1 * v1) + (v2 * v2));
  }
  const R h_mean = R(0.5) * (a[DIM + 2] + b[DIM + 2]);
  const R p_mom = IsF32<R>::value ? R(0.5) * (mom_p<R, DIM>(a) + mom_p<R, DIM>(b)) : pbar;
  F[0] = rho_mean * vn;
#pragma unroll
  for (int d = 0; d < DIM; ++d) F[1 + d] = rho_mean * vn * vbar[d] + p_mom * met[d];
  F[DIM + 1] = rho_mean * (h_mean + ke_mean) * vn;
}

// Central flux of HLL/LLF/Roe (include/HLLFlux.hpp:21-51): average of the
// physical Euler fluxes contracted with the averaged metric.  qa/qb are the
// conserved states, a/b the node data (aux = total enthalpy H).
template <typename R, int DIM>
__device__ __forceinline__ void vol_central(const R *qa, const R *qb, const R *a, const R *b,
                                            const R *met, R *F) {
  const R ia = fdiv(R(1), a[0]), ib = fdiv(R(1), b[0]);
  R acc0 = R(0), accE = R(0);
  R accm[DIM];
#pragma unroll
  for (int i = 0; i < DIM; ++i) accm[i] = R(0);
#pragma unroll
  for (int d = 0; d < DIM; ++d) {
    acc0 += R(0.5) * (qa[1 + d] + qb[1 + d]) * met[d];
#pragma unroll
    for (int i = 0; i < DIM; ++i) {
      R fa = qa[1 + i] * qa[1 + d] * ia, fb = qb[1 + i] * qb[1 + d] * ib;
      if (i == d) { fa += mom_p<R, DIM>(a); fb += mom_p<R, DIM>(b); }
      accm[i] += R(0.5) * (fa + fb) * met[d];
    }
    accE += R(0.5) * (qa[1 + d] * a[DIM + 2] + qb[1 + d] * b[DIM + 2]) * met[d];
  }
  F[0] = acc0;
#pragma unroll
  for (int i = 0; i < DIM; ++i) F[1 + i] = accm[i];
  F[DIM + 1] = accE;
}

// ---- surface fluxes ------------------------------------------------------
// A face state: the conserved state q, its raw stored form d (FP32: the
// offset u - qref, so that jumps d2 - d1 are exact; FP64: q itself), the
// pressure p and the pressure entering momentum fluxes pp (FP32: p - p_ref).
template <typename R, int DIM>
struct FState {
  R q[DIM + 2], d[DIM + 2], p, pp;
  R dv[DIM];  // FP32 perturbation form: v - v_r
};

template <typename R, int DIM>
__device__ __forceinline__ void make_fstate(const GasT<R> &g, const R *raw, FState<R, DIM> &s) {
  if constexpr (IsF32<R>::value) {
#pragma unroll
    for (int k = 0; k < DIM + 2; ++k) { s.d[k] = raw[k]; s.q[k] = g.qref[k] + raw[k]; }
    if (g.pert) {
      // deviations as in node_prims' perturbation form
      R v2 = R(0), vrdv = R(0), dvdv = R(0);
#pragma unroll
      for (int d = 0; d < DIM; ++d) {
        s.dv[d] = fdiv(raw[1 + d] - raw[0] * g.v_r[d], s.q[0]);
        const R v = g.v_r[d] + s.dv[d];
        v2 += v * v;
        vrdv += g.v_r[d] * s.dv[d];
        dvdv += s.dv[d] * s.dv[d];
      }
      s.pp = g.gm1 * (raw[DIM + 1] - (R(0.5) * raw[0] * v2 + g.rho_r * (vrdv + R(0.5) * dvdv)));
    } else {
      const R ke = ke_density<R, DIM>(s.q);
      s.pp = g.gm1 * (raw[DIM + 1] - (ke - g.ke_ref));
    }
    s.p = g.p_ref + s.pp;
  } else {
#pragma unroll
    for (int k = 0; k < DIM + 2; ++k) { s.d[k] = raw[k]; s.q[k] = raw[k]; }
    s.p = pressure<R, DIM>(g, s.q);
    s.pp = s.p;
  }
}

// Full conserved state from its stored form (adds qref in FP32).
template <typename R, int DIM>
__device__ __forceinline__ void reconstruct(const GasT<R> &g, const R *raw, R *q) {
#pragma unroll
  for (int k = 0; k < DIM + 2; ++k) {
    if constexpr (IsF32<R>::value) q[k] = g.qref[k] + raw[k];
    else q[k] = raw[k];
  }
}

template <typename R, int DIM>
struct NState { R inv_rho, p, pp, H; };

template <typename R, int DIM>
__device__ __forceinline__ NState<R, DIM> nstate(const FState<R, DIM> &f) {
  NState<R, DIM> s;
  s.inv_rho = R(1) / f.q[0];
  s.p = f.p;
  s.pp = f.pp;
  s.H = (f.q[DIM + 1] + s.p) * s.inv_rho;
  return s;
}
// include/NavierStokesFlux.hpp:64-103
template <typename R, int DIM>
__device__ __forceinline__ R normal_flux(const R *q, const NState<R, DIM> &s, const R *n, int eq) {
  R r = R(0);
#pragma unroll
  for (int dir = 0; dir < DIM; ++dir) {
    const R m = q[1 + dir];
    R pf;
    if (eq == 0) pf = m;
    else if (eq <= DIM) {
      const int c = eq - 1;
      pf = q[1 + c] * m * s.inv_rho;
      if (c == dir) pf += s.pp;
    } else pf = m * s.H;
    r += pf * n[dir];
  }
  return r;
}

// FP32 perturbation form of normal_flux: component eq of (F(q) - F(q_ref)).n
// from the state's deviations d (raw working copy), dv = v - v_r and the
// pressure deviation pp:
//   mass      d_m.n
//   momentum  d_(m_c) (v.n) + m_rc (dv.n) + pp n_c
//   energy    (d_E + pp)(v.n) + (E_r + p_r)(dv.n)
template <int DIM>
__device__ __forceinline__ float normal_flux_dev(const GasT<float> &g, const FState<float, DIM> &s,
                                                 const NState<float, DIM> &ns, const float *n, int eq) {
  float vn = 0.f, dvn = 0.f, dmn = 0.f;
#pragma unroll
  for (int d = 0; d < DIM; ++d) {
    vn += s.q[1 + d] * ns.inv_rho * n[d];
    dvn += s.dv[d] * n[d];
    dmn += s.d[1 + d] * n[d];
  }
  if (eq == 0) return dmn;
  if (eq <= DIM) return s.d[eq] * vn + g.qref[eq] * dvn + s.pp * n[eq - 1];
  return (s.d[DIM + 1] + s.pp) * vn + g.Hr * dvn;
}

// component eq of the normal flux: F(q).n (FP64; FP32 without a reference
// state, the pressure entering as its fluctuation) or its deviation
// (FP32 perturbation form)
template <typename R, int DIM>
__device__ __forceinline__ R normal_flux_s(const GasT<R> &g, const FState<R, DIM> &s,
                                           const NState<R, DIM> &ns, const R *n, int eq) {
  if constexpr (IsF32<R>::value) {
    if (g.pert) return normal_flux_dev<DIM>(g, s, ns, n, eq);
  }
  return normal_flux<R, DIM>(s.q, ns, n, eq);
}

// include/DissipationOperator.hpp:57-172
template <typename R, int DIM>
__device__ __forceinline__ void roe_dissipation(const GasT<R> &g, const FState<R, DIM> &A,
                                                const FState<R, DIM> &B, const R *n, R *diss) {
  const int E = DIM + 1;
  const R *q1 = A.q, *q2 = B.q;
  R vn1 = R(0), vn2 = R(0), vn_roe = R(0), nor_mag = R(0);
  const R rho1 = q1[0], rho2 = q2[0];
  const R p1 = A.p, p2 = B.p;
  const R H1 = (q1[E] + p1) / rho1, H2 = (q2[E] + p2) / rho2;
  R roe[DIM + 2];
  const R ratio = rsqrt_(rho2 / rho1);
  const R a = R(1) / (ratio + R(1));
  const R b = a * ratio;
  roe[0] = ratio * rho1;
  roe[E] = a * H1 + b * H2;
  R del_mom[DIM];
  R ke = R(0);
#pragma unroll
  for (int d = 0; d < DIM; ++d) {
    nor_mag += n[d] * n[d];
    const R v1 = q1[1 + d] / rho1, v2 = q2[1 + d] / rho2;
    del_mom[d] = v2 - v1;
    roe[1 + d] = a * v1 + b * v2;
    ke += R(0.5) * roe[1 + d] * roe[1 + d];
    vn1 += v1 * n[d];
    vn2 += v2 * n[d];
    vn_roe += roe[1 + d] * n[d];
  }
  nor_mag = rsqrt_(nor_mag);
  const R inm = R(1) / nor_mag;
  vn1 *= inm;
  vn2 *= inm;
  vn_roe *= inm;
  const R c_roe = rsqrt_((g.gamma - R(1)) * (roe[E] - ke));
  const R c1 = rsqrt_(g.gamma * p1 / rho1), c2 = rsqrt_(g.gamma * p2 / rho2);
  R e0, e2;
  {
    const R er = vn_roe - c_roe;
    const R eps = rmax(R(0), rmax(er - (vn1 - c1), (vn2 - c2) - er));
    e0 = (rabs(er) < eps) ? R(0.5) * (eps + (er * er) / eps) : rabs(er);
  }
  {
    const R er = vn_roe + c_roe;
    const R eps = rmax(R(0), rmax(er - (vn1 + c1), (vn2 + c2) - er));
    e2 = (rabs(er) < eps) ? R(0.5) * (eps + (er * er) / eps) : rabs(er);
  }
  const R e1 = rabs(vn_roe);
  const R del_rho = B.d[0] - A.d[0];
  const R del_vn = vn2 - vn1;
  const R del_p = B.pp - A.pp;
  const R ov_csq = R(1) / (c_roe * c_roe);
  const R pov_csq = del_p * ov_csq;
  const R rhoc_del_vn = roe[0] * del_vn * c_roe * ov_csq;
  const R aVn = e1 * (del_rho - pov_csq);
  const R aVn_rho = e1 * roe[0];
  const R aL = R(0.5) * (e0 * (pov_csq - rhoc_del_vn));
  const R aR = R(0.5) * (e2 * (pov_csq + rhoc_del_vn));
  diss[0] = R(0.5) * (aVn + aL + aR);
  R de = R(0);
#pragma unroll
  for (int d = 0; d < DIM; ++d) {
    R dm = R(0.5) * (aVn * roe[1 + d] + aVn_rho * (del_mom[d] - n[d] * inm * del_vn));
    dm += R(0.5) * (aL * (roe[1 + d] - n[d] * inm * c_roe) + aR * (roe[1 + d] + n[d] * inm * c_roe));
    diss[1 + d] = dm;
    de += R(0.5) * aVn_rho * (roe[1 + d] * del_mom[d]);
  }
  de -= R(0.5) * aVn_rho * vn_roe * del_vn;
  de += R(0.5) * aVn * ke + R(0.5) * aL * (roe[E] - vn_roe * c_roe) +
        R(0.5) * aR * (roe[E] + vn_roe * c_roe);
  diss[E] = de;
#pragma unroll
  for (int e = 0; e < DIM + 2; ++e) diss[e] *= nor_mag;
}

// include/DissipationOperator.hpp:174-232
template <typename R, int DIM>
__device__ __forceinline__ void scalar_dissipation(const GasT<R> &g, const FState<R, DIM> &A,
                                                   const FState<R, DIM> &B, const R *n, R *diss) {
  const int E = DIM + 1;
  const R *q1 = A.q, *q2 = B.q;
  const R rho1 = q1[0], rho2 = q2[0];
  const R rho_mean = R(0.5) * (rho1 + rho2);
  const R drho = B.d[0] - A.d[0];
  const R p1 = A.p, p2 = B.p;
  R vn1 = R(0), vn2 = R(0), nor_mag = R(0), de = R(0);
#pragma unroll
  for (int d = 0; d < DIM; ++d) {
    nor_mag += n[d] * n[d];
    const R v1 = q1[1 + d] / rho1, v2 = q2[1 + d] / rho2;
    const R dv = v2 - v1;
    const R vbar = R(0.5) * (v1 + v2);
    vn1 += v1 * n[d];
    vn2 += v2 * n[d];
    de += R(0.5) * drho * v1 * v2 + rho_mean * dv * vbar;
  }
  nor_mag = rsqrt_(nor_mag);
  const R lmax = rmax(rabs(vn1) + rsqrt_(g.gamma * p1 / rho1) * nor_mag,
                      rabs(vn2) + rsqrt_(g.gamma * p2 / rho2) * nor_mag);
  const R beta1 = R(0.5) * rho1 / p1, beta2 = R(0.5) * rho2 / p2;
  const R beta_ln = log_mean(beta1, beta2);
  de += R(0.5) * drho * g.inv_gm1 / beta_ln + R(0.5) * rho_mean * g.inv_gm1 * (R(1) / beta2 - R(1) / beta1);
  diss[0] = R(0.5) * lmax * drho;
#pragma unroll
  for (int d = 0; d < DIM; ++d) diss[1 + d] = R(0.5) * lmax * (B.d[1 + d] - A.d[1 + d]);
  diss[E] = de * (R(0.5) * lmax);
}

enum SurfKind { SURF_CHANDRASHEKAR = 0, SURF_RANOCHA = 1, SURF_PIROZZOLI = 2, SURF_HLL = 3,
                SURF_LLF = 4, SURF_ROE = 5, SURF_LTEEC = 6 };

template <typename R, int DIM, int SURF>
__device__ __forceinline__ void surface_flux(const GasT<R> &g, const FState<R, DIM> &A,
                                             const FState<R, DIM> &B, const R *n, R *F) {
  constexpr int E = DIM + 1;
  const R *q1 = A.q, *q2 = B.q;
  if (SURF == SURF_CHANDRASHEKAR) {
    // include/ChandrashekarFlux.hpp:91-155
    const R rho1 = q1[0], rho2 = q2[0];
    const R rho_ln = log_mean(rho1, rho2);
    R mom[DIM];
    R hhat = R(0), vn = R(0);
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
      const R v1 = q1[1 + d] / rho1, v2 = q2[1 + d] / rho2;
      const R vbar = R(0.5) * (v1 + v2);
      vn += vbar * n[d];
      mom[d] = rho_ln * vbar;
      hhat += -R(0.25) * (v1 * v1 + v2 * v2) + vbar * vbar;
    }
    const R p1 = A.p, p2 = B.p;
    const R beta1 = R(0.5) * rho1 / p1, beta2 = R(0.5) * rho2 / p2;
    const R beta_ln = log_mean(beta1, beta2);
    const R p_hat = R(0.5) * (rho1 + rho2) / (beta1 + beta2);
    hhat += R(0.5) / beta_ln * g.gm1_av_inv + p_hat / rho_ln;
    R p_mom = p_hat;
    if constexpr (IsF32<R>::value) p_mom = (beta1 * A.pp + beta2 * B.pp) / (beta1 + beta2);
    R diss[DIM + 2];
    scalar_dissipation<R, DIM>(g, A, B, n, diss);
    F[0] = rho_ln * vn - diss[0];
#pragma unroll
    for (int d = 0; d < DIM; ++d) F[1 + d] = vn * mom[d] + p_mom * n[d] - diss[1 + d];
    F[E] = rho_ln * vn * hhat - diss[E];
  } else if (SURF == SURF_RANOCHA) {
    // include/RanochaFlux.hpp:81-134
    const R rho1 = q1[0], rho2 = q2[0];
    const R rho_ln = log_mean(rho1, rho2);
    const R p1 = A.p, p2 = B.p;
    const R pbar = IsF32<R>::value ? R(0.5) * (A.pp + B.pp) : R(0.5) * (p1 + p2);
    R vbar[DIM];
    R ke = R(0), vn = R(0), fe = R(0);
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
      const R v1 = q1[1 + d] / rho1, v2 = q2[1 + d] / rho2;
      vbar[d] = R(0.5) * (v1 + v2);
      vn += vbar[d] * n[d];
      ke += R(0.5) * (v1 * v2);
      fe += (R(0.5) * (p1 * v2 + p2 * v1)) * n[d];
    }
    const R inv_beta_ln = (p1 * p2) / log_mean(rho1 * p2, rho2 * p1);
    const R ie = inv_beta_ln * g.inv_gm1;
    R diss[DIM + 2];
    roe_dissipation<R, DIM>(g, A, B, n, diss);
    F[0] = rho_ln * vn - diss[0];
#pragma unroll
    for (int d = 0; d < DIM; ++d) F[1 + d] = rho_ln * vn * vbar[d] + pbar * n[d] - diss[1 + d];
    F[E] = fe + (rho_ln * (ie + ke) * vn - diss[E]);
  } else if (SURF == SURF_PIROZZOLI) {
    // include/PirozzoliFlux.hpp:73-120
    const R rho1 = q1[0], rho2 = q2[0];
    const R rho_mean = R(0.5) * (rho1 + rho2);
    const R ke1 = ke_density<R, DIM>(q1), ke2 = ke_density<R, DIM>(q2);
    const R p1 = A.p, p2 = B.p;
    const R pbar = IsF32<R>::value ? R(0.5) * (A.pp + B.pp) : R(0.5) * (p1 + p2);
    R vbar[DIM];
    R ke_mean = R(0), vn = R(0);
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
      const R v1 = q1[1 + d] / rho1, v2 = q2[1 + d] / rho2;
      vbar[d] = R(0.5) * (v1 + v2);
      vn += vbar[d] * n[d];
      ke_mean += R(0.25) * ((v1 * v1) + (v2 * v2));
    }
    R h_mean;
    if constexpr (IsF32<R>::value)
      h_mean = R(0.5) * ((p1 * g.gm1_inv) / rho1 + p1 / rho1 + (p2 * g.gm1_inv) / rho2 + p2 / rho2);
    else
      h_mean = R(0.5) * ((q1[E] - ke1) / rho1 + p1 / rho1 + (q2[E] - ke2) / rho2 + p2 / rho2);
    R diss[DIM + 2];
    roe_dissipation<R, DIM>(g, A, B, n, diss);
    F[0] = rho_mean * vn - diss[0];
#pragma unroll
    for (int d = 0; d < DIM; ++d) F[1 + d] = rho_mean * vn * vbar[d] + pbar * n[d] - diss[1 + d];
    F[E] = rho_mean * (h_mean + ke_mean) * vn - diss[E];
  } else if (SURF == SURF_HLL) {
    // include/HLLFlux.hpp:53-116
    const NState<R, DIM> L = nstate<R, DIM>(A), Rs = nstate<R, DIM>(B);
    R un1 = R(0), un2 = R(0), nn = R(0);
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
      un1 += (q1[1 + d] / q1[0]) * n[d];
      un2 += (q2[1 + d] / q2[0]) * n[d];
      nn += n[d] * n[d];
    }
    const R nm = rsqrt_(nn);
    const R c1 = rsqrt_(g.gamma * L.p / q1[0]) * nm, c2 = rsqrt_(g.gamma * Rs.p / q2[0]) * nm;
    const R sL1 = un1 - c1, sL2 = un2 - c2, sR1 = un1 + c1, sR2 = un2 + c2;
    const R sL = (sL1 < sL2) ? sL1 : sL2;
    const R sR = (sR1 > sR2) ? sR1 : sR2;
#pragma unroll
    for (int e = 0; e < DIM + 2; ++e) {
      const R fn1 = normal_flux_s<R, DIM>(g, A, L, n, e), fn2 = normal_flux_s<R, DIM>(g, B, Rs, n, e);
      if (sL >= R(0)) F[e] = fn1;
      else if (sR <= R(0)) F[e] = fn2;
      else F[e] = (sR * fn1 - sL * fn2 + sL * sR * (B.d[e] - A.d[e])) / (sR - sL);
    }
  } else if (SURF == SURF_LLF) {
    // include/LaxFriedrichsFlux.hpp:188-211, include/NavierStokesFlux.hpp:16-41
    const NState<R, DIM> L = nstate<R, DIM>(A), Rs = nstate<R, DIM>(B);
    R vn1 = R(0), vn2 = R(0), nn = R(0);
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
      vn1 += (q1[1 + d] / q1[0]) * n[d];
      vn2 += (q2[1 + d] / q2[0]) * n[d];
      nn += n[d] * n[d];
    }
    const R nm = rsqrt_(nn);
    const R lmax = rmax(rabs(vn1) + rsqrt_(g.gamma * L.p / q1[0]) * nm,
                        rabs(vn2) + rsqrt_(g.gamma * Rs.p / q2[0]) * nm);
#pragma unroll
    for (int e = 0; e < DIM + 2; ++e) {
      const R nl = normal_flux_s<R, DIM>(g, A, L, n, e), nr = normal_flux_s<R, DIM>(g, B, Rs, n, e);
      F[e] = R(0.5) * (nl + nr) - R(0.5) * lmax * (B.d[e] - A.d[e]);
    }
  } else {
    // include/RoeFlux.hpp:42-149
    const NState<R, DIM> left = nstate<R, DIM>(A), right = nstate<R, DIM>(B);
    R nm2 = R(0);
#pragma unroll
    for (int d = 0; d < DIM; ++d) nm2 += n[d] * n[d];
    const R nm = rsqrt_(nm2);
    const R inv_nm = R(1) / nm;
    const R rhoL = q1[0], rhoR = q2[0];
    const R pL = left.p, pR = right.p;
    const R rootL = rsqrt_(rhoL), rootR = rsqrt_(rhoR);
    const R rsi = R(1) / (rootL + rootR);
    const R rho_roe = rootL * rootR;
    const R HL = (q1[E] + pL) / rhoL, HR = (q2[E] + pR) / rhoR;
    const R H = (rootL * HL + rootR * HR) * rsi;
    R u[DIM], du_t[DIM], nh[DIM];
    R u2 = R(0), un = R(0), dun = R(0);
    R du[DIM];
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
      const R uL = q1[1 + d] / rhoL, uR = q2[1 + d] / rhoR;
      nh[d] = n[d] * inv_nm;
      u[d] = (rootL * uL + rootR * uR) * rsi;
      du[d] = uR - uL;
      u2 += u[d] * u[d];
      un += u[d] * nh[d];
      dun += du[d] * nh[d];
    }
    const R a2 = (g.gamma - R(1)) * (H - R(0.5) * u2);
    const R a = rsqrt_(a2);
    const R dp = right.pp - left.pp, drho = B.d[0] - A.d[0];
    const R am = R(0.5) * (dp - rho_roe * a * dun) / a2;
    const R ap = R(0.5) * (dp + rho_roe * a * dun) / a2;
    const R az = drho - dp / a2;
    const R lm = rabs(un - a) * nm, lz = rabs(un) * nm, lp = rabs(un + a) * nm;
#pragma unroll
    for (int d = 0; d < DIM; ++d) du_t[d] = du[d] - dun * nh[d];
    R diss[DIM + 2];
    diss[0] = lm * am + lz * az + lp * ap;
#pragma unroll
    for (int d = 0; d < DIM; ++d)
      diss[1 + d] = lm * am * (u[d] - a * nh[d]) + lz * (az * u[d] + rho_roe * du_t[d]) +
                    lp * ap * (u[d] + a * nh[d]);
    R udt = R(0);
#pragma unroll
    for (int d = 0; d < DIM; ++d) udt += u[d] * du_t[d];
    diss[E] = lm * am * (H - a * un) + lz * (R(0.5) * az * u2 + rho_roe * udt) + lp * ap * (H + a * un);
#pragma unroll
    for (int e = 0; e < DIM + 2; ++e) {
      const R central = R(0.5) * (normal_flux_s<R, DIM>(g, A, left, n, e) + normal_flux_s<R, DIM>(g, B, right, n, e));
      F[e] = central - R(0.5) * diss[e];
    }
  }
}

// ---- viscous flux: include/NavierStokesFlux.hpp:160-290 --------------------
// dp[d*(DIM+2) + eq] = gradient of the primitive (rho, u, p) in direction d.
// Returns vf[eq*DIM + dir]; the mass row is zero.
template <typename R, int DIM>
__device__ __forceinline__ void viscous_flux(const GasT<R> &g, const R *q, const R *dp, R *vf) {
  constexpr int NEQ = DIM + 2, E = DIM + 1;
  const R mu = viscosity<R, DIM>(g, q);
  const R kappa = mu * g.cp * g.Pr_inv;
  const R rho = q[0];
  const R p = pressure<R, DIM>(g, q);
  const R pressor = fdiv(p, rho);
  const R fac = fdiv(g.gm1_inv, g.cv * rho);
  R div = R(0);
#pragma unroll
  for (int i = 0; i < DIM; ++i) div += dp[i * NEQ + 1 + i];
#pragma unroll
  for (int d = 0; d < DIM; ++d) vf[d] = R(0);
#pragma unroll
  for (int dir = 0; dir < DIM; ++dir) {
    R ef = kappa * (fac * (dp[dir * NEQ + E] - pressor * dp[dir * NEQ + 0]));
#pragma unroll
    for (int mom = 0; mom < DIM; ++mom) {
      R tau;
      if (mom == dir) tau = mu * (R(2) * dp[dir * NEQ + 1 + mom] - g.mu_bulk * div);
      else tau = mu * (dp[dir * NEQ + 1 + mom] + dp[mom * NEQ + 1 + dir]);
      vf[(1 + mom) * DIM + dir] = tau;
    }
#pragma unroll
    for (int mom = 0; mom < DIM; ++mom) ef += fdiv(q[1 + mom], rho) * vf[(1 + mom) * DIM + dir];
    vf[E * DIM + dir] = ef;
  }
}

// Per-node gas quantities shared by the entropy-to-primitive gradient map and
// the viscous flux at one node, each formed once: the same operations as
// grad_entropy_to_prim and viscous_flux evaluate (and so the same results),
// without repeating the divisions for every gradient direction.
template <typename R, int DIM>
struct NodeGas {
  R rho, ke, p, p_rho;  // p_rho = p / rho
  R v[DIM];             // q[1+d] / rho
};
template <typename R, int DIM>
__device__ __forceinline__ NodeGas<R, DIM> node_gas(const GasT<R> &g, const R *q) {
  NodeGas<R, DIM> s;
  s.rho = q[0];
  s.ke = ke_density<R, DIM>(q);
  s.p = g.gm1 * (q[DIM + 1] - s.ke);
  s.p_rho = fdiv(s.p, s.rho);
#pragma unroll
  for (int d = 0; d < DIM; ++d) s.v[d] = fdiv(q[1 + d], s.rho);
  return s;
}
// grad_entropy_to_prim with the node's quantities precomputed
template <typename R, int DIM>
__device__ __forceinline__ void grad_entropy_to_prim_ng(const NodeGas<R, DIM> &s, const R *q, const R *dE,
                                                        R *dP) {
  constexpr int E = DIM + 1;
  const R ie = q[E] - s.ke;
  R drho = R(0);
#pragma unroll
  for (int d = 0; d < DIM; ++d) {
    dP[1 + d] = s.p_rho * (dE[1 + d] + s.v[d] * dE[E]);
    drho += q[1 + d] * dP[1 + d];
  }
  drho = s.rho * dE[0] - dE[E] * (s.ke - ie) + fdiv(s.rho * drho, s.p);
  dP[0] = drho;
  dP[E] = s.p_rho * (dP[0] + s.p * dE[E]);
}
// viscosity() with the node's pressure precomputed
template <typename R, int DIM>
__device__ __forceinline__ R viscosity_ng(const GasT<R> &g, const NodeGas<R, DIM> &s) {
  if (g.sutherland) {
    const R T = s.p / (s.rho * g.R_gas);
    const R Trel = T / g.T0;
    const R T0pTs = g.T0 + g.Ts;
    return g.mu0 * T0pTs * Trel * rsqrt_(Trel) / (T + g.Ts);
  }
  return g.mu;
}

// viscous_flux with the node's quantities precomputed
template <typename R, int DIM>
__device__ __forceinline__ void viscous_flux_ng(const GasT<R> &g, const R *q, const NodeGas<R, DIM> &s,
                                                const R *dp, R *vf) {
  constexpr int NEQ = DIM + 2, E = DIM + 1;
  const R mu = viscosity_ng<R, DIM>(g, s);
  const R kappa = mu * g.cp * g.Pr_inv;
  const R fac = fdiv(g.gm1_inv, g.cv * s.rho);
  R div = R(0);
#pragma unroll
  for (int i = 0; i < DIM; ++i) div += dp[i * NEQ + 1 + i];
#pragma unroll
  for (int d = 0; d < DIM; ++d) vf[d] = R(0);
#pragma unroll
  for (int dir = 0; dir < DIM; ++dir) {
    R ef = kappa * (fac * (dp[dir * NEQ + E] - s.p_rho * dp[dir * NEQ + 0]));
#pragma unroll
    for (int mom = 0; mom < DIM; ++mom) {
      R tau;
      if (mom == dir) tau = mu * (R(2) * dp[dir * NEQ + 1 + mom] - g.mu_bulk * div);
      else tau = mu * (dp[dir * NEQ + 1 + mom] + dp[mom * NEQ + 1 + dir]);
      vf[(1 + mom) * DIM + dir] = tau;
    }
#pragma unroll
    for (int mom = 0; mom < DIM; ++mom) ef += s.v[mom] * vf[(1 + mom) * DIM + dir];
    vf[E * DIM + dir] = ef;
  }
}

// include/EOS.hpp:206-234: entropy variables (s_rho, beta*u, -beta), beta = rho/p
template <typename R, int DIM>
__device__ __forceinline__ void entropy_vars(const GasT<R> &g, const R *q, R *w) {
  const R rho = q[0];
  const R ke = ke_density<R, DIM>(q);
  const R p = g.gm1 * (q[DIM + 1] - ke);
  const R s = rlog(p) - g.gamma * rlog(rho);
  const R beta = fdiv(rho, p);
  const R v2o2 = fdiv(ke, rho);
  w[0] = fdiv(g.gamma - s, g.gamma - R(1)) - beta * v2o2;
#pragma unroll
  for (int d = 0; d < DIM; ++d) w[1 + d] = beta * fdiv(q[1 + d], rho);
  w[DIM + 1] = -beta;
}

// include/EOS.hpp:236-263: gradient of entropy variables -> gradient of (rho,u,p)
template <typename R, int DIM>
__device__ __forceinline__ void grad_entropy_to_prim(const GasT<R> &g, const R *q, const R *dE, R *dP) {
  constexpr int E = DIM + 1;
  const R rho = q[0];
  const R ke = ke_density<R, DIM>(q);
  const R p = g.gm1 * (q[E] - ke);
  const R ie = q[E] - ke;
  R drho = R(0);
#pragma unroll
  for (int d = 0; d < DIM; ++d) {
    dP[1 + d] = fdiv(p, rho) * (dE[1 + d] + fdiv(q[1 + d], rho) * dE[E]);
    drho += q[1 + d] * dP[1 + d];
  }
  drho = rho * dE[0] - dE[E] * (ke - ie) + fdiv(rho * drho, p);
  dP[0] = drho;
  dP[E] = fdiv(p, rho) * (dP[0] + p * dE[E]);
}

// Local face index lf (0:x-,1:x+,2:y-,3:y+,4:z-,5:z+) and face point fp ->
// element-local lexicographic node.
template <int DIM>
__device__ __forceinline__ int trace_node(int N, int lf, int fp) {
  const int dir = lf >> 1;
  const int pos = (lf & 1) ? N - 1 : 0;
  if (DIM == 2) return dir == 0 ? pos + N * fp : fp + N * pos;
  const int a = fp % N, b = fp / N;
  if (dir == 0) return pos + N * (a + N * b);
  if (dir == 1) return a + N * (pos + N * b);
  return a + N * (b + N * pos);
}

// ---- LTE Helmholtz gas at a node with its recovered temperature T ---------
// Per-node staging of the LTEEC volume kernel: conserved state, T, the table
// cell of (rho, T) and the free-energy jet there (lte_jet).
enum : int { LTE_P_T = 0, LTE_P_XI = 1, LTE_P_ETA = 2, LTE_P_DR = 3, LTE_P_DT = 4, LTE_P_OFF = 5,
             LTE_P_H = 6, LTE_P_HR = 7, LTE_P_HT = 8, LTE_P_HRR = 9, LTE_P_HRT = 10,
             LTE_P_COUNT = 11 };

__device__ __forceinline__ LteJet lte_unpack_jet(const double *x /* LTE_P_* block */) {
  LteJet j;
  j.H = x[LTE_P_H];
  j.Hr = x[LTE_P_HR];
  j.HT = x[LTE_P_HT];
  j.Hrr = x[LTE_P_HRR];
  j.HrT = x[LTE_P_HRT];
  j.c2 = 0.0;  // volume fluxes do not use it
  return j;
}

__device__ __forceinline__ LteEval lte_unpack(const double *x /* LTE_P_* block */, double rho, int nx) {
  LteEval s;
  s.cell.off = (int)x[LTE_P_OFF];
  s.cell.nx = nx;
  s.cell.dr = x[LTE_P_DR];
  s.cell.dt = x[LTE_P_DT];
  s.xi = x[LTE_P_XI];
  s.eta = x[LTE_P_ETA];
  s.rho = rho;
  s.T = x[LTE_P_T];
  s.valid = true;
  return s;
}

// include/LTEHelmholtzGasEOS.hpp:144-157: (beta (g - |u|^2/2), beta u, -beta)
template <int DIM>
__device__ __forceinline__ void lte_entropy_vars(const LteDev &t, const double *q, double T, int cell,
                                                 double *w) {
  const LteEval s = lte_at_cell(t, q[0], T, cell);
  const double beta = 1 / s.T;
  double m2 = 0.0;
#pragma unroll
  for (int d = 0; d < DIM; ++d) m2 += q[1 + d] * q[1 + d];
  const double kinetic = (0.5 * m2 / q[0]) / q[0];
  w[0] = beta * (lte_gibbs(t, s) - kinetic);
#pragma unroll
  for (int d = 0; d < DIM; ++d) w[1 + d] = beta * (q[1 + d] / q[0]);
  w[DIM + 1] = -beta;
}

// include/LTEHelmholtzGasEOS.hpp:159-172: the energy slot carries grad T
template <int DIM>
__device__ __forceinline__ void lte_grad_entropy_to_prim(const double *q, double T, const double *dE,
                                                         double *dP) {
  constexpr int E = DIM + 1;
  dP[0] = 0.0;
#pragma unroll
  for (int d = 0; d < DIM; ++d) dP[1 + d] = T * dE[1 + d] + T * (q[1 + d] / q[0]) * dE[E];
  dP[E] = T * T * dE[E];
}

// include/NavierStokesFlux.hpp:160-290 with the LTE transport planes
// (include/LTETransport.hpp:33-65) and grad T taken from the energy slot
// (include/LTEHelmholtzGasEOS.hpp:133-142).
template <int DIM>
__device__ __forceinline__ void lte_viscous_flux(const GasT<double> &g, const double *q, double T,
                                                 int cell, const double *dp, double *vf) {
  constexpr int NEQ = DIM + 2, E = DIM + 1;
  const LteEval s = lte_at_cell(g.lte, q[0], T, cell);
  const double mu = lte_transport(g.lte, s, 4);
  const double kappa = lte_transport(g.lte, s, 5);
  const double rho = q[0];
  double div = 0.0;
#pragma unroll
  for (int i = 0; i < DIM; ++i) div += dp[i * NEQ + 1 + i];
#pragma unroll
  for (int d = 0; d < DIM; ++d) vf[d] = 0.0;
#pragma unroll
  for (int dir = 0; dir < DIM; ++dir) {
    double ef = kappa * dp[dir * NEQ + E];
#pragma unroll
    for (int mom = 0; mom < DIM; ++mom) {
      double tau;
      if (mom == dir) tau = mu * (2.0 * dp[dir * NEQ + 1 + mom] - g.mu_bulk * div);
      else tau = mu * (dp[dir * NEQ + 1 + mom] + dp[mom * NEQ + 1 + dir]);
      vf[(1 + mom) * DIM + dir] = tau;
    }
#pragma unroll
    for (int mom = 0; mom < DIM; ++mom) ef += (q[1 + mom] / rho) * vf[(1 + mom) * DIM + dir];
    vf[E * DIM + dir] = ef;
  }
}

}  // namespace thx
