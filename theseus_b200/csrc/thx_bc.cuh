// thx_bc.cuh -- boundary conditions at boundary face points (FP64).
//
// One thread per boundary face point evaluates the boundary flux of the
// face's condition from the interior trace and stores it where the volume
// kernel's lift reads face fluxes; the lift adds the boundary faces after
// the interior ones.  Restates include/bc_kernels.hpp:138-279 and
// include/Flow.hpp:54-170 in the reference's operation order.
#pragma once
#include "thx_device.cuh"
#include "theseus_b200.h"

namespace thx {

// Kernel arguments of the boundary faces of one case.
struct BndArgs {
  const double *u;         // state L-vector
  int ne, N, nbf;
  int f0;                  // face slot of boundary face 0 in fstar
  const int *bdr_elem, *bdr_lface, *bdr_bc;
  const double *normal;    // [nbf][nfp][dim]
  const thx_bc *bcs;
  const double *bc_data;
  const double *bgrad;     // NS: primitive gradients at the points [nbf][nfp][dim][dim+2]
  double *fstar;           // [f][eq][fp]
  GasT<double> gas;
};

// Exterior minus interior entropy variables w at a boundary point, the jump
// of the BR1 lift (include/bc_kernels.hpp:32-135); zero for the conditions
// without an exterior entropy state.
template <int DIM>
__device__ __forceinline__ void bc_grad_flux(const GasT<double> &g, const thx_bc &bc, const double *data,
                                             const double *w, double *F) {
  constexpr int NEQ = DIM + 2, E = DIM + 1;
#pragma unroll
  for (int k = 0; k < NEQ; ++k) F[k] = 0.0;
  if (bc.type == THX_BC_PRESCRIBED_STATE) {
    double qb[NEQ], e[NEQ];
#pragma unroll
    for (int k = 0; k < NEQ; ++k) qb[k] = data[bc.data_index + k];
    entropy_vars<double, DIM>(g, qb, e);
#pragma unroll
    for (int k = 0; k < NEQ; ++k) F[k] = e[k] - w[k];
  } else if (bc.type == THX_BC_NOSLIP_ADIABATIC) {
    const double *vw = data + bc.data_index;
    const double v = -w[E];
    F[0] = w[0];
#pragma unroll
    for (int d = 0; d < DIM; ++d) F[1 + d] = vw[d] * v;
    F[E] = -v;
#pragma unroll
    for (int k = 0; k < NEQ; ++k) F[k] -= w[k];
  } else if (bc.type == THX_BC_NOSLIP_ISOTHERMAL) {
    const double *bd = data + bc.data_index;
    const double beta = 1.0 / (g.R_gas * bd[DIM]);  // include/EOS.hpp:41-46
    F[0] = w[0];
#pragma unroll
    for (int d = 0; d < DIM; ++d) F[1 + d] = bd[d] * beta;
    F[E] = -beta;
#pragma unroll
    for (int k = 0; k < NEQ; ++k) F[k] -= w[k];
  }
}

// Normal viscous flux n . F_v from the primitive gradients dp[dir][eq]
// (include/NavierStokesFlux.hpp:296-355, Cartesian), in its own order.
template <int DIM>
__device__ __forceinline__ void viscous_normal_flux(const GasT<double> &g, const double *q, const double *dp,
                                                    const double *n, double *flux) {
  constexpr int NEQ = DIM + 2, E = DIM + 1;
  const double mu = viscosity<double, DIM>(g, q);
  const double kappa = mu * g.cp * g.Pr_inv;
  double divergence = 0.0;
#pragma unroll
  for (int d = 0; d < DIM; ++d) divergence += dp[d * NEQ + 1 + d];
  const double rho = q[0];
  const double pressor = pressure<double, DIM>(g, q) / rho;
  const double fac = g.gm1_inv / (g.cv * rho);
  double gT[DIM];
#pragma unroll
  for (int d = 0; d < DIM; ++d) gT[d] = fac * (dp[d * NEQ + E] - pressor * dp[d * NEQ + 0]);
#pragma unroll
  for (int k = 0; k < NEQ; ++k) flux[k] = 0.0;
  double energy_flux = 0.0;
#pragma unroll
  for (int c = 0; c < DIM; ++c) {
    double traction = 0.0;
#pragma unroll
    for (int d = 0; d < DIM; ++d) {
      const double stress = c == d ? mu * (2.0 * dp[d * NEQ + 1 + c] - g.mu_bulk * divergence)
                                   : mu * (dp[d * NEQ + 1 + c] + dp[c * NEQ + 1 + d]);
      traction += n[d] * stress;
    }
    flux[1 + c] = traction;
    energy_flux += (q[1 + c] / q[0]) * traction;
  }
#pragma unroll
  for (int d = 0; d < DIM; ++d) energy_flux += n[d] * kappa * gT[d];
  flux[E] = energy_flux;
}

// Momentum of the wall-rotated state, component c (include/Flow.hpp:77-150):
// c = 0 along the unit normal, then the tangent chosen by the smallest
// normal component, then their cross product.
template <int DIM>
__device__ __forceinline__ double wall_momentum(const double *q, const double *n, double inv, int c) {
  const double nx = n[0] * inv, ny = n[1] * inv, nz = DIM > 2 ? n[2] * inv : 0.0;
  double x = nx, y = ny, z = nz;
  if (c > 0) {
    double tx, ty, tz;
    if (DIM == 2) {
      tx = -ny; ty = nx; tz = 0.0;
    } else if (rabs(nx) <= rabs(ny) && rabs(nx) <= rabs(nz)) {
      tx = 0.0; ty = nz; tz = -ny;
    } else if (rabs(ny) <= rabs(nx) && rabs(ny) <= rabs(nz)) {
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
  if (DIM == 3) r += q[3] * z;
  return r;
}

// p* of the 1-D Riemann problem against a slip wall with (unnormalised)
// normal n (include/Flow.hpp:54-75 on the rotated view, :155-170).
template <int DIM>
__device__ __forceinline__ double slipwall_pstar_normal(const GasT<double> &g, const double *q,
                                                       const double *n) {
  double mag2 = 0.0;
#pragma unroll
  for (int d = 0; d < DIM; ++d) mag2 += n[d] * n[d];
  if (mag2 == 0.0) return 0.0;
  const double inv = 1.0 / sqrt(mag2);
  const double rho = q[0];
  double m2 = 0.0;
#pragma unroll
  for (int c = 0; c < DIM; ++c) {
    const double m = wall_momentum<DIM>(q, n, inv, c);
    m2 += m * m;
  }
  const double ke = 0.5 * m2 / rho;
  const double p = g.gm1 * (q[DIM + 1] - ke);
  const double c = sqrt(g.gamma * p / rho);
  const double v = wall_momentum<DIM>(q, n, inv, 0) / rho;
  const double gamma = g.gamma;
  const double gammaP1 = gamma + 1.;
  const double gammaM1 = gamma - 1.;
  const double gammaP1Inverse = 1.0 / gammaP1;
  const double gammaM1Inverse = 1.0 / gammaM1;
  if (v > 0.0)
    return (p + 0.25 * v * gammaP1 * rho *
                    (v + sqrt(v * v + 8.0 * gammaP1Inverse * p * (gammaM1 * gammaP1Inverse + 1.0) / rho)));
  const double base = 1.0 + 0.5 * gammaM1 * v / c;
  return p * pow(base < 0.0001 ? 0.0001 : base, 2.0 * gamma * gammaM1Inverse);
}

// Inviscid boundary flux (include/bc_kernels.hpp:219-279); the surface flux
// is the configured interior one.
template <int DIM, int SURF>
__device__ __forceinline__ void bc_inviscid(const GasT<double> &g, const thx_bc &bc, const double *data,
                                            const double *q, const double *n, double *F) {
  constexpr int NEQ = DIM + 2;
  FState<double, DIM> s1, s2;
  switch (bc.type) {
    case THX_BC_SLIP_WALL: {
      const double ps = slipwall_pstar_normal<DIM>(g, q, n);
#pragma unroll
      for (int k = 0; k < NEQ; ++k) F[k] = 0.0;
#pragma unroll
      for (int d = 0; d < DIM; ++d) F[1 + d] = ps * n[d];
      return;
    }
    case THX_BC_SUPERSONIC_OUTFLOW:
      make_fstate<double, DIM>(g, q, s1);
      surface_flux<double, DIM, SURF>(g, s1, s1, n, F);
      return;
    case THX_BC_PRESCRIBED_STATE:
    case THX_BC_SUPERSONIC_INFLOW: {
      double qb[NEQ];
#pragma unroll
      for (int k = 0; k < NEQ; ++k) qb[k] = data[bc.data_index + k];
      make_fstate<double, DIM>(g, q, s1);
      make_fstate<double, DIM>(g, qb, s2);
      surface_flux<double, DIM, SURF>(g, s1, s2, n, F);
      return;
    }
    case THX_BC_SYMMETRY: {
      // mirror the momentum about the face (include/bc_kernels.hpp:248-271)
      double qb[NEQ], un[DIM];
#pragma unroll
      for (int k = 0; k < NEQ; ++k) qb[k] = q[k];
      double fac = 0.0;
#pragma unroll
      for (int d = 0; d < DIM; ++d) {
        un[d] = n[d];
        fac += (un[d] * un[d]);
      }
      fac = 1.0 / sqrt(fac);
#pragma unroll
      for (int d = 0; d < DIM; ++d) un[d] *= fac;
      double nv = 0.0;
#pragma unroll
      for (int d = 0; d < DIM; ++d) nv += q[1 + d] * un[d];
#pragma unroll
      for (int d = 0; d < DIM; ++d) qb[1 + d] = -2.0 * nv * un[d] + q[1 + d];
      make_fstate<double, DIM>(g, q, s1);
      make_fstate<double, DIM>(g, qb, s2);
      surface_flux<double, DIM, SURF>(g, s1, s2, n, F);
      return;
    }
    default:
#pragma unroll
      for (int k = 0; k < NEQ; ++k) F[k] = 0.0;
      return;
  }
}

// Viscous boundary flux (include/bc_kernels.hpp:154-217, 281-374): the
// inviscid conditions; the exterior state minus the interior viscous flux;
// the no-slip walls from the wall pressure p* and the normal viscous flux
// with the wall's heat flux or temperature.
template <int DIM, int SURF>
__device__ __forceinline__ void bc_viscous(const GasT<double> &g, const thx_bc &bc, const double *data,
                                           const double *q, const double *dp, const double *n, double *F) {
  constexpr int NEQ = DIM + 2, E = DIM + 1;
  switch (bc.type) {
    case THX_BC_PRESCRIBED_STATE: {
      bc_inviscid<DIM, SURF>(g, bc, data, q, n, F);
      double vf[NEQ * DIM];
      viscous_flux<double, DIM>(g, q, dp, vf);
#pragma unroll
      for (int d = 0; d < DIM; ++d) vf[d] = 0.0;  // mass row
#pragma unroll
      for (int k = 0; k < NEQ; ++k)
#pragma unroll
        for (int d = 0; d < DIM; ++d) F[k] -= vf[k * DIM + d] * n[d];
      return;
    }
    case THX_BC_NOSLIP_ADIABATIC: {
      const double *vw = data + bc.data_index;
      const double ps = slipwall_pstar_normal<DIM>(g, q, n);
      viscous_normal_flux<DIM>(g, q, dp, n, F);
      double mag2 = 0.0;
#pragma unroll
      for (int d = 0; d < DIM; ++d) mag2 += n[d] * n[d];
      double ef = vw[DIM] * sqrt(mag2);
#pragma unroll
      for (int d = 0; d < DIM; ++d) ef += vw[d] * F[1 + d];
      F[E] = ef;
#pragma unroll
      for (int k = 0; k < NEQ; ++k) F[k] = -F[k];
#pragma unroll
      for (int d = 0; d < DIM; ++d) F[1 + d] += ps * n[d];
      return;
    }
    case THX_BC_NOSLIP_ISOTHERMAL: {
      const double *vw = data + bc.data_index;
      const double ps = slipwall_pstar_normal<DIM>(g, q, n);
      viscous_normal_flux<DIM>(g, q, dp, n, F);
#pragma unroll
      for (int d = 0; d < DIM; ++d) F[E] -= (q[1 + d] / q[0]) * F[1 + d];
#pragma unroll
      for (int d = 0; d < DIM; ++d) F[E] += vw[d] * F[1 + d];
#pragma unroll
      for (int k = 0; k < NEQ; ++k) F[k] = -F[k];
#pragma unroll
      for (int d = 0; d < DIM; ++d) F[1 + d] += ps * n[d];
      return;
    }
    default:
      bc_inviscid<DIM, SURF>(g, bc, data, q, n, F);
      return;
  }
}

template <int DIM, int SURF, bool NS>
__global__ void __launch_bounds__(128) bnd_face_kernel(const BndArgs a) {
  constexpr int NEQ = DIM + 2;
  const int N = a.N;
  const int nfp = DIM == 2 ? N : N * N;
  const int nd = DIM == 2 ? N * N : N * N * N;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)a.nbf * nfp) return;
  const int b = (int)(t / nfp), fp = (int)(t % nfp);
  const long long L = (long long)a.ne * nd;
  const long long i = (long long)a.bdr_elem[b] * nd + trace_node<DIM>(N, a.bdr_lface[b], fp);
  double q[NEQ], F[NEQ];
#pragma unroll
  for (int k = 0; k < NEQ; ++k) q[k] = a.u[k * L + i];
  const double *n = a.normal + ((long long)b * nfp + fp) * DIM;
  if constexpr (NS)
    bc_viscous<DIM, SURF>(a.gas, a.bcs[a.bdr_bc[b]], a.bc_data, q,
                          a.bgrad + ((long long)b * nfp + fp) * DIM * NEQ, n, F);
  else
    bc_inviscid<DIM, SURF>(a.gas, a.bcs[a.bdr_bc[b]], a.bc_data, q, n, F);
  const int f = a.f0 + b;
#pragma unroll
  for (int k = 0; k < NEQ; ++k) a.fstar[((long long)f * NEQ + k) * nfp + fp] = F[k];
}

}  // namespace thx
