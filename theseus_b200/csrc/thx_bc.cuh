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
  double *fstar;           // [f][eq][fp]
  GasT<double> gas;
};

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

template <int DIM, int SURF>
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
  bc_inviscid<DIM, SURF>(a.gas, a.bcs[a.bdr_bc[b]], a.bc_data, q, n, F);
  const int f = a.f0 + b;
#pragma unroll
  for (int k = 0; k < NEQ; ++k) a.fstar[((long long)f * NEQ + k) * nfp + fp] = F[k];
}

}  // namespace thx
