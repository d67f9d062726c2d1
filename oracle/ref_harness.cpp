// ref_harness.cpp -- TEST INFRASTRUCTURE ONLY.
//
// Drives the reference's own header-only kernels (fluxes, gas model,
// DGSEMIntegrator point kernels) compiled from the reference sources with the
// stand-in headers in oracle/ref_shim/.  The MFEM-owned glue (element/face
// restriction and its transpose, face loop) is restated here exactly as in
// the oracle.  Built by oracle/build_ref.sh into oracle/_ref/libthx_ref.so; it
// is used to pin the oracle restatement and to generate tests/golden/.
#include "GasModel.hpp"
#include "DGSEMIntegrator.hpp"
#include "ChandrashekarFlux.hpp"
#include "RanochaFlux.hpp"
#include "PirozzoliFlux.hpp"
#include "RoeFlux.hpp"
#include "HLLFlux.hpp"
#include "LaxFriedrichsFlux.hpp"
#include "LTEGasModel.hpp"
#include "LTEECFlux.hpp"
#include "bc_kernels.hpp"

#include "theseus_b200.h"

#include <vector>

namespace {

using Gas = Theseus::IdealGasModel;

// Runtime-selected (volume, surface) pair built from the reference's own
// per-class kernels.
struct PairFlux {
  int vol = 0, surf = 0;
  template <typename G>
  void ComputeVolumeFlux(const G &g, const double *q1, const double *q2, const double *m1,
                         const double *m2, double *F) const {
    switch (vol) {
      case THX_FLUX_CHANDRASHEKAR: Theseus::ChandrashekarFlux::ComputeVolumeFluxKernel(g, q1, q2, m1, m2, F); break;
      case THX_FLUX_RANOCHA: Theseus::RanochaFlux::ComputeVolumeFluxKernel(g, q1, q2, m1, m2, F); break;
      case THX_FLUX_PIROZZOLI: Theseus::PirozzoliFlux::ComputeVolumeFluxKernel(g, q1, q2, m1, m2, F); break;
      case THX_FLUX_HLL: Theseus::HLLFlux::ComputeVolumeFluxKernel(g, q1, q2, m1, m2, F); break;
      case THX_FLUX_LLF: Theseus::LaxFriedrichsFlux::ComputeVolumeFluxKernel(g, q1, q2, m1, m2, F); break;
      default: Theseus::RoeFlux::ComputeVolumeFluxKernel(g, q1, q2, m1, m2, F); break;
    }
  }
  template <typename G>
  void ComputeFaceFlux(const G &g, const double *qm, const double *qp, const double *n,
                       double *F) const {
    switch (surf) {
      case THX_FLUX_CHANDRASHEKAR: Theseus::ChandrashekarFlux::ComputeFaceFluxKernel(g, qm, qp, n, F); break;
      case THX_FLUX_RANOCHA: Theseus::RanochaFlux::ComputeFaceFluxKernel(g, qm, qp, n, F); break;
      case THX_FLUX_PIROZZOLI: Theseus::PirozzoliFlux::ComputeFaceFluxKernel(g, qm, qp, n, F); break;
      case THX_FLUX_HLL: Theseus::HLLFlux::ComputeFaceFluxKernel(g, qm, qp, n, F); break;
      case THX_FLUX_LLF: Theseus::LaxFriedrichsFlux::ComputeFaceFluxKernel(g, qm, qp, n, F); break;
      default: Theseus::RoeFlux::ComputeFaceFluxKernel(g, qm, qp, n, F); break;
    }
  }
};

// Duck-typed context, the pattern of tests/viscous_volume_tests.cpp:9-17.
template <class GasT, class FluxT>
struct CtxT {
  int dim, num_equations, ndof_scalar_el, Np_x, Np_y, Np_z, num_face_points;
  bool axisymmetric = false;
  GasT gas;
  FluxT iflux;
  const double *D_d, *Dhat_d, *Dhat2_d, *subcell_weights_d;
  const double *bc_vector_d = nullptr, *bc_scalar_d = nullptr;  // boundary payloads
  int iface_idx(int side, int fp, int eq) const {
    return (side * num_equations + eq) * num_face_points + fp;
  }
};
using Ctx = CtxT<Gas, PairFlux>;
using LteGas = Theseus::LTEHelmholtzGas;
using LteCtx = CtxT<LteGas, Theseus::LTEECFlux::InviscidFlux>;

// The reference's table data from the oracle's arrays.
struct LteData {
  Theseus::HelmholtzTable::Data data;
  Theseus::HelmholtzTable::Layout layout;
  explicit LteData(const thx_lte_table *t) {
    layout.nx = t->nx;
    layout.ny = t->ny;
    auto fill = [](mfem::Vector &v, const double *src, int n) {
      v.SetSize(n);
      for (int i = 0; i < n; ++i) v[i] = src[i];
    };
    fill(data.rho_grid, t->rho_grid, t->nx);
    fill(data.T_grid, t->T_grid, t->ny);
    fill(data.e_grid, t->e_grid, t->ny);
    fill(data.lte_table, t->planes, 6 * t->nx * t->ny);
    fill(data.inv_table, t->inverse, t->nx * t->ny);
  }
  LteGas gas(const thx_config &c, int dim) const {
    Theseus::PhysicsConstants phys(c.gamma, c.Pr, c.R_gas, c.mu, c.mu0);
    phys.mu_bulk = c.mu_bulk;
    return LteGas(phys, Theseus::StateLayout(dim, 1), Theseus::HelmholtzTable::HostView(data, layout));
  }
};

Gas make_gas(const thx_config &c, int dim) {
  Theseus::PhysicsConstants phys(c.gamma, c.Pr, c.R_gas, c.mu, c.mu0);
  phys.mu_bulk = c.mu_bulk;
  return Gas(phys, Theseus::StateLayout(dim, 1));
}

// [0,1] LGL rule and operators, passed in by the caller (the same arrays the
// oracle uses), so that only the kernels differ.
struct Setup {
  int dim, N, nd, nfp, neq, ne, nf;
  std::vector<double> D, Dhat, Dhat2, w;
};

int trace_node(int dim, int N, int lf, int fp) {
  const int dir = lf / 2;
  const int pos = (lf % 2) ? N - 1 : 0;
  if (dim == 2) return dir == 0 ? pos + N * fp : fp + N * pos;
  const int a = fp % N, b = fp / N;
  if (dir == 0) return pos + N * (a + N * b);
  if (dir == 1) return a + N * (pos + N * b);
  return a + N * (b + N * pos);
}

}  // namespace

namespace {
// Full RHS on a byNODES L-vector, driving the reference point kernels.
//  D, Dhat, Dhat2: [i*Np+l] operator arrays; w: LGL weights on [0,1]
//  alpha: per-element blending coefficient (NULL = no blending)
//  sub_xi/eta/zeta: subcell metrics in the reference layout
template <class C>
int rhs_impl(const C &ctx, const C &fvctx, const thx_geometry *geo, const thx_config *cfg,
             const double *alpha, const double *sub_xi, const double *sub_eta,
             const double *sub_zeta, const double *u, double *dudt) {
  const int dim = geo->dim, N = geo->order + 1;
  const int nd = dim == 2 ? N * N : N * N * N;
  const int nfp = dim == 2 ? N : N * N;
  const int neq = dim + 2, ne = geo->num_elements, nf = geo->num_faces;
  const size_t L = (size_t)ne * nd;
  const bool ns = cfg->flow_model == THX_FLOW_NAVIER_STOKES;

  // E-vector [e][eq][node] (restr_v->Mult)
  std::vector<double> Ue((size_t)neq * L), dUe((size_t)neq * L, 0.0);
  // faces of each element in ascending (face, side) order: the order in
  // which the serial restriction transpose adds face contributions
  std::vector<std::vector<std::pair<int, int>>> elem_faces(ne);
  for (int f = 0; f < nf; ++f)
    for (int s = 0; s < 2; ++s) elem_faces[geo->face_elem[2 * f + s]].push_back({f, s});
#pragma omp parallel for schedule(static)
  for (int e = 0; e < ne; ++e)
    for (int q = 0; q < neq; ++q)
      for (int a = 0; a < nd; ++a) Ue[((size_t)e * neq + q) * nd + a] = u[q * L + (size_t)e * nd + a];
  const int dd = dim * dim;

  // NS: gradients (E-layout per direction), reference kernels
  std::vector<double> gradE;
  if (ns) {
    std::vector<double> Se((size_t)neq * L);
#pragma omp parallel for schedule(static)
    for (int e = 0; e < ne; ++e)
      for (int a = 0; a < nd; ++a) {
        double q[5], s[5];
        for (int k = 0; k < neq; ++k) q[k] = Ue[((size_t)e * neq + k) * nd + a];
        Theseus::PointStateView S{q};
        Theseus::PointStateViewRW E{s};
        ctx.gas.entropy_state(S, E);
        for (int k = 0; k < neq; ++k) Se[((size_t)e * neq + k) * nd + a] = s[k];
      }
    gradE.assign((size_t)dim * neq * L, 0.0);
#pragma omp parallel for schedule(static)
    for (int e = 0; e < ne; ++e) {
      double *gp[3] = {nullptr, nullptr, nullptr};
      for (int c = 0; c < dim; ++c) gp[c] = gradE.data() + (size_t)c * neq * L + (size_t)e * neq * nd;
      for (int a = 0; a < nd; ++a)
        Theseus::DGSEMIntegrator::AssembleGradVolumePointKernel(
            ctx, Se.data() + (size_t)e * neq * nd, geo->jac + (size_t)e * nd,
            geo->metric + (size_t)e * nd * dd, a, gp);
    }
    // interior-face lift: per face restriction [side][eq][fp], kernel; the
    // transpose adds the stored face results element by element, in face order
    const size_t fstride = (size_t)dim * 2 * neq * nfp;
    std::vector<double> rfall((size_t)nf * fstride);
    std::vector<double> acc((size_t)dim * neq * L, 0.0);
#pragma omp parallel for schedule(static)
    for (int f = 0; f < nf; ++f) {
      std::vector<double> uf(2 * neq * nfp);
      double *rf = rfall.data() + (size_t)f * fstride;
      for (int s = 0; s < 2; ++s) {
        const int e = geo->face_elem[2 * f + s], lf = geo->face_lface[2 * f + s];
        for (int fp = 0; fp < nfp; ++fp)
          for (int q = 0; q < neq; ++q)
            uf[(s * neq + q) * nfp + fp] = Se[((size_t)e * neq + q) * nd + trace_node(dim, N, lf, fp)];
      }
      double *rp[3] = {rf, rf + 2 * neq * nfp, rf + 4 * neq * nfp};
      for (int fp = 0; fp < nfp; ++fp)
        Theseus::DGSEMIntegrator::AssembleGradInteriorFacePointKernel(
            ctx, uf.data(), geo->face_normal + ((size_t)f * nfp + fp) * dim,
            geo->face_wminus[(size_t)f * nfp + fp], geo->face_wplus[(size_t)f * nfp + fp], fp, rp);
    }
#pragma omp parallel for schedule(static)
    for (int e = 0; e < ne; ++e)
      for (const auto &fs : elem_faces[e]) {
        const int f = fs.first, s = fs.second, lf = geo->face_lface[2 * f + s];
        const double *rf = rfall.data() + (size_t)f * fstride;
        for (int c = 0; c < dim; ++c)
          for (int fp = 0; fp < nfp; ++fp)
            for (int q = 0; q < neq; ++q)
              acc[(size_t)c * neq * L + ((size_t)e * neq + q) * nd + trace_node(dim, N, lf, fp)] +=
                  rf[(size_t)c * 2 * neq * nfp + (s * neq + q) * nfp + fp];
      }
    for (size_t i = 0; i < gradE.size(); ++i) gradE[i] += acc[i];
    // boundary faces: the reference's boundary point kernel per face point,
    // restr_b transpose in boundary-face order, then added
    if (geo->num_bdr_faces > 0) {
      C bctx = ctx;
      bctx.bc_vector_d = geo->bc_data;
      std::vector<double> accb((size_t)dim * neq * L, 0.0);
      std::vector<double> uf((size_t)neq * nfp), rb((size_t)3 * neq * nfp);
      for (int b = 0; b < geo->num_bdr_faces; ++b) {
        const thx_bc &tb = geo->bcs[geo->bdr_bc[b]];
        Theseus::BCDescriptor bd{};
        bd.type = tb.type;
        bd.data_index = tb.data_index;
        const int e = geo->bdr_elem[b], lf = geo->bdr_lface[b];
        for (int fp = 0; fp < nfp; ++fp)
          for (int q = 0; q < neq; ++q)
            uf[q * nfp + fp] = Se[((size_t)e * neq + q) * nd + trace_node(dim, N, lf, fp)];
        std::fill(rb.begin(), rb.end(), 0.0);
        double *rp[3] = {rb.data(), rb.data() + neq * nfp, rb.data() + 2 * neq * nfp};
        for (int fp = 0; fp < nfp; ++fp)
          Theseus::DGSEMIntegrator::AssembleGradBoundaryPointKernel(
              bctx, bd, uf.data(), geo->bdr_normal + ((size_t)b * nfp + fp) * dim,
              geo->bdr_weight[(size_t)b * nfp + fp], fp, rp);
        for (int c = 0; c < dim; ++c)
          for (int fp = 0; fp < nfp; ++fp)
            for (int q = 0; q < neq; ++q)
              accb[(size_t)c * neq * L + ((size_t)e * neq + q) * nd + trace_node(dim, N, lf, fp)] +=
                  rp[c][q * nfp + fp];
      }
      for (size_t i = 0; i < gradE.size(); ++i) gradE[i] += accb[i];
    }
    // entropy gradient -> primitive gradient
    for (int c = 0; c < dim; ++c)
#pragma omp parallel for schedule(static)
      for (int e = 0; e < ne; ++e)
        for (int a = 0; a < nd; ++a) {
          double q[5], dS[5], dP[5];
          for (int k = 0; k < neq; ++k) {
            q[k] = Ue[((size_t)e * neq + k) * nd + a];
            dS[k] = gradE[(size_t)c * neq * L + ((size_t)e * neq + k) * nd + a];
          }
          Theseus::PointStateView CV{q};
          Theseus::PointStateView DS{dS};
          Theseus::PointStateViewRW DP{dP};
          ctx.gas.grad_entropy_to_grad_prim(CV, DS, DP);
          for (int k = 0; k < neq; ++k) gradE[(size_t)c * neq * L + ((size_t)e * neq + k) * nd + a] = dP[k];
        }
  }

  const int nxi = (N + 1) * N * (dim > 2 ? N : 1), neta = N * (N + 1) * (dim > 2 ? N : 1),
            nzeta = N * N * (N + 1);
#pragma omp parallel for schedule(dynamic, 16)
  for (int e = 0; e < ne; ++e) {
    std::vector<double> vflux((size_t)dim * neq * nd), dUfv((size_t)neq * nd);
    const double *ue = Ue.data() + (size_t)e * neq * nd;
    double *du = dUe.data() + (size_t)e * neq * nd;
    const double *J = geo->jac + (size_t)e * nd;
    const double *M = geo->metric + (size_t)e * nd * dd;
    for (int a = 0; a < nd; ++a) Theseus::DGSEMIntegrator::AssembleVolumePointKernel(ctx, ue, J, M, a, du);
    if (alpha && alpha[e] > 1e-16) {
      Theseus::DGSEMIntegrator::ComputeFVFluxesKernel(
          fvctx, ue, J, sub_xi + (size_t)e * nxi * dim,
          dim > 1 ? sub_eta + (size_t)e * neta * dim : nullptr,
          dim > 2 ? sub_zeta + (size_t)e * nzeta * dim : nullptr, dUfv.data());
      for (int v = 0; v < neq * nd; ++v) du[v] = (1.0 - alpha[e]) * du[v] + alpha[e] * dUfv[v];
    }
    if (ns) {
      const double *g0 = gradE.data() + (size_t)e * neq * nd;
      const double *g1 = gradE.data() + (size_t)neq * L + (size_t)e * neq * nd;
      const double *g2 = dim > 2 ? gradE.data() + 2 * (size_t)neq * L + (size_t)e * neq * nd : nullptr;
      for (int a = 0; a < nd; ++a)
        Theseus::DGSEMIntegrator::ComputeViscousVolumeFluxPointKernel(ctx, ue, M, nullptr, g0, g1, g2, a,
                                                                      vflux.data());
      for (int a = 0; a < nd; ++a)
        Theseus::DGSEMIntegrator::AssembleViscousVolumePointKernel(ctx, ue, J, M, nullptr, g0, g1, g2,
                                                                   vflux.data(), a, du);
    }
  }
  // restr_v->AddMultTranspose into zeroed dudt
#pragma omp parallel for schedule(static)
  for (int e = 0; e < ne; ++e)
    for (int q = 0; q < neq; ++q)
      for (int a = 0; a < nd; ++a) dudt[q * L + (size_t)e * nd + a] = dUe[((size_t)e * neq + q) * nd + a];
  // interior faces: face results stored, then added element by element in face order
  std::vector<double> rfall((size_t)nf * 2 * neq * nfp), acc((size_t)neq * L, 0.0);
#pragma omp parallel for schedule(static)
  for (int f = 0; f < nf; ++f) {
    std::vector<double> uf(2 * neq * nfp), gf((size_t)3 * 2 * neq * nfp, 0.0);
    double *rf = rfall.data() + (size_t)f * 2 * neq * nfp;
    for (int s = 0; s < 2; ++s) {
      const int e = geo->face_elem[2 * f + s], lf = geo->face_lface[2 * f + s];
      for (int fp = 0; fp < nfp; ++fp)
        for (int q = 0; q < neq; ++q) {
          const int a = trace_node(dim, N, lf, fp);
          uf[(s * neq + q) * nfp + fp] = Ue[((size_t)e * neq + q) * nd + a];
          if (ns)
            for (int c = 0; c < dim; ++c)
              gf[(size_t)c * 2 * neq * nfp + (s * neq + q) * nfp + fp] =
                  gradE[(size_t)c * neq * L + ((size_t)e * neq + q) * nd + a];
        }
    }
    for (int fp = 0; fp < nfp; ++fp) {
      const double *nr = geo->face_normal + ((size_t)f * nfp + fp) * dim;
      const double wm = geo->face_wminus[(size_t)f * nfp + fp], wp = geo->face_wplus[(size_t)f * nfp + fp];
      if (ns)
        Theseus::DGSEMIntegrator::AssembleViscousFacePointKernel(
            ctx, uf.data(), nr, wm, wp, gf.data(), gf.data() + 2 * neq * nfp,
            gf.data() + 4 * neq * nfp, 0.0, fp, rf);
      else
        Theseus::DGSEMIntegrator::AssembleFacePointKernel(ctx, uf.data(), nr, wm, wp, fp, rf);
    }
  }
#pragma omp parallel for schedule(static)
  for (int e = 0; e < ne; ++e)
    for (const auto &fs : elem_faces[e]) {
      const int f = fs.first, s = fs.second, lf = geo->face_lface[2 * f + s];
      const double *rf = rfall.data() + (size_t)f * 2 * neq * nfp;
      for (int fp = 0; fp < nfp; ++fp)
        for (int q = 0; q < neq; ++q)
          acc[q * L + (size_t)e * nd + trace_node(dim, N, lf, fp)] += rf[(s * neq + q) * nfp + fp];
    }
  for (size_t i = 0; i < (size_t)neq * L; ++i) dudt[i] += acc[i];
  // boundary faces (include/EulerOperator_impl.hpp:292-392) with the
  // reference's own boundary kernel; restr_b transpose in boundary-face order
  if (geo->num_bdr_faces > 0) {
    C bctx = ctx;
    bctx.bc_vector_d = geo->bc_data;
    std::vector<double> accb((size_t)neq * L, 0.0);
    for (int b = 0; b < geo->num_bdr_faces; ++b) {
      const thx_bc &tb = geo->bcs[geo->bdr_bc[b]];
      Theseus::BCDescriptor bd{};
      bd.type = tb.type;
      bd.data_index = tb.data_index;
      const int e = geo->bdr_elem[b], lf = geo->bdr_lface[b];
      for (int fp = 0; fp < nfp; ++fp) {
        const int a = trace_node(dim, N, lf, fp);
        double state1[Theseus::MAXEQ], fluxN[Theseus::MAXEQ];
        for (int q = 0; q < neq; ++q) state1[q] = Ue[((size_t)e * neq + q) * nd + a];
        const double *nr = geo->bdr_normal + ((size_t)b * nfp + fp) * dim;
        if (ns) {
          double gx[Theseus::MAXEQ], gy[Theseus::MAXEQ], gz[Theseus::MAXEQ] = {0};
          for (int q = 0; q < neq; ++q) {
            gx[q] = gradE[((size_t)e * neq + q) * nd + a];
            gy[q] = gradE[(size_t)neq * L + ((size_t)e * neq + q) * nd + a];
            if (dim > 2) gz[q] = gradE[2 * (size_t)neq * L + ((size_t)e * neq + q) * nd + a];
          }
          Theseus::BC::ApplyViscousBoundaryCondition(bctx, bd, state1, gx, gy, gz, nr, 0.0, fluxN);
        } else {
          Theseus::BC::ApplyBoundaryConditionInviscid(bctx, bd, state1, nr, fluxN);
        }
        const double scale = -geo->bdr_weight[(size_t)b * nfp + fp];
        for (int q = 0; q < neq; ++q) accb[q * L + (size_t)e * nd + a] += scale * fluxN[q];
      }
    }
    for (size_t i = 0; i < (size_t)neq * L; ++i) dudt[i] += accb[i];
  }
  return 0;
}

}  // namespace

extern "C" {

int ref_volume_flux(int flux, const thx_config *cfg, int dim, const double *q1, const double *q2,
                    const double *m1, const double *m2, double *F) {
  Gas g = make_gas(*cfg, dim);
  PairFlux pf;
  pf.vol = flux;
  pf.ComputeVolumeFlux(g, q1, q2, m1, m2, F);
  return 0;
}

int ref_face_flux(int flux, const thx_config *cfg, int dim, const double *qm, const double *qp,
                  const double *n, double *F) {
  Gas g = make_gas(*cfg, dim);
  PairFlux pf;
  pf.surf = flux;
  pf.ComputeFaceFlux(g, qm, qp, n, F);
  return 0;
}

int ref_entropy_vars(const thx_config *cfg, int dim, const double *q, double *w) {
  Gas g = make_gas(*cfg, dim);
  Theseus::PointStateView S{q};
  Theseus::PointStateViewRW E{w};
  g.entropy_state(S, E);
  return 0;
}

int ref_viscous_flux(const thx_config *cfg, int dim, const double *q, const double *dprim,
                     double *vf_out) {
  Gas g = make_gas(*cfg, dim);
  double vf[Theseus::MAXEQ][Theseus::MAXDIM];
  const int neq = dim + 2;
  Theseus::NavierStokesFlux::ComputeViscousFluxKernel(g, q, dprim, dprim + neq,
                                                     dim > 2 ? dprim + 2 * neq : dprim, vf);
  for (int e = 0; e < neq; ++e)
    for (int d = 0; d < dim; ++d) vf_out[e * dim + d] = vf[e][d];
  return 0;
}

int ref_rhs(const thx_geometry *geo, const thx_config *cfg, const double *D, const double *Dhat,
            const double *Dhat2, const double *w, const double *alpha, const double *sub_xi,
            const double *sub_eta, const double *sub_zeta, const double *u, double *dudt) {
  const int dim = geo->dim, N = geo->order + 1;
  const int nd = dim == 2 ? N * N : N * N * N;
  const int nfp = dim == 2 ? N : N * N;
  Ctx ctx{dim, dim + 2, nd, N, N, dim > 2 ? N : 1, nfp, false, make_gas(*cfg, dim), PairFlux{},
          D, Dhat, Dhat2, w};
  ctx.iflux.vol = cfg->volume_flux;
  ctx.iflux.surf = cfg->surface_flux;
  Ctx fvctx = ctx;
  fvctx.iflux.surf = cfg->fv_flux;
  return rhs_impl(ctx, fvctx, geo, cfg, alpha, sub_xi, sub_eta, sub_zeta, u, dudt);
}

// The same driver with the reference's LTE Helmholtz gas and LTEEC flux.
int ref_rhs_lte(const thx_geometry *geo, const thx_config *cfg, const thx_lte_table *t,
                const double *D, const double *Dhat, const double *Dhat2, const double *w,
                const double *u, double *dudt) {
  const int dim = geo->dim, N = geo->order + 1;
  const int nd = dim == 2 ? N * N : N * N * N;
  const int nfp = dim == 2 ? N : N * N;
  LteData data(t);
  LteCtx ctx{dim, dim + 2, nd, N, N, dim > 2 ? N : 1, nfp, false, data.gas(*cfg, dim),
             Theseus::LTEECFlux::InviscidFlux{}, D, Dhat, Dhat2, w};
  try {
    return rhs_impl(ctx, ctx, geo, cfg, nullptr, nullptr, nullptr, nullptr, u, dudt);
  } catch (const std::exception &) {
    return THX_ERR_NUMERICS;
  }
}

int ref_lte_point(const thx_lte_table *t, double rho, double T, double *out) {
  LteData data(t);
  const auto tables = Theseus::HelmholtzTable::HostView(data.data, data.layout);
  const auto s = Theseus::HelmholtzEOS::At(tables, rho, T);
  if (!s.valid) return THX_ERR_NUMERICS;
  out[0] = s.pressure(); out[1] = s.energy(); out[2] = s.gibbs(); out[3] = s.cv();
  out[4] = s.sound_speed_squared();
  out[5] = s.transport<Theseus::HelmholtzTable::Layout::mu_idx>(tables);
  out[6] = s.transport<Theseus::HelmholtzTable::Layout::lambda_idx>(tables);
  return THX_OK;
}

int ref_lte_temperature(const thx_lte_table *t, double rho, double e, double *T, int *status) {
  LteData data(t);
  const auto tables = Theseus::HelmholtzTable::HostView(data.data, data.layout);
  const auto r = Theseus::HelmholtzEOS::TemperatureFromEnergy(tables, rho, e);
  *T = r.temperature;
  *status = (int)r.status;
  return THX_OK;
}

int ref_lte_flux(const thx_lte_table *t, const thx_config *cfg, int dim, int face,
                 const double *q1, const double *q2, const double *d1, const double *d2,
                 double *F) {
  LteData data(t);
  const LteGas gas = data.gas(*cfg, dim);
  try {
    if (face) Theseus::LTEECFlux::ComputeFaceFluxKernel(gas, q1, q2, d1, F);
    else Theseus::LTEECFlux::ComputeVolumeFluxKernel(gas, q1, q2, d1, d2, F);
  } catch (const std::exception &) {
    return THX_ERR_NUMERICS;
  }
  return THX_OK;
}

}  // extern "C"
