// thx_api.cu -- the C ABI (include/theseus_b200.h): operator set-up on the
// device, kernel selection, right-hand side, fused SSP-RK3 steps, stability
// estimate and status.  No CPU fallback exists: without a CUDA device every
// compute entry point returns THX_ERR_NO_DEVICE.
#include "thx_operator.cuh"
#include "thx_host.h"
#include "thx_time.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

using namespace thx;

namespace {

// Pack a [outer][inner][block] array, dropping the outer and/or inner
// dimension where every entry is bitwise equal along it.
//   returns strides (outer stride, inner stride) in units of `block`.
void pack_strided(const double *src, long long outer, long long inner, int block, bool full,
                  std::vector<double> &dst, long long &os, long long &is) {
  auto eqb = [&](long long a, long long b) {
    return std::memcmp(src + a * block, src + b * block, sizeof(double) * block) == 0;
  };
  bool inner_const = !full, outer_same = !full;
  if (!full) {
    for (long long o = 0; o < outer && inner_const; ++o)
      for (long long i = 1; i < inner; ++i)
        if (!eqb(o * inner + i, o * inner)) { inner_const = false; break; }
    for (long long o = 1; o < outer && outer_same; ++o)
      if (std::memcmp(src + o * inner * block, src, sizeof(double) * inner * block) != 0) outer_same = false;
  }
  if (outer_same && inner_const) {
    dst.assign(src, src + block);
    os = 0; is = 0;
  } else if (outer_same) {
    dst.assign(src, src + inner * block);
    os = 0; is = block;
  } else if (inner_const) {
    dst.resize(outer * block);
    for (long long o = 0; o < outer; ++o) std::memcpy(dst.data() + o * block, src + o * inner * block, sizeof(double) * block);
    os = block; is = 0;
  } else {
    dst.assign(src, src + outer * inner * block);
    os = inner * block; is = block;
  }
}

template <typename R>
GasT<R> make_gas(const thx_config &c, int dim) {
  GasT<R> g;
  for (int k = 0; k < 5; ++k) g.qref[k] = R(0);
  g.ke_ref = R(0);
  g.p_ref = R(0);
  if (IsF32<R>::value) {
    // reference state of the FP32 working copy and its pressure
    double m2 = 0.0;
    for (int d = 0; d < dim; ++d) m2 += c.state_offset[1 + d] * c.state_offset[1 + d];
    const double rho = c.state_offset[0];
    const double ke = rho > 0.0 ? 0.5 * m2 / rho : 0.0;
    for (int k = 0; k < dim + 2; ++k) g.qref[k] = (R)c.state_offset[k];
    g.ke_ref = (R)ke;
    const double pr = (c.gamma - 1.0) * (c.state_offset[dim + 1] - ke);
    g.p_ref = (R)pr;
    // perturbation form of the fluxes about the offset state: for the
    // Chandrashekar volume flux with physical-flux surface fluxes (and subcell
    // fluxes), and an offset that is a physical state
    auto physical_face = [](int f) { return f == THX_FLUX_HLL || f == THX_FLUX_LLF || f == THX_FLUX_ROE; };
    g.pert = (c.volume_flux == THX_FLUX_CHANDRASHEKAR && physical_face(c.surface_flux) &&
              (!c.blending || physical_face(c.fv_flux)) && rho > 0.0 && pr > 0.0 &&
              !c.mixed_flux_no_perturbation) ? 1 : 0;
    g.rho_r = (R)rho;
    double v2 = 0.0;
    for (int d = 0; d < 3; ++d) {
      const double v = (d < dim && rho > 0.0) ? c.state_offset[1 + d] / rho : 0.0;
      g.v_r[d] = (R)v;
      v2 += v * v;
    }
    g.p_r = (R)pr;
    const double beta = pr > 0.0 ? 0.5 * rho / pr : 0.0;
    g.beta_r = (R)beta;
    const double gav = 2.0 / (c.gamma + c.gamma - 2.0);
    g.h_r = beta > 0.0 ? (R)(0.5 / beta * gav + 0.5 * v2 + pr / rho) : R(0);
    g.Hr = (R)(c.state_offset[dim + 1] + pr);
  } else {
    g.pert = 0;
    g.rho_r = g.p_r = g.beta_r = g.h_r = g.Hr = R(0);
    g.v_r[0] = g.v_r[1] = g.v_r[2] = R(0);
  }
  const double gm1 = c.gamma - 1.0;
  const double gm1_inv = 1.0 / gm1;
  const double cp = (c.gamma * gm1_inv) * c.R_gas;
  g.gamma = (R)c.gamma;
  g.gm1 = (R)gm1;
  g.gm1_inv = (R)gm1_inv;
  g.R_gas = (R)c.R_gas;
  g.cp = (R)cp;
  g.Pr_inv = (R)(1.0 / c.Pr);
  g.mu = (R)c.mu;
  g.mu0 = (R)c.mu0;
  g.mu_bulk = (R)c.mu_bulk;
  g.T0 = (R)c.T0;
  g.Ts = (R)c.Ts;
  g.gm1_av_inv = (R)(2.0 / (c.gamma + c.gamma - 2.0));
  g.inv_gm1 = (R)(1.0 / (c.gamma - 1.0));
  g.cv = (R)(cp / c.gamma);
  g.sutherland = c.sutherland;
  return g;
}

// Operator whose buffers are being allocated on this thread: in pool mode
// (batch engine) allocations are stream-ordered on its set-up stream.
thread_local thx_operator_s *t_alloc_owner = nullptr;

struct AllocOwner {
  explicit AllocOwner(thx_operator_s *h) { t_alloc_owner = h; }
  ~AllocOwner() { t_alloc_owner = nullptr; }
};

bool pool_mode() { return t_alloc_owner && t_alloc_owner->pool; }

template <typename T>
int dev_alloc(T **p, size_t n, std::vector<void *> &track) {
  *p = nullptr;
  if (n == 0) n = 1;
  const cudaError_t e = pool_mode()
      ? cudaMallocFromPoolAsync((void **)p, n * sizeof(T), t_alloc_owner->pool, t_alloc_owner->setup_stream)
      : cudaMalloc((void **)p, n * sizeof(T));
  if (e != cudaSuccess) {
    *p = nullptr;
    return cuda_failed(e, pool_mode() ? "cudaMallocFromPoolAsync" : "cudaMalloc", THX_ERR_OUT_OF_MEMORY);
  }
  track.push_back(*p);
  return THX_OK;
}

// Host-to-device copy of set-up data; stream-ordered in pool mode (pageable
// sources are staged before the call returns).
int to_device(void *dst, const void *src, size_t bytes) {
  if (pool_mode() && t_alloc_owner->ring)
    return t_alloc_owner->ring->copy(dst, src, bytes, t_alloc_owner->setup_stream);
  const cudaError_t e = pool_mode()
      ? cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, t_alloc_owner->setup_stream)
      : cudaMemcpy(dst, src, bytes, cudaMemcpyHostToDevice);
  return e == cudaSuccess ? THX_OK : THX_ERR_CUDA;
}

int dev_zero(void *dst, size_t bytes) {
  if (pool_mode() && t_alloc_owner->ring) {
    // through the upload ring: the set-up stream then holds copies only,
    // which the copy engines run while persistent kernels fill every SM
    thread_local std::vector<unsigned char> zeros;
    if (zeros.size() < bytes) zeros.assign(bytes, 0);
    return t_alloc_owner->ring->copy(dst, zeros.data(), bytes, t_alloc_owner->setup_stream);
  }
  const cudaError_t e = pool_mode() ? cudaMemsetAsync(dst, 0, bytes, t_alloc_owner->setup_stream)
                                    : cudaMemset(dst, 0, bytes);
  return e == cudaSuccess ? THX_OK : THX_ERR_CUDA;
}

template <typename T>
int upload(T **p, const T *src, size_t n, std::vector<void *> &track) {
  int st = dev_alloc(p, n, track);
  if (st) return st;
  return to_device(*p, src, n * sizeof(T));
}

int upload_both(const std::vector<double> &h, double **d64, float **d32, bool want32,
                std::vector<void *> &track) {
  int st = upload(d64, h.data(), h.size(), track);
  if (st) return st;
  if (want32) {
    std::vector<float> f(h.begin(), h.end());
    st = upload(d32, f.data(), f.size(), track);
  } else {
    *d32 = nullptr;
  }
  return st;
}

}  // namespace


namespace {

struct DeviceGuard {
  int prev = -1;
  bool ok = true;
  explicit DeviceGuard(int dev) {
    if (cudaGetDevice(&prev) != cudaSuccess) { prev = -1; ok = false; cudaGetLastError(); return; }
    if (prev != dev && cudaSetDevice(dev) != cudaSuccess) { ok = false; cudaGetLastError(); }
  }
  ~DeviceGuard() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

bool pick_order_kernels(thx_operator_s *h, int vk) {
  const bool ns = h->ns;
  const bool bl = h->blend;
#define THX_PICK(P, D, NN)                                                  \
  if (h->dim == D && h->N == NN) {                                          \
    auto k = order_kernels_##P##_##D##_##NN();                              \
    const bool tma = h->cfg.volume_staging == 1 && !bl;                    \
    if (P == 0) {                                                           \
      h->vol64 = reinterpret_cast<VolLaunch<double>>(tma ? k.vol_tma[vk][ns ? 1 : 0]      \
                                                         : k.vol[vk][ns ? 1 : 0][bl ? 1 : 0]); \
      h->grad64 = reinterpret_cast<GradLaunch<double>>(k.grad);             \
      h->blend64 = reinterpret_cast<BlendLaunch<double>>(k.blend);          \
      h->fv64 = reinterpret_cast<VolLaunch<double>>(k.fv);                  \
    } else {                                                                \
      h->vol32 = reinterpret_cast<VolLaunch<float>>(tma ? k.vol_tma[vk][ns ? 1 : 0]       \
                                                        : k.vol[vk][ns ? 1 : 0][bl ? 1 : 0]); \
      h->grad32 = reinterpret_cast<GradLaunch<float>>(k.grad);              \
      h->blend32 = reinterpret_cast<BlendLaunch<float>>(k.blend);           \
      h->fv32 = reinterpret_cast<VolLaunch<float>>(k.fv);                   \
    }                                                                       \
    return true;                                                            \
  }
  if (!h->mixed) {
    THX_FOR_ORDERS(THX_PICK, 0, 2)
    THX_FOR_ORDERS(THX_PICK, 0, 3)
  } else {
    THX_FOR_ORDERS(THX_PICK, 1, 2)
    THX_FOR_ORDERS(THX_PICK, 1, 3)
  }
#undef THX_PICK
  return false;
}

bool pick_lte_kernels(thx_operator_s *h) {
  const int ns = h->ns ? 1 : 0;
#define THX_PICK_LTE(P, D, NN)                      \
  if (h->dim == D && h->N == NN) {                  \
    const LteKernels k = lte_kernels_##D##_##NN();  \
    h->vol64 = k.vol[ns];                           \
    h->grad64 = k.grad;                             \
    found = true;                                   \
  }
  bool found = false;
  THX_FOR_ORDERS(THX_PICK_LTE, 0, 2)
  THX_FOR_ORDERS(THX_PICK_LTE, 0, 3)
#undef THX_PICK_LTE
  if (!found) return false;
  const LteFaceKernels f = h->dim == 2 ? lte_face_kernels_2() : lte_face_kernels_3();
  h->face64 = f.face[ns];
  return true;
}

void pick_face_kernels(thx_operator_s *h) {
  const int s = h->cfg.surface_flux, ns = h->ns ? 1 : 0;
  if (!h->mixed) {
    FaceKernels0 k = h->dim == 2 ? face_kernels_0_2() : face_kernels_0_3();
    h->face64 = k.face[s][ns];
    h->bnd64 = k.bnd[s][ns];
    h->ent64 = k.entropy;
  } else {
    FaceKernels1 k = h->dim == 2 ? face_kernels_1_2() : face_kernels_1_3();
    h->face32 = k.face[s][ns];
    h->ent32 = k.entropy;
  }
}

void free_all(thx_operator_s *h) {
  if (h->hp_in) cudaStreamSynchronize(h->hp_in);
  if (h->hp_out) cudaStreamSynchronize(h->hp_out);
  for (cudaEvent_t &e : h->hp_ev)
    if (e) { cudaEventDestroy(e); e = nullptr; }
  if (h->hp_in) { cudaStreamDestroy(h->hp_in); h->hp_in = nullptr; }
  if (h->hp_out) { cudaStreamDestroy(h->hp_out); h->hp_out = nullptr; }
  for (void *p : h->allocs) {
    if (h->pool) cudaFreeAsync(p, h->setup_stream);
    else cudaFree(p);
  }
  h->allocs.clear();
}

// Subcell-FV metrics of one element (include/dgsem_cache_utilities.hpp:641-763),
// node-indexed as in the reference; D row-major [l*N+m].
void subcell_element(int dim, int N, const double *metric_el, const double *D, const double *w,
                     double *xi, double *eta, double *zeta) {
  const int Nx = N, Ny = N, Nz = dim > 2 ? N : 1;
  const int nxi = (Nx + 1) * Ny * Nz, neta = Nx * (Ny + 1) * Nz, nzeta = Nx * Ny * (Nz + 1);
  std::memset(xi, 0, sizeof(double) * nxi * dim);
  if (eta) std::memset(eta, 0, sizeof(double) * neta * dim);
  if (zeta) std::memset(zeta, 0, sizeof(double) * nzeta * dim);
  auto M = [&](int node, int row, int d) { return metric_el[(node * dim + row) * dim + d]; };
  for (int k = 0; k < Nz; ++k)
    for (int j = 0; j < Ny; ++j)
      for (int i = 1; i < Nx; ++i)
        for (int d = 0; d < dim; ++d) {
          const int line = k * Ny * Nx + j * Nx;
          double nrm = M(line, 0, d);
          for (int l = 0; l < i; ++l) {
            double sum = 0.0;
            for (int m = 0; m < Nx; ++m) sum += M(line + m, 0, d) * D[l * Nx + m];
            sum *= w[l];
            nrm += sum;
          }
          xi[(line + i) * dim + d] = nrm;
        }
  if (dim > 1 && eta)
    for (int k = 0; k < Nz; ++k)
      for (int i = 0; i < Nx; ++i)
        for (int j = 1; j < Ny; ++j)
          for (int d = 0; d < dim; ++d) {
            const int line = k * Ny * Nx + i;
            double nrm = M(line, 1, d);
            for (int l = 0; l < j; ++l) {
              double sum = 0.0;
              for (int m = 0; m < Ny; ++m) sum += M(line + m * Nx, 1, d) * D[l * Nx + m];
              sum *= w[l];
              nrm += sum;
            }
            eta[(k * Ny * Nx + j * Nx + i) * dim + d] = nrm;
          }
  if (dim > 2 && zeta)
    for (int j = 0; j < Ny; ++j)
      for (int i = 0; i < Nx; ++i)
        for (int k = 1; k < Nz; ++k)
          for (int d = 0; d < dim; ++d) {
            const int line = j * Nx + i;
            double nrm = M(line, 2, d);
            for (int l = 0; l < k; ++l) {
              double sum = 0.0;
              for (int m = 0; m < Nz; ++m) sum += M(line + m * Ny * Nx, 2, d) * D[l * Nx + m];
              sum *= w[l];
              nrm += sum;
            }
            zeta[(k * Ny * Nx + line) * dim + d] = nrm;
          }
}

// Copies a donor operator's device geometry (factors, face tables, element-to-
// face table, operators, subcell metrics, modal transform) into h by pointer:
// h does not own them.  The donor must be built from the same mesh, order,
// precision, blending and geometry layout, periodic, and outlive h.
void share_geometry(thx_operator_s *h, const thx_operator_s *d) {
  h->lay = d->lay;
  h->jac64 = d->jac64; h->jac32 = d->jac32;
  h->met64 = d->met64; h->met32 = d->met32;
  h->nrm64 = d->nrm64; h->nrm32 = d->nrm32;
  h->wm64 = d->wm64; h->wm32 = d->wm32;
  h->wp64 = d->wp64; h->wp32 = d->wp32;
  h->face_elem = d->face_elem; h->face_lface = d->face_lface;
  h->face_order = d->face_order; h->elem_face = d->elem_face;
  h->ops64 = d->ops64; h->ops32 = d->ops32;
  h->D64 = d->D64; h->D32 = d->D32;
  for (int k = 0; k < 3; ++k) { h->sub64[k] = d->sub64[k]; h->sub32[k] = d->sub32[k]; }
  h->vinv = d->vinv;
}

int create_impl(const thx_geometry *g, const thx_config *cfg, thx_operator_s *h,
                const thx_lte_table *table = nullptr, const thx_operator_s *donor = nullptr) {
  AllocOwner owner(h);
  h->cfg = *cfg;
  h->dim = g->dim;
  h->order = g->order;
  h->N = g->order + 1;
  h->nd = g->dim == 2 ? h->N * h->N : h->N * h->N * h->N;
  h->nfp = g->dim == 2 ? h->N : h->N * h->N;
  h->neq = g->dim + 2;
  h->ne = g->num_elements;
  h->nf = g->num_faces;
  h->L = (long long)h->ne * h->nd;
  h->mixed = cfg->precision == THX_PRECISION_FP32_MIXED;
  h->ns = cfg->flow_model == THX_FLOW_NAVIER_STOKES;
  h->blend = cfg->blending != 0;
  h->nbf = g->num_bdr_faces > 0 ? g->num_bdr_faces : 0;
  if (h->nbf > 0) {
    // boundary faces: FP64, ideal gas
    if (!g->bdr_elem || !g->bdr_lface || !g->bdr_normal || !g->bdr_weight || !g->bdr_bc || !g->bcs ||
        g->num_bcs <= 0 || g->bc_data_len < 0 || (g->bc_data_len > 0 && !g->bc_data))
      return THX_ERR_INVALID_ARGUMENT;
    // FP32-mixed: Euler only, the boundary-adjacent blocks evaluated in FP64
    // (FP64 islands); the LTE gas has no boundary conditions here
    if (table || (h->mixed && cfg->flow_model == THX_FLOW_NAVIER_STOKES)) return THX_ERR_UNSUPPORTED;
    for (int i = 0; i < g->num_bcs; ++i) {
      const thx_bc &bc = g->bcs[i];
      if (bc.type < THX_BC_SLIP_WALL || bc.type > THX_BC_NOSLIP_ISOTHERMAL) return THX_ERR_INVALID_ARGUMENT;
      if (bc.type == THX_BC_AXIS) return THX_ERR_UNSUPPORTED;
      if ((bc.type == THX_BC_PRESCRIBED_STATE || bc.type == THX_BC_SUPERSONIC_INFLOW) &&
          (bc.data_index < 0 || bc.data_index + g->dim + 2 > g->bc_data_len))
        return THX_ERR_INVALID_ARGUMENT;
    }
    for (int b = 0; b < h->nbf; ++b)
      if (g->bdr_bc[b] < 0 || g->bdr_bc[b] >= g->num_bcs) return THX_ERR_INVALID_ARGUMENT;
  }
  h->g64 = make_gas<double>(*cfg, g->dim);
  h->g32 = make_gas<float>(*cfg, g->dim);
  for (int k = 0; k < 5; ++k) h->off.v[k] = (k < g->dim + 2) ? cfg->state_offset[k] : 0.0;
  const int vk = (cfg->volume_flux == THX_FLUX_CHANDRASHEKAR) ? VOL_CHANDRASHEKAR
               : (cfg->volume_flux == THX_FLUX_RANOCHA)     ? VOL_RANOCHA
               : (cfg->volume_flux == THX_FLUX_PIROZZOLI)   ? VOL_PIROZZOLI
                                                            : VOL_CENTRAL;
  h->lte = table != nullptr;
  if (h->lte) {
    if (!pick_lte_kernels(h)) return THX_ERR_UNSUPPORTED;
  } else {
    if (!pick_order_kernels(h, vk)) return THX_ERR_UNSUPPORTED;
    pick_face_kernels(h);
  }
  const bool full = cfg->geometry_layout == 1;
  const int dim = h->dim, N = h->N, nd = h->nd, nfp = h->nfp, MB = dim * dim;
  const bool w32 = h->mixed;
  auto &A = h->allocs;
  int st;
  if (h->lte) {
    // device copy of the table; node temperatures
    const size_t nx = (size_t)table->nx, ny = (size_t)table->ny;
    double *rho = nullptr, *T = nullptr, *e = nullptr, *planes = nullptr, *inv = nullptr;
    if ((st = upload(&rho, table->rho_grid, nx, A))) return st;
    if ((st = upload(&T, table->T_grid, ny, A))) return st;
    if ((st = upload(&e, table->e_grid, ny, A))) return st;
    if ((st = upload(&planes, table->planes, 6 * nx * ny, A))) return st;
    if ((st = upload(&inv, table->inverse, nx * ny, A))) return st;
    h->g64.lte.nx = table->nx;
    h->g64.lte.ny = table->ny;
    h->g64.lte.rho = rho;
    h->g64.lte.T = T;
    h->g64.lte.e = e;
    h->g64.lte.planes = planes;
    h->g64.lte.inv = inv;
    if ((st = dev_alloc(&h->Tn, (size_t)h->L, A))) return st;
    h->g64.Tn = h->Tn;
    if ((st = dev_alloc(&h->Cn, (size_t)h->L, A))) return st;
    h->g64.Cn = h->Cn;
  }
  // a donor's device geometry is shared, not rebuilt (batch engine: cases
  // that name the same mesh)
  if (donor && (donor->dim != dim || donor->order != h->order || donor->ne != h->ne ||
                donor->nf != h->nf || donor->nbf != 0 || h->nbf != 0 || donor->mixed != h->mixed ||
                donor->blend != h->blend || donor->cfg.geometry_layout != cfg->geometry_layout))
    return THX_ERR_INVALID_ARGUMENT;
  if (donor) share_geometry(h, donor);
  // geometry
  std::vector<double> tmp;
  if (!donor) {
  pack_strided(g->jac, h->ne, nd, 1, full, tmp, h->lay.jac_es, h->lay.jac_ns);
  if ((st = upload_both(tmp, &h->jac64, &h->jac32, w32, A))) return st;
  pack_strided(g->metric, h->ne, nd, MB, full, tmp, h->lay.met_es, h->lay.met_ns);
  if ((st = upload_both(tmp, &h->met64, &h->met32, w32, A))) return st;
  pack_strided(g->face_normal, h->nf, nfp, dim, full, tmp, h->lay.n_fs, h->lay.n_ps);
  // normals are indexed as (f*n_fs + fp*n_ps)*DIM: convert block strides to point units
  h->lay.n_fs /= dim;
  h->lay.n_ps /= dim;
  if ((st = upload_both(tmp, &h->nrm64, &h->nrm32, w32, A))) return st;
  {
    // lift weights share one layout
    std::vector<double> both((size_t)h->nf * nfp * 2);
    for (long long i = 0; i < (long long)h->nf * nfp; ++i) {
      both[2 * i] = g->face_wminus[i];
      both[2 * i + 1] = g->face_wplus[i];
    }
    long long fs, ps;
    pack_strided(both.data(), h->nf, nfp, 2, full, tmp, fs, ps);
    h->lay.w_fs = fs / 2;
    h->lay.w_ps = ps / 2;
    std::vector<double> wm(tmp.size() / 2), wp(tmp.size() / 2);
    for (size_t i = 0; i < wm.size(); ++i) { wm[i] = tmp[2 * i]; wp[i] = tmp[2 * i + 1]; }
    if ((st = upload_both(wm, &h->wm64, &h->wm32, w32, A))) return st;
    if ((st = upload_both(wp, &h->wp64, &h->wp32, w32, A))) return st;
  }
  // connectivity
  if ((st = upload(&h->face_elem, g->face_elem, (size_t)2 * h->nf, A))) return st;
  if ((st = upload(&h->face_lface, g->face_lface, (size_t)2 * h->nf, A))) return st;
  {
    // face-kernel processing order: interior faces by minus-side element
    // (stable), so that the CTAs in flight gather from a narrow element window
    std::vector<int> order(h->nf);
    for (int f = 0; f < h->nf; ++f) order[f] = f;
    std::stable_sort(order.begin(), order.end(),
                     [&](int x, int y) { return g->face_elem[2 * x] < g->face_elem[2 * y]; });
    if ((st = upload(&h->face_order, order.data(), order.size(), A))) return st;
  }
  {
    std::vector<int> ef((size_t)h->ne * 2 * dim, -1);
    for (int f = 0; f < h->nf; ++f)
      for (int s = 0; s < 2; ++s) {
        const int e = g->face_elem[2 * f + s], lf = g->face_lface[2 * f + s];
        if (e < 0 || e >= h->ne || lf < 0 || lf >= 2 * dim) return THX_ERR_INVALID_ARGUMENT;
        ef[(size_t)e * 2 * dim + lf] = 2 * f + s;
      }
    // boundary faces take face slots nf .. nf+nbf-1 (minus side only)
    for (int b = 0; b < h->nbf; ++b) {
      const int e = g->bdr_elem[b], lf = g->bdr_lface[b];
      if (e < 0 || e >= h->ne || lf < 0 || lf >= 2 * dim) return THX_ERR_INVALID_ARGUMENT;
      ef[(size_t)e * 2 * dim + lf] = 2 * (h->nf + b);
    }
    if ((st = upload(&h->elem_face, ef.data(), ef.size(), A))) return st;
  }
  if (h->nbf > 0) {
    if ((st = upload(&h->bdr_elem, g->bdr_elem, (size_t)h->nbf, A))) return st;
    if ((st = upload(&h->bdr_lface, g->bdr_lface, (size_t)h->nbf, A))) return st;
    if ((st = upload(&h->bdr_bc, g->bdr_bc, (size_t)h->nbf, A))) return st;
    if ((st = upload(&h->bdr_nrm, g->bdr_normal, (size_t)h->nbf * nfp * dim, A))) return st;
    if ((st = upload(&h->bdr_w, g->bdr_weight, (size_t)h->nbf * nfp, A))) return st;
    if ((st = upload(&h->bcs, g->bcs, (size_t)g->num_bcs, A))) return st;
    if ((st = upload(&h->bc_data, g->bc_data, (size_t)std::max(1, (int)g->bc_data_len), A))) return st;
    if (h->ns && (st = dev_alloc(&h->bgrad, (size_t)h->nbf * nfp * dim * h->neq, A))) return st;
  }
  }  // !donor
  // operators
  std::vector<double> x(N), w(N), D(N * N), Dh(N * N), Dh2(N * N);
  lgl_rule(N, x.data(), w.data());
  derivative_operators(N, x.data(), w.data(), D.data(), Dh.data(), Dh2.data());
  if (!donor) {
    std::vector<double> ops(2 * N * N + N);
    std::memcpy(ops.data(), Dh2.data(), sizeof(double) * N * N);
    std::memcpy(ops.data() + N * N, Dh.data(), sizeof(double) * N * N);
    std::memcpy(ops.data() + 2 * N * N, w.data(), sizeof(double) * N);
    if ((st = upload_both(ops, &h->ops64, &h->ops32, w32, A))) return st;
    if ((st = upload_both(D, &h->D64, &h->D32, w32, A))) return st;
  }
  // scratch
  const size_t fsz = (size_t)(h->nf + h->nbf) * h->neq * nfp;
  if (h->mixed) {
    float *p;
    if ((st = dev_alloc(&p, fsz, A))) return st;
    h->fstar = p;
    if (h->ns) { if ((st = dev_alloc(&p, (size_t)dim * (h->neq - 1) * h->L, A))) return st; h->vflux = p; }
  } else {
    double *p;
    if ((st = dev_alloc(&p, fsz, A))) return st;
    h->fstar = p;
    if (h->ns) { if ((st = dev_alloc(&p, (size_t)dim * (h->neq - 1) * h->L, A))) return st; h->vflux = p; }
    if (h->ns && !h->lte) { if ((st = dev_alloc(&p, (size_t)h->neq * h->L, A))) return st; h->svars = p; }
  }
  if ((st = dev_alloc(&h->status, 1, A))) return st;
  if ((st = dev_alloc(&h->stab, 3, A))) return st;
  if ((st = dev_alloc(&h->dtd, 1, A))) return st;
  if ((st = dev_zero(h->status, sizeof(unsigned)))) return st;
  if ((st = dev_alloc(&h->alpha, h->ne, A))) return st;
  if ((st = dev_alloc(&h->eta, h->ne, A))) return st;
  if ((st = dev_zero(h->alpha, sizeof(double) * h->ne))) return st;
  if ((st = dev_zero(h->eta, sizeof(double) * h->ne))) return st;
  if (h->blend) {
    const size_t nfv = (size_t)h->L * h->neq;
    if (h->mixed) {
      float *p;
      if ((st = dev_alloc(&p, nfv, A))) return st;
      h->fvrate = p;
    } else {
      double *p;
      if ((st = dev_alloc(&p, nfv, A))) return st;
      h->fvrate = p;
    }
  }
  // blending: modal transform and subcell metrics
  h->threshold = cfg->modal_threshold > 0 ? cfg->modal_threshold
                                          : 0.5 * std::pow(10.0, -1.8 * std::pow((double)h->order, 0.25));
  if (h->blend && !donor) {
    std::vector<double> vinv(N * N);
    if (!legendre_vinv(N, x.data(), vinv.data())) return THX_ERR_NUMERICS;
    if ((st = upload(&h->vinv, vinv.data(), vinv.size(), A))) return st;
    const int Nz = dim > 2 ? N : 1;
    const long long nsub[3] = {(long long)(N + 1) * N * Nz * dim, (long long)N * (N + 1) * Nz * dim,
                               (long long)N * N * (N + 1) * dim};
    const bool shared = h->lay.met_es == 0;
    const long long nel = shared ? 1 : h->ne;
    std::vector<double> xi(nsub[0] * nel), et(nsub[1] * nel), ze(dim > 2 ? nsub[2] * nel : 1);
    std::vector<double> mel((size_t)nd * MB);
    for (long long e = 0; e < nel; ++e) {
      for (int a = 0; a < nd; ++a)
        std::memcpy(mel.data() + (size_t)a * MB, g->metric + ((size_t)e * nd + a) * MB, sizeof(double) * MB);
      subcell_element(dim, N, mel.data(), D.data(), w.data(), xi.data() + e * nsub[0],
                      et.data() + e * nsub[1], dim > 2 ? ze.data() + e * nsub[2] : nullptr);
    }
    for (int d = 0; d < 3; ++d) h->lay.sub_es[d] = shared ? 0 : nsub[d];
    if ((st = upload_both(xi, &h->sub64[0], &h->sub32[0], w32, A))) return st;
    if ((st = upload_both(et, &h->sub64[1], &h->sub32[1], w32, A))) return st;
    if (dim > 2 && (st = upload_both(ze, &h->sub64[2], &h->sub32[2], w32, A))) return st;
  }
  // stability scales (include/StabilityEstimate.hpp:61-92)
  {
    static const double adv_cal[] = {0.0, 2.19706891727, 5.41995189335, 9.64849524786,
                                     14.7297419321, 20.5984751391, 27.2141622680, 34.5459214016,
                                     42.5691944324, 51.2637780299, 60.6126232210, 70.6010566044,
                                     81.2162499718};
    static const double dif_cal[] = {0.0, 4.0, 25.5969429388, 82.9000427145, 203.470468982,
                                     426.230394541, 799.733889878, 1383.0975821, 2244.38177282,
                                     3461.2550528, 5121.29136549, 7321.77632194, 10169.7148876};
    const int p = h->order;
    h->adv_scale = (p > 0 && p < 13) ? 1.05 * adv_cal[p] : 0.65 * (p + 1) * (p + 1);
    h->dif_scale = (p > 0 && p < 13) ? 1.25 * dif_cal[p] : 0.5 * std::pow(p + 1.0, 4);
    h->surf_scale = h->adv_scale / (1.0 / w[0]);
  }
  // FP64 islands of the FP32-mixed Euler path: the blocks holding a blended
  // element (unless switched off) and the blocks next to a boundary face
  if (h->mixed && !h->ns && !h->lte && ((h->blend && !cfg->mixed_blended_fp32) || h->nbf > 0)) {
    bool found = false;
#define THX_PICK_ISL(P, D, NN)                                   \
    if (h->dim == D && h->N == NN) {                             \
      auto k = order_kernels_0_##D##_##NN();                     \
      h->isl_vol = k.voll[vk];                                   \
      h->isl_fv = k.fvl;                                         \
      h->isl_blend = k.blendl;                                   \
      found = true;                                              \
    }
    THX_FOR_ORDERS(THX_PICK_ISL, 0, 2)
    THX_FOR_ORDERS(THX_PICK_ISL, 0, 3)
#undef THX_PICK_ISL
    const FaceKernels0 fk = dim == 2 ? face_kernels_0_2() : face_kernels_0_3();
    h->isl_face = fk.facel[cfg->surface_flux];
    h->isl_bnd = fk.bnd[cfg->surface_flux][0];
    if (!found || !h->isl_vol || !h->isl_fv || !h->isl_blend || !h->isl_face || (h->nbf > 0 && !h->isl_bnd))
      return THX_ERR_UNSUPPORTED;
    h->isl_epb = std::max(1, 256 / nd);
    const int nblk = (h->ne + h->isl_epb - 1) / h->isl_epb;
    h->isl_alpha_in = h->blend && !cfg->mixed_blended_fp32;
    if (h->nbf > 0) {
      // blocks next to a boundary face are islands at every right-hand side
      std::vector<int> stat(nblk, 0);
      for (int b = 0; b < h->nbf; ++b) stat[g->bdr_elem[b] / h->isl_epb] = 1;
      if ((st = upload(&h->isl_static, stat.data(), stat.size(), A))) return st;
    }
    if ((st = dev_alloc(&h->isl_flag, (size_t)nblk, A))) return st;
    if ((st = dev_alloc(&h->isl_blocks, (size_t)nblk, A))) return st;
    if ((st = dev_alloc(&h->isl_faces, (size_t)std::max(1, h->nf), A))) return st;
    if ((st = dev_alloc(&h->isl_count, 2, A))) return st;
    if ((st = dev_alloc(&h->isl_fstar, (size_t)(h->nf + h->nbf) * h->neq * nfp, A))) return st;
    if ((st = dev_alloc(&h->isl_alpha, (size_t)h->ne, A))) return st;
    if ((st = dev_alloc(&h->isl_eta, (size_t)h->ne, A))) return st;
    if ((st = dev_alloc(&h->isl_fvrate, (size_t)h->L * h->neq, A))) return st;
    if ((st = dev_zero(h->isl_alpha, sizeof(double) * h->ne))) return st;
    h->islands = true;
  }
  // kernel attributes (dynamic shared memory)
  cudaError_t ce;
  if (h->mixed) {
    VolArgs<float> va{};
    GradArgs<float> ga{};
    ce = h->vol32(va, 0, 1);
    if (ce == cudaSuccess && h->ns) ce = h->grad32(ga, 0, 1);
    if (ce == cudaSuccess && h->blend) ce = h->fv32(va, 0, 1);
    if (ce == cudaSuccess && h->islands) {
      VolArgs<double> v64{};
      ce = h->isl_vol(v64, nullptr, nullptr, 0, 1);
      if (ce == cudaSuccess) ce = h->isl_fv(v64, nullptr, nullptr, 0, 1);
    }
  } else {
    VolArgs<double> va{};
    GradArgs<double> ga{};
    ce = h->vol64(va, 0, 1);
    if (ce == cudaSuccess && h->ns) ce = h->grad64(ga, 0, 1);
    if (ce == cudaSuccess && h->blend && h->fv64) ce = h->fv64(va, 0, 1);
  }
  if (ce != cudaSuccess) { cudaGetLastError(); return THX_ERR_CUDA; }
  char buf[512];
  std::snprintf(buf, sizeof(buf),
                "dim=%d p=%d ne=%d nf=%d flow=%s gas=%s vol=%d surf=%d fv=%d blend=%d prec=%s "
                "layout jac(%lld,%lld) met(%lld,%lld) nrm(%lld,%lld) w(%lld,%lld) sub(%lld)",
                dim, h->order, h->ne, h->nf, h->ns ? "ns" : "euler", h->lte ? "lte" : "ideal",
                cfg->volume_flux, cfg->surface_flux, cfg->fv_flux, cfg->blending,
                h->mixed ? "fp32-mixed" : "fp64",
                h->lay.jac_es, h->lay.jac_ns, h->lay.met_es, h->lay.met_ns, h->lay.n_fs, h->lay.n_ps,
                h->lay.w_fs, h->lay.w_ps, h->lay.sub_es[0]);
  h->desc = buf;
  return THX_OK;
}

template <typename R>
struct Geo {
  const R *jac, *met, *nrm, *wm, *wp, *sub[3], *ops, *D;
};
Geo<double> geo(thx_operator_s *h, double *) {
  return {h->jac64, h->met64, h->nrm64, h->wm64, h->wp64, {h->sub64[0], h->sub64[1], h->sub64[2]}, h->ops64, h->D64};
}
Geo<float> geo(thx_operator_s *h, float *) {
  return {h->jac32, h->met32, h->nrm32, h->wm32, h->wp32, {h->sub32[0], h->sub32[1], h->sub32[2]}, h->ops32, h->D32};
}
VolLaunch<double> volk(thx_operator_s *h, double *) { return h->vol64; }
VolLaunch<float> volk(thx_operator_s *h, float *) { return h->vol32; }
EntropyLaunch<double> entk(thx_operator_s *h, double *) { return h->ent64; }
EntropyLaunch<float> entk(thx_operator_s *h, float *) { return h->ent32; }
GradLaunch<double> gradk(thx_operator_s *h, double *) { return h->grad64; }
GradLaunch<float> gradk(thx_operator_s *h, float *) { return h->grad32; }
BlendLaunch<double> blendk(thx_operator_s *h, double *) { return h->blend64; }
VolLaunch<double> fvk(thx_operator_s *h, double *) { return h->fv64; }
VolLaunch<float> fvk(thx_operator_s *h, float *) { return h->fv32; }
BlendLaunch<float> blendk(thx_operator_s *h, float *) { return h->blend32; }
FaceLaunch<double> facek(thx_operator_s *h, double *) { return h->face64; }
FaceLaunch<float> facek(thx_operator_s *h, float *) { return h->face32; }
const GasT<double> &gas(thx_operator_s *h, double *) { return h->g64; }
const GasT<float> &gas(thx_operator_s *h, float *) { return h->g32; }

}  // namespace

namespace thx {

template <typename R>
void op_args(thx_operator_s *h, const R *u, R *du, int stage, double dt, double *um, double *y,
             float *yf, GradArgs<R> &ga, FaceArgs<R> &fa, VolArgs<R> &va) {
  R *tag = nullptr;
  const Geo<R> G = geo(h, tag);
  const GasT<R> &g = gas(h, tag);
  R *vfl = reinterpret_cast<R *>(h->vflux);
  R *fst = reinterpret_cast<R *>(h->fstar);
  ga = GradArgs<R>{};
  ga.u = u; ga.vflux = vfl; ga.ne = h->ne;
  ga.jac = G.jac; ga.jac_es = h->lay.jac_es; ga.jac_ns = h->lay.jac_ns;
  ga.met = G.met; ga.met_es = h->lay.met_es; ga.met_ns = h->lay.met_ns;
  ga.elem_face = h->elem_face; ga.face_elem = h->face_elem; ga.face_lface = h->face_lface;
  ga.normal = G.nrm; ga.n_fs = h->lay.n_fs; ga.n_ps = h->lay.n_ps;
  ga.wm = G.wm; ga.wp = G.wp; ga.w_fs = h->lay.w_fs; ga.w_ps = h->lay.w_ps;
  ga.D = G.D; ga.gas = g; ga.status = h->status;
  ga.svars = reinterpret_cast<const R *>(h->svars);
  ga.nf_int = h->nf;
  if constexpr (IsF32<R>::value) {
    ga.bw = nullptr;
  } else {
    ga.bw = h->nbf > 0 ? h->bdr_w : nullptr;
    ga.bnrm = h->bdr_nrm; ga.bdr_bc = h->bdr_bc; ga.bcs = h->bcs; ga.bc_data = h->bc_data;
    ga.bgrad = h->bgrad;
  }
  fa = FaceArgs<R>{};
  fa.u = u; fa.ne = h->ne; fa.nf = h->nf; fa.N = h->N;
  fa.face_elem = h->face_elem; fa.face_lface = h->face_lface;
  fa.normal = G.nrm; fa.n_fs = h->lay.n_fs; fa.n_ps = h->lay.n_ps;
  fa.vflux = vfl; fa.fstar = fst; fa.gas = g;
  fa.order = h->face_order;
  va = VolArgs<R>{};
  va.u = u; va.du = du; va.ne = h->ne;
  va.jac = G.jac; va.jac_es = h->lay.jac_es; va.jac_ns = h->lay.jac_ns;
  va.met = G.met; va.met_es = h->lay.met_es; va.met_ns = h->lay.met_ns;
  va.elem_face = h->elem_face; va.fstar = fst;
  va.wm = G.wm; va.wp = G.wp; va.w_fs = h->lay.w_fs; va.w_ps = h->lay.w_ps;
  va.vflux = vfl;
  va.nf_int = h->nf;
  if constexpr (IsF32<R>::value) va.bw = nullptr;
  else va.bw = h->bdr_w;
  va.alpha = h->blend ? h->alpha : nullptr;
  va.fvrate = h->blend ? reinterpret_cast<R *>(h->fvrate) : nullptr;
  for (int d = 0; d < 3; ++d) { va.sub[d] = G.sub[d]; va.sub_es[d] = h->lay.sub_es[d]; }
  va.fv_flux = h->cfg.fv_flux;
  va.gas = g;
  va.ops = G.ops;
  va.stage = stage; va.dt = dt; va.um = um; va.y = y; va.yf = yf;
  for (int k = 0; k < 5; ++k) va.off[k] = IsF32<R>::value ? h->off.v[k] : 0.0;
  va.status = h->status;
}

template void op_args<double>(thx_operator_s *, const double *, double *, int, double, double *,
                              double *, float *, GradArgs<double> &, FaceArgs<double> &,
                              VolArgs<double> &);
template void op_args<float>(thx_operator_s *, const float *, float *, int, double, double *,
                             double *, float *, GradArgs<float> &, FaceArgs<float> &,
                             VolArgs<float> &);

}  // namespace thx

namespace {

// One right-hand side: [T recovery] [indicator] [gradient] face fluxes,
// volume+lift.  stage 0 writes du; stages 1..3 apply the SSP-RK3 update in place.
// FP32-mixed: u64 is the FP64 state the working copy u was narrowed from
// (the FP64 islands read it).
template <typename R>
int run_rhs(thx_operator_s *h, const R *u, R *du, cudaStream_t s, int stage, double dt,
            double *um, double *y, float *yf, cudaEvent_t *ev = nullptr, double *du64 = nullptr,
            const double *dt_dev = nullptr, const double *u64 = nullptr, bool narrow_in_grad = false) {
  R *tag = nullptr;
  if (ev) cudaEventRecord(ev[0], s);
  GradArgs<R> ga;
  FaceArgs<R> fa;
  VolArgs<R> va;
  op_args<R>(h, u, du, stage, dt, um, y, yf, ga, fa, va);
  va.du64 = du64;
  va.dt_dev = dt_dev;
  if constexpr (IsF32<R>::value) {
    if (narrow_in_grad) {
      // the gradient kernel narrows the FP64 state into the working copy
      ga.u64 = u64;
      ga.yf = h->yf;
      for (int k = 0; k < 5; ++k) ga.off[k] = h->off.v[k];
    }
  }
  if constexpr (!IsF32<R>::value) {
    if (h->lte) {
      cudaError_t te = h->dim == 2
          ? launch_lte_temperature<2>(u, h->L, h->g64.lte, h->Tn, h->Cn, h->status, s)
          : launch_lte_temperature<3>(u, h->L, h->g64.lte, h->Tn, h->Cn, h->status, s);
      if (te != cudaSuccess) return THX_ERR_CUDA;
    }
  }
  if (h->blend) {
    BlendArgs<R> b;
    b.u = u; b.ne = h->ne; b.vinv = h->vinv; b.gas = gas(h, tag);
    b.threshold = h->threshold; b.sharpness = h->cfg.sharpness;
    b.alpha_min = h->cfg.alpha_min; b.alpha_max = h->cfg.alpha_max;
    b.alpha = h->alpha; b.eta = h->eta;
    if (blendk(h, tag)(b, s) != cudaSuccess) return THX_ERR_CUDA;
  }
  // FP64 islands: list the blocks holding a blended element and their faces,
  // then the FP64 indicator of those blocks
  const bool isl = IsF32<R>::value && h->islands && u64;
  GradArgs<double> ga64;
  FaceArgs<double> fa64;
  VolArgs<double> va64;
  if (isl) {
    const int nblk = (h->ne + h->isl_epb - 1) / h->isl_epb;
    if (cudaMemsetAsync(h->isl_count, 0, 2 * sizeof(int), s) != cudaSuccess) return THX_ERR_CUDA;
    island_blocks_kernel<R><<<(nblk + 255) / 256, 256, 0, s>>>(
        h->ne, h->isl_epb, h->isl_alpha_in ? h->alpha : nullptr, h->isl_static, h->isl_flag,
        h->isl_blocks, h->isl_count);
    if (h->nf > 0)
      island_faces_kernel<<<(h->nf + 255) / 256, 256, 0, s>>>(h->nf, h->isl_epb, h->face_elem, h->isl_flag,
                                                              h->isl_faces, h->isl_count + 1);
    BlendArgs<double> b;
    b.u = u64; b.ne = h->ne; b.vinv = h->vinv; b.gas = h->g64;
    b.threshold = h->threshold; b.sharpness = h->cfg.sharpness;
    b.alpha_min = h->cfg.alpha_min; b.alpha_max = h->cfg.alpha_max;
    b.alpha = h->isl_alpha; b.eta = h->isl_eta;
    if (h->blend && h->isl_blend(b, h->isl_blocks, h->isl_count, s) != cudaSuccess) return THX_ERR_CUDA;
    op_args<double>(h, u64, du64, stage, dt, um, y, yf, ga64, fa64, va64);
    fa64.fstar = h->isl_fstar;
    fa64.order = h->isl_faces;
    va64.fstar = h->isl_fstar;
    va64.alpha = h->isl_alpha;
    va64.fvrate = h->isl_fvrate;
    va64.yf = yf;
    va64.dt_dev = dt_dev;
    for (int k = 0; k < 5; ++k) va64.off[k] = h->off.v[k];
    va.skip_block = h->isl_flag;
  }
  if (ev) cudaEventRecord(ev[1], s);
  // FP64 Navier-Stokes (ideal gas): the entropy variables of every node
  // first, read by the gradient kernel
  if (h->svars &&
      entk(h, tag)(u, h->L, gas(h, tag), reinterpret_cast<R *>(h->svars), s) != cudaSuccess)
    return THX_ERR_CUDA;
  if (h->ns && gradk(h, tag)(ga, s, 0) != cudaSuccess) return THX_ERR_CUDA;
  if (ev) cudaEventRecord(ev[2], s);
  if (facek(h, tag)(fa, s) != cudaSuccess) return THX_ERR_CUDA;
  if (isl && h->isl_face(fa64, h->isl_count + 1, s) != cudaSuccess) return THX_ERR_CUDA;
  if (isl && h->nbf > 0) {
    // boundary faces in FP64 into the islands' face fluxes
    BndArgs ba;
    ba.u = u64; ba.ne = h->ne; ba.N = h->N; ba.nbf = h->nbf; ba.f0 = h->nf;
    ba.bdr_elem = h->bdr_elem; ba.bdr_lface = h->bdr_lface; ba.bdr_bc = h->bdr_bc;
    ba.normal = h->bdr_nrm; ba.bcs = h->bcs; ba.bc_data = h->bc_data; ba.bgrad = h->bgrad;
    ba.fstar = h->isl_fstar; ba.gas = h->g64;
    if (h->isl_bnd(ba, s) != cudaSuccess) return THX_ERR_CUDA;
  }
  if constexpr (!IsF32<R>::value) {
    if (h->nbf > 0) {
      BndArgs ba;
      ba.u = u; ba.ne = h->ne; ba.N = h->N; ba.nbf = h->nbf; ba.f0 = h->nf;
      ba.bdr_elem = h->bdr_elem; ba.bdr_lface = h->bdr_lface; ba.bdr_bc = h->bdr_bc;
      ba.normal = h->bdr_nrm; ba.bcs = h->bcs; ba.bc_data = h->bc_data; ba.bgrad = h->bgrad;
      ba.fstar = reinterpret_cast<double *>(h->fstar); ba.gas = h->g64;
      if (h->bnd64(ba, s) != cudaSuccess) return THX_ERR_CUDA;
    }
  }
  if (ev) cudaEventRecord(ev[3], s);
  if (isl && h->blend) {
    // the FP64 subcell rate of the listed blocks
    if (h->isl_fv(va64, h->isl_blocks, h->isl_count, s, 0) != cudaSuccess) return THX_ERR_CUDA;
  }
  // the FP32 subcell rate, for blended elements outside the islands
  if (h->blend && !(isl && h->isl_alpha_in) && fvk(h, tag)(va, s, 0) != cudaSuccess) return THX_ERR_CUDA;
  if (volk(h, tag)(va, s, 0) != cudaSuccess) return THX_ERR_CUDA;
  if (isl && h->isl_vol(va64, h->isl_blocks, h->isl_count, s, 0) != cudaSuccess) return THX_ERR_CUDA;
  if (ev) cudaEventRecord(ev[4], s);
  return THX_OK;
}

int check_device() {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n <= 0) {
    cudaGetLastError();
    return THX_ERR_NO_DEVICE;
  }
  return THX_OK;
}

}  // namespace

namespace {

// Narrow the FP64 state to the FP32 working copy (mixed mode).
int to_working_copy(thx_operator_s *h, const double *u, cudaStream_t s) {
  const long long n = h->L * h->neq;
  int st;
  if (!h->yf && (st = dev_alloc(&h->yf, (size_t)n, h->allocs))) return st;
  const int gridn = (int)std::min<long long>((h->L + 255) / 256, 1LL << 24);  // one node per thread
  if (h->dim == 2) to_working<2><<<gridn, 256, 0, s>>>(h->L, u, h->yf, h->off, h->g64.gm1, h->status);
  else to_working<3><<<gridn, 256, 0, s>>>(h->L, u, h->yf, h->off, h->g64.gm1, h->status);
  return cudaGetLastError() == cudaSuccess ? THX_OK : THX_ERR_CUDA;
}

int rhs_mixed(thx_operator_s *h, const double *u, double *dudt, cudaStream_t s, cudaEvent_t *ev) {
  // the volume kernel writes the FP32 rate widened to FP64 directly.  Navier-
  // Stokes without blending: the gradient kernel, the first to read the state,
  // narrows it into the working copy (one pass over the FP64 state fewer);
  // otherwise the indicator or the face kernel reads the copy first and a
  // separate narrowing pass runs ahead.
  const bool in_grad = h->ns && !h->blend && !h->lte && !h->islands;
  int st;
  if (!h->yf && (st = dev_alloc(&h->yf, (size_t)(h->L * h->neq), h->allocs))) return st;
  if (!in_grad && (st = to_working_copy(h, u, s))) return st;
  return run_rhs<float>(h, h->yf, nullptr, s, 0, 0.0, nullptr, nullptr, nullptr, ev, dudt, nullptr, u,
                        in_grad);
}

}  // namespace

namespace thx {

int op_create(const thx_geometry *g, const thx_config *cfg, thx_operator_s *h,
              const thx_lte_table *table, const thx_operator_s *donor) {
  try {
    return create_impl(g, cfg, h, table, donor);
  } catch (...) {
    return THX_ERR_OUT_OF_MEMORY;
  }
}

void op_free(thx_operator_s *h) { free_all(h); }

int op_to_working_copy(thx_operator_s *h, const double *u, cudaStream_t s) {
  return to_working_copy(h, u, s);
}

}  // namespace thx


namespace thx {

// Stability rates of state u into h->stab (ordered bit patterns of the
// advective, surface and diffusive rates), stream-ordered
// (include/RHSOperator_impl.hpp:10-270).
int stability_rates(thx_operator_s *h, const double *u, cudaStream_t s) {
  StabArgs a;
  a.u = u; a.ne = h->ne; a.N = h->N;
  a.jac = h->jac64; a.jac_es = h->lay.jac_es; a.jac_ns = h->lay.jac_ns;
  a.met = h->met64; a.met_es = h->lay.met_es; a.met_ns = h->lay.met_ns;
  a.face_elem = h->face_elem; a.face_lface = h->face_lface; a.nf = h->nf;
  a.normal = h->nrm64; a.n_fs = h->lay.n_fs; a.n_ps = h->lay.n_ps;
  a.wm = h->wm64; a.wp = h->wp64; a.w_fs = h->lay.w_fs; a.w_ps = h->lay.w_ps;
  a.gas = h->g64;
  a.adv_scale = h->adv_scale; a.dif_scale = h->dif_scale; a.surf_scale = h->surf_scale;
  a.viscous = h->ns ? 1 : 0;
  a.out = h->stab;
  a.nbf = h->nbf;
  a.bdr_elem = h->bdr_elem; a.bdr_lface = h->bdr_lface; a.bdr_bc = h->bdr_bc;
  a.bnrm = h->bdr_nrm; a.bw = h->bdr_w; a.bcs = h->bcs; a.bc_data = h->bc_data;
  if (cudaMemsetAsync(h->stab, 0, sizeof(unsigned long long) * 3, s) != cudaSuccess) return THX_ERR_CUDA;
  const long long work = h->L + (long long)(h->nf + h->nbf) * h->nfp;
  const int grid = (int)std::min<long long>((work + 255) / 256, 148LL * 8);
  if (h->dim == 2) stability_kernel<2><<<grid, 256, 0, s>>>(a);
  else stability_kernel<3><<<grid, 256, 0, s>>>(a);
  return cudaGetLastError() == cudaSuccess ? THX_OK : THX_ERR_CUDA;
}

// The device side of the clocked time loop: one thread advances the
// thx_time_loop record in device memory around each SSP-RK3 step.
__device__ inline double total_rate_of(const unsigned long long *rates) {
  const double adv = __longlong_as_double((long long)rates[0]);
  const double sur = __longlong_as_double((long long)rates[1]);
  const double dif = __longlong_as_double((long long)rates[2]);
  return (adv > sur ? adv : sur) + dif;
}

// Initial nominal step of a variable-dt loop (src/Simulation.cpp:1150-1158).
__global__ void time_loop_init_kernel(thx_time_loop *L, const unsigned long long *rates, double cfl,
                                      unsigned *status) {
  if (threadIdx.x != 0 || blockIdx.x != 0 || L->done || L->dt > 0.0) return;
  const double total = total_rate_of(rates);
  if (total > 0.0) L->dt = cfl / total;
  else atomicOr(status, STATUS_NONFINITE);
}

__global__ void time_loop_begin_kernel(thx_time_loop *L, double *dt, double *history) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const double s = time_loop_begin(*L);
  *dt = s;
  if (history) *history = s;
}

__global__ void time_loop_end_kernel(thx_time_loop *L, const double *dt,
                                     const unsigned long long *rates, double cfl, unsigned *status) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const double total = cfl > 0.0 ? total_rate_of(rates) : 0.0;
  if (!time_loop_end(*L, *dt, total, cfl)) atomicOr(status, STATUS_NONFINITE);
}

}  // namespace thx

extern "C" {

const char *thx_version(void) { return "theseus-b200 0.1 (sm_100a)"; }

const char *thx_last_cuda_failure(void) { return thx::last_cuda_failure; }

const char *thx_status_string(int status) {
  switch (status) {
    case THX_OK: return "ok";
    case THX_ERR_INVALID_ARGUMENT: return "invalid argument";
    case THX_ERR_UNSUPPORTED: return "unsupported configuration";
    case THX_ERR_CUDA: return "CUDA runtime error";
    case THX_ERR_NO_DEVICE: return "no CUDA device (no CPU fallback exists)";
    case THX_ERR_OUT_OF_MEMORY: return "out of device memory";
    case THX_ERR_NUMERICS: return "numerical status flag set";
    case THX_ERR_BUSY: return "busy: the case does not fit the memory budget now";
    case THX_ERR_IO: return "checkpoint file I/O failed";
  }
  return "unknown status";
}

void thx_config_default(thx_config *c) {
  if (!c) return;
  std::memset(c, 0, sizeof(*c));
  c->flow_model = THX_FLOW_EULER;
  c->volume_flux = THX_FLUX_CHANDRASHEKAR;
  c->surface_flux = THX_FLUX_CHANDRASHEKAR;
  c->fv_flux = THX_FLUX_LLF;
  c->precision = THX_PRECISION_FP64;
  c->gamma = 1.4;
  c->Pr = 0.72;
  c->R_gas = 287.05;
  c->mu = 0.02;
  c->mu0 = 1.716e-5;
  c->mu_bulk = 2.0 / 3.0;
  c->T0 = 273.15;
  c->Ts = 110.4;
  c->alpha_max = 0.5;
  c->alpha_min = 0.001;
  c->sharpness = 9.21024;
  c->modal_threshold = 0.0;
}

int thx_create(const thx_geometry *g, const thx_config *cfg, thx_handle *out) {
  if (!g || !cfg || !out) return THX_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  if (g->dim < 2 || g->dim > 3 || g->order < 1 || g->num_elements <= 0 || g->num_faces < 0 ||
      !g->jac || !g->metric || (g->num_faces > 0 && (!g->face_elem || !g->face_lface ||
                                                     !g->face_normal || !g->face_wminus ||
                                                     !g->face_wplus)))
    return THX_ERR_INVALID_ARGUMENT;
  if (cfg->volume_flux < 0 || cfg->volume_flux >= THX_FLUX_COUNT || cfg->surface_flux < 0 ||
      cfg->surface_flux >= THX_FLUX_COUNT || cfg->fv_flux < 0 || cfg->fv_flux >= THX_FLUX_COUNT ||
      (cfg->flow_model != THX_FLOW_EULER && cfg->flow_model != THX_FLOW_NAVIER_STOKES) ||
      (cfg->precision != THX_PRECISION_FP64 && cfg->precision != THX_PRECISION_FP32_MIXED) ||
      !(cfg->gamma > 1.0) || !(cfg->Pr > 0.0))
    return THX_ERR_INVALID_ARGUMENT;
  if (g->order + 1 < 3 || g->order + 1 > 6) return THX_ERR_UNSUPPORTED;
  // the LTEEC flux needs the LTE Helmholtz gas (thx_create_lte)
  if (cfg->volume_flux == THX_FLUX_LTEEC || cfg->surface_flux == THX_FLUX_LTEEC ||
      cfg->fv_flux == THX_FLUX_LTEEC)
    return THX_ERR_UNSUPPORTED;
  int st = check_device();
  if (st) return st;
  thx_operator_s *h = new (std::nothrow) thx_operator_s();
  if (!h) return THX_ERR_OUT_OF_MEMORY;
  cudaGetDevice(&h->device);
  try {
    st = create_impl(g, cfg, h);
  } catch (...) {
    st = THX_ERR_OUT_OF_MEMORY;
  }
  if (st) {
    free_all(h);
    delete h;
    return st;
  }
  *out = h;
  return THX_OK;
}

int thx_create_lte(const thx_geometry *g, const thx_config *cfg, const thx_lte_table *table,
                   thx_handle *out) {
  if (!g || !cfg || !table || !out) return THX_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  if (g->dim < 2 || g->dim > 3 || g->order < 1 || g->num_elements <= 0 || g->num_faces < 0 ||
      !g->jac || !g->metric || (g->num_faces > 0 && (!g->face_elem || !g->face_lface ||
                                                     !g->face_normal || !g->face_wminus ||
                                                     !g->face_wplus)))
    return THX_ERR_INVALID_ARGUMENT;
  if ((cfg->flow_model != THX_FLOW_EULER && cfg->flow_model != THX_FLOW_NAVIER_STOKES) ||
      !(cfg->Pr > 0.0))
    return THX_ERR_INVALID_ARGUMENT;
  // the LTE gas is served by the LTEEC flux on volume and faces, in FP64,
  // without subcell blending
  if (cfg->volume_flux != THX_FLUX_LTEEC || cfg->surface_flux != THX_FLUX_LTEEC ||
      cfg->precision != THX_PRECISION_FP64 || cfg->blending)
    return THX_ERR_UNSUPPORTED;
  if (g->order + 1 < 3 || g->order + 1 > 6) return THX_ERR_UNSUPPORTED;
  if (table->nx < 2 || table->ny < 2 || !table->rho_grid || !table->T_grid || !table->e_grid ||
      !table->planes || !table->inverse)
    return THX_ERR_INVALID_ARGUMENT;
  // grids strictly increasing (the cell search bisects them)
  const double *grids[3] = {table->rho_grid, table->T_grid, table->e_grid};
  const int counts[3] = {table->nx, table->ny, table->ny};
  for (int k = 0; k < 3; ++k)
    for (int i = 0; i < counts[k]; ++i)
      if (!std::isfinite(grids[k][i]) || (i > 0 && !(grids[k][i] > grids[k][i - 1])))
        return THX_ERR_INVALID_ARGUMENT;
  if ((long long)table->nx * table->ny > (1LL << 26)) return THX_ERR_INVALID_ARGUMENT;
  int st = check_device();
  if (st) return st;
  thx_operator_s *h = new (std::nothrow) thx_operator_s();
  if (!h) return THX_ERR_OUT_OF_MEMORY;
  cudaGetDevice(&h->device);
  try {
    st = create_impl(g, cfg, h, table);
  } catch (...) {
    st = THX_ERR_OUT_OF_MEMORY;
  }
  if (st) {
    free_all(h);
    delete h;
    return st;
  }
  *out = h;
  return THX_OK;
}

int thx_destroy(thx_handle h) {
  if (!h) return THX_ERR_INVALID_ARGUMENT;
  {
    DeviceGuard dg(h->device);
    free_all(h);
  }
  delete h;
  return THX_OK;
}

int thx_rhs(thx_handle h, const void *u, void *dudt, void *stream) {
  if (!h || !u || !dudt) return THX_ERR_INVALID_ARGUMENT;
  DeviceGuard dg(h->device);
  if (!dg.ok) return THX_ERR_CUDA;
  cudaStream_t s = (cudaStream_t)stream;
  if (h->mixed) return rhs_mixed(h, (const double *)u, (double *)dudt, s, nullptr);
  return run_rhs<double>(h, (const double *)u, (double *)dudt, s, 0, 0.0, nullptr, nullptr, nullptr);
}

int thx_rhs_host(thx_handle h, int n, const double *const *u_host, double *const *dudt_host, void *stream) {
  if (!h || n < 0 || (n > 0 && (!u_host || !dudt_host))) return THX_ERR_INVALID_ARGUMENT;
  for (int i = 0; i < n; ++i)
    if (!u_host[i] || !dudt_host[i]) return THX_ERR_INVALID_ARGUMENT;
  DeviceGuard dg(h->device);
  if (!dg.ok) return THX_ERR_CUDA;
  cudaStream_t s = (cudaStream_t)stream;
  const size_t count = (size_t)h->L * h->neq, bytes = sizeof(double) * count;
  int st;
  for (int b = 0; b < 2; ++b) {
    if (!h->hp_u[b] && (st = dev_alloc(&h->hp_u[b], count, h->allocs))) return st;
    if (!h->hp_du[b] && (st = dev_alloc(&h->hp_du[b], count, h->allocs))) return st;
  }
  if (!h->hp_in) {
    THX_CU(cudaStreamCreateWithFlags(&h->hp_in, cudaStreamNonBlocking));
    THX_CU(cudaStreamCreateWithFlags(&h->hp_out, cudaStreamNonBlocking));
    for (cudaEvent_t &e : h->hp_ev) THX_CU(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  }
  cudaEvent_t start = h->hp_ev[0], *in = h->hp_ev + 1, *done = h->hp_ev + 3, *out = h->hp_ev + 5;
  // nothing starts before the work already queued on the caller's stream
  THX_CU(cudaEventRecord(start, s));
  THX_CU(cudaStreamWaitEvent(h->hp_in, start, 0));
  THX_CU(cudaStreamWaitEvent(h->hp_out, start, 0));
  for (int i = 0; i < n; ++i) {
    const int b = i & 1;
    // copy in once the right-hand side two states back has read this buffer
    if (i >= 2) THX_CU(cudaStreamWaitEvent(h->hp_in, done[b], 0));
    THX_CU(cudaMemcpyAsync(h->hp_u[b], u_host[i], bytes, cudaMemcpyHostToDevice, h->hp_in));
    THX_CU(cudaEventRecord(in[b], h->hp_in));
    THX_CU(cudaStreamWaitEvent(s, in[b], 0));
    // overwrite the rate buffer once its previous copy-out is done
    if (i >= 2) THX_CU(cudaStreamWaitEvent(s, out[b], 0));
    if ((st = h->mixed ? rhs_mixed(h, h->hp_u[b], h->hp_du[b], s, nullptr)
                       : run_rhs<double>(h, h->hp_u[b], h->hp_du[b], s, 0, 0.0, nullptr, nullptr, nullptr)))
      return st;
    THX_CU(cudaEventRecord(done[b], s));
    THX_CU(cudaStreamWaitEvent(h->hp_out, done[b], 0));
    THX_CU(cudaMemcpyAsync(dudt_host[i], h->hp_du[b], bytes, cudaMemcpyDeviceToHost, h->hp_out));
    THX_CU(cudaEventRecord(out[b], h->hp_out));
  }
  // the caller's stream resumes after the last copy-out
  for (int b = 0; b < 2 && b < n; ++b) THX_CU(cudaStreamWaitEvent(s, out[(n - 1 - b) & 1], 0));
  return THX_OK;
}

int thx_rk3_steps(thx_handle h, double *u, double dt, int nsteps, void *stream) {
  if (!h || !u || nsteps < 0 || !std::isfinite(dt)) return THX_ERR_INVALID_ARGUMENT;
  DeviceGuard dg(h->device);
  if (!dg.ok) return THX_ERR_CUDA;
  cudaStream_t s = (cudaStream_t)stream;
  const long long n = h->L * h->neq;
  int st;
  if (!h->y && (st = dev_alloc(&h->y, (size_t)n, h->allocs))) return st;
  if (h->mixed && (st = to_working_copy(h, u, s))) return st;
  for (int step = 0; step < nsteps; ++step) {
    if (h->mixed) {
      for (int stage = 1; stage <= 3; ++stage)
        if ((st = run_rhs<float>(h, h->yf, nullptr, s, stage, dt, u, h->y, h->yf, nullptr, nullptr,
                                 nullptr, stage == 1 ? u : h->y)))
          return st;
    } else {
      if ((st = run_rhs<double>(h, u, nullptr, s, 1, dt, u, h->y, nullptr))) return st;
      if ((st = run_rhs<double>(h, h->y, nullptr, s, 2, dt, u, h->y, nullptr))) return st;
      if ((st = run_rhs<double>(h, h->y, nullptr, s, 3, dt, u, h->y, nullptr))) return st;
    }
  }
  return THX_OK;
}

int thx_rk3_steps_cfl(thx_handle h, double *u, double cfl, int nsteps, double *dt_history,
                      void *stream) {
  if (!h || !u || nsteps < 0 || !(cfl > 0.0)) return THX_ERR_INVALID_ARGUMENT;
  if (h->lte) return THX_ERR_UNSUPPORTED;  // ideal-gas rates only
  DeviceGuard dg(h->device);
  if (!dg.ok) return THX_ERR_CUDA;
  cudaStream_t s = (cudaStream_t)stream;
  const long long n = h->L * h->neq;
  int st;
  if (!h->y && (st = dev_alloc(&h->y, (size_t)n, h->allocs))) return st;
  if (h->mixed && (st = to_working_copy(h, u, s))) return st;
  for (int step = 0; step < nsteps; ++step) {
    // dt from the stability rates of the step's initial state, on the device
    if ((st = stability_rates(h, u, s))) return st;
    cfl_dt_kernel<<<1, 1, 0, s>>>(h->stab, cfl, h->dtd, dt_history ? dt_history + step : nullptr,
                                  h->status);
    if (cudaGetLastError() != cudaSuccess) return THX_ERR_CUDA;
    if (h->mixed) {
      for (int stage = 1; stage <= 3; ++stage)
        if ((st = run_rhs<float>(h, h->yf, nullptr, s, stage, 0.0, u, h->y, h->yf, nullptr, nullptr,
                                 h->dtd, stage == 1 ? u : h->y)))
          return st;
    } else {
      if ((st = run_rhs<double>(h, u, nullptr, s, 1, 0.0, u, h->y, nullptr, nullptr, nullptr, h->dtd))) return st;
      if ((st = run_rhs<double>(h, h->y, nullptr, s, 2, 0.0, u, h->y, nullptr, nullptr, nullptr, h->dtd))) return st;
      if ((st = run_rhs<double>(h, h->y, nullptr, s, 3, 0.0, u, h->y, nullptr, nullptr, nullptr, h->dtd))) return st;
    }
  }
  return THX_OK;
}

void thx_time_loop_defaults(thx_time_loop *loop) {
  if (!loop) return;
  std::memset(loop, 0, sizeof(*loop));
  loop->t_final = INFINITY;
  loop->max_dt_growth = 1.2;
  loop->next_output = INFINITY;
  loop->output_dt = 0.01;
  loop->refined_output_dt = 0.01;
  loop->refine_time = 2.0;
  loop->next_checkpoint = INFINITY;
  loop->checkpoint_dt = 0.01;
  loop->max_cycles = -1;
  loop->output_cycles = 100;
}

int thx_time_event_reached(double t, double event_time) { return thx::time_event_reached(t, event_time) ? 1 : 0; }

double thx_limit_time_step_to_events(double step, double t, const double *events, int n) {
  return thx::limit_step_to_events(step, t, events, events ? n : 0);
}

int thx_step_limit_reached(int64_t cycle, int64_t max_cycles) {
  return thx::step_limit_reached(cycle, max_cycles) ? 1 : 0;
}

double thx_time_loop_begin(thx_time_loop *loop) { return loop ? thx::time_loop_begin(*loop) : 0.0; }

void thx_time_loop_end(thx_time_loop *loop, double dt_taken, double total_rate, double cfl) {
  if (loop) thx::time_loop_end(*loop, dt_taken, total_rate, cfl);
}

int thx_rk3_time_loop(thx_handle h, double *u, double cfl, int ncycles, thx_time_loop *loop,
                      double *dt_history, void *stream) {
  if (!h || !u || !loop || ncycles < 0) return THX_ERR_INVALID_ARGUMENT;
  if (cfl > 0.0 && h->lte) return THX_ERR_UNSUPPORTED;  // ideal-gas rates only
  DeviceGuard dg(h->device);
  if (!dg.ok) return THX_ERR_CUDA;
  cudaStream_t s = (cudaStream_t)stream;
  const long long n = h->L * h->neq;
  int st;
  if (!h->y && (st = dev_alloc(&h->y, (size_t)n, h->allocs))) return st;
  if (h->mixed && (st = to_working_copy(h, u, s))) return st;
  const bool variable = cfl > 0.0;
  if (variable) {
    if ((st = stability_rates(h, u, s))) return st;
    time_loop_init_kernel<<<1, 1, 0, s>>>(loop, h->stab, cfl, h->status);
  }
  for (int c = 0; c < ncycles; ++c) {
    time_loop_begin_kernel<<<1, 1, 0, s>>>(loop, h->dtd, dt_history ? dt_history + c : nullptr);
    if (cudaGetLastError() != cudaSuccess) return THX_ERR_CUDA;
    if (h->mixed) {
      for (int stage = 1; stage <= 3; ++stage)
        if ((st = run_rhs<float>(h, h->yf, nullptr, s, stage, 0.0, u, h->y, h->yf, nullptr, nullptr,
                                 h->dtd, stage == 1 ? u : h->y)))
          return st;
    } else {
      if ((st = run_rhs<double>(h, u, nullptr, s, 1, 0.0, u, h->y, nullptr, nullptr, nullptr, h->dtd))) return st;
      if ((st = run_rhs<double>(h, h->y, nullptr, s, 2, 0.0, u, h->y, nullptr, nullptr, nullptr, h->dtd))) return st;
      if ((st = run_rhs<double>(h, h->y, nullptr, s, 3, 0.0, u, h->y, nullptr, nullptr, nullptr, h->dtd))) return st;
    }
    if (variable && (st = stability_rates(h, u, s))) return st;
    time_loop_end_kernel<<<1, 1, 0, s>>>(loop, h->dtd, h->stab, cfl, h->status);
    if (cudaGetLastError() != cudaSuccess) return THX_ERR_CUDA;
  }
  return THX_OK;
}

int thx_blending_coefficients(thx_handle h, double *alpha_dev, double *eta_dev, void *stream) {
  if (!h) return THX_ERR_INVALID_ARGUMENT;
  DeviceGuard dg(h->device);
  cudaStream_t s = (cudaStream_t)stream;
  if (alpha_dev && cudaMemcpyAsync(alpha_dev, h->alpha, sizeof(double) * h->ne, cudaMemcpyDeviceToDevice, s) != cudaSuccess)
    return THX_ERR_CUDA;
  if (eta_dev && cudaMemcpyAsync(eta_dev, h->eta, sizeof(double) * h->ne, cudaMemcpyDeviceToDevice, s) != cudaSuccess)
    return THX_ERR_CUDA;
  return THX_OK;
}

int thx_integral_measures(thx_handle h, const double *u, double *out) {
  if (!h || !u || !out) return THX_ERR_INVALID_ARGUMENT;
  DeviceGuard dg(h->device);
  if (!dg.ok) return THX_ERR_CUDA;
  double *el = nullptr;
  if (cudaMalloc(&el, sizeof(double) * 9 * (size_t)h->ne) != cudaSuccess) {
    cudaGetLastError();
    return THX_ERR_OUT_OF_MEMORY;
  }
  MeasureArgs a;
  a.u = u; a.ne = h->ne; a.N = h->N;
  a.jac = h->jac64; a.jac_es = h->lay.jac_es; a.jac_ns = h->lay.jac_ns;
  a.w = h->ops64 + 2 * h->N * h->N;
  a.gas = h->g64; a.lte = h->lte ? 1 : 0; a.out = el; a.status = h->status;
  const int grid = (h->ne + 127) / 128;
  if (h->dim == 2) measures_kernel<2><<<grid, 128>>>(a);
  else measures_kernel<3><<<grid, 128>>>(a);
  std::vector<double> hv((size_t)9 * h->ne);
  const bool ok = cudaGetLastError() == cudaSuccess &&
                  cudaMemcpy(hv.data(), el, sizeof(double) * hv.size(), cudaMemcpyDeviceToHost) == cudaSuccess;
  cudaFree(el);
  if (!ok) return THX_ERR_CUDA;
  double r[9] = {0, 0, 0, 1e32, 0, 1e32, 0, 1e32, 0};
  for (int e = 0; e < h->ne; ++e) {
    const double *v = hv.data() + (size_t)9 * e;
    r[0] += v[0]; r[1] += v[1]; r[2] += v[2];
    r[3] = std::min(r[3], v[3]); r[4] = std::max(r[4], v[4]);
    r[5] = std::min(r[5], v[5]); r[6] = std::max(r[6], v[6]);
    r[7] = std::min(r[7], v[7]); r[8] = std::max(r[8], v[8]);
  }
  for (int k = 0; k < 9; ++k) out[k] = r[k];
  return THX_OK;
}

int thx_estimate_dt(thx_handle h, const double *u, double cfl, double *dt_out, double *rates_out) {
  if (!h || !u || !dt_out) return THX_ERR_INVALID_ARGUMENT;
  if (h->lte) return THX_ERR_UNSUPPORTED;  // ideal-gas rates only
  DeviceGuard dg(h->device);
  if (!dg.ok) return THX_ERR_CUDA;
  int st = thx::stability_rates(h, u, 0);
  if (st) return st;
  unsigned long long r[3];
  if (cudaMemcpy(r, h->stab, sizeof(r), cudaMemcpyDeviceToHost) != cudaSuccess) return THX_ERR_CUDA;
  double rates[3];
  for (int i = 0; i < 3; ++i) std::memcpy(&rates[i], &r[i], sizeof(double));
  if (rates_out) std::memcpy(rates_out, rates, sizeof(rates));
  const double total = std::max(rates[0], rates[1]) + rates[2];
  if (!(total > 0.0)) return THX_ERR_NUMERICS;
  *dt_out = cfl / total;
  return THX_OK;
}

int thx_read_status(thx_handle h, uint32_t *flags, void *stream) {
  if (!h || !flags) return THX_ERR_INVALID_ARGUMENT;
  DeviceGuard dg(h->device);
  cudaStream_t s = (cudaStream_t)stream;
  unsigned v = 0;
  if (cudaMemcpyAsync(&v, h->status, sizeof(unsigned), cudaMemcpyDeviceToHost, s) != cudaSuccess) return THX_ERR_CUDA;
  if (cudaStreamSynchronize(s) != cudaSuccess) return THX_ERR_CUDA;
  if (cudaMemsetAsync(h->status, 0, sizeof(unsigned), s) != cudaSuccess) return THX_ERR_CUDA;
  *flags = v;
  return THX_OK;
}

int thx_rhs_profile(thx_handle h, const void *u, void *dudt, void *stream, double *ms) {
  if (!h || !u || !dudt || !ms) return THX_ERR_INVALID_ARGUMENT;
  DeviceGuard dg(h->device);
  if (!dg.ok) return THX_ERR_CUDA;
  cudaStream_t s = (cudaStream_t)stream;
  cudaEvent_t ev[5];
  for (int i = 0; i < 5; ++i)
    if (cudaEventCreate(&ev[i]) != cudaSuccess) return THX_ERR_CUDA;
  int st = h->mixed ? rhs_mixed(h, (const double *)u, (double *)dudt, s, ev)
                    : run_rhs<double>(h, (const double *)u, (double *)dudt, s, 0, 0.0, nullptr, nullptr, nullptr, ev);
  if (st == THX_OK && cudaEventSynchronize(ev[4]) != cudaSuccess) st = THX_ERR_CUDA;
  for (int i = 0; i < 4 && st == THX_OK; ++i) {
    float t = 0.f;
    if (cudaEventElapsedTime(&t, ev[i], ev[i + 1]) != cudaSuccess) st = THX_ERR_CUDA;
    ms[i] = t;
  }
  for (int i = 0; i < 5; ++i) cudaEventDestroy(ev[i]);
  return st;
}

int thx_describe(thx_handle h, char *buf, size_t len) {
  if (!h || !buf || len == 0) return THX_ERR_INVALID_ARGUMENT;
  std::snprintf(buf, len, "%s", h->desc.c_str());
  return THX_OK;
}

}  // extern "C"
