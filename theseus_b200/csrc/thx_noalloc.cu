// thx_noalloc.cu -- an Euler right-hand side that allocates no device memory.
//
// Some hosts cannot let a library call cudaMalloc: a solver whose device
// memory is owned by its own pool (a memory manager that must account for
// every byte, or a caching allocator that has already reserved nearly all of
// HBM), or a time loop that must not pay cudaMalloc's implicit device-wide
// synchronisation.  thx_rhs_euler_noalloc serves them: the caller passes the
// state, the result and device-resident geometry, and the only scratch the
// kernels need -- the face-flux buffer, the element-to-face table and the
// derivative operators -- lives in one file-scope __device__ array that every
// GPU loading this library holds until the process exits.
//
// The array is shared by all calls and keeps the previous call's contents, so
// everything that must start from a known value is rewritten on every call.
// Calls that overlap on the GPU (two streams, or two host threads) race on it.
// Each call's status bits (non-positive state, a kernel that could not run, an
// out-of-range face table entry) are copied, stream-ordered, to a word the
// caller passes.
#include "thx_launch.cuh"
#include "thx_host.h"

#include <cstring>
#include <mutex>
#include <vector>

namespace {

// 8 MiB: fits, e.g., a 16^3 p=3 or a 12^3 p=4 hex mesh (3-D) and a 128^2 p=5
// quad mesh (2-D).
constexpr size_t kScratchBytes = size_t(8) << 20;
constexpr int kMaxDevices = 64;

__device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

std::mutex g_mutex;
void *g_scratch_addr[kMaxDevices] = {nullptr};

size_t round256(size_t n) { return (n + 255) & ~size_t(255); }

// Address of this device's copy of the array (host code may not use the
// array's name as a device address).  Looked up once per device, with that
// device current.
int scratch_address(int dev, unsigned char **out) {
  if (dev < 0 || dev >= kMaxDevices) return THX_ERR_UNSUPPORTED;
  std::lock_guard<std::mutex> lock(g_mutex);
  if (!g_scratch_addr[dev]) {
    void *p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) {
      cudaGetLastError();
      return THX_ERR_CUDA;
    }
    g_scratch_addr[dev] = p;
  }
  *out = static_cast<unsigned char *>(g_scratch_addr[dev]);
  return THX_OK;
}

struct OpsParam {
  double v[2 * 6 * 6 + 6];
  int n;
};

__global__ void noalloc_fill_ops(const OpsParam p, double *dst) {
  for (int i = threadIdx.x; i < p.n; i += blockDim.x) dst[i] = p.v[i];
}

// Copies the face tables into the scratch array with every entry checked:
// an entry whose element or local face is out of range is replaced by
// (element 0, local face 0), which the face kernel can read without leaving
// the state arrays, is left out of the element-to-face table, and sets
// THX_STATUS_FACE_TABLE; noalloc_poison_bad_faces later gives such a face NaN fluxes.
__global__ void noalloc_face_tables(int nf, int ne, int dim, const int *face_elem,
                                    const int *face_lface, int *fe_ok, int *fl_ok, int *elem_face,
                                    unsigned *status) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 2 * nf) return;
  const int f = t >> 1, s = t & 1;
  const int e = face_elem[t], lf = face_lface[t];
  if (e < 0 || e >= ne || lf < 0 || lf >= 2 * dim) {
    fe_ok[t] = 0;
    fl_ok[t] = 0;
    atomicOr(status, THX_STATUS_FACE_TABLE);
    return;
  }
  fe_ok[t] = e;
  fl_ok[t] = lf;
  elem_face[e * 2 * dim + lf] = 2 * f + s;
}

// NaN fluxes on every face with an out-of-range table entry (either side).
__global__ void noalloc_poison_bad_faces(int nf, int ne, int dim, int nfp, int neq,
                                         const int *face_elem, const int *face_lface,
                                         double *fstar) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= nf) return;
  bool bad = false;
  for (int s = 0; s < 2; ++s) {
    const int e = face_elem[2 * f + s], lf = face_lface[2 * f + s];
    if (e < 0 || e >= ne || lf < 0 || lf >= 2 * dim) bad = true;
  }
  if (!bad) return;
  const double nan = __longlong_as_double(0x7ff8000000000000LL);
  for (int i = 0; i < neq * nfp; ++i) fstar[(long long)f * neq * nfp + i] = nan;
}

}  // namespace

extern "C" int thx_rhs_euler_noalloc(const thx_geometry *g, const thx_config *cfg, const double *u,
                                     double *dudt, unsigned int *status_out, void *stream) {
  using namespace thx;
  if (!g || !cfg || !u || !dudt || !g->jac || !g->metric || !g->face_elem || !g->face_lface ||
      !g->face_normal || !g->face_wminus || !g->face_wplus)
    return THX_ERR_INVALID_ARGUMENT;
  if (g->dim < 2 || g->dim > 3 || g->num_elements <= 0 || g->num_faces <= 0)
    return THX_ERR_INVALID_ARGUMENT;
  if (g->num_bdr_faces > 0) return THX_ERR_UNSUPPORTED;  // periodic meshes only
  if (cfg->flow_model != THX_FLOW_EULER || cfg->precision != THX_PRECISION_FP64 || cfg->blending)
    return THX_ERR_UNSUPPORTED;
  if (cfg->volume_flux < 0 || cfg->volume_flux >= THX_FLUX_LTEEC || cfg->surface_flux < 0 ||
      cfg->surface_flux >= THX_FLUX_LTEEC || !(cfg->gamma > 1.0))
    return THX_ERR_INVALID_ARGUMENT;
  const int dim = g->dim, N = g->order + 1;
  if (N < 3 || N > 6) return THX_ERR_UNSUPPORTED;
  const int nd = dim == 2 ? N * N : N * N * N;
  const int nfp = dim == 2 ? N : N * N;
  const int neq = dim + 2, ne = g->num_elements, nf = g->num_faces;
  // scratch layout: [ops][status][elem_face][checked face tables][face fluxes]
  const size_t ops_bytes = round256(sizeof(double) * (2 * N * N + N));
  const size_t status_bytes = 256;
  const size_t ef_bytes = round256(sizeof(int) * (size_t)ne * 2 * dim);
  const size_t ft_bytes = round256(sizeof(int) * (size_t)nf * 2);
  const size_t fs_bytes = round256(sizeof(double) * (size_t)nf * nfp * neq);
  if (ops_bytes + status_bytes + ef_bytes + 2 * ft_bytes + fs_bytes > kScratchBytes)
    return THX_ERR_INVALID_ARGUMENT;

  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) { cudaGetLastError(); return THX_ERR_NO_DEVICE; }
  unsigned char *base = nullptr;
  int st = scratch_address(dev, &base);
  if (st) return st;
  double *ops = reinterpret_cast<double *>(base);
  unsigned *status = reinterpret_cast<unsigned *>(base + ops_bytes);
  int *elem_face = reinterpret_cast<int *>(base + ops_bytes + status_bytes);
  int *fe_ok = reinterpret_cast<int *>(base + ops_bytes + status_bytes + ef_bytes);
  int *fl_ok = reinterpret_cast<int *>(base + ops_bytes + status_bytes + ef_bytes + ft_bytes);
  double *fstar = reinterpret_cast<double *>(base + ops_bytes + status_bytes + ef_bytes + 2 * ft_bytes);
  cudaStream_t s = (cudaStream_t)stream;

  // derivative operators (host arithmetic, passed by value)
  OpsParam op;
  op.n = 2 * N * N + N;
  {
    std::vector<double> x(N), w(N), D(N * N), Dh(N * N), Dh2(N * N);
    lgl_rule(N, x.data(), w.data());
    derivative_operators(N, x.data(), w.data(), D.data(), Dh.data(), Dh2.data());
    std::memcpy(op.v, Dh2.data(), sizeof(double) * N * N);
    std::memcpy(op.v + N * N, Dh.data(), sizeof(double) * N * N);
    std::memcpy(op.v + 2 * N * N, w.data(), sizeof(double) * N);
  }
  noalloc_fill_ops<<<1, 128, 0, s>>>(op, ops);
  if (cudaMemsetAsync(status, 0, sizeof(unsigned), s) != cudaSuccess) return THX_ERR_CUDA;
  if (cudaMemsetAsync(elem_face, 0xff, sizeof(int) * (size_t)ne * 2 * dim, s) != cudaSuccess)
    return THX_ERR_CUDA;
  noalloc_face_tables<<<(2 * nf + 255) / 256, 256, 0, s>>>(nf, ne, dim, g->face_elem, g->face_lface,
                                                           fe_ok, fl_ok, elem_face, status);
  if (cudaGetLastError() != cudaSuccess) return THX_ERR_CUDA;

  // the same face and volume kernels as thx_rhs, on the full per-node layout
  const GasT<double> gas = [&] {
    GasT<double> r{};
    const double gm1 = cfg->gamma - 1.0, gm1_inv = 1.0 / gm1;
    const double cp = (cfg->gamma * gm1_inv) * cfg->R_gas;
    r.gamma = cfg->gamma; r.gm1 = gm1; r.gm1_inv = gm1_inv; r.R_gas = cfg->R_gas; r.cp = cp;
    r.Pr_inv = 1.0 / cfg->Pr; r.mu = cfg->mu; r.mu0 = cfg->mu0; r.mu_bulk = cfg->mu_bulk;
    r.T0 = cfg->T0; r.Ts = cfg->Ts; r.gm1_av_inv = 2.0 / (cfg->gamma + cfg->gamma - 2.0);
    r.inv_gm1 = 1.0 / (cfg->gamma - 1.0); r.cv = cp / cfg->gamma; r.sutherland = cfg->sutherland;
    return r;
  }();
  FaceKernels0 fk = dim == 2 ? face_kernels_0_2() : face_kernels_0_3();
  FaceArgs<double> fa{};  // value-initialised: order (face processing order) stays null
  fa.u = u; fa.ne = ne; fa.nf = nf; fa.N = N;
  fa.face_elem = fe_ok; fa.face_lface = fl_ok;
  fa.normal = g->face_normal; fa.n_fs = nfp; fa.n_ps = 1;
  fa.vflux = nullptr; fa.fstar = fstar; fa.gas = gas;
  if (fk.face[cfg->surface_flux][0](fa, s) != cudaSuccess) return THX_ERR_CUDA;
  noalloc_poison_bad_faces<<<(nf + 127) / 128, 128, 0, s>>>(nf, ne, dim, nfp, neq, g->face_elem,
                                                             g->face_lface, fstar);
  if (cudaGetLastError() != cudaSuccess) return THX_ERR_CUDA;

  const int vk = (cfg->volume_flux == THX_FLUX_CHANDRASHEKAR) ? VOL_CHANDRASHEKAR
               : (cfg->volume_flux == THX_FLUX_RANOCHA)     ? VOL_RANOCHA
               : (cfg->volume_flux == THX_FLUX_PIROZZOLI)   ? VOL_PIROZZOLI
                                                            : VOL_CENTRAL;
  VolLaunch<double> vol = nullptr;
#define THX_NOALLOC_PICK(P, D, NN) \
  if (dim == D && N == NN) vol = order_kernels_##P##_##D##_##NN().vol[vk][0][0];
  THX_FOR_ORDERS(THX_NOALLOC_PICK, 0, 2)
  THX_FOR_ORDERS(THX_NOALLOC_PICK, 0, 3)
#undef THX_NOALLOC_PICK
  if (!vol) return THX_ERR_UNSUPPORTED;
  if (vol(VolArgs<double>{}, s, 1) != cudaSuccess) { cudaGetLastError(); return THX_ERR_CUDA; }
  VolArgs<double> va{};
  va.u = u; va.du = dudt; va.ne = ne;
  va.jac = g->jac; va.jac_es = nd; va.jac_ns = 1;
  va.met = g->metric; va.met_es = (long long)nd * dim * dim; va.met_ns = dim * dim;
  va.elem_face = elem_face; va.fstar = fstar;
  va.wm = g->face_wminus; va.wp = g->face_wplus; va.w_fs = nfp; va.w_ps = 1;
  va.nf_int = nf; va.bw = nullptr;  // periodic: every face is interior
  va.vflux = nullptr; va.alpha = nullptr;
  va.fv_flux = cfg->fv_flux; va.gas = gas; va.ops = ops;
  va.stage = 0; va.status = status;
  if (vol(va, s, 0) != cudaSuccess) return THX_ERR_CUDA;
  // the status word, stream-ordered, to the caller's device or page-locked
  // host word
  if (status_out &&
      cudaMemcpyAsync(status_out, status, sizeof(unsigned), cudaMemcpyDefault, s) != cudaSuccess) {
    cudaGetLastError();
    return THX_ERR_CUDA;
  }
  return THX_OK;
}
