// thx_operator.cuh -- internal: the operator object behind thx_handle, shared
// by the C ABI unit (thx_api.cu) and the batch engine (thx_engine.cu).
#pragma once
#include "thx_launch.cuh"
#include "theseus_b200.h"

#include <cstring>
#include <string>
#include <vector>

#include <cstdio>
#include <deque>
#include <mutex>

#include <chrono>

#include "thx_ring.h"

namespace thx {

// The CUDA call that failed last on this thread inside the library, with the
// runtime's error name ("" until one fails); read by thx_last_cuda_failure.
inline thread_local char last_cuda_failure[192] = "";
inline int cuda_failed(cudaError_t e, const char *call, int status = THX_ERR_CUDA) {
  std::snprintf(last_cuda_failure, sizeof(last_cuda_failure), "%s: %s", call, cudaGetErrorName(e));
  cudaGetLastError();
  return status;
}
#define THX_CU(call)                                           \
  do {                                                         \
    const cudaError_t thx_e_ = (call);                         \
    if (thx_e_ != cudaSuccess) return thx::cuda_failed(thx_e_, #call); \
  } while (0)

// Pinned host staging ring for stream-ordered uploads: a copy is written into
// the ring on the host and sent with cudaMemcpyAsync, so the call neither
// waits for the stream nor goes through the driver's pageable path.  Space
// is reclaimed in FIFO order once each copy's event has completed.
class HostRing {
 public:
  ~HostRing() {
    for (cudaEvent_t ev : busy_) cudaEventDestroy(ev);
    for (cudaEvent_t ev : spare_) cudaEventDestroy(ev);
    if (buf_) cudaFreeHost(buf_);
  }
  int init(size_t bytes) {
    if (cudaHostAlloc((void **)&buf_, bytes, cudaHostAllocDefault) != cudaSuccess) {
      cudaGetLastError();
      buf_ = nullptr;
      return THX_ERR_OUT_OF_MEMORY;
    }
    space_.reset(bytes);
    return THX_OK;
  }
  // host -> device copy of `bytes` on stream s through the ring (copies of
  // more than half the ring go directly)
  int copy(void *dst, const void *src, size_t bytes, cudaStream_t s) {
    std::lock_guard<std::mutex> lock(mu_);
    const size_t need = (bytes + 255) & ~size_t(255);
    if (!buf_ || need > space_.capacity() / 2) {
      const cudaError_t e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s);
      return e == cudaSuccess ? THX_OK : cuda_failed(e, "cudaMemcpyAsync(upload)");
    }
    size_t off;
    const auto t0 = std::chrono::steady_clock::now();
    while (!space_.place(need, &off)) {  // wait for the oldest copy
      const cudaError_t e = cudaEventSynchronize(busy_.front());
      if (e != cudaSuccess) return cuda_failed(e, "cudaEventSynchronize(upload ring)");
      spare_.push_back(busy_.front());
      busy_.pop_front();
      space_.pop();
    }
    const auto t1 = std::chrono::steady_clock::now();
    std::memcpy(buf_ + off, src, bytes);
    const auto t2 = std::chrono::steady_clock::now();
    wait_s_ += std::chrono::duration<double>(t1 - t0).count();
    copy_s_ += std::chrono::duration<double>(t2 - t1).count();
    cudaError_t e = cudaMemcpyAsync(dst, buf_ + off, bytes, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return cuda_failed(e, "cudaMemcpyAsync(upload ring)");
    cudaEvent_t ev;
    if (!spare_.empty()) {
      ev = spare_.back();
      spare_.pop_back();
    } else if ((e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming)) != cudaSuccess) {
      return cuda_failed(e, "cudaEventCreate(upload ring)");
    }
    // the span is live from here on: its bytes are read by the queued copy
    busy_.push_back(ev);
    space_.push(off, need);
    if ((e = cudaEventRecord(ev, s)) != cudaSuccess) {
      // unrecorded: the event would report complete at once, so wait for the
      // stream before the span can be reused
      cudaStreamSynchronize(s);
      return cuda_failed(e, "cudaEventRecord(upload ring)");
    }
    return THX_OK;
  }
  // host seconds spent waiting for space and copying into the ring
  void times(double *wait_s, double *copy_s) {
    std::lock_guard<std::mutex> lock(mu_);
    *wait_s = wait_s_;
    *copy_s = copy_s_;
  }

 private:
  std::mutex mu_;
  double wait_s_ = 0.0, copy_s_ = 0.0;
  unsigned char *buf_ = nullptr;
  RingSpace space_;
  std::deque<cudaEvent_t> busy_;  // one per live span, oldest first
  std::vector<cudaEvent_t> spare_;
};

// Strides of the (possibly compressed) geometry arrays on the device.
struct Layout {
  long long jac_es = 0, jac_ns = 0, met_es = 0, met_ns = 0;
  long long n_fs = 0, n_ps = 0, w_fs = 0, w_ps = 0;
  long long sub_es[3] = {0, 0, 0};
};

}  // namespace thx

struct thx_operator_s {
  int device = 0;
  thx_config cfg{};
  int dim = 0, order = 0, N = 0, nd = 0, nfp = 0, neq = 0, ne = 0, nf = 0;
  long long L = 0;
  bool mixed = false, ns = false, blend = false;
  thx::Layout lay;
  double *jac64 = nullptr, *met64 = nullptr, *nrm64 = nullptr, *wm64 = nullptr, *wp64 = nullptr;
  double *sub64[3] = {nullptr, nullptr, nullptr}, *ops64 = nullptr, *D64 = nullptr;
  float *jac32 = nullptr, *met32 = nullptr, *nrm32 = nullptr, *wm32 = nullptr, *wp32 = nullptr;
  float *sub32[3] = {nullptr, nullptr, nullptr}, *ops32 = nullptr, *D32 = nullptr;
  int *face_elem = nullptr, *face_lface = nullptr, *elem_face = nullptr;
  void *fstar = nullptr, *vflux = nullptr;  // face fluxes; NS physical viscous flux
  void *svars = nullptr;     // FP64 NS (ideal gas): entropy variables of every node
  int *face_order = nullptr; // interior faces sorted by their minus-side element
  double *alpha = nullptr, *eta = nullptr, *vinv = nullptr;
  void *fvrate = nullptr;  // subcell FV rate of blended elements (blending only)
  // boundary faces: face slots nf .. nf+nbf-1 of fstar/elem_face
  int nbf = 0;
  int *bdr_elem = nullptr, *bdr_lface = nullptr, *bdr_bc = nullptr;
  double *bdr_nrm = nullptr, *bdr_w = nullptr, *bc_data = nullptr;
  double *bgrad = nullptr;   // NS: primitive gradients at the boundary points
  thx_bc *bcs = nullptr;
  unsigned *status = nullptr;
  unsigned long long *stab = nullptr;
  double *dtd = nullptr;   // device-side CFL time step (thx_rk3_steps_cfl)
  double *y = nullptr;
  float *yf = nullptr;
  thx::Offsets off{};    // FP32 working-copy offsets (mixed mode)
  thx::VolLaunch<double> vol64 = nullptr;
  thx::GradLaunch<double> grad64 = nullptr;
  thx::BlendLaunch<double> blend64 = nullptr;
  thx::VolLaunch<double> fv64 = nullptr;
  thx::FaceLaunch<double> face64 = nullptr;
  thx::EntropyLaunch<double> ent64 = nullptr;
  // FP32-mixed Euler with blending: FP64 islands (blocks holding blended
  // elements and their faces evaluated in FP64; thx_kernels.cuh)
  bool islands = false;
  int isl_epb = 1;
  int *isl_flag = nullptr, *isl_blocks = nullptr, *isl_faces = nullptr;
  int *isl_count = nullptr;  // [0] blocks, [1] faces
  int *isl_static = nullptr; // blocks next to a boundary face (islands at every RHS)
  bool isl_alpha_in = false; // blended blocks are islands
  thx::BndLaunch isl_bnd = nullptr;
  double *isl_fstar = nullptr, *isl_alpha = nullptr, *isl_eta = nullptr, *isl_fvrate = nullptr;
  thx::VolListLaunch<double> isl_vol = nullptr, isl_fv = nullptr;
  thx::BlendListLaunch<double> isl_blend = nullptr;
  thx::FaceListLaunch<double> isl_face = nullptr;
  thx::EntropyLaunch<float> ent32 = nullptr;
  thx::BndLaunch bnd64 = nullptr;   // boundary faces (FP64 Euler)
  thx::VolLaunch<float> vol32 = nullptr;
  thx::GradLaunch<float> grad32 = nullptr;
  thx::BlendLaunch<float> blend32 = nullptr;
  thx::VolLaunch<float> fv32 = nullptr;
  thx::FaceLaunch<float> face32 = nullptr;
  thx::GasT<double> g64;
  thx::GasT<float> g32;
  bool lte = false;        // LTE Helmholtz gas (g64.lte, g64.Tn on the device)
  double *Tn = nullptr;    // recovered node temperatures [elem][node]
  int *Cn = nullptr;       // their table cells (lte_at's cell.off; -1: none)
  double threshold = 0.0;
  double adv_scale = 0.0, dif_scale = 0.0, surf_scale = 0.0;
  std::vector<void *> allocs;
  // stream-ordered allocation (batch engine): when pool is set, device
  // buffers come from it on setup_stream and uploads are asynchronous there
  cudaMemPool_t pool = nullptr;
  cudaStream_t setup_stream = nullptr;
  thx::HostRing *ring = nullptr;  // pinned staging of uploads (may be null)
  // host-buffer pipeline (thx_rhs_host): two device state/rate buffers, a
  // copy-in and a copy-out stream and their events
  double *hp_u[2] = {nullptr, nullptr}, *hp_du[2] = {nullptr, nullptr};
  cudaStream_t hp_in = nullptr, hp_out = nullptr;
  cudaEvent_t hp_ev[7] = {};  // start, in[2], rhs[2], out[2]
  std::string desc;
};

namespace thx {

// Builds the operator's device data (geometry, operators, scratch, kernel
// choice); LTE gas when table != nullptr.  On failure the caller frees.
int op_create(const thx_geometry *g, const thx_config *cfg, thx_operator_s *h,
              const thx_lte_table *table, const thx_operator_s *donor = nullptr);
void op_free(thx_operator_s *h);

// Kernel arguments of one right-hand side (stage 0: du = L(u); stages 1..3:
// fused SSP-RK3 stage on um / y, with the FP32 working copy yf).
template <typename R>
void op_args(thx_operator_s *h, const R *u, R *du, int stage, double dt, double *um, double *y,
             float *yf, GradArgs<R> &ga, FaceArgs<R> &fa, VolArgs<R> &va);

// FP32 working copy yf = float(u - offset) of the FP64 state (mixed mode).
int op_to_working_copy(thx_operator_s *h, const double *u, cudaStream_t s);

}  // namespace thx
