// thx_operator.cuh -- internal: the operator object behind thx_handle, shared
// by the C ABI unit (thx_api.cu) and the batch engine (thx_engine.cu).
#pragma once
#include "thx_launch.cuh"
#include "theseus_b200.h"

#include <string>
#include <vector>

namespace thx {

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
  double *alpha = nullptr, *eta = nullptr, *vinv = nullptr;
  unsigned *status = nullptr;
  unsigned long long *stab = nullptr;
  double *y = nullptr;
  float *yf = nullptr;
  float *kf = nullptr;   // FP32 right-hand side scratch of thx_rhs (mixed mode)
  thx::Offsets off{};    // FP32 working-copy offsets (mixed mode)
  thx::VolLaunch<double> vol64 = nullptr;
  thx::GradLaunch<double> grad64 = nullptr;
  thx::BlendLaunch<double> blend64 = nullptr;
  thx::FaceLaunch<double> face64 = nullptr;
  thx::VolLaunch<float> vol32 = nullptr;
  thx::GradLaunch<float> grad32 = nullptr;
  thx::BlendLaunch<float> blend32 = nullptr;
  thx::FaceLaunch<float> face32 = nullptr;
  thx::GasT<double> g64;
  thx::GasT<float> g32;
  bool lte = false;        // LTE Helmholtz gas (g64.lte, g64.Tn on the device)
  double *Tn = nullptr;    // recovered node temperatures [elem][node]
  double threshold = 0.0;
  double adv_scale = 0.0, dif_scale = 0.0, surf_scale = 0.0;
  std::vector<void *> allocs;
  // stream-ordered allocation (batch engine): when pool is set, device
  // buffers come from it on setup_stream and uploads are asynchronous there
  cudaMemPool_t pool = nullptr;
  cudaStream_t setup_stream = nullptr;
  std::string desc;
};

namespace thx {

// Builds the operator's device data (geometry, operators, scratch, kernel
// choice); LTE gas when table != nullptr.  On failure the caller frees.
int op_create(const thx_geometry *g, const thx_config *cfg, thx_operator_s *h,
              const thx_lte_table *table);
void op_free(thx_operator_s *h);

// Kernel arguments of one right-hand side (stage 0: du = L(u); stages 1..3:
// fused SSP-RK3 stage on um / y, with the FP32 working copy yf).
template <typename R>
void op_args(thx_operator_s *h, const R *u, R *du, int stage, double dt, double *um, double *y,
             float *yf, GradArgs<R> &ga, FaceArgs<R> &fa, VolArgs<R> &va);

// FP32 working copy yf = float(u - offset) of the FP64 state (mixed mode).
int op_to_working_copy(thx_operator_s *h, const double *u, cudaStream_t s);

}  // namespace thx
