// thx_launch.cuh -- typed launchers for the kernel templates and the names of
// the per-(precision, dimension, order) instantiation units.
#pragma once
#include "thx_kernels.cuh"
#include "thx_bc.cuh"

#include <algorithm>

namespace thx {

using PREC_T_0 = double;
using PREC_T_1 = float;

template <typename R> using VolLaunch = cudaError_t (*)(const VolArgs<R> &, cudaStream_t, int prepare);
template <typename R> using FaceLaunch = cudaError_t (*)(const FaceArgs<R> &, cudaStream_t);
template <typename R> using GradLaunch = cudaError_t (*)(const GradArgs<R> &, cudaStream_t, int prepare);
template <typename R> using BlendLaunch = cudaError_t (*)(const BlendArgs<R> &, cudaStream_t);
// batched persistent forms: (argument table, work list, device work count,
// grid size, stream, prepare)
template <typename R>
using VolBatchLaunch = cudaError_t (*)(const VolArgs<R> *, const BatchWork *, const int *, int,
                                       cudaStream_t, int);
template <typename R>
using GradBatchLaunch = cudaError_t (*)(const GradArgs<R> *, const BatchWork *, const int *, int,
                                        cudaStream_t, int);
template <typename R>
using FaceBatchLaunch = cudaError_t (*)(const FaceArgs<R> *, const BatchWork *, const int *, int,
                                        cudaStream_t, int);

template <typename R, int DIM, int N, int VOL, bool NS, bool BLEND>
constexpr size_t volume_smem_bytes(bool metric_per_node) {
  return VolSmem<R, DIM, N, VOL, NS, BLEND>::bytes(metric_per_node);
}

template <typename R, int DIM, int N, int VOL, bool NS, bool BLEND>
cudaError_t launch_volume(const VolArgs<R> &a, cudaStream_t s, int prepare) {
  using S = Shape<DIM, N>;
  static_assert(S::PAIRS >= S::ND, "subcell FV rate aliases the pair-flux buffer");
  constexpr int MINB = VolMinBlocks<R, VOL, BLEND>::value;
  if (prepare) {
    const int bytes = (int)volume_smem_bytes<R, DIM, N, VOL, NS, BLEND>(true);
    if constexpr (MINB > 0)
      return cudaFuncSetAttribute(volume_kernel_mb<R, DIM, N, VOL, NS, BLEND, MINB>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    else
      return cudaFuncSetAttribute(volume_kernel<R, DIM, N, VOL, NS, BLEND>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  }
  if (a.ne <= 0) return cudaSuccess;
  const size_t smem = volume_smem_bytes<R, DIM, N, VOL, NS, BLEND>(a.met_ns != 0);
  const int grid = (a.ne + S::EPB - 1) / S::EPB;
  if constexpr (MINB > 0) volume_kernel_mb<R, DIM, N, VOL, NS, BLEND, MINB><<<grid, S::THREADS, smem, s>>>(a);
  else volume_kernel<R, DIM, N, VOL, NS, BLEND><<<grid, S::THREADS, smem, s>>>(a);
  return cudaGetLastError();
}

// Persistent, bulk-copy-staged volume kernel (no blending): as many CTAs as
// fit on the device at once, each walking the element blocks.
template <typename R, int DIM, int N, int VOL, bool NS>
cudaError_t launch_volume_tma(const VolArgs<R> &a, cudaStream_t s, int prepare) {
  using S = Shape<DIM, N>;
  using T_ = VolTmaSmem<R, DIM, N, VOL, NS, false>;
  constexpr int MINB = VolMinBlocks<R, VOL, false>::value;
  auto kern = volume_tma_kernel<R, DIM, N, VOL, NS, false, MINB>;
  static int cap[2] = {0, 0};  // resident CTAs on the device: metric per element / per node
  if (prepare) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)T_::bytes(true));
    if (e != cudaSuccess) return e;
    int dev = 0, sms = 0;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
    for (int m = 0; m < 2; ++m) {
      int per = 0;
      if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kern, S::THREADS, T_::bytes(m == 1))) !=
          cudaSuccess)
        return e;
      cap[m] = (per > 0 ? per : 1) * sms;
    }
    return cudaSuccess;
  }
  if (a.ne <= 0) return cudaSuccess;
  const int m = a.met_ns != 0 ? 1 : 0;
  const int nblocks = (a.ne + S::EPB - 1) / S::EPB;
  const int grid = std::min(nblocks, cap[m] > 0 ? cap[m] : 148);
  kern<<<grid, S::THREADS, T_::bytes(a.met_ns != 0), s>>>(a);
  return cudaGetLastError();
}

template <typename R, int DIM, int SURF, bool NS>
cudaError_t launch_face(const FaceArgs<R> &a, cudaStream_t s) {
  const int nfp = DIM == 2 ? a.N : a.N * a.N;
  const long long total = (long long)a.nf * nfp;
  if (total <= 0) return cudaSuccess;
  const int grid = (int)((total + 127) / 128);
  if constexpr (SURF == SURF_LTEEC) face_kernel_lte<DIM, NS><<<grid, 128, 0, s>>>(a);
  else if constexpr (IsF32<R>::value) face_kernel_f32<DIM, SURF, NS><<<grid, 128, 0, s>>>(a);
  else face_kernel_f64<DIM, SURF, NS><<<grid, 128, 0, s>>>(a);
  return cudaGetLastError();
}

template <typename R, int DIM, int N, bool LTE = false>
cudaError_t launch_grad(const GradArgs<R> &a, cudaStream_t s, int prepare) {
  using S = Shape<DIM, N>;
  constexpr size_t smem = grad_smem_bytes<R, DIM, N>();
  if constexpr (LTE) {
    if (prepare)
      return cudaFuncSetAttribute(grad_kernel_lte<DIM, N>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)smem);
    if (a.ne <= 0) return cudaSuccess;
    grad_kernel_lte<DIM, N><<<(a.ne + S::EPB - 1) / S::EPB, S::THREADS, smem, s>>>(a);
  } else {
    if (prepare)
      return cudaFuncSetAttribute(grad_kernel<R, DIM, N, LTE>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (a.ne <= 0) return cudaSuccess;
    const int grid = (a.ne + S::EPB - 1) / S::EPB;
    grad_kernel<R, DIM, N, LTE><<<grid, S::THREADS, smem, s>>>(a);
  }
  return cudaGetLastError();
}

// Gradient from precomputed entropy variables (a.svars, entropy_kernel).
template <typename R, int DIM, int N>
cudaError_t launch_grad_sv(const GradArgs<R> &a, cudaStream_t s, int prepare) {
  using S = Shape<DIM, N>;
  constexpr size_t smem = grad_sv_smem_bytes<R, DIM, N>();
  if (prepare)
    return cudaFuncSetAttribute(grad_sv_kernel<R, DIM, N>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)smem);
  if (a.ne <= 0) return cudaSuccess;
  if (!a.svars) return cudaErrorInvalidValue;
  const int grid = (a.ne + S::EPB - 1) / S::EPB;
  grad_sv_kernel<R, DIM, N><<<grid, S::THREADS, smem, s>>>(a);
  return cudaGetLastError();
}

template <typename R>
using EntropyLaunch = cudaError_t (*)(const R *, long long, const GasT<R> &, R *, cudaStream_t);

template <typename R, int DIM>
cudaError_t launch_entropy(const R *u, long long L, const GasT<R> &g, R *sv, cudaStream_t s) {
  if (L <= 0) return cudaSuccess;
  entropy_kernel<R, DIM><<<(unsigned)((L + 255) / 256), 256, 0, s>>>(u, L, g, sv);
  return cudaGetLastError();
}

template <int DIM>
cudaError_t launch_lte_temperature(const double *u, long long L, const LteDev &t, double *Tn,
                                   int *Cn, unsigned *status, cudaStream_t s) {
  if (L <= 0) return cudaSuccess;
  const int grid = (int)std::min<long long>((L + 255) / 256, 148LL * 8);
  lte_temperature_kernel<DIM><<<grid, 256, 0, s>>>(u, L, t, Tn, Cn, status);
  return cudaGetLastError();
}

template <typename R, int DIM, int N, int VOL, bool NS, int EPBX = 0>
cudaError_t launch_volume_batched(const VolArgs<R> *args, const BatchWork *work, const int *nwork,
                                  int grid, cudaStream_t s, int prepare) {
  using S = Shape<DIM, N, EPBX>;
  constexpr size_t smem = VolSmem<R, DIM, N, VOL, NS, false, EPBX>::bytes(true);
  if (prepare)
    return cudaFuncSetAttribute(volume_batched<R, DIM, N, VOL, NS, EPBX>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (grid <= 0) return cudaSuccess;
  volume_batched<R, DIM, N, VOL, NS, EPBX><<<grid, S::THREADS, smem, s>>>(args, work, nwork);
  return cudaGetLastError();
}

template <typename R, int DIM, int N, int EPBX = 0>
cudaError_t launch_grad_batched(const GradArgs<R> *args, const BatchWork *work, const int *nwork,
                                int grid, cudaStream_t s, int prepare) {
  using S = Shape<DIM, N, EPBX>;
  constexpr size_t smem = grad_smem_bytes<R, DIM, N, EPBX>();
  if (prepare)
    return cudaFuncSetAttribute(grad_batched<R, DIM, N, EPBX>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (grid <= 0) return cudaSuccess;
  grad_batched<R, DIM, N, EPBX><<<grid, S::THREADS, smem, s>>>(args, work, nwork);
  return cudaGetLastError();
}

// Elements per CTA of the batched kernels' half-size variant (0: none, the
// full-size CTA already holds one element).
template <int DIM, int N>
constexpr int half_epb() {
  return Shape<DIM, N>::EPB >= 2 ? Shape<DIM, N>::EPB / 2 : 0;
}

template <typename R, int DIM, int SURF, bool NS>
cudaError_t launch_face_batched(const FaceArgs<R> *args, const BatchWork *work, const int *nwork,
                                int grid, cudaStream_t s, int prepare) {
  if (prepare || grid <= 0) return cudaSuccess;
  face_batched<R, DIM, SURF, NS><<<grid, 128, 0, s>>>(args, work, nwork);
  return cudaGetLastError();
}

// FP64 islands: walkers over device-side lists (grid fixed, length read on
// the device)
template <typename R>
using VolListLaunch = cudaError_t (*)(const VolArgs<R> &, const int *, const int *, cudaStream_t, int);
template <typename R>
using BlendListLaunch = cudaError_t (*)(const BlendArgs<R> &, const int *, const int *, cudaStream_t);
template <typename R>
using FaceListLaunch = cudaError_t (*)(const FaceArgs<R> &, const int *, cudaStream_t);
constexpr int kIslandGrid = 148 * 4;

template <typename R, int DIM, int N, int VOL>
cudaError_t launch_volume_list(const VolArgs<R> &a, const int *list, const int *count, cudaStream_t s,
                               int prepare) {
  using S = Shape<DIM, N>;
  const int bytes = (int)volume_smem_bytes<R, DIM, N, VOL, false, true>(true);
  if (prepare)
    return cudaFuncSetAttribute(volume_list_kernel<R, DIM, N, VOL>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  const size_t smem = volume_smem_bytes<R, DIM, N, VOL, false, true>(a.met_ns != 0);
  volume_list_kernel<R, DIM, N, VOL><<<kIslandGrid, S::THREADS, smem, s>>>(a, list, count);
  return cudaGetLastError();
}

template <typename R, int DIM, int N>
cudaError_t launch_fv_list(const VolArgs<R> &a, const int *list, const int *count, cudaStream_t s,
                           int prepare) {
  using S = Shape<DIM, N>;
  constexpr size_t smem = FvSmem<R, DIM, N>::bytes();
  if (prepare)
    return cudaFuncSetAttribute(fv_list_kernel<R, DIM, N>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)smem);
  fv_list_kernel<R, DIM, N><<<kIslandGrid, S::THREADS, smem, s>>>(a, list, count);
  return cudaGetLastError();
}

template <typename R, int DIM, int N>
cudaError_t launch_blend_list(const BlendArgs<R> &a, const int *list, const int *count, cudaStream_t s) {
  blend_warp_kernel<R, DIM, N><<<kIslandGrid, 32 * kBlendWarps, 0, s>>>(a, list, count);
  return cudaGetLastError();
}

template <typename R, int DIM, int SURF>
cudaError_t launch_face_list(const FaceArgs<R> &a, const int *count, cudaStream_t s) {
  face_list_kernel<R, DIM, SURF><<<148 * 8, 128, 0, s>>>(a, count);
  return cudaGetLastError();
}

using BndLaunch = cudaError_t (*)(const BndArgs &, cudaStream_t);

template <int DIM, int SURF, bool NS>
cudaError_t launch_bnd(const BndArgs &a, cudaStream_t s) {
  const int nfp = DIM == 2 ? a.N : a.N * a.N;
  const long long total = (long long)a.nbf * nfp;
  if (total <= 0) return cudaSuccess;
  bnd_face_kernel<DIM, SURF, NS><<<(unsigned)((total + 127) / 128), 128, 0, s>>>(a);
  return cudaGetLastError();
}

template <typename R, int DIM, int N>
cudaError_t launch_fv(const VolArgs<R> &a, cudaStream_t s, int prepare) {
  using S = Shape<DIM, N>;
  constexpr size_t smem = FvSmem<R, DIM, N>::bytes();
  if (prepare)
    return cudaFuncSetAttribute(fv_kernel<R, DIM, N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (a.ne <= 0 || !a.alpha || !a.fvrate) return cudaSuccess;
  const int grid = (a.ne + S::EPB - 1) / S::EPB;
  fv_kernel<R, DIM, N><<<grid, S::THREADS, smem, s>>>(a);
  return cudaGetLastError();
}

template <typename R, int DIM, int N>
cudaError_t launch_blend(const BlendArgs<R> &a, cudaStream_t s) {
  if (a.ne <= 0) return cudaSuccess;
  const int grid = (a.ne + kBlendWarps - 1) / kBlendWarps;  // one warp per element
  blend_warp_kernel<R, DIM, N><<<grid, 32 * kBlendWarps, 0, s>>>(a, nullptr, nullptr);
  return cudaGetLastError();
}

template <typename R>
struct OrderKernelsT {
  VolLaunch<R> vol[4][2][2];     // [volume flux][ns][blend]
  VolLaunch<R> vol_tma[4][2];    // bulk-copy-staged, no blending: [volume flux][ns]
  GradLaunch<R> grad;
  BlendLaunch<R> blend;
  VolLaunch<R> fv;               // subcell FV rate of blended elements
  VolBatchLaunch<R> volb[4][2];  // [volume flux][ns]
  GradBatchLaunch<R> gradb;
  // half-size CTAs (epb_half elements each; 0 and null when EPB is 1)
  int epb, epb_half;
  VolBatchLaunch<R> volb_half[4][2];
  GradBatchLaunch<R> gradb_half;
  // FP64 islands (Euler, blending; set in the FP64 units only)
  VolListLaunch<R> voll[4];      // [volume flux]
  VolListLaunch<R> fvl;
  BlendListLaunch<R> blendl;
};
template <typename R>
struct FaceKernelsT {
  FaceLaunch<R> face[6][2];      // [surface flux][ns]
  FaceBatchLaunch<R> faceb[6][2];
  BndLaunch bnd[6][2];           // boundary faces [surface flux][ns] (FP64)
  EntropyLaunch<R> entropy;      // entropy variables of every node (NS)
  FaceListLaunch<R> facel[6];    // FP64 islands: listed faces (Euler; FP64 units only)
};
using OrderKernels0 = OrderKernelsT<double>;
using OrderKernels1 = OrderKernelsT<float>;
using FaceKernels0 = FaceKernelsT<double>;
using FaceKernels1 = FaceKernelsT<float>;
// LTE Helmholtz gas, FP64: LTEEC volume kernel [euler|ns], gradient, face
// flux [euler|ns].
struct LteKernels { VolLaunch<double> vol[2]; GradLaunch<double> grad; };
struct LteFaceKernels { FaceLaunch<double> face[2]; };

#define THX_DECLARE_ORDER(P, D, N) OrderKernels##P order_kernels_##P##_##D##_##N();
#define THX_DECLARE_FACE(P, D) FaceKernels##P face_kernels_##P##_##D();
#define THX_FOR_ORDERS(X, P, D) X(P, D, 3) X(P, D, 4) X(P, D, 5) X(P, D, 6)
THX_FOR_ORDERS(THX_DECLARE_ORDER, 0, 2)
THX_FOR_ORDERS(THX_DECLARE_ORDER, 0, 3)
THX_FOR_ORDERS(THX_DECLARE_ORDER, 1, 2)
THX_FOR_ORDERS(THX_DECLARE_ORDER, 1, 3)
#define THX_DECLARE_LTE(P, D, N) LteKernels lte_kernels_##D##_##N();
THX_FOR_ORDERS(THX_DECLARE_LTE, 0, 2)
THX_FOR_ORDERS(THX_DECLARE_LTE, 0, 3)
LteFaceKernels lte_face_kernels_2();
LteFaceKernels lte_face_kernels_3();
THX_DECLARE_FACE(0, 2)
THX_DECLARE_FACE(0, 3)
THX_DECLARE_FACE(1, 2)
THX_DECLARE_FACE(1, 3)

}  // namespace thx
