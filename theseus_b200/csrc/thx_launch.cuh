// thx_launch.cuh -- typed launchers for the kernel templates and the names of
// the per-(precision, dimension, order) instantiation units.
#pragma once
#include "thx_kernels.cuh"

namespace thx {

using PREC_T_0 = double;
using PREC_T_1 = float;

template <typename R> using VolLaunch = cudaError_t (*)(const VolArgs<R> &, cudaStream_t, int prepare);
template <typename R> using FaceLaunch = cudaError_t (*)(const FaceArgs<R> &, cudaStream_t);
template <typename R> using GradLaunch = cudaError_t (*)(const GradArgs<R> &, cudaStream_t, int prepare);
template <typename R> using BlendLaunch = cudaError_t (*)(const BlendArgs<R> &, cudaStream_t);

template <typename R, int DIM, int N, int VOL, bool NS, bool BLEND>
constexpr size_t volume_smem_bytes(bool metric_per_node) {
  using S = Shape<DIM, N>;
  constexpr bool NEEDQ = (VOL == VOL_CENTRAL) || BLEND;
  constexpr size_t region = (size_t)S::EPB * (S::NPRIM * S::ND + S::PAIRS * S::NEQ);
  constexpr size_t visc = NS ? (size_t)S::EPB * DIM * (S::NEQ - 1) * S::ND : 0;
  const size_t met = (size_t)S::EPB * (metric_per_node ? S::ND * DIM * DIM : DIM * DIM);
  return sizeof(R) * (S::OPS + (region > visc ? region : visc) +
                      (NEEDQ ? (size_t)S::EPB * S::NEQ * S::ND : 0) + met);
}

template <typename R, int DIM, int N, int VOL, bool NS, bool BLEND>
cudaError_t launch_volume(const VolArgs<R> &a, cudaStream_t s, int prepare) {
  using S = Shape<DIM, N>;
  static_assert(S::PAIRS >= S::ND, "subcell FV rate aliases the pair-flux buffer");
  if (prepare)
    return cudaFuncSetAttribute(volume_kernel<R, DIM, N, VOL, NS, BLEND>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)volume_smem_bytes<R, DIM, N, VOL, NS, BLEND>(true));
  if (a.ne <= 0) return cudaSuccess;
  const size_t smem = volume_smem_bytes<R, DIM, N, VOL, NS, BLEND>(a.met_ns != 0);
  const int grid = (a.ne + S::EPB - 1) / S::EPB;
  volume_kernel<R, DIM, N, VOL, NS, BLEND><<<grid, S::THREADS, smem, s>>>(a);
  return cudaGetLastError();
}

template <typename R, int DIM, int SURF, bool NS>
cudaError_t launch_face(const FaceArgs<R> &a, cudaStream_t s) {
  const int nfp = DIM == 2 ? a.N : a.N * a.N;
  const long long total = (long long)a.nf * nfp;
  if (total <= 0) return cudaSuccess;
  const int grid = (int)((total + 127) / 128);
  face_kernel<R, DIM, SURF, NS><<<grid, 128, 0, s>>>(a);
  return cudaGetLastError();
}

template <typename R, int DIM, int N>
cudaError_t launch_grad(const GradArgs<R> &a, cudaStream_t s, int prepare) {
  using S = Shape<DIM, N>;
  constexpr size_t smem = sizeof(R) * (S::DPAD + (size_t)S::EPB * S::NEQ * S::ND);
  if (prepare)
    return cudaFuncSetAttribute(grad_kernel<R, DIM, N>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)smem);
  if (a.ne <= 0) return cudaSuccess;
  const int grid = (a.ne + S::EPB - 1) / S::EPB;
  grad_kernel<R, DIM, N><<<grid, S::THREADS, smem, s>>>(a);
  return cudaGetLastError();
}

template <typename R, int DIM, int N>
cudaError_t launch_blend(const BlendArgs<R> &a, cudaStream_t s) {
  using S = Shape<DIM, N>;
  if (a.ne <= 0) return cudaSuccess;
  const int grid = (a.ne + S::EPB - 1) / S::EPB;
  blend_kernel<R, DIM, N><<<grid, S::THREADS, 0, s>>>(a);
  return cudaGetLastError();
}

struct OrderKernels0 { VolLaunch<double> vol[4][2][2]; GradLaunch<double> grad; BlendLaunch<double> blend; };
struct OrderKernels1 { VolLaunch<float> vol[4][2][2]; GradLaunch<float> grad; BlendLaunch<float> blend; };
struct FaceKernels0 { FaceLaunch<double> face[6][2]; };
struct FaceKernels1 { FaceLaunch<float> face[6][2]; };

#define THX_DECLARE_ORDER(P, D, N) OrderKernels##P order_kernels_##P##_##D##_##N();
#define THX_DECLARE_FACE(P, D) FaceKernels##P face_kernels_##P##_##D();
#define THX_FOR_ORDERS(X, P, D) X(P, D, 3) X(P, D, 4) X(P, D, 5) X(P, D, 6)
THX_FOR_ORDERS(THX_DECLARE_ORDER, 0, 2)
THX_FOR_ORDERS(THX_DECLARE_ORDER, 0, 3)
THX_FOR_ORDERS(THX_DECLARE_ORDER, 1, 2)
THX_FOR_ORDERS(THX_DECLARE_ORDER, 1, 3)
THX_DECLARE_FACE(0, 2)
THX_DECLARE_FACE(0, 3)
THX_DECLARE_FACE(1, 2)
THX_DECLARE_FACE(1, 3)

}  // namespace thx
