// thx_trials.cu -- tensor-core trial of the element-local derivative
// contraction of the BR1 gradient (include/DGSEMIntegrator.hpp:764-850):
// for every element, direction d and field k, dS/dxi_d at each node is the
// LGL derivative matrix D (N x N) applied along the node's tensor line.
// Per element and direction this is a small GEMM, dr^T = S^T D^T, with
// S^T of (lines x fields) rows and N columns.
//
// Two forms of the same contraction, each one CTA per element with the
// element's fields staged in shared memory:
//   SIMT: one thread per node, the N-term sums on the FP64 (or FP32) pipe;
//   MMA:  warp-level tensor-core tiles -- FP64 mma.sync.m8n8k4 (rows of S^T
//         padded to 8, K = N padded to a multiple of 4, 8 output columns of
//         which N are used), or for FP32 mma.sync.m16n8k8 with TF32 operands
//         split into high and low parts (three products, hi*hi + hi*lo +
//         lo*hi, recover FP32 accuracy).
// Both write, per node, sum over (d, k) of c_(d,k) dS_k/dxi_d with fixed
// coefficients c = 1 + (d*NEQ + k)/8, in the same order, so the two outputs
// differ only by the rounding inside the contraction.  The trial exists to
// measure which pipe wins at these sizes; the product kernels use the SIMT
// form.
#include "theseus_b200.h"
#include "thx_kernels.cuh"

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

namespace {

using thx::Shape;

template <int DIM, int N>
struct Tr {
  static constexpr int ND = DIM == 2 ? N * N : N * N * N;
  static constexpr int NEQ = DIM + 2;
  static constexpr int NLINE = ND / N;
  static constexpr int ROWS = NLINE * NEQ;  // rows of S^T per direction
  static constexpr int THREADS = ((ND + 31) / 32) * 32 < 128 ? 128 : ((ND + 31) / 32) * 32;
};

template <int DIM, int N>
__device__ __forceinline__ int tr_line_node(int dir, int line, int pos) {
  return thx::line_node<DIM, N>(dir, line, pos);
}

template <typename R, int DIM, int N>
__device__ __forceinline__ R weighted_sum(const R *sDr, int n) {
  // sDr[(d*NEQ + k)*ND + n]
  using T = Tr<DIM, N>;
  R s = R(0);
#pragma unroll
  for (int d = 0; d < DIM; ++d)
#pragma unroll
    for (int k = 0; k < T::NEQ; ++k) s += (R(1) + R(d * T::NEQ + k) / R(8)) * sDr[(d * T::NEQ + k) * T::ND + n];
  return s;
}

template <typename R, int DIM, int N>
__global__ void __launch_bounds__(Tr<DIM, N>::THREADS) contraction_simt(const R *__restrict__ S, long long L,
                                                                     const R *__restrict__ D, int ne,
                                                                     R *__restrict__ out) {
  using T = Tr<DIM, N>;
  __shared__ R sD[N * N];
  __shared__ R sS[T::NEQ * T::ND];
  const int e = blockIdx.x, tid = threadIdx.x;
  if (e >= ne) return;
  for (int i = tid; i < N * N; i += blockDim.x) sD[i] = D[i];
  for (int i = tid; i < T::NEQ * T::ND; i += blockDim.x)
    sS[i] = S[(long long)(i / T::ND) * L + (long long)e * T::ND + i % T::ND];
  __syncthreads();
  if (tid >= T::ND) return;
  int c[3];
  thx::node_coords<DIM, N>(tid, c);
  R s = R(0);
#pragma unroll
  for (int d = 0; d < DIM; ++d) {
    const int me = c[d], line = thx::line_of<DIM, N>(d, c);
#pragma unroll
    for (int k = 0; k < T::NEQ; ++k) {
      R dr = R(0);
#pragma unroll
      for (int l = 0; l < N; ++l) dr += sD[me * N + l] * sS[k * T::ND + tr_line_node<DIM, N>(d, line, l)];
      s += (R(1) + R(d * T::NEQ + k) / R(8)) * dr;
    }
  }
  out[(long long)e * T::ND + tid] = s;
}

// FP64: mma.sync.aligned.m8n8k4.row.col.f64 -- A 8x4 (row = lane/4, col =
// lane%4), B 4x8 (row = lane%4, col = lane/4), C 8x8 (row = lane/4,
// cols 2*(lane%4) + {0,1}).  A = S^T tile (rows: (line, field) pairs),
// B = D^T (rows: l, cols: output position i).
__device__ __forceinline__ void dmma_8x8x4(double &c0, double &c1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
               : "+d"(c0), "+d"(c1)
               : "d"(a), "d"(b));
}

template <int DIM, int N>
__global__ void __launch_bounds__(Tr<DIM, N>::THREADS) contraction_dmma(const double *__restrict__ S, long long L,
                                                                     const double *__restrict__ D, int ne,
                                                                     double *__restrict__ out) {
  using T = Tr<DIM, N>;
  constexpr int KS = (N + 3) / 4;                 // k-steps of 4
  constexpr int TILES = (T::ROWS + 7) / 8;        // 8-row tiles of S^T per direction
  __shared__ double sD[N * N];
  __shared__ double sS[T::NEQ * T::ND];
  __shared__ double sDr[DIM * T::NEQ * T::ND];
  const int e = blockIdx.x, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int nwarps = blockDim.x >> 5;
  if (e >= ne) return;
  for (int i = tid; i < N * N; i += blockDim.x) sD[i] = D[i];
  for (int i = tid; i < T::NEQ * T::ND; i += blockDim.x)
    sS[i] = S[(long long)(i / T::ND) * L + (long long)e * T::ND + i % T::ND];
  __syncthreads();
  const int g = lane >> 2, t4 = lane & 3;
  for (int job = warp; job < DIM * TILES; job += nwarps) {
    const int d = job / TILES, tile = job % TILES;
    const int row = tile * 8 + g;               // this lane's A row: (line, field)
    const int line = row / T::NEQ, k = row % T::NEQ;
    double c0 = 0.0, c1 = 0.0;
#pragma unroll
    for (int ks = 0; ks < KS; ++ks) {
      const int l = ks * 4 + t4;
      const double a = (row < T::ROWS && l < N) ? sS[k * T::ND + tr_line_node<DIM, N>(d, line, l)] : 0.0;
      const int i = g;                          // B column: output position
      const double b = (l < N && i < N) ? sD[i * N + l] : 0.0;
      dmma_8x8x4(c0, c1, a, b);
    }
    // C row g is (line, field) of row tile*8 + g; columns 2*t4, 2*t4 + 1 are positions
    const int crow = tile * 8 + g;
    if (crow < T::ROWS) {
      const int cl = crow / T::NEQ, ck = crow % T::NEQ;
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        const int i = 2 * t4 + j;
        if (i < N) sDr[(d * T::NEQ + ck) * T::ND + tr_line_node<DIM, N>(d, cl, i)] = j ? c1 : c0;
      }
    }
  }
  __syncthreads();
  if (tid < T::ND) out[(long long)e * T::ND + tid] = weighted_sum<double, DIM, N>(sDr, tid);
}

// FP32: mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 -- A 16x8 (a0:(g,t)
// a1:(g+8,t) a2:(g,t+4) a3:(g+8,t+4)), B 8x8 (b0:(t,g) b1:(t+4,g)), C 16x8
// (c0:(g,2t) c1:(g,2t+1) c2:(g+8,2t) c3:(g+8,2t+1)); g = lane/4, t = lane%4.
__device__ __forceinline__ uint32_t to_tf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}
__device__ __forceinline__ void mma_tf32(float *c, const uint32_t *a, const uint32_t *b) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

template <int DIM, int N, int PASSES>
__global__ void __launch_bounds__(Tr<DIM, N>::THREADS) contraction_tf32(const float *__restrict__ S, long long L,
                                                                     const float *__restrict__ D, int ne,
                                                                     float *__restrict__ out) {
  using T = Tr<DIM, N>;
  static_assert(N <= 8, "K padded to 8");
  constexpr int TILES = (T::ROWS + 15) / 16;
  __shared__ float sD[N * N];
  __shared__ float sS[T::NEQ * T::ND];
  __shared__ float sDr[DIM * T::NEQ * T::ND];
  const int e = blockIdx.x, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int nwarps = blockDim.x >> 5;
  if (e >= ne) return;
  for (int i = tid; i < N * N; i += blockDim.x) sD[i] = D[i];
  for (int i = tid; i < T::NEQ * T::ND; i += blockDim.x)
    sS[i] = S[(long long)(i / T::ND) * L + (long long)e * T::ND + i % T::ND];
  __syncthreads();
  const int g = lane >> 2, t4 = lane & 3;
  for (int job = warp; job < DIM * TILES; job += nwarps) {
    const int d = job / TILES, tile = job % TILES;
    float av[4], bv[2];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int row = tile * 16 + g + ((q & 1) ? 8 : 0);
      const int l = t4 + ((q & 2) ? 4 : 0);
      const int line = row / T::NEQ, k = row % T::NEQ;
      av[q] = (row < T::ROWS && l < N) ? sS[k * T::ND + tr_line_node<DIM, N>(d, line, l)] : 0.f;
    }
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      const int l = t4 + (q ? 4 : 0), i = g;
      bv[q] = (l < N && i < N) ? sD[i * N + l] : 0.f;
    }
    uint32_t ahi[4], alo[4], bhi[2], blo[2];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      ahi[q] = to_tf32(av[q]);
      alo[q] = to_tf32(av[q] - __uint_as_float(ahi[q]));
    }
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      bhi[q] = to_tf32(bv[q]);
      blo[q] = to_tf32(bv[q] - __uint_as_float(bhi[q]));
    }
    float c[4] = {0.f, 0.f, 0.f, 0.f};
    if (PASSES == 3) {
      mma_tf32(c, alo, bhi);
      mma_tf32(c, ahi, blo);
    }
    mma_tf32(c, ahi, bhi);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int crow = tile * 16 + g + ((q & 2) ? 8 : 0);
      const int i = 2 * t4 + (q & 1);
      if (crow < T::ROWS && i < N) {
        const int cl = crow / T::NEQ, ck = crow % T::NEQ;
        sDr[(d * T::NEQ + ck) * T::ND + tr_line_node<DIM, N>(d, cl, i)] = c[q];
      }
    }
  }
  __syncthreads();
  if (tid < T::ND) out[(long long)e * T::ND + tid] = weighted_sum<float, DIM, N>(sDr, tid);
}

template <typename F>
int time_launches(F launch, int reps, cudaStream_t s, double *ms_out) {
  cudaEvent_t a, b;
  if (cudaEventCreate(&a) != cudaSuccess) return THX_ERR_CUDA;
  if (cudaEventCreate(&b) != cudaSuccess) { cudaEventDestroy(a); return THX_ERR_CUDA; }
  launch();  // warm-up
  cudaEventRecord(a, s);
  for (int r = 0; r < reps; ++r) launch();
  cudaEventRecord(b, s);
  int st = THX_OK;
  if (cudaGetLastError() != cudaSuccess || cudaEventSynchronize(b) != cudaSuccess) st = THX_ERR_CUDA;
  float ms = 0.f;
  if (st == THX_OK && cudaEventElapsedTime(&ms, a, b) != cudaSuccess) st = THX_ERR_CUDA;
  *ms_out = ms / reps;
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  return st;
}

}  // namespace

extern "C" int thx_trial_contraction(int dim, int order, int num_elements, int precision, int form,
                                     const void *fields, const double *D_host, void *out, int reps,
                                     double *ms, void *stream) {
  if (!fields || !D_host || !out || !ms || num_elements <= 0 || reps <= 0) return THX_ERR_INVALID_ARGUMENT;
  if (dim != 3 || order != 4) return THX_ERR_UNSUPPORTED;
  constexpr int DIM = 3, N = 5;
  using T = Tr<DIM, N>;
  cudaStream_t s = (cudaStream_t)stream;
  const long long L = (long long)num_elements * T::ND;
  const int ne = num_elements;
  if (precision == THX_PRECISION_FP64) {
    double *dD = nullptr;
    if (cudaMalloc(&dD, sizeof(double) * N * N) != cudaSuccess) { cudaGetLastError(); return THX_ERR_OUT_OF_MEMORY; }
    cudaMemcpy(dD, D_host, sizeof(double) * N * N, cudaMemcpyHostToDevice);
    const double *S = (const double *)fields;
    double *o = (double *)out;
    int st;
    if (form == 0)
      st = time_launches([&] { contraction_simt<double, DIM, N><<<ne, T::THREADS, 0, s>>>(S, L, dD, ne, o); }, reps, s, ms);
    else if (form == 1)
      st = time_launches([&] { contraction_dmma<DIM, N><<<ne, T::THREADS, 0, s>>>(S, L, dD, ne, o); }, reps, s, ms);
    else
      st = THX_ERR_INVALID_ARGUMENT;
    cudaFree(dD);
    return st;
  }
  if (precision == THX_PRECISION_FP32_MIXED) {
    float Df[N * N];
    for (int i = 0; i < N * N; ++i) Df[i] = (float)D_host[i];
    float *dD = nullptr;
    if (cudaMalloc(&dD, sizeof(float) * N * N) != cudaSuccess) { cudaGetLastError(); return THX_ERR_OUT_OF_MEMORY; }
    cudaMemcpy(dD, Df, sizeof(float) * N * N, cudaMemcpyHostToDevice);
    const float *S = (const float *)fields;
    float *o = (float *)out;
    int st;
    if (form == 0)
      st = time_launches([&] { contraction_simt<float, DIM, N><<<ne, T::THREADS, 0, s>>>(S, L, dD, ne, o); }, reps, s, ms);
    else if (form == 1)
      st = time_launches([&] { contraction_tf32<DIM, N, 1><<<ne, T::THREADS, 0, s>>>(S, L, dD, ne, o); }, reps, s, ms);
    else if (form == 2)
      st = time_launches([&] { contraction_tf32<DIM, N, 3><<<ne, T::THREADS, 0, s>>>(S, L, dD, ne, o); }, reps, s, ms);
    else
      st = THX_ERR_INVALID_ARGUMENT;
    cudaFree(dD);
    return st;
  }
  return THX_ERR_INVALID_ARGUMENT;
}
