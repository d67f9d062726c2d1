// thx_kernels.cuh -- CUDA kernels of the DGSEM right-hand side on sm_100a.
//
// Layouts (all in HBM, R = double or float):
//   state / rate     u[eq][elem][node]      (MFEM byNODES L-vector, node lexicographic)
//   viscous flux     fv[d][eq-1][elem][node] (physical viscous flux, NS only;
//                    its mass row is identically zero and is not stored)
//   face fluxes      fs[face][eq][fp]       (unweighted F*, inviscid minus viscous)
//   geometry         jac[e*jac_es + n*jac_ns], metric block of DIM*DIM per node
//                    at met[e*met_es + n*met_ns]; strides are 0 where the host
//                    found the factor constant (exactly) over nodes/elements.
//
// Kernel structure per right-hand side:
//   NS only : grad_kernel   element-local BR1 gradient of entropy variables with
//             the interior-face lift, converted to primitive gradients and on to
//             the physical viscous flux, which is what the other kernels read.
//   always  : face_kernel   one thread per face point: F*(u-,u+,n) (- n.avg(F_v)).
//   always  : volume_kernel one CTA per EPB elements: flux differencing with every
//             symmetric pair evaluated once, optional subcell-FV blend, viscous
//             divergence, surface lift from fs; writes dudt once.
#pragma once
#include "thx_device.cuh"
#include "thx_bc.cuh"

namespace thx {

template <int DIM, int N, int EPBX = 0>
struct Shape {
  static constexpr int ND = DIM == 2 ? N * N : N * N * N;
  static constexpr int NFP = DIM == 2 ? N : N * N;
  static constexpr int NEQ = DIM + 2;
  // elements per CTA: as many as fit 256 threads, or EPBX when given (the
  // batched kernels' half-size variant)
  static constexpr int EPB = EPBX > 0 ? EPBX : (256 / ND) > 0 ? 256 / ND : 1;
  static constexpr int THREADS = ((EPB * ND + 31) / 32) * 32;
  static constexpr int NP = N * (N - 1) / 2;  // pairs per line
  static constexpr int NLINE = ND / N;
  static constexpr int PAIRS = NLINE * NP;     // pairs per element and direction
  static constexpr int OPS = ((2 * N * N + N + 7) / 8) * 8;  // Dhat2 | Dhat | w, padded
  static constexpr int DPAD = ((N * N + 7) / 8) * 8;
};

// Node index of position `pos` on tensor line `line` along direction dir.
template <int DIM, int N>
__device__ __forceinline__ int line_node(int dir, int line, int pos) {
  if (DIM == 2) return dir == 0 ? pos + N * line : line + N * pos;
  if (dir == 0) return pos + N * line;
  if (dir == 1) return (line % N) + N * (pos + N * (line / N));
  return line + N * N * pos;
}
template <int DIM, int N>
__device__ __forceinline__ void node_coords(int n, int *c) {
  c[0] = n % N;
  c[1] = (n / N) % N;
  c[2] = DIM == 3 ? n / (N * N) : 0;
}
template <int DIM, int N>
__device__ __forceinline__ int line_of(int dir, const int *c) {
  if (DIM == 2) return dir == 0 ? c[1] : c[0];
  if (dir == 0) return c[1] + N * c[2];
  if (dir == 1) return c[0] + N * c[2];
  return c[0] + N * c[1];
}
// Face point of a node on a face normal to `dir` (same order as trace_node).
template <int DIM, int N>
__device__ __forceinline__ int face_point(int dir, const int *c) {
  if (DIM == 2) return dir == 0 ? c[1] : c[0];
  if (dir == 0) return c[1] + N * c[2];
  if (dir == 1) return c[0] + N * c[2];
  return c[0] + N * c[1];
}
template <int N>
__device__ __forceinline__ int pair_index(int lo, int hi) {
  return lo * (N - 1) - (lo * (lo - 1)) / 2 + (hi - lo - 1);
}
template <int N>
__device__ __forceinline__ void pair_decode(int k, int &a, int &b) {
  a = 0;
#pragma unroll
  for (int s = 0; s < N - 1; ++s) {
    if (k >= N - 1 - a) { k -= N - 1 - a; ++a; }
  }
  b = a + 1 + k;
}

// Status bits written by kernels (read by thx_read_status).  STATUS_LAUNCH:
// a kernel was given less dynamic shared memory than its layout needs and
// returned without doing any work.
// STATUS_EOS: an LTE temperature recovery failed or left the table.
enum : unsigned { STATUS_NONPOSITIVE = 1u, STATUS_NONFINITE = 2u, STATUS_LAUNCH = 4u,
                  STATUS_EOS = 8u };

// Density and pressure of an FP64 conserved state both positive (NaN fails).
template <int DIM>
__device__ __forceinline__ bool fp64_state_positive(const double *q, double gm1) {
  double m2 = 0.0;
#pragma unroll
  for (int d = 0; d < DIM; ++d) m2 += q[1 + d] * q[1 + d];
  const double p = gm1 * (q[DIM + 1] - 0.5 * m2 / q[0]);
  return q[0] > 0.0 && p > 0.0;
}

__device__ __forceinline__ unsigned dynamic_smem_bytes() {
  unsigned v;
  asm volatile("mov.u32 %0, %%dynamic_smem_size;" : "=r"(v));
  return v;
}

// Shared-memory layout of the volume kernel, in elements of R:
// [ops | prim + pair fluxes, or the viscous flux | state (NEEDQ) | metric].
template <typename R, int DIM, int N, int VOL, bool NS, bool BLEND, int EPBX = 0>
struct VolSmem {
  using S = Shape<DIM, N, EPBX>;
  static constexpr bool NEEDQ = VOL == VOL_CENTRAL;
  static constexpr int PRIM = VOL == VOL_LTEEC ? S::NEQ + LTE_P_COUNT : nprim<R, DIM>();
  static constexpr int REGION = S::EPB * (PRIM * S::ND + S::PAIRS * S::NEQ);
  static constexpr int VISC = NS ? S::EPB * DIM * (S::NEQ - 1) * S::ND : 0;
  static constexpr int SHARED = REGION > VISC ? REGION : VISC;
  static constexpr int STATE = NEEDQ ? S::EPB * S::NEQ * S::ND : 0;
  // pair table: (lower node | upper node << 16) of every pair, per direction
  static constexpr int PTAB = (DIM * S::PAIRS * 4 + (int)sizeof(R) - 1) / (int)sizeof(R);
  __host__ __device__ static constexpr size_t bytes(bool metric_per_node) {
    return sizeof(R) * ((size_t)S::OPS + SHARED + STATE + PTAB +
                        (size_t)S::EPB * (metric_per_node ? S::ND * DIM * DIM : DIM * DIM));
  }
};

template <typename R>
struct VolArgs {
  const R *u;
  R *du;
  double *du64;  // stage 0: write the rate widened to FP64 here instead of du
  int ne;
  const R *jac;
  long long jac_es, jac_ns;
  const R *met;
  long long met_es, met_ns;
  const int *elem_face;   // [e][2*DIM] = 2*face + side
  const R *fstar;         // [f][eq][fp]
  const R *wm, *wp;       // lift weights
  long long w_fs, w_ps;
  int nf_int;             // faces at or past nf_int are boundary faces
  const R *bw;            // boundary lift weights [b][fp], face slot nf_int + b
  const R *vflux;         // NS physical viscous flux [dir][eq-1][elem][node]
  const double *alpha;    // per-element blending coefficient or nullptr
  const R *sub[3];        // subcell metrics (reference layout), element stride sub_es
  long long sub_es[3];
  int fv_flux;            // SurfKind for the subcell FV fluxes
  R *fvrate;              // subcell FV rate [elem][eq][node] of blended elements (fv_kernel)
  GasT<R> gas;
  const R *ops;           // [Dhat2 N*N | Dhat N*N | w N]
  // fused SSP-RK3 stage (stage==0: plain dudt)
  int stage;
  double dt;
  const double *dt_dev;   // when set, the stage's dt is read here (device-side CFL step)
  double *um;             // FP64 master state (read every stage, written by stage 3)
  double *y;              // FP64 stage state (written by stages 1 and 2)
  float *yf;              // FP32 working copy of the next RHS input (mixed mode) or nullptr
  double off[5];          // yf = (float)(y - off[eq])
  unsigned *status;
  // FP32-mixed with FP64 islands: blocks (of EPB elements) flagged here are
  // evaluated by the FP64 kernels instead; this kernel skips them
  const int *skip_block;
};

// Surface flux with a run-time selector (used on subcell faces).  Inlined:
// a call would pass the states and the gas record through local memory.
template <typename R, int DIM>
__device__ __forceinline__ void surface_flux_rt(int kind, const GasT<R> &g, const FState<R, DIM> &A,
                                             const FState<R, DIM> &B, const R *n, R *F) {
  switch (kind) {
    case SURF_CHANDRASHEKAR: surface_flux<R, DIM, SURF_CHANDRASHEKAR>(g, A, B, n, F); break;
    case SURF_RANOCHA: surface_flux<R, DIM, SURF_RANOCHA>(g, A, B, n, F); break;
    case SURF_PIROZZOLI: surface_flux<R, DIM, SURF_PIROZZOLI>(g, A, B, n, F); break;
    case SURF_HLL: surface_flux<R, DIM, SURF_HLL>(g, A, B, n, F); break;
    case SURF_ROE: surface_flux<R, DIM, SURF_ROE>(g, A, B, n, F); break;
    default: surface_flux<R, DIM, SURF_LLF>(g, A, B, n, F); break;
  }
}

// One CTA's work of the volume kernel: elements [block*EPB, block*EPB + EPB).
// Shared by the one-case kernel (block = blockIdx.x) and the batched
// persistent kernel (block from its work list).
// Stride (in R) between the NEQ arrays of a block's state staged in shared
// memory: EPB*ND rounded up to 16 bytes, so every array starts 16-byte aligned.
template <typename R, int DIM, int N, int EPBX = 0>
__host__ __device__ constexpr int stage_kstride() {
  using S = Shape<DIM, N, EPBX>;
  return (int)(((size_t)S::EPB * S::ND * sizeof(R) + 15) / 16 * 16 / sizeof(R));
}

// su: the block's state staged in shared memory (array k at k*stage_kstride,
// element el's node n at el*ND + n), or nullptr to read it from a.u.
template <typename R, int DIM, int N, int VOL, bool NS, bool BLEND, int EPBX = 0>
__device__ __forceinline__ void volume_body(const VolArgs<R> &a, const int block,
                                            const R *su = nullptr) {
  using S = Shape<DIM, N, EPBX>;
  static_assert(VOL != VOL_LTEEC || (!BLEND && !IsF32<R>::value), "LTEEC: FP64, no blending");
  using L_ = VolSmem<R, DIM, N, VOL, NS, BLEND, EPBX>;
  constexpr int ND = S::ND, NEQ = S::NEQ, EPB = S::EPB, NPRIM = L_::PRIM, PAIRS = S::PAIRS;
  constexpr int MB = DIM * DIM;
  constexpr bool NEEDQ = L_::NEEDQ;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  if (a.skip_block && a.skip_block[block]) return;  // block-uniform: before any barrier
  if (dynamic_smem_bytes() < L_::bytes(a.met_ns != 0)) {
    if (threadIdx.x == 0) atomicOr(a.status, STATUS_LAUNCH);
    return;
  }
  // [ops | prim | pair fluxes | state (NEEDQ) | metric]; the viscous flux of the
  // NS phase reuses the prim + pair-flux region, the FV rate the pair fluxes.
  R *sOps = reinterpret_cast<R *>(smem_raw);              // 2*N*N + N (padded)
  R *sPrim = sOps + S::OPS;                               // [EPB][NPRIM][ND]
  R *sFB = sPrim + EPB * NPRIM * ND;                      // [EPB][PAIRS][NEQ]
  R *sQ = sPrim + L_::SHARED;                             // [EPB][NEQ][ND] if NEEDQ
  unsigned *sPT = reinterpret_cast<unsigned *>(sQ + L_::STATE);  // [DIM][PAIRS]
  R *sMet = sQ + L_::STATE + L_::PTAB;                    // per node or once per element
  R *sFv = sPrim;                                         // [EPB][DIM][NEQ-1][ND] (NS)
  const int mns = a.met_ns != 0 ? MB : 0;                 // metric node stride in smem
  const int mbk = a.met_ns != 0 ? ND * MB : MB;           // metric element block in smem

  const int tid = threadIdx.x;
  const int e0 = block * EPB;
  const long long L = (long long)a.ne * ND;
  for (int i = tid; i < 2 * N * N + N; i += blockDim.x) sOps[i] = a.ops[i];
  for (int i = tid; i < DIM * PAIRS; i += blockDim.x) {
    const int dir = i / PAIRS, pidx = i % PAIRS;
    int pa, pb;
    pair_decode<N>(pidx % S::NP, pa, pb);
    const int line = pidx / S::NP;
    sPT[i] = (unsigned)line_node<DIM, N>(dir, line, pa) | ((unsigned)line_node<DIM, N>(dir, line, pb) << 16);
  }
  const R *sD2 = sOps;
  const R *sDh = sOps + N * N;
  const R *sW = sOps + 2 * N * N;

  // stage states, node data and metric
  const int el = tid / ND, n = tid % ND;
  const int e = e0 + el;
  const bool active = (el < EPB) && (e < a.ne);
  if (active) {
    R q[NEQ];
    if (su) {
#pragma unroll
      for (int k = 0; k < NEQ; ++k) q[k] = su[k * stage_kstride<R, DIM, N, EPBX>() + el * ND + n];
    } else {
#pragma unroll
      for (int k = 0; k < NEQ; ++k) q[k] = a.u[k * L + (long long)e * ND + n];
    }
    if constexpr (VOL == VOL_LTEEC) {
      // conserved state, recovered T, its table cell and the pressure
      const double T = a.gas.Tn[(long long)e * ND + n];
      const LteEval sv = lte_at_cell(a.gas.lte, q[0], T, a.gas.Cn[(long long)e * ND + n]);
      R pr[NPRIM];
#pragma unroll
      for (int k = 0; k < NEQ; ++k) pr[k] = q[k];
      pr[NEQ + LTE_P_T] = T;
      pr[NEQ + LTE_P_XI] = sv.xi;
      pr[NEQ + LTE_P_ETA] = sv.eta;
      pr[NEQ + LTE_P_DR] = sv.cell.dr;
      pr[NEQ + LTE_P_DT] = sv.cell.dt;
      pr[NEQ + LTE_P_OFF] = (double)sv.cell.off;
      const LteJet jv = lte_jet(a.gas.lte, sv);
      pr[NEQ + LTE_P_H] = jv.H;
      pr[NEQ + LTE_P_HR] = jv.Hr;
      pr[NEQ + LTE_P_HT] = jv.HT;
      pr[NEQ + LTE_P_HRR] = jv.Hrr;
      pr[NEQ + LTE_P_HRT] = jv.HrT;
#pragma unroll
      for (int k = 0; k < NPRIM; ++k) sPrim[(el * NPRIM + k) * ND + n] = pr[k];
      if (!sv.valid || !(q[0] > 0.0)) atomicOr(a.status, STATUS_EOS);
    } else {
      R pr[NPRIM];
      node_prims<R, DIM, VOL>(a.gas, q, pr);
#pragma unroll
      for (int k = 0; k < NPRIM; ++k) sPrim[(el * NPRIM + k) * ND + n] = pr[k];
      if (NEEDQ) {
#pragma unroll
        for (int k = 0; k < NEQ; ++k) sQ[(el * NEQ + k) * ND + n] = q[k];
      }
      // FP64 path: positivity of the state read here.  FP32-mixed: checked
      // on the FP64 master state instead (to_working, the RK stage epilogue)
      if (!IsF32<R>::value && (!(pr[0] > R(0)) || !(pr[DIM + 1] > R(0))))
        atomicOr(a.status, STATUS_NONPOSITIVE);
    }
    if (mns != 0 || n == 0) {
      const R *mp = a.met + (long long)e * a.met_es + (long long)n * a.met_ns;
#pragma unroll
      for (int k = 0; k < MB; ++k) sMet[el * mbk + n * mns + k] = mp[k];
    }
  }
  __syncthreads();

  int c[3];
  node_coords<DIM, N>(n, c);
  R rate[NEQ];
#pragma unroll
  for (int k = 0; k < NEQ; ++k) rate[k] = R(0);

  // directions unrolled: 2 % faster than rolled (32^3 p=4, FP64 and FP32);
  // rolled for the LTEEC flux, whose spills it would multiply
  constexpr int DIR_UNROLL = VOL == VOL_LTEEC ? 1 : DIM;
#pragma unroll DIR_UNROLL
  for (int dir = 0; dir < DIM; ++dir) {
    // pair phase: every symmetric pair once, in (lower, upper) order
    for (int t = tid; t < EPB * PAIRS; t += S::THREADS) {  // launched with S::THREADS
      const int pel = t / PAIRS, pidx = t % PAIRS;
      if (e0 + pel >= a.ne) continue;
      const unsigned nn = sPT[dir * PAIRS + pidx];
      const int na = (int)(nn & 0xffffu), nb = (int)(nn >> 16);
      R A[NPRIM], B[NPRIM], met[DIM], F[NEQ];
#pragma unroll
      for (int k = 0; k < NPRIM; ++k) {
        A[k] = sPrim[(pel * NPRIM + k) * ND + na];
        B[k] = sPrim[(pel * NPRIM + k) * ND + nb];
      }
      if (mns == 0) {
        // one metric per element: 0.5*(m+m) == m
#pragma unroll
        for (int d = 0; d < DIM; ++d) met[d] = sMet[pel * mbk + dir * DIM + d];
      } else {
#pragma unroll
        for (int d = 0; d < DIM; ++d)
          met[d] = R(0.5) * (sMet[pel * mbk + na * mns + dir * DIM + d] + sMet[pel * mbk + nb * mns + dir * DIM + d]);
      }
      if constexpr (VOL == VOL_LTEEC) {
        // include/LTEECFlux.hpp:11-84: the averaged metric passed as both rows
        // (0.5*(m+m) == m exactly)
        const LteEval sa = lte_unpack(A + NEQ, A[0], a.gas.lte.nx);
        const LteEval sb = lte_unpack(B + NEQ, B[0], a.gas.lte.nx);
        lte_ec_flux<DIM, false>(a.gas.lte, A, B, sa, sb, lte_unpack_jet(A + NEQ),
                                lte_unpack_jet(B + NEQ), met, met, F);
      } else if (VOL == VOL_CHANDRASHEKAR) vol_chandrashekar<R, DIM>(a.gas, A, B, met, F);
      else if (VOL == VOL_RANOCHA) vol_ranocha<R, DIM>(a.gas, A, B, met, F);
      else if (VOL == VOL_PIROZZOLI) vol_pirozzoli<R, DIM>(a.gas, A, B, met, F);
      else {
        R RA[NEQ], RB[NEQ], QA[NEQ], QB[NEQ];
#pragma unroll
        for (int k = 0; k < NEQ; ++k) {
          RA[k] = sQ[(pel * NEQ + k) * ND + na];
          RB[k] = sQ[(pel * NEQ + k) * ND + nb];
        }
        reconstruct<R, DIM>(a.gas, RA, QA);
        reconstruct<R, DIM>(a.gas, RB, QB);
        vol_central<R, DIM>(QA, QB, A, B, met, F);
      }
#pragma unroll
      for (int k = 0; k < NEQ; ++k) sFB[(pel * PAIRS + pidx) * NEQ + k] = F[k];
    }
    __syncthreads();
    // node phase: rate_i += sum_m Dhat2(i,m) F(i,m) in m order
    if (active) {
      const int me = c[dir];
      const int line = line_of<DIM, N>(dir, c);
#pragma unroll
      for (int m = 0; m < N; ++m) {
        if (m == me) continue;
        const int lo = m < me ? m : me, hi = m < me ? me : m;
        const int pidx = line * S::NP + pair_index<N>(lo, hi);
        const R coef = sD2[me * N + m];
#pragma unroll
        for (int k = 0; k < NEQ; ++k) rate[k] += coef * sFB[(el * PAIRS + pidx) * NEQ + k];
      }
    }
    __syncthreads();
  }

  R du[NEQ];
  R J = R(1);
  if (active) {
    J = a.jac[(long long)e * a.jac_es + (long long)n * a.jac_ns];
    const R s = R(-1) / J;
#pragma unroll
    for (int k = 0; k < NEQ; ++k) du[k] = s * rate[k];
  }

  // subcell finite-volume blend (include/EulerOperator_impl.hpp:134-152):
  // fv_kernel has stored the FV rate of every blended element
  if (BLEND && a.alpha != nullptr && active) {
    const double al = a.alpha[e];
    if (al > 1e-16) {
      const R af = (R)al, ad = (R)(1.0 - al);
#pragma unroll
      for (int k = 0; k < NEQ; ++k) du[k] = ad * du[k] + af * a.fvrate[((long long)e * NEQ + k) * ND + n];
    }
  }

  if (NS) {
    // contravariant viscous flux per node (include/DGSEMIntegrator.hpp:486-524)
    // from the physical viscous flux that grad_kernel stored; the mass row of
    // the viscous flux is zero and is not stored.
    constexpr int NV = NEQ - 1;
    if (active) {
      R vf[NV * DIM];
#pragma unroll
      for (int pd = 0; pd < DIM; ++pd)
#pragma unroll
        for (int k = 0; k < NV; ++k)
          vf[k * DIM + pd] = a.vflux[((long long)pd * NV + k) * L + (long long)e * ND + n];
      const R *row = sMet + el * mbk + n * mns;
#pragma unroll
      for (int dir = 0; dir < DIM; ++dir)
#pragma unroll
        for (int k = 0; k < NV; ++k) {
          R f = R(0);
#pragma unroll
          for (int pd = 0; pd < DIM; ++pd) f += row[dir * DIM + pd] * vf[k * DIM + pd];
          sFv[((el * DIM + dir) * NV + k) * ND + n] = f;
        }
    }
    __syncthreads();
    // weak-form divergence with Dhat (include/DGSEMIntegrator.hpp:526-622)
    if (active) {
      R dv[NV];
#pragma unroll
      for (int k = 0; k < NV; ++k) dv[k] = R(0);
#pragma unroll
      for (int dir = 0; dir < DIM; ++dir) {
        const int me = c[dir];
        const int line = line_of<DIM, N>(dir, c);
#pragma unroll
        for (int l = 0; l < N; ++l) {
          const int s = line_node<DIM, N>(dir, line, l);
          const R co = sDh[me * N + l];
#pragma unroll
          for (int k = 0; k < NV; ++k) dv[k] += co * sFv[((el * DIM + dir) * NV + k) * ND + s];
        }
      }
      const R sc = R(1) / J;
#pragma unroll
      for (int k = 0; k < NV; ++k) du[1 + k] += sc * dv[k];
    }
  }

  if (!active) return;
  // surface lift: interior faces summed first, then added (restr_f
  // transpose; +=); then the boundary faces the same way (restr_b)
#pragma unroll 1
  for (int pass = 0; pass < ((!IsF32<R>::value && a.bw) ? 2 : 1); ++pass) {
    R acc[NEQ];
#pragma unroll
    for (int k = 0; k < NEQ; ++k) acc[k] = R(0);
    bool any = false;
#pragma unroll
    for (int dir = 0; dir < DIM; ++dir) {
      const int me = c[dir];
      if (me != 0 && me != N - 1) continue;
      const int lf = 2 * dir + (me == N - 1 ? 1 : 0);
      const int fs = a.elem_face[e * 2 * DIM + lf];
      if (fs < 0) continue;
      const int f = fs >> 1, side = fs & 1;
      const int fp = face_point<DIM, N>(dir, c);
      R w;
      if (!IsF32<R>::value && a.bw && f >= a.nf_int) {  // boundary face (FP64 only)
        if (pass == 0) continue;
        w = -a.bw[(long long)(f - a.nf_int) * S::NFP + fp];
      } else {
        if (pass == 1) continue;
        const long long wi = (long long)f * a.w_fs + (long long)fp * a.w_ps;
        w = side == 0 ? -a.wm[wi] : a.wp[wi];
      }
#pragma unroll
      for (int k = 0; k < NEQ; ++k) acc[k] += w * a.fstar[((long long)f * NEQ + k) * S::NFP + fp];
      any = true;
    }
    if (any) {
#pragma unroll
      for (int k = 0; k < NEQ; ++k) du[k] += acc[k];
    }
  }
  const long long base = (long long)e * ND + n;
  if (a.stage == 0) {
    if (a.du64) {
#pragma unroll
      for (int k = 0; k < NEQ; ++k) a.du64[k * L + base] = (double)du[k];
    } else {
#pragma unroll
      for (int k = 0; k < NEQ; ++k) a.du[k * L + base] = du[k];
    }
  } else {
    // fused SSP-RK3 stage in the arithmetic order of mfem::RK3SSPSolver::Step
    const double dt = a.dt_dev ? *a.dt_dev : a.dt;
    // every load before the first store: the state arrays may alias as far
    // as the compiler knows, so interleaving would serialise the round trips
    double umv[NEQ], yv[NEQ];
#pragma unroll
    for (int k = 0; k < NEQ; ++k) {
      const long long i = k * L + base;
      umv[k] = a.um[i];
      yv[k] = a.stage == 1 ? 0.0 : a.y[i];
    }
    double ynew[NEQ];
#pragma unroll
    for (int k = 0; k < NEQ; ++k) {
      const double kk = (double)du[k];
      double y;
      if (a.stage == 1) {
        y = umv[k] + dt * kk;
      } else if (a.stage == 2) {
        y = yv[k] + dt * kk;
        y = 0.75 * umv[k] + 0.25 * y;
      } else {
        y = yv[k] + dt * kk;
        y = (1.0 / 3.0) * umv[k] + (2.0 / 3.0) * y;
        // a device-side step of 0 (a finished time loop, or no valid rate)
        // leaves the state exactly as it was
        if (a.dt_dev && dt == 0.0) y = umv[k];
      }
      ynew[k] = y;
    }
#pragma unroll
    for (int k = 0; k < NEQ; ++k) {
      const long long i = k * L + base;
      if (a.stage == 3) {
        if (!(a.dt_dev && dt == 0.0)) a.um[i] = ynew[k];
      } else {
        a.y[i] = ynew[k];
      }
      if (a.yf) a.yf[i] = (float)(ynew[k] - a.off[k]);
    }
    if constexpr (IsF32<R>::value) {
      // FP32-mixed: positivity of the new FP64 stage state, in FP64
      if (!fp64_state_positive<DIM>(ynew, (double)a.gas.gm1)) atomicOr(a.status, STATUS_NONPOSITIVE);
    }
  }
}

// Subcell finite-volume rate of the blended elements (include/DGSEMIntegrator.hpp:338-483):
// along every tensor line, first-order fluxes F_j between neighbouring
// subcells j, j+1 with the run-time FV face flux; node i of the line gets
// (F_{i-1} - F_i) / (J_i w_i) (F_{-1} = F_{N-1} = 0), summed over directions
// in direction order.  All subcell faces of a block are evaluated in
// parallel, then each node forms its rate.  Blocks without a blended element
// return at once; the volume kernel blends the stored rate in.  Kept apart
// from the volume kernel, whose register count it would otherwise set.
template <typename R, int DIM, int N>
struct FvSmem {
  using S = Shape<DIM, N>;
  static constexpr int FACES = DIM * S::NLINE * (N - 1);  // subcell faces per element
  static constexpr size_t bytes() {
    return sizeof(R) * (8 + (size_t)S::EPB * S::NEQ * S::ND + (size_t)S::EPB * FACES * S::NEQ);
  }
};

template <typename R, int DIM, int N>
__device__ __forceinline__ void fv_body(const VolArgs<R> &a, const int block) {
  using S = Shape<DIM, N>;
  constexpr int ND = S::ND, NEQ = S::NEQ, EPB = S::EPB, NL = S::NLINE;
  constexpr int FACES = FvSmem<R, DIM, N>::FACES;
  const int e0 = block * EPB;
  bool any = false;
  for (int k = 0; k < EPB; ++k)
    if (e0 + k < a.ne && a.alpha[e0 + k] > 1e-16) any = true;
  if (!any) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  if (dynamic_smem_bytes() < FvSmem<R, DIM, N>::bytes()) {
    if (threadIdx.x == 0) atomicOr(a.status, STATUS_LAUNCH);
    return;
  }
  R *sW = reinterpret_cast<R *>(smem_raw);  // quadrature weights (8 slots)
  R *sQ = sW + 8;                           // [EPB][NEQ][ND] state
  R *sF = sQ + EPB * NEQ * ND;              // [EPB][DIM][NL][N-1][NEQ] subcell fluxes
  const int tid = threadIdx.x;
  const long long L = (long long)a.ne * ND;
  for (int i = tid; i < N; i += blockDim.x) sW[i] = a.ops[2 * N * N + i];
  const int el = tid / ND, n = tid % ND;
  const int e = e0 + el;
  const bool active = (el < EPB) && (e < a.ne);
  if (active) {
#pragma unroll
    for (int k = 0; k < NEQ; ++k) sQ[(el * NEQ + k) * ND + n] = a.u[k * L + (long long)e * ND + n];
  }
  __syncthreads();
  // subcell face fluxes: face j of a line lies between its nodes j and j+1,
  // with the subcell normal stored at node j+1
  for (int t = tid; t < EPB * FACES; t += blockDim.x) {
    const int fel = t / FACES;
    const int r = t - fel * FACES;
    const int dir = r / (NL * (N - 1));
    const int r2 = r - dir * (NL * (N - 1));
    const int line = r2 / (N - 1), j = r2 - line * (N - 1);
    const int fe = e0 + fel;
    if (fe >= a.ne || !(a.alpha[fe] > 1e-16)) continue;
    const int id1 = line_node<DIM, N>(dir, line, j), id2 = line_node<DIM, N>(dir, line, j + 1);
    R raw[NEQ], fn[NEQ], nrm[DIM];
    FState<R, DIM> s1, s2;
#pragma unroll
    for (int k = 0; k < NEQ; ++k) raw[k] = sQ[(fel * NEQ + k) * ND + id1];
    make_fstate<R, DIM>(a.gas, raw, s1);
#pragma unroll
    for (int k = 0; k < NEQ; ++k) raw[k] = sQ[(fel * NEQ + k) * ND + id2];
    make_fstate<R, DIM>(a.gas, raw, s2);
    const R *sub = a.sub[dir] + (long long)fe * a.sub_es[dir];
#pragma unroll
    for (int d = 0; d < DIM; ++d) nrm[d] = sub[id2 * DIM + d];
    surface_flux_rt<R, DIM>(a.fv_flux, a.gas, s1, s2, nrm, fn);
#pragma unroll
    for (int k = 0; k < NEQ; ++k) sF[((long long)fel * FACES + r) * NEQ + k] = fn[k];
  }
  __syncthreads();
  if (!active || !(a.alpha[e] > 1e-16)) return;
  int c[3];
  node_coords<DIM, N>(n, c);
  const R J = a.jac[(long long)e * a.jac_es + (long long)n * a.jac_ns];
  R rate[NEQ];
#pragma unroll
  for (int dir = 0; dir < DIM; ++dir) {
    const int i = c[dir];
    const int line = line_of<DIM, N>(dir, c);
    const R *Fl = sF + ((long long)el * FACES + (dir * NL + line) * (N - 1)) * NEQ;
    const R s = J * sW[i];
#pragma unroll
    for (int k = 0; k < NEQ; ++k) {
      const R fm = i > 0 ? Fl[(i - 1) * NEQ + k] : R(0);
      const R fp = i < N - 1 ? Fl[i * NEQ + k] : R(0);
      const R d = (fm - fp) / s;
      rate[k] = dir == 0 ? d : rate[k] + d;
    }
  }
#pragma unroll
  for (int k = 0; k < NEQ; ++k) a.fvrate[((long long)e * NEQ + k) * ND + n] = rate[k];
}

template <typename R, int DIM, int N>
__global__ void __launch_bounds__(Shape<DIM, N>::THREADS) fv_kernel(const VolArgs<R> a) {
  fv_body<R, DIM, N>(a, blockIdx.x);
}

template <typename R, int DIM, int N, int VOL, bool NS, bool BLEND>
__global__ void __launch_bounds__(Shape<DIM, N>::THREADS) volume_kernel(const VolArgs<R> a) {
  volume_body<R, DIM, N, VOL, NS, BLEND>(a, blockIdx.x);
}

// The same with MINB CTAs per SM required.  FP64 takes four (8 % faster
// than the compiler's three); the LTEEC flux takes two (left alone the
// compiler gives it the whole register file and one CTA).
template <typename R, int DIM, int N, int VOL, bool NS, bool BLEND, int MINB>
__global__ void __launch_bounds__(Shape<DIM, N>::THREADS, MINB) volume_kernel_mb(const VolArgs<R> a) {
  volume_body<R, DIM, N, VOL, NS, BLEND>(a, blockIdx.x);
}

// ---- TMA-staged volume kernel ---------------------------------------------
// Persistent CTAs walk the element blocks; while a CTA evaluates one block,
// the bulk-copy engine (cp.async.bulk, completion counted on an mbarrier)
// brings the state of its next block into the other half of a double buffer
// in shared memory, so the state loads of a block never wait on HBM.  Each
// of the NEQ state arrays of a block is one contiguous run of EPB*ND values
// (byNODES layout); a block whose runs are not 16-byte aligned, or not a
// multiple of 16 bytes long, is staged with ordinary loads instead.
// Waits are bounded: a copy that has not landed within kTmaWaitNs of the
// global timer sets STATUS_TIMEOUT and the CTA stops.
enum : unsigned { STATUS_TIMEOUT = 32u };
constexpr unsigned long long kTmaWaitNs = 1000000000ull;  // one second

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ unsigned smem_addr(const void *p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(unsigned long long *bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned long long *bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void mbar_arrive(unsigned long long *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}
// true once the phase with the given parity has completed
__device__ __forceinline__ bool mbar_try_wait(unsigned long long *bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ bool mbar_wait_bounded(unsigned long long *bar, unsigned parity) {
  if (mbar_try_wait(bar, parity)) return true;
  const unsigned long long t0 = global_ns();
  while (global_ns() - t0 < kTmaWaitNs)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, unsigned bytes,
                                         unsigned long long *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}

template <typename R, int DIM, int N, int VOL, bool NS, bool BLEND>
struct VolTmaSmem {
  using S = Shape<DIM, N>;
  static constexpr size_t base(bool metric_per_node) {
    return (VolSmem<R, DIM, N, VOL, NS, BLEND>::bytes(metric_per_node) + 15) / 16 * 16;
  }
  static constexpr size_t buf_elems = (size_t)S::NEQ * stage_kstride<R, DIM, N>();
  static constexpr size_t bytes(bool metric_per_node) {
    return base(metric_per_node) + 2 * buf_elems * sizeof(R) + 2 * sizeof(unsigned long long);
  }
};

// Thread 0: stage block `blk` into buffer `dst` (bulk copies counted on bar),
// or report that the block needs ordinary loads (returns false).
template <typename R, int DIM, int N>
__device__ __forceinline__ bool tma_stage_issue(const VolArgs<R> &a, int blk, R *dst,
                                                unsigned long long *bar) {
  using S = Shape<DIM, N>;
  constexpr int ND = S::ND, NEQ = S::NEQ, EPB = S::EPB;
  const int e0 = blk * EPB;
  const int cnt = min(EPB, a.ne - e0);
  const unsigned bytes = (unsigned)(cnt * ND * (int)sizeof(R));
  const long long L = (long long)a.ne * ND;
  bool ok = (bytes % 16u) == 0;
#pragma unroll
  for (int k = 0; k < NEQ; ++k)
    ok = ok && ((reinterpret_cast<uintptr_t>(a.u + k * L + (long long)e0 * ND) & 15u) == 0);
  if (!ok) return false;
  mbar_expect_tx(bar, bytes * NEQ);
#pragma unroll
  for (int k = 0; k < NEQ; ++k)
    bulk_g2s(dst + k * stage_kstride<R, DIM, N>(), a.u + k * L + (long long)e0 * ND, bytes, bar);
  return true;
}

template <typename R, int DIM, int N, int VOL, bool NS, bool BLEND, int MINB>
__global__ void __launch_bounds__(Shape<DIM, N>::THREADS, MINB > 0 ? MINB : 1)
volume_tma_kernel(const VolArgs<R> a) {
  using S = Shape<DIM, N>;
  using T_ = VolTmaSmem<R, DIM, N, VOL, NS, BLEND>;
  constexpr int ND = S::ND, NEQ = S::NEQ, EPB = S::EPB;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const bool mpn = a.met_ns != 0;
  if (dynamic_smem_bytes() < T_::bytes(mpn)) {
    if (threadIdx.x == 0) atomicOr(a.status, STATUS_LAUNCH);
    return;
  }
  R *buf0 = reinterpret_cast<R *>(smem_raw + T_::base(mpn));
  R *bufs[2] = {buf0, buf0 + T_::buf_elems};
  unsigned long long *bars = reinterpret_cast<unsigned long long *>(buf0 + 2 * T_::buf_elems);
  __shared__ int s_bulk[2];  // buffer staged by bulk copy (1) or to be loaded (0)
  __shared__ int s_fail;
  const int nblocks = (a.ne + EPB - 1) / EPB;
  const int tid = threadIdx.x;
  if (tid == 0) {
    mbar_init(&bars[0], 1);
    mbar_init(&bars[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    s_fail = 0;
    s_bulk[0] = s_bulk[1] = 0;
    if ((int)blockIdx.x < nblocks) s_bulk[0] = tma_stage_issue<R, DIM, N>(a, blockIdx.x, bufs[0], &bars[0]);
  }
  __syncthreads();
  unsigned phase[2] = {0u, 0u};
  bool pending[2] = {s_bulk[0] != 0, false};  // a copy into the buffer not yet waited for
  const long long L = (long long)a.ne * ND;
  int it = 0;
  for (int blk = blockIdx.x; blk < nblocks; blk += gridDim.x, ++it) {
    const int b = it & 1;
    // the other buffer was last read before the previous iteration's final
    // barrier: refill it with the next block
    const int nxt = blk + gridDim.x;
    if (tid == 0)
      s_bulk[b ^ 1] = nxt < nblocks ? tma_stage_issue<R, DIM, N>(a, nxt, bufs[b ^ 1], &bars[b ^ 1]) : 0;
    if (s_bulk[b]) {
      if (!mbar_wait_bounded(&bars[b], phase[b])) s_fail = 1;
    } else {
      // ordinary loads into the buffer
      const int e0 = blk * EPB;
      for (int i = tid; i < EPB * ND; i += blockDim.x) {
        if (e0 * ND + i >= L) continue;
#pragma unroll
        for (int k = 0; k < NEQ; ++k) bufs[b][k * stage_kstride<R, DIM, N>() + i] = a.u[k * L + (long long)e0 * ND + i];
      }
    }
    __syncthreads();
    pending[b ^ 1] = s_bulk[b ^ 1] != 0;
    if (s_fail) break;
    if (s_bulk[b]) {
      phase[b] ^= 1u;
      pending[b] = false;
    }
    volume_body<R, DIM, N, VOL, NS, BLEND>(a, blk, bufs[b]);
    __syncthreads();  // shared memory and the buffer are free for the next block
  }
  if (s_fail) {
    if (tid == 0) atomicOr(a.status, STATUS_TIMEOUT);
    // give the copies still in flight a bounded chance to land before exit
    for (int q = 0; q < 2; ++q)
      if (pending[q]) mbar_wait_bounded(&bars[q], phase[q]);
  }
}

template <typename R, int VOL, bool BLEND>
struct VolMinBlocks {
  static constexpr int value = VOL == VOL_LTEEC ? 2 : (!IsF32<R>::value ? 4 : 6);
};

// ---------------------------------------------------------------------------
template <typename R>
struct FaceArgs {
  const R *u;
  int ne, nf, N;
  const int *face_elem, *face_lface;
  const R *normal;
  long long n_fs, n_ps;
  const R *vflux;
  R *fstar;
  GasT<R> gas;
  // processing order of the faces (nullptr: face order): faces sorted by
  // their minus-side element, so that the traces the CTAs in flight gather
  // belong to a narrow window of elements and come from L2 (in face order
  // the x-, y- and z-faces each sweep all of u and of the viscous flux)
  const int *order;
};

// Face point t (face order[t / nfp], point t % nfp) of one case.
template <typename R, int DIM, int SURF, bool NS>
__device__ __forceinline__ void face_body(const FaceArgs<R> &a, const long long t) {
  constexpr int NEQ = DIM + 2;
  const int N = a.N;
  const int nfp = DIM == 2 ? N : N * N;
  const int nd = DIM == 2 ? N * N : N * N * N;
  if (t >= (long long)a.nf * nfp) return;
  const int fi = (int)(t / nfp), fp = (int)(t % nfp);
  const int f = a.order ? a.order[fi] : fi;
  const long long L = (long long)a.ne * nd;
  const int em = a.face_elem[2 * f], ep = a.face_elem[2 * f + 1];
  const long long im = (long long)em * nd + trace_node<DIM>(N, a.face_lface[2 * f], fp);
  const long long ip = (long long)ep * nd + trace_node<DIM>(N, a.face_lface[2 * f + 1], fp);
  R qm[NEQ], qp[NEQ], nrm[DIM], F[NEQ];
#pragma unroll
  for (int k = 0; k < NEQ; ++k) { qm[k] = a.u[k * L + im]; qp[k] = a.u[k * L + ip]; }
  const R *np = a.normal + ((long long)f * a.n_fs + (long long)fp * a.n_ps) * DIM;
#pragma unroll
  for (int d = 0; d < DIM; ++d) nrm[d] = np[d];
  if constexpr (SURF == SURF_LTEEC) {
    // include/LTEECFlux.hpp:86-99 with the Lax dissipation
    // (include/DissipationOperator.hpp:15-55); T recovered per node
    static_assert(!IsF32<R>::value, "LTEEC: FP64 only");
    const LteEval sm = lte_at_cell(a.gas.lte, qm[0], a.gas.Tn[im], a.gas.Cn[im]);
    const LteEval sp = lte_at_cell(a.gas.lte, qp[0], a.gas.Tn[ip], a.gas.Cn[ip]);
    lte_ec_flux<DIM, true>(a.gas.lte, qm, qp, sm, sp, lte_face_jet(a.gas.lte, sm),
                           lte_face_jet(a.gas.lte, sp), nrm, nrm, F);
  } else {
    FState<R, DIM> A, B;
    make_fstate<R, DIM>(a.gas, qm, A);
    make_fstate<R, DIM>(a.gas, qp, B);
    surface_flux<R, DIM, SURF>(a.gas, A, B, nrm, F);
  }
  if (NS) {
    // include/DGSEMIntegrator.hpp:261-316: F* -= n . avg(F_v), with the physical
    // viscous flux of both traces as stored by grad_kernel (mass row zero)
    constexpr int NV = NEQ - 1;
#pragma unroll
    for (int k = 0; k < NV; ++k)
#pragma unroll
      for (int d = 0; d < DIM; ++d) {
        const R vm = a.vflux[((long long)d * NV + k) * L + im];
        const R vp = a.vflux[((long long)d * NV + k) * L + ip];
        F[1 + k] -= nrm[d] * (R(0.5) * (vm + vp));
      }
  }
#pragma unroll
  for (int k = 0; k < NEQ; ++k) a.fstar[((long long)f * NEQ + k) * nfp + fp] = F[k];
}

// The face kernels: one thread per face point, each precision compiled for
// its own number of resident 128-thread CTAs per SM.  FP64: eight (64
// registers, some spills; 0.166 -> 0.158 ms at 32^3 p=4 NS against the
// compiler's 92 registers at five CTAs; six, ten and twelve CTAs were no
// faster or slower).  FP32: ten (48 registers; 2 % faster than the
// compiler's 62 at eight).
template <int DIM, int SURF, bool NS>
__global__ void __launch_bounds__(128, 8) face_kernel_f64(const FaceArgs<double> a) {
  face_body<double, DIM, SURF, NS>(a, (long long)blockIdx.x * blockDim.x + threadIdx.x);
}
template <int DIM, int SURF, bool NS>
__global__ void __launch_bounds__(128, 10) face_kernel_f32(const FaceArgs<float> a) {
  face_body<float, DIM, SURF, NS>(a, (long long)blockIdx.x * blockDim.x + threadIdx.x);
}

// The LTEEC face flux: the same body compiled for four resident CTAs per SM
// (128 registers).  Left to itself the compiler takes 255 registers and two
// CTAs fit; with the spills of the bounded form it is still 15 % faster (24^3
// p=4: 0.244 -> 0.208 ms; three CTAs, 168 registers: 0.215 ms).
template <int DIM, bool NS>
__global__ void __launch_bounds__(128, 4) face_kernel_lte(const FaceArgs<double> a) {
  face_body<double, DIM, SURF_LTEEC, NS>(a, (long long)blockIdx.x * blockDim.x + threadIdx.x);
}

// ---------------------------------------------------------------------------
template <typename R>
struct GradArgs {
  const R *u;
  R *vflux;   // physical viscous flux [dir][eq-1][elem][node] (mass row omitted)
  int ne;
  const R *jac;
  long long jac_es, jac_ns;
  const R *met;
  long long met_es, met_ns;
  const int *elem_face, *face_elem, *face_lface;
  const R *normal;
  long long n_fs, n_ps;
  const R *wm, *wp;
  long long w_fs, w_ps;
  const R *D;  // N*N
  GasT<R> gas;
  const R *svars;  // entropy variables of every node [eq][elem][node] (SV kernels)
  unsigned *status;
  // boundary faces (FP64 ideal gas; bw == nullptr: none): face slots
  // nf_int + b, lift weights bw[b][fp], outward normals bnrm[b][fp][dim],
  // conditions; the primitive gradients at the boundary points go to bgrad
  int nf_int;
  const double *bw, *bnrm;
  const int *bdr_bc;
  const thx_bc *bcs;
  const double *bc_data;
  double *bgrad;  // [b][fp][dim][dim+2]
  // FP32-mixed right-hand side of an FP64 state (u64 set): the kernel reads
  // the FP64 state, narrows it as the to_working kernel does,
  // (float)(u64 - off), writes its own nodes' working copy to yf for the
  // face and volume kernels that follow, and checks their FP64 positivity;
  // u is not read.  Neighbour traces are narrowed from u64 as well, so no
  // CTA reads a working copy another CTA is writing.
  const double *u64;
  float *yf;
  double off[5];
};

template <typename R, int DIM, int N, int EPBX = 0>
__host__ __device__ constexpr size_t grad_smem_bytes() {
  using S = Shape<DIM, N, EPBX>;
  return sizeof(R) * (S::DPAD + (size_t)S::EPB * S::NEQ * (S::ND + 2 * DIM * S::NFP));
}

// Entropy variables of every node (include/EOS.hpp:206-234, as
// include/NSOperator_impl.hpp:11-78 forms them), written once per right-hand
// side: the gradient kernel reads its nodes and its neighbours' face traces
// from here instead of evaluating them (2.2 evaluations per node, each two
// logarithms and seven divisions).
template <typename R, int DIM>
__global__ void __launch_bounds__(256) entropy_kernel(const R *__restrict__ u, long long L,
                                                      const GasT<R> gas, R *__restrict__ sv) {
  constexpr int NEQ = DIM + 2;
  const long long i = (long long)blockIdx.x * 256 + threadIdx.x;
  if (i >= L) return;
  R raw[NEQ], q[NEQ], w[NEQ];
#pragma unroll
  for (int k = 0; k < NEQ; ++k) raw[k] = u[k * L + i];
  reconstruct<R, DIM>(gas, raw, q);
  entropy_vars<R, DIM>(gas, q, w);
#pragma unroll
  for (int k = 0; k < NEQ; ++k) sv[k * L + i] = w[k];
}

// BR1 gradient (include/NSOperator_impl.hpp:11-159,194-517;
// include/DGSEMIntegrator.hpp:764-850,1011-1044).  SV: the entropy variables
// come from a.svars (entropy_kernel) instead of being evaluated here.
// NARROW: compiled with the FP32-mixed reading of an FP64 state (GradArgs::u64);
// the batched kernels, which never take it, leave it out.
template <typename R, int DIM, int N, bool LTE, bool SV = false, int EPBX = 0, bool NARROW = false>
__device__ __forceinline__ void grad_body(const GradArgs<R> &a, const int block) {
  static_assert(!LTE || !IsF32<R>::value, "LTE gas: FP64 only");
  using S = Shape<DIM, N, EPBX>;
  constexpr int ND = S::ND, NEQ = S::NEQ, EPB = S::EPB, NFP = S::NFP, NLF = 2 * DIM;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  R *sD = reinterpret_cast<R *>(smem_raw);   // N*N (padded)
  R *sS = sD + S::DPAD;                      // [EPB][NEQ][ND] own entropy variables
  R *sN = sS + EPB * NEQ * ND;               // [EPB][2*DIM][NEQ][NFP] neighbour traces
  if (dynamic_smem_bytes() < grad_smem_bytes<R, DIM, N, EPBX>()) {
    if (threadIdx.x == 0 && a.status) atomicOr(a.status, STATUS_LAUNCH);
    return;
  }
  const int tid = threadIdx.x;
  for (int i = tid; i < N * N; i += blockDim.x) sD[i] = a.D[i];
  const int el = tid / ND, n = tid % ND;
  const int e0 = block * EPB;
  const int e = e0 + el;
  const bool active = (el < EPB) && (e < a.ne);
  const long long L = (long long)a.ne * ND;
  R q[NEQ];
  if (active) {
    R raw[NEQ];
    if (NARROW && IsF32<R>::value && a.u64) {
      double d[NEQ];
#pragma unroll
      for (int k = 0; k < NEQ; ++k) d[k] = a.u64[k * L + (long long)e * ND + n];
#pragma unroll
      for (int k = 0; k < NEQ; ++k) {
        raw[k] = (R)(d[k] - a.off[k]);
        a.yf[k * L + (long long)e * ND + n] = (float)raw[k];
      }
      if (!fp64_state_positive<DIM>(d, (double)a.gas.gm1)) atomicOr(a.status, STATUS_NONPOSITIVE);
    } else {
#pragma unroll
      for (int k = 0; k < NEQ; ++k) raw[k] = a.u[k * L + (long long)e * ND + n];
    }
    reconstruct<R, DIM>(a.gas, raw, q);
    R w[NEQ];
    if constexpr (SV) {
#pragma unroll
      for (int k = 0; k < NEQ; ++k) w[k] = a.svars[k * L + (long long)e * ND + n];
    } else if constexpr (LTE) {
      lte_entropy_vars<DIM>(a.gas.lte, q, a.gas.Tn[(long long)e * ND + n], a.gas.Cn[(long long)e * ND + n], w);
    } else {
      entropy_vars<R, DIM>(a.gas, q, w);
    }
#pragma unroll
    for (int k = 0; k < NEQ; ++k) sS[(el * NEQ + k) * ND + n] = w[k];
  }
  // entropy variables of the neighbour's trace at every face point of the
  // CTA's elements, one converged task per face point
  for (int t = tid; t < EPB * NLF * NFP; t += S::THREADS) {  // launched with S::THREADS
    const int tel = t / (NLF * NFP), lf = (t / NFP) % NLF, fp = t % NFP;
    const int te = e0 + tel;
    if (te >= a.ne) continue;
    const int fs = a.elem_face[te * NLF + lf];
    if (fs < 0) continue;
    const int f = fs >> 1, side = fs & 1;
    if (a.bw && f >= a.nf_int) continue;  // boundary face: no neighbour
    const int eo = a.face_elem[2 * f + 1 - side];
    const int no = trace_node<DIM>(N, a.face_lface[2 * f + 1 - side], fp);
    R so[NEQ];
    if constexpr (SV) {
#pragma unroll
      for (int k = 0; k < NEQ; ++k) so[k] = a.svars[k * L + (long long)eo * ND + no];
    } else {
      R ro[NEQ], qo[NEQ];
      if (NARROW && IsF32<R>::value && a.u64) {
#pragma unroll
        for (int k = 0; k < NEQ; ++k) ro[k] = (R)(a.u64[k * L + (long long)eo * ND + no] - a.off[k]);
      } else {
#pragma unroll
        for (int k = 0; k < NEQ; ++k) ro[k] = a.u[k * L + (long long)eo * ND + no];
      }
      reconstruct<R, DIM>(a.gas, ro, qo);
      if constexpr (LTE)
        lte_entropy_vars<DIM>(a.gas.lte, qo, a.gas.Tn[(long long)eo * ND + no], a.gas.Cn[(long long)eo * ND + no],
                              so);
      else entropy_vars<R, DIM>(a.gas, qo, so);
    }
#pragma unroll
    for (int k = 0; k < NEQ; ++k) sN[((tel * NLF + lf) * NEQ + k) * NFP + fp] = so[k];
  }
  __syncthreads();
  if (!active) return;
  int c[3];
  node_coords<DIM, N>(n, c);
  R dref[DIM][NEQ];
#pragma unroll
  for (int dir = 0; dir < DIM; ++dir) {
    const int me = c[dir];
    const int line = line_of<DIM, N>(dir, c);
#pragma unroll
    for (int k = 0; k < NEQ; ++k) dref[dir][k] = R(0);
#pragma unroll
    for (int l = 0; l < N; ++l) {
      const int s = line_node<DIM, N>(dir, line, l);
      const R co = sD[me * N + l];
#pragma unroll
      for (int k = 0; k < NEQ; ++k) dref[dir][k] += sS[(el * NEQ + k) * ND + s] * co;
    }
  }
  const R invJ = R(1) / a.jac[(long long)e * a.jac_es + (long long)n * a.jac_ns];
  const R *adj = a.met + (long long)e * a.met_es + (long long)n * a.met_ns;
  R adjr[DIM * DIM];
#pragma unroll
  for (int k = 0; k < DIM * DIM; ++k) adjr[k] = adj[k];
  R g[DIM][NEQ];
#pragma unroll
  for (int cc = 0; cc < DIM; ++cc)
#pragma unroll
    for (int k = 0; k < NEQ; ++k) {
      R s = dref[0][k] * adjr[0 * DIM + cc];
#pragma unroll
      for (int dir = 1; dir < DIM; ++dir) s += dref[dir][k] * adjr[dir * DIM + cc];
      g[cc][k] = invJ * s;
    }
  // interior-face lift: w * 0.5 (S+ - S-) n_c, faces summed then added
  {
    R acc[DIM][NEQ];
    bool any = false;
#pragma unroll
    for (int cc = 0; cc < DIM; ++cc)
#pragma unroll
      for (int k = 0; k < NEQ; ++k) acc[cc][k] = R(0);
#pragma unroll
    for (int dir = 0; dir < DIM; ++dir) {
      const int me = c[dir];
      if (me != 0 && me != N - 1) continue;
      const int lf = 2 * dir + (me == N - 1 ? 1 : 0);
      const int fs = a.elem_face[e * 2 * DIM + lf];
      if (fs < 0) continue;
      const int f = fs >> 1, side = fs & 1;
      if (a.bw && f >= a.nf_int) continue;  // boundary face: below
      const int fp = face_point<DIM, N>(dir, c);
      R so[NEQ];
#pragma unroll
      for (int k = 0; k < NEQ; ++k) so[k] = sN[((el * NLF + lf) * NEQ + k) * NFP + fp];
      const long long wi = (long long)f * a.w_fs + (long long)fp * a.w_ps;
      const R w = side == 0 ? a.wm[wi] : a.wp[wi];
      const R *nr = a.normal + ((long long)f * a.n_fs + (long long)fp * a.n_ps) * DIM;
#pragma unroll
      for (int k = 0; k < NEQ; ++k) {
        const R sown = sS[(el * NEQ + k) * ND + n];
        const R jump = side == 0 ? R(0.5) * (so[k] - sown) : R(0.5) * (sown - so[k]);
#pragma unroll
        for (int cc = 0; cc < DIM; ++cc) acc[cc][k] += w * (jump * nr[cc]);
      }
      any = true;
    }
    if (any) {
#pragma unroll
      for (int cc = 0; cc < DIM; ++cc)
#pragma unroll
        for (int k = 0; k < NEQ; ++k) g[cc][k] += acc[cc][k];
    }
  }
  // boundary faces (include/NSOperator_impl.hpp:285-404,
  // include/DGSEMIntegrator.hpp:1068-1094): w_b (exterior - interior entropy
  // variables) n_c, the node's boundary faces summed then added
  if constexpr (!IsF32<R>::value && !LTE) {
    if (a.bw) {
      R accb[DIM][NEQ];
      bool anyb = false;
#pragma unroll
      for (int cc = 0; cc < DIM; ++cc)
#pragma unroll
        for (int k = 0; k < NEQ; ++k) accb[cc][k] = R(0);
#pragma unroll
      for (int dir = 0; dir < DIM; ++dir) {
        const int me = c[dir];
        if (me != 0 && me != N - 1) continue;
        const int lf = 2 * dir + (me == N - 1 ? 1 : 0);
        const int fs = a.elem_face[e * 2 * DIM + lf];
        if (fs < 0 || (fs >> 1) < a.nf_int) continue;
        const int b = (fs >> 1) - a.nf_int;
        const long long bp = (long long)b * NFP + face_point<DIM, N>(dir, c);
        R w[NEQ], fl[NEQ];
#pragma unroll
        for (int k = 0; k < NEQ; ++k) w[k] = sS[(el * NEQ + k) * ND + n];
        bc_grad_flux<DIM>(a.gas, a.bcs[a.bdr_bc[b]], a.bc_data, w, fl);
        const R scale = a.bw[bp];
        const R *nr = a.bnrm + bp * DIM;
#pragma unroll
        for (int k = 0; k < NEQ; ++k)
#pragma unroll
          for (int cc = 0; cc < DIM; ++cc) accb[cc][k] += scale * (fl[k] * nr[cc]);
        anyb = true;
      }
      if (anyb) {
#pragma unroll
        for (int cc = 0; cc < DIM; ++cc)
#pragma unroll
          for (int k = 0; k < NEQ; ++k) g[cc][k] += accb[cc][k];
      }
    }
  }
  // entropy gradient -> primitive gradient, then the physical viscous flux
  // (include/NavierStokesFlux.hpp:160-290) that the face and volume kernels use
  R dp[DIM * NEQ];
  R vf[NEQ * DIM];
  if constexpr (LTE) {
    const double T = a.gas.Tn[(long long)e * ND + n];
#pragma unroll
    for (int cc = 0; cc < DIM; ++cc) lte_grad_entropy_to_prim<DIM>(q, T, g[cc], dp + cc * NEQ);
    lte_viscous_flux<DIM>(a.gas, q, T, a.gas.Cn[(long long)e * ND + n], dp, vf);
  } else {
    const NodeGas<R, DIM> ng = node_gas<R, DIM>(a.gas, q);
#pragma unroll
    for (int cc = 0; cc < DIM; ++cc) grad_entropy_to_prim_ng<R, DIM>(ng, q, g[cc], dp + cc * NEQ);
    viscous_flux_ng<R, DIM>(a.gas, q, ng, dp, vf);
  }
  constexpr int NV = NEQ - 1;
#pragma unroll
  for (int d = 0; d < DIM; ++d)
#pragma unroll
    for (int k = 0; k < NV; ++k)
      a.vflux[((long long)d * NV + k) * L + (long long)e * ND + n] = vf[(1 + k) * DIM + d];
  // primitive gradients at this node's boundary points, for the viscous
  // boundary fluxes
  if constexpr (!IsF32<R>::value && !LTE) {
    if (a.bw) {
#pragma unroll
      for (int dir = 0; dir < DIM; ++dir) {
        const int me = c[dir];
        if (me != 0 && me != N - 1) continue;
        const int fs = a.elem_face[e * 2 * DIM + 2 * dir + (me == N - 1 ? 1 : 0)];
        if (fs < 0 || (fs >> 1) < a.nf_int) continue;
        const long long bp = (long long)((fs >> 1) - a.nf_int) * NFP + face_point<DIM, N>(dir, c);
#pragma unroll
        for (int i = 0; i < DIM * NEQ; ++i) a.bgrad[bp * DIM * NEQ + i] = dp[i];
      }
    }
  }
}

// Shared memory of the gradient kernel that reads precomputed entropy
// variables: D | own entropy variables [EPB][NEQ][ND] | own conserved state
// [EPB][NEQ][ND] | lift data [EPB][2*DIM][NEQ+1+DIM][NFP] (the jump -- or the
// boundary flux --, the weight and the normal of every face point) | face
// kinds [EPB][2*DIM] (0 none, 1 interior, 2 boundary).
template <typename R, int DIM, int N>
__host__ __device__ constexpr size_t grad_sv_smem_bytes() {
  using S = Shape<DIM, N>;
  return sizeof(R) * (S::DPAD + 2 * (size_t)S::EPB * S::NEQ * S::ND +
                      (size_t)S::EPB * 2 * DIM * (S::NEQ + 1 + DIM) * S::NFP) +
         sizeof(int) * (size_t)S::EPB * 2 * DIM;
}

// The BR1 gradient of grad_body with the entropy variables read from a.svars
// and the work laid out for fewer registers: the face-point tasks stage each
// lift term's factors -- the jump 0.5 (S+ - S-) of interior faces or the
// boundary flux of bc_grad_flux, the weight and the normal -- in shared
// memory, and each node then forms w (jump n_c) per (component, variable),
// sums its faces' terms in face order and adds the sum, as grad_body does;
// the reference-direction derivatives are folded into the physical gradient
// one direction at a time, and the viscous flux is stored as it is formed.
// Same operations in the same order as grad_body, so the results are
// identical.
template <typename R, int DIM, int N>
__device__ __forceinline__ void grad_body_sv(const GradArgs<R> &a, const int block) {
  using S = Shape<DIM, N>;
  constexpr int ND = S::ND, NEQ = S::NEQ, EPB = S::EPB, NFP = S::NFP, NLF = 2 * DIM;
  constexpr int NJ = NEQ + 1 + DIM;  // jump, weight, normal per face point
  extern __shared__ __align__(16) unsigned char smem_raw[];
  R *sD = reinterpret_cast<R *>(smem_raw);   // N*N (padded)
  R *sS = sD + S::DPAD;                      // [EPB][NEQ][ND]
  R *sQ = sS + EPB * NEQ * ND;               // [EPB][NEQ][ND]
  R *sJ = sQ + EPB * NEQ * ND;               // [EPB][NLF][NJ][NFP]
  int *sK = reinterpret_cast<int *>(sJ + EPB * NLF * NJ * NFP);  // [EPB][NLF]
  if (dynamic_smem_bytes() < grad_sv_smem_bytes<R, DIM, N>()) {
    if (threadIdx.x == 0 && a.status) atomicOr(a.status, STATUS_LAUNCH);
    return;
  }
  const int tid = threadIdx.x;
  for (int i = tid; i < N * N; i += blockDim.x) sD[i] = a.D[i];
  const int el = tid / ND, n = tid % ND;
  const int e0 = block * EPB;
  const int e = e0 + el;
  const bool active = (el < EPB) && (e < a.ne);
  const long long L = (long long)a.ne * ND;
  if (active) {
    R raw[NEQ], q[NEQ];
#pragma unroll
    for (int k = 0; k < NEQ; ++k) {
      raw[k] = a.u[k * L + (long long)e * ND + n];
      sS[(el * NEQ + k) * ND + n] = a.svars[k * L + (long long)e * ND + n];
    }
    reconstruct<R, DIM>(a.gas, raw, q);
#pragma unroll
    for (int k = 0; k < NEQ; ++k) sQ[(el * NEQ + k) * ND + n] = q[k];
  }
  for (int t = tid; t < EPB * NLF; t += blockDim.x) {
    const int te = e0 + t / NLF;
    int kind = 0;
    if (te < a.ne) {
      const int fs = a.elem_face[te * NLF + t % NLF];
      if (fs >= 0) kind = (a.bw && (fs >> 1) >= a.nf_int) ? 2 : 1;
    }
    sK[t] = kind;
  }
  __syncthreads();
  // lift factors of every face point of the CTA's elements (unrolled: the
  // neighbours' gathers of the iterations issue together)
#pragma unroll
  for (int t = tid; t < EPB * NLF * NFP; t += S::THREADS) {  // launched with S::THREADS
    const int tel = t / (NLF * NFP), lf = (t / NFP) % NLF, fp = t % NFP;
    const int te = e0 + tel;
    if (te >= a.ne) continue;
    const int fs = a.elem_face[te * NLF + lf];
    if (fs < 0) continue;
    const int f = fs >> 1, side = fs & 1;
    const int nown = trace_node<DIM>(N, lf, fp);
    R *dst = sJ + ((tel * NLF + lf) * NJ) * NFP + fp;
    if (a.bw && f >= a.nf_int) {
      // boundary face (include/NSOperator_impl.hpp:285-404,
      // include/DGSEMIntegrator.hpp:1068-1094): w_b (exterior - interior) n_c
      if constexpr (!IsF32<R>::value) {
        const int b = f - a.nf_int;
        const long long bp = (long long)b * NFP + fp;
        R w[NEQ], fl[NEQ];
#pragma unroll
        for (int k = 0; k < NEQ; ++k) w[k] = sS[(tel * NEQ + k) * ND + nown];
        bc_grad_flux<DIM>(a.gas, a.bcs[a.bdr_bc[b]], a.bc_data, w, fl);
#pragma unroll
        for (int k = 0; k < NEQ; ++k) dst[k * NFP] = fl[k];
        dst[NEQ * NFP] = a.bw[bp];
#pragma unroll
        for (int cc = 0; cc < DIM; ++cc) dst[(NEQ + 1 + cc) * NFP] = a.bnrm[bp * DIM + cc];
      }
      continue;
    }
    // interior face: w * 0.5 (S+ - S-) n_c
    const int eo = a.face_elem[2 * f + 1 - side];
    const int no = trace_node<DIM>(N, a.face_lface[2 * f + 1 - side], fp);
#pragma unroll
    for (int k = 0; k < NEQ; ++k) {
      const R so = a.svars[k * L + (long long)eo * ND + no];
      const R sown = sS[(tel * NEQ + k) * ND + nown];
      dst[k * NFP] = side == 0 ? R(0.5) * (so - sown) : R(0.5) * (sown - so);
    }
    const long long wi = (long long)f * a.w_fs + (long long)fp * a.w_ps;
    dst[NEQ * NFP] = side == 0 ? a.wm[wi] : a.wp[wi];
    const R *nr = a.normal + ((long long)f * a.n_fs + (long long)fp * a.n_ps) * DIM;
#pragma unroll
    for (int cc = 0; cc < DIM; ++cc) dst[(NEQ + 1 + cc) * NFP] = nr[cc];
  }
  __syncthreads();
  if (!active) return;
  int c[3];
  node_coords<DIM, N>(n, c);
  const R *adj = a.met + (long long)e * a.met_es + (long long)n * a.met_ns;
  // physical gradient: sum over directions of D-derivative x adjugate row
  R g[DIM][NEQ];
#pragma unroll
  for (int dir = 0; dir < DIM; ++dir) {
    const int me = c[dir];
    const int line = line_of<DIM, N>(dir, c);
    R dr[NEQ];
#pragma unroll
    for (int k = 0; k < NEQ; ++k) dr[k] = R(0);
    // unrolled: the shared-memory loads of the N terms issue together (same
    // accumulation order; 2 % faster than the rolled loop at 80 registers)
#pragma unroll
    for (int l = 0; l < N; ++l) {
      const int s = line_node<DIM, N>(dir, line, l);
      const R co = sD[me * N + l];
#pragma unroll
      for (int k = 0; k < NEQ; ++k) dr[k] += sS[(el * NEQ + k) * ND + s] * co;
    }
#pragma unroll
    for (int cc = 0; cc < DIM; ++cc) {
      const R ar = adj[dir * DIM + cc];
#pragma unroll
      for (int k = 0; k < NEQ; ++k) {
        if (dir == 0) g[cc][k] = dr[k] * ar;
        else g[cc][k] += dr[k] * ar;
      }
    }
  }
  {
    const R invJ = R(1) / a.jac[(long long)e * a.jac_es + (long long)n * a.jac_ns];
#pragma unroll
    for (int cc = 0; cc < DIM; ++cc)
#pragma unroll
      for (int k = 0; k < NEQ; ++k) g[cc][k] = invJ * g[cc][k];
  }
  // lift: interior faces summed, then added; then the boundary faces
  int jb[DIM], kinds[DIM];
  bool any_i = false, any_b = false;
#pragma unroll
  for (int dir = 0; dir < DIM; ++dir) {
    const int me = c[dir];
    const bool tr = me == 0 || me == N - 1;
    const int lf = 2 * dir + (me == N - 1 ? 1 : 0);
    kinds[dir] = tr ? sK[el * NLF + lf] : 0;
    jb[dir] = ((el * NLF + lf) * NJ) * NFP + face_point<DIM, N>(dir, c);
    any_i |= kinds[dir] == 1;
    any_b |= kinds[dir] == 2;
  }
#pragma unroll
  for (int pass = 1; pass <= 2; ++pass) {
    if (!(pass == 1 ? any_i : any_b)) continue;
#pragma unroll
    for (int cc = 0; cc < DIM; ++cc)
#pragma unroll
      for (int k = 0; k < NEQ; ++k) {
        R acc = R(0);
#pragma unroll
        for (int dir = 0; dir < DIM; ++dir)
          if (kinds[dir] == pass) {
            const R *j = sJ + jb[dir];
            acc += j[NEQ * NFP] * (j[k * NFP] * j[(NEQ + 1 + cc) * NFP]);
          }
        g[cc][k] += acc;
      }
  }
  // entropy gradient -> primitive gradient (in place), then the physical
  // viscous flux (include/NavierStokesFlux.hpp:160-290), stored as formed
  const R *q = sQ + el * NEQ * ND + n;  // q[k * ND]
  R qv[NEQ];
#pragma unroll
  for (int k = 0; k < NEQ; ++k) qv[k] = q[k * ND];
  const NodeGas<R, DIM> ng = node_gas<R, DIM>(a.gas, qv);
#pragma unroll
  for (int cc = 0; cc < DIM; ++cc) {
    R dpc[NEQ];
    grad_entropy_to_prim_ng<R, DIM>(ng, qv, g[cc], dpc);
#pragma unroll
    for (int k = 0; k < NEQ; ++k) g[cc][k] = dpc[k];
  }
  const R *dp = &g[0][0];  // dp[d*NEQ + eq]
  constexpr int NV = NEQ - 1, E = DIM + 1;
  const long long base = (long long)e * ND + n;
  {
    const R mu = viscosity_ng<R, DIM>(a.gas, ng);
    const R kappa = mu * a.gas.cp * a.gas.Pr_inv;
    const R rho = ng.rho;
    const R pressor = ng.p_rho;
    const R fac = fdiv(a.gas.gm1_inv, a.gas.cv * rho);
    R div = R(0);
#pragma unroll
    for (int i = 0; i < DIM; ++i) div += dp[i * NEQ + 1 + i];
#pragma unroll
    for (int dir = 0; dir < DIM; ++dir) {
      R ef = kappa * (fac * (dp[dir * NEQ + E] - pressor * dp[dir * NEQ + 0]));
#pragma unroll
      for (int mom = 0; mom < DIM; ++mom) {
        R tau;
        if (mom == dir) tau = mu * (R(2) * dp[dir * NEQ + 1 + mom] - a.gas.mu_bulk * div);
        else tau = mu * (dp[dir * NEQ + 1 + mom] + dp[mom * NEQ + 1 + dir]);
        a.vflux[((long long)dir * NV + mom) * L + base] = tau;
        ef += ng.v[mom] * tau;
      }
      a.vflux[((long long)dir * NV + DIM) * L + base] = ef;
    }
  }
  // primitive gradients at this node's boundary points, for the viscous
  // boundary fluxes
  if constexpr (!IsF32<R>::value) {
    if (any_b) {
#pragma unroll
      for (int dir = 0; dir < DIM; ++dir) {
        if (kinds[dir] != 2) continue;
        const int me = c[dir];
        const int fs = a.elem_face[e * NLF + 2 * dir + (me == N - 1 ? 1 : 0)];
        const long long bp = (long long)((fs >> 1) - a.nf_int) * NFP + face_point<DIM, N>(dir, c);
#pragma unroll
        for (int i = 0; i < DIM * NEQ; ++i) a.bgrad[bp * DIM * NEQ + i] = dp[i];
      }
    }
  }
}

template <typename R, int DIM, int N, bool LTE, bool SV = false>
__global__ void __launch_bounds__(Shape<DIM, N>::THREADS) grad_kernel(const GradArgs<R> a) {
  grad_body<R, DIM, N, LTE, SV, 0, IsF32<R>::value>(a, blockIdx.x);
}

// The LTE gradient: the same body compiled for three resident CTAs per SM
// (80 registers; the compiler's own 124 fit two): 0.279 -> 0.235 ms at 24^3
// p=4 (four CTAs, 64 registers with heavier spills: 0.243 ms).
template <int DIM, int N>
__global__ void __launch_bounds__(Shape<DIM, N>::THREADS, 3) grad_kernel_lte(const GradArgs<double> a) {
  grad_body<double, DIM, N, true, false>(a, blockIdx.x);
}

// The gradient kernel that reads precomputed entropy variables, bounded to
// three CTAs per SM (four spill about 230 bytes per thread at 64 registers).
template <typename R, int DIM, int N>
__global__ void __launch_bounds__(Shape<DIM, N>::THREADS, 3) grad_sv_kernel(const GradArgs<R> a) {
  grad_body_sv<R, DIM, N>(a, blockIdx.x);
}

// ---------------------------------------------------------------------------
// LTE temperature recovery, once per node and right-hand side
// (include/LTEHelmholtzGasEOS.hpp:59-76 evaluates it on every gas query; the
// face, gradient and volume kernels read the stored T instead).
template <int DIM>
__global__ void __launch_bounds__(256, 2) lte_temperature_kernel(const double *u, long long L, LteDev t,
                                                              double *Tn, int *Cn, unsigned *status) {
  constexpr int NEQ = DIM + 2;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < L; i += stride) {
    double q[NEQ];
#pragma unroll
    for (int k = 0; k < NEQ; ++k) q[k] = u[k * L + i];
    double m2 = 0.0;
#pragma unroll
    for (int d = 0; d < DIM; ++d) m2 += q[1 + d] * q[1 + d];
    const double ke = 0.5 * m2 / q[0];
    const double ei = (q[DIM + 1] - ke) / q[0];
    int st;
    const double T = lte_temperature(t, q[0], ei, &st);
    Tn[i] = T;
    // the node's table cell, read by the kernels that evaluate the gas here
    const LteEval s = lte_at(t, q[0], T);
    Cn[i] = s.valid ? s.cell.off : -1;
    if (st != LTE_CONVERGED) atomicOr(status, STATUS_EOS);
  }
}

// ---------------------------------------------------------------------------
// Persson-Peraire indicator (include/RHSOperator_impl.hpp:355-527): modal
// energy of p*rho with the tensor-product Legendre transform applied by sum
// factorisation (V^-1 = V1^-1 (x) V1^-1 (x) V1^-1).
template <typename R>
struct BlendArgs {
  const R *u;
  int ne;
  const double *vinv;  // N*N, row = degree
  GasT<R> gas;
  double threshold, sharpness, alpha_min, alpha_max;
  double *alpha, *eta;
};

// The indicator of one element by one warp: lanes own nodes lane, lane+32,
// ...; the sum-factorised transform runs through two warp-private shared
// buffers (__syncwarp between directions) and the mode sums through a fixed
// shuffle tree -- no block-wide barrier (include/RHSOperator_impl.hpp:355-437:
// modal energy of p*rho, eta, the sigmoid alpha with its alpha_min/alpha_max
// clipping).
template <typename R, int DIM, int N>
__device__ __forceinline__ void blend_element_warp(const BlendArgs<R> &a, const int e, const double *sV,
                                                   double *bufA, double *bufB) {
  using S = Shape<DIM, N>;
  constexpr int ND = S::ND, NEQ = S::NEQ, J = (ND + 31) / 32;
  const int lane = threadIdx.x & 31;
  const long long L = (long long)a.ne * ND;
#pragma unroll
  for (int j = 0; j < J; ++j) {
    const int n = lane + 32 * j;
    if (n < ND) {
      R raw[NEQ], q[NEQ];
#pragma unroll
      for (int k = 0; k < NEQ; ++k) raw[k] = a.u[k * L + (long long)e * ND + n];
      reconstruct<R, DIM>(a.gas, raw, q);
      bufA[n] = (double)(pressure<R, DIM>(a.gas, q) * q[0]);
    }
  }
  __syncwarp();
  double *src = bufA, *dst = bufB;
#pragma unroll
  for (int dir = 0; dir < DIM; ++dir) {
#pragma unroll
    for (int j = 0; j < J; ++j) {
      const int n = lane + 32 * j;
      if (n < ND) {
        int c[3];
        node_coords<DIM, N>(n, c);
        const int line = line_of<DIM, N>(dir, c);
        double s = 0.0;
#pragma unroll
        for (int l = 0; l < N; ++l) s += sV[c[dir] * N + l] * src[line_node<DIM, N>(dir, line, l)];
        dst[n] = s;
      }
    }
    __syncwarp();
    double *t = src; src = dst; dst = t;
  }
  double mm = 0.0, m1 = 0.0, m2 = 0.0;
#pragma unroll
  for (int j = 0; j < J; ++j) {
    const int n = lane + 32 * j;
    if (n < ND) {
      int c[3];
      node_coords<DIM, N>(n, c);
      int mx = c[0];
#pragma unroll
      for (int d = 1; d < DIM; ++d) mx = c[d] > mx ? c[d] : mx;
      const double mode = src[n];
      const double sq = mode * mode;
      mm += sq;
      if (mx <= N - 2) m1 += sq;
      if (mx <= N - 3) m2 += sq;
    }
  }
#pragma unroll
  for (int off = 16; off >= 1; off >>= 1) {
    mm += __shfl_xor_sync(0xffffffffu, mm, off);
    m1 += __shfl_xor_sync(0xffffffffu, m1, off);
    m2 += __shfl_xor_sync(0xffffffffu, m2, off);
  }
  __syncwarp();  // the buffers are free for the warp's next element
  if (lane == 0) {
    const double eps = 1.0e-30;
    double val = 0.0;
    if (mm > eps) {
      val = 1.0 - m1 / mm;
      if (m1 > eps) val = fmax(val, 1.0 - m2 / m1);
      else val = 1.0;
    }
    const double et = fmin(fmax(val, 0.0), 1.0);
    double al = 1.0 / (1.0 + exp(-a.sharpness * (et - a.threshold) / a.threshold));
    if (al < a.alpha_min) al = 0.0;
    else if (al > 1.0 - a.alpha_min) al = 1.0;
    a.alpha[e] = fmin(al, a.alpha_max);
    if (a.eta) a.eta[e] = et;
  }
}

constexpr int kBlendWarps = 8;

// Elements [e_begin + i) for i over the grid's warps (nsel: element count;
// list: nullptr, or blocks of EPB elements to take the elements from).
template <typename R, int DIM, int N>
__global__ void __launch_bounds__(32 * kBlendWarps) blend_warp_kernel(const BlendArgs<R> a,
                                                                      const int *__restrict__ list,
                                                                      const int *__restrict__ count) {
  using S = Shape<DIM, N>;
  constexpr int ND = S::ND;
  __shared__ double sV[N * N];
  __shared__ double sBuf[kBlendWarps][2][ND];
  for (int i = threadIdx.x; i < N * N; i += blockDim.x) sV[i] = a.vinv[i];
  __syncthreads();
  const int w = threadIdx.x >> 5;
  const long long nitems = list ? (long long)(*count) * S::EPB : (long long)a.ne;
  for (long long it = (long long)blockIdx.x * kBlendWarps + w; it < nitems;
       it += (long long)gridDim.x * kBlendWarps) {
    const int e = list ? list[it / S::EPB] * S::EPB + (int)(it % S::EPB) : (int)it;
    if (e >= a.ne) continue;  // warp-uniform
    blend_element_warp<R, DIM, N>(a, e, sV, sBuf[w][0], sBuf[w][1]);
  }
}


// ---------------------------------------------------------------------------
// SSP-RK3 stage updates (mfem::RK3SSPSolver::Step order) for the unfused path.
// Conversions between the FP64 L-vector and the FP32 working copy u - off.
struct Offsets { double v[5]; };
// FP32 working copy of an FP64 state, node by node, with the positivity of
// the FP64 state checked in FP64 (density and pressure; gm1 = gamma - 1).
template <int DIM>
static __global__ void to_working(long long L, const double *__restrict__ src, float *__restrict__ dst,
                                  Offsets off, double gm1, unsigned *status) {
  constexpr int NEQ = DIM + 2;
  const long long stride = (long long)gridDim.x * blockDim.x;
  bool bad = false;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < L; i += stride) {
    double q[NEQ];
#pragma unroll
    for (int k = 0; k < NEQ; ++k) q[k] = src[k * L + i];  // all loads in flight before the stores
#pragma unroll
    for (int k = 0; k < NEQ; ++k) dst[k * L + i] = (float)(q[k] - off.v[k]);
    if (!fp64_state_positive<DIM>(q, gm1)) bad = true;
  }
  if (bad && status) atomicOr(status, STATUS_NONPOSITIVE);
}

// ---------------------------------------------------------------------------
// Integral measures (include/RHSOperator_impl.hpp:530-717): one thread per
// element sums rho, |m|^2/(2 rho) and rho E over its nodes in node order,
// weighted by J * (w_a w_b w_c), and finds the extrema of pressure,
// temperature and density; the host combines the elements in order.
struct MeasureArgs {
  const double *u;
  int ne, N;
  const double *jac;
  long long jac_es, jac_ns;
  const double *w;  // LGL weights on [0,1]
  GasT<double> gas;
  int lte;
  double *out;      // [e][9]
  unsigned *status;
};

template <int DIM>
__global__ void __launch_bounds__(128) measures_kernel(const MeasureArgs a) {
  constexpr int NEQ = DIM + 2;
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= a.ne) return;
  const int N = a.N, nd = DIM == 2 ? N * N : N * N * N;
  const long long L = (long long)a.ne * nd;
  double m_i = 0, k_i = 0, e_i = 0, pn = 1e32, px = 0, tn = 1e32, tx = 0, dn = 1e32, dx = 0;
  bool bad = false;
  for (int n = 0; n < nd; ++n) {
    double q[NEQ];
#pragma unroll
    for (int k = 0; k < NEQ; ++k) q[k] = a.u[k * L + (long long)e * nd + n];
    const int ia = n % N, ib = (n / N) % N, ic = n / (N * N);
    double W = a.w[ia] * a.w[ib];
    if (DIM == 3) W = W * a.w[ic];
    const double measure = a.jac[(long long)e * a.jac_es + (long long)n * a.jac_ns] * W;
    const double rho = q[0];
    const double kin = ke_density<double, DIM>(q);
    const double rhoE = q[DIM + 1];
    double press, temper;
    if (a.lte) {
      const LteEval sv = lte_state<DIM>(a.gas.lte, q, &bad);
      press = sv.valid ? lte_pressure(a.gas.lte, sv) : 0.0;
      temper = sv.T;
    } else {
      press = pressure<double, DIM>(a.gas, q);
      temper = press / (q[0] * a.gas.R_gas);
    }
    m_i += rho * measure;
    k_i += kin * measure;
    e_i += rhoE * measure;
    tn = fmin(tn, temper); tx = fmax(tx, temper);
    dn = fmin(dn, rho); dx = fmax(dx, rho);
    pn = fmin(pn, press); px = fmax(px, press);
  }
  double *o = a.out + (long long)e * 9;
  o[0] = m_i; o[1] = k_i; o[2] = e_i;
  o[3] = pn; o[4] = px; o[5] = tn; o[6] = tx; o[7] = dn; o[8] = dx;
  if (bad) atomicOr(a.status, STATUS_EOS);
}

// ---------------------------------------------------------------------------
// Stability rates (include/RHSOperator_impl.hpp:10-174) reduced on device.
struct StabArgs {
  const double *u;
  int ne, N;
  const double *jac;
  long long jac_es, jac_ns;
  const double *met;
  long long met_es, met_ns;
  const int *face_elem, *face_lface;
  int nf;
  const double *normal;
  long long n_fs, n_ps;
  const double *wm, *wp;
  long long w_fs, w_ps;
  GasT<double> gas;
  double adv_scale, dif_scale, surf_scale;
  int viscous;
  unsigned long long *out;  // [3] as ordered bit patterns of non-negative doubles
  // boundary points
  int nbf;
  const int *bdr_elem, *bdr_lface, *bdr_bc;
  const double *bnrm, *bw;
  const thx_bc *bcs;
  const double *bc_data;
};

template <int DIM>
__global__ void stability_kernel(const StabArgs a) {
  constexpr int NEQ = DIM + 2;
  const int N = a.N;
  const int nd = DIM == 2 ? N * N : N * N * N;
  const int nfp = DIM == 2 ? N : N * N;
  const long long L = (long long)a.ne * nd;
  const long long nface_pts = (long long)a.nf * nfp;
  const long long nbnd_pts = (long long)a.nbf * nfp;
  double adv = 0.0, dif = 0.0, sur = 0.0;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < L + nface_pts + nbnd_pts;
       t += stride) {
    if (t < L) {
      const long long e = t / nd, n = t % nd;
      double q[NEQ];
#pragma unroll
      for (int k = 0; k < NEQ; ++k) q[k] = a.u[k * L + t];
      const double ij = 1.0 / a.jac[e * a.jac_es + n * a.jac_ns];
      const double *M = a.met + e * a.met_es + n * a.met_ns;
      const double snd = sound_speed<double, DIM>(a.gas, q);
      double ds = 0.0, mss = 0.0;
#pragma unroll
      for (int rd = 0; rd < DIM; ++rd) {
        double vdm = 0.0, mn2 = 0.0;
#pragma unroll
        for (int pd = 0; pd < DIM; ++pd) {
          const double v = M[rd * DIM + pd];
          vdm += (q[1 + pd] / q[0]) * v;
          mn2 += v * v;
        }
        ds += (fabs(vdm) + snd * sqrt(mn2)) * ij;
        mss += mn2 * ij * ij;
      }
      adv = fmax(adv, a.adv_scale * ds);
      if (a.viscous) {
        const double mu = viscosity<double, DIM>(a.gas, q);
        const double lon = (2.0 - a.gas.mu_bulk) * mu;
        const double md = fmax(mu, lon) / q[0];
        const double td = (mu * a.gas.cp * a.gas.Pr_inv) * a.gas.gamma / (q[0] * a.gas.cp);
        dif = fmax(dif, a.dif_scale * fmax(md, td) * mss);
      }
    } else if (t >= L + nface_pts) {
      // boundary point (include/RHSOperator_impl.hpp:176-268)
      const long long bpt = t - L - nface_pts;
      const int b = (int)(bpt / nfp), fp = (int)(bpt % nfp);
      const long long e = a.bdr_elem[b];
      const long long node = trace_node<DIM>(N, a.bdr_lface[b], fp);
      double q[NEQ];
#pragma unroll
      for (int k = 0; k < NEQ; ++k) q[k] = a.u[k * L + e * nd + node];
      const double *nr = a.bnrm + bpt * DIM;
      double n2 = 0.0, vn = 0.0;
#pragma unroll
      for (int d = 0; d < DIM; ++d) {
        n2 += nr[d] * nr[d];
        vn += (q[1 + d] / q[0]) * nr[d];
      }
      double ws = fabs(vn) + sound_speed<double, DIM>(a.gas, q) * sqrt(n2);
      const thx_bc bc = a.bcs[a.bdr_bc[b]];
      if (bc.type == THX_BC_PRESCRIBED_STATE || bc.type == THX_BC_SUPERSONIC_INFLOW) {
        double qe[NEQ];
#pragma unroll
        for (int k = 0; k < NEQ; ++k) qe[k] = a.bc_data[bc.data_index + k];
        if (a.viscous) {
          const double ij = 1.0 / a.jac[e * a.jac_es + node * a.jac_ns];
          const double *M = a.met + e * a.met_es + node * a.met_ns;
          double mss = 0.0;
#pragma unroll
          for (int rd = 0; rd < DIM; ++rd) {
            double mn2 = 0.0;
#pragma unroll
            for (int pd = 0; pd < DIM; ++pd) mn2 += M[rd * DIM + pd] * M[rd * DIM + pd];
            mss += mn2 * ij * ij;
          }
          const double mu = viscosity<double, DIM>(a.gas, qe);
          const double lon = (2.0 - a.gas.mu_bulk) * mu;
          const double md = fmax(mu, lon) / qe[0];
          const double td = (mu * a.gas.cp * a.gas.Pr_inv) * a.gas.gamma / (qe[0] * a.gas.cp);
          dif = fmax(dif, a.dif_scale * fmax(md, td) * mss);
        }
        double ve = 0.0;
#pragma unroll
        for (int d = 0; d < DIM; ++d) ve += (qe[1 + d] / qe[0]) * nr[d];
        ws = fmax(ws, fabs(ve) + sound_speed<double, DIM>(a.gas, qe) * sqrt(n2));
      }
      sur = fmax(sur, ws * fabs(a.bw[bpt]) * a.surf_scale);
    } else {
      const long long fpt = t - L;
      const int f = (int)(fpt / nfp), fp = (int)(fpt % nfp);
      const long long im = (long long)a.face_elem[2 * f] * nd + trace_node<DIM>(N, a.face_lface[2 * f], fp);
      const long long ip = (long long)a.face_elem[2 * f + 1] * nd + trace_node<DIM>(N, a.face_lface[2 * f + 1], fp);
      double qm[NEQ], qp[NEQ];
#pragma unroll
      for (int k = 0; k < NEQ; ++k) { qm[k] = a.u[k * L + im]; qp[k] = a.u[k * L + ip]; }
      const double *nr = a.normal + ((long long)f * a.n_fs + (long long)fp * a.n_ps) * DIM;
      double n2 = 0.0, vm = 0.0, vp = 0.0;
#pragma unroll
      for (int d = 0; d < DIM; ++d) {
        n2 += nr[d] * nr[d];
        vm += (qm[1 + d] / qm[0]) * nr[d];
        vp += (qp[1 + d] / qp[0]) * nr[d];
      }
      const double nm = sqrt(n2);
      const double ws = fmax(fabs(vm) + sound_speed<double, DIM>(a.gas, qm) * nm,
                             fabs(vp) + sound_speed<double, DIM>(a.gas, qp) * nm);
      const long long wi = (long long)f * a.w_fs + (long long)fp * a.w_ps;
      sur = fmax(sur, ws * fmax(fabs(a.wm[wi]), fabs(a.wp[wi])) * a.surf_scale);
    }
  }
  // warp reduce then one atomic per warp
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    adv = fmax(adv, __shfl_xor_sync(0xffffffffu, adv, o));
    dif = fmax(dif, __shfl_xor_sync(0xffffffffu, dif, o));
    sur = fmax(sur, __shfl_xor_sync(0xffffffffu, sur, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMax(&a.out[0], (unsigned long long)__double_as_longlong(adv));
    atomicMax(&a.out[1], (unsigned long long)__double_as_longlong(sur));
    atomicMax(&a.out[2], (unsigned long long)__double_as_longlong(dif));
  }
}


// dt = cfl / (max(advective, surface) + diffusive) from the stability
// kernel's rates (src/Simulation.cpp:1150-1160), on the device, so that a
// variable-dt time loop needs no host round trip; a non-positive total sets
// the numerics flag and dt = 0.
static __global__ void cfl_dt_kernel(const unsigned long long *rates, double cfl, double *dt, double *history,
                              unsigned *status) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const double adv = __longlong_as_double((long long)rates[0]);
  const double sur = __longlong_as_double((long long)rates[1]);
  const double dif = __longlong_as_double((long long)rates[2]);
  const double total = (adv > sur ? adv : sur) + dif;
  double d = 0.0;
  if (total > 0.0) d = cfl / total;
  else atomicOr(status, STATUS_NONFINITE);
  *dt = d;
  if (history) *history = d;
}

// ---------------------------------------------------------------------------
// Batched persistent forms: one launch serves every case of a batch group.
// work[w] names a per-case argument record (item) and a CTA-sized block of
// that case; a fixed grid walks the list, whose length *nwork is read on the
// device, so a captured graph stays valid while cases come and go.
struct BatchWork {
  int item;
  int block;
};

// A work item's argument record copied into shared memory by the whole CTA
// (one coalesced read): the body then reads its fields at shared-memory
// latency, as a one-case kernel reads its parameters from the constant bank,
// instead of one dependent global load per field.
template <typename A>
__device__ __forceinline__ void stage_record(unsigned char *dst, const A *src) {
  static_assert(sizeof(A) % 8 == 0 && alignof(A) >= 8, "8-byte words");
  const unsigned long long *s = reinterpret_cast<const unsigned long long *>(src);
  unsigned long long *d = reinterpret_cast<unsigned long long *>(dst);
  for (int i = threadIdx.x; i < (int)(sizeof(A) / 8); i += blockDim.x) d[i] = s[i];
}

// The batched volume kernel is compiled for four resident 256-thread CTAs per
// SM (eight of the half-size CTAs): 64 registers a thread.  Bounded to the
// FP32 one-case kernel's six CTAs (40 registers) its persistent loop spills
// about 100 bytes per thread and runs 4-8 % slower (2-D).
template <typename R, int DIM, int N, int EPBX>
constexpr int vol_batch_min_blocks() {
  return 4 * Shape<DIM, N>::THREADS / Shape<DIM, N, EPBX>::THREADS;
}
template <typename R, int DIM, int N, int VOL, bool NS, int EPBX = 0>
__global__ void __launch_bounds__(Shape<DIM, N, EPBX>::THREADS, (vol_batch_min_blocks<R, DIM, N, EPBX>()))
volume_batched(const VolArgs<R> *__restrict__ args, const BatchWork *__restrict__ work,
               const int *__restrict__ nwork) {
  __shared__ __align__(16) unsigned char sa[sizeof(VolArgs<R>)];
  const int n = *nwork;
  for (int w = blockIdx.x; w < n; w += gridDim.x) {
    __syncthreads();  // the previous item's shared memory is free
    const BatchWork it = work[w];
    stage_record(sa, &args[it.item]);
    __syncthreads();
    volume_body<R, DIM, N, VOL, NS, false, EPBX>(*reinterpret_cast<const VolArgs<R> *>(sa), it.block);
  }
}

template <typename R, int DIM, int N, int EPBX = 0>
__global__ void __launch_bounds__(Shape<DIM, N, EPBX>::THREADS)
grad_batched(const GradArgs<R> *__restrict__ args, const BatchWork *__restrict__ work,
             const int *__restrict__ nwork) {
  __shared__ __align__(16) unsigned char sa[sizeof(GradArgs<R>)];
  const int n = *nwork;
  for (int w = blockIdx.x; w < n; w += gridDim.x) {
    __syncthreads();
    const BatchWork it = work[w];
    stage_record(sa, &args[it.item]);
    __syncthreads();
    grad_body<R, DIM, N, false, false, EPBX>(*reinterpret_cast<const GradArgs<R> *>(sa), it.block);
  }
}

// face work blocks are 128 face points; compiled for eight resident CTAs per
// SM in FP32 (the register budget of the one-case FP32 face kernel)
template <typename R, int DIM, int SURF, bool NS>
__global__ void __launch_bounds__(128, IsF32<R>::value ? 8 : 5)
face_batched(const FaceArgs<R> *__restrict__ args, const BatchWork *__restrict__ work,
             const int *__restrict__ nwork) {
  __shared__ __align__(16) unsigned char sa[sizeof(FaceArgs<R>)];
  const int n = *nwork;
  for (int w = blockIdx.x; w < n; w += gridDim.x) {
    __syncthreads();
    const BatchWork it = work[w];
    stage_record(sa, &args[it.item]);
    __syncthreads();
    face_body<R, DIM, SURF, NS>(*reinterpret_cast<const FaceArgs<R> *>(sa),
                                (long long)it.block * 128 + threadIdx.x);
  }
}

// ---------------------------------------------------------------------------
// FP64 islands of the FP32-mixed Euler path with blending.  The blended
// (troubled) elements are where FP32 rounding of the state matters: a blast
// core's energy density is large while its pressure may be small.  After the
// FP32 indicator, every block (of EPB elements) holding a blended element is
// flagged and listed, and so is every face touching a flagged block; the
// FP64 kernels then evaluate the indicator, the face fluxes, the subcell FV
// rate and the volume term with the stage update for exactly those blocks
// and faces from the FP64 stage state, while the FP32 volume kernel skips
// the flagged blocks.  The list walkers are persistent grids that read the
// list length on the device, so a captured graph stays valid.

// flag[b] = block b holds an element with alpha > 0 (alpha may be null) or is
// flagged in stat (may be null: blocks next to a boundary face); flagged
// blocks are appended to list (count zeroed beforehand)
template <typename R>
__global__ void island_blocks_kernel(int ne, int epb, const double *__restrict__ alpha,
                                     const int *__restrict__ stat, int *__restrict__ flag,
                                     int *__restrict__ list, int *count) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  const int nb = (ne + epb - 1) / epb;
  if (b >= nb) return;
  bool any = stat && stat[b];
  for (int k = 0; alpha && k < epb; ++k) {
    const int e = b * epb + k;
    if (e < ne && alpha[e] > 0.0) any = true;
  }
  flag[b] = any ? 1 : 0;
  if (any) list[atomicAdd(count, 1)] = b;
}

// faces with a side in a flagged block, appended to list (count zeroed beforehand)
static __global__ void island_faces_kernel(int nf, int epb, const int *__restrict__ face_elem,
                                    const int *__restrict__ flag, int *__restrict__ list, int *count) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= nf) return;
  if (flag[face_elem[2 * f] / epb] || flag[face_elem[2 * f + 1] / epb]) list[atomicAdd(count, 1)] = f;
}

template <typename R, int DIM, int N, int VOL>
__global__ void __launch_bounds__(Shape<DIM, N>::THREADS, 4)
volume_list_kernel(const VolArgs<R> a, const int *__restrict__ list, const int *__restrict__ count) {
  const int n = *count;
  for (int w = blockIdx.x; w < n; w += gridDim.x) {
    __syncthreads();  // the previous block's shared memory is free
    volume_body<R, DIM, N, VOL, false, true>(a, list[w]);
  }
}

template <typename R, int DIM, int N>
__global__ void __launch_bounds__(Shape<DIM, N>::THREADS)
fv_list_kernel(const VolArgs<R> a, const int *__restrict__ list, const int *__restrict__ count) {
  const int n = *count;
  for (int w = blockIdx.x; w < n; w += gridDim.x) {
    __syncthreads();
    fv_body<R, DIM, N>(a, list[w]);
  }
}

// face points of the listed faces (a.order = the face list)
template <typename R, int DIM, int SURF>
__global__ void __launch_bounds__(128)
face_list_kernel(const FaceArgs<R> a, const int *__restrict__ count) {
  const int nfp = DIM == 2 ? a.N : a.N * a.N;
  const long long total = (long long)(*count) * nfp;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x)
    face_body<R, DIM, SURF, false>(a, t);
}

}  // namespace thx
