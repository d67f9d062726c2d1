// Mesh set-up for straight-sided (bi/trilinear) cells: the face table on the
// host and the geometric factors on the device.
//
// Replaces the reference's MFEM set-up of the DGSEM caches
// (include/dgsem_cache_utilities.hpp:83-215 SetupGeometricTerms, 470-513
// AssembleElementVolumeGeometricTerms, 516-639 AssembleInteriorFaceGeometryTerms):
// at every LGL node the Jacobian determinant and the rows of the adjugate
// Jacobian (the metric terms), at every face point the minus element's
// outward, face-Jacobian-scaled normal and the lift weights 1/(w0 J) of both
// sides.  Reference coordinates are [0,1]^d.  Cells are given by their 2^d
// vertices in lexicographic order of the reference coordinates (x fastest)
// and must be oriented along the mesh's axes, so that local face 2d / 2d+1 is
// the -/+ face of direction d and the two sides of a face list their face
// points in the same order (the structured meshes of the reference's cases).
#include "theseus_b200.h"
#include "thx_host.h"

#include <algorithm>
#include <array>
#include <cuda_runtime.h>
#include <tuple>
#include <vector>

namespace {

constexpr int kMaxNodes = 16;

struct LglNodes {
  double x[kMaxNodes];
  double w0;
};

__device__ __forceinline__ int cell_trace_node(int dim, int N, int lf, int fp) {
  const int dir = lf >> 1;
  const int pos = (lf & 1) ? N - 1 : 0;
  if (dim == 2) return dir == 0 ? pos + N * fp : fp + N * pos;
  const int a = fp % N, b = fp / N;
  if (dir == 0) return pos + N * (a + N * b);
  if (dir == 1) return a + N * (pos + N * b);
  return a + N * (b + N * pos);
}

// One thread per (element, node): Jacobian determinant, adjugate rows and
// (optionally) the node's physical coordinates.
template <int DIM>
__global__ void cell_volume_kernel(int ne, int N, LglNodes r, const double *__restrict__ corners,
                                   double *__restrict__ jac, double *__restrict__ metric,
                                   double *__restrict__ coords) {
  const int nd = DIM == 2 ? N * N : N * N * N;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)ne * nd) return;
  const int e = (int)(t / nd), n = (int)(t % nd);
  const double a = r.x[n % N], b = r.x[(n / N) % N];
  const double *c = corners + (size_t)e * (1 << DIM) * DIM;
  if (DIM == 2) {
    // X0 (0,0) = c0, X1 (1,0) = c1, X2 (1,1) = c3, X3 (0,1) = c2
    double dxi[2], deta[2], pos[2];
    for (int d = 0; d < 2; ++d) {
      const double X0 = c[0 * 2 + d], X1 = c[1 * 2 + d], X2 = c[3 * 2 + d], X3 = c[2 * 2 + d];
      dxi[d] = (1 - b) * (X1 - X0) + b * (X2 - X3);
      deta[d] = (1 - a) * (X3 - X0) + a * (X2 - X1);
      pos[d] = (1 - a) * (1 - b) * X0 + a * (1 - b) * X1 + a * b * X2 + (1 - a) * b * X3;
    }
    jac[t] = dxi[0] * deta[1] - deta[0] * dxi[1];
    double *m = metric + t * 4;
    m[0] = deta[1];
    m[1] = -deta[0];
    m[2] = -dxi[1];
    m[3] = dxi[0];
    if (coords)
      for (int d = 0; d < 2; ++d) coords[(size_t)d * ne * nd + t] = pos[d];
  } else {
    const double g = r.x[n / (N * N)];
    double da[3], db[3], dc[3], pos[3];
    for (int d = 0; d < 3; ++d) {
      const double *v = c + d;
      auto C = [&](int k) { return v[k * 3]; };
      da[d] = (1 - b) * (1 - g) * (C(1) - C(0)) + b * (1 - g) * (C(3) - C(2)) + (1 - b) * g * (C(5) - C(4)) +
              b * g * (C(7) - C(6));
      db[d] = (1 - a) * (1 - g) * (C(2) - C(0)) + a * (1 - g) * (C(3) - C(1)) + (1 - a) * g * (C(6) - C(4)) +
              a * g * (C(7) - C(5));
      dc[d] = (1 - a) * (1 - b) * (C(4) - C(0)) + a * (1 - b) * (C(5) - C(1)) + (1 - a) * b * (C(6) - C(2)) +
              a * b * (C(7) - C(3));
      pos[d] = (1 - a) * (1 - b) * (1 - g) * C(0) + a * (1 - b) * (1 - g) * C(1) + (1 - a) * b * (1 - g) * C(2) +
               a * b * (1 - g) * C(3) + (1 - a) * (1 - b) * g * C(4) + a * (1 - b) * g * C(5) +
               (1 - a) * b * g * C(6) + a * b * g * C(7);
    }
    double *m = metric + t * 9;
    // adjugate rows: db x dc, dc x da, da x db
    m[0] = db[1] * dc[2] - db[2] * dc[1];
    m[1] = db[2] * dc[0] - db[0] * dc[2];
    m[2] = db[0] * dc[1] - db[1] * dc[0];
    m[3] = dc[1] * da[2] - dc[2] * da[1];
    m[4] = dc[2] * da[0] - dc[0] * da[2];
    m[5] = dc[0] * da[1] - dc[1] * da[0];
    m[6] = da[1] * db[2] - da[2] * db[1];
    m[7] = da[2] * db[0] - da[0] * db[2];
    m[8] = da[0] * db[1] - da[1] * db[0];
    jac[t] = da[0] * m[0] + da[1] * m[1] + da[2] * m[2];
    if (coords)
      for (int d = 0; d < 3; ++d) coords[(size_t)d * ne * nd + t] = pos[d];
  }
}

// One thread per (face, face point): the minus element's adjugate row of the
// face direction at the trace node (outward: negated on a - face) and the
// lift weights of both sides; boundary faces (minus side only) after them.
// Face entries that name no element or local face of the mesh get NaN
// outputs instead of a read outside the arrays.
template <int DIM>
__global__ void cell_face_kernel(int ne, int N, LglNodes r, const double *__restrict__ jac,
                                 const double *__restrict__ metric, int nf, const int32_t *__restrict__ fe,
                                 const int32_t *__restrict__ fl, double *__restrict__ normal,
                                 double *__restrict__ wm, double *__restrict__ wp, int nbf,
                                 const int32_t *__restrict__ be, const int32_t *__restrict__ bl,
                                 double *__restrict__ bnormal, double *__restrict__ bw) {
  const int nd = DIM == 2 ? N * N : N * N * N;
  const int nfp = DIM == 2 ? N : N * N;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long nint = (long long)nf * nfp;
  if (t >= nint + (long long)nbf * nfp) return;
  const bool bdr = t >= nint;
  const long long s = bdr ? t - nint : t;
  const int f = (int)(s / nfp), fp = (int)(s % nfp);
  const int e = bdr ? be[f] : fe[2 * f], lf = bdr ? bl[f] : fl[2 * f];
  double *out = (bdr ? bnormal : normal) + s * DIM;
  const int ep = bdr ? 0 : fe[2 * f + 1], lp = bdr ? 0 : fl[2 * f + 1];
  if (e < 0 || e >= ne || lf < 0 || lf >= 2 * DIM || ep < 0 || ep >= ne || lp < 0 || lp >= 2 * DIM) {
    const double nan = __longlong_as_double(0x7ff8000000000000LL);
    for (int d = 0; d < DIM; ++d) out[d] = nan;
    if (bdr) bw[s] = nan;
    else wm[s] = wp[s] = nan;
    return;
  }
  const long long node = (long long)e * nd + cell_trace_node(DIM, N, lf, fp);
  const double *row = metric + (node * DIM + (lf >> 1)) * DIM;
  for (int d = 0; d < DIM; ++d) out[d] = (lf & 1) ? row[d] : 0.0 - row[d];
  const double w = 1.0 / (r.w0 * jac[node]);
  if (bdr) {
    bw[s] = w;
  } else {
    wm[s] = w;
    const long long np_ = (long long)ep * nd + cell_trace_node(DIM, N, lp, fp);
    wp[s] = 1.0 / (r.w0 * jac[np_]);
  }
}

}  // namespace

extern "C" {

int thx_cell_faces(int dim, int ne, const int64_t *vertex_ids, int32_t *face_elem, int32_t *face_lface,
                   int32_t *num_faces, int32_t *bdr_elem, int32_t *bdr_lface, int32_t *num_bdr_faces) {
  if ((dim != 2 && dim != 3) || ne <= 0 || !vertex_ids || !num_faces || !num_bdr_faces)
    return THX_ERR_INVALID_ARGUMENT;
  const int nv = 1 << dim, nfv = 1 << (dim - 1);
  // every local face keyed by its sorted vertex ids; equal keys end up
  // adjacent after one sort
  struct Side {
    std::array<int64_t, 4> key;
    int e, lf;
  };
  std::vector<Side> sides((size_t)ne * 2 * dim);
  for (int e = 0; e < ne; ++e)
    for (int lf = 0; lf < 2 * dim; ++lf) {
      const int dir = lf >> 1, side = lf & 1;
      Side &sd = sides[(size_t)e * 2 * dim + lf];
      sd.key = {-1, -1, -1, -1};
      sd.e = e;
      sd.lf = lf;
      int m = 0;
      for (int v = 0; v < nv; ++v)
        if (((v >> dir) & 1) == side) sd.key[m++] = vertex_ids[(size_t)e * nv + v];
      std::sort(sd.key.begin(), sd.key.begin() + nfv);
    }
  std::sort(sides.begin(), sides.end(), [](const Side &a, const Side &b) {
    return a.key != b.key ? a.key < b.key : (a.e != b.e ? a.e < b.e : a.lf < b.lf);
  });
  std::vector<std::tuple<int, int, int, int, int>> faces;
  std::vector<std::tuple<int, int, int>> bfaces;
  for (size_t i = 0; i < sides.size();) {
    size_t j = i + 1;
    while (j < sides.size() && sides[j].key == sides[i].key) ++j;
    if (j - i == 2) {
      std::pair<int, int> m{sides[i].e, sides[i].lf}, p{sides[i + 1].e, sides[i + 1].lf};
      if ((m.second & 1) == 0) std::swap(m, p);  // minus side: the element whose + face it is
      if (p.second != m.second - 1) return THX_ERR_INVALID_ARGUMENT;  // faces not aligned
      faces.emplace_back(m.second >> 1, m.first, m.second, p.first, p.second);
    } else if (j - i == 1) {
      bfaces.emplace_back(sides[i].lf >> 1, sides[i].e, sides[i].lf);
    } else {
      return THX_ERR_INVALID_ARGUMENT;  // non-manifold face
    }
    i = j;
  }
  std::sort(faces.begin(), faces.end());
  std::sort(bfaces.begin(), bfaces.end());
  *num_faces = (int32_t)faces.size();
  *num_bdr_faces = (int32_t)bfaces.size();
  if (face_elem && face_lface)
    for (size_t f = 0; f < faces.size(); ++f) {
      face_elem[2 * f] = std::get<1>(faces[f]);
      face_lface[2 * f] = std::get<2>(faces[f]);
      face_elem[2 * f + 1] = std::get<3>(faces[f]);
      face_lface[2 * f + 1] = std::get<4>(faces[f]);
    }
  if (bdr_elem && bdr_lface)
    for (size_t b = 0; b < bfaces.size(); ++b) {
      bdr_elem[b] = std::get<1>(bfaces[b]);
      bdr_lface[b] = std::get<2>(bfaces[b]);
    }
  return THX_OK;
}

int thx_cell_geometry(int dim, int order, int ne, const double *corners, int nf, const int32_t *face_elem,
                      const int32_t *face_lface, int nbf, const int32_t *bdr_elem, const int32_t *bdr_lface,
                      double *jac, double *metric, double *face_normal, double *face_wminus,
                      double *face_wplus, double *bdr_normal, double *bdr_weight, double *node_coords,
                      void *stream) {
  const int N = order + 1;
  if ((dim != 2 && dim != 3) || order < 1 || N > kMaxNodes || ne <= 0 || nf < 0 || nbf < 0 || !corners ||
      !jac || !metric)
    return THX_ERR_INVALID_ARGUMENT;
  if (nf > 0 && (!face_elem || !face_lface || !face_normal || !face_wminus || !face_wplus))
    return THX_ERR_INVALID_ARGUMENT;
  if (nbf > 0 && (!bdr_elem || !bdr_lface || !bdr_normal || !bdr_weight)) return THX_ERR_INVALID_ARGUMENT;
  LglNodes r{};
  double w[kMaxNodes];
  thx::lgl_rule(N, r.x, w);
  r.w0 = w[0];
  cudaStream_t s = (cudaStream_t)stream;
  const int nd = dim == 2 ? N * N : N * N * N, nfp = dim == 2 ? N : N * N;
  const long long nv = (long long)ne * nd;
  const int vgrid = (int)((nv + 255) / 256);
  if (dim == 2) cell_volume_kernel<2><<<vgrid, 256, 0, s>>>(ne, N, r, corners, jac, metric, node_coords);
  else cell_volume_kernel<3><<<vgrid, 256, 0, s>>>(ne, N, r, corners, jac, metric, node_coords);
  if (cudaGetLastError() != cudaSuccess) return THX_ERR_CUDA;
  const long long nfw = (long long)(nf + nbf) * nfp;
  if (nfw > 0) {
    const int fgrid = (int)((nfw + 255) / 256);
    if (dim == 2)
      cell_face_kernel<2><<<fgrid, 256, 0, s>>>(ne, N, r, jac, metric, nf, face_elem, face_lface, face_normal,
                                                face_wminus, face_wplus, nbf, bdr_elem, bdr_lface, bdr_normal,
                                                bdr_weight);
    else
      cell_face_kernel<3><<<fgrid, 256, 0, s>>>(ne, N, r, jac, metric, nf, face_elem, face_lface, face_normal,
                                                face_wminus, face_wplus, nbf, bdr_elem, bdr_lface, bdr_normal,
                                                bdr_weight);
    if (cudaGetLastError() != cudaSuccess) return THX_ERR_CUDA;
  }
  return THX_OK;
}

}  // extern "C"
