// thx_host.cpp -- host-side set-up that MFEM performs for the reference:
// Legendre-Gauss-Lobatto rule on [0,1], derivative operators, periodic
// Cartesian box meshes with their geometric factors, and the 1-D Legendre
// transform of the Persson-Peraire indicator.  No device work happens here.
#include "thx_host.h"

#include <cmath>
#include <cstring>
#include <vector>

namespace thx {

// LGL rule on [0,1]: end points plus the roots of P'_{N} (Newton on the
// Legendre three-term recurrence); weights 2/(N(N+1) P_N(z)^2) halved.
void lgl_rule(int np, double *x, double *w) {
  const int N = np - 1;
  for (int i = 0; i < np; ++i) {
    double z = -std::cos(M_PI * i / N);
    double p0 = 1.0, p1 = z;
    for (int it = 0; it < 100; ++it) {
      p0 = 1.0;
      p1 = z;
      for (int k = 2; k <= N; ++k) {
        const double p2 = ((2.0 * k - 1.0) * z * p1 - (k - 1.0) * p0) / k;
        p0 = p1;
        p1 = p2;
      }
      const double dz = (z * p1 - p0) / (np * p1);
      z -= dz;
      if (std::fabs(dz) < 1e-16) break;
    }
    p0 = 1.0;
    p1 = z;
    for (int k = 2; k <= N; ++k) {
      const double p2 = ((2.0 * k - 1.0) * z * p1 - (k - 1.0) * p0) / k;
      p0 = p1;
      p1 = p2;
    }
    x[i] = 0.5 * (z + 1.0);
    w[i] = 1.0 / (N * np * p1 * p1);
  }
  x[0] = 0.0;
  x[np - 1] = 1.0;
}

// D(i,l) = l'_l(x_i) from barycentric weights; Dhat = D with the weak-form
// boundary terms; Dhat2 = 2D with boundary terms
// (include/dgsem_cache_utilities.hpp:123-181).  Row-major [i*N+l].
void derivative_operators(int np, const double *x, const double *w, double *D, double *Dhat,
                          double *Dhat2) {
  std::vector<double> wb(np, 1.0);
  for (int i = 1; i < np; ++i)
    for (int j = 0; j < i; ++j) {
      wb[j] *= (x[j] - x[i]);
      wb[i] *= (x[i] - x[j]);
    }
  for (int i = 0; i < np; ++i) wb[i] = 1.0 / wb[i];
  for (int k = 0; k < np * np; ++k) D[k] = 0.0;
  for (int l = 0; l < np; ++l)
    for (int i = 0; i < np; ++i)
      if (l != i) {
        D[i * np + l] = wb[l] / wb[i] / (x[i] - x[l]);
        D[i * np + i] -= D[i * np + l];
      }
  for (int k = 0; k < np * np; ++k) {
    Dhat[k] = D[k];
    Dhat2[k] = 2.0 * D[k];
  }
  Dhat[0] += 1.0 / w[0];
  Dhat[np * np - 1] -= 1.0 / w[np - 1];
  Dhat2[0] += 1.0 / w[0];
  Dhat2[np * np - 1] -= 1.0 / w[np - 1];
}

// Inverse of the 1-D shifted-Legendre Vandermonde V(i,k) = P_k(2 x_i - 1)
// (src/ModalBasis.cpp:115-140 builds the tensor product of these).  Output
// row k (degree), column i (node).  Gauss-Jordan with partial pivoting.
bool legendre_vinv(int np, const double *x, double *vinv) {
  std::vector<double> A(np * np), I(np * np, 0.0);
  for (int i = 0; i < np; ++i) {
    const double z = 2.0 * x[i] - 1.0;
    double Pm = 1.0, P = z;
    A[i * np + 0] = 1.0;
    if (np > 1) A[i * np + 1] = z;
    for (int n = 1; n + 1 < np; ++n) {
      const double Pn = ((2.0 * n + 1.0) * z * P - n * Pm) / (n + 1.0);
      Pm = P;
      P = Pn;
      A[i * np + n + 1] = Pn;
    }
    I[i * np + i] = 1.0;
  }
  for (int c = 0; c < np; ++c) {
    int piv = c;
    for (int r = c + 1; r < np; ++r)
      if (std::fabs(A[r * np + c]) > std::fabs(A[piv * np + c])) piv = r;
    if (A[piv * np + c] == 0.0) return false;
    for (int k = 0; k < np; ++k) {
      std::swap(A[c * np + k], A[piv * np + k]);
      std::swap(I[c * np + k], I[piv * np + k]);
    }
    const double inv = 1.0 / A[c * np + c];
    for (int k = 0; k < np; ++k) { A[c * np + k] *= inv; I[c * np + k] *= inv; }
    for (int r = 0; r < np; ++r) {
      if (r == c) continue;
      const double f = A[r * np + c];
      for (int k = 0; k < np; ++k) { A[r * np + k] -= f * A[c * np + k]; I[r * np + k] -= f * I[c * np + k]; }
    }
  }
  // I = V^{-1}: rows indexed by degree k, columns by node i
  std::memcpy(vinv, I.data(), sizeof(double) * np * np);
  return true;
}

}  // namespace thx

extern "C" {

int thx_sizes(int dim, int order, int32_t *nodes_per_element, int32_t *points_per_face,
              int32_t *num_equations) {
  if (dim < 2 || dim > 3 || order < 1) return THX_ERR_INVALID_ARGUMENT;
  const int N = order + 1;
  if (nodes_per_element) *nodes_per_element = dim == 2 ? N * N : N * N * N;
  if (points_per_face) *points_per_face = dim == 2 ? N : N * N;
  if (num_equations) *num_equations = dim + 2;
  return THX_OK;
}

int thx_lgl(int np, double *x, double *w) {
  if (np < 2 || !x || !w) return THX_ERR_INVALID_ARGUMENT;
  thx::lgl_rule(np, x, w);
  return THX_OK;
}

int thx_box_counts(int dim, const int32_t *n, int32_t *num_elements, int32_t *num_faces) {
  if (dim < 2 || dim > 3 || !n) return THX_ERR_INVALID_ARGUMENT;
  long long ne = 1;
  for (int d = 0; d < dim; ++d) {
    if (n[d] < 1) return THX_ERR_INVALID_ARGUMENT;
    ne *= n[d];
  }
  if (ne * dim > 0x7fffffffLL) return THX_ERR_INVALID_ARGUMENT;
  if (num_elements) *num_elements = (int32_t)ne;
  if (num_faces) *num_faces = (int32_t)(ne * dim);
  return THX_OK;
}

// Periodic box: element (ex,ey,ez) = ex + nx*(ey + ny*ez); faces ordered by
// normal direction then by minus element, the minus element being the one on
// the low side (the wrap face has the last element as minus side).  The
// affine map x = lo + h*(e + xi) gives J = prod h, adj(J) = diag(prod_{d'!=d} h),
// CalcOrtho normal h-scaled, lift weight 1/(w0 J).
int thx_box_geometry(int dim, int order, const int32_t *n, const double *lo, const double *hi,
                     double *jac, double *metric, int32_t *face_elem, int32_t *face_lface,
                     double *face_normal, double *face_wminus, double *face_wplus,
                     double *node_coords) {
  int32_t ne32, nf32;
  int st = thx_box_counts(dim, n, &ne32, &nf32);
  if (st) return st;
  if (order < 1 || order > 16 || !lo || !hi || !jac || !metric || !face_elem || !face_lface ||
      !face_normal || !face_wminus || !face_wplus)
    return THX_ERR_INVALID_ARGUMENT;
  const int Np = order + 1;
  const int nd = dim == 2 ? Np * Np : Np * Np * Np;
  const int nfp = dim == 2 ? Np : Np * Np;
  const int nn[3] = {n[0], n[1], dim > 2 ? n[2] : 1};
  double h[3] = {1.0, 1.0, 1.0};
  for (int d = 0; d < dim; ++d) {
    if (!(hi[d] > lo[d])) return THX_ERR_INVALID_ARGUMENT;
    h[d] = (hi[d] - lo[d]) / nn[d];
  }
  std::vector<double> x(Np), w(Np);
  thx::lgl_rule(Np, x.data(), w.data());
  const double J = dim == 2 ? h[0] * h[1] : h[0] * h[1] * h[2];
  const long long ne = ne32;
  const long long L = ne * nd;
  for (long long e = 0; e < ne; ++e) {
    const int ex = (int)(e % nn[0]), ey = (int)((e / nn[0]) % nn[1]), ez = (int)(e / (nn[0] * nn[1]));
    for (int a = 0; a < nd; ++a) {
      jac[e * nd + a] = J;
      double *M = metric + (e * nd + a) * dim * dim;
      for (int r = 0; r < dim * dim; ++r) M[r] = 0.0;
      for (int dir = 0; dir < dim; ++dir) {
        double v = 1.0;
        for (int d = 0; d < dim; ++d)
          if (d != dir) v *= h[d];
        M[dir * dim + dir] = v;
      }
      if (node_coords) {
        const int i = a % Np, j = (a / Np) % Np, k = a / (Np * Np);
        node_coords[0 * L + e * nd + a] = lo[0] + h[0] * (ex + x[i]);
        node_coords[1 * L + e * nd + a] = lo[1] + h[1] * (ey + x[j]);
        if (dim > 2) node_coords[2 * L + e * nd + a] = lo[2] + h[2] * (ez + x[k]);
      }
    }
  }
  long long f = 0;
  const double wlift = 1.0 / (w[0] * J);
  for (int dir = 0; dir < dim; ++dir)
    for (long long e = 0; e < ne; ++e) {
      int ix[3] = {(int)(e % nn[0]), (int)((e / nn[0]) % nn[1]), (int)(e / (nn[0] * nn[1]))};
      ix[dir] = (ix[dir] + 1) % nn[dir];
      face_elem[2 * f] = (int32_t)e;
      face_elem[2 * f + 1] = ix[0] + nn[0] * (ix[1] + nn[1] * ix[2]);
      face_lface[2 * f] = 2 * dir + 1;
      face_lface[2 * f + 1] = 2 * dir;
      double area = 1.0;
      for (int d = 0; d < dim; ++d)
        if (d != dir) area *= h[d];
      for (int fp = 0; fp < nfp; ++fp) {
        for (int d = 0; d < dim; ++d) face_normal[(f * nfp + fp) * dim + d] = d == dir ? area : 0.0;
        face_wminus[f * nfp + fp] = wlift;
        face_wplus[f * nfp + fp] = wlift;
      }
      ++f;
    }
  return THX_OK;
}

}  // extern "C"
