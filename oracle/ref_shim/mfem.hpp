// Stand-in for the few MFEM names that the reference's pointwise headers
// (fluxes, gas models, DGSEMIntegrator point kernels) touch, so that those
// headers compile on a machine without MFEM.  TEST INFRASTRUCTURE ONLY; it
// contains declarations and a std::vector-backed Vector, no MFEM code.
#pragma once
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <iostream>
#include <memory>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>
#define MFEM_HOST_DEVICE
#define MFEM_ABORT(msg) do { std::ostringstream s_; s_ << msg; throw std::runtime_error(s_.str()); } while (0)
#define MFEM_VERIFY(c, msg) do { if (!(c)) MFEM_ABORT(msg); } while (0)
#define MFEM_ASSERT(c, msg) do {} while (0)
namespace mfem {
using real_t = double;
inline real_t infinity() { return HUGE_VAL; }
class Vector {
  std::vector<real_t> d;
 public:
  Vector() = default;
  explicit Vector(int n) : d(n) {}
  int Size() const { return (int)d.size(); }
  void SetSize(int n) { d.resize(n); }
  real_t *GetData() { return d.data(); }
  const real_t *GetData() const { return d.data(); }
  const real_t *Read(bool = true) const { return d.data(); }
  const real_t *HostRead() const { return d.data(); }
  real_t *Write(bool = true) { return d.data(); }
  real_t *HostWrite() { return d.data(); }
  real_t *ReadWrite(bool = true) { return d.data(); }
  real_t *HostReadWrite() { return d.data(); }
  void UseDevice(bool = true) {}
  real_t &operator[](int i) { return d[i]; }
  real_t operator[](int i) const { return d[i]; }
  real_t &operator()(int i) { return d[i]; }
  real_t operator()(int i) const { return d[i]; }
  void Reciprocal() { for (auto &x : d) x = 1.0 / x; }
  Vector &operator=(real_t v) { for (auto &x : d) x = v; return *this; }
};
template <typename F> void forall(int n, F &&f) { for (int i = 0; i < n; ++i) f(i); }
template <class T> class Array {
 public:
  Array(); explicit Array(int);
  int Size() const; void SetSize(int); T &operator[](int); const T &operator[](int) const;
  T &operator()(int); Array &operator=(const T &); const T *Read(bool = true) const; const T *HostRead() const;
  T *Write(bool = true); T *HostWrite(); T *ReadWrite(bool = true); void UseDevice(bool = true) const; T Max() const;
  void Append(const T &);
};
template <class T> class Array2D { public: int NumRows() const; void GetRow(int, Array<T> &) const; T &operator()(int, int); };
class DenseMatrix { public: DenseMatrix(); explicit DenseMatrix(int); void SetSize(int); double &operator()(int, int);
  double operator()(int, int) const; void GetRow(int, Vector &) const; void Transpose(); double *Data();
  DenseMatrix &operator=(double); DenseMatrix &operator*=(double); };
struct IntegrationPoint { double x, y, z, weight; void Get(double *, int) const; };
class IntegrationRule { public: int GetNPoints() const; IntegrationPoint &IntPoint(int); const IntegrationPoint &IntPoint(int) const; };
struct Quadrature1D { enum { GaussLobatto = 1 }; };
struct Geometry { enum Type { POINT, SEGMENT, TRIANGLE, SQUARE, TETRAHEDRON, CUBE }; };
class IntegrationRules { public: IntegrationRules(int, int); const IntegrationRule &Get(int, int); };
class ElementTransformation; class FaceElementTransformations;
class ElementRestrictionOperator; class FaceRestriction; class FaceQuadratureSpace;
class Mesh; class DG_FECollection; class FiniteElementSpace; class ParFiniteElementSpace; class ParGridFunction;
enum class FaceType { Interior, Boundary };
class ParMesh { public: int GetNumFaces() const; int GetNBE() const; int GetBdrElementFaceIndex(int) const;
  const Array<int> &GetFaceIndices(FaceType) const; const Array<int> &GetBdrFaceAttributes() const;
  FaceElementTransformations *GetSharedFaceTransformationsByLocalIndex(int, bool); };
enum class ElementDofOrdering { NATIVE, LEXICOGRAPHIC };
enum class L2FaceValues { SingleValued, DoubleValued };
void CalcOrtho(const DenseMatrix &, Vector &);
}  // namespace mfem
