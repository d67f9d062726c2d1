// Test-only stand-in for the few MFEM types that the library's
// MFEMRHSOperator adapter (include/theseus_b200/RHSOperator.hpp) touches:
// Vector (device-readable data through Read/Write), Operator,
// TimeDependentOperator, ODESolver and RK3SSPSolver, the solver the
// reference's Simulation selects (src/Simulation.cpp:265-268).  It holds no
// MFEM code: Vector keeps its data in CUDA managed memory, so the device
// pointer Read()/Write() hand out is also readable on the host after a
// synchronisation, and RK3SSPSolver::Step is the published Shu-Osher SSP-RK3
// written with the linear combinations mfem::add forms (z = x + a y,
// z = a x + b y), evaluated on the host.
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <stdexcept>

namespace mfem {

class Vector {
 public:
  Vector() = default;
  explicit Vector(int n) { SetSize(n); }
  Vector(const Vector &) = delete;
  Vector &operator=(const Vector &) = delete;
  ~Vector() { if (d_) cudaFree(d_); }
  void SetSize(int n) {
    if (n == n_) return;
    if (d_) cudaFree(d_);
    d_ = nullptr;
    n_ = n;
    if (n > 0 && cudaMallocManaged(&d_, sizeof(double) * (size_t)n) != cudaSuccess)
      throw std::runtime_error("cudaMallocManaged failed");
  }
  int Size() const { return n_; }
  const double *Read(bool = true) const { return d_; }
  double *Write(bool = true) { return d_; }
  double *ReadWrite(bool = true) { return d_; }
  const double *HostRead() const { cudaDeviceSynchronize(); return d_; }
  double *HostWrite() { cudaDeviceSynchronize(); return d_; }
  double *HostReadWrite() { cudaDeviceSynchronize(); return d_; }
  double &operator[](int i) { return d_[i]; }
  double operator[](int i) const { return d_[i]; }

 private:
  double *d_ = nullptr;
  int n_ = 0;
};

// z = x + a y
inline void add(const Vector &x, double a, const Vector &y, Vector &z) {
  const double *xp = x.HostRead(), *yp = y.HostRead();
  double *zp = z.HostWrite();
  for (int i = 0; i < z.Size(); ++i) zp[i] = xp[i] + a * yp[i];
}
// z = a x + b y
inline void add(double a, const Vector &x, double b, const Vector &y, Vector &z) {
  const double *xp = x.HostRead(), *yp = y.HostRead();
  double *zp = z.HostWrite();
  for (int i = 0; i < z.Size(); ++i) zp[i] = a * xp[i] + b * yp[i];
}

class Operator {
 public:
  explicit Operator(int s = 0) : height(s), width(s) {}
  virtual ~Operator() = default;
  int Height() const { return height; }
  int Width() const { return width; }
  virtual void Mult(const Vector &x, Vector &y) const = 0;

 protected:
  int height, width;
};

class TimeDependentOperator : public Operator {
 public:
  explicit TimeDependentOperator(int n = 0, double t0 = 0.0) : Operator(n), t(t0) {}
  virtual void SetTime(double t_) { t = t_; }
  double GetTime() const { return t; }

 protected:
  double t;
};

class ODESolver {
 public:
  virtual ~ODESolver() = default;
  virtual void Init(TimeDependentOperator &f_) { f = &f_; }
  virtual void Step(Vector &x, double &t, double &dt) = 0;

 protected:
  TimeDependentOperator *f = nullptr;
};

class RK3SSPSolver : public ODESolver {
 public:
  void Init(TimeDependentOperator &f_) override {
    ODESolver::Init(f_);
    y.SetSize(f_.Height());
    k.SetSize(f_.Height());
  }
  void Step(Vector &x, double &t, double &dt) override {
    f->SetTime(t);
    f->Mult(x, k);
    add(x, dt, k, y);                      // y = x + dt k
    f->SetTime(t + dt);
    f->Mult(y, k);
    add(y, dt, k, y);                      // y = y + dt k
    add(3.0 / 4.0, x, 1.0 / 4.0, y, y);    // y = 3/4 x + 1/4 y
    f->SetTime(t + dt / 2);
    f->Mult(y, k);
    add(y, dt, k, y);                      // y = y + dt k
    add(1.0 / 3.0, x, 2.0 / 3.0, y, x);    // x = 1/3 x + 2/3 y
    t += dt;
  }

 private:
  Vector y, k;
};

}  // namespace mfem
