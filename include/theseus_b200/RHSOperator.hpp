// RHSOperator.hpp -- C++ host side of the B200 DGSEM right-hand side.
//
// Header-only classes over the C ABI of theseus_b200.h that keep the
// reference's operator interface, so a C++ caller of
//   Theseus::RHSOperator<PhysicsT>::Mult(const mfem::Vector &u, mfem::Vector &dudt)
//   (include/RHSOperator.hpp:100,172 of the reference)
// can switch to these kernels:
//
//   theseus_b200::Geometry g = theseus_b200::Geometry::PeriodicBox(3, 4, {32,32,32}, lo, hi);
//   theseus_b200::NSOperator op(g, theseus_b200::Selection{"ranocha", "hll"}, physics);
//   op.Mult(u_dev, dudt_dev, stream);           // device L-vectors, byNODES
//
// Errors surface as std::runtime_error carrying the library's status string,
// in the spirit of the reference's MFEM_VERIFY / std::invalid_argument.
//
// With THESEUS_B200_WITH_MFEM defined (and MFEM on the include path) the header
// also defines MFEMRHSOperator, an mfem::TimeDependentOperator whose Mult reads
// and writes mfem::Vector device memory -- the object an mfem::ODESolver such as
// RK3SSPSolver drives (src/Simulation.cpp:256-285,1255 of the reference).
#pragma once

#include <array>
#include <cctype>
#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "../theseus_b200.h"

namespace theseus_b200 {

inline void check(int status, const char *what) {
  if (status != THX_OK)
    throw std::runtime_error(std::string(what) + ": " + thx_status_string(status));
}

// Geometric factors in the thx_geometry layout, owned on the host.
// Boundary faces (empty: periodic) follow the reference's boundary cache:
// element and local face, outward normals, lift weights, the condition of
// each face and the condition table with its packed payloads.
struct Geometry {
  int dim = 0, order = 0, num_elements = 0, num_faces = 0;
  std::vector<double> jac, metric, face_normal, face_wminus, face_wplus, coords;
  std::vector<int32_t> face_elem, face_lface;
  std::vector<int32_t> bdr_elem, bdr_lface, bdr_bc;
  std::vector<double> bdr_normal, bdr_weight, bc_data;
  std::vector<thx_bc> bcs;

  int nodes_per_element() const { int32_t n = 0; thx_sizes(dim, order, &n, nullptr, nullptr); return n; }
  int points_per_face() const { int32_t n = 0; thx_sizes(dim, order, nullptr, &n, nullptr); return n; }
  int num_equations() const { return dim + 2; }
  // Height of the byNODES L-vector (num_equations x elements x nodes).
  long long height() const { return (long long)num_equations() * num_elements * nodes_per_element(); }

  thx_geometry view() const {
    thx_geometry g{};
    g.dim = dim; g.order = order; g.num_elements = num_elements; g.num_faces = num_faces;
    g.jac = jac.data(); g.metric = metric.data();
    g.face_elem = face_elem.data(); g.face_lface = face_lface.data();
    g.face_normal = face_normal.data(); g.face_wminus = face_wminus.data();
    g.face_wplus = face_wplus.data();
    g.num_bdr_faces = (int32_t)bdr_elem.size();
    if (g.num_bdr_faces > 0) {
      g.bdr_elem = bdr_elem.data(); g.bdr_lface = bdr_lface.data(); g.bdr_bc = bdr_bc.data();
      g.bdr_normal = bdr_normal.data(); g.bdr_weight = bdr_weight.data();
      g.num_bcs = (int32_t)bcs.size(); g.bcs = bcs.data();
      g.bc_data_len = (int32_t)bc_data.size(); g.bc_data = bc_data.data();
    }
    return g;
  }

  // Periodic Cartesian box (stands in for MFEM's mesh and geometric-factor set-up).
  static Geometry PeriodicBox(int dim, int order, std::array<int32_t, 3> n, std::array<double, 3> lo,
                              std::array<double, 3> hi, bool with_coords = false) {
    Geometry g;
    g.dim = dim;
    g.order = order;
    int32_t ne = 0, nf = 0;
    check(thx_box_counts(dim, n.data(), &ne, &nf), "thx_box_counts");
    g.num_elements = ne;
    g.num_faces = nf;
    const size_t nd = (size_t)g.nodes_per_element(), nfp = (size_t)g.points_per_face();
    g.jac.resize((size_t)ne * nd);
    g.metric.resize((size_t)ne * nd * dim * dim);
    g.face_elem.resize((size_t)nf * 2);
    g.face_lface.resize((size_t)nf * 2);
    g.face_normal.resize((size_t)nf * nfp * dim);
    g.face_wminus.resize((size_t)nf * nfp);
    g.face_wplus.resize((size_t)nf * nfp);
    if (with_coords) g.coords.resize((size_t)dim * ne * nd);
    check(thx_box_geometry(dim, order, n.data(), lo.data(), hi.data(), g.jac.data(), g.metric.data(),
                           g.face_elem.data(), g.face_lface.data(), g.face_normal.data(),
                           g.face_wminus.data(), g.face_wplus.data(),
                           with_coords ? g.coords.data() : nullptr),
          "thx_box_geometry");
    return g;
  }
};

// Volume / surface / subcell-FV numerical fluxes by the reference's selection
// strings (include/SimFactory_impl.hpp:75-128 of the reference).
inline int FluxFromString(std::string s) {
  for (auto &c : s) c = (char)std::tolower((unsigned char)c);
  if (s.empty() || s.rfind("chan", 0) == 0) return THX_FLUX_CHANDRASHEKAR;
  if (s == "ranocha") return THX_FLUX_RANOCHA;
  if (s == "piflux" || s.rfind("pi", 0) == 0) return THX_FLUX_PIROZZOLI;
  if (s == "hll") return THX_FLUX_HLL;
  if (s == "roe") return THX_FLUX_ROE;
  if (s == "llf" || s == "lfr" || s == "laxfriedrichs" || s == "lax_friedrichs" || s.rfind("lax", 0) == 0)
    return THX_FLUX_LLF;
  throw std::invalid_argument("unknown numerical flux '" + s +
                              "'; supported: Chandrashekar, Ranocha, Pirozzoli, LLF/LFR, HLL, Roe");
}

struct Selection {
  std::string volume = "chandrashekar";
  std::string surface = "";    // empty: same class as the volume flux (the reference's coupling)
  std::string subcell = "llf";
};

// Mirror of include/StabilityEstimate.hpp:38-54 of the reference.
struct StabilityEstimate {
  double advective_rate = 0.0, surface_rate = 0.0, diffusive_rate = 0.0;
  double TotalRate() const { return (advective_rate > surface_rate ? advective_rate : surface_rate) + diffusive_rate; }
};

class RHSOperator {
 public:
  RHSOperator(const Geometry &g, const thx_config &cfg) : cfg_(cfg), height_(g.height()) {
    const thx_geometry view = g.view();
    thx_handle h = nullptr;
    check(thx_create(&view, &cfg_, &h), "thx_create");
    h_.reset(h);
  }
  virtual ~RHSOperator() = default;

  long long Height() const { return height_; }
  const thx_config &Config() const { return cfg_; }

  // dudt = L(u) on device L-vectors (double for FP64, float for FP32-mixed).
  void Mult(const void *u_dev, void *dudt_dev, void *stream = nullptr) const {
    check(thx_rhs(h_.get(), u_dev, dudt_dev, stream), "thx_rhs");
  }
  // nsteps SSP-RK3 steps on the FP64 master state, in place.
  void RK3Steps(double *u_dev, double dt, int nsteps, void *stream = nullptr) const {
    check(thx_rk3_steps(h_.get(), u_dev, dt, nsteps, stream), "thx_rk3_steps");
  }
  // ncycles of the reference's clocked loop (src/Simulation.cpp:1150-1335) on
  // the FP64 state; loop_dev is a thx_time_loop in device memory (fill it
  // on the host with TimeLoopDefaults and copy it over); cfl > 0: variable dt.
  void RunTimeLoop(double *u_dev, double cfl, int ncycles, thx_time_loop *loop_dev,
                   double *dt_history_dev = nullptr, void *stream = nullptr) const {
    check(thx_rk3_time_loop(h_.get(), u_dev, cfl, ncycles, loop_dev, dt_history_dev, stream),
          "thx_rk3_time_loop");
  }
  // dudt_host[i] = L(u_host[i]) for FP64 host L-vectors; the transfers of
  // neighbouring states overlap the kernels (page-locked buffers).  Ordered on
  // `stream`: synchronise it before reading the rates.
  void MultHost(int n, const double *const *u_host, double *const *dudt_host, void *stream = nullptr) const {
    check(thx_rhs_host(h_.get(), n, u_host, dudt_host, stream), "thx_rhs_host");
  }
  StabilityEstimate EstimateStability(const double *u_dev) const {
    double dt = 0.0, r[3] = {0, 0, 0};
    check(thx_estimate_dt(h_.get(), u_dev, 1.0, &dt, r), "thx_estimate_dt");
    return {r[0], r[1], r[2]};
  }
  void BlendingCoefficients(double *alpha_dev, double *eta_dev, void *stream = nullptr) const {
    check(thx_blending_coefficients(h_.get(), alpha_dev, eta_dev, stream), "thx_blending_coefficients");
  }
  uint32_t ReadStatus(void *stream = nullptr) const {
    uint32_t f = 0;
    check(thx_read_status(h_.get(), &f, stream), "thx_read_status");
    return f;
  }
  std::string Describe() const {
    char buf[1024];
    check(thx_describe(h_.get(), buf, sizeof(buf)), "thx_describe");
    return buf;
  }

 protected:
  static thx_config MakeConfig(int flow, const Selection &sel, thx_config physics) {
    physics.flow_model = flow;
    physics.volume_flux = FluxFromString(sel.volume);
    physics.surface_flux = sel.surface.empty() ? physics.volume_flux : FluxFromString(sel.surface);
    physics.fv_flux = FluxFromString(sel.subcell);
    return physics;
  }

 private:
  struct Deleter { void operator()(thx_operator_s *h) const { if (h) thx_destroy(h); } };
  thx_config cfg_;
  long long height_;
  std::unique_ptr<thx_operator_s, Deleter> h_;
};

// The reference's runTime defaults for the time loop, with the given final
// time, fixed or first step (<= 0 with cfl > 0: from the stability
// estimate), cycle limit (<= 0: none) and output interval (<= 0: no output).
inline thx_time_loop TimeLoopDefaults(double t_final, double dt, long long max_cycles, double output_dt) {
  thx_time_loop L;
  thx_time_loop_defaults(&L);
  L.t_final = t_final;
  L.dt = dt;
  L.max_cycles = max_cycles;
  if (output_dt > 0.0) {
    L.output_dt = L.refined_output_dt = output_dt;
    L.next_output = L.t + output_dt;
  }
  return L;
}

// Default physics (the reference's runtime JSON defaults).
inline thx_config DefaultPhysics() {
  thx_config c;
  thx_config_default(&c);
  return c;
}

class EulerOperator : public RHSOperator {
 public:
  EulerOperator(const Geometry &g, const Selection &sel = {}, thx_config physics = DefaultPhysics())
      : RHSOperator(g, MakeConfig(THX_FLOW_EULER, sel, physics)) {}
};

class NSOperator : public RHSOperator {
 public:
  NSOperator(const Geometry &g, const Selection &sel = {}, thx_config physics = DefaultPhysics())
      : RHSOperator(g, MakeConfig(THX_FLOW_NAVIER_STOKES, sel, physics)) {}
};

}  // namespace theseus_b200

#ifdef THESEUS_B200_WITH_MFEM
#include "mfem.hpp"
namespace theseus_b200 {
// mfem::TimeDependentOperator front end: the drop-in replacement of
// Theseus::RHSOperatorBase for an mfem::ODESolver.  The L2 space must be
// byNODES with lexicographic element DOFs (the reference's choice,
// include/Simulation.hpp:68-69), so u is already the library's L-vector.
class MFEMRHSOperator : public mfem::TimeDependentOperator {
 public:
  explicit MFEMRHSOperator(std::shared_ptr<RHSOperator> op)
      : mfem::TimeDependentOperator((int)op->Height()), op_(std::move(op)) {}
  void Mult(const mfem::Vector &u, mfem::Vector &dudt) const override {
    op_->Mult(u.Read(), dudt.Write());
  }
  StabilityEstimate EstimateStability(const mfem::Vector &u) const {
    return op_->EstimateStability(u.Read());
  }

 private:
  std::shared_ptr<RHSOperator> op_;
};
}  // namespace theseus_b200
#endif
