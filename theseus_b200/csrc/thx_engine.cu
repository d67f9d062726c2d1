// thx_engine.cu -- batch engine: many independent cases advanced together by
// persistent kernels launched from CUDA graphs (C ABI in
// include/theseus_b200.h, "batch engine").
//
// Cases with the same (dimension, order, flow model) form a group.  A group
// owns, on the device, one argument record per case and SSP-RK3 stage (the
// same VolArgs / FaceArgs / GradArgs a one-case right-hand side uses) and the
// work lists of its persistent kernels (CTA-sized blocks of every case).  Its
// CUDA graph holds `steps_per_launch` SSP-RK3 steps of [gradient] face volume
// launches whose grids are fixed and whose work counts are read on the
// device, so admitting or retiring a case rewrites the tables between graph
// launches and never re-captures the graph.  Each case keeps its own buffers
// (allocated stream-ordered from a memory pool on the engine's set-up stream,
// so admission overlaps the running groups), which makes every result
// bit-identical to the same case run alone.
//
// The volume kernel's grid (CTAs per SM) is tuned online per group: the first
// launches try each candidate, cost = device time / work items, and the
// cheapest is kept.
#include "thx_operator.cuh"

#include <algorithm>
#include <chrono>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <tuple>
#include <vector>

using namespace thx;

namespace {

constexpr int kFaceBlock = 128;  // face points per face work item

size_t round_up(size_t n) { return (n + 255) & ~size_t(255); }

// Upper bound of the device bytes of one case (geometry counted uncompressed).
size_t case_bytes(const thx_geometry *g, const thx_config *cfg, int flow) {
  const int dim = g->dim, N = g->order + 1;
  const size_t nd = dim == 2 ? N * N : N * N * N, nfp = dim == 2 ? N : N * N;
  const size_t neq = dim + 2, ne = g->num_elements, nf = g->num_faces, L = ne * nd;
  const bool mixed = cfg->precision == THX_PRECISION_FP32_MIXED;
  const bool ns = flow == THX_FLOW_NAVIER_STOKES;
  const size_t s = mixed ? 4 : 8, gs = mixed ? 12 : 8;  // working / geometry element bytes
  size_t b = 0;
  b += round_up(L * neq * 8) * 2;                             // master state, stage copy
  if (mixed) b += round_up(L * neq * 4);                      // FP32 working copy
  b += round_up(nf * nfp * neq * s);                          // face fluxes
  if (ns) b += round_up((size_t)dim * (neq - 1) * L * s);     // viscous flux
  b += round_up(L * gs) + round_up(L * dim * dim * gs);       // J, metric
  b += round_up(nf * nfp * dim * gs) + 2 * round_up(nf * nfp * gs);  // normals, lift weights
  b += round_up(nf * 2 * 4) * 2 + round_up(ne * 2 * dim * 4); // connectivity
  b += round_up(ne * 8) * 2 + 4096;                           // alpha, eta, operators, status
  return b;
}

struct EngineCase {
  int64_t id = 0;
  thx_operator_s *h = nullptr;
  double *u = nullptr;     // FP64 master state
  double dt = 0.0;
  int steps_left = 0;
  size_t bytes = 0;
  cudaEvent_t done = nullptr;
  cudaEvent_t ready = nullptr;  // recorded on the set-up stream after the case's uploads
  bool finished = false;   // all steps enqueued; done recorded
  bool fetching = false;   // a fetch is copying the result
  // the case's kernel arguments of SSP-RK3 stages 1..3 (VolArgs, FaceArgs,
  // GradArgs per stage), packed once at admission: they do not change while
  // the case runs, so rewriting a group's tables is a copy
  std::vector<unsigned char> packed;
};

struct EngineBase {
  virtual ~EngineBase() {}
  virtual int admit(const thx_geometry *g, const thx_case *c, const double *u0, int64_t *id) = 0;
  virtual int advance() = 0;
  virtual int poll(int64_t *ids, int cap, int *count) = 0;
  virtual int fetch(int64_t id, double *u_host) = 0;
  virtual void stats(thx_engine_stats *st) = 0;
  virtual int groups(thx_engine_group *out, int cap) = 0;
};

template <typename R>
struct Group {
  int dim = 0, N = 0;
  bool ns = false;
  int epb = 1, nfp = 1;  // epb: elements per CTA of the current tables
  int epb_full = 1, epb_half = 0;
  std::vector<EngineCase *> cases;
  // admitted cases whose set-up may still run on the set-up stream: they join
  // `cases` once their ready event has completed, so a group's launches never
  // wait on the set-up stream
  std::vector<EngineCase *> pending;
  bool dirty = true;
  cudaStream_t stream = nullptr;
  // device tables: [stage 1..3][cap] argument records, work lists, counts
  VolArgs<R> *dvol = nullptr;
  FaceArgs<R> *dface = nullptr;
  GradArgs<R> *dgrad = nullptr;
  BatchWork *dwv = nullptr, *dwf = nullptr;
  int *dcount = nullptr;  // [0] volume/gradient work, [1] face work
  int cap_cases = 0, cap_wv = 0, cap_wf = 0;
  // pinned staging of the tables, a ring of three: with at most two launches
  // queued, the copies out of the slot about to be refilled have finished,
  // so a rewrite does not wait for the GPU (with the engine lock held)
  static constexpr int kStaging = 3;
  unsigned char *staging[kStaging] = {nullptr, nullptr, nullptr};
  size_t staging_bytes[kStaging] = {0, 0, 0};
  cudaEvent_t staged[kStaging] = {nullptr, nullptr, nullptr};
  int stage_pos = 0;
  std::vector<unsigned char *> retired;  // outgrown staging buffers
  int nwv = 0, nwf = 0;
  long long nodes = 0;  // solution nodes of the cases in the tables
  // kernels and graph
  VolBatchLaunch<R> volb = nullptr, volb_half = nullptr;
  FaceBatchLaunch<R> faceb = nullptr;
  GradBatchLaunch<R> gradb = nullptr, gradb_half = nullptr;
  cudaGraphExec_t exec = nullptr;
  // grids of the persistent kernels in the captured graph
  struct Grids {
    int vol = 0, face = 0, grad = 0;
    bool half = false;  // half-size CTAs for the volume and gradient kernels
    bool operator==(const Grids &o) const {
      return vol == o.vol && face == o.face && grad == o.grad && half == o.half;
    }
  };
  Grids exec_grids;
  // launches in flight: at most two per group, so that newly admitted cases
  // join after a short queue
  cudaEvent_t ring[2] = {nullptr, nullptr};
  int ring_pos = 0;
  // online tuning: coordinate search over the elements per CTA (full or
  // half-size CTAs), then the volume grid, the face grid and (Navier-Stokes)
  // the gradient grid, each over a few multiples of the SM count; cost =
  // device time of a launch / (case nodes x steps); every tuning launch
  // advances real cases
  Grids best;
  double best_cost = -1.0;
  int tune_axis = 0, tune_index = 0;  // 0 CTA size, 1 volume, 2 face, 3 gradient; 4: done
  int tune_rep = 0;                   // timings taken of the current candidate
  bool members_changed = true;        // cases joined or left since the last launch
  int unsteady = 0;                   // candidate launches deferred in a row
  bool tuned = false;
  Grids timing_grids;
  cudaEvent_t t0 = nullptr, t1 = nullptr;
  bool timing = false;
  long long timing_work = 0;
};

template <typename R>
class Engine final : public EngineBase {
  static constexpr size_t kPackedStage = sizeof(VolArgs<R>) + sizeof(FaceArgs<R>) + sizeof(GradArgs<R>);

 public:
  Engine(const thx_config &cfg, size_t budget, int k) : cfg_(cfg), budget_(budget), k_(k) {}

  int init() {
    if (cudaGetDevice(&device_) != cudaSuccess) return THX_ERR_NO_DEVICE;
    if (cudaDeviceGetAttribute(&sms_, cudaDevAttrMultiProcessorCount, device_) != cudaSuccess)
      return THX_ERR_CUDA;
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device_;
    THX_CU(cudaMemPoolCreate(&pool_, &props));
    uint64_t keep = ~uint64_t(0);  // keep freed memory in the pool
    cudaMemPoolSetAttribute(pool_, cudaMemPoolAttrReleaseThreshold, &keep);
    // set-up work (uploads, the working-copy conversion) at the highest
    // priority: its small kernels take the first free CTA slots between the
    // persistent batched kernels
    int least = 0, greatest = 0;
    THX_CU(cudaDeviceGetStreamPriorityRange(&least, &greatest));
    THX_CU(cudaStreamCreateWithPriority(&setup_, cudaStreamNonBlocking, greatest));
    if (ring_.init(size_t(256) << 20) != THX_OK) return THX_ERR_OUT_OF_MEMORY;
    return THX_OK;
  }

  ~Engine() override {
    for (auto &kv : groups_) {
      Group<R> &G = *kv.second;
      if (G.stream) cudaStreamSynchronize(G.stream);
    }
    if (setup_) cudaStreamSynchronize(setup_);
    for (auto &kv : cases_) release(kv.second.get(), false);
    cases_.clear();
    for (auto &kv : groups_) destroy_group(*kv.second);
    if (setup_) cudaStreamSynchronize(setup_);
    for (auto &kv : donors_) {
      op_free(kv.second);
      delete kv.second;
    }
    donors_.clear();
    if (setup_) {
      cudaStreamSynchronize(setup_);
      cudaStreamDestroy(setup_);
    }
    for (Bounce &b : bounce_) cudaFreeHost(b.ptr);
    if (pool_) cudaMemPoolDestroy(pool_);
  }

  // Validation and the budget reservation happen under the engine lock; the
  // operator set-up (host packing, stream-ordered allocations and uploads on
  // the set-up stream) runs outside it, so one thread can admit while another
  // advances the running groups.
  int admit(const thx_geometry *g, const thx_case *c, const double *u0, int64_t *id) override {
    if (!g || !c || !u0 || !id) return THX_ERR_INVALID_ARGUMENT;
    if (c->nsteps < 0 || !(c->dt > 0.0) || !(c->mu >= 0.0) ||
        (c->flow_model != THX_FLOW_EULER && c->flow_model != THX_FLOW_NAVIER_STOKES) ||
        (c->flow_model == THX_FLOW_NAVIER_STOKES && !(c->Pr > 0.0)))
      return THX_ERR_INVALID_ARGUMENT;
    if (g->dim < 2 || g->dim > 3 || g->num_elements <= 0 || g->num_faces < 0 || !g->jac ||
        !g->metric || (g->num_faces > 0 && (!g->face_elem || !g->face_lface || !g->face_normal ||
                                            !g->face_wminus || !g->face_wplus)))
      return THX_ERR_INVALID_ARGUMENT;
    if (g->order + 1 < 3 || g->order + 1 > 6) return THX_ERR_UNSUPPORTED;
    if (g->num_bdr_faces > 0) return THX_ERR_UNSUPPORTED;  // batched kernels: periodic meshes
    const size_t bytes = case_bytes(g, &cfg_, c->flow_model);
    const double t0 = now();
    {
      std::lock_guard<std::mutex> lock(mu_);
      t_lock_ += now() - t0;
      if (bytes_ + bytes > budget_) return THX_ERR_BUSY;
      bytes_ += bytes;  // reserved
    }
    const double t1 = now();
    auto unreserve = [&](int st) {
      std::lock_guard<std::mutex> lock(mu_);
      bytes_ -= bytes;
      return st;
    };
    thx_config cc = cfg_;
    cc.flow_model = c->flow_model;
    cc.mu = c->mu;
    cc.Pr = c->Pr;
    for (int k = 0; k < 5; ++k) cc.state_offset[k] = c->state_offset[k];
    // cases naming the same mesh share one device copy of its geometry
    const thx_operator_s *donor = nullptr;
    if (c->geometry_key != 0) {
      std::lock_guard<std::mutex> dl(donor_mu_);
      auto it = donors_.find(c->geometry_key);
      if (it != donors_.end()) {
        donor = it->second;
      } else {
        thx_operator_s *d = new (std::nothrow) thx_operator_s();
        if (!d) return unreserve(THX_ERR_OUT_OF_MEMORY);
        d->device = device_;
        d->pool = pool_;
        d->setup_stream = setup_;
        d->ring = &ring_;
        const int dst = op_create(g, &cc, d, nullptr);
        if (dst) {
          op_free(d);
          delete d;
          return unreserve(dst);
        }
        donors_[c->geometry_key] = d;
        donor = d;
      }
    }
    auto ec = std::make_unique<EngineCase>();
    thx_operator_s *h = new (std::nothrow) thx_operator_s();
    if (!h) return unreserve(THX_ERR_OUT_OF_MEMORY);
    h->device = device_;
    h->pool = pool_;
    h->setup_stream = setup_;
    h->ring = &ring_;
    ec->h = h;
    auto fail = [&](int st) {
      op_free(h);
      delete h;
      ec->h = nullptr;
      if (ec->done) cudaEventDestroy(ec->done);
      if (ec->ready) cudaEventDestroy(ec->ready);
      ec->done = ec->ready = nullptr;
      return unreserve(st);
    };
    int st = op_create(g, &cc, h, nullptr, donor);
    if (st) return fail(st);
    const size_t n = (size_t)h->L * h->neq;
    if ((st = alloc(h, &ec->u, n)) || (st = alloc(h, &h->y, n)) ||
        (h->mixed && (st = alloc(h, &h->yf, n))))
      return fail(st);
    ec->dt = c->dt;
    ec->packed.resize(3 * kPackedStage);
    for (int stage = 1; stage <= 3; ++stage) {
      VolArgs<R> va;
      FaceArgs<R> fa;
      GradArgs<R> ga;
      const R *in;
      if constexpr (IsF32<R>::value) in = h->yf;
      else in = stage == 1 ? ec->u : h->y;
      op_args<R>(h, in, nullptr, stage, ec->dt, ec->u, h->y, h->yf, ga, fa, va);
      unsigned char *pk = ec->packed.data() + (size_t)(stage - 1) * kPackedStage;
      std::memcpy(pk, &va, sizeof(va));
      std::memcpy(pk + sizeof(va), &fa, sizeof(fa));
      std::memcpy(pk + sizeof(va) + sizeof(fa), &ga, sizeof(ga));
    }
    const double t2 = now();
    if (ring_.copy(ec->u, u0, n * sizeof(double), setup_) != THX_OK ||
        (h->mixed && upload_working_copy(h, u0) != THX_OK) ||
        cudaEventCreateWithFlags(&ec->done, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&ec->ready, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventRecord(ec->ready, setup_) != cudaSuccess) {
      cudaGetLastError();
      return fail(THX_ERR_CUDA);
    }
    const double t3 = now();
    std::lock_guard<std::mutex> lock(mu_);
    t_lock_ += now() - t3;
    t_setup_ += t2 - t1;
    t_copy_ += t3 - t2;
    Group<R> *G = nullptr;
    if ((st = group_for(h, &G))) {
      ec->bytes = bytes;
      release(ec.get(), true);
      return st;
    }
    ec->id = next_id_++;
    ec->steps_left = c->nsteps;
    ec->bytes = bytes;
    G->pending.push_back(ec.get());
    *id = ec->id;
    cases_[ec->id] = std::move(ec);
    return THX_OK;
  }

  // The FP32 working copy of an admitted case's initial state, narrowed on
  // the host exactly as the to_working kernel narrows it, (float)(u - offset),
  // with its FP64 positivity check, and uploaded through the ring: the
  // set-up stream holds no kernel, whose CTAs would wait for the persistent
  // kernels of the running groups to leave an SM.
  int upload_working_copy(thx_operator_s *h, const double *u0) {
    const long long L = h->L;
    const int neq = h->neq, dim = h->dim;
    thread_local std::vector<float> wf;
    wf.resize((size_t)L * neq);
    for (int k = 0; k < neq; ++k) {
      const double o = h->off.v[k];
      const double *src = u0 + (size_t)k * L;
      float *dst = wf.data() + (size_t)k * L;
      for (long long i = 0; i < L; ++i) dst[i] = (float)(src[i] - o);
    }
    bool bad = false;
    const double gm1 = h->g64.gm1;
    for (long long i = 0; i < L && !bad; ++i) {
      double m2 = 0.0;
      for (int d = 0; d < dim; ++d) m2 += u0[(size_t)(1 + d) * L + i] * u0[(size_t)(1 + d) * L + i];
      const double rho = u0[i];
      const double p = gm1 * (u0[(size_t)(dim + 1) * L + i] - 0.5 * m2 / rho);
      bad = !(rho > 0.0 && p > 0.0);
    }
    int st = ring_.copy(h->yf, wf.data(), wf.size() * sizeof(float), setup_);
    if (!st && bad) {
      static const unsigned flag = STATUS_NONPOSITIVE;
      st = ring_.copy(h->status, &flag, sizeof(flag), setup_);
    }
    return st;
  }

  int advance() override {
    std::lock_guard<std::mutex> lock(mu_);
    const double t0 = now();
    ++n_advance_;
    for (auto &kv : groups_) {
      int st = advance_group(*kv.second);
      if (st) return st;
    }
    t_advance_ += now() - t0;
    return THX_OK;
  }

  int poll(int64_t *ids, int cap, int *count) override {
    std::lock_guard<std::mutex> lock(mu_);
    if (!count || (cap > 0 && !ids)) return THX_ERR_INVALID_ARGUMENT;
    int n = 0;
    for (auto &kv : cases_) {
      EngineCase *c = kv.second.get();
      if (!c->finished || c->fetching || n >= cap) continue;
      const cudaError_t q = cudaEventQuery(c->done);
      if (q == cudaSuccess) ids[n++] = c->id;
      else if (q != cudaErrorNotReady) return cuda_failed(q, "cudaEventQuery(case done)");
    }
    *count = n;
    return THX_OK;
  }

  // The copy to the host runs outside the engine lock, so that fetching one
  // case does not hold up advancing the others.
  int fetch(int64_t id, double *u_host) override {
    EngineCase *c = nullptr;
    size_t n = 0;
    {
      std::lock_guard<std::mutex> lock(mu_);
      auto it = cases_.find(id);
      if (it == cases_.end() || !u_host) return THX_ERR_INVALID_ARGUMENT;
      c = it->second.get();
      if (!c->finished || c->fetching) return THX_ERR_BUSY;
      c->fetching = true;
      n = (size_t)c->h->L * c->h->neq;
    }
    const double t0 = now();
    // through a pinned bounce buffer (a device-to-pageable copy would take the
    // driver's slow path)
    const size_t bytes = n * sizeof(double);
    Bounce b = take_bounce(bytes);
    cudaStream_t fs = nullptr;
    cudaError_t e = b.ptr ? cudaStreamCreateWithFlags(&fs, cudaStreamNonBlocking) : cudaErrorMemoryAllocation;
    if (e == cudaSuccess) e = cudaStreamWaitEvent(fs, c->done, 0);
    if (e == cudaSuccess) e = cudaMemcpyAsync(b.ptr, c->u, bytes, cudaMemcpyDeviceToHost, fs);
    if (e == cudaSuccess) e = cudaStreamSynchronize(fs);
    if (e == cudaSuccess) std::memcpy(u_host, b.ptr, bytes);
    if (fs) cudaStreamDestroy(fs);
    give_bounce(b);
    std::lock_guard<std::mutex> lock(mu_);
    t_fetch_ += now() - t0;
    if (e != cudaSuccess) {
      c->fetching = false;
      return cuda_failed(e, "result copy");
    }
    release(c, true);
    cases_.erase(id);
    ++done_;
    return THX_OK;
  }

  int groups(thx_engine_group *out, int cap) override {
    std::lock_guard<std::mutex> lock(mu_);
    int n = 0;
    for (auto &kv : groups_) {
      Group<R> &G = *kv.second;
      if (n < cap) {
        thx_engine_group &o = out[n];
        o.dim = G.dim;
        o.order = G.N - 1;
        o.navier_stokes = G.ns ? 1 : 0;
        o.active_cases = (int32_t)(G.cases.size() + G.pending.size());
        o.tuned = G.tuned ? 1 : 0;
        o.volume_grid = G.best.vol;
        o.face_grid = G.best.face;
        o.gradient_grid = G.ns ? G.best.grad : 0;
        o.elements_per_block = G.best.half ? G.epb_half : G.epb_full;
        o.best_cost_ms = G.best_cost;
      }
      ++n;
    }
    return n;
  }

  void stats(thx_engine_stats *st) override {
    std::lock_guard<std::mutex> lock(mu_);
    st->active_cases = (int32_t)cases_.size();
    st->groups = (int32_t)groups_.size();
    st->bytes_in_use = (int64_t)bytes_;
    st->launches = launches_;
    st->cases_done = done_;
    st->admit_lock_s = t_lock_;
    st->admit_setup_s = t_setup_;
    st->admit_copy_s = t_copy_;
    st->advance_s = t_advance_;
    st->fetch_copy_s = t_fetch_;
    uint64_t v = 0;
    st->pool_reserved_bytes =
        cudaMemPoolGetAttribute(pool_, cudaMemPoolAttrReservedMemCurrent, &v) == cudaSuccess ? (int64_t)v : -1;
    v = 0;
    st->pool_used_bytes =
        cudaMemPoolGetAttribute(pool_, cudaMemPoolAttrUsedMemCurrent, &v) == cudaSuccess ? (int64_t)v : -1;
    st->advance_calls = n_advance_;
    st->advance_tables_s = t_tables_;
    st->advance_launch_s = t_launch_;
    st->table_bytes = table_bytes_;
    ring_.times(&st->ring_wait_s, &st->ring_copy_s);
  }

 private:
  using Key = std::tuple<int, int, bool>;

  struct Bounce {
    unsigned char *ptr = nullptr;
    size_t size = 0;
  };
  Bounce take_bounce(size_t bytes) {
    {
      std::lock_guard<std::mutex> lock(bounce_mu_);
      for (size_t i = 0; i < bounce_.size(); ++i)
        if (bounce_[i].size >= bytes) {
          Bounce b = bounce_[i];
          bounce_.erase(bounce_.begin() + i);
          return b;
        }
    }
    Bounce b;
    b.size = std::max(bytes, size_t(8) << 20);
    if (cudaHostAlloc((void **)&b.ptr, b.size, cudaHostAllocDefault) != cudaSuccess) {
      cudaGetLastError();
      b.ptr = nullptr;
    }
    return b;
  }
  void give_bounce(const Bounce &b) {
    if (!b.ptr) return;
    std::lock_guard<std::mutex> lock(bounce_mu_);
    bounce_.push_back(b);
  }

  template <typename T>
  int alloc(thx_operator_s *h, T **p, size_t n) {
    const cudaError_t e = cudaMallocFromPoolAsync((void **)p, n * sizeof(T), pool_, setup_);
    if (e != cudaSuccess) {
      *p = nullptr;
      return cuda_failed(e, "cudaMallocFromPoolAsync(case state)", THX_ERR_OUT_OF_MEMORY);
    }
    h->allocs.push_back(*p);
    return THX_OK;
  }

  // free a case's buffers after its last work (stream-ordered on set-up)
  void release(EngineCase *c, bool account) {
    if (c->done) cudaStreamWaitEvent(setup_, c->done, 0);
    if (c->h) {
      op_free(c->h);
      delete c->h;
      c->h = nullptr;
    }
    if (c->done) cudaEventDestroy(c->done);
    c->done = nullptr;
    if (c->ready) cudaEventDestroy(c->ready);
    c->ready = nullptr;
    if (account) bytes_ -= c->bytes;
  }

  int group_for(thx_operator_s *h, Group<R> **out) {
    const Key key(h->dim, h->N, h->ns);
    auto it = groups_.find(key);
    if (it != groups_.end()) {
      *out = it->second.get();
      return THX_OK;
    }
    auto G = std::make_unique<Group<R>>();
    G->dim = h->dim;
    G->N = h->N;
    G->ns = h->ns;
    G->nfp = h->nfp;
    const int vk = (cfg_.volume_flux == THX_FLUX_CHANDRASHEKAR) ? VOL_CHANDRASHEKAR
                 : (cfg_.volume_flux == THX_FLUX_RANOCHA)     ? VOL_RANOCHA
                 : (cfg_.volume_flux == THX_FLUX_PIROZZOLI)   ? VOL_PIROZZOLI
                                                              : VOL_CENTRAL;
    const int ns = h->ns ? 1 : 0;
    pick_kernels(*G, vk, ns);
    if (!G->volb || !G->faceb || !G->gradb) return THX_ERR_UNSUPPORTED;
    if (G->epb_half > 0 && (!G->volb_half || !G->gradb_half)) return THX_ERR_UNSUPPORTED;
    G->epb = G->epb_full;
    if (G->volb(nullptr, nullptr, nullptr, 0, nullptr, 1) != cudaSuccess ||
        G->gradb(nullptr, nullptr, nullptr, 0, nullptr, 1) != cudaSuccess ||
        (G->epb_half > 0 && (G->volb_half(nullptr, nullptr, nullptr, 0, nullptr, 1) != cudaSuccess ||
                             G->gradb_half(nullptr, nullptr, nullptr, 0, nullptr, 1) != cudaSuccess))) {
      cudaGetLastError();
      return THX_ERR_CUDA;
    }
    if (cudaStreamCreateWithFlags(&G->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&G->staged[0], cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&G->staged[1], cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&G->staged[2], cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreate(&G->t0) != cudaSuccess || cudaEventCreate(&G->t1) != cudaSuccess ||
        cudaEventCreateWithFlags(&G->ring[0], cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&G->ring[1], cudaEventDisableTiming) != cudaSuccess) {
      cudaGetLastError();
      return THX_ERR_CUDA;
    }
    G->best.vol = 4 * sms_;
    G->best.face = 8 * sms_;
    G->best.grad = 2 * sms_;
    G->tune_axis = next_axis(*G, 0);
    *out = G.get();
    groups_[key] = std::move(G);
    return THX_OK;
  }

  void pick_kernels(Group<R> &G, int vk, int ns);

  void destroy_group(Group<R> &G) {
    if (G.stream) cudaStreamSynchronize(G.stream);
    if (G.exec) cudaGraphExecDestroy(G.exec);
    cudaFree(G.dvol);
    cudaFree(G.dface);
    cudaFree(G.dgrad);
    cudaFree(G.dwv);
    cudaFree(G.dwf);
    cudaFree(G.dcount);
    for (int i = 0; i < Group<R>::kStaging; ++i) {
      if (G.staging[i]) cudaFreeHost(G.staging[i]);
      if (G.staged[i]) cudaEventDestroy(G.staged[i]);
    }
    for (unsigned char *p : G.retired) cudaFreeHost(p);
    if (G.t0) cudaEventDestroy(G.t0);
    if (G.t1) cudaEventDestroy(G.t1);
    for (cudaEvent_t ev : G.ring)
      if (ev) cudaEventDestroy(ev);
    if (G.stream) cudaStreamDestroy(G.stream);
  }

  // Rewrite the group's argument tables and work lists (between launches).
  int upload_tables(Group<R> &G) {
    const int nc = (int)G.cases.size();
    int nwv = 0, nwf = 0;
    for (EngineCase *c : G.cases) {
      nwv += (c->h->ne + G.epb - 1) / G.epb;
      nwf += (int)(((long long)c->h->nf * G.nfp + kFaceBlock - 1) / kFaceBlock);
    }
    bool grow = nc > G.cap_cases || nwv > G.cap_wv || nwf > G.cap_wf;
    if (grow) {
      // Stream-ordered reallocation on the group's stream: the old tables are
      // freed after the launches in flight that read them, and nothing here
      // waits for the device (cudaMalloc/cudaFree would synchronise it with
      // every other group's launches).  A graph in flight is released by the
      // runtime when it completes.
      auto grow_to = [](int need, int have) { return std::max(need, std::max(64, 2 * have)); };
      const int cc = nc > G.cap_cases ? grow_to(nc, G.cap_cases) : G.cap_cases;
      const int cv = nwv > G.cap_wv ? grow_to(nwv, G.cap_wv) : G.cap_wv;
      const int cf = nwf > G.cap_wf ? grow_to(nwf, G.cap_wf) : G.cap_wf;
      void *old[5] = {G.dvol, G.dface, G.dgrad, G.dwv, G.dwf};
      G.dvol = nullptr; G.dface = nullptr; G.dgrad = nullptr; G.dwv = nullptr; G.dwf = nullptr;
      if (G.exec) {
        cudaGraphExecDestroy(G.exec);
        G.exec = nullptr;
      }
      for (void *q : old)
        if (q) cudaFreeAsync(q, G.stream);
      auto get = [&](void **q, size_t bytes) {
        return cudaMallocFromPoolAsync(q, bytes, pool_, G.stream) == cudaSuccess;
      };
      if (!get((void **)&G.dvol, sizeof(VolArgs<R>) * 3 * cc) ||
          !get((void **)&G.dface, sizeof(FaceArgs<R>) * 3 * cc) ||
          !get((void **)&G.dgrad, sizeof(GradArgs<R>) * 3 * cc) ||
          !get((void **)&G.dwv, sizeof(BatchWork) * cv) || !get((void **)&G.dwf, sizeof(BatchWork) * cf) ||
          (!G.dcount && !get((void **)&G.dcount, sizeof(int) * 2))) {
        G.cap_cases = G.cap_wv = G.cap_wf = 0;
        return cuda_failed(cudaGetLastError(), "cudaMallocFromPoolAsync(group tables)", THX_ERR_OUT_OF_MEMORY);
      }
      G.cap_cases = cc;
      G.cap_wv = cv;
      G.cap_wf = cf;
    }
    const size_t bv = sizeof(VolArgs<R>) * 3 * nc, bf = sizeof(FaceArgs<R>) * 3 * nc;
    const size_t bg = sizeof(GradArgs<R>) * 3 * nc;
    const size_t bw = sizeof(BatchWork) * (size_t)(nwv + nwf);
    const size_t need = bv + bf + bg + bw + 2 * sizeof(int) + 64;
    const int slot = G.stage_pos;
    THX_CU(cudaEventSynchronize(G.staged[slot]));  // this slot's last copies are done
    if (need > G.staging_bytes[slot]) {
      // cudaFreeHost would synchronise the device: the outgrown buffer is
      // kept until the group is destroyed (at most the final size again)
      if (G.staging[slot]) G.retired.push_back(G.staging[slot]);
      G.staging[slot] = nullptr;
      G.staging_bytes[slot] = std::max(need, std::max(size_t(1) << 20, 2 * G.staging_bytes[slot]));
      const cudaError_t e =
          cudaHostAlloc((void **)&G.staging[slot], G.staging_bytes[slot], cudaHostAllocDefault);
      if (e != cudaSuccess) {
        G.staging_bytes[slot] = 0;
        return cuda_failed(e, "cudaHostAlloc(table staging)", THX_ERR_OUT_OF_MEMORY);
      }
    }
    unsigned char *stg = G.staging[slot];
    VolArgs<R> *hv = reinterpret_cast<VolArgs<R> *>(stg);
    FaceArgs<R> *hf = reinterpret_cast<FaceArgs<R> *>(stg + bv);
    GradArgs<R> *hg = reinterpret_cast<GradArgs<R> *>(stg + bv + bf);
    BatchWork *hw = reinterpret_cast<BatchWork *>(stg + bv + bf + bg);
    int *hc = reinterpret_cast<int *>(stg + bv + bf + bg + bw);
    int wv = 0, wf = 0;
    for (int i = 0; i < nc; ++i) {
      EngineCase *c = G.cases[i];
      thx_operator_s *h = c->h;
      for (int stage = 1; stage <= 3; ++stage) {
        const int j = (stage - 1) * nc + i;
        const unsigned char *pk = c->packed.data() + (size_t)(stage - 1) * kPackedStage;
        std::memcpy(&hv[j], pk, sizeof(VolArgs<R>));
        std::memcpy(&hf[j], pk + sizeof(VolArgs<R>), sizeof(FaceArgs<R>));
        std::memcpy(&hg[j], pk + sizeof(VolArgs<R>) + sizeof(FaceArgs<R>), sizeof(GradArgs<R>));
      }
      const int nb = (h->ne + G.epb - 1) / G.epb;
      for (int b = 0; b < nb; ++b) hw[wv++] = BatchWork{i, b};
    }
    for (int i = 0; i < nc; ++i) {
      thx_operator_s *h = G.cases[i]->h;
      const int nb = (int)(((long long)h->nf * G.nfp + kFaceBlock - 1) / kFaceBlock);
      for (int b = 0; b < nb; ++b) hw[nwv + wf++] = BatchWork{i, b};
    }
    hc[0] = nwv;
    hc[1] = nwf;
    // the argument records of stage s start at s*nc; the graph indexes
    // tables by capacity, so place each stage block at s*cap
    for (int stage = 0; stage < 3; ++stage) {
      if (cudaMemcpyAsync(G.dvol + (size_t)stage * G.cap_cases, hv + (size_t)stage * nc,
                          sizeof(VolArgs<R>) * nc, cudaMemcpyHostToDevice, G.stream) != cudaSuccess ||
          cudaMemcpyAsync(G.dface + (size_t)stage * G.cap_cases, hf + (size_t)stage * nc,
                          sizeof(FaceArgs<R>) * nc, cudaMemcpyHostToDevice, G.stream) != cudaSuccess ||
          cudaMemcpyAsync(G.dgrad + (size_t)stage * G.cap_cases, hg + (size_t)stage * nc,
                          sizeof(GradArgs<R>) * nc, cudaMemcpyHostToDevice, G.stream) != cudaSuccess)
        return cuda_failed(cudaGetLastError(), "argument table upload");
    }
    if ((nwv && cudaMemcpyAsync(G.dwv, hw, sizeof(BatchWork) * nwv, cudaMemcpyHostToDevice, G.stream) != cudaSuccess) ||
        (nwf && cudaMemcpyAsync(G.dwf, hw + nwv, sizeof(BatchWork) * nwf, cudaMemcpyHostToDevice, G.stream) != cudaSuccess) ||
        cudaMemcpyAsync(G.dcount, hc, sizeof(int) * 2, cudaMemcpyHostToDevice, G.stream) != cudaSuccess ||
        cudaEventRecord(G.staged[slot], G.stream) != cudaSuccess)
      return cuda_failed(cudaGetLastError(), "work list upload");
    table_bytes_ += (int64_t)(bv + bf + bg + bw + 2 * sizeof(int));
    G.stage_pos = (slot + 1) % Group<R>::kStaging;
    G.nwv = nwv;
    G.nodes = 0;
    for (EngineCase *c : G.cases) G.nodes += c->h->L;
    G.nwf = nwf;
    G.dirty = false;
    return THX_OK;
  }

  int capture(Group<R> &G, const typename Group<R>::Grids &gr) {
    if (G.exec) {
      cudaGraphExecDestroy(G.exec);
      G.exec = nullptr;
    }
    const int grid = gr.vol, gf = gr.face, gg = gr.grad;
    const VolBatchLaunch<R> volb = gr.half ? G.volb_half : G.volb;
    const GradBatchLaunch<R> gradb = gr.half ? G.gradb_half : G.gradb;
    cudaGraph_t graph = nullptr;
    THX_CU(cudaStreamBeginCapture(G.stream, cudaStreamCaptureModeRelaxed));
    cudaError_t e = cudaSuccess;
    for (int step = 0; step < k_ && e == cudaSuccess; ++step)
      for (int stage = 0; stage < 3 && e == cudaSuccess; ++stage) {
        const size_t o = (size_t)stage * G.cap_cases;
        if (G.ns) e = gradb(G.dgrad + o, G.dwv, G.dcount, gg, G.stream, 0);
        if (e == cudaSuccess) e = G.faceb(G.dface + o, G.dwf, G.dcount + 1, gf, G.stream, 0);
        if (e == cudaSuccess) e = volb(G.dvol + o, G.dwv, G.dcount, grid, G.stream, 0);
      }
    const cudaError_t ee = cudaStreamEndCapture(G.stream, &graph);
    if (e != cudaSuccess || ee != cudaSuccess || !graph) {
      if (graph) cudaGraphDestroy(graph);
      return e != cudaSuccess ? cuda_failed(e, "batched launch under capture")
                              : cuda_failed(ee, "cudaStreamEndCapture");
    }
    e = cudaGraphInstantiate(&G.exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) {
      G.exec = nullptr;
      return cuda_failed(e, "cudaGraphInstantiate");
    }
    G.exec_grids = gr;
    return THX_OK;
  }

  // candidate `index` on the current tuning axis (false when the axis is done)
  static int axis_size(const Group<R> &G, int axis) {
    if (axis == 0) return G.epb_half > 0 ? 2 : 0;
    if (axis == 3) return G.ns ? 3 : 0;
    return 3;
  }
  bool tune_candidate(const Group<R> &G, int index, typename Group<R>::Grids &out) const {
    static const int vol_m[] = {1, 2, 4}, face_m[] = {4, 8, 16}, grad_m[] = {1, 2, 4};
    if (index >= axis_size(G, G.tune_axis)) return false;
    out = G.best;
    if (G.tune_axis == 0) out.half = index == 1;
    else if (G.tune_axis == 1) out.vol = vol_m[index] * sms_;
    else if (G.tune_axis == 2) out.face = face_m[index] * sms_;
    else out.grad = grad_m[index] * sms_;
    return true;
  }
  // the next axis with candidates (4: the search is done)
  static int next_axis(const Group<R> &G, int axis) {
    while (axis < 4 && axis_size(G, axis) == 0) ++axis;
    return axis;
  }

  // collect the timing of the previous tuning launch, if it has finished
  void collect_timing(Group<R> &G) {
    if (!G.timing) return;
    if (cudaEventQuery(G.t1) != cudaSuccess) {
      cudaGetLastError();
      return;
    }
    float ms = 0.f;
    G.timing = false;
    if (cudaEventElapsedTime(&ms, G.t0, G.t1) == cudaSuccess && G.timing_work > 0) {
      const double c = ms / (double)G.timing_work;
      if (G.best_cost < 0.0 || c < G.best_cost) {
        G.best_cost = c;
        G.best = G.timing_grids;
      }
    }
    // every candidate is timed on two launches; the better one counts
    if (++G.tune_rep < 2) return;
    G.tune_rep = 0;
    if (++G.tune_index >= axis_size(G, G.tune_axis)) {
      G.tune_index = 0;
      G.tune_axis = next_axis(G, G.tune_axis + 1);
      if (G.tune_axis >= 4) G.tuned = true;
      // a new axis starts from the best so far: its cost is re-measured
      else G.best_cost = -1.0;
    }
  }

  int advance_group(Group<R> &G) {
    collect_timing(G);
    // admitted cases join once their set-up has finished on the device
    for (size_t i = 0; i < G.pending.size();) {
      EngineCase *c = G.pending[i];
      const cudaError_t q = cudaEventQuery(c->ready);
      if (q == cudaErrorNotReady) {
        ++i;
        continue;
      }
      if (q != cudaSuccess) return cuda_failed(q, "cudaEventQuery(case set-up)");
      G.cases.push_back(c);
      G.pending.erase(G.pending.begin() + i);
      G.members_changed = true;
      G.dirty = true;
    }
    // cases with fewer steps left than a launch holds finish one at a time
    for (size_t i = 0; i < G.cases.size();) {
      EngineCase *c = G.cases[i];
      if (c->steps_left < k_) {
        if (c->steps_left > 0) {
          int st = thx_rk3_steps(c->h, c->u, c->dt, c->steps_left, G.stream);
          if (st) return st;
        }
        c->steps_left = 0;
        c->finished = true;
        THX_CU(cudaEventRecord(c->done, G.stream));
        G.cases.erase(G.cases.begin() + i);
        G.members_changed = true;
        G.dirty = true;
      } else {
        ++i;
      }
    }
    if (G.cases.empty()) return THX_OK;
    {
      const cudaError_t q = cudaEventQuery(G.ring[G.ring_pos]);
      if (q == cudaErrorNotReady) return THX_OK;  // two launches still queued
      if (q != cudaSuccess) return cuda_failed(q, "cudaEventQuery(launch ring)");
    }
    int st;
    typename Group<R>::Grids grids = G.best;
    bool measure = false;
    if (!G.tuned && !G.timing && tune_candidate(G, G.tune_index, grids)) {
      // time a candidate on a launch with the same cases as the one before
      // (a launch that cases joined or left runs a different load); after
      // four such launches in a row, time it anyway
      if (G.members_changed && G.unsteady < 4) {
        ++G.unsteady;
        grids = G.exec ? G.exec_grids : G.best;
      } else {
        measure = true;
        G.unsteady = 0;
      }
    } else if (!G.tuned && G.timing && G.exec) {
      grids = G.exec_grids;
    }
    // the work lists follow the CTA size
    const int epb = grids.half ? G.epb_half : G.epb_full;
    if (epb != G.epb) {
      G.epb = epb;
      G.dirty = true;
    }
    const double ta = now();
    if (G.dirty && (st = upload_tables(G))) return st;
    const double tb = now();
    t_tables_ += tb - ta;
    if (!G.exec || !(G.exec_grids == grids)) {
      if ((st = capture(G, grids))) return st;
    }
    if (measure) cudaEventRecord(G.t0, G.stream);
    THX_CU(cudaGraphLaunch(G.exec, G.stream));
    if (measure) {
      cudaEventRecord(G.t1, G.stream);
      G.timing = true;
      G.timing_grids = grids;
      G.timing_work = G.nodes * k_;
    }
    ++launches_;
    G.members_changed = false;
    t_launch_ += now() - tb;
    THX_CU(cudaEventRecord(G.ring[G.ring_pos], G.stream));
    G.ring_pos ^= 1;
    for (size_t i = 0; i < G.cases.size();) {
      EngineCase *c = G.cases[i];
      c->steps_left -= k_;
      if (c->steps_left == 0) {
        c->finished = true;
        THX_CU(cudaEventRecord(c->done, G.stream));
        G.cases.erase(G.cases.begin() + i);
        G.members_changed = true;
        G.dirty = true;
      } else {
        ++i;
      }
    }
    return THX_OK;
  }

  thx_config cfg_;
  size_t budget_;
  int k_;
  int device_ = 0, sms_ = 148;
  cudaMemPool_t pool_ = nullptr;
  cudaStream_t setup_ = nullptr;
  HostRing ring_;                 // pinned staging of admission uploads
  std::mutex bounce_mu_;
  std::vector<Bounce> bounce_;    // pinned buffers of result copies
  std::map<Key, std::unique_ptr<Group<R>>> groups_;
  std::map<int64_t, std::unique_ptr<EngineCase>> cases_;
  size_t bytes_ = 0;
  int64_t next_id_ = 1, launches_ = 0, done_ = 0;
  // host time accounting (seconds)
  double t_lock_ = 0, t_setup_ = 0, t_copy_ = 0, t_advance_ = 0, t_fetch_ = 0;
  double t_tables_ = 0, t_launch_ = 0;
  int64_t n_advance_ = 0, table_bytes_ = 0;
  static double now() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
  }
  std::mutex mu_;
  // device geometry shared by cases with the same thx_case::geometry_key
  std::mutex donor_mu_;
  std::map<int64_t, thx_operator_s *> donors_;
};

template <>
void Engine<double>::pick_kernels(Group<double> &G, int vk, int ns) {
#define THX_PICKB(P, D, NN)                                 \
  if (G.dim == D && G.N == NN) {                            \
    const OrderKernels0 k = order_kernels_##P##_##D##_##NN(); \
    G.volb = k.volb[vk][ns];                                \
    G.gradb = k.gradb;                                      \
    G.epb_full = k.epb;                                     \
    G.epb_half = k.epb_half;                                \
    G.volb_half = k.volb_half[vk][ns];                      \
    G.gradb_half = k.gradb_half;                            \
  }
  THX_FOR_ORDERS(THX_PICKB, 0, 2)
  THX_FOR_ORDERS(THX_PICKB, 0, 3)
#undef THX_PICKB
  const FaceKernels0 f = G.dim == 2 ? face_kernels_0_2() : face_kernels_0_3();
  G.faceb = f.faceb[cfg_.surface_flux][ns];
}

template <>
void Engine<float>::pick_kernels(Group<float> &G, int vk, int ns) {
#define THX_PICKB(P, D, NN)                                 \
  if (G.dim == D && G.N == NN) {                            \
    const OrderKernels1 k = order_kernels_##P##_##D##_##NN(); \
    G.volb = k.volb[vk][ns];                                \
    G.gradb = k.gradb;                                      \
    G.epb_full = k.epb;                                     \
    G.epb_half = k.epb_half;                                \
    G.volb_half = k.volb_half[vk][ns];                      \
    G.gradb_half = k.gradb_half;                            \
  }
  THX_FOR_ORDERS(THX_PICKB, 1, 2)
  THX_FOR_ORDERS(THX_PICKB, 1, 3)
#undef THX_PICKB
  const FaceKernels1 f = G.dim == 2 ? face_kernels_1_2() : face_kernels_1_3();
  G.faceb = f.faceb[cfg_.surface_flux][ns];
}

}  // namespace

struct thx_engine_s {
  EngineBase *impl = nullptr;
  int device = 0;
};

extern "C" {

int thx_case_footprint(const thx_geometry *g, const thx_config *cfg, int flow_model, size_t *bytes) {
  if (!g || !cfg || !bytes || g->dim < 2 || g->dim > 3 || g->order < 1 || g->num_elements <= 0 ||
      g->num_faces < 0)
    return THX_ERR_INVALID_ARGUMENT;
  *bytes = case_bytes(g, cfg, flow_model);
  return THX_OK;
}

int thx_engine_create(const thx_config *cfg, size_t hbm_budget, int steps_per_launch, thx_engine *out) {
  if (!cfg || !out || steps_per_launch < 1 || steps_per_launch > 1000) return THX_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  if (cfg->blending || cfg->volume_flux < 0 || cfg->volume_flux >= THX_FLUX_LTEEC ||
      cfg->surface_flux < 0 || cfg->surface_flux >= THX_FLUX_LTEEC)
    return THX_ERR_UNSUPPORTED;  // ideal gas, no subcell blending
  if (cfg->precision != THX_PRECISION_FP64 && cfg->precision != THX_PRECISION_FP32_MIXED)
    return THX_ERR_INVALID_ARGUMENT;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n <= 0) {
    cudaGetLastError();
    return THX_ERR_NO_DEVICE;
  }
  thx_engine_s *e = new (std::nothrow) thx_engine_s();
  if (!e) return THX_ERR_OUT_OF_MEMORY;
  cudaGetDevice(&e->device);
  int st;
  if (cfg->precision == THX_PRECISION_FP32_MIXED) {
    auto *impl = new (std::nothrow) Engine<float>(*cfg, hbm_budget, steps_per_launch);
    st = impl ? impl->init() : THX_ERR_OUT_OF_MEMORY;
    e->impl = impl;
  } else {
    auto *impl = new (std::nothrow) Engine<double>(*cfg, hbm_budget, steps_per_launch);
    st = impl ? impl->init() : THX_ERR_OUT_OF_MEMORY;
    e->impl = impl;
  }
  if (st) {
    delete e->impl;
    delete e;
    return st;
  }
  *out = e;
  return THX_OK;
}

int thx_engine_destroy(thx_engine e) {
  if (!e) return THX_ERR_INVALID_ARGUMENT;
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(e->device);
  delete e->impl;
  cudaSetDevice(prev);
  delete e;
  return THX_OK;
}

#define THX_ENGINE_CALL(expr)          \
  int prev = 0;                        \
  cudaGetDevice(&prev);                \
  if (prev != e->device) cudaSetDevice(e->device); \
  const int st = (expr);               \
  if (prev != e->device) cudaSetDevice(prev);      \
  return st;

int thx_engine_admit(thx_engine e, const thx_geometry *g, const thx_case *c, const double *u0,
                     int64_t *id) {
  if (!e) return THX_ERR_INVALID_ARGUMENT;
  THX_ENGINE_CALL(e->impl->admit(g, c, u0, id))
}

int thx_engine_advance(thx_engine e) {
  if (!e) return THX_ERR_INVALID_ARGUMENT;
  THX_ENGINE_CALL(e->impl->advance())
}

int thx_engine_poll(thx_engine e, int64_t *ids, int cap, int *count) {
  if (!e) return THX_ERR_INVALID_ARGUMENT;
  THX_ENGINE_CALL(e->impl->poll(ids, cap, count))
}

int thx_engine_fetch(thx_engine e, int64_t id, double *u_host) {
  if (!e) return THX_ERR_INVALID_ARGUMENT;
  THX_ENGINE_CALL(e->impl->fetch(id, u_host))
}

int thx_engine_get_stats(thx_engine e, thx_engine_stats *out) {
  if (!e || !out) return THX_ERR_INVALID_ARGUMENT;
  e->impl->stats(out);
  return THX_OK;
}

int thx_engine_groups(thx_engine e, thx_engine_group *out, int cap, int *count) {
  if (!e || !count || cap < 0 || (cap > 0 && !out)) return THX_ERR_INVALID_ARGUMENT;
  *count = e->impl->groups(out, cap);
  return THX_OK;
}

#undef THX_ENGINE_CALL

}  // extern "C"
