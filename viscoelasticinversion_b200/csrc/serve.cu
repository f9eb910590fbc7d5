// serve.cu — a request server over the step: forward solves and misfit
// gradients submitted from any host thread, run by a few worker threads
// ("lanes") on one CUDA stream per resident request, so the work of
// several requests overlaps on the device.
//
// The reference solves one problem per call and has no server
// (sciml_solver/ViscoelasticProblem.jl:273-309).  Scheduling here:
//  * admission: a request is admitted when its device footprint (estimated
//    from its grid, mechanisms, precision and step count) fits the HBM
//    budget next to the requests already resident; one that could never
//    fit is refused at submit (VI_ERR_BUDGET);
//  * continuous batching by time slices: requests join and leave between
//    slices of slice_steps steps; each slice goes to the resident request
//    with the least remaining work (grid cells x steps left, x3 for a
//    gradient), so a short request that arrives while a long one runs
//    preempts it at the next slice boundary (shortest remaining work
//    first, which minimises mean latency);
//  * gradient requests run in slices too: vi_gradient runs on a thread of
//    the request's own that yields after every slice_steps step units (a
//    forward or recompute step 1, an adjoint step 2), and while L - 1 lanes
//    run gradient slices an idle forward request goes first;
//  * lanes: each lane takes the next slice of the best idle resident
//    request and issues it on that request's stream; with L lanes the L
//    requests with the least remaining work advance at the same time (a
//    gradient occupies one lane while the others keep the forward solves
//    going, small grids run beside large ones).
// Each request has its own plan and device buffers, so its results do not
// depend on what else is resident (the sliced stepping is bitwise equal to
// one vi_step call).  Latency is measured from submit to the moment the
// results are in the caller's host buffers.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "nvtx.cuh"
#include "plan.cuh"

using Clock = std::chrono::steady_clock;

namespace vb {
namespace {

// A gradient request runs vi_gradient on a thread of its own, which yields
// after every slice (plan yield hook): a lane that picks the request hands
// it a budget of slice_steps step units and waits until the thread has
// enqueued them or finished, so a gradient holds a lane one slice at a
// time, as a forward request does.
struct GradRun {
  std::thread th;
  std::mutex mu;
  std::condition_variable cv;
  long long budget = 0;   // units the thread may still enqueue
  bool running = false;   // a lane handed it a budget and waits for the yield
  bool abort = false;     // the request is being released unfinished
  bool done = false;
  int rc = VI_OK;
  std::string msg;
  double J = 0;
  long long units = 0;    // enqueued so far (1 per forward step, 2 per adjoint step)
};

int grad_yield(void *ctx, int units) {
  auto *g = static_cast<GradRun *>(ctx);
  std::unique_lock<std::mutex> lk(g->mu);
  g->units += units;
  g->budget -= units;
  if (g->budget <= 0 && !g->abort) {
    g->running = false;
    g->cv.notify_all();
    g->cv.wait(lk, [&] { return g->running || g->abort; });
  }
  return g->abort ? 1 : 0;
}

struct Req {
  uint64_t ticket = 0;
  vi_request rq{};
  std::vector<vi_source> src;
  std::vector<vi_receiver> rec;
  int state = VI_REQ_QUEUED;
  int err = VI_OK;
  std::string msg;
  Clock::time_point t_submit, t_done;
  int64_t footprint = 0;
  // resident state (used by the lane that holds the request)
  vi_plan *plan = nullptr;
  void *buf = nullptr;
  vi_medium md{};
  vi_fields fd{};
  vi_shot shot{};
  void *obs_dev = nullptr;
  double *grad_dev = nullptr;
  int done_steps = 0;
  cudaStream_t st = nullptr;  // the request's own stream: its slices stay in order
  bool busy = false;          // a lane is advancing it (under the server lock)
  uint64_t last_turn = 0;     // round robin: when it last got a slice
  std::shared_ptr<GradRun> gr;  // gradient requests, once started
  bool started = false;         // has had a slice (under the server lock)
};

size_t esize_of(const vi_config &c) { return c.precision == VI_F64 ? 8 : 4; }

// Remaining work of a request in grid-cell steps (the scheduling key; a
// gradient costs about three forward passes, a TTI step about two).
double remaining_work(const Req &q) {
  const vi_request &r = q.rq;
  const double cells = (double)r.cfg.nx * r.cfg.nz;
  const double left = (double)(r.nt - q.done_steps);
  return cells * left * (r.kind == VI_REQ_GRADIENT ? 3.0 : 1.0) * (r.cfg.medium == VI_MEDIUM_TTI ? 2.0 : 1.0);
}

// Device bytes a request holds while resident (plan workspace included,
// rounded up): medium, state, the fused path's second state copy, CPML
// strips, wavelets and traces; for a gradient the checkpoints and segment
// slots, the adjoint state and scratch, observed traces and FP64 planes.
int64_t footprint(const vi_request &r) {
  const vi_config &c = r.cfg;
  const int64_t np = (int64_t)c.nx * c.nz, e = (int64_t)esize_of(c);
  const int64_t ns = 5 + 3 * (int64_t)c.nsls;
  const int64_t pml = c.pml_thickness > 0 ? c.pml_thickness : 0;
  const int64_t psi = 2 * 4 * (2 * pml * c.nz + c.nx * 2 * pml) * e;
  const int64_t tr = 2 * (int64_t)r.nrec * r.nt * e;
  const int64_t wav = (int64_t)r.nsrc * (r.wavelet_nt > 0 ? r.wavelet_nt : 0) * e;
  int64_t b = (8 + 2 * ns + 6) * np * e + psi + 2 * tr + wav + (16 << 20);
  if (r.kind == VI_REQ_GRADIENT) {
    int64_t K = 1;
    while (K * K < r.nt) ++K;
    const int64_t nck = (r.nt + K - 1) / K;
    const int64_t slot = ns * np * e + psi / 2;
    b += (nck + K + 2) * slot + 13 * np * e + 8 * np * 8 + tr;
  }
  return b;
}

}  // namespace
}  // namespace vb

using namespace vb;

struct vi_server {
  vi_serve_config cfg{};
  std::vector<std::thread> lanes;
  // plans of finished requests, reused by later requests with the same
  // configuration (destroying a plan frees device memory, which
  // synchronises the whole device and would stall the other lanes)
  std::mutex plan_mu;
  std::vector<vi_plan *> plan_cache;
  std::mutex mu;
  std::condition_variable cv;
  std::deque<std::shared_ptr<Req>> queue;
  std::vector<std::shared_ptr<Req>> active;  // resident (admitted and staged)
  std::unordered_map<uint64_t, std::shared_ptr<Req>> all;
  uint64_t next_ticket = 1;
  uint64_t turn = 0;
  int admitting = 0;  // admitted, still being staged by a lane
  bool stopping = false;
  int64_t used = 0;
};

namespace {

// up to 64 plans and 16 GB of plan workspace are kept; beyond that the
// oldest is destroyed (a device-wide free)
constexpr size_t kPlanCache = 64;
constexpr size_t kPlanCacheBytes = 16ull << 30;

bool same_config(const vi_config &a, const vi_config &b) { return std::memcmp(&a, &b, sizeof(a)) == 0; }

// A plan for config c: a cached one when there is one, else a new one.
int take_plan(vi_server *s, const vi_config &c, vi_plan **out) {
  {
    std::lock_guard<std::mutex> lk(s->plan_mu);
    for (size_t k = 0; k < s->plan_cache.size(); ++k) {
      vi_plan *p = s->plan_cache[k];
      if (same_config(p->cfg, c)) {
        s->plan_cache.erase(s->plan_cache.begin() + (long)k);
        *out = p;
        return VI_OK;
      }
    }
  }
  return vi_plan_create(&c, out);
}

// Keeps a finished request's plan for reuse (oldest evicted beyond the cap).
void give_plan(vi_server *s, vi_plan *p) {
  std::vector<vi_plan *> evict;
  {
    std::lock_guard<std::mutex> lk(s->plan_mu);
    s->plan_cache.push_back(p);
    size_t bytes = 0;
    for (vi_plan *c : s->plan_cache) bytes += c->bytes;
    while (s->plan_cache.size() > 1 && (s->plan_cache.size() > kPlanCache || bytes > kPlanCacheBytes)) {
      bytes -= s->plan_cache.front()->bytes;
      evict.push_back(s->plan_cache.front());
      s->plan_cache.erase(s->plan_cache.begin());
    }
  }
  for (vi_plan *c : evict) vi_plan_destroy(c);
}

template <typename T>
int admit_impl(vi_server *s, Req &q) {
  const vi_request &r = q.rq;
  const vi_config &c = r.cfg;
  const size_t np = (size_t)c.nx * c.nz;
  int rc = cuda_check(cudaStreamCreateWithFlags(&q.st, cudaStreamNonBlocking), "serve: create stream");
  if (rc) return rc;
  if ((rc = take_plan(s, c, &q.plan))) return rc;
  const int ns = 5 + 3 * c.nsls;
  const int nmed = 8;
  const size_t tr = 2 * (size_t)r.nrec * r.nt;
  const size_t wav = (size_t)r.nsrc * (r.wavelet_nt > 0 ? r.wavelet_nt : 0);
  const bool grad = r.kind == VI_REQ_GRADIENT;
  size_t elems = (nmed + ns) * np + wav + tr + (grad ? tr : 0) + 64;
  size_t bytes = elems * sizeof(T) + (grad ? 8 * np * sizeof(double) + 256 : 0);
  // stream-ordered: no device-wide synchronisation, so other lanes run on
  if ((rc = cuda_check(cudaMallocAsync(&q.buf, bytes, q.st), "serve: allocate request buffers"))) return rc;
  T *base = (T *)q.buf;
  const void *hp[8] = {r.medium_host.rho, r.medium_host.c11, r.medium_host.c13, r.medium_host.c15,
                       r.medium_host.c33, r.medium_host.c35, r.medium_host.c55, r.medium_host.tau};
  const void **dp[8] = {&q.md.rho, &q.md.c11, &q.md.c13, &q.md.c15, &q.md.c33, &q.md.c35, &q.md.c55, &q.md.tau};
  for (int k = 0; k < 8; ++k) {
    *dp[k] = nullptr;
    if (hp[k]) {
      T *d = base + k * np;
      if ((rc = cuda_check(cudaMemcpyAsync(d, hp[k], np * sizeof(T), cudaMemcpyHostToDevice, q.st),
                           "serve: upload medium")))
        return rc;
      *dp[k] = d;
    }
  }
  T *state = base + nmed * np;
  if ((rc = cuda_check(cudaMemsetAsync(state, 0, ns * np * sizeof(T), q.st), "serve: zero state"))) return rc;
  q.fd.vx = state;
  q.fd.vz = state + np;
  q.fd.sxx = state + 2 * np;
  q.fd.szz = state + 3 * np;
  q.fd.sxz = state + 4 * np;
  q.fd.m = c.nsls ? state + 5 * np : nullptr;
  q.fd.m_plane_stride = (long long)np;
  T *w = state + ns * np;
  T *t = w + wav;
  if (wav && (rc = cuda_check(cudaMemcpyAsync(w, r.wavelet_host, wav * sizeof(T), cudaMemcpyHostToDevice, q.st),
                              "serve: upload wavelets")))
    return rc;
  if (tr && (rc = cuda_check(cudaMemsetAsync(t, 0, tr * sizeof(T), q.st), "serve: zero traces"))) return rc;
  if (grad) {
    T *o = t + tr;
    if ((rc = cuda_check(cudaMemcpyAsync(o, r.obs_host, tr * sizeof(T), cudaMemcpyHostToDevice, q.st),
                         "serve: upload observed traces")))
      return rc;
    q.obs_dev = o;
    uintptr_t gp = ((uintptr_t)(o + tr) + 255) / 256 * 256;
    q.grad_dev = (double *)gp;
  }
  q.shot.nsrc = r.nsrc;
  q.shot.src_host = q.src.empty() ? nullptr : q.src.data();
  q.shot.wavelet_dev = w;
  q.shot.wavelet_nt = r.wavelet_nt;
  q.shot.nrec = r.nrec;
  q.shot.rec_host = q.rec.empty() ? nullptr : q.rec.data();
  q.shot.traces_dev = t;
  q.shot.traces_nt = r.nt;
  if ((rc = vi_plan_reset(q.plan, q.st))) return rc;
  return cuda_check(cudaStreamSynchronize(q.st), "serve: stage request");
}

int admit(vi_server *s, Req &q) {
  return q.rq.cfg.precision == VI_F64 ? admit_impl<double>(s, q) : admit_impl<float>(s, q);
}

void release(vi_server *s, Req &q) {
  if (q.gr && q.gr->th.joinable()) {  // a gradient left unfinished: stop its thread
    {
      std::lock_guard<std::mutex> lk(q.gr->mu);
      q.gr->abort = true;
      q.gr->cv.notify_all();
    }
    q.gr->th.join();
  }
  q.gr.reset();
  if (q.buf) cudaFreeAsync(q.buf, q.st);
  q.buf = nullptr;
  if (q.st) cudaStreamSynchronize(q.st);
  if (q.plan) give_plan(s, q.plan);
  q.plan = nullptr;
  if (q.st) cudaStreamDestroy(q.st);
  q.st = nullptr;
}

// Runs the request's next slice; sets *finished when the request is done.
int advance(vi_server *s, Req &q, bool *finished) {
  NvtxRange nr(q.rq.kind == VI_REQ_GRADIENT ? "vi_serve: gradient request" : "vi_serve: forward slice");
  const vi_request &r = q.rq;
  const size_t es = esize_of(r.cfg);
  int rc;
  if (r.kind == VI_REQ_GRADIENT) {
    if (!q.gr) {
      q.gr = std::make_shared<GradRun>();
      GradRun *g = q.gr.get();
      Req *qp = &q;
      const int dev = s->cfg.device;
      g->th = std::thread([g, qp, dev] {
        cudaSetDevice(dev);
        {
          std::unique_lock<std::mutex> lk(g->mu);
          g->cv.wait(lk, [&] { return g->running || g->abort; });
        }
        const vi_request &rr = qp->rq;
        // checkpoints every ceil(sqrt(nt)) steps, as the admission estimate
        // assumes (checkpoint_every 0 may keep every state in HBM)
        const int K = (int)std::ceil(std::sqrt((double)rr.nt));
        double J = 0;
        int grc = VI_ERR_STATE;
        std::string msg = "gradient: stopped";
        if (!g->abort) {
          qp->plan->yield_fn = grad_yield;
          qp->plan->yield_ctx = g;
          grc = vi_gradient(qp->plan, &qp->md, &qp->shot, rr.nt, qp->obs_dev, K, 0, qp->grad_dev, &J, qp->st);
          qp->plan->yield_fn = nullptr;
          qp->plan->yield_ctx = nullptr;
          if (grc) msg = vi_last_error();
        }
        std::lock_guard<std::mutex> lk(g->mu);
        g->rc = grc;
        if (grc) g->msg = msg;
        g->J = J;
        g->done = true;
        g->running = false;
        g->cv.notify_all();
      });
    }
    GradRun &g = *q.gr;
    {
      std::unique_lock<std::mutex> lk(g.mu);
      g.budget = s->cfg.slice_steps;
      g.running = true;
      g.cv.notify_all();
      g.cv.wait(lk, [&] { return !g.running; });
      q.done_steps = (int)std::min<long long>(r.nt, g.units / 4);
      if (!g.done) {
        *finished = false;
        return VI_OK;
      }
    }
    g.th.join();
    if (g.rc) return set_error(g.rc, g.msg);
    const double J = g.J;
    const size_t np = (size_t)r.cfg.nx * r.cfg.nz;
    if ((rc = cuda_check(cudaMemcpyAsync(r.grad_host, q.grad_dev, 8 * np * sizeof(double), cudaMemcpyDeviceToHost,
                                         q.st),
                         "serve: download gradient")))
      return rc;
    if (r.misfit_host) *r.misfit_host = J;
  } else {
    int n = s->cfg.slice_steps;
    if (n > r.nt - q.done_steps) n = r.nt - q.done_steps;
    if ((rc = vi_step(q.plan, &q.md, &q.fd, &q.shot, q.done_steps, n, 0, q.st))) return rc;
    q.done_steps += n;
    if (q.done_steps < r.nt) {
      *finished = false;
      return VI_OK;
    }
    if ((rc = vi_plan_status(q.plan, q.st))) return rc;
  }
  const size_t tr = 2 * (size_t)r.nrec * r.nt;
  if (tr && r.traces_host &&
      (rc = cuda_check(cudaMemcpyAsync(r.traces_host, q.shot.traces_dev, tr * es, cudaMemcpyDeviceToHost, q.st),
                       "serve: download traces")))
    return rc;
  if ((rc = cuda_check(cudaStreamSynchronize(q.st), "serve: finish request"))) return rc;
  *finished = true;
  return VI_OK;
}

void finish(vi_server *s, const std::shared_ptr<Req> &q, int rc) {
  release(s, *q);
  std::lock_guard<std::mutex> lk(s->mu);
  q->err = rc;
  if (rc) q->msg = vi_last_error();
  q->state = rc ? VI_REQ_FAILED : VI_REQ_DONE;
  q->t_done = Clock::now();
  s->used -= q->footprint;
  s->cv.notify_all();
}

// true when the front of the queue may be admitted now
bool can_admit(const vi_server *s) {
  return !s->queue.empty() && (int)s->active.size() + s->admitting < s->cfg.max_active &&
         s->used + s->queue.front()->footprint <= s->cfg.hbm_budget_bytes;
}

// the idle resident request the policy picks next (nullptr if none).  A
// gradient holds its lane for its whole length, so while lanes - 1 lanes
// run gradients an idle forward request goes first: the forward stream is
// never left without a lane
std::shared_ptr<Req> pick_idle(vi_server *s) {
  int grads = 0, open_grads = 0;
  bool idle_fwd = false;
  for (auto &q : s->active) {
    if (q->busy && q->rq.kind == VI_REQ_GRADIENT) ++grads;
    if (q->started && q->rq.kind == VI_REQ_GRADIENT) ++open_grads;
    if (!q->busy && q->rq.kind != VI_REQ_GRADIENT) idle_fwd = true;
  }
  const bool hold_grads = s->cfg.lanes > 1 && grads >= s->cfg.lanes - 1 && idle_fwd;
  // at most `lanes` gradients in progress at once, as when each ran whole:
  // a started gradient holds its checkpoint workspace until it ends
  const bool hold_new_grads = open_grads >= s->cfg.lanes;
  std::shared_ptr<Req> best;
  for (auto &q : s->active) {
    if (q->busy) continue;
    if (hold_grads && q->rq.kind == VI_REQ_GRADIENT) continue;
    if (hold_new_grads && !q->started && q->rq.kind == VI_REQ_GRADIENT) continue;
    if (!best) {
      best = q;
    } else if (s->cfg.policy == VI_SERVE_ROUND_ROBIN ? q->last_turn < best->last_turn
                                                      : remaining_work(*q) < remaining_work(*best)) {
      best = q;
    }
  }
  return best;
}

void lane_main(vi_server *s) {
  cudaSetDevice(s->cfg.device);
  for (;;) {
    std::shared_ptr<Req> adm, pick;
    {
      std::unique_lock<std::mutex> lk(s->mu);
      const auto drained = [&] {
        return s->stopping && s->queue.empty() && s->active.empty() && s->admitting == 0;
      };
      s->cv.wait(lk, [&] { return can_admit(s) || pick_idle(s) != nullptr || drained(); });
      if (can_admit(s)) {
        adm = s->queue.front();
        s->queue.pop_front();
        s->used += adm->footprint;
        adm->state = VI_REQ_RUNNING;
        ++s->admitting;
      } else if ((pick = pick_idle(s))) {
        pick->busy = true;
        pick->started = true;
        pick->last_turn = ++s->turn;
      } else {
        return;  // drained
      }
    }
    if (adm) {
      const int rc = admit(s, *adm);
      if (rc) {
        {
          std::lock_guard<std::mutex> lk(s->mu);
          --s->admitting;
        }
        finish(s, adm, rc);
        continue;
      }
      std::lock_guard<std::mutex> lk(s->mu);
      --s->admitting;
      s->active.push_back(adm);
      s->cv.notify_all();
      continue;
    }
    bool fin = false;
    const int rc = advance(s, *pick, &fin);
    if (rc || fin) {
      {
        std::lock_guard<std::mutex> lk(s->mu);
        for (size_t k = 0; k < s->active.size(); ++k)
          if (s->active[k] == pick) {
            s->active.erase(s->active.begin() + (long)k);
            break;
          }
      }
      finish(s, pick, rc);
    } else {
      std::lock_guard<std::mutex> lk(s->mu);
      pick->busy = false;
      s->cv.notify_all();
    }
  }
}

}  // namespace

extern "C" int vi_serve_start(const vi_serve_config *cfg, vi_server **out) {
  if (!cfg || !out) return set_error(VI_ERR_ARG, "serve: NULL argument");
  int ndev = 0;
  int rc = cuda_check(cudaGetDeviceCount(&ndev), "cudaGetDeviceCount");
  if (rc) return rc;
  if (cfg->device < 0 || cfg->device >= ndev) return set_error(VI_ERR_ARG, "serve: no such device");
  auto *s = new vi_server();
  s->cfg = *cfg;
  if (s->cfg.slice_steps <= 0) s->cfg.slice_steps = 1024;
  if (s->cfg.max_active <= 0) s->cfg.max_active = 64;
  if (s->cfg.hbm_budget_bytes <= 0) s->cfg.hbm_budget_bytes = 150LL * 1000 * 1000 * 1000;
  if (s->cfg.policy != VI_SERVE_ROUND_ROBIN) s->cfg.policy = VI_SERVE_SHORTEST_FIRST;
  // two lanes measured best on the mixed request stream (one for the long
  // solves, one for the short ones; more lanes make the large solves share
  // the GPU with each other)
  if (s->cfg.lanes <= 0) s->cfg.lanes = 2;
  if (s->cfg.lanes > 16) s->cfg.lanes = 16;
  if ((rc = cuda_check(cudaSetDevice(cfg->device), "cudaSetDevice"))) {
    delete s;
    return rc;
  }
  for (int k = 0; k < s->cfg.lanes; ++k) s->lanes.emplace_back(lane_main, s);
  *out = s;
  return VI_OK;
}

extern "C" int vi_serve_submit(vi_server *s, const vi_request *r, uint64_t *ticket) {
  if (!s || !r || !ticket) return set_error(VI_ERR_ARG, "serve: NULL argument");
  if (r->kind != VI_REQ_FORWARD && r->kind != VI_REQ_GRADIENT) return set_error(VI_ERR_ARG, "serve: unknown request kind");
  if (r->nt <= 0) return set_error(VI_ERR_ARG, "serve: nt must be positive");
  if (r->nsrc < 0 || r->nrec < 0) return set_error(VI_ERR_ARG, "serve: negative source/receiver count");
  if (r->nsrc > 0 && (!r->src_host || !r->wavelet_host || r->wavelet_nt <= 0))
    return set_error(VI_ERR_ARG, "serve: sources need src_host and wavelet_host");
  if (r->nrec > 0 && (!r->rec_host || !r->traces_host)) return set_error(VI_ERR_ARG, "serve: receivers need rec_host and traces_host");
  if (r->kind == VI_REQ_GRADIENT && (!r->obs_host || !r->grad_host || r->nrec <= 0))
    return set_error(VI_ERR_ARG, "serve: gradient requests need receivers, obs_host and grad_host");
  if (!r->medium_host.rho) return set_error(VI_ERR_ARG, "serve: medium_host is incomplete");
  auto q = std::make_shared<Req>();
  q->rq = *r;
  q->src.assign(r->src_host, r->src_host + r->nsrc);
  q->rec.assign(r->rec_host, r->rec_host + r->nrec);
  q->footprint = footprint(*r);
  if (q->footprint > s->cfg.hbm_budget_bytes)
    return set_error(VI_ERR_BUDGET, "serve: request needs " + std::to_string(q->footprint) +
                                        " device bytes, more than the budget " +
                                        std::to_string(s->cfg.hbm_budget_bytes));
  std::lock_guard<std::mutex> lk(s->mu);
  if (s->stopping) return set_error(VI_ERR_STATE, "serve: server is stopping");
  q->ticket = s->next_ticket++;
  q->t_submit = Clock::now();
  s->all[q->ticket] = q;
  s->queue.push_back(q);
  *ticket = q->ticket;
  s->cv.notify_all();
  return VI_OK;
}

extern "C" int vi_serve_poll(vi_server *s, uint64_t ticket, int32_t *state, double *latency_ms) {
  if (!s || !state) return set_error(VI_ERR_ARG, "serve: NULL argument");
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->all.find(ticket);
  if (it == s->all.end()) return set_error(VI_ERR_ARG, "serve: unknown ticket");
  const Req &q = *it->second;
  *state = q.state;
  const auto end = (q.state == VI_REQ_DONE || q.state == VI_REQ_FAILED) ? q.t_done : Clock::now();
  if (latency_ms) *latency_ms = std::chrono::duration<double, std::milli>(end - q.t_submit).count();
  if (q.state == VI_REQ_FAILED) return set_error(q.err, "serve: request failed: " + q.msg);
  return VI_OK;
}

extern "C" int vi_serve_wait(vi_server *s, uint64_t ticket, double timeout_s, int32_t *state) {
  if (!s || !state) return set_error(VI_ERR_ARG, "serve: NULL argument");
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->all.find(ticket);
  if (it == s->all.end()) return set_error(VI_ERR_ARG, "serve: unknown ticket");
  auto q = it->second;
  auto done = [&] { return q->state == VI_REQ_DONE || q->state == VI_REQ_FAILED; };
  if (timeout_s < 0)
    s->cv.wait(lk, done);
  else
    s->cv.wait_for(lk, std::chrono::duration<double>(timeout_s), done);
  *state = q->state;
  if (q->state == VI_REQ_FAILED) return set_error(q->err, "serve: request failed: " + q->msg);
  return VI_OK;
}

extern "C" int vi_serve_stop(vi_server *s) {
  if (!s) return set_error(VI_ERR_ARG, "serve: NULL argument");
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stopping = true;
    s->cv.notify_all();
  }
  for (auto &t : s->lanes)
    if (t.joinable()) t.join();
  for (vi_plan *p : s->plan_cache) vi_plan_destroy(p);
  delete s;
  return VI_OK;
}
