// batch.cu — many shots of different grids and step counts advancing
// together: one kernel launch per time step covers the tiles of every shot
// still running, and the whole sequence of launches is one CUDA graph.
//
// Each shot keeps its own plan (CPML tables and ψ, the second state copy,
// source/receiver lists); the batch adds device arrays of per-shot step
// arguments, extras and tensor maps (both ping-pong parities) that the
// batched TMA kernel indexes per tile.  Shots are processed in descending
// step-count order so the shots active at step it are a prefix of the
// order and a launch covers items [0, prefix[active]).
//
// Kernel forms: the TMA-staged fused step (one launch per time step; two-
// stage persistent tiles or one-stage tiles), the split pair (a velocity
// and a stress launch per time step, in place; TTI memory variables and
// psi ping-pong by step parity), or per shot (each shot's own vi_step time
// loop, one shot after the other: the fastest when every shot fills the
// GPU by itself).  The autotuner picks the form by timing a
// few steps of each on the bound shots and caches the choice per (medium,
// precision, mechanisms, grid set).
#include <algorithm>
#include <cstring>
#include <map>
#include <mutex>
#include <numeric>
#include <string>
#include <thread>
#include <vector>

#include "fused_tma.cuh"
#include "nvtx.cuh"
#include "plan.cuh"
#include "split.cuh"

struct vi_batch {
  int n = 0;
  int kind = 0, precision = 0, nsls = 0, device = 0, nsm = 148;
  std::vector<vi_plan *> plans;
  std::vector<vi_medium> med;
  std::vector<vi_fields> fields;
  std::vector<int> nt;
  std::vector<std::vector<vi_source>> src;
  std::vector<std::vector<vi_receiver>> rec;
  std::vector<vi_shot> shot;
  std::vector<char> bound;
  // device arrays
  void *dev = nullptr;
  size_t dev_bytes = 0;
  int *err = nullptr;
  // cached graph of the whole run (valid while nothing is re-bound)
  cudaGraphExec_t graph = nullptr;
  int graph_form = -1;
  bool dirty = true;
  int form = -1;  // kernel form: -1 untuned, 0 one-stage, 1 two-stage persistent, 2 split pair
  std::vector<int> order;
  std::vector<int> prefix;
  int max_nt = 0;
  bool afda = false;  // some shot has the H-AFDA free surface
  // concurrent per-shot form: its streams and their fork / join events
  std::vector<cudaStream_t> streams;
  std::vector<cudaEvent_t> joins;
  cudaEvent_t fork = nullptr;
};

namespace vb {

constexpr int kFormOneStage = 0, kFormTwoStage = 1, kFormSplit = 2, kFormPerShot = 3, kFormStreams = 4;
constexpr int kBatchStreams = 8;  // streams of the concurrent per-shot form

static std::map<std::string, int> g_tuned;  // kernel form chosen per problem class
static std::mutex g_tuned_mu;               // batches may run on several host threads

static std::string tune_key(const vi_batch *b) {
  std::vector<std::pair<int, int>> g;
  for (int i = 0; i < b->n; ++i) g.emplace_back(b->plans[i]->cfg.nx, b->plans[i]->cfg.nz);
  std::sort(g.begin(), g.end());
  g.erase(std::unique(g.begin(), g.end()), g.end());
  std::string k = std::to_string(b->kind) + "/" + std::to_string(b->precision) + "/" +
                  std::to_string(b->nsls);
  for (auto &p : g) k += "/" + std::to_string(p.first) + "x" + std::to_string(p.second);
  return k;
}

// Processing order (descending step count, so the shots active at step it
// form a prefix) and the longest step count.
static void set_order(vi_batch *b) {
  b->order.resize(b->n);
  std::iota(b->order.begin(), b->order.end(), 0);
  std::stable_sort(b->order.begin(), b->order.end(), [&](int x, int y) { return b->nt[x] > b->nt[y]; });
  b->max_nt = b->n ? b->nt[b->order[0]] : 0;
}

// Builds every per-shot device structure for one kernel form and uploads it.
template <typename T>
static int prepare(vi_batch *b, int form, cudaStream_t st, BatchDev<T> &bd) {
  // one tile list serves both merged split kernels: their tilings must agree
  static_assert(SplitGeom<T>::TX == SplitStressGeomBatch<T>::TX && SplitGeom<T>::TZ == SplitStressGeomBatch<T>::TZ &&
                    SplitGeom<T>::TX == SplitTtiGeomBatch<T>::TX && SplitGeom<T>::TZ == SplitTtiGeomBatch<T>::TZ,
                "merged split kernels share one tiling");
  const bool split = form == kFormSplit;
  const bool tti = b->kind == VI_MEDIUM_TTI;
  TmaBoxes bx{};
  if (!split) {
    bx = tma_boxes(b->kind, b->nsls, (int)sizeof(T), form == kFormTwoStage);
    if (!bx.ok) return set_error(VI_ERR_ARG, "batch: the TMA-staged step does not fit this medium");
  }
  const int n = b->n;
  std::vector<StepArgs<T>> args(2 * n);
  std::vector<FusedExtras<T>> ext(n);
  std::vector<TmaMaps> maps(split ? 0 : 2 * n);
  std::vector<SplitMaps> smaps(split ? n : 0);
  std::vector<int> ntiles(n);
  long long kept = 0;  // planes the split kernels keep in L2, over every shot
  for (int i = 0; i < n; ++i) kept += 5LL * b->plans[i]->cfg.nx * b->plans[i]->cfg.nz * (long long)sizeof(T);
  int rc;
  for (int i = 0; i < n; ++i) {
    vi_plan *p = b->plans[i];
    const vi_config &c = p->cfg;
    const size_t np = (size_t)c.nx * c.nz;
    const int nstate = 5 + 3 * c.nsls;
    if (!p->alt) {
      size_t have = 0;
      if ((rc = ensure_buffer(p, &p->alt, &have, nstate * np * sizeof(T)))) return rc;
      if ((rc = cuda_check(cudaMemsetAsync(p->alt, 0, nstate * np * sizeof(T), st), "zero alt state")))
        return rc;
    }
    if ((rc = stage_shot<T>(p, &b->shot[i], st))) return rc;
    int ntx, ntz;
    std::vector<int> off;
    std::vector<int4> ent;
    if (split)
      build_tile_lists(c.nx, c.nz, SplitGeom<T>::TX, SplitGeom<T>::TZ, 0, &b->shot[i], off, ent, ntx, ntz);
    else
      build_tile_lists(c.nx, c.nz, bx.TX, bx.TZ, bx.HV, &b->shot[i], off, ent, ntx, ntz);
    int *d_off = nullptr;
    int4 *d_ent = nullptr;
    if ((rc = stage_tile_lists(p, off, ent, st, &d_off, &d_ent))) return rc;
    ntiles[i] = ntx * ntz;
    StepArgs<T> a = make_args<T>(p, &b->med[i], &b->fields[i]);
    T *user[5] = {a.vx, a.vz, a.sxx, a.szz, a.sxz};
    T *alt = (T *)p->alt;
    T *alt_st[5];
    for (int q = 0; q < 5; ++q) alt_st[q] = alt + q * np;
    T *psix0 = (T *)p->psix, *psiz0 = (T *)p->psiz;
    p->psi_cur = 0;  // a batch run starts from rest: psi is reset below
    if (split) {
      if (!split_eligible<T>(p, a))
        return set_error(VI_ERR_ARG, "batch: the split step needs 16-byte aligned planes");
      if (b->precision == VI_F32C) {
        // compensated stress accumulation, as the shot's own split step
        if (!p->slo) {
          size_t have = 0;
          if ((rc = ensure_buffer(p, &p->slo, &have, 3 * np * sizeof(uint16_t)))) return rc;
          if ((rc = cuda_check(cudaMemsetAsync(p->slo, 0, 3 * np * sizeof(uint16_t), st), "zero stress residues")))
            return rc;
          p->slo_valid = true;
        }
        a.slo = (uint16_t *)p->slo;
        a.slo_plane = (long long)np;
      }
      for (int par = 0; par < 2; ++par) {
        // sigma and v in place; TTI: M and psi from parity par to the other
        StepArgs<T> s = a;
        const int pin = tti ? par : 0, pout = tti ? 1 - par : 0;
        if (tti) {
          s.m = par == 0 ? a.m : alt + 5 * np;
          s.mstride = par == 0 ? a.mstride : (long long)np;
          s.m_o = par == 0 ? alt + 5 * np : a.m;
          s.mstride_o = par == 0 ? (long long)np : a.mstride;
        }
        s.psix = psix0 ? psix0 + pin * kPsiPerSet * p->psix_plane : nullptr;
        s.psix_o = psix0 ? psix0 + pout * kPsiPerSet * p->psix_plane : nullptr;
        s.psiz = psiz0 ? psiz0 + pin * kPsiPerSet * p->psiz_plane : nullptr;
        s.psiz_o = psiz0 ? psiz0 + pout * kPsiPerSet * p->psiz_plane : nullptr;
        args[2 * i + par] = s;
      }
      const int bw = tti ? SplitTtiGeomBatch<T>::BW : SplitStressGeomBatch<T>::BW;
      const int bh = tti ? SplitTtiGeomBatch<T>::BH : SplitStressGeomBatch<T>::BH;
      if ((rc = encode_map(&smaps[i].a, a.vx, (int)sizeof(T), c.nx, c.nz, 1, 0, bw, bh, 1))) return rc;
      if ((rc = encode_map(&smaps[i].b, a.vz, (int)sizeof(T), c.nx, c.nz, 1, 0, bw, bh, 1))) return rc;
      smaps[i].c = smaps[i].b;
    }
    for (int par = 0; par < (split ? 0 : 2); ++par) {
      StepArgs<T> s = a;
      T *const *in = par == 0 ? user : alt_st;
      T *const *out = par == 0 ? alt_st : user;
      s.vx = in[0]; s.vz = in[1]; s.sxx = in[2]; s.szz = in[3]; s.sxz = in[4];
      s.vx_o = out[0]; s.vz_o = out[1]; s.sxx_o = out[2]; s.szz_o = out[3]; s.sxz_o = out[4];
      s.m = par == 0 ? a.m : alt + 5 * np;
      s.mstride = par == 0 ? a.mstride : (long long)np;
      s.m_o = par == 0 ? alt + 5 * np : a.m;
      s.mstride_o = par == 0 ? (long long)np : a.mstride;
      s.psix = psix0 ? psix0 + par * kPsiPerSet * p->psix_plane : nullptr;
      s.psix_o = psix0 ? psix0 + (1 - par) * kPsiPerSet * p->psix_plane : nullptr;
      s.psiz = psiz0 ? psiz0 + par * kPsiPerSet * p->psiz_plane : nullptr;
      s.psiz_o = psiz0 ? psiz0 + (1 - par) * kPsiPerSet * p->psiz_plane : nullptr;
      args[2 * i + par] = s;
      if ((rc = encode_parity<T>(maps[2 * i + par], bx, c, in, s.m, s.mstride, s))) return rc;
    }
    FusedExtras<T> &x = ext[i];
    x.ntx = ntx;
    x.fs = c.free_surface;
    x.it = 0;
    x.tile_off = d_off;
    x.tile_ent = d_ent;
    x.amp = (const T *)p->damp;
    const vi_shot &sh = b->shot[i];
    x.wavelet = sh.nsrc ? (const T *)sh.wavelet_dev : nullptr;
    x.wnt = sh.nsrc ? sh.wavelet_nt : 0;
    x.traces = sh.nrec ? (T *)sh.traces_dev : nullptr;
    x.tnt = sh.nrec ? sh.traces_nt : 0;
    x.nrec = sh.nrec;
    x.err = b->err;
    x.l2hint = l2_hints_fit(kept, p->l2_bytes);
  }
  // descending step count: the shots active at step it form a prefix
  set_order(b);
  b->prefix.assign(n + 1, 0);
  for (int q = 0; q < n; ++q) b->prefix[q + 1] = b->prefix[q] + ntiles[b->order[q]];
  // (shot, tile) of every item, so a CTA finds its tile with one load
  std::vector<int2> items((size_t)b->prefix[n]);
  for (int q = 0; q < n; ++q)
    for (int t = 0; t < ntiles[b->order[q]]; ++t) items[(size_t)b->prefix[q] + t] = make_int2(b->order[q], t);
  // one device block: args | ext | maps | smaps | prefix | order | items
  auto up = [](size_t x) { return (x + 127) / 128 * 128; };
  const size_t o_args = 0, o_ext = up(o_args + args.size() * sizeof(StepArgs<T>));
  const size_t o_maps = up(o_ext + ext.size() * sizeof(FusedExtras<T>));
  const size_t o_smaps = up(o_maps + maps.size() * sizeof(TmaMaps));
  const size_t o_pre = up(o_smaps + smaps.size() * sizeof(SplitMaps));
  const size_t o_ord = up(o_pre + b->prefix.size() * sizeof(int));
  const size_t o_items = up(o_ord + b->order.size() * sizeof(int));
  const size_t total = up(o_items + items.size() * sizeof(int2));
  if (b->dev_bytes < total) {
    if (b->dev) cudaFree(b->dev);
    b->dev = nullptr;
    b->dev_bytes = 0;
    if (cudaMalloc(&b->dev, total) != cudaSuccess) {
      cudaGetLastError();
      return set_error(VI_ERR_BUDGET, "batch: cudaMalloc of the shot table failed");
    }
    b->dev_bytes = total;
  }
  std::vector<char> host(total, 0);
  std::memcpy(host.data() + o_args, args.data(), args.size() * sizeof(StepArgs<T>));
  std::memcpy(host.data() + o_ext, ext.data(), ext.size() * sizeof(FusedExtras<T>));
  std::memcpy(host.data() + o_maps, maps.data(), maps.size() * sizeof(TmaMaps));
  std::memcpy(host.data() + o_smaps, smaps.data(), smaps.size() * sizeof(SplitMaps));
  std::memcpy(host.data() + o_pre, b->prefix.data(), b->prefix.size() * sizeof(int));
  std::memcpy(host.data() + o_ord, b->order.data(), b->order.size() * sizeof(int));
  std::memcpy(host.data() + o_items, items.data(), items.size() * sizeof(int2));
  if ((rc = cuda_check(cudaMemcpyAsync(b->dev, host.data(), total, cudaMemcpyHostToDevice, st),
                       "upload batch table")))
    return rc;
  if ((rc = cuda_check(cudaStreamSynchronize(st), "upload batch table"))) return rc;
  char *d = (char *)b->dev;
  bd.args = (const StepArgs<T> *)(d + o_args);
  bd.ext = (const FusedExtras<T> *)(d + o_ext);
  bd.maps = (const TmaMaps *)(d + o_maps);
  bd.smaps = (const SplitMaps *)(d + o_smaps);
  bd.prefix = (const int *)(d + o_pre);
  bd.order = (const int *)(d + o_ord);
  bd.items = (const int2 *)(d + o_items);
  bd.nshots = n;
  bd.err = b->err;
  return VI_OK;
}

// Items (tiles of active shots) at step it.
static int items_at(const vi_batch *b, int it) {
  int a = 0;
  while (a < b->n && b->nt[b->order[a]] > it) ++a;
  return b->prefix[a];
}

template <typename T>
static int launch_steps(vi_batch *b, const BatchDev<T> &bd, int form, int it0, int it1,
                        cudaStream_t st) {
  for (int it = it0; it < it1; ++it) {
    const int nitems = items_at(b, it);
    if (nitems == 0) break;
    int rc;
    if (form == kFormSplit) {
      // each launch overlaps the tail of the previous one and waits for it
      // at entry (programmatic dependent launch), as the one-shot pair does
      rc = launch_split_vel_batch<T>(b->kind, b->afda, bd, it, nitems, st, it > it0);
      if (!rc)
        rc = launch_split_stress_batch<T>(b->kind, b->nsls, b->precision == VI_F32C, b->afda, bd, it, nitems, st, true);
    } else {
      rc = launch_fused_tma_batch<T>(b->kind, b->nsls, bd, it, nitems, b->nsm, form == kFormTwoStage, st);
    }
    if (rc) return rc;
  }
  return cuda_check(cudaGetLastError(), "batch launch");
}

// Zeroes every shot's fields and psi (the state a forward solve starts from).
template <typename T>
static int reset_state(vi_batch *b, cudaStream_t st) {
  int rc;
  for (int i = 0; i < b->n; ++i) {
    vi_plan *p = b->plans[i];
    const size_t pb = (size_t)p->cfg.nx * p->cfg.nz * sizeof(T);
    const vi_fields &f = b->fields[i];
    void *planes[5] = {f.vx, f.vz, f.sxx, f.szz, f.sxz};
    for (void *q : planes)
      if ((rc = cuda_check(cudaMemsetAsync(q, 0, pb, st), "reset fields"))) return rc;
    for (int q = 0; q < 3 * p->cfg.nsls; ++q)
      if ((rc = cuda_check(cudaMemsetAsync((char *)f.m + q * f.m_plane_stride * sizeof(T), 0, pb, st),
                           "reset memory variables")))
        return rc;
    if ((rc = vi_plan_reset(p, st))) return rc;
  }
  return VI_OK;
}


// The per-shot form: steps [it0, it1) of every shot (capped at its step
// count) through vi_step, one shot after the other.
static int per_shot_steps(vi_batch *b, int it0, int it1, cudaStream_t st) {
  for (int q = 0; q < b->n; ++q) {
    const int i = b->order[q];
    const int n = std::min(it1, b->nt[i]) - it0;
    if (n <= 0) continue;
    const int rc = vi_step(b->plans[i], &b->med[i], &b->fields[i], &b->shot[i], it0, n, 0, st);
    if (rc) return rc;
  }
  return VI_OK;
}

// The concurrent per-shot form: every shot through its own vi_step calls,
// as in the per-shot form, spread over kBatchStreams streams so that shots
// which do not fill the GPU run beside one another (each with the
// single-shot kernels).  Largest work first, each shot to the stream with
// the least work queued; one host thread per stream issues its shots, so a
// call that waits on the host for its stream (it stages the shot's lists)
// holds up no other stream, and the launches are issued in parallel.  The
// streams fork from and join back into st.
static int streams_steps(vi_batch *b, int it0, int it1, cudaStream_t st) {
  int rc;
  if (b->streams.empty()) {
    b->streams.assign(kBatchStreams, nullptr);
    b->joins.assign(kBatchStreams, nullptr);
    for (int k = 0; k < kBatchStreams; ++k) {
      if ((rc = cuda_check(cudaStreamCreateWithFlags(&b->streams[k], cudaStreamNonBlocking), "batch stream")))
        return rc;
      if ((rc = cuda_check(cudaEventCreateWithFlags(&b->joins[k], cudaEventDisableTiming), "batch event")))
        return rc;
    }
    if ((rc = cuda_check(cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming), "batch event"))) return rc;
  }
  if ((rc = cuda_check(cudaEventRecord(b->fork, st), "fork"))) return rc;
  for (cudaStream_t q : b->streams)
    if ((rc = cuda_check(cudaStreamWaitEvent(q, b->fork, 0), "fork wait"))) return rc;
  std::vector<std::pair<double, int>> work;  // (cells x steps, shot)
  for (int i = 0; i < b->n; ++i) {
    const int n = std::min(it1, b->nt[i]) - it0;
    if (n > 0) work.push_back({(double)b->plans[i]->cfg.nx * b->plans[i]->cfg.nz * n, i});
  }
  std::stable_sort(work.begin(), work.end(), [](const auto &x, const auto &y) { return x.first > y.first; });
  std::vector<double> load(kBatchStreams, 0.0);
  std::vector<std::vector<int>> mine(kBatchStreams);
  for (const auto &wk : work) {
    const int k = (int)(std::min_element(load.begin(), load.end()) - load.begin());
    mine[k].push_back(wk.second);
    load[k] += wk.first;
  }
  std::vector<int> rcs(kBatchStreams, VI_OK);
  std::vector<std::string> msgs(kBatchStreams);
  std::vector<std::thread> th;
  for (int k = 0; k < kBatchStreams; ++k) {
    if (mine[k].empty()) continue;
    th.emplace_back([&, k] {
      cudaSetDevice(b->device);
      for (int i : mine[k]) {
        const int n = std::min(it1, b->nt[i]) - it0;
        if ((rcs[k] = vi_step(b->plans[i], &b->med[i], &b->fields[i], &b->shot[i], it0, n, 0, b->streams[k]))) {
          msgs[k] = vi_last_error();
          return;
        }
      }
    });
  }
  for (auto &t : th) t.join();
  for (int k = 0; k < kBatchStreams; ++k)
    if (rcs[k]) return set_error(rcs[k], msgs[k]);
  for (int k = 0; k < kBatchStreams; ++k) {
    if ((rc = cuda_check(cudaEventRecord(b->joins[k], b->streams[k]), "join"))) return rc;
    if ((rc = cuda_check(cudaStreamWaitEvent(st, b->joins[k], 0), "join wait"))) return rc;
  }
  return VI_OK;
}

// Marginal time of 8 more steps of every shot for one form (the time of
// 16 steps minus that of 8), so one-time costs per call — host staging of
// the per-shot form — do not decide between forms.
template <typename F>
static int time_marginal(F run_steps, cudaStream_t st, int max_nt, float *ms) {
  const int s1 = std::min(8, max_nt), s2 = std::min(16, max_nt);
  int rc = run_steps(0, 2);  // warm-up
  if (rc) return rc;
  float t[2] = {0, 0};
  const int n[2] = {s1, s2};
  for (int k = 0; k < 2; ++k) {
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, st);
    rc = run_steps(0, n[k]);
    cudaEventRecord(e1, st);
    cudaEventSynchronize(e1);
    cudaEventElapsedTime(&t[k], e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc) return rc;
  }
  *ms = s2 > s1 ? t[1] - t[0] : t[1];
  return VI_OK;
}

template <typename T>
static int tune(vi_batch *b, cudaStream_t st) {
  const std::string key = tune_key(b);
  {
    std::lock_guard<std::mutex> lk(g_tuned_mu);
    auto hit = g_tuned.find(key);
    if (hit != g_tuned.end()) {
      b->form = hit->second;
      return VI_OK;
    }
  }
  set_order(b);
  float best = 1e30f;
  int choice = kFormTwoStage;
  // double precision has one fused form (two stages do not fit); compensated
  // FP32 and the H-AFDA surface run on the split pair only
  const int forms[5] = {kFormPerShot, kFormStreams, kFormSplit, kFormTwoStage, kFormOneStage};
  const int nforms = (b->precision == VI_F32C || b->afda) ? 3 : sizeof(T) == 4 ? 5 : 4;
  for (int f = 0; f < nforms; ++f) {
    const int form = forms[f];
    float ms = 0;
    int rc;
    if (form == kFormPerShot) {
      rc = time_marginal([&](int a, int e) { return per_shot_steps(b, a, e, st); }, st, b->max_nt, &ms);
    } else if (form == kFormStreams) {
      rc = time_marginal([&](int a, int e) { return streams_steps(b, a, e, st); }, st, b->max_nt, &ms);
    } else {
      BatchDev<T> bd;
      rc = prepare<T>(b, form, st, bd);
      if (rc == VI_ERR_ARG) continue;
      if (rc) return rc;
      rc = time_marginal([&](int a, int e) { return launch_steps<T>(b, bd, form, a, e, st); }, st, b->max_nt, &ms);
    }
    if (rc) return rc;
    if (ms < best) {
      best = ms;
      choice = form;
    }
  }
  b->form = choice;
  {
    std::lock_guard<std::mutex> lk(g_tuned_mu);
    g_tuned[key] = choice;
  }
  // tuning advanced the shots: put them back at rest
  return reset_state<T>(b, st);
}

// Sets kernel attributes (outside a capture) for a form.
template <typename T>
static int set_up_form(vi_batch *b, const BatchDev<T> &bd, int form, cudaStream_t st) {
  if (form == kFormSplit)
    return launch_split_stress_batch<T>(b->kind, b->nsls, b->precision == VI_F32C, b->afda, bd, 0, 0, st, false);
  return launch_fused_tma_batch<T>(b->kind, b->nsls, bd, 0, 0, b->nsm, form == kFormTwoStage, st);
}

template <typename T>
static int run_impl(vi_batch *b, int flags, cudaStream_t st) {
  for (int i = 0; i < b->n; ++i)
    if (!b->bound[i]) return set_error(VI_ERR_STATE, "batch: shot " + std::to_string(i) + " is not bound");
  int rc = cuda_check(cudaSetDevice(b->device), "cudaSetDevice");
  if (rc) return rc;
  const bool use_graph = (flags & VI_BATCH_NO_GRAPH) == 0;
  if (b->form < 0 || (flags & VI_BATCH_RETUNE)) {
    if (flags & VI_BATCH_RETUNE) {
      std::lock_guard<std::mutex> lk(g_tuned_mu);
      g_tuned.erase(tune_key(b));
    }
    if ((rc = tune<T>(b, st))) return rc;
    b->dirty = true;
  }
  const int form = b->form;
  for (int i = 0; i < b->n; ++i)
    if ((rc = vi_plan_reset(b->plans[i], st))) return rc;
  if (form == kFormPerShot || form == kFormStreams) {
    set_order(b);
    for (int i = 0; i < b->n; ++i) b->plans[i]->psi_cur = 0;
    if ((rc = form == kFormStreams ? streams_steps(b, 0, b->max_nt, st) : per_shot_steps(b, 0, b->max_nt, st)))
      return rc;
    return cuda_check(cudaGetLastError(), "batch run");
  }
  if (b->dirty || !use_graph || b->graph_form != form) {
    BatchDev<T> bd;
    if ((rc = prepare<T>(b, form, st, bd))) return rc;
    if (b->graph) {
      cudaGraphExecDestroy(b->graph);
      b->graph = nullptr;
    }
    if (use_graph) {
      if ((rc = set_up_form<T>(b, bd, form, st))) return rc;
      cudaStream_t cs;
      if ((rc = cuda_check(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking), "capture stream")))
        return rc;
      cudaGraph_t g = nullptr;
      rc = cuda_check(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal), "begin capture");
      if (!rc) {
        const int lrc = launch_steps<T>(b, bd, form, 0, b->max_nt, cs);
        rc = cuda_check(cudaStreamEndCapture(cs, &g), "end capture");
        if (!rc) rc = lrc;
      }
      if (!rc) rc = cuda_check(cudaGraphInstantiate(&b->graph, g, 0), "instantiate graph");
      if (g) cudaGraphDestroy(g);
      cudaStreamDestroy(cs);
      if (rc) return rc;
      b->graph_form = form;
      b->dirty = false;
    } else {
      if ((rc = launch_steps<T>(b, bd, form, 0, b->max_nt, st))) return rc;
    }
  }
  if (use_graph && (rc = cuda_check(cudaGraphLaunch(b->graph, st), "graph launch"))) return rc;
  // shots with an odd step count end in the plan's copy: bring them back
  // (the fused forms ping-pong the whole state, the split pair only the
  // TTI memory variables)
  for (int i = 0; i < b->n; ++i) {
    if (b->nt[i] % 2 == 0) continue;
    if (form == kFormSplit && b->kind != VI_MEDIUM_TTI) continue;
    vi_plan *p = b->plans[i];
    const size_t np = (size_t)p->cfg.nx * p->cfg.nz;
    T *alt = (T *)p->alt;
    const vi_fields &f = b->fields[i];
    if (form != kFormSplit) {
      void *user[5] = {f.vx, f.vz, f.sxx, f.szz, f.sxz};
      for (int q = 0; q < 5; ++q)
        if ((rc = cuda_check(cudaMemcpyAsync(user[q], alt + q * np, np * sizeof(T), cudaMemcpyDeviceToDevice, st),
                             "copy back fields")))
          return rc;
    }
    for (int q = 0; q < 3 * p->cfg.nsls; ++q)
      if ((rc = cuda_check(cudaMemcpyAsync((T *)f.m + q * f.m_plane_stride, alt + (5 + q) * np,
                                           np * sizeof(T), cudaMemcpyDeviceToDevice, st),
                           "copy back memory variables")))
        return rc;
  }
  // the fused forms do not fold the finite check into their stress pass:
  // check every shot's stresses once at the end of the run
  if (form != kFormSplit)
    for (int i = 0; i < b->n; ++i) {
      const vi_fields &f = b->fields[i];
      const vi_plan *p = b->plans[i];
      if ((rc = launch_finite_check<T>(f.sxx, f.szz, f.sxz, (long long)p->cfg.nx * p->cfg.nz, b->err, b->nsm, st)))
        return rc;
    }
  return cuda_check(cudaGetLastError(), "batch run");
}

}  // namespace vb

using namespace vb;

extern "C" int vi_batch_create(const vi_config *cfgs, int32_t nshots, vi_batch **out) {
  if (!out || !cfgs || nshots <= 0) return set_error(VI_ERR_ARG, "batch: bad arguments");
  *out = nullptr;
  for (int i = 1; i < nshots; ++i)
    if (cfgs[i].medium != cfgs[0].medium || cfgs[i].precision != cfgs[0].precision ||
        cfgs[i].nsls != cfgs[0].nsls)
      return set_error(VI_ERR_ARG, "batch: shots must share medium kind, precision and nsls");
  vi_batch *b = new vi_batch();
  b->n = nshots;
  b->kind = cfgs[0].medium;
  b->precision = cfgs[0].precision;
  b->nsls = cfgs[0].nsls;
  cudaGetDevice(&b->device);
  if (cudaDeviceGetAttribute(&b->nsm, cudaDevAttrMultiProcessorCount, b->device) != cudaSuccess)
    b->nsm = 148;
  for (int i = 0; i < nshots; ++i)
    if ((cfgs[i].nx % 4) != 0) {
      delete b;
      return set_error(VI_ERR_ARG, "batch: every shot needs nx % 4 == 0 (TMA-staged tiles)");
    }
  b->plans.assign(nshots, nullptr);
  for (int i = 0; i < nshots; ++i) {
    int rc = vi_plan_create(&cfgs[i], &b->plans[i]);
    if (rc) {
      vi_batch_destroy(b);
      return rc;
    }
    b->afda |= cfgs[i].free_surface == kFsAfda;
  }
  b->med.assign(nshots, vi_medium{});
  b->fields.assign(nshots, vi_fields{});
  b->nt.assign(nshots, 0);
  b->src.resize(nshots);
  b->rec.resize(nshots);
  b->shot.assign(nshots, vi_shot{});
  b->bound.assign(nshots, 0);
  if (cudaMalloc(&b->err, 16) != cudaSuccess || cudaMemset(b->err, 0, 16) != cudaSuccess) {
    cudaGetLastError();
    vi_batch_destroy(b);
    return set_error(VI_ERR_BUDGET, "batch: error word allocation failed");
  }
  *out = b;
  return VI_OK;
}

extern "C" int vi_batch_destroy(vi_batch *b) {
  if (!b) return VI_OK;
  if (b->graph) cudaGraphExecDestroy(b->graph);
  if (b->dev) cudaFree(b->dev);
  if (b->err) cudaFree(b->err);
  for (cudaStream_t q : b->streams)
    if (q) cudaStreamDestroy(q);
  for (cudaEvent_t e : b->joins)
    if (e) cudaEventDestroy(e);
  if (b->fork) cudaEventDestroy(b->fork);
  for (vi_plan *p : b->plans) vi_plan_destroy(p);
  delete b;
  return VI_OK;
}

extern "C" int vi_batch_set_shot(vi_batch *b, int32_t i, const vi_medium *med_dev,
                                 const vi_fields *fields_dev, const vi_shot *shot, int32_t nt) {
  if (!b || i < 0 || i >= b->n) return set_error(VI_ERR_ARG, "batch: bad shot index");
  if (nt < 0) return set_error(VI_ERR_ARG, "batch: negative step count");
  vi_plan *p = b->plans[i];
  int rc = check_medium(p, med_dev);
  if (rc) return rc;
  rc = check_fields(p, fields_dev);
  if (rc) return rc;
  b->med[i] = *med_dev;
  b->fields[i] = *fields_dev;
  b->nt[i] = nt;
  vi_shot s{};
  if (shot) {
    s = *shot;
    b->src[i].assign(shot->src_host, shot->src_host + (shot->nsrc > 0 ? shot->nsrc : 0));
    b->rec[i].assign(shot->rec_host, shot->rec_host + (shot->nrec > 0 ? shot->nrec : 0));
    s.src_host = b->src[i].data();
    s.rec_host = b->rec[i].data();
  }
  b->shot[i] = s;
  b->bound[i] = 1;
  b->dirty = true;
  return VI_OK;
}

extern "C" int vi_batch_run(vi_batch *b, int32_t flags, void *stream) {
  if (!b) return set_error(VI_ERR_ARG, "batch is NULL");
  NvtxRange nr("vi_batch_run");
  cudaStream_t st = (cudaStream_t)stream;
  return b->precision == VI_F64 ? run_impl<double>(b, flags, st) : run_impl<float>(b, flags, st);
}

extern "C" int vi_batch_status(vi_batch *b, void *stream, int32_t *kernel_form) {
  if (!b) return set_error(VI_ERR_ARG, "batch is NULL");
  int rc = cuda_check(cudaStreamSynchronize((cudaStream_t)stream), "batch status");
  if (rc) return rc;
  if (kernel_form) *kernel_form = b->form;
  int flag = 0;
  rc = cuda_check(cudaMemcpy(&flag, b->err, sizeof(int), cudaMemcpyDeviceToHost), "read error word");
  if (rc) return rc;
  // the per-shot forms report through each shot's plan
  for (int i = 0; i < b->n; ++i) {
    int pf = 0;
    if ((rc = cuda_check(cudaMemcpy(&pf, b->plans[i]->errflag, sizeof(int), cudaMemcpyDeviceToHost),
                         "read plan error word")))
      return rc;
    if (pf) cudaMemset(b->plans[i]->errflag, 0, sizeof(int));
    flag |= pf;
  }
  if (flag) {
    cudaMemset(b->err, 0, sizeof(int));
    if (flag & kErrTimeout) return set_error(VI_ERR_TIMEOUT, "batch: a bounded device wait gave up");
    return set_error(VI_ERR_NONFINITE, "batch: a stress value came out NaN or infinite");
  }
  return VI_OK;
}
