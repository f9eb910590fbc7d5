// noalloc.cu — vi_step_noalloc: the plain in-place step (the path of
// vi_step kernel_variant 1) with every device buffer it needs beyond the
// plan, the medium and the caller's fields taken from one file-scope static
// device array instead of the plan's grow-on-demand workspace.
//
// Who needs it: callers that must not allocate or free device memory in the
// middle of a run.  cudaMalloc / cudaFree can synchronize the device and so
// stall every other stream of a serving process that shares the GPU; a
// process whose HBM is fully reserved by a memory pool cannot grow; and code
// running on a thread that holds an allocator's lock must not re-enter it.
// vi_step's plain path allocates its six strain planes and its source /
// receiver lists on first use; this entry point never does.
//
// Contract:
//  * The static array holds VI_NOALLOC_SCRATCH_BYTES bytes: the six strain
//    planes (6 * nx * nz reals of the plan's precision) followed by the
//    source list (int4 + one amplitude per source) and the receiver list
//    (int2 per receiver), each block 256-byte aligned.  Larger problems are
//    rejected with VI_ERR_ARG before anything runs.
//  * Set-up: every call, with the plan's device current, looks up the
//    array's device address in the current context with
//    cudaGetSymbolAddress (a table lookup once the module is loaded), so the
//    address cannot go stale across a cudaDeviceReset or a change of
//    context.  The first call on a device loads the module that holds the
//    array: make that first call before any stream capture.
//  * With sources or receivers, the call stages their lists from its own
//    stack frame and blocks the host thread on the stream until they are
//    on the device (cudaStreamSynchronize).
//  * What must start at zero: the strain planes outside the update region,
//    which the neighbour averages read and the strain pass never writes.
//    Each call clears all six planes with cudaMemsetAsync on its stream
//    before its first step, because another grid may have used the array.
//  * The array is one per device and per process: calls that overlap in
//    time on one device (different streams, threads or plans) race on it.
//    Serialize them.
#include <cstdint>
#include <string>

#include "plain.cuh"
#include "plan.cuh"

namespace vb {

static __device__ __align__(256) unsigned char g_noalloc_scratch[VI_NOALLOC_SCRATCH_BYTES];

namespace {

constexpr int kMaxSources = 256;  // host packing buffer on the stack

// Device address of the static array in the current context.  In host
// code the array's name is only a host-side stand-in: a kernel given
// &g_noalloc_scratch would fault or, where the GPU can reach host memory,
// write the wrong memory, so the address always comes from the runtime.
int scratch_address(void **out) {
  void *ptr = nullptr;
  const int rc = cuda_check(cudaGetSymbolAddress(&ptr, g_noalloc_scratch), "cudaGetSymbolAddress");
  if (rc) return rc;
  *out = ptr;
  return VI_OK;
}

size_t align256(size_t n) { return (n + 255) / 256 * 256; }

bool inside(const vi_config &c, int i, int j) { return i >= L && i < c.nx - L && j >= L && j < c.nz - L; }

template <typename T>
int noalloc_impl(vi_plan *p, const vi_medium *m, vi_fields *f, const vi_shot *s, int it0, int nsteps,
                 cudaStream_t st) {
  int rc = check_medium(p, m);
  if (rc) return rc;
  if ((rc = check_fields(p, f))) return rc;
  if (p->cfg.precision == VI_F32C)
    return set_error(VI_ERR_ARG, "noalloc: the plain step has no compensated FP32 (VI_F32C) form");
  if (nsteps < 0) return set_error(VI_ERR_ARG, "nsteps must be >= 0");
  const int nsrc = s ? s->nsrc : 0, nrec = s ? s->nrec : 0;
  if (nsrc < 0 || nrec < 0) return set_error(VI_ERR_ARG, "negative source/receiver count");
  if (nsrc > kMaxSources) return set_error(VI_ERR_ARG, "noalloc: at most 256 sources");
  if (nsrc > 0 && (!s->src_host || !s->wavelet_dev || s->wavelet_nt < 0))
    return set_error(VI_ERR_ARG, "sources need src_host and wavelet_dev");
  if (nrec > 0 && !s->rec_host) return set_error(VI_ERR_ARG, "receivers need rec_host");
  if (nrec > 0 && s->traces_nt > 0 && !s->traces_dev) return set_error(VI_ERR_ARG, "receivers need traces_dev");
  const vi_config &c = p->cfg;
  const size_t np = (size_t)c.nx * c.nz;
  const size_t o_src = align256(6 * np * sizeof(T));
  const size_t o_amp = o_src + align256((size_t)nsrc * sizeof(int4));
  const size_t o_rec = o_amp + align256((size_t)nsrc * sizeof(T));
  const size_t need = o_rec + (size_t)nrec * sizeof(int2);
  if (need > (size_t)VI_NOALLOC_SCRATCH_BYTES)
    return set_error(VI_ERR_ARG, "noalloc: needs " + std::to_string(need) + " bytes of static scratch, limit " +
                                     std::to_string((size_t)VI_NOALLOC_SCRATCH_BYTES) +
                                     " (6 strain planes + source/receiver lists)");
  int4 hs[kMaxSources];
  T ha[kMaxSources];
  for (int q = 0; q < nsrc; ++q) {
    const vi_source &v = s->src_host[q];
    if (!inside(c, v.i, v.j)) return set_error(VI_ERR_ARG, "source " + std::to_string(q) + " outside the update region");
    if (v.kind < VI_SRC_EXPLOSIVE || v.kind > VI_SRC_FORCE_Z) return set_error(VI_ERR_ARG, "unknown source kind");
    hs[q] = make_int4(v.i, v.j, v.kind, 0);
    ha[q] = (T)v.amp;
  }
  for (int r = 0; r < nrec; ++r) {
    const vi_receiver &v = s->rec_host[r];
    if (!inside(c, v.i, v.j)) return set_error(VI_ERR_ARG, "receiver " + std::to_string(r) + " outside the update region");
  }
  if ((rc = cuda_check(cudaSetDevice(p->device), "cudaSetDevice"))) return rc;
  void *base = nullptr;
  if ((rc = scratch_address(&base))) return rc;
  unsigned char *b = (unsigned char *)base;
  if ((rc = cuda_check(cudaMemsetAsync(b, 0, 6 * np * sizeof(T), st), "noalloc: clear strain planes"))) return rc;
  if (nsrc > 0) {
    if ((rc = cuda_check(cudaMemcpyAsync(b + o_src, hs, nsrc * sizeof(int4), cudaMemcpyHostToDevice, st),
                         "noalloc: copy sources")))
      return rc;
    if ((rc = cuda_check(cudaMemcpyAsync(b + o_amp, ha, nsrc * sizeof(T), cudaMemcpyHostToDevice, st),
                         "noalloc: copy amplitudes")))
      return rc;
  }
  if (nrec > 0)  // vi_receiver is {int32 i, int32 j}: the int2 layout the kernels read
    if ((rc = cuda_check(cudaMemcpyAsync(b + o_rec, s->rec_host, nrec * sizeof(int2), cudaMemcpyHostToDevice, st),
                         "noalloc: copy receivers")))
      return rc;
  if (nsrc > 0 || nrec > 0)  // the packed source lists live on this stack frame
    if ((rc = cuda_check(cudaStreamSynchronize(st), "noalloc: stage lists"))) return rc;
  StepArgs<T> a = make_args<T>(p, m, f);
  PlainExtras<T> x;
  x.scratch = (T *)b;
  x.fs = c.free_surface;
  x.src = (const int4 *)(b + o_src);
  x.amp = (const T *)(b + o_amp);
  x.nsrc = nsrc;
  x.wavelet = nsrc ? (const T *)s->wavelet_dev : nullptr;
  x.wnt = nsrc ? s->wavelet_nt : 0;
  x.rec = (const int2 *)(b + o_rec);
  x.nrec = nrec;
  x.traces = nrec ? (T *)s->traces_dev : nullptr;
  x.tnt = nrec ? s->traces_nt : 0;
  // in place on the plan's current psi set, as vi_step's plain path
  const int cur = p->psi_cur;
  if (a.psix) a.psix = a.psix_o = (T *)p->psix + cur * kPsiPerSet * p->psix_plane;
  if (a.psiz) a.psiz = a.psiz_o = (T *)p->psiz + cur * kPsiPerSet * p->psiz_plane;
  for (int k = 0; k < nsteps; ++k) plain_step<T>(a, x, c.medium, it0 + k, st);
  p->last_kernel = 1;
  return cuda_check(cudaGetLastError(), "noalloc step launch");
}

}  // namespace
}  // namespace vb

using namespace vb;

extern "C" int vi_step_noalloc(vi_plan *p, const vi_medium *med, vi_fields *f, const vi_shot *shot,
                               int32_t it0, int32_t nsteps, void *stream) {
  if (!p) return set_error(VI_ERR_ARG, "plan is NULL");
  cudaStream_t st = (cudaStream_t)stream;
  return p->cfg.precision == VI_F64 ? noalloc_impl<double>(p, med, f, shot, it0, nsteps, st)
                                    : noalloc_impl<float>(p, med, f, shot, it0, nsteps, st);
}
