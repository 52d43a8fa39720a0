// C-ABI of the B200 FDTD engine: device buffers, launches, CUDA-graph replay
// of the step loop, read-back and checkpointing.
//
// The reference's run() (src/simulation/simulation_hd.cu:106-257) builds ~47
// launches per step from per-object agencies and runs them on the default
// stream.  Here one step is 2-5 launches on the handle's own stream, captured
// into a CUDA graph of `graph_steps` steps and replayed; the step index lives
// in device memory (bumped once per captured chunk) so a captured chunk is
// valid for any starting step.
#include <cuda_runtime.h>
#include <unistd.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "handle.h"
#include "kernels.cuh"
#include "labc.cuh"
#include "xfb_internal.h"

using namespace xfb;

namespace {
thread_local std::string g_err;
}

namespace xfb {

int set_err(xfb_handle* h, int code, const std::string& m) {
  if (h) h->err = m;
  g_err = m;
  return code;
}

int cuda_err(xfb_handle* h, cudaError_t e, const char* what) {
  return set_err(h, XFB_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}



void free_device(xfb_handle* h) {
  for (auto& kv : h->graphs) cudaGraphExecDestroy(kv.second);
  h->graphs.clear();
  for (auto& b : h->bufs)
    if (b.owner) cudaFree(b.p);
  h->bufs.clear();
  h->bytes = 0;
  h->arena = nullptr;
  h->arena_left = 0;
  h->movie_out.clear();
  h->movie_frames.clear();
  h->labc_on = false;
  h->labc_w = nullptr;
  h->labc_hist = nullptr;
  h->step_err = nullptr;
  h->ade_runs = nullptr;
  h->n_ade_runs = -1;
  h->rb_dev = nullptr;  // one of bufs
  for (int q = 0; q < 2; ++q) {
    if (h->rb_host[q]) cudaFreeHost(h->rb_host[q]);
    if (h->rb_ev[q]) cudaEventDestroy(h->rb_ev[q]);
    h->rb_host[q] = nullptr;
    h->rb_ev[q] = nullptr;
  }
  h->inited = false;
}

namespace {
constexpr size_t kArenaMax = 32u << 20;     // larger buffers get their own cudaMalloc
constexpr size_t kArenaChunk = 256u << 20;  // chunk the smaller ones are carved from
constexpr size_t kAlign = 256;

// One cudaMalloc of `bytes`, listed as an owner buffer (freed with the device
// state; not part of the checkpoint state, whose parts are listed separately).
int device_malloc(xfb_handle* h, void** out, size_t bytes) {
  void* p = nullptr;
  const cudaError_t e = cudaMalloc(&p, bytes);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return set_err(h, XFB_ERR_OOM, "cudaMalloc of " + std::to_string(bytes) + " bytes failed: " + cudaGetErrorString(e));
  }
  h->bufs.push_back({p, 0, false, true});
  h->bytes += bytes;
  *out = p;
  return XFB_OK;
}
}  // namespace

// A zeroed device buffer of `bytes`, listed (with `state`) for the checkpoint.
// Buffers up to kArenaMax come out of the handle's current chunk.  While host
// threads fault in large result arrays (xfb_host_prefault), every cudaMalloc
// waits on the process's memory map, so init keeps their number small.
int alloc(xfb_handle* h, void** out, size_t bytes, bool state) {
  *out = nullptr;
  if (bytes == 0) return XFB_OK;
  void* p = nullptr;
  if (bytes <= kArenaMax) {
    const size_t need = (bytes + kAlign - 1) / kAlign * kAlign;
    if (h->arena_left < need) {
      void* chunk;
      if (int rc = device_malloc(h, &chunk, kArenaChunk)) return rc;
      h->arena = static_cast<char*>(chunk);
      h->arena_left = kArenaChunk;
    }
    p = h->arena;
    h->arena += need;
    h->arena_left -= need;
  } else if (int rc = device_malloc(h, &p, bytes)) {
    return rc;
  }
  const cudaError_t e = cudaMemsetAsync(p, 0, bytes, h->stream);
  if (e != cudaSuccess) return cuda_err(h, e, "cudaMemsetAsync");
  h->bufs.push_back({p, bytes, state, false});
  *out = p;
  return XFB_OK;
}

int alloc_block(xfb_handle* h, void** out, int n, size_t bytes, bool state) {
  for (int q = 0; q < n; ++q) out[q] = nullptr;
  if (n <= 0 || bytes == 0) return XFB_OK;
  const size_t each = (bytes + kAlign - 1) / kAlign * kAlign;
  void* base;
  if (int rc = device_malloc(h, &base, each * n)) return rc;
  const cudaError_t e = cudaMemsetAsync(base, 0, each * n, h->stream);
  if (e != cudaSuccess) return cuda_err(h, e, "cudaMemsetAsync");
  for (int q = 0; q < n; ++q) {
    out[q] = static_cast<char*>(base) + q * each;
    h->bufs.push_back({out[q], bytes, state, false});
  }
  return XFB_OK;
}


int copy(xfb_handle* h, void* dst, const void* src, size_t bytes, cudaMemcpyKind kind) {
  if (bytes == 0) return XFB_OK;
  XFB_CUDA(h, cudaMemcpyAsync(dst, src, bytes, kind, h->stream));
  XFB_CUDA(h, cudaStreamSynchronize(h->stream));
  if (kind == cudaMemcpyHostToDevice) h->h2d_bytes += static_cast<long long>(bytes);
  if (kind == cudaMemcpyDeviceToHost) h->d2h_bytes += static_cast<long long>(bytes);
  return XFB_OK;
}

long long roundup(long long v, long long m) { return (v + m - 1) / m * m; }

bool fused(const xfb_handle* h) { return h->path == XFB_PATH_FUSED; }
bool plain(const xfb_handle* h) { return h->path == XFB_PATH_PLAIN; }
// field set holding the state after h->step steps
int cur_set(const xfb_handle* h) { return fused(h) ? static_cast<int>(h->step & 1) : 0; }
void* field_ptr(const xfb_handle* h, int set, int q) { return set ? h->f1[q] : h->f[q]; }

// element offset of component index (i, j, k) in the padded layout
long long off3(const xfb_handle* h, int i, int j, int k) { return i * h->sx + j * h->sy + k; }

void comp_shape(const Compiled& c, int f, int s[3]) {
  s[0] = c.nx + (f == XFB_EY || f == XFB_EZ || f == XFB_HX ? 1 : 0);
  s[1] = c.ny + (f == XFB_EX || f == XFB_EZ || f == XFB_HY ? 1 : 0);
  s[2] = c.nz + (f == XFB_EX || f == XFB_EY || f == XFB_HZ ? 1 : 0);
  if (c.dim == 2) s[2] = 1;
}

int nf_face_points(const Compiled& c, int face) {
  const FaceGeom g = face_geom(c, face);
  return g.ni * g.nj * g.nk;
}

// ---------------------------------------------------------------------------
int launches_per_step(const xfb_handle* h) {
  const Compiled& c = h->c;
  if (plain(h)) {
    int faces = 0;
    for (int f = 0; f < 6; ++f) faces += c.pml[f] > 0;
    return 6 + 2 * faces + (c.tfsf_on ? 24 : 0) + (c.nf_on ? 1 : 0) + (c.td_on ? 2 : 0) + (c.probes.empty() ? 0 : 1) +
           static_cast<int>(c.movies.size());
  }
  int bulk = 2;
  if (fused(h)) {
    bulk = c.dim == 2 ? 1
                      : (h->n_step_items[step_tile_index(h->tj)] > 0 ? 1 : 0) + (h->ade_deferred ? 1 : 0) +
                            (h->lines_on ? 1 : 0);  // k_tfsf_lines
  }
  if (h->tb_on) return 1;  // one blocked launch per tb_steps steps, probes recorded inside
  return bulk + (c.nf_on ? 1 : 0) + (c.td_on ? 2 : 0) + (c.probes.empty() ? 0 : 1) +
         static_cast<int>(c.movies.size());
}

int batch_err(xfb_batch* b, int code, const std::string& m) {
  if (b) b->err = m;
  g_err = m;
  return code;
}

void batch_free(xfb_batch* b) {
  for (auto& kv : b->graphs) cudaGraphExecDestroy(kv.second);
  b->graphs.clear();
  void* ps[11] = {b->scenes,  b->maps,           b->items[0],       b->items[1],       b->items[2],     b->t_dev,
                  b->err_dev, b->pscene_items[0], b->pscene_items[1], b->pscene_items[2], b->queue};  // pitems alias items
  for (void* p : ps) cudaFree(p);
  b->scenes = b->maps = nullptr;
  for (int t = 0; t < kStepTileCount; ++t) {
    b->items[t] = nullptr;
    b->n_items[t] = 0;
    b->pitems[t] = nullptr;
    b->pscene_items[t] = nullptr;
  }
  b->queue = nullptr;
  b->t_dev = nullptr;
  b->err_dev = nullptr;
  b->inited = false;
}

// A handle that a batch steps may only be read, not stepped or re-sized.
int not_batched(xfb_handle* h) {
  if (h && h->batch) return set_err(h, XFB_ERR_STATE, "the handle is stepped by a batch (xfb_batch_destroy releases it)");
  return XFB_OK;
}

// Join the handle's prefault threads (before any write into caller memory).
void wait_prefault(xfb_handle* h) {
  for (auto& t : h->prefault) t.join();
  h->prefault.clear();
  h->pf_queue.clear();
  h->pf_active = 0;
}

// A prefault worker: takes queued parts until none is left and takes the
// write fault of every page of each by an atomic add of zero to one byte of
// the page inside the part (contents unchanged; one fault per huge page where
// the range is madvised for them).
void prefault_worker(xfb_handle* h) {
  const uintptr_t page = static_cast<uintptr_t>(sysconf(_SC_PAGESIZE));
  for (;;) {
    std::pair<char*, char*> r;
    {
      std::lock_guard<std::mutex> lk(h->pf_mu);
      if (h->pf_queue.empty()) {
        --h->pf_active;
        return;
      }
      r = h->pf_queue.back();
      h->pf_queue.pop_back();
    }
    char* p = r.first;
    while (p < r.second) {
      __atomic_fetch_add(p, static_cast<char>(0), __ATOMIC_RELAXED);
      p = reinterpret_cast<char*>((reinterpret_cast<uintptr_t>(p) / page + 1) * page);
    }
  }
}

// Queue [ptr, ptr + bytes) for the handle's prefault pool (64 MiB parts) and
// start workers up to the pool size; false when that fails.
bool queue_prefault(xfb_handle* h, void* ptr, size_t bytes) {
  if (!bytes) return true;
  const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
  const int max_threads = static_cast<int>(std::max(1u, std::min(12u, hw * 3 / 4)));
  const size_t part = 64u << 20;
  char* base = static_cast<char*>(ptr);
  try {
    std::lock_guard<std::mutex> lk(h->pf_mu);
    for (size_t o = 0; o < bytes; o += part) h->pf_queue.emplace_back(base + o, base + std::min(bytes, o + part));
    while (h->pf_active < max_threads) {
      h->prefault.emplace_back(prefault_worker, h);
      ++h->pf_active;
    }
  } catch (const std::exception&) {
    wait_prefault(h);
    return false;
  }
  return true;
}

// Fault in a large caller destination with the pool before a read-back writes
// it: the pool takes fresh pages several times faster than the read-back's
// own writes would.  A failure only leaves the faults to the read-back.
void prefault_now(xfb_handle* h, void* ptr, size_t bytes) {
  if (bytes >= (8u << 20)) queue_prefault(h, ptr, bytes);
  wait_prefault(h);
}

int check_handle(xfb_handle* h, bool need_init) {
  if (!h) return set_err(nullptr, XFB_ERR_INVALID, "null handle");
  if (need_init && !h->inited) return set_err(h, XFB_ERR_STATE, "handle not initialised (call xfb_init or xfb_run)");
  if (h->inited) {
    cudaError_t e = cudaSetDevice(h->device);
    if (e != cudaSuccess) return cuda_err(h, e, "cudaSetDevice");
  }
  return XFB_OK;
}

}  // namespace xfb

// ---------------------------------------------------------------------------
// Scratch of xfb_far_field_static: a fixed device array instead of per-call
// allocations, for callers that must not allocate device memory after start-up.
// Layout: theta[kFarStaticMaxAngles], phi[kFarStaticMaxAngles],
// out[4 * kFarStaticMaxAngles] (192 KiB per device that loads the library, held
// until the process exits).  Device code could name the array directly; host
// code only holds a host-side stand-in for it, so the device address is fetched
// with cudaGetSymbolAddress once per device, with that device current.
namespace {
constexpr int kFarStaticMaxAngles = XFB_FAR_FIELD_STATIC_MAX_ANGLES;
static __device__ __align__(256) double g_far_scratch[6 * kFarStaticMaxAngles];

std::mutex g_far_scratch_mu;
double* g_far_scratch_dev[256] = {};  // per device ordinal

int far_scratch_for(xfb_handle* h, double** out) {
  if (h->device < 0 || h->device >= 256) return set_err(h, XFB_ERR_RANGE, "device ordinal outside the scratch table");
  std::lock_guard<std::mutex> lock(g_far_scratch_mu);
  if (!g_far_scratch_dev[h->device]) {
    double* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(reinterpret_cast<void**>(&p), g_far_scratch);
    if (e != cudaSuccess) return cuda_err(h, e, "cudaGetSymbolAddress(far-field scratch)");
    g_far_scratch_dev[h->device] = p;
  }
  *out = g_far_scratch_dev[h->device];
  return XFB_OK;
}
}  // namespace

extern "C" {

int xfb_abi_version(void) { return XFB_ABI_VERSION; }

const char* xfb_status_string(int s) {
  switch (s) {
    case XFB_OK: return "ok";
    case XFB_ERR_INVALID: return "invalid argument";
    case XFB_ERR_CUDA: return "CUDA error";
    case XFB_ERR_OOM: return "out of memory";
    case XFB_ERR_STATE: return "invalid state";
    case XFB_ERR_RANGE: return "out of range";
    case XFB_ERR_NUMERIC: return "non-finite values";
    case XFB_ERR_TIMEOUT: return "device wait timed out";
    case XFB_ERR_NO_DEVICE: return "no CUDA device";
  }
  return "unknown status";
}

const char* xfb_last_error(const xfb_handle* h) { return h ? h->err.c_str() : g_err.c_str(); }

int xfb_create(const xfb_scene* scene, xfb_handle** out) {
  if (!scene || !out) return set_err(nullptr, XFB_ERR_INVALID, "null scene or output pointer");
  *out = nullptr;
  std::unique_ptr<xfb_handle> h(new (std::nothrow) xfb_handle());
  if (!h) return set_err(nullptr, XFB_ERR_OOM, "host allocation failed");
  std::string err;
  int rc;
  try {
    rc = compile_scene(*scene, h->c, &err);
  } catch (const std::bad_alloc&) {
    return set_err(nullptr, XFB_ERR_OOM, "host allocation failed while compiling the scene");
  }
  if (rc) return set_err(nullptr, rc, err);
  h->esize = h->c.prec == XFB_FP64 ? 8 : 4;
  *out = h.release();
  g_err.clear();
  return XFB_OK;
}

int xfb_create_from_arrays(const xfb_core_arrays* arrays, xfb_handle** out) {
  if (!arrays || !out) return set_err(nullptr, XFB_ERR_INVALID, "null arrays or output pointer");
  *out = nullptr;
  std::unique_ptr<xfb_handle> h(new (std::nothrow) xfb_handle());
  if (!h) return set_err(nullptr, XFB_ERR_OOM, "host allocation failed");
  std::string err;
  int rc;
  try {
    rc = compile_arrays(*arrays, h->c, &err);
  } catch (const std::bad_alloc&) {
    return set_err(nullptr, XFB_ERR_OOM, "host allocation failed while reading the arrays");
  }
  if (rc) return set_err(nullptr, rc, err);
  h->esize = h->c.prec == XFB_FP64 ? 8 : 4;
  *out = h.release();
  g_err.clear();
  return XFB_OK;
}

int xfb_destroy(xfb_handle* h) {
  if (!h) return XFB_OK;
  if (int rc = not_batched(h)) return rc;
  wait_prefault(h);
  if (h->device >= 0) {
    cudaSetDevice(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    free_device(h);
    if (h->stream) cudaStreamDestroy(h->stream);
  }
  delete h;
  return XFB_OK;
}

int xfb_set_launch_hint(xfb_handle* h, const unsigned grid[3], const unsigned block[3]) {
  if (!h || !grid || !block) return set_err(h, XFB_ERR_INVALID, "null argument");
  for (int a = 0; a < 3; ++a) {
    h->hint_grid[a] = grid[a] ? grid[a] : 1;
    h->hint_block[a] = block[a] ? block[a] : 1;
  }
  const unsigned threads = h->hint_block[0] * h->hint_block[1] * h->hint_block[2];
  if (threads % 32 == 0 && threads <= 1024 && threads >= 32) {
    h->tk = 32;
    h->tj = static_cast<int>(threads / 32);
  }
  for (auto& kv : h->graphs) cudaGraphExecDestroy(kv.second);
  h->graphs.clear();
  return XFB_OK;
}

int xfb_set_device(xfb_handle* h, int ordinal) {
  if (!h) return set_err(nullptr, XFB_ERR_INVALID, "null handle");
  if (h->device >= 0) return set_err(h, XFB_ERR_STATE, "device already chosen (set it before the first xfb_init)");
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
    cudaGetLastError();
    return set_err(h, XFB_ERR_NO_DEVICE, "no CUDA device available");
  }
  if (ordinal < 0 || ordinal >= n) return set_err(h, XFB_ERR_RANGE, "device ordinal out of range");
  XFB_CUDA(h, cudaSetDevice(ordinal));
  h->device = ordinal;
  XFB_CUDA(h, cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
  return XFB_OK;
}

int xfb_set_kernel_path(xfb_handle* h, int path) {
  if (!h) return set_err(nullptr, XFB_ERR_INVALID, "null handle");
  if (path < XFB_PATH_AUTO || path > XFB_PATH_PLAIN) return set_err(h, XFB_ERR_INVALID, "unknown kernel path");
  if (h->inited) return set_err(h, XFB_ERR_STATE, "set the kernel path before xfb_init");
  h->path = path;
  return XFB_OK;
}

int xfb_set_temporal_block(xfb_handle* h, int steps) {
  if (!h) return set_err(nullptr, XFB_ERR_INVALID, "null handle");
  if (steps < 0 || (steps > 0 && (steps % 2 == 0 || steps > 31)))
    return set_err(h, XFB_ERR_INVALID, "steps per launch must be 0 (off) or odd, at most 31");
  if (h->inited) return set_err(h, XFB_ERR_STATE, "set the temporal blocking before xfb_init");
  h->tb_steps = steps;
  return XFB_OK;
}

int xfb_set_coeff_storage(xfb_handle* h, int storage) {
  if (!h) return set_err(nullptr, XFB_ERR_INVALID, "null handle");
  if (storage < XFB_COEFF_NATIVE || storage > XFB_COEFF_BF16) return set_err(h, XFB_ERR_INVALID, "unknown coefficient storage");
  if (h->inited) return set_err(h, XFB_ERR_STATE, "set the coefficient storage before xfb_init");
  h->coeff_storage = storage;
  return XFB_OK;
}

int xfb_set_graph(xfb_handle* h, int enabled, int steps_per_graph) {
  if (!h) return set_err(nullptr, XFB_ERR_INVALID, "null handle");
  if (steps_per_graph < 1 || steps_per_graph > 4096) return set_err(h, XFB_ERR_INVALID, "steps_per_graph must be in [1, 4096]");
  h->graph_on = enabled ? 1 : 0;
  h->graph_steps = steps_per_graph;
  return XFB_OK;
}

int xfb_prepare_tables(xfb_handle* h, long long total_steps) {
  if (!h) return set_err(nullptr, XFB_ERR_INVALID, "null handle");
  if (total_steps < 0 || total_steps > (1LL << 31)) return set_err(h, XFB_ERR_INVALID, "total_steps out of range");
  size_tables(h->c, total_steps);
  return XFB_OK;
}

int xfb_init(xfb_handle* h, long long total_steps) {
  if (!h) return set_err(nullptr, XFB_ERR_INVALID, "null handle");
  if (int rc = not_batched(h)) return rc;
  h->slab_pending = false;
  if (is_slab(h) && (h->path == XFB_PATH_SPLIT || h->path == XFB_PATH_PLAIN))
    return set_err(h, XFB_ERR_INVALID, "x slabs run on the one-sweep path");
  if (total_steps < 0 || total_steps > (1LL << 31)) return set_err(h, XFB_ERR_INVALID, "total_steps out of range");
  if (h->c.inc_given && total_steps > h->c.inc_steps)
    return set_err(h, XFB_ERR_RANGE, "the run is longer than the incident tables the arrays handed over");
  if (h->device < 0) {
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0) {
      cudaGetLastError();
      return set_err(h, XFB_ERR_NO_DEVICE, "no CUDA device available");
    }
    XFB_CUDA(h, cudaGetDevice(&h->device));
    XFB_CUDA(h, cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
  }
  XFB_CUDA(h, cudaSetDevice(h->device));
  XFB_CUDA(h, cudaStreamSynchronize(h->stream));
  free_device(h);
  size_tables(h->c, total_steps);
  if (h->path == XFB_PATH_PLAIN && (h->c.dim != 3 || h->c.ade_kind != XFB_ADE_NONE))
    return set_err(h, XFB_ERR_INVALID, "the plain path handles 3-D scenes without dispersive media only");
  if (h->path == XFB_PATH_AUTO) h->path = XFB_PATH_FUSED;
  int rc;
  try {
    rc = h->c.prec == XFB_FP64 ? init_device<double>(h) : init_device<float>(h);
  } catch (const std::bad_alloc&) {
    rc = set_err(h, XFB_ERR_OOM, "host allocation failed during init");
  }
  if (rc) {
    free_device(h);
    return rc;
  }
  h->step = 0;
  h->inited = true;
  return XFB_OK;
}

int xfb_step(xfb_handle* h, long long n) {
  int rc = check_handle(h, true);
  if (rc || (rc = not_batched(h))) return rc;
  if (is_slab(h)) return set_err(h, XFB_ERR_STATE, "an x slab steps through xfb_slab_update / xfb_slab_record");
  if (n < 0) return set_err(h, XFB_ERR_INVALID, "negative step count");
  if (h->step + n > h->c.total_steps)
    return set_err(h, XFB_ERR_RANGE, "steps beyond the count xfb_init sized the run for");
  return h->c.prec == XFB_FP64 ? run_steps<double>(h, n) : run_steps<float>(h, n);
}

// Waits for the handle's stream and reads the step kernel's error flag: a
// staging wait that ran out makes every later sync and read-back of the run
// return XFB_ERR_TIMEOUT (the step's results are incomplete) until the next
// xfb_init.
static int step_status(xfb_handle* h) {
  XFB_CUDA(h, cudaStreamSynchronize(h->stream));
  XFB_CUDA(h, cudaGetLastError());
  if (h->step_err) {
    int e = 0;
    XFB_CUDA(h, cudaMemcpyAsync(&e, h->step_err, sizeof(e), cudaMemcpyDeviceToHost, h->stream));
    XFB_CUDA(h, cudaStreamSynchronize(h->stream));
    if (e)
      return set_err(h, XFB_ERR_TIMEOUT,
                     "one-sweep step: a staging copy did not complete within the wait limit; the run's results "
                     "are incomplete (xfb_init starts it over)");
  }
  return XFB_OK;
}

int xfb_sync(xfb_handle* h) {
  int rc = check_handle(h, true);
  if (rc) return rc;
  return step_status(h);
}

int xfb_set_wait_limit(xfb_handle* h, int polls) {
  int rc = check_handle(h, true);
  if (rc || (rc = not_batched(h))) return rc;
  if (polls < 0) return set_err(h, XFB_ERR_INVALID, "negative poll limit");
  if (!h->step_err) return set_err(h, XFB_ERR_STATE, "only the 3-D one-sweep step has bounded waits");
  return copy(h, h->step_err + 1, &polls, sizeof(int), cudaMemcpyHostToDevice);
}

int xfb_timed_step(xfb_handle* h, long long n, double* ms) {
  int rc = check_handle(h, true);
  if (rc || (rc = not_batched(h))) return rc;
  if (!ms) return set_err(h, XFB_ERR_INVALID, "null output");
  cudaEvent_t a, b;
  XFB_CUDA(h, cudaEventCreate(&a));
  XFB_CUDA(h, cudaEventCreate(&b));
  XFB_CUDA(h, cudaStreamSynchronize(h->stream));
  cudaEventRecord(a, h->stream);
  rc = xfb_step(h, n);
  cudaEventRecord(b, h->stream);
  cudaError_t e = cudaEventSynchronize(b);
  float t = 0;
  if (e == cudaSuccess) e = cudaEventElapsedTime(&t, a, b);
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  if (rc) return rc;
  if (e != cudaSuccess) return cuda_err(h, e, "timed step");
  *ms = t;
  return XFB_OK;
}

int xfb_profile_kernels(xfb_handle* h, long long n, double* ms, long long* launches) {
  int rc = check_handle(h, true);
  if (rc || (rc = not_batched(h))) return rc;
  if (!ms || !launches || n < 0) return set_err(h, XFB_ERR_INVALID, "bad arguments");
  if (h->step + n > h->c.total_steps) return set_err(h, XFB_ERR_RANGE, "steps beyond the count xfb_init sized the run for");
  XFB_CUDA(h, cudaStreamSynchronize(h->stream));
  return h->c.prec == XFB_FP64 ? profile_steps<double>(h, n, ms, launches) : profile_steps<float>(h, n, ms, launches);
}

int xfb_run(xfb_handle* h, long long n) {
  int rc = xfb_init(h, n);
  if (rc) return rc;
  if ((rc = xfb_step(h, n))) return rc;
  return xfb_sync(h);
}

int xfb_get_grid_info(const xfb_handle* h, xfb_grid_info* o) {
  if (!h || !o) return set_err(nullptr, XFB_ERR_INVALID, "null argument");
  const Compiled& c = h->c;
  std::memset(o, 0, sizeof(*o));
  o->dim = c.dim; o->precision = c.prec;
  o->nx = c.nx; o->ny = c.ny; o->nz = c.nz;
  o->dx = c.dx; o->dy = c.dy; o->dz = c.dz; o->dt = c.dt;
  for (int a = 0; a < 3; ++a) o->origin[a] = c.origin[a];
  o->n_materials = c.n_mat;
  o->ade_kind = c.ade_kind; o->ade_poles = c.ade_poles;
  if (c.tfsf_on) for (int q = 0; q < 6; ++q) o->tfsf_box[q] = c.tf[q];
  if (c.nf_on) for (int q = 0; q < 6; ++q) o->nf2ff_box[q] = c.nf[q];
  o->n_freqs = static_cast<int>(c.freqs.size());
  o->current_step = h->step;
  o->total_steps = c.total_steps;
  o->device_bytes = h->bytes;
  if (h->n_disp_cells < 0) {  // counted once: the material ids do not change
    long long nd = 0;
    if (c.ade_kind != XFB_ADE_NONE) {
      bool disp[256] = {};
      for (int m = 0; m < c.n_mat; ++m) disp[m] = c.ade_mat[static_cast<size_t>(m) * kAdeMat] != 0;
      const long long n = static_cast<long long>(c.mat_id.size());
      const uint8_t* id = c.mat_id.data();
#pragma omp parallel for reduction(+ : nd) schedule(static)
      for (long long q = 0; q < n; ++q) nd += disp[id[q]];
    }
    h->n_disp_cells = nd;
  }
  o->n_dispersive_cells = h->n_disp_cells;
  o->launches_per_step = launches_per_step(h);
  o->kernel_path = h->path;
  o->h2d_bytes = h->h2d_bytes;
  o->d2h_bytes = h->d2h_bytes;
  if (c.td_on) for (int q = 0; q < 6; ++q) o->nf2ff_td_box[q] = c.td[q];
  return XFB_OK;
}

int xfb_read_field(xfb_handle* h, int f, double* dst, size_t len) {
  int rc = check_handle(h, true);
  if (rc) return rc;
  wait_prefault(h);
  if (f < 0 || f > 5 || !dst) return set_err(h, XFB_ERR_INVALID, "bad field or buffer");
  if (!h->f[f]) return set_err(h, XFB_ERR_INVALID, "component not present in a 2-D (TMz) scene");
  int s[3];
  comp_shape(h->c, f, s);
  const size_t n = static_cast<size_t>(s[0]) * s[1] * s[2];
  if (len < n) return set_err(h, XFB_ERR_RANGE, "destination too small");
  if (!h->batch && (rc = step_status(h))) return rc;
  prefault_now(h, dst, n * sizeof(double));
  return h->c.prec == XFB_FP64 ? read_field_t<double>(h, f, dst) : read_field_t<float>(h, f, dst);
}

int xfb_host_prefault(xfb_handle* h, void* ptr, size_t bytes) {
  if (!h || (!ptr && bytes)) return set_err(h, XFB_ERR_INVALID, "null handle or range");
  if (!queue_prefault(h, ptr, bytes)) return set_err(h, XFB_ERR_OOM, "could not queue the range or start host threads");
  return XFB_OK;
}

int xfb_host_prefault_wait(xfb_handle* h) {
  if (!h) return set_err(nullptr, XFB_ERR_INVALID, "null handle");
  wait_prefault(h);
  return XFB_OK;
}

int xfb_write_field(xfb_handle* h, int f, const double* src, size_t len) {
  int rc = check_handle(h, true);
  if (rc) return rc;
  if (f < 0 || f > 5 || !src) return set_err(h, XFB_ERR_INVALID, "bad field or buffer");
  if (!h->f[f]) return set_err(h, XFB_ERR_INVALID, "component not present in a 2-D (TMz) scene");
  int s[3];
  comp_shape(h->c, f, s);
  if (len < static_cast<size_t>(s[0]) * s[1] * s[2]) return set_err(h, XFB_ERR_RANGE, "source too small");
  return h->c.prec == XFB_FP64 ? write_field_t<double>(h, f, src) : write_field_t<float>(h, f, src);
}

int xfb_read_probe(xfb_handle* h, int id, double* dst, size_t len, long long* n_written) {
  int rc = check_handle(h, true);
  if (rc) return rc;
  wait_prefault(h);
  if (id < 0 || id >= static_cast<int>(h->c.probes.size())) return set_err(h, XFB_ERR_RANGE, "probe id out of range");
  const long long n = h->step;
  if (len < static_cast<size_t>(n)) return set_err(h, XFB_ERR_RANGE, "destination too small");
  if (!h->batch && (rc = step_status(h))) return rc;
  if (n > 0 && (rc = copy(h, dst, h->probe_out + id * h->c.total_steps, n * sizeof(double), cudaMemcpyDeviceToHost))) return rc;
  if (n_written) *n_written = n;
  return XFB_OK;
}

int xfb_movie_shape(const xfb_handle* h, int id, int s[4]) {
  if (!h || !s) return set_err(nullptr, XFB_ERR_INVALID, "null argument");
  if (id < 0 || id >= static_cast<int>(h->c.movies.size())) return set_err(const_cast<xfb_handle*>(h), XFB_ERR_RANGE, "movie id out of range");
  const xfb_movie& mv = h->c.movies[id];
  s[0] = static_cast<int>((h->c.total_steps + mv.interval - 1) / mv.interval);
  for (int a = 0; a < 3; ++a) s[1 + a] = mv.hi[a] - mv.lo[a];
  return XFB_OK;
}

int xfb_read_movie(xfb_handle* h, int id, double* dst, size_t len) {
  int rc = check_handle(h, true);
  if (rc) return rc;
  wait_prefault(h);
  int s[4];
  if ((rc = xfb_movie_shape(h, id, s))) return rc;
  const size_t n = static_cast<size_t>(s[0]) * s[1] * s[2] * s[3];
  if (len < n) return set_err(h, XFB_ERR_RANGE, "destination too small");
  if (!h->batch && (rc = step_status(h))) return rc;
  if (n && (rc = copy(h, dst, h->movie_out[id], n * sizeof(double), cudaMemcpyDeviceToHost))) return rc;
  return XFB_OK;
}

int xfb_nf2ff_face_shape(const xfb_handle* h, int face, int s[3]) {
  if (!h || !s) return set_err(nullptr, XFB_ERR_INVALID, "null argument");
  if (!h->c.nf_on) return set_err(const_cast<xfb_handle*>(h), XFB_ERR_STATE, "scene has no NF2FF box");
  if (face < 0 || face > 5) return set_err(const_cast<xfb_handle*>(h), XFB_ERR_RANGE, "face out of range");
  const FaceGeom g = face_geom(h->c, face);
  s[0] = g.ni; s[1] = g.nj; s[2] = g.nk;
  return XFB_OK;
}

// Accumulates the NF2FF surface samples still in the ring (k_nf2ff keeps the
// samples of up to kNfRing steps before it adds them), so the accumulators
// hold every step taken.  Enqueued on the stream that steps the handle (the
// batch's stream while a batch steps it); launches kernels only.
static int nf2ff_flush(xfb_handle* h) {
  if (!h->c.nf_on || !h->nf_ring) return XFB_OK;
  cudaStream_t s = h->batch ? h->batch->stream : h->stream;
  const Compiled& c = h->c;
  NfP nf{};
  nf.nfreq = static_cast<int>(c.freqs.size());
  for (int q = 0; q < 6; ++q) nf.box[q] = c.nf[q];
  for (int q = 0; q < 7; ++q) nf.off[q] = h->nf_off[q];
  nf.npts = h->nf_npts;
  nf.acc = h->nf_acc; nf.te = h->te; nf.th = h->th;
  nf.total_steps = c.total_steps;
  nf.ring = h->nf_ring;
  nf.done = h->nf_done;
  nf.own_lo = own_lo(h);
  nf.own_hi = own_hi(h);
  k_nf2ff_flush<<<static_cast<unsigned>((h->nf_npts + 255) / 256), 256, 0, s>>>(nf, h->step);
  k_nf2ff_done<<<1, 1, 0, s>>>(h->nf_done, h->step);
  XFB_CUDA(h, cudaGetLastError());
  if (s != h->stream) XFB_CUDA(h, cudaStreamSynchronize(s));
  return XFB_OK;
}

int xfb_read_nf2ff(xfb_handle* h, int freq, int face, int which, double* dst, size_t len) {
  int rc = check_handle(h, true);
  if (rc) return rc;
  wait_prefault(h);
  int s[3];
  if ((rc = xfb_nf2ff_face_shape(h, face, s))) return rc;
  if (freq < 0 || freq >= static_cast<int>(h->c.freqs.size()) || which < 0 || which > 3)
    return set_err(h, XFB_ERR_RANGE, "frequency or current index out of range");
  const size_t n = static_cast<size_t>(s[0]) * s[1] * s[2];
  if (len < 2 * n) return set_err(h, XFB_ERR_RANGE, "destination too small (complex interleaved)");
  if ((rc = nf2ff_flush(h))) return rc;
  if (!h->batch && (rc = step_status(h))) return rc;
  const double2* src = h->nf_acc + (static_cast<long long>(freq) * 4 + which) * h->nf_npts + h->nf_off[face];
  if ((rc = copy(h, dst, src, n * sizeof(double2), cudaMemcpyDeviceToHost))) return rc;
  return XFB_OK;
}

int xfb_read_nf2ff_all(xfb_handle* h, int freq, double* dst, size_t len, long long* points) {
  int rc = check_handle(h, true);
  if (rc) return rc;
  wait_prefault(h);
  if (!h->c.nf_on) return set_err(h, XFB_ERR_STATE, "scene has no NF2FF box");
  if (freq < 0 || freq >= static_cast<int>(h->c.freqs.size())) return set_err(h, XFB_ERR_RANGE, "frequency index out of range");
  const size_t n = 4 * static_cast<size_t>(h->nf_npts);
  if (points) *points = h->nf_npts;
  if (!dst) return set_err(h, XFB_ERR_INVALID, "null destination");
  if (len < 2 * n) return set_err(h, XFB_ERR_RANGE, "destination too small (complex interleaved)");
  if ((rc = nf2ff_flush(h))) return rc;
  if (!h->batch && (rc = step_status(h))) return rc;
  prefault_now(h, dst, n * sizeof(double2));
  const double2* src = h->nf_acc + static_cast<long long>(freq) * 4 * h->nf_npts;
  return h->c.prec == XFB_FP64 ? read_bytes_t<double>(h, dst, src, n * sizeof(double2))
                               : read_bytes_t<float>(h, dst, src, n * sizeof(double2));
}

int xfb_far_field(xfb_handle* h, int freq, int n, const double* theta, const double* phi, double* out) {
  int rc = check_handle(h, true);
  if (rc) return rc;
  wait_prefault(h);
  if (!h->c.nf_on) return set_err(h, XFB_ERR_STATE, "scene has no NF2FF box");
  if (freq < 0 || freq >= static_cast<int>(h->c.freqs.size())) return set_err(h, XFB_ERR_RANGE, "frequency index out of range");
  if (n < 0 || (n > 0 && (!theta || !phi || !out))) return set_err(h, XFB_ERR_INVALID, "bad angle arrays");
  if (n == 0) return XFB_OK;
  if ((rc = nf2ff_flush(h))) return rc;
  // angle and output buffers of this call, released on every return path
  // (after the stream has finished with them)
  struct Scratch {
    xfb_handle* h;
    double* p[3] = {nullptr, nullptr, nullptr};
    ~Scratch() {
      cudaStreamSynchronize(h->stream);
      for (double* q : p) cudaFree(q);
    }
  } sb{h};
  XFB_CUDA(h, cudaMalloc(&sb.p[0], n * sizeof(double)));
  XFB_CUDA(h, cudaMalloc(&sb.p[1], n * sizeof(double)));
  XFB_CUDA(h, cudaMalloc(&sb.p[2], 4 * n * sizeof(double)));
  double *d_th = sb.p[0], *d_ph = sb.p[1], *d_out = sb.p[2];
  XFB_CUDA(h, cudaMemcpyAsync(d_th, theta, n * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  XFB_CUDA(h, cudaMemcpyAsync(d_ph, phi, n * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  FarP fp{};
  const Compiled& c = h->c;
  for (int q = 0; q < 6; ++q) fp.box[q] = c.nf[q];
  for (int q = 0; q < 7; ++q) fp.off[q] = h->nf_off[q];
  fp.npts = h->nf_npts;
  fp.acc = h->nf_acc + static_cast<long long>(freq) * 4 * h->nf_npts;
  for (int a = 0; a < 3; ++a) fp.origin[a] = c.origin[a];
  fp.d[0] = c.dx; fp.d[1] = c.dy; fp.d[2] = c.dz;
  fp.k = 2 * kPi * c.freqs[freq] / c0();
  fp.eta = std::sqrt(kMu0 / kEps0);
  fp.theta = d_th; fp.phi = d_ph; fp.out = d_out;
  k_far<<<n, 256, 0, h->stream>>>(fp);
  XFB_CUDA(h, cudaGetLastError());
  XFB_CUDA(h, cudaMemcpyAsync(out, d_out, 4 * n * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  XFB_CUDA(h, cudaStreamSynchronize(h->stream));
  return XFB_OK;
}

int xfb_far_field_static(xfb_handle* h, int freq, int n, const double* theta, const double* phi, double* out) {
  int rc = check_handle(h, true);  // makes the handle's device current
  if (rc) return rc;
  wait_prefault(h);
  if (!h->c.nf_on) return set_err(h, XFB_ERR_STATE, "scene has no NF2FF box");
  if (freq < 0 || freq >= static_cast<int>(h->c.freqs.size())) return set_err(h, XFB_ERR_RANGE, "frequency index out of range");
  if (n < 0 || (n > 0 && (!theta || !phi || !out))) return set_err(h, XFB_ERR_INVALID, "bad angle arrays");
  if (n > kFarStaticMaxAngles)
    return set_err(h, XFB_ERR_RANGE,
                   "xfb_far_field_static takes at most " + std::to_string(kFarStaticMaxAngles) +
                       " angles per call (its scratch is a fixed device array); got " + std::to_string(n));
  if (n == 0) return XFB_OK;
  if ((rc = nf2ff_flush(h))) return rc;
  double* scratch = nullptr;
  if ((rc = far_scratch_for(h, &scratch))) return rc;
  double* d_th = scratch;
  double* d_ph = scratch + kFarStaticMaxAngles;
  double* d_out = scratch + 2 * kFarStaticMaxAngles;
  XFB_CUDA(h, cudaMemcpyAsync(d_th, theta, n * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  XFB_CUDA(h, cudaMemcpyAsync(d_ph, phi, n * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  FarP fp{};
  const Compiled& c = h->c;
  for (int q = 0; q < 6; ++q) fp.box[q] = c.nf[q];
  for (int q = 0; q < 7; ++q) fp.off[q] = h->nf_off[q];
  fp.npts = h->nf_npts;
  fp.acc = h->nf_acc + static_cast<long long>(freq) * 4 * h->nf_npts;
  for (int a = 0; a < 3; ++a) fp.origin[a] = c.origin[a];
  fp.d[0] = c.dx; fp.d[1] = c.dy; fp.d[2] = c.dz;
  fp.k = 2 * kPi * c.freqs[freq] / c0();
  fp.eta = std::sqrt(kMu0 / kEps0);
  fp.theta = d_th; fp.phi = d_ph; fp.out = d_out;  // k_far writes all 4 outputs of every angle
  k_far<<<n, 256, 0, h->stream>>>(fp);
  XFB_CUDA(h, cudaGetLastError());
  XFB_CUDA(h, cudaMemcpyAsync(out, d_out, 4 * n * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  XFB_CUDA(h, cudaStreamSynchronize(h->stream));
  return XFB_OK;
}

int xfb_nf2ff_td_bins(const xfb_handle* h, long long* n_bins) {
  if (!h || !n_bins) return set_err(nullptr, XFB_ERR_INVALID, "null argument");
  if (!h->c.td_on) return set_err(const_cast<xfb_handle*>(h), XFB_ERR_STATE, "scene has no time-domain NF2FF box");
  *n_bins = h->c.td_bins;
  return XFB_OK;
}

int xfb_read_nf2ff_td(xfb_handle* h, int which, double* dst, size_t len) {
  int rc = check_handle(h, true);
  if (rc) return rc;
  wait_prefault(h);
  if (!h->c.td_on) return set_err(h, XFB_ERR_STATE, "scene has no time-domain NF2FF box");
  if (which < 0 || which > 5 || !dst) return set_err(h, XFB_ERR_INVALID, "potential index must be 0..5 (W_x..U_z)");
  const size_t n = static_cast<size_t>(h->c.td_bins);
  if (len < n) return set_err(h, XFB_ERR_RANGE, "destination too small");
  if (!h->batch && (rc = step_status(h))) return rc;
  if (h->batch) XFB_CUDA(h, cudaStreamSynchronize(h->batch->stream));
  return copy(h, dst, h->td_pot + static_cast<size_t>(which) * n, n * sizeof(double), cudaMemcpyDeviceToHost);
}

int xfb_far_field_td(xfb_handle* h, double* e_theta, double* e_phi, size_t len) {
  int rc = check_handle(h, true);
  if (rc) return rc;
  wait_prefault(h);
  if (!h->c.td_on) return set_err(h, XFB_ERR_STATE, "scene has no time-domain NF2FF box");
  const size_t n = static_cast<size_t>(h->c.td_bins);
  if (!e_theta || !e_phi || len < n) return set_err(h, XFB_ERR_RANGE, "destination too small");
  std::vector<double> p(6 * n);
  for (int q = 0; q < 6; ++q)
    if ((rc = xfb_read_nf2ff_td(h, q, p.data() + q * n, n))) return rc;
  const double th = h->c.td_theta, ph = h->c.td_phi;
  const double st = std::sin(th), ct = std::cos(th), sp = std::sin(ph), cp = std::cos(ph);
  const double eta = std::sqrt(kMu0 / kEps0);
  const double f = 1.0 / (4 * kPi * kTdC0 * h->c.dt);
  for (size_t b = 0; b < n; ++b) {
    const double wx = p[b], wy = p[n + b], wz = p[2 * n + b], ux = p[3 * n + b], uy = p[4 * n + b], uz = p[5 * n + b];
    const double w_th = wx * ct * cp + wy * ct * sp - wz * st, w_ph = -wx * sp + wy * cp;
    const double u_th = ux * ct * cp + uy * ct * sp - uz * st, u_ph = -ux * sp + uy * cp;
    e_theta[b] = -f * (u_ph + eta * w_th);
    e_phi[b] = f * (u_th - eta * w_ph);
  }
  return XFB_OK;
}

// ---- x-slab decomposition ---------------------------------------------------

int xfb_set_slab(xfb_handle* h, int i0, int i1) {
  if (!h) return set_err(nullptr, XFB_ERR_INVALID, "null handle");
  if (h->inited) return set_err(h, XFB_ERR_STATE, "set the slab before xfb_init");
  const Compiled& c = h->c;
  if (c.dim != 3) return set_err(h, XFB_ERR_INVALID, "x slabs are 3-D");
  if (i0 < 0 || i1 > c.nx || i1 <= i0) return set_err(h, XFB_ERR_RANGE, "slab planes outside [0, nx)");
  if (c.nx >= 65536 || c.ny >= 65536 || c.nz >= 65536) return set_err(h, XFB_ERR_INVALID, "x slabs need sides below 65536 cells");
  // the H halo plane below a slab is recomputed from the read set; its x-CPML
  // psi would be another slab's, so no split may put it in an x slab
  for (int s0 : {i0, i1})
    if (s0 > 0 && s0 < c.nx && (s0 - 1 < c.pml[0] || s0 - 1 >= c.nx - c.pml[1]))
      return set_err(h, XFB_ERR_RANGE, "a slab boundary's plane below lies in the x CPML");
  h->slab_i0 = i0;
  h->slab_i1 = i1;
  return XFB_OK;
}

int xfb_get_slab(const xfb_handle* h, int* i0, int* i1) {
  if (!h || !i0 || !i1) return set_err(nullptr, XFB_ERR_INVALID, "null argument");
  *i0 = is_slab(h) ? h->slab_i0 : 0;
  *i1 = is_slab(h) ? h->slab_i1 : h->c.nx;
  return XFB_OK;
}

int xfb_slab_update(xfb_handle* h) {
  int rc = check_handle(h, true);
  if (rc) return rc;
  if (!is_slab(h)) return set_err(h, XFB_ERR_STATE, "not an x slab (xfb_set_slab)");
  if (h->slab_pending) return set_err(h, XFB_ERR_STATE, "the previous update awaits xfb_slab_record");
  if (h->step + 1 > h->c.total_steps) return set_err(h, XFB_ERR_RANGE, "steps beyond the count xfb_init sized the run for");
  return h->c.prec == XFB_FP64 ? slab_update<double>(h) : slab_update<float>(h);
}

int xfb_slab_record(xfb_handle* h) {
  int rc = check_handle(h, true);
  if (rc) return rc;
  if (!h->slab_pending) return set_err(h, XFB_ERR_STATE, "no update awaits its record");
  return h->c.prec == XFB_FP64 ? slab_record<double>(h) : slab_record<float>(h);
}

// The buffers of one exchange side in the set the pending update wrote:
// which = 0 the first owned plane (sent down), 1 the last owned plane (sent
// up), 2 the lower halo (received from below), 3 the upper halo (received
// from above).  Six field planes; the upward direction (1, 2) also carries
// the H-side psi of the y and z CPML slabs at that plane, which the H halo of
// the slab above reads.
static int slab_buffers(xfb_handle* h, int which, void* ptrs[10], size_t sizes[10], int* n) {
  const int plane[4] = {h->slab_i0, h->slab_i1 - 1, h->slab_i0 - 1, h->slab_i1};
  const long long p = plane[which];
  if (p < 0 || p > h->c.nx) return set_err(h, XFB_ERR_RANGE, "the slab has no halo on that side (grid wall)");
  const int set = static_cast<int>((h->step + 1) & 1);  // the set the pending update wrote
  int q = 0;
  for (int f = 0; f < 6; ++f, ++q) {
    ptrs[q] = static_cast<char*>(field_ptr(h, set, f)) + p * h->sx * h->esize;
    sizes[q] = static_cast<size_t>(h->sx) * h->esize;
  }
  if (which == 1 || which == 2) {
    void* const* hp = set ? h->psi_h1 : h->psi + 6;  // hy_x hz_x hz_y hx_y hx_z hy_z
    const long long ys = h->ysx, zs = h->zsx;
    if (ys > 0)
      for (int r : {2, 3}) {
        ptrs[q] = static_cast<char*>(hp[r]) + p * ys * h->esize;
        sizes[q++] = static_cast<size_t>(ys) * h->esize;
      }
    if (zs > 0 && h->c.pml[4] + h->c.pml[5] > 0)
      for (int r : {4, 5}) {
        ptrs[q] = static_cast<char*>(hp[r]) + p * zs * h->esize;
        sizes[q++] = static_cast<size_t>(zs) * h->esize;
      }
  }
  *n = q;
  return XFB_OK;
}

int xfb_slab_planes(xfb_handle* h, int which, void* ptrs[10], size_t sizes[10], int* n) {
  int rc = check_handle(h, true);
  if (rc) return rc;
  if (!is_slab(h) || !h->slab_pending) return set_err(h, XFB_ERR_STATE, "planes exist between xfb_slab_update and xfb_slab_record");
  if (which < 0 || which > 3 || !ptrs || !sizes || !n) return set_err(h, XFB_ERR_INVALID, "which must be 0..3");
  return slab_buffers(h, which, ptrs, sizes, n);
}

int xfb_slab_exchange(xfb_handle* lo, xfb_handle* hi) {
  if (!lo || !hi) return set_err(nullptr, XFB_ERR_INVALID, "null handle");
  int rc = check_handle(lo, true);
  if (rc || (rc = check_handle(hi, true))) return rc;
  if (!is_slab(lo) || !is_slab(hi) || lo->slab_i1 != hi->slab_i0)
    return set_err(lo, XFB_ERR_INVALID, "the slabs are not neighbours (lo's end must be hi's start)");
  if (!lo->slab_pending || !hi->slab_pending || lo->step != hi->step)
    return set_err(lo, XFB_ERR_STATE, "both slabs must hold the update of the same step");
  if (lo->sx != hi->sx || lo->esize != hi->esize) return set_err(lo, XFB_ERR_INVALID, "the slabs have different layouts");
  // the updates have finished on both devices before their planes move
  XFB_CUDA(hi, cudaSetDevice(hi->device));
  XFB_CUDA(hi, cudaStreamSynchronize(hi->stream));
  XFB_CUDA(lo, cudaSetDevice(lo->device));
  XFB_CUDA(lo, cudaStreamSynchronize(lo->stream));
  void *up_src[10], *up_dst[10], *dn_src[10], *dn_dst[10];
  size_t up_sz[10], up_dsz[10], dn_sz[10], dn_dsz[10];
  int nus, nud, nds, ndd;
  if ((rc = slab_buffers(lo, 1, up_src, up_sz, &nus)) || (rc = slab_buffers(hi, 2, up_dst, up_dsz, &nud)) ||
      (rc = slab_buffers(hi, 0, dn_src, dn_sz, &nds)) || (rc = slab_buffers(lo, 3, dn_dst, dn_dsz, &ndd)))
    return rc;
  if (nus != nud || nds != ndd) return set_err(lo, XFB_ERR_INVALID, "the slabs' exchange lists differ");
  for (int q = 0; q < nus; ++q)
    XFB_CUDA(lo, cudaMemcpyPeerAsync(up_dst[q], hi->device, up_src[q], lo->device, up_sz[q], lo->stream));
  for (int q = 0; q < nds; ++q)
    XFB_CUDA(lo, cudaMemcpyPeerAsync(dn_dst[q], lo->device, dn_src[q], hi->device, dn_sz[q], lo->stream));
  XFB_CUDA(lo, cudaStreamSynchronize(lo->stream));
  return XFB_OK;
}

int xfb_state_size(const xfb_handle* h, size_t* bytes) {
  if (!h || !bytes) return set_err(nullptr, XFB_ERR_INVALID, "null argument");
  if (!h->inited) return set_err(const_cast<xfb_handle*>(h), XFB_ERR_STATE, "handle not initialised");
  size_t s = sizeof(long long);
  for (const Buf& b : h->bufs)
    if (b.state) s += b.bytes;
  *bytes = s;
  return XFB_OK;
}

int xfb_get_state(xfb_handle* h, void* dst, size_t len) {
  int rc = check_handle(h, true);
  if (rc) return rc;
  wait_prefault(h);
  size_t need;
  if ((rc = xfb_state_size(h, &need))) return rc;
  if (!dst || len < need) return set_err(h, XFB_ERR_RANGE, "state buffer too small");
  if ((rc = nf2ff_flush(h))) return rc;  // the state holds accumulators, not the sample ring
  XFB_CUDA(h, cudaStreamSynchronize(h->stream));
  char* o = static_cast<char*>(dst);
  std::memcpy(o, &h->step, sizeof(long long));
  o += sizeof(long long);
  for (const Buf& b : h->bufs)
    if (b.state) {
      if ((rc = copy(h, o, b.p, b.bytes, cudaMemcpyDeviceToHost))) return rc;
      o += b.bytes;
    }
  return XFB_OK;
}

int xfb_set_state(xfb_handle* h, const void* src, size_t len) {
  int rc = check_handle(h, true);
  if (rc || (rc = not_batched(h))) return rc;
  size_t need;
  if ((rc = xfb_state_size(h, &need))) return rc;
  if (!src || len < need) return set_err(h, XFB_ERR_RANGE, "state buffer too small");
  XFB_CUDA(h, cudaStreamSynchronize(h->stream));
  const char* o = static_cast<const char*>(src);
  long long step;
  std::memcpy(&step, o, sizeof(long long));
  if (step < 0 || step > h->c.total_steps) return set_err(h, XFB_ERR_INVALID, "state step outside this run");
  o += sizeof(long long);
  for (const Buf& b : h->bufs)
    if (b.state) {
      if ((rc = copy(h, b.p, o, b.bytes, cudaMemcpyHostToDevice))) return rc;
      o += b.bytes;
    }
  h->step = step;
  return XFB_OK;
}

int xfb_check_finite(xfb_handle* h, long long* bad) {
  int rc = check_handle(h, true);
  if (rc) return rc;
  XFB_CUDA(h, cudaMemsetAsync(h->scratch_u64, 0, sizeof(unsigned long long), h->stream));
  if (h->c.prec == XFB_FP64) launch_nonfinite<double>(h);
  else launch_nonfinite<float>(h);
  unsigned long long n = 0;
  XFB_CUDA(h, cudaMemcpyAsync(&n, h->scratch_u64, sizeof(n), cudaMemcpyDeviceToHost, h->stream));
  XFB_CUDA(h, cudaStreamSynchronize(h->stream));
  if (bad) *bad = static_cast<long long>(n);
  if (n) return set_err(h, XFB_ERR_NUMERIC, std::to_string(n) + " non-finite field values");
  return XFB_OK;
}

int xfb_compiled_view_get(const xfb_handle* h, xfb_compiled_view* v) {
  if (!h || !v) return set_err(nullptr, XFB_ERR_INVALID, "null argument");
  const Compiled& c = h->c;
  std::memset(v, 0, sizeof(*v));
  v->dim = c.dim; v->nx = c.nx; v->ny = c.ny; v->nz = c.nz;
  v->dx = c.dx; v->dy = c.dy; v->dz = c.dz; v->dt = c.dt;
  v->material_id = c.mat_id.data();
  v->n_materials = c.n_mat;
  v->coeff = c.coeff.data();
  v->ade_kind = c.ade_kind; v->ade_poles = c.ade_poles;
  v->ade_mat = c.ade_mat.data();
  v->ade_pole = c.ade_pole.data();
  for (int q = 0; q < 6; ++q) v->pml_cells[q] = c.pml[q];
  for (int a = 0; a < 3; ++a) {
    v->pml_ae[a] = c.pml_ae[a].data(); v->pml_be[a] = c.pml_be[a].data();
    v->pml_ah[a] = c.pml_ah[a].data(); v->pml_bh[a] = c.pml_bh[a].data();
  }
  v->tfsf_enabled = c.tfsf_on;
  for (int q = 0; q < 6; ++q) v->tfsf_box[q] = c.tf[q];
  for (int a = 0; a < 3; ++a) {
    v->tfsf_proj_int[a] = c.proj_int[a].data();
    v->tfsf_proj_half[a] = c.proj_half[a].data();
    v->tfsf_transform_e[a] = c.tr_e[a]; v->tfsf_transform_h[a] = c.tr_h[a];
    v->tfsf_ca[a] = c.ca[a]; v->tfsf_cb[a] = c.cb[a];
  }
  v->aux_nl = c.aux_nl;
  v->aux_ceih = c.aux_ceih; v->aux_chie = c.aux_chie; v->aux_abc = c.aux_abc;
  v->aux_source = c.aux_source.data();
  v->total_steps = c.total_steps;
  v->nf2ff_enabled = c.nf_on;
  for (int q = 0; q < 6; ++q) v->nf2ff_box[q] = c.nf[q];
  v->n_freqs = static_cast<int>(c.freqs.size());
  v->freqs = c.freqs.data();
  v->nf2ff_te = c.te.data();
  v->nf2ff_th = c.th.data();
  v->nf2ff_td_enabled = c.td_on;
  for (int q = 0; q < 6; ++q) v->nf2ff_td_box[q] = c.td[q];
  v->nf2ff_td_theta = c.td_theta;
  v->nf2ff_td_phi = c.td_phi;
  v->nf2ff_td_bins = c.td_bins;
  for (int a = 0; a < 3; ++a) v->origin[a] = c.origin[a];
  for (int q = 0; q < 6; ++q) v->ade_box[q] = c.ade_box[q];
  return XFB_OK;
}


// ---- learned absorbing boundary -----------------------------------------------

int xfb_labc_wall_cells(const xfb_handle* h, long long* cells) {
  if (!h || !cells) return set_err(nullptr, XFB_ERR_INVALID, "null argument");
  *cells = labc_layout(h->c.nx, h->c.ny, h->c.nz).off[12];
  return XFB_OK;
}

int xfb_set_learned_abc(xfb_handle* h, const float* weights, int n_weights) {
  int rc = check_handle(h, true);
  if (rc || (rc = not_batched(h))) return rc;
  for (auto& kv : h->graphs) cudaGraphExecDestroy(kv.second);  // the step's launch list changes
  h->graphs.clear();
  if (!weights) {
    h->labc_on = false;
    return XFB_OK;
  }
  if (n_weights != kMlpParams) return set_err(h, XFB_ERR_INVALID, "weight count must be xfb_mlp_param_count()");
  if (!fused(h) || h->c.dim != 3) return set_err(h, XFB_ERR_STATE, "the learned boundary runs on the 3-D one-sweep path");
  if (is_slab(h)) return set_err(h, XFB_ERR_STATE, "the learned boundary runs on whole grids, not x slabs");
  for (int f = 0; f < 6; ++f)
    if (h->c.pml[f]) return set_err(h, XFB_ERR_INVALID, "the learned boundary replaces the CPML: the scene must have none");
  // BF16 weights, round to nearest even
  std::vector<uint16_t> wb(kMlpParams);
  for (int q = 0; q < kMlpParams; ++q) {
    uint32_t u;
    std::memcpy(&u, &weights[q], 4);
    if ((u & 0x7f800000u) == 0x7f800000u && (u & 0x7fffffu)) wb[q] = 0x7fc0;
    else wb[q] = static_cast<uint16_t>((u + 0x7fffu + ((u >> 16) & 1u)) >> 16);
  }
  if (!h->labc_w) {
    if ((rc = alloc(h, &h->labc_w, kMlpParams * sizeof(uint16_t), false))) return rc;
    void* p = nullptr;
    if ((rc = alloc(h, &p, 2 * labc_layout(h->c.nx, h->c.ny, h->c.nz).off[12] * sizeof(float), true))) return rc;
    h->labc_hist = static_cast<float*>(p);
  }
  if ((rc = copy(h, h->labc_w, wb.data(), wb.size() * sizeof(uint16_t), cudaMemcpyHostToDevice))) return rc;
  h->labc_on = true;
  return XFB_OK;
}

// ---- batches of scenes -------------------------------------------------------

int xfb_batch_create(xfb_handle* const* handles, int n, xfb_batch** out) {
  if (!handles || n <= 0 || !out) return set_err(nullptr, XFB_ERR_INVALID, "null handles or output, or n <= 0");
  *out = nullptr;
  for (int q = 0; q < n; ++q) {
    xfb_handle* h = handles[q];
    if (!h) return set_err(nullptr, XFB_ERR_INVALID, "null handle in the batch");
    if (h->batch) return set_err(h, XFB_ERR_STATE, "handle already belongs to a batch");
    if (h->c.dim != 3) return set_err(h, XFB_ERR_INVALID, "batches hold 3-D scenes only");
    if (is_slab(h)) return set_err(h, XFB_ERR_INVALID, "batches hold whole scenes, not x slabs");
    if (h->c.prec != handles[0]->c.prec) return set_err(h, XFB_ERR_INVALID, "all scenes of a batch share one precision");
    for (int r = 0; r < q; ++r)
      if (handles[r] == h) return set_err(h, XFB_ERR_INVALID, "a handle appears twice in the batch");
  }
  xfb_batch* b = new (std::nothrow) xfb_batch();
  if (!b) return set_err(nullptr, XFB_ERR_OOM, "host allocation failed");
  b->hs.assign(handles, handles + n);
  b->prec = handles[0]->c.prec;
  for (xfb_handle* h : b->hs) h->batch = b;
  *out = b;
  return XFB_OK;
}

int xfb_batch_set_tile(xfb_batch* b, int rows) {
  if (!b) return set_err(nullptr, XFB_ERR_INVALID, "null batch");
  if (rows != 0 && rows != 8 && rows != 14 && rows != 16)
    return batch_err(b, XFB_ERR_INVALID, "tile rows must be 0 (autotune), 8, 14 or 16");
  b->tile_req = rows;
  b->tile = -1;
  return XFB_OK;
}

int xfb_batch_set_launch(xfb_batch* b, int launch) {
  if (!b) return set_err(nullptr, XFB_ERR_INVALID, "null batch");
  if (launch != XFB_BATCH_AUTO && launch != XFB_BATCH_PER_STEP && launch != XFB_BATCH_PERSISTENT)
    return batch_err(b, XFB_ERR_INVALID, "launch form must be XFB_BATCH_AUTO, XFB_BATCH_PER_STEP or XFB_BATCH_PERSISTENT");
  if (b->inited && launch == XFB_BATCH_PERSISTENT && !b->persist_ok)
    return batch_err(b, XFB_ERR_INVALID, "persistent batch launches need scenes without monitors or a separate ADE pass");
  b->launch_req = launch;
  b->launch = -1;
  b->tile = -1;
  return XFB_OK;
}

int xfb_batch_launch_form(const xfb_batch* b, int* launch) {
  if (!b || !launch) return set_err(nullptr, XFB_ERR_INVALID, "null batch or output");
  *launch = b->launch < 0 ? 0 : b->launch;
  return XFB_OK;
}

int xfb_batch_init(xfb_batch* b, long long total_steps) {
  if (!b) return set_err(nullptr, XFB_ERR_INVALID, "null batch");
  if (b->inited) {
    cudaSetDevice(b->device);
    cudaStreamSynchronize(b->stream);
    batch_free(b);
  }
  int dev = b->hs[0]->device;
  if (dev < 0) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
      cudaGetLastError();
      return batch_err(b, XFB_ERR_NO_DEVICE, "no CUDA device available");
    }
    if (cudaGetDevice(&dev) != cudaSuccess) return batch_err(b, XFB_ERR_CUDA, "cudaGetDevice");
  }
  b->device = dev;
  b->cells = 0;
  for (xfb_handle* h : b->hs) {
    if (h->device >= 0 && h->device != dev) return batch_err(b, XFB_ERR_INVALID, "all scenes of a batch run on one device");
    h->batch = nullptr;  // xfb_init is refused for batched handles
    if (h->device < 0) cudaSetDevice(dev);  // xfb_init adopts the current device
    h->path = XFB_PATH_FUSED;
    int rc = xfb_init(h, total_steps);
    h->batch = b;
    if (rc) return batch_err(b, rc, "scene init failed: " + h->err);
    b->cells += static_cast<long long>(h->c.nx) * h->c.ny * h->c.nz;
  }
  if (cudaSetDevice(dev) != cudaSuccess) return batch_err(b, XFB_ERR_CUDA, "cudaSetDevice");
  if (!b->stream && cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess)
    return batch_err(b, XFB_ERR_CUDA, "cudaStreamCreate");
  int rc;
  try {
    rc = b->prec == XFB_FP64 ? batch_init<double>(b) : batch_init<float>(b);
  } catch (const std::bad_alloc&) {
    rc = batch_err(b, XFB_ERR_OOM, "host allocation failed during batch init");
  }
  if (rc) return rc;
  b->step = 0;
  b->total = total_steps;
  b->tile = -1;
  b->launch = -1;
  b->inited = true;
  return XFB_OK;
}

int xfb_batch_step(xfb_batch* b, long long n) {
  if (!b) return set_err(nullptr, XFB_ERR_INVALID, "null batch");
  if (!b->inited) return batch_err(b, XFB_ERR_STATE, "batch not initialised (call xfb_batch_init)");
  if (n < 0) return batch_err(b, XFB_ERR_INVALID, "negative step count");
  if (b->step + n > b->total) return batch_err(b, XFB_ERR_RANGE, "steps beyond the count xfb_batch_init sized the run for");
  if (cudaSetDevice(b->device) != cudaSuccess) return batch_err(b, XFB_ERR_CUDA, "cudaSetDevice");
  return b->prec == XFB_FP64 ? batch_run<double>(b, n) : batch_run<float>(b, n);
}

int xfb_batch_sync(xfb_batch* b) {
  if (!b) return set_err(nullptr, XFB_ERR_INVALID, "null batch");
  if (!b->inited) return batch_err(b, XFB_ERR_STATE, "batch not initialised");
  cudaSetDevice(b->device);
  cudaError_t e = cudaStreamSynchronize(b->stream);
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e != cudaSuccess) return batch_err(b, XFB_ERR_CUDA, cudaGetErrorString(e));
  if (b->err_dev) {
    int flag = 0;
    e = cudaMemcpy(&flag, b->err_dev, sizeof(int), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return batch_err(b, XFB_ERR_CUDA, cudaGetErrorString(e));
    if (flag)
      return batch_err(b, XFB_ERR_TIMEOUT,
                       "batch step: a staging copy did not complete within the wait limit; the batch's results are "
                       "incomplete (xfb_batch_init starts it over)");
  }
  return XFB_OK;
}

int xfb_batch_set_wait_limit(xfb_batch* b, int polls) {
  if (!b) return set_err(nullptr, XFB_ERR_INVALID, "null batch");
  if (!b->inited) return batch_err(b, XFB_ERR_STATE, "batch not initialised");
  if (polls < 0) return batch_err(b, XFB_ERR_INVALID, "negative poll limit");
  cudaSetDevice(b->device);
  cudaError_t e = cudaMemcpyAsync(b->err_dev + 1, &polls, sizeof(int), cudaMemcpyHostToDevice, b->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
  if (e != cudaSuccess) return batch_err(b, XFB_ERR_CUDA, cudaGetErrorString(e));
  return XFB_OK;
}

int xfb_batch_timed_step(xfb_batch* b, long long n, double* ms) {
  int rc = xfb_batch_sync(b);
  if (rc) return rc;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, b->stream);
  rc = xfb_batch_step(b, n);
  cudaEventRecord(e1, b->stream);
  cudaEventSynchronize(e1);
  float t = 0;
  cudaEventElapsedTime(&t, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (ms) *ms = t;
  return rc ? rc : xfb_batch_sync(b);
}

int xfb_batch_info(const xfb_batch* b, long long* cells, int* tile_rows, int* work_items) {
  if (!b) return set_err(nullptr, XFB_ERR_INVALID, "null batch");
  if (cells) *cells = b->cells;
  const int t = b->tile < 0 ? 1 : b->tile;
  if (tile_rows) *tile_rows = b->tile < 0 ? 0 : kStepTileRows[t];
  if (work_items) *work_items = b->n_items[t];
  return XFB_OK;
}

const char* xfb_batch_last_error(const xfb_batch* b) { return b ? b->err.c_str() : g_err.c_str(); }

int xfb_batch_destroy(xfb_batch* b) {
  if (!b) return XFB_OK;
  if (b->inited) {
    cudaSetDevice(b->device);
    cudaStreamSynchronize(b->stream);
  }
  for (xfb_handle* h : b->hs) {
    h->batch = nullptr;
    // the handle's own step counter continues from where the batch left it
    if (h->inited && h->t_dev) {
      cudaMemcpyAsync(h->t_dev, &h->step, sizeof(long long), cudaMemcpyHostToDevice, h->stream);
      cudaStreamSynchronize(h->stream);
    }
  }
  batch_free(b);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
  return XFB_OK;
}

}  // extern "C"
