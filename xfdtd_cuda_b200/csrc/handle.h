// Engine handle shared by the C-ABI (api.cu) and the per-precision engine
// translation units (engine_f32.cu, engine_f64.cu).
#pragma once

#include <cuda.h>  // CUtensorMap
#include <cuda_runtime.h>

#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "xfb_internal.h"

namespace xfb {
struct Buf {
  void* p = nullptr;
  size_t bytes = 0;
  bool state = false;  // part of the checkpoint state
  bool owner = true;   // p is a cudaMalloc base (freed with the handle's device state)
};

}  // namespace xfb

struct xfb_batch;
struct xfb_handle {
  using Buf = xfb::Buf;
  xfb::Compiled c;
  std::string err;
  // xfb_host_prefault: ranges (64 MiB parts) queued for a pool of host
  // threads (three quarters of the cores, at most 12) that fault them in;
  // every call that writes caller memory joins the pool first
  std::vector<std::thread> prefault;
  mutable long long n_disp_cells = -1;  // cells of dispersive materials (grid info), once counted
  std::vector<std::pair<char*, char*>> pf_queue;
  std::mutex pf_mu;
  int pf_active = 0;
  int device = -1;
  cudaStream_t stream = nullptr;
  bool inited = false;
  long long step = 0;
  unsigned hint_grid[3] = {1, 1, 1}, hint_block[3] = {1, 1, 1};
  int tk = 32, tj = 16;
  int path = XFB_PATH_AUTO;  // resolved at init: XFB_PATH_SPLIT or XFB_PATH_FUSED
  int graph_on = 1, graph_steps = 64;
  int coeff_storage = XFB_COEFF_NATIVE;  // rounding of the update-coefficient LUT (xfb_set_coeff_storage)
  // 2-D temporal blocking (k_step2_tb): steps per launch (odd; 0: one launch
  // per step), whether init enabled it, the tile rows / columns, and the
  // second set of the E-side psi (ez_x, ez_y) it alternates with psi[1], psi[2]
  int tb_steps = 9;
  bool tb_on = false;
  int tb_ti = 0, tb_tj = 0;
  void* psi_e1[2] = {};
  std::map<int, cudaGraphExec_t> graphs;
  std::vector<Buf> bufs;
  size_t bytes = 0;
  // device buffers up to kArenaMax bytes are carved from chunks of one
  // cudaMalloc each (fewer driver calls at init): the free part of the last chunk
  char* arena = nullptr;
  size_t arena_left = 0;
  int esize = 4;
  // field layout
  long long sx = 0, sy = 0, nzp = 0, elems = 0, guard = 0;
  void* f[6] = {};    // field set 0
  void* f1[6] = {};   // field set 1 (one-sweep path: step t reads set t&1, writes the other)
  uint8_t* mid = nullptr;
  void* lut8 = nullptr;       // [n_mat][8] compact coefficients (one-sweep path)
  uint8_t* mat_disp = nullptr;
  void* lut = nullptr;
  // CPML
  void* prof[12] = {};  // ae0 ae1 ae2 be0 be1 be2 ah0 ah1 ah2 bh0 bh1 bh2
  void* psi[12] = {};   // ey_x ez_x ez_y ex_y ex_z ey_z hy_x hz_x hz_y hx_y hx_z hy_z
  void* psi_h1[6] = {}; // H-side psi of field set 1 (one-sweep path)
  long long ysx = 0, zsx = 0, zsy = 0;
  // TFSF
  double* proj[6] = {};
  double* e_aux = nullptr;   // [total_steps + 1][nl + 1] incident E of every step
  double* h_aux = nullptr;   // [total_steps][nl] incident H of every half step
  double* src = nullptr;
  // ADE
  void* ade_mat = nullptr;
  void* ade_pole = nullptr;
  void* J = nullptr;
  void* Jp = nullptr;
  void* Ep = nullptr;
  long long bsx = 0, bsy = 0, bn = 0;
  // NF2FF
  double2* nf_acc = nullptr;
  double* nf_ring = nullptr;     // [kNfRing][4][npts] surface samples not yet accumulated
  long long* nf_done = nullptr;  // steps accumulated by the last flush
  double2* te = nullptr;
  double2* th = nullptr;
  int nf_off[7] = {};
  long long nf_npts = 0;
  // time-domain NF2FF (k_nftd_chunks / k_nftd_bins)
  void* td_ent = nullptr;     // int4 per point
  double* td_tsd = nullptr;   // delay in steps per point
  double* td_prev = nullptr;  // [2][td_n]
  long long td_n = 0;
  void* td_chunk = nullptr;   // int4 per chunk
  int td_nchunks = 0;
  double* td_part = nullptr;  // [td_nchunks][6]
  int* td_offs = nullptr;
  int* td_list = nullptr;
  double* td_pot = nullptr;   // [6][td_bins]
  // monitors
  long long* probe_idx = nullptr;
  int* probe_field = nullptr;
  double* probe_out = nullptr;
  std::vector<double*> movie_out;
  std::vector<long long> movie_frames;
  long long* t_dev = nullptr;
  unsigned long long* scratch_u64 = nullptr;
  int* scratch_err = nullptr;  // blocked 2-D kernel: 2 when a tile's region outgrew its psi tables
  void* plain_c[18] = {};  // per-cell coefficient arrays of the plain path
  // one-sweep step work items per tile configuration
  // (int4: k tile | region kind << 16, j tile, first plane, end plane)
  void* step_items[2] = {};
  int n_step_items[2] = {};
  // staging tensor maps of the one-sweep kernel per tile configuration and
  // read set (six field components, then the material ids), the bulk-store
  // maps of its lean interior items per tile configuration and write set
  // (Ex Ey Ez Hx Hy Hz), and its error flag (1: a staging wait ran out)
  CUtensorMap stage_maps[3][2][7];
  CUtensorMap store_maps[3][2][6];
  int* step_err = nullptr;
  // TFSF line tables of the one-sweep step, filled every step by
  // k_tfsf_lines (or, in a batch, k_tfsf_lines_batch; yh, ye: rows of pitch
  // line_ykp; zh, ze: rows of pitch line_zjp), and their tensor maps per tile
  // configuration.  Off without a TFSF source.
  bool lines_on = false;
  void* line_tab[4] = {};
  long long line_ykp = 0, line_zjp = 0;
  CUtensorMap line_maps[3][4];
  // ADE applied by k_ade_box after the one-sweep step (no dispersive cell
  // takes a TFSF or CPML correction)
  bool ade_deferred = false;
  // its work list: runs of dispersive cells (k_ade_runs); -1: no list (k_ade_box)
  void* ade_runs = nullptr;
  int n_ade_runs = -1;
  // set while a batch steps this handle (xfb_batch_*)
  xfb_batch* batch = nullptr;
  // learned absorbing boundary (xfb_set_learned_abc): BF16 weights and the
  // E(w, n-1), E(w+s, n-1) history planes of every wall
  bool labc_on = false;
  void* labc_w = nullptr;
  float* labc_hist = nullptr;
  // field read-back (read_field_t): a device gather buffer of kReadChunk
  // elements of the compute type, two pinned host buffers of the same size
  // (chunk c lands in buffer c & 1 while the host widens chunk c - 1 to
  // double), their completion events; allocated by the first read-back
  void* rb_dev = nullptr;
  void* rb_host[2] = {};
  cudaEvent_t rb_ev[2] = {};
  // bytes this handle has copied host -> device and device -> host
  long long h2d_bytes = 0, d2h_bytes = 0;
  // x-slab decomposition (xfb_set_slab): the handle updates cells
  // [slab_i0, slab_i1) along x of the full grid; planes slab_i0 - 1 and
  // slab_i1 are halos, refilled between xfb_slab_update and xfb_slab_record
  // (xfb_slab_exchange, or the host's own collective); -1: the whole grid
  int slab_i0 = 0, slab_i1 = -1;
  bool slab_pending = false;  // an update awaits its record
};

// A batch of scenes stepped together: one launch of the one-sweep kernel per
// step over the work items of every scene, or one persistent launch for a
// chunk of steps (k_step3_persist).  The handles stay owned by the caller;
// the batch owns only its tables, stream, counters and graphs.
struct xfb_batch {
  std::vector<xfb_handle*> hs;
  std::string err;
  int device = 0;
  int prec = XFB_FP32;
  cudaStream_t stream = nullptr;
  bool inited = false;
  long long step = 0, total = 0, cells = 0;
  int tile_req = 0;   // 0: autotune, else 8, 14 or 16 rows
  int tile = -1;      // tile configuration in use (-1 until chosen)
  int graph_steps = 64;
  void* scenes = nullptr;   // BatchScene<T>[n]
  void* maps = nullptr;     // BatchMaps[n]: tensor maps of every scene
  int* err_dev = nullptr;   // 1: a staging wait of the step kernel ran out
  void* items[3] = {};      // per tile configuration
  int n_items[3] = {};
  long long* t_dev = nullptr;
  std::map<int, cudaGraphExec_t> graphs;
  // persistent launches (XFB_BATCH_PERSISTENT): work lists (the per-step
  // lists, aliased), items per scene, and the queue (ticket counter, then one
  // finished-item counter per scene)
  int launch_req = XFB_BATCH_AUTO;  // xfb_batch_set_launch
  int launch = -1;                  // XFB_BATCH_PER_STEP or XFB_BATCH_PERSISTENT (-1 until chosen)
  bool persist_ok = false;          // no scene records monitors or runs a separate ADE pass
  void* pitems[3] = {};
  void* pscene_items[3] = {};
  unsigned* queue = nullptr;
  long long lines_work = 0;  // TFSF line entries of the largest scene (0: no scene has a TFSF source)
};

namespace xfb {

// ---- helpers (api.cu) ----------------------------------------------------
int set_err(xfb_handle* h, int code, const std::string& m);
int cuda_err(xfb_handle* h, cudaError_t e, const char* what);

#define XFB_CUDA(h, call)                                   \
  do {                                                      \
    cudaError_t e_ = (call);                                \
    if (e_ != cudaSuccess) return cuda_err((h), e_, #call); \
  } while (0)

template <typename T>
T* as(void* p) { return static_cast<T*>(p); }

void free_device(xfb_handle* h);
int alloc(xfb_handle* h, void** out, size_t bytes, bool state);
// n zeroed buffers of `bytes` each (256-byte aligned) from one cudaMalloc.
int alloc_block(xfb_handle* h, void** out, int n, size_t bytes, bool state);
// Every host<->device copy of the library goes through this: it is issued on
// the handle's stream (a non-blocking stream, which the legacy default stream
// does not order against) and waited for, so it lands after the zero-fill of
// alloc() and after every kernel already queued, and the host buffer may be
// released on return.
int copy(xfb_handle* h, void* dst, const void* src, size_t bytes, cudaMemcpyKind kind);

template <typename T>
int upload(xfb_handle* h, void** out, const std::vector<double>& v, bool state = false) {
  std::vector<T> tmp(v.begin(), v.end());
  int rc = alloc(h, out, tmp.size() * sizeof(T), state);
  if (rc) return rc;
  if (!tmp.empty()) return copy(h, *out, tmp.data(), tmp.size() * sizeof(T), cudaMemcpyHostToDevice);
  return XFB_OK;
}

long long roundup(long long v, long long m);
bool fused(const xfb_handle* h);
// tile configuration of the one-sweep kernel picked by the launch hint's rows
inline int step_tile_index(int tj) { return tj <= 8 ? 0 : 1; }
// tile rows of the one-sweep kernel's configurations; single scenes use the
// first two, a batch autotunes over all three
constexpr int kStepTileCount = 3;
constexpr int kStepTileRows[kStepTileCount] = {8, 16, 14};
bool plain(const xfb_handle* h);
inline bool is_slab(const xfb_handle* h) { return h->slab_i1 >= 0; }
// planes i whose cells and monitors this handle owns (the last slab also owns
// the node plane i = nx of the E components)
inline int own_lo(const xfb_handle* h) { return is_slab(h) ? h->slab_i0 : 0; }
inline int own_hi(const xfb_handle* h) {
  return is_slab(h) && h->slab_i1 < h->c.nx ? h->slab_i1 : h->c.nx + 1;
}
int cur_set(const xfb_handle* h);
void* field_ptr(const xfb_handle* h, int set, int q);
long long off3(const xfb_handle* h, int i, int j, int k);
void comp_shape(const Compiled& c, int f, int s[3]);
int nf_face_points(const Compiled& c, int face);
int launches_per_step(const xfb_handle* h);
int check_handle(xfb_handle* h, bool need_init);

// ---- engine (engine.cuh, instantiated for float and double) -------------
template <typename T> int init_device(xfb_handle* h);
template <typename T> int run_steps(xfb_handle* h, long long n);
template <typename T> int slab_update(xfb_handle* h);
template <typename T> int slab_record(xfb_handle* h);
template <typename T> int profile_steps(xfb_handle* h, long long n, double* ms, long long* launches);
template <typename T> int read_field_t(xfb_handle* h, int f, double* dst);
template <typename T> int read_bytes_t(xfb_handle* h, void* dst, const void* src, size_t bytes);
template <typename T> int write_field_t(xfb_handle* h, int f, const double* src);
template <typename T> void launch_nonfinite(xfb_handle* h);
template <typename T> int batch_init(xfb_batch* b);
template <typename T> int batch_run(xfb_batch* b, long long n);
void batch_free(xfb_batch* b);
int batch_err(xfb_batch* b, int code, const std::string& m);

}  // namespace xfb
