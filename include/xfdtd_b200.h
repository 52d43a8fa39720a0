/*
 * xfdtd_b200.h -- C-ABI of the B200-native FDTD engine.
 *
 * This is the drop-in boundary for the GPU path of XFDTD_CUDA.  The reference
 * exposes one C++ class, xfdtd::cuda::SimulationHD
 * (include/xfdtd_cuda/simulation/simulation_hd.cuh:37-88), built from an
 * XFDTD_CORE xfdtd::Simulation.  XFDTD_CORE (the host scene library) is not
 * part of the reference, so the scene enters here as a plain description
 * (xfb_scene) and the engine compiles it on the host (voxelisation, update
 * coefficients, CPML profiles, TFSF geometry, NF2FF surfaces) exactly where
 * XFDTD_CORE's Simulation::init would have done it.
 *
 * Conventions
 *  - Every call returns an int status (XFB_OK == 0).  No C++ exception crosses
 *    this boundary.  xfb_last_error() gives the message of the last failure on
 *    a handle (thread-local message for calls without a handle).
 *  - A handle owns one CUDA stream on the device that was current when it was
 *    created.  A handle is not thread-safe.
 *  - Grid indices follow the reference layout: row-major (i, j, k), k fastest
 *    (include/xfdtd_cuda/tensor.cuh:203-212); the box has nx*ny*nz cells and the
 *    Yee component shapes are Ex (nx, ny+1, nz+1), Ey (nx+1, ny, nz+1),
 *    Ez (nx+1, ny+1, nz), Hx (nx+1, ny, nz), Hy (nx, ny+1, nz),
 *    Hz (nx, ny, nz+1).  In 2-D (TMz) nz == 1.
 *  - All host-side read-back buffers are double precision, whatever precision
 *    the device computes in.
 */
#ifndef XFDTD_B200_H_
#define XFDTD_B200_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define XFB_ABI_VERSION 2

/* ---- status codes ------------------------------------------------------- */
#define XFB_OK 0
#define XFB_ERR_INVALID 1   /* bad argument or scene                        */
#define XFB_ERR_CUDA 2      /* CUDA runtime error                            */
#define XFB_ERR_OOM 3       /* device or host allocation failed              */
#define XFB_ERR_STATE 4     /* call not allowed in the current state         */
#define XFB_ERR_RANGE 5     /* index / id out of range                       */
#define XFB_ERR_NUMERIC 6   /* non-finite value detected by the watchdog      */
#define XFB_ERR_TIMEOUT 7   /* a bounded device wait gave up                 */
#define XFB_ERR_NO_DEVICE 8 /* no CUDA device available                      */

/* ---- enumerations ------------------------------------------------------- */
enum xfb_precision { XFB_FP32 = 0, XFB_FP64 = 1 };
enum xfb_field { XFB_EX = 0, XFB_EY = 1, XFB_EZ = 2, XFB_HX = 3, XFB_HY = 4, XFB_HZ = 5 };
enum xfb_face { XFB_XN = 0, XFB_XP = 1, XFB_YN = 2, XFB_YP = 3, XFB_ZN = 4, XFB_ZP = 5 };
enum xfb_shape { XFB_SHAPE_CUBE = 0, XFB_SHAPE_SPHERE = 1, XFB_SHAPE_CYLINDER = 2 };
enum xfb_pole_kind {
  XFB_POLE_DEBYE = 0,    /* p = {delta_eps, tau}                         */
  XFB_POLE_DRUDE = 1,    /* p = {omega_p, gamma}                         */
  XFB_POLE_LORENTZ = 2,  /* p = {delta_eps, omega_0, delta}              */
  XFB_POLE_MLORENTZ = 3  /* p = {a0, a1, b0, b1, b2}:
                            chi(w) = (a0 + a1 jw) / (b0 + b1 jw + b2 (jw)^2) */
};
enum xfb_waveform { XFB_WAVE_GAUSSIAN = 0, XFB_WAVE_COS_GAUSSIAN = 1 };
/* surface-current selector of one NF2FF face (reference: ja, jb, ma, mb,
 * src/include/nf2ff/frequency_domain/nf2ff_frequency_domain_data.cuh:336) */
enum xfb_current { XFB_JA = 0, XFB_JB = 1, XFB_MA = 2, XFB_MB = 3 };
/* which E update the scene needs (the reference picks one updator for the
 * whole grid: src/simulation/simulation_hd.cu:407-503) */
enum xfb_ade_kind { XFB_ADE_NONE = 0, XFB_ADE_DEBYE = 1, XFB_ADE_DRUDE = 2, XFB_ADE_MLORENTZ = 3 };
/* How a 3-D time step is executed.  SPLIT: an H half-step kernel and an E
 * half-step kernel (the reference's updateH/updateE split, correctors fused).
 * FUSED: one kernel per step that sweeps the grid once (H and E together,
 * ping-pong field buffers).  PLAIN: the reference's own GPU structure kept as
 * a baseline -- 18 per-cell coefficient arrays, one launch per field
 * component with flat (i, j, k) indexing, CPML and TFSF corrections as
 * separate launches per face (src/include/updator/update_scheme.cuh:132-197,
 * src/boundary/pml_corrector.cu:9-291,
 * src/waveform_source/tfsf/tfsf_corrector.cu:155-271); 3-D scenes without
 * dispersive media only.  AUTO: FUSED (3-D and 2-D TMz). */
enum xfb_kernel_path { XFB_PATH_AUTO = 0, XFB_PATH_SPLIT = 1, XFB_PATH_FUSED = 2, XFB_PATH_PLAIN = 3 };

#define XFB_MAX_POLES 4
#define XFB_MAX_MATERIALS 255

/* ---- scene description -------------------------------------------------- */
typedef struct xfb_pole {
  int kind; /* enum xfb_pole_kind */
  double p[5];
} xfb_pole;

typedef struct xfb_material {
  double eps_r;   /* relative permittivity (eps_inf of a dispersive medium) */
  double mu_r;    /* relative permeability                                  */
  double sigma_e; /* electric conductivity, S/m                              */
  double sigma_m; /* magnetic conductivity, Ohm/m                            */
  int is_pec;     /* perfect electric conductor: E held at zero              */
  int n_poles;    /* 0 .. XFB_MAX_POLES dispersive poles                     */
  xfb_pole poles[XFB_MAX_POLES];
} xfb_material;

/* Shapes.  CUBE: p[0..2] min corner, p[3..5] size (may be +inf).
 * SPHERE: p[0..2] centre, p[3] radius.
 * CYLINDER: p[0..2] centre of the circular section, p[3] radius, p[4] axis
 * (0=x, 1=y, 2=z), p[5] length along the axis centred on the centre (+inf:
 * infinite).  The last object containing a cell centre decides its material. */
typedef struct xfb_object {
  int shape;
  int material;
  double p[8];
} xfb_object;

typedef struct xfb_pml {
  int cells[6];        /* CPML thickness per face (enum xfb_face); 0 = PEC wall */
  double order_m;      /* polynomial grading order (default 3)              */
  double sigma_ratio;  /* sigma_max / sigma_opt (default 1)                  */
  double alpha_max;    /* CFS alpha at the interface (default 0.05)         */
} xfb_pml;

typedef struct xfb_tfsf {
  int enabled;
  int inset[3];        /* cells between the inner domain edge and the TF box */
  double theta, phi, psi; /* incidence direction and polarisation, rad     */
  int waveform;        /* enum xfb_waveform                                  */
  double tau, t0, freq;   /* waveform parameters (s, s, Hz)                  */
} xfb_tfsf;

typedef struct xfb_nf2ff {
  int enabled;
  int inset[3];        /* cells between the inner domain edge and the box    */
  int n_freqs;
  const double* freqs; /* Hz */
} xfb_nf2ff;

/* Time-domain near-to-far-field transformation for one observation
 * direction: the retarded-time potentials of the equivalent surface currents
 * on a box (the reference's NFFFTTimeDomain path,
 * src/nf2ff/time_domain/nf2ff_time_domain_data.cu:113-175,
 * nf2ff_time_domain_hd.cu:1-234). */
typedef struct xfb_nf2ff_td {
  int enabled;
  int inset[3];        /* cells between the inner domain edge and the box    */
  double theta, phi;   /* observation direction, rad                        */
} xfb_nf2ff_td;

typedef struct xfb_probe {
  int field;           /* enum xfb_field */
  int index[3];        /* component index (i, j, k) */
} xfb_probe;

typedef struct xfb_movie {
  int field;           /* enum xfb_field */
  int lo[3], hi[3];    /* half-open component-index box */
  int interval;        /* a frame every `interval` steps, starting at step 0 */
} xfb_movie;

typedef struct xfb_scene {
  int dim;             /* 3 or 2 (TMz: Ez, Hx, Hy) */
  int precision;       /* enum xfb_precision */
  double dx, dy, dz;
  double courant;      /* dt = courant / (c * sqrt(sum 1/d^2)) */
  double domain_min[3];   /* physical corner of the inner domain (no PML) */
  int domain_cells[3];    /* inner cells per axis (nz = 1 in 2-D) */
  int n_materials;        /* materials[0] is the background */
  const xfb_material* materials;
  int n_objects;
  const xfb_object* objects;
  xfb_pml pml;
  xfb_tfsf tfsf;
  xfb_nf2ff nf2ff;
  int n_probes;
  const xfb_probe* probes;
  int n_movies;
  const xfb_movie* movies;
  xfb_nf2ff_td nf2ff_td;
} xfb_scene;

/* ---- grid information --------------------------------------------------- */
typedef struct xfb_grid_info {
  int dim, precision;
  int nx, ny, nz;            /* total cells including CPML */
  double dx, dy, dz, dt;
  double origin[3];          /* physical position of node (0,0,0) */
  int n_materials;
  int ade_kind;              /* enum xfb_ade_kind */
  int ade_poles;
  int tfsf_box[6];           /* is, ie, js, je, ks, ke (nodes) or zeros */
  int nf2ff_box[6];          /* is, ie, js, je, ks, ke (nodes) or zeros */
  int n_freqs;
  long long current_step;    /* steps taken since the last init */
  long long total_steps;     /* steps the last init sized its buffers for */
  size_t device_bytes;       /* device memory held by the handle */
  long long n_dispersive_cells; /* cells whose material has ADE poles */
  int launches_per_step;     /* engine kernels one time step launches */
  int kernel_path;           /* enum xfb_kernel_path in use (after init) */
  int nf2ff_td_box[6];       /* time-domain NF2FF box (nodes) or zeros */
  long long h2d_bytes;       /* bytes the handle has copied host -> device */
  long long d2h_bytes;       /* bytes the handle has copied device -> host */
} xfb_grid_info;

typedef struct xfb_handle xfb_handle;

/* ---- lifecycle ---------------------------------------------------------- */

/* Compile a scene on the host (no device work).  Replaces the reference
 * constructor SimulationHD(xfdtd::Simulation*)
 * (include/xfdtd_cuda/simulation/simulation_hd.cuh:39) together with the
 * XFDTD_CORE Simulation::init it triggers (src/simulation/simulation_hd.cu:259-267). */
int xfb_create(const xfb_scene* scene, xfb_handle** out);

/* Release every device and host resource.  Replaces ~SimulationHD and
 * SimulationHD::releaseDevice (simulation_hd.cuh:41,47). */
int xfb_destroy(xfb_handle* h);

/* Device ordinal the handle will use (default: the device current at the
 * first xfb_init).  Must be called before the first xfb_init. */
int xfb_set_device(xfb_handle* h, int ordinal);

/* Launch-shape hint.  Replaces SimulationHD::setGridDim / setBlockDim
 * (simulation_hd.cuh:53,55).  The engine sizes its own grid; the thread count
 * of the block hint (bx*by*bz, a multiple of 32, at most 1024) selects the
 * bulk-update tile: 32 lanes along k times (threads/32) rows along j. */
int xfb_set_launch_hint(xfb_handle* h, const unsigned grid[3], const unsigned block[3]);

/* Allocate and zero device state for a run of `total_steps` steps (sizes the
 * movie, probe and NF2FF-transform buffers).  Replaces SimulationHD::init
 * (simulation_hd.cuh:51) plus copyHostToDevice (simulation_hd.cuh:43). */
int xfb_init(xfb_handle* h, long long total_steps);

/* Reference run(n) (simulation_hd.cuh:49; src/simulation/simulation_hd.cu:106-257):
 * re-initialise for n steps, advance n steps, wait for the device.  Results
 * stay on the device until read. */
int xfb_run(xfb_handle* h, long long n_steps);

/* Advance n more steps from the current state (no re-initialisation; n must
 * not take the run beyond the steps xfb_init sized for).  Asynchronous. */
int xfb_step(xfb_handle* h, long long n_steps);

/* Block until the handle's stream is idle; reports device-side errors.
 * XFB_ERR_TIMEOUT: a bounded wait of the step kernel ran out (see
 * xfb_set_wait_limit); the run's results are incomplete, and this sync and
 * every read-back return the same status until the next xfb_init. */
int xfb_sync(xfb_handle* h);

/* Diagnostics, no counterpart in the reference.  The 3-D one-sweep step
 * stages its planes with asynchronous bulk copies and waits for each with a
 * bounded poll loop (default limit 4194304 polls, far beyond any copy's
 * latency).  A wait that runs out lets the copies in flight land, ends its
 * work item and sets the handle's error flag instead of hanging the device.
 * This call sets the limit (after xfb_init; 0 makes every wait give up at
 * once, which tests use to exercise that path without a device fault). */
int xfb_set_wait_limit(xfb_handle* h, int polls);

/* Advance n steps bracketed by CUDA events on the handle's stream (after a
 * synchronize); *ms = elapsed device time of the n steps. */
int xfb_timed_step(xfb_handle* h, long long n, double* ms);

/* Kernel classes of one time step, for xfb_profile_kernels (XFB_K_AUX: the
 * per-step TFSF line values of the one-sweep 3-D step). */
enum xfb_kernel_class {
  XFB_K_UPDATE_H = 0, XFB_K_AUX = 1, XFB_K_UPDATE_E = 2, XFB_K_NF2FF = 3, XFB_K_PROBE = 4,
  XFB_K_MOVIE = 5, XFB_K_STEP = 6, XFB_K_CORRECT = 7, XFB_K_COUNT = 8
};
/* Advance n steps launching every kernel individually with CUDA events around
 * it; ms[c] = summed device time and launches[c] = launch count of class c
 * (arrays of XFB_K_COUNT). */
int xfb_profile_kernels(xfb_handle* h, long long n, double* ms, long long* launches);

/* Select the 3-D kernel path (enum xfb_kernel_path); before xfb_init. */
int xfb_set_kernel_path(xfb_handle* h, int path);

/* 2-D TMz scenes on the one-sweep path: steps advanced per launch by the
 * temporally blocked kernel (each CTA advances its tile plus a halo of that
 * many cells in shared memory and records its probes every step), odd, at
 * most 31; default 9; 0 launches once per step.  Scenes with movie monitors
 * or CPML slabs wider than a tile's psi tables step once per launch.  Results
 * are identical either way.  Before xfb_init. */
int xfb_set_temporal_block(xfb_handle* h, int steps);

/* Storage trial of the update coefficients, no counterpart in the reference
 * (its 18 per-cell coefficient arrays are FP64, fdtd_coefficient.cuh:15-168).
 * NATIVE keeps them in the compute precision; FP16 / BF16 round every entry
 * of the material LUT to that 16-bit format at xfb_init (the arithmetic
 * stays in the compute precision), to measure what 16-bit storage would cost
 * in accuracy.  The LUT sits in shared memory, not on the HBM stream, so
 * 16-bit storage would save no bandwidth.  Before xfb_init. */
enum xfb_coeff_storage { XFB_COEFF_NATIVE = 0, XFB_COEFF_FP16 = 1, XFB_COEFF_BF16 = 2 };
int xfb_set_coeff_storage(xfb_handle* h, int storage);

/* Use CUDA-graph replay of the step loop (default 1) and the steps per
 * captured graph (default 64). */
int xfb_set_graph(xfb_handle* h, int enabled, int steps_per_graph);

int xfb_get_grid_info(const xfb_handle* h, xfb_grid_info* out);

/* ---- read-back (reference copyDeviceToHost, simulation_hd.cuh:45) -------- */

/* One field component in its reference shape, converted to double. */
int xfb_read_field(xfb_handle* h, int field, double* dst, size_t dst_len);
/* Fault in the pages of a host range that results will be read into (a
 * field or NF2FF destination), on background host threads, and return at
 * once; contents are unchanged.  A read into fresh memory otherwise pays the
 * page faults of every destination page (about 5x slower than into resident
 * memory), so a caller that allocates its result arrays ahead of a run (as
 * XFDTD_CORE allocates the host fields in Simulation::init) lets the faults
 * run while the device initialises and steps (it may be called between
 * xfb_create and xfb_init for that).  The range must stay allocated
 * until the handle's next read, far-field or get_state call,
 * xfb_host_prefault_wait or xfb_destroy; each of these waits for the threads
 * first. */
int xfb_host_prefault(xfb_handle* h, void* ptr, size_t bytes);
int xfb_host_prefault_wait(xfb_handle* h);

/* Overwrite one field component (reference shape, double) - initial values. */
int xfb_write_field(xfb_handle* h, int field, const double* src, size_t src_len);
/* Time series of probe `id` (one value per step taken, double). */
int xfb_read_probe(xfb_handle* h, int id, double* dst, size_t dst_len, long long* n_written);
/* Movie frames of monitor `id`: [frames, lo..hi box] in double; the reference
 * MovieMonitor<F>::update frame rule (src/monitor/movie_monitor.cu:17-46). */
int xfb_movie_shape(const xfb_handle* h, int id, int shape_out[4]);
int xfb_read_movie(xfb_handle* h, int id, double* dst, size_t dst_len);
/* NF2FF surface current `which` (enum xfb_current) of `face` at frequency
 * `freq`: complex, interleaved (re, im), face extent shape.  The reference
 * NF2FFFrequencyDomainData<D>::calculateJ/M accumulators
 * (src/nf2ff/frequency_domain/nf2ff_frequency_domain.data.cu:80-194). */
int xfb_nf2ff_face_shape(const xfb_handle* h, int face, int shape_out[3]);
int xfb_read_nf2ff(xfb_handle* h, int freq, int face, int which, double* dst, size_t dst_len);
/* All surface currents of frequency `freq` in one read: [which 0..3][points],
 * complex interleaved, the six faces one after another in face order, each
 * in its xfb_nf2ff_face_shape (so face f of current w starts at point
 * w * points + the sizes of faces 0..f-1).  dst_len >= 8 * points doubles;
 * *points (optional) receives the face points of all six faces. */
int xfb_read_nf2ff_all(xfb_handle* h, int freq, double* dst, size_t dst_len, long long* points);
/* Far field from the accumulated surface currents, computed on the device.
 * For each (theta[i], phi[i]) writes 4 doubles: Re/Im E_theta, Re/Im E_phi of
 * r*E (the e^{-jkr} factor removed), in the e^{+jwt} phasor convention of the
 * DFT.  Replaces XFDTD_CORE NFFFTFrequencyDomain::processFarField, which the
 * reference calls on the host (test/dielectric_sphere_scatter.cu:85-91). */
int xfb_far_field(xfb_handle* h, int freq, int n_angles, const double* theta,
                  const double* phi, double* out);

/* Same far field as xfb_far_field, computed without allocating device memory.
 * No counterpart in the reference.  For hosts that cannot allocate on the
 * device once they are running: frameworks that hand the solver a fixed
 * device-memory budget at start-up and treat any later cudaMalloc as a fault,
 * and latency-bound loops where cudaMalloc/cudaFree would stall the device.
 * xfb_far_field allocates its angle and output buffers per call; this entry
 * point uses one fixed device array of the library instead (192 KiB on every
 * device that loads the library, kept until process exit), so it accepts at
 * most XFB_FAR_FIELD_STATIC_MAX_ANGLES angles per call and returns
 * XFB_ERR_RANGE beyond that.  The caller still passes the host angle and
 * output arrays.  The first call on a device looks the array's device address
 * up (cudaGetSymbolAddress) and caches it; make that first call before any
 * stream capture.  All calls on a device share the one array: calls that
 * overlap on the GPU (e.g. two handles on different streams) race, so keep
 * them apart.  Nothing needs clearing between calls: every output entry of the
 * n angles is rewritten by each call. */
#define XFB_FAR_FIELD_STATIC_MAX_ANGLES 4096
int xfb_far_field_static(xfb_handle* h, int freq, int n_angles, const double* theta,
                         const double* phi, double* out);

/* Time-domain NF2FF (scene.nf2ff_td).  Every step adds, for every face point
 * and both field kinds, the time difference of the interpolated tangential
 * field times the face area into the time bins of its retarded arrival, with
 * linear weights between two bins (nf2ff_time_domain_data.cu:150-170):
 * W from the electric surface current J = n x H, U from the magnetic surface
 * current M = -n x E, each a vector of x, y, z components, summed over the
 * six faces.  The reference runs this update on one GPU thread because its
 * reduction over face points was never written (nf2ff_time_domain_data.cu:174,
 * 213-223); here every face point has a thread and the bins are summed by a
 * deterministic two-level reduction, so results do not depend on the launch
 * and match a sequential sum to round-off.  Bin n is observation time n*dt
 * after the wave leaves the box point farthest along the direction. */
int xfb_nf2ff_td_bins(const xfb_handle* h, long long* n_bins);
/* which = 0, 1, 2: W_x, W_y, W_z; 3, 4, 5: U_x, U_y, U_z (n_bins doubles). */
int xfb_read_nf2ff_td(xfb_handle* h, int which, double* dst, size_t dst_len);
/* r E_theta(t_n) and r E_phi(t_n), n < n_bins, from the potentials
 * (Luebbers et al., IEEE Trans. Antennas Propag. 39(4), 1991):
 * r E_theta = -(U_phi + eta W_theta) / (4 pi c dt),
 * r E_phi = (U_theta - eta W_phi) / (4 pi c dt).  Replaces XFDTD_CORE
 * NFFFTTimeDomain::processFarField. */
int xfb_far_field_td(xfb_handle* h, double* e_theta, double* e_phi, size_t len);

/* ---- learned absorbing boundary --------------------------------------------
 * No counterpart in the reference.  A small MLP (8 -> 64 -> 64 -> 1, tanh,
 * BF16 weights, FP32 accumulation) corrects the first-order Mur value of the
 * tangential E of every outer wall cell at step n+1, from a 3-cell-deep
 * stencil (the wall plane and the two planes inside it at steps n-1, n, n+1,
 * plus a transverse Laplacian, all divided by their largest magnitude), in
 * place of a CPML layer; all-zero weights give the plain Mur boundary.  The network
 * is trained on the device by xfb_mlp_train on samples taken from the
 * engine's own CPML runs (xfdtd_cuda_b200/labc.py builds them). */
/* Number of MLP parameters (layout W1[64][8], b1[64], W2[64][64], b2[64], w3[64], b3). */
int xfb_mlp_param_count(void);
/* Mean squared error of the network with weights w (rounded to BF16 for the
 * forward pass) over n samples (x: [n][8], y: [n]) and its gradient with
 * respect to the weights; computed on the device. */
int xfb_mlp_loss_grad(const float* x, const float* y, int n, const float* w, double* loss, float* grad);
/* Full-batch Adam on the device for iters steps from w_init; w_out gets the
 * FP32 master weights, loss_curve (may be NULL) the loss before each step. */
int xfb_mlp_train(const float* x, const float* y, int n, int iters, float lr, const float* w_init, float* w_out,
                  double* loss_curve);
const char* xfb_mlp_last_error(void);
/* Use the network on every wall of a 3-D one-sweep scene without CPML (after
 * xfb_init; NULL weights switch it off).  The walls stay PEC without it. */
int xfb_set_learned_abc(xfb_handle* h, const float* weights, int n_weights);
/* Wall cells the learned boundary updates per step. */
int xfb_labc_wall_cells(const xfb_handle* h, long long* cells);

/* ---- batches of scenes ---------------------------------------------------
 * No counterpart in the reference (whose SimulationHD runs one scene per
 * object).  A batch steps many 3-D scenes of one precision together: every
 * step is one launch of the one-sweep kernel over the work items of all
 * scenes, plus one launch for all TFSF auxiliary grids, replayed from CUDA
 * graphs.  Results are identical to stepping each scene alone.  The handles
 * stay owned by the caller and are read as usual (xfb_read_field, ...) after
 * xfb_batch_sync; while in a batch they cannot be stepped, initialised or
 * destroyed on their own (XFB_ERR_STATE). */
typedef struct xfb_batch xfb_batch;
/* Group n created handles (same precision, 3-D, one device). */
int xfb_batch_create(xfb_handle* const* handles, int n, xfb_batch** out);
/* Tile rows of the one-sweep kernel: 0 = autotune on the first steps (default), 8, 14 or 16. */
int xfb_batch_set_tile(xfb_batch* b, int rows);
/* How the steps are launched.  XFB_BATCH_PER_STEP: one launch of the
 * one-sweep kernel per step.  XFB_BATCH_PERSISTENT: one launch per chunk of
 * steps (up to the graph chunk), whose resident CTAs take the work items of
 * all steps from a device queue; an item of step s starts once every item of
 * step s - 1 of its scene is done (bounded waits, XFB_ERR_TIMEOUT as for the
 * staging waits), so a scene's next step overlaps the end of the current
 * step of the others.  Only for batches whose scenes record no monitors (NF2FF,
 * probes, movies) and run no separate ADE pass, which the per-step form
 * launches between steps; otherwise XFB_ERR_INVALID.  XFB_BATCH_AUTO (default)
 * times both on the first steps, together with the tile rows, and keeps the
 * faster. */
enum xfb_batch_launch { XFB_BATCH_AUTO = 0, XFB_BATCH_PER_STEP = 1, XFB_BATCH_PERSISTENT = 2 };
int xfb_batch_set_launch(xfb_batch* b, int launch);
/* The launch form in use (0 before the first step). */
int xfb_batch_launch_form(const xfb_batch* b, int* launch);
/* xfb_init every scene for total_steps steps (one-sweep path) and build the batch's work list. */
int xfb_batch_init(xfb_batch* b, long long total_steps);
/* Advance every scene n steps (asynchronous). */
int xfb_batch_step(xfb_batch* b, long long n);
/* XFB_ERR_TIMEOUT as for xfb_sync when a bounded wait of the step ran out. */
int xfb_batch_sync(xfb_batch* b);
/* Poll limit of the batch step's bounded waits (after xfb_batch_init), as
 * xfb_set_wait_limit. */
int xfb_batch_set_wait_limit(xfb_batch* b, int polls);
/* n steps between CUDA events on the batch's stream; *ms = device time. */
int xfb_batch_timed_step(xfb_batch* b, long long n, double* ms);
/* Cells per step over all scenes, tile rows in use (0 before the first step), work items per step. */
int xfb_batch_info(const xfb_batch* b, long long* cells, int* tile_rows, int* work_items);
const char* xfb_batch_last_error(const xfb_batch* b);
/* Release the batch; its handles become independent again. */
int xfb_batch_destroy(xfb_batch* b);

/* ---- x-slab decomposition -----------------------------------------------
 * No counterpart in the reference (its one multi-node path is XFDTD_CORE's
 * CPU MPI).  A handle can update only the cells [i0, i1) along x of its
 * scene, so N handles on N devices step one grid together.  Every step is:
 * xfb_slab_update on every slab (the one-sweep update of the owned planes;
 * the H plane below the slab is recomputed from the halo), then the halo
 * exchange -- each slab's first owned plane to the lower neighbour's upper
 * halo, its last owned plane to the upper neighbour's lower halo (the six
 * components of the set the update wrote, and upward the H-side psi of the y
 * and z CPML slabs) -- then xfb_slab_record on every slab (monitors of the
 * owned planes, step counter).  Monitors record only what a slab owns (probes,
 * movie planes, NF2FF face points and time-domain sums by plane), so the sum
 * over the slabs of every read-back is the whole grid's.  The arrays are
 * allocated at full size on every device.  A slab boundary s must leave the
 * plane s - 1 outside the x CPML; learned boundaries and batches take whole
 * grids only. */
int xfb_set_slab(xfb_handle* h, int i0, int i1);  /* before xfb_init */
int xfb_get_slab(const xfb_handle* h, int* i0, int* i1);
int xfb_slab_update(xfb_handle* h);
/* The device buffers of one side of the exchange, in the set the pending
 * update wrote: which = 0 the first owned plane (sent down), 1 the last owned
 * plane (sent up), 2 the lower halo (received from below), 3 the upper halo
 * (received from above).  *n buffers (at most 10): the plane of Ex Ey Ez Hx
 * Hy Hz, and on the upward direction (1 and 2) also the plane of the H-side
 * CPML psi of the y and z slabs, which the H halo of the slab above reads.
 * Buffer q of side 1 of a slab goes to buffer q of side 2 of the slab above;
 * buffer q of side 0 to buffer q of side 3 of the slab below.  Between update
 * and record only. */
int xfb_slab_planes(xfb_handle* h, int which, void* ptrs[10], size_t sizes[10], int* n);
/* The exchange between two neighbouring slabs of one process (peer copies,
 * same or different devices; waits for both updates, returns when done). */
int xfb_slab_exchange(xfb_handle* lo, xfb_handle* hi);
int xfb_slab_record(xfb_handle* h);

/* ---- checkpoint / resume ------------------------------------------------ */
/* Byte size of the full solver state (fields, CPML psi, ADE state, TFSF
 * auxiliary grid, NF2FF accumulators, monitors, step counter). */
int xfb_state_size(const xfb_handle* h, size_t* bytes);
int xfb_get_state(xfb_handle* h, void* dst, size_t dst_len);
int xfb_set_state(xfb_handle* h, const void* src, size_t src_len);

/* ---- status -------------------------------------------------------------- */
/* Scan the fields for non-finite values; *bad = number of non-finite entries.
 * Returns XFB_ERR_NUMERIC when any is found. */
int xfb_check_finite(xfb_handle* h, long long* bad);
const char* xfb_last_error(const xfb_handle* h);
const char* xfb_status_string(int status);
int xfb_abi_version(void);

/* ---- scenes compiled by XFDTD_CORE ----------------------------------------
 * The arrays XFDTD_CORE's Simulation::init computes and the reference's *HD
 * wrappers copy to the device (src/simulation/simulation_hd.cu:259-398:
 * FDTDCoefficientHD, fdtd_coefficient_hd.cu:9-51; PMLCorrectorHD,
 * pml_corrector_hd.cu:8-34; TFSFCorrectorHD, tfsf_corrector_hd.cu:9-73;
 * the NF2FF and monitor wrappers; ADEMethodStorageHD, ade_method_hd.cu:5-24),
 * as plain host arrays.  include/xfdtd_b200/xfdtd_core_adapter.hpp fills this
 * struct from an xfdtd::Simulation.  3-D scenes; every array is row-major
 * (k fastest) and is read, not kept, by xfb_create_from_arrays. */
typedef struct xfb_core_arrays {
  int precision;                /* enum xfb_precision of the device engine  */
  int nx, ny, nz;               /* cells, CPML included                      */
  double dx, dy, dz, dt;
  double origin[3];             /* position of node (0, 0, 0)                */
  /* the 18 FDTDCoefficient arrays (cexe cexhy cexhz ceye ceyhz ceyhx ceze
   * cezhx cezhy chxh chxey chxez chyh chyez chyex chzh chzex chzey), each in
   * the shape of its field (Ex (nx, ny+1, nz+1) ... Hz (nx, ny, nz+1)) */
  const double* coeff[18];
  /* ADE (enum xfb_ade_kind, NONE without dispersive media): per cell
   * (nx, ny, nz) the dispersive flag, ceep and cejsum; per cell and pole
   * (nx, ny, nz, poles) cjj cjjp cjen cje cjep cjsj cjsjp */
  int ade_kind, ade_poles;
  const double* ade_cell[3];
  const double* ade_pole[7];
  /* CPML thickness per face and the profiles along each axis: a/b of the E
   * nodes (length n + 1), of the H half nodes (length n), zero outside */
  int pml[6];
  const double* pml_ae[3];
  const double* pml_be[3];
  const double* pml_ah[3];
  const double* pml_bh[3];
  /* TFSF: box nodes, projections (length box_n + 1 and box_n + 2), field
   * transforms, ca/cb per axis, and the incident tables: e_inc row t = E at
   * t dt (aux_nl + 1 entries, inc_steps + 1 rows), h_inc row t = H at
   * (t + 1/2) dt (aux_nl entries, inc_steps rows) */
  int tfsf_enabled;
  int tfsf_box[6];
  const double* tfsf_proj_int[3];
  const double* tfsf_proj_half[3];
  double tfsf_transform_e[3], tfsf_transform_h[3], tfsf_ca[3], tfsf_cb[3];
  int aux_nl;
  long long inc_steps;
  const double* e_inc;
  const double* h_inc;
  /* frequency-domain NF2FF: box nodes and frequencies */
  int nf2ff_enabled;
  int nf2ff_box[6];
  int n_freqs;
  const double* freqs;
  /* time-domain NF2FF: box nodes and the observation direction (rad) */
  int nf2ff_td_enabled;
  int nf2ff_td_box[6];
  double nf2ff_td_theta, nf2ff_td_phi;
  int n_probes;
  const xfb_probe* probes;
  int n_movies;
  const xfb_movie* movies;
} xfb_core_arrays;

/* A handle from arrays XFDTD_CORE compiled: the replacement of
 * SimulationHD(xfdtd::Simulation*) for callers that keep XFDTD_CORE.  Cells
 * whose 18 coefficients (and ADE coefficients) are bitwise equal share a
 * material of the engine's coefficient table: at most 255 distinct sets, each
 * of the isotropic form the update uses (cexhy = -ceyhx, ...), else
 * XFB_ERR_INVALID.  xfb_init may not size a run beyond inc_steps. */
int xfb_create_from_arrays(const xfb_core_arrays* arrays, xfb_handle** out);

/* ---- compiled-scene export (host only; used by the CPU restatement) ------ */
/* The arrays the host scene compiler produced, i.e. what XFDTD_CORE would hand
 * to the reference's *HD wrappers.  Pointers stay valid until xfb_destroy. */
typedef struct xfb_compiled_view {
  int dim, nx, ny, nz;
  double dx, dy, dz, dt;
  const uint8_t* material_id;   /* [nx][ny][nz] cell material index          */
  int n_materials;
  const double* coeff;          /* [n_materials][18] cexe cexhy cexhz ceye ceyhz
                                   ceyhx ceze cezhx cezhy chxh chxey chxez chyh
                                   chyez chyex chzh chzex chzey               */
  int ade_kind, ade_poles;
  const double* ade_mat;        /* [n_materials][3] is_dispersive ceep cejsum */
  const double* ade_pole;       /* [n_materials][poles][7] cjj cjjp cjen cje
                                   cjep cjsj cjsjp                            */
  int pml_cells[6];
  const double* pml_ae[3];      /* per axis, length n_axis+1 (E nodes)        */
  const double* pml_be[3];
  const double* pml_ah[3];      /* per axis, length n_axis (H half nodes)     */
  const double* pml_bh[3];
  int tfsf_enabled;
  int tfsf_box[6];
  const double* tfsf_proj_int[3];  /* length box_n+1 */
  const double* tfsf_proj_half[3]; /* length box_n+2 */
  double tfsf_transform_e[3], tfsf_transform_h[3];
  double tfsf_ca[3], tfsf_cb[3];
  int aux_nl;                   /* aux E nodes 0..nl, H nodes 0..nl-1        */
  double aux_ceih, aux_chie, aux_abc;
  const double* aux_source;     /* E source at aux node 0, index t = time t*dt;
                                   length total_steps+1 (valid after init)    */
  long long total_steps;
  int nf2ff_enabled;
  int nf2ff_box[6];
  int n_freqs;
  const double* freqs;
  const double* nf2ff_te;       /* [n_freqs][total_steps] complex (re,im)    */
  const double* nf2ff_th;
  int nf2ff_td_enabled;
  int nf2ff_td_box[6];          /* is ie js je ks ke (nodes)                 */
  double nf2ff_td_theta, nf2ff_td_phi;
  long long nf2ff_td_bins;      /* time bins of the potentials (after init)  */
  double origin[3];             /* physical position of node (0, 0, 0)      */
  int ade_box[6];               /* i0 i1 j0 j1 k0 k1: cell bounds of the
                                   dispersive cells (all 0 when none)        */
} xfb_compiled_view;

int xfb_compiled_view_get(const xfb_handle* h, xfb_compiled_view* out);

/* Host only: size the step-count dependent tables (TFSF source samples,
 * NF2FF DFT kernels) for a run of total_steps steps without touching a
 * device, so xfb_compiled_view_get exposes them.  xfb_init calls it. */
int xfb_prepare_tables(xfb_handle* h, long long total_steps);

#ifdef __cplusplus
}
#endif

#endif /* XFDTD_B200_H_ */
