"""ctypes binding of the engine's C-ABI (include/xfdtd_b200.h).

The shared library is built in-tree (xfdtd_cuda_b200/libxfdtd_b200.so).  There
is no fallback path: if the library is missing or fails to load, every entry
point raises.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "libxfdtd_b200.so"

XFB_OK = 0
XFB_ERR_INVALID, XFB_ERR_CUDA, XFB_ERR_OOM, XFB_ERR_STATE = 1, 2, 3, 4
XFB_ERR_RANGE, XFB_ERR_NUMERIC, XFB_ERR_TIMEOUT, XFB_ERR_NO_DEVICE = 5, 6, 7, 8
XFB_FP32, XFB_FP64 = 0, 1
EX, EY, EZ, HX, HY, HZ = range(6)
XN, XP, YN, YP, ZN, ZP = range(6)
SHAPE_CUBE, SHAPE_SPHERE, SHAPE_CYLINDER = 0, 1, 2
POLE_DEBYE, POLE_DRUDE, POLE_LORENTZ, POLE_MLORENTZ = 0, 1, 2, 3
WAVE_GAUSSIAN, WAVE_COS_GAUSSIAN = 0, 1
JA, JB, MA, MB = 0, 1, 2, 3
ADE_NONE, ADE_DEBYE, ADE_DRUDE, ADE_MLORENTZ = 0, 1, 2, 3
MAX_POLES = 4
FAR_FIELD_STATIC_MAX_ANGLES = 4096  # XFB_FAR_FIELD_STATIC_MAX_ANGLES
BATCH_AUTO, BATCH_PER_STEP, BATCH_PERSISTENT = 0, 1, 2  # xfb_batch_set_launch
K_UPDATE_H, K_AUX, K_UPDATE_E, K_NF2FF, K_PROBE, K_MOVIE, K_STEP, K_CORRECT, K_COUNT = range(9)
KERNEL_NAMES = ("k_h3/k_h2 (H half-step)", "k_tfsf_lines (TFSF line values of the step)", "k_e3/k_e2 (E half-step)", "k_nf2ff",
                "k_probe", "k_movie", "k_step3 (one-sweep H+E step)",
                "boundary corrections (plain CPML/TFSF launches; k_labc_apply of the learned boundary)")
PATH_AUTO, PATH_SPLIT, PATH_FUSED, PATH_PLAIN = 0, 1, 2, 3
COEFF_NATIVE, COEFF_FP16, COEFF_BF16 = 0, 1, 2


class Pole(C.Structure):
    _fields_ = [("kind", C.c_int), ("p", C.c_double * 5)]


class Material(C.Structure):
    _fields_ = [
        ("eps_r", C.c_double), ("mu_r", C.c_double), ("sigma_e", C.c_double), ("sigma_m", C.c_double),
        ("is_pec", C.c_int), ("n_poles", C.c_int), ("poles", Pole * MAX_POLES),
    ]


class Object(C.Structure):
    _fields_ = [("shape", C.c_int), ("material", C.c_int), ("p", C.c_double * 8)]


class Pml(C.Structure):
    _fields_ = [("cells", C.c_int * 6), ("order_m", C.c_double), ("sigma_ratio", C.c_double), ("alpha_max", C.c_double)]


class Tfsf(C.Structure):
    _fields_ = [
        ("enabled", C.c_int), ("inset", C.c_int * 3), ("theta", C.c_double), ("phi", C.c_double), ("psi", C.c_double),
        ("waveform", C.c_int), ("tau", C.c_double), ("t0", C.c_double), ("freq", C.c_double),
    ]


class Nf2ff(C.Structure):
    _fields_ = [("enabled", C.c_int), ("inset", C.c_int * 3), ("n_freqs", C.c_int), ("freqs", C.POINTER(C.c_double))]


class Nf2ffTd(C.Structure):
    _fields_ = [("enabled", C.c_int), ("inset", C.c_int * 3), ("theta", C.c_double), ("phi", C.c_double)]


class Probe(C.Structure):
    _fields_ = [("field", C.c_int), ("index", C.c_int * 3)]


class Movie(C.Structure):
    _fields_ = [("field", C.c_int), ("lo", C.c_int * 3), ("hi", C.c_int * 3), ("interval", C.c_int)]


class Scene(C.Structure):
    _fields_ = [
        ("dim", C.c_int), ("precision", C.c_int),
        ("dx", C.c_double), ("dy", C.c_double), ("dz", C.c_double), ("courant", C.c_double),
        ("domain_min", C.c_double * 3), ("domain_cells", C.c_int * 3),
        ("n_materials", C.c_int), ("materials", C.POINTER(Material)),
        ("n_objects", C.c_int), ("objects", C.POINTER(Object)),
        ("pml", Pml), ("tfsf", Tfsf), ("nf2ff", Nf2ff),
        ("n_probes", C.c_int), ("probes", C.POINTER(Probe)),
        ("n_movies", C.c_int), ("movies", C.POINTER(Movie)),
        ("nf2ff_td", Nf2ffTd),
    ]


class GridInfo(C.Structure):
    _fields_ = [
        ("dim", C.c_int), ("precision", C.c_int), ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
        ("dx", C.c_double), ("dy", C.c_double), ("dz", C.c_double), ("dt", C.c_double),
        ("origin", C.c_double * 3), ("n_materials", C.c_int), ("ade_kind", C.c_int), ("ade_poles", C.c_int),
        ("tfsf_box", C.c_int * 6), ("nf2ff_box", C.c_int * 6), ("n_freqs", C.c_int),
        ("current_step", C.c_longlong), ("total_steps", C.c_longlong), ("device_bytes", C.c_size_t),
        ("n_dispersive_cells", C.c_longlong), ("launches_per_step", C.c_int), ("kernel_path", C.c_int),
        ("nf2ff_td_box", C.c_int * 6), ("h2d_bytes", C.c_longlong), ("d2h_bytes", C.c_longlong),
    ]


_dp = C.POINTER(C.c_double)


class CoreArrays(C.Structure):
    """xfb_core_arrays: a scene as the arrays XFDTD_CORE compiles."""
    _fields_ = [
        ("precision", C.c_int), ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
        ("dx", C.c_double), ("dy", C.c_double), ("dz", C.c_double), ("dt", C.c_double), ("origin", C.c_double * 3),
        ("coeff", _dp * 18), ("ade_kind", C.c_int), ("ade_poles", C.c_int), ("ade_cell", _dp * 3), ("ade_pole", _dp * 7),
        ("pml", C.c_int * 6), ("pml_ae", _dp * 3), ("pml_be", _dp * 3), ("pml_ah", _dp * 3), ("pml_bh", _dp * 3),
        ("tfsf_enabled", C.c_int), ("tfsf_box", C.c_int * 6), ("tfsf_proj_int", _dp * 3), ("tfsf_proj_half", _dp * 3),
        ("tfsf_transform_e", C.c_double * 3), ("tfsf_transform_h", C.c_double * 3), ("tfsf_ca", C.c_double * 3),
        ("tfsf_cb", C.c_double * 3), ("aux_nl", C.c_int), ("inc_steps", C.c_longlong), ("e_inc", _dp), ("h_inc", _dp),
        ("nf2ff_enabled", C.c_int), ("nf2ff_box", C.c_int * 6), ("n_freqs", C.c_int), ("freqs", _dp),
        ("nf2ff_td_enabled", C.c_int), ("nf2ff_td_box", C.c_int * 6), ("nf2ff_td_theta", C.c_double),
        ("nf2ff_td_phi", C.c_double), ("n_probes", C.c_int), ("probes", C.POINTER(Probe)), ("n_movies", C.c_int), ("movies", C.POINTER(Movie)),
    ]


class CompiledView(C.Structure):
    _fields_ = [
        ("dim", C.c_int), ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
        ("dx", C.c_double), ("dy", C.c_double), ("dz", C.c_double), ("dt", C.c_double),
        ("material_id", C.POINTER(C.c_uint8)), ("n_materials", C.c_int), ("coeff", _dp),
        ("ade_kind", C.c_int), ("ade_poles", C.c_int), ("ade_mat", _dp), ("ade_pole", _dp),
        ("pml_cells", C.c_int * 6),
        ("pml_ae", _dp * 3), ("pml_be", _dp * 3), ("pml_ah", _dp * 3), ("pml_bh", _dp * 3),
        ("tfsf_enabled", C.c_int), ("tfsf_box", C.c_int * 6),
        ("tfsf_proj_int", _dp * 3), ("tfsf_proj_half", _dp * 3),
        ("tfsf_transform_e", C.c_double * 3), ("tfsf_transform_h", C.c_double * 3),
        ("tfsf_ca", C.c_double * 3), ("tfsf_cb", C.c_double * 3),
        ("aux_nl", C.c_int), ("aux_ceih", C.c_double), ("aux_chie", C.c_double), ("aux_abc", C.c_double),
        ("aux_source", _dp), ("total_steps", C.c_longlong),
        ("nf2ff_enabled", C.c_int), ("nf2ff_box", C.c_int * 6), ("n_freqs", C.c_int), ("freqs", _dp),
        ("nf2ff_te", _dp), ("nf2ff_th", _dp),
        ("nf2ff_td_enabled", C.c_int), ("nf2ff_td_box", C.c_int * 6), ("nf2ff_td_theta", C.c_double),
        ("nf2ff_td_phi", C.c_double), ("nf2ff_td_bins", C.c_longlong), ("origin", C.c_double * 3),
        ("ade_box", C.c_int * 6),
    ]


# (name, restype, argtypes) of every exported entry point in include/xfdtd_b200.h
_H = C.c_void_p
SIGNATURES = [
    ("xfb_abi_version", C.c_int, []),
    ("xfb_status_string", C.c_char_p, [C.c_int]),
    ("xfb_last_error", C.c_char_p, [_H]),
    ("xfb_create", C.c_int, [C.POINTER(Scene), C.POINTER(_H)]),
    ("xfb_create_from_arrays", C.c_int, [C.POINTER(CoreArrays), C.POINTER(_H)]),
    ("xfb_destroy", C.c_int, [_H]),
    ("xfb_set_device", C.c_int, [_H, C.c_int]),
    ("xfb_set_launch_hint", C.c_int, [_H, C.POINTER(C.c_uint), C.POINTER(C.c_uint)]),
    ("xfb_init", C.c_int, [_H, C.c_longlong]),
    ("xfb_run", C.c_int, [_H, C.c_longlong]),
    ("xfb_step", C.c_int, [_H, C.c_longlong]),
    ("xfb_sync", C.c_int, [_H]),
    ("xfb_set_wait_limit", C.c_int, [_H, C.c_int]),
    ("xfb_timed_step", C.c_int, [_H, C.c_longlong, C.POINTER(C.c_double)]),
    ("xfb_profile_kernels", C.c_int, [_H, C.c_longlong, C.POINTER(C.c_double), C.POINTER(C.c_longlong)]),
    ("xfb_set_graph", C.c_int, [_H, C.c_int, C.c_int]),
    ("xfb_set_kernel_path", C.c_int, [_H, C.c_int]),
    ("xfb_set_coeff_storage", C.c_int, [_H, C.c_int]),
    ("xfb_set_temporal_block", C.c_int, [_H, C.c_int]),
    ("xfb_get_grid_info", C.c_int, [_H, C.POINTER(GridInfo)]),
    ("xfb_read_field", C.c_int, [_H, C.c_int, _dp, C.c_size_t]),
    ("xfb_host_prefault", C.c_int, [_H, C.c_void_p, C.c_size_t]),
    ("xfb_host_prefault_wait", C.c_int, [_H]),
    ("xfb_write_field", C.c_int, [_H, C.c_int, _dp, C.c_size_t]),
    ("xfb_read_probe", C.c_int, [_H, C.c_int, _dp, C.c_size_t, C.POINTER(C.c_longlong)]),
    ("xfb_movie_shape", C.c_int, [_H, C.c_int, C.c_int * 4]),
    ("xfb_read_movie", C.c_int, [_H, C.c_int, _dp, C.c_size_t]),
    ("xfb_nf2ff_face_shape", C.c_int, [_H, C.c_int, C.c_int * 3]),
    ("xfb_read_nf2ff", C.c_int, [_H, C.c_int, C.c_int, C.c_int, _dp, C.c_size_t]),
    ("xfb_read_nf2ff_all", C.c_int, [_H, C.c_int, _dp, C.c_size_t, C.POINTER(C.c_longlong)]),
    ("xfb_far_field", C.c_int, [_H, C.c_int, C.c_int, _dp, _dp, _dp]),
    ("xfb_far_field_static", C.c_int, [_H, C.c_int, C.c_int, _dp, _dp, _dp]),
    ("xfb_nf2ff_td_bins", C.c_int, [_H, C.POINTER(C.c_longlong)]),
    ("xfb_read_nf2ff_td", C.c_int, [_H, C.c_int, _dp, C.c_size_t]),
    ("xfb_far_field_td", C.c_int, [_H, _dp, _dp, C.c_size_t]),
    ("xfb_mlp_param_count", C.c_int, []),
    ("xfb_mlp_loss_grad", C.c_int, [C.POINTER(C.c_float), C.POINTER(C.c_float), C.c_int, C.POINTER(C.c_float),
                                    C.POINTER(C.c_double), C.POINTER(C.c_float)]),
    ("xfb_mlp_train", C.c_int, [C.POINTER(C.c_float), C.POINTER(C.c_float), C.c_int, C.c_int, C.c_float,
                                C.POINTER(C.c_float), C.POINTER(C.c_float), C.POINTER(C.c_double)]),
    ("xfb_mlp_last_error", C.c_char_p, []),
    ("xfb_set_learned_abc", C.c_int, [_H, C.POINTER(C.c_float), C.c_int]),
    ("xfb_labc_wall_cells", C.c_int, [_H, C.POINTER(C.c_longlong)]),
    ("xfb_batch_create", C.c_int, [C.POINTER(C.c_void_p), C.c_int, C.POINTER(C.c_void_p)]),
    ("xfb_batch_set_tile", C.c_int, [C.c_void_p, C.c_int]),
    ("xfb_batch_set_launch", C.c_int, [C.c_void_p, C.c_int]),
    ("xfb_batch_launch_form", C.c_int, [C.c_void_p, C.POINTER(C.c_int)]),
    ("xfb_batch_init", C.c_int, [C.c_void_p, C.c_longlong]),
    ("xfb_batch_step", C.c_int, [C.c_void_p, C.c_longlong]),
    ("xfb_batch_sync", C.c_int, [C.c_void_p]),
    ("xfb_batch_set_wait_limit", C.c_int, [C.c_void_p, C.c_int]),
    ("xfb_batch_timed_step", C.c_int, [C.c_void_p, C.c_longlong, C.POINTER(C.c_double)]),
    ("xfb_batch_info", C.c_int, [C.c_void_p, C.POINTER(C.c_longlong), C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    ("xfb_batch_last_error", C.c_char_p, [C.c_void_p]),
    ("xfb_batch_destroy", C.c_int, [C.c_void_p]),
    ("xfb_set_slab", C.c_int, [_H, C.c_int, C.c_int]),
    ("xfb_get_slab", C.c_int, [_H, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    ("xfb_slab_update", C.c_int, [_H]),
    ("xfb_slab_planes", C.c_int, [_H, C.c_int, C.c_void_p * 10, C.c_size_t * 10, C.POINTER(C.c_int)]),
    ("xfb_slab_exchange", C.c_int, [_H, _H]),
    ("xfb_slab_record", C.c_int, [_H]),
    ("xfb_state_size", C.c_int, [_H, C.POINTER(C.c_size_t)]),
    ("xfb_get_state", C.c_int, [_H, C.c_void_p, C.c_size_t]),
    ("xfb_set_state", C.c_int, [_H, C.c_void_p, C.c_size_t]),
    ("xfb_check_finite", C.c_int, [_H, C.POINTER(C.c_longlong)]),
    ("xfb_compiled_view_get", C.c_int, [_H, C.POINTER(CompiledView)]),
    ("xfb_prepare_tables", C.c_int, [_H, C.c_longlong]),
]

_lib = None


def load(path: Path | str | None = None) -> C.CDLL:
    """Load libxfdtd_b200.so (built in-tree) and declare every signature."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    # XFB_LIBRARY selects another build of the same library (same C-ABI)
    p = Path(path) if path else Path(os.environ.get("XFB_LIBRARY", LIB_PATH))
    if not p.exists():
        raise RuntimeError(
            f"{p} is missing: build it with `python -m xfdtd_cuda_b200.build` "
            "(the engine has no CPU fallback)")
    lib = C.CDLL(str(p))
    for name, res, args in SIGNATURES:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib


class XfbError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"[{status}] {message}")
        self.status = status


def check(status: int, handle=None) -> None:
    if status != XFB_OK:
        lib = load()
        msg = lib.xfb_last_error(handle)
        raise XfbError(status, (msg or b"").decode() or lib.xfb_status_string(status).decode())
