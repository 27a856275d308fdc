"""ctypes binding of libpetchb200.so (the C ABI declared in include/petch_b200.h).

Every call takes raw device pointers; the helpers here turn torch CUDA tensors into pointers and
raise PetchError on a non-zero status.  There is no CPU fallback: if the library is missing the
first call raises.
"""
import ctypes
import os

import torch

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libpetchb200.so")

P = ctypes.c_void_p
I = ctypes.c_int  # noqa: E741
L = ctypes.c_longlong
F = ctypes.c_float
D = ctypes.c_double

U = ctypes.c_uint32
LLP = ctypes.POINTER(ctypes.c_longlong)


class Domain(ctypes.Structure):
    """petch_domain"""
    _fields_ = [("lx", F), ("ly", F), ("lz", F), ("z_src", F), ("periodic", I)]


class IonParams(ctypes.Structure):
    """petch_ion_params"""
    _fields_ = [(n, F) for n in ("meanE", "sigmaE", "A_sp", "Eth_sp", "B_sp", "A_ie", "Eth_ie",
                                 "A_p", "Eth_p", "inflect", "minang", "n_l", "A_en", "minE",
                                 "thrmin", "thrmax", "sigma")]


class ChemParams(ctypes.Structure):
    """petch_chem_params"""
    _fields_ = [(n, D) for n in ("ionFlux", "Fflux", "Oflux", "k_sigma", "beta_sigma", "rho",
                                 "rate_scale", "fnorm_E", "fnorm_O", "s_F", "s_O", "Yie", "Ysp",
                                 "Yp", "B_sp")] + [("yield_angular", I), ("chemistry", I)]


class BatchItem(ctypes.Structure):
    """petch_batch_item."""
    _fields_ = [("mesh", ctypes.c_void_p), ("dom", Domain), ("ion", IonParams),
                ("bare", ctypes.c_void_p), ("out", ctypes.c_void_p), ("ang", ctypes.c_void_p),
                ("n_rays", ctypes.c_int), ("seed", ctypes.c_uint32)]


class BatchGrid(ctypes.Structure):
    """petch_batch_grid."""
    _fields_ = [("phi", ctypes.c_void_p), ("tmp", ctypes.c_void_p), ("ua", ctypes.c_void_p),
                ("ub", ctypes.c_void_p), ("F", ctypes.c_void_p), ("mask_phi", ctypes.c_void_p),
                ("mask_idx", ctypes.c_void_p), ("n_mask", ctypes.c_int),
                ("active", ctypes.c_void_p), ("n_active", ctypes.c_void_p),
                ("max_active", ctypes.c_int), ("nx", ctypes.c_int), ("ny", ctypes.c_int),
                ("nz", ctypes.c_int), ("dx", ctypes.c_double), ("dt", ctypes.c_double),
                ("stats", ctypes.c_void_p), ("hdr", ctypes.c_void_p), ("sub", ctypes.c_void_p),
                ("hold", ctypes.c_void_p)]


class BatchTangent(ctypes.Structure):
    """petch_batch_tangent."""
    _fields_ = [("dout", ctypes.c_void_p), ("dbare", ctypes.c_void_p)]


class BatchTangentGrid(ctypes.Structure):
    """petch_batch_tangent_grid."""
    _fields_ = [("dphi", ctypes.c_void_p), ("dtmp", ctypes.c_void_p), ("dF", ctypes.c_void_p),
                ("mask", ctypes.c_void_p), ("du_a", ctypes.c_void_p), ("du_b", ctypes.c_void_p)]


class StepConfig(ctypes.Structure):
    """petch_step_config."""
    _fields_ = [("nx", I), ("ny", I), ("nz", I), ("dx", D), ("Lx", D), ("Ly", D), ("Lz", D),
                ("sub_top", D), ("mask_th", D), ("trench_width", D), ("hole", I), ("dt", D),
                ("n_ion", I), ("n_neu", I), ("seed_offset", I), ("max_tris", I), ("n_fp", I),
                ("warm_start", I), ("n_smooth", I), ("smooth_alpha", F), ("betaE", F),
                ("betaO", F), ("dom", Domain), ("ion", IonParams), ("chem", ChemParams)]


class StepStatus(ctypes.Structure):
    """petch_step_status."""
    _fields_ = [("steps", I), ("faces", I), ("max_faces", I), ("trace_errors", I),
                ("mesh_errors", I), ("nonfinite", I), ("nsub", I), ("nsub_max", I), ("vmax", F),
                ("queries", L)]


DP = ctypes.POINTER(Domain)
IP = ctypes.POINTER(IonParams)
CP = ctypes.POINTER(ChemParams)

# name -> argtypes (restype is int status for all of them)
SIGNATURES = {
    "petch_abi_version": [],
    "petch_launch_count": [LLP],
    "petch_last_error": [ctypes.c_char_p, I],
    "petch_seed_level_set": [P, P, I, I, I, D, D, D, D, D, D, I, P],
    "petch_advect": [P, P, P, P, P, I, I, I, F, F, I, P],
    "petch_reinit_eik": [P, P, P, P, I, I, I, D, F, F, I, I, P],
    "petch_reinit_eik_noalloc": [P, P, I, I, I, D, F, F, I, I, P],
    "petch_mesh_layout": [I, I, LLP, I, LLP],
    "petch_mesh_scratch_bytes": [I, I, I, I, LLP],
    "petch_mesh_build": [P, I, I, I, D, D, D, D, D, D, I, P, I, I, P, L, P],
    "petch_trace_ions": [P, I, I, DP, IP, U, I, P, P, P, P],
    "petch_trace_neutrals": [P, I, I, DP, P, F, U, U, I, P, P, P],
    "petch_trace_legacy": [P, I, I, DP, I, F, F, I, I, F, F, U, I, P, P, P, P],
    "petch_trace_electrons": [P, I, I, DP, F, U, I, P, P, P],
    "petch_trace_neutral_pair": [P, I, I, DP, P, F, F, U, U, U, I, P, P, P, P],
    "petch_extend_velocity": [P, I, I, P, P, I, I, I, D, D, P, P, I, P, P, I, P, P],
    "petch_warmstart": [P, I, I, P, P, I, I, P, P, P],
    "petch_norm_smooth": [P, I, I, P, F, F, F, I, I, F, P, P, P, P],
    "petch_ion_post": [P, I, I, P, P, F, I, F, P, P, P, P, P, P, P],
    "petch_cos_ratio": [P, I, I, P, P, P, P],
    "petch_belen_bare": [P, I, I, CP, P, P, P, P, P, P, P, P],
    "petch_surface_rate": [P, I, I, CP, P, P, P, P, P, P, P, P, P, P],
    "petch_advect_sparse": [P, P, P, P, P, I, P, I, I, I, I, F, F, I, P],
    "petch_raycast": [P, I, I, P, P, I, F, P, P, P, P],
    "petch_tracer_config": [I, I, I],
    "petch_tally_aggregation": [I],
    "petch_stencil_config": [I, I],
    "petch_tracer_settings": [P],
    "petch_tracer_grouping": [I],
    "petch_nearest_face": [P, I, I, P, I, F, P, P, P],
    "petch_gas_normals": [P, I, I, P, I, I, I, D, P, P],
    "petch_trace_ff": [P, I, I, DP, P, U, I, P, P, P],
    "petch_ff_scratch_bytes": [I, I, LLP],
    "petch_ff_matrix": [P, I, I, P, I, P, P, P, P, L, P],
    "petch_radiosity_solve": [P, I, I, P, P, P, I, P, D, D, I, P, P, P, P],
    "petch_radiosity_solve_tangent": [P, I, I, P, P, P, I, P, P, D, D, I, P, P, P, P, P, P],
    "petch_radiosity_gmres_scratch_bytes": [I, I, LLP],
    "petch_radiosity_gmres": [P, I, I, P, P, P, I, P, D, D, I, I, P, P, L, P, P],
    "petch_dda_scratch_bytes": [I, I, I, I, I, LLP],
    "petch_dda_prepare": [P, I, I, I, D, D, I, I, P, I, P, P, P, P, P, I, P, L, P],
    "petch_dda_solve": [I, I, I, I, I, P, D, D, I, P, L, P, P, P],
    "petch_knudsen_scratch_bytes": [I, I, LLP],
    "petch_knudsen_prepare": [P, I, I, I, D, D, I, P, I, P, P, D, D, D, P, L, P],
    "petch_knudsen_solve": [I, I, P, P, D, D, I, D, D, I, D, D, D, D, P, L, P, P, P],
    "petch_knudsen_profile": [I, I, P, P, D, P, L, P, P],
    "petch_knudsen_slices": [I, I, P, L, P, P, P],
    "petch_charging_floor_stats": [P, I, P, P, P, P, D, D, D, I, D, D, P, P],
    "petch_charging_apply": [P, I, P, P, D, D, D, I, D, P, P, D, P, P, P, P, P],
    "petch_zero_below": [P, I, P, D, P, P],
    "petch_electron_shadow": [P, I, P, D, D, D, P, P],
    "petch_column_floors": [P, I, I, I, P, I, P, P],
    "petch_extend_velocity_centroid": [P, I, I, P, P, I, I, I, D, D, P, P, I, P, P, I, P, P],
    "petch_reinit_pde": [P, P, P, P, I, I, I, D, I, P],
    "petch_gaussian_smooth": [P, P, P, P, P, I, I, I, D, D, P],
    "petch_redep_scratch_bytes": [I, LLP],
    "petch_trace_redep": [P, I, I, DP, P, P, F, U, I, P, P, P, L, P, P],
    "petch_redep_apply": [P, I, I, P, P, I, F, P, P, P, P],
    "petch_trace_batch": [I, P, I, I, I, F, P, U, U, P, P],
    "petch_trace_batch_pair": [P, I, I, I, F, F, P, U, U, U, P, P],
    "petch_prepare_device": [],
    "petch_set_deterministic": [P, L],
    "petch_trace_ions_tangent": [P, I, I, DP, IP, U, I, P, P, P, P, P],
    "petch_trace_neutrals_tangent": [P, I, I, DP, P, P, F, U, U, I, P, P, P, P],
    "petch_trace_neutral_pair_tangent": [P, I, I, DP, P, P, F, F, U, U, U, I, P, P, P, P, P, P],
    "petch_norm_smooth_tangent": [P, I, I, P, P, F, F, F, I, I, F, I, P, P, P, P],
    "petch_belen_bare_tangent": [P, I, I, CP, P, P, P, P, P, P, P, P, P, P, P, P],
    "petch_surface_rate_tangent": [P, I, I, CP, P, P, P, P, P, P, P, P, P, P, P, P, P, P, P, P],
    "petch_extend_tangent": [P, I, I, P, I, I, I, D, D, P, P, P, P],
    "petch_warmstart_tangent": [P, I, I, P, P, P, I, I, P, P, P],
    "petch_advect_tangent": [P, P, P, P, P, P, P, P, I, I, I, F, F, I, P],
    "petch_reinit_tangent": [P, P, P, P, P, P, I, I, I, D, F, F, I, P],
    "petch_batch_advect": [P, I, P],
    "petch_batch_reinit": [P, I, D, P],
    "petch_batch_step_advance": [P, P],
    "petch_trace_batch_tangent": [I, P, P, I, I, I, F, P, U, U, P, P],
    "petch_trace_batch_pair_tangent": [P, P, P, I, I, I, F, F, P, U, U, U, P, P],
    "petch_batch_advect_tangent": [P, P, I, P],
    "petch_batch_reinit_tangent": [P, P, I, D, P],
    "petch_extend_velocity_dual": [P, I, I, P, P, I, I, I, D, D, P, P, P, P, I, P, P, I, P, P],
    "petch_warmstart_dual": [P, I, I, P, P, P, I, I, P, P, P, P],
    "petch_plan": [ctypes.POINTER(StepConfig), P, I, ctypes.POINTER(P), P],
    "petch_step": [P, P],
    "petch_plan_status": [P, ctypes.POINTER(StepStatus), P],
    "petch_plan_seek": [P, L],
    "petch_plan_timing": [P, I],
    "petch_plan_trace_ms": [P, ctypes.POINTER(ctypes.c_float)],
    "petch_plan_mask": [P, P, P],
    "petch_destroy": [P],
}

# The library's tracer configuration at load (bvh_width, steps_per_round, keep_lanes): what
# petch_tracer_config restores to.
TRACER_DEFAULT = (2, 32, 16)
TRACER_GROUPING_DEFAULT = 2

_det_scratch = None


def set_deterministic(max_entries):
    """Deterministic (order-independent, bit-reproducible) tallies for every later trace call,
    with device scratch for max_entries tally entries (8 bytes each; a batch of B instances of
    capacity MT needs about 5 * B * MT); max_entries = 0 switches back to float atomics."""
    import torch
    global _det_scratch
    if max_entries <= 0:
        call("petch_set_deterministic", None, 0)
        _det_scratch = None
        return
    nbytes = 8 * int(max_entries) + 256 * 64
    _det_scratch = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
    call("petch_set_deterministic", _det_scratch.data_ptr(), nbytes)

_lib = None


class PetchError(RuntimeError):
    def __init__(self, status, what, msg):
        super().__init__(f"{what} failed with status {status}: {msg}")
        self.status = status


def lib():
    """The loaded library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with petch_b200.build.build()")
        so = ctypes.CDLL(LIB_PATH)
        for name, args in SIGNATURES.items():
            fn = getattr(so, name)
            fn.argtypes = args
            fn.restype = ctypes.c_int
        _lib = so
    return _lib


def last_error():
    buf = ctypes.create_string_buffer(512)
    lib().petch_last_error(buf, 512)
    return buf.value.decode(errors="replace")


def call(name, *args):
    """Invoke `name`; raise PetchError unless it returns PETCH_OK."""
    rc = getattr(lib(), name)(*args)
    if rc != 0:
        raise PetchError(rc, name, last_error())
    return rc


def ptr(t):
    """Device pointer of a CUDA tensor (None -> NULL)."""
    if t is None:
        return None
    if not t.is_cuda:
        raise ValueError("expected a CUDA tensor")
    if not t.is_contiguous():
        raise ValueError("expected a contiguous tensor")
    return t.data_ptr()


def launch_count():
    """Kernel launches enqueued by libpetchb200.so so far."""
    n = ctypes.c_longlong()
    call("petch_launch_count", ctypes.byref(n))
    return int(n.value)


def stream_ptr(stream=None):
    s = stream if stream is not None else torch.cuda.current_stream()
    return s.cuda_stream
