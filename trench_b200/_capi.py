"""ctypes binding of libtrench_b200.so (the C ABI in include/trench_b200.h).

The library is built in-tree by ``trench_b200.build``; TRENCH_B200_LIB may name
another build of the same ABI (for comparing kernel variants).  Loading fails
loudly: there is no CPU fallback anywhere in this package.
"""
import ctypes
import os
from pathlib import Path

HERE = Path(__file__).resolve().parent
LIB_PATH = Path(os.environ.get("TRENCH_B200_LIB", HERE / "libtrench_b200.so"))

TB_OK = 0
TB_ERR_ARG = 1
TB_ERR_CUDA = 2
TB_ERR_DEVICE = 3
TB_ERR_KERNEL = 4
TB_ERR_CONVERGENCE = 5
PRECISION = {"f64": 0, "f32": 1}

_vp = ctypes.c_void_p
_i32 = ctypes.c_int32
_i64 = ctypes.c_int64
_dbl = ctypes.c_double


class TraceArgs(ctypes.Structure):
    """Mirror of ``tb_trace_args``; field order and types follow the header."""
    _fields_ = [
        ("n", _i64),
        ("d_x", _vp), ("d_y", _vp), ("d_vx", _vp), ("d_vy", _vp),
        ("d_qm", _vp), ("d_spc", _vp),
        ("d_ex", _vp), ("d_ey", _vp),
        ("d_phi", _vp), ("d_wface", _vp),
        ("max_steps", ctypes.c_int), ("step_budget", ctypes.c_int),
        ("cfl", _dbl),
        ("tapered", ctypes.c_int),
        ("d_rf_ex", _vp), ("d_rf_ey", _vp), ("d_rf_phi", _vp),
        ("d_wave", _vp),
        ("n_phase", ctypes.c_int),
        ("period", _dbl), ("dt_max", _dbl), ("bound_vs", _dbl), ("bound_vm", _dbl),
        ("d_clock", _vp),
        ("record", ctypes.c_int),
        ("d_endpoints", _vp), ("d_slots", _vp), ("d_paths", _vp), ("d_path_len", _vp),
        ("path_stride", ctypes.c_int),
        ("d_counts", _vp), ("d_totals", _vp),
        ("d_status", _vp), ("d_hit", _vp), ("d_steps", _vp),
        ("write_state", ctypes.c_int),
    ]


class StepDesc(ctypes.Structure):
    """Mirror of ``tb_step_desc``."""
    _fields_ = [
        ("m", ctypes.c_int),
        ("d_surf", _vp), ("d_sflag", _vp),
        ("d_rho_s", _vp), ("d_rho_prev", _vp), ("d_work", _vp),
        ("d_leak_M", _vp), ("d_leak_h", _vp), ("d_g_s", _vp),
        ("c_slot", ctypes.c_int),
        ("floating", ctypes.c_int), ("driven", ctypes.c_int),
        ("q_macro", _dbl), ("dx", _dbl), ("C_cond", _dbl), ("Te", _dbl), ("dt_batch", _dbl),
        ("leak_norm", _dbl), ("bottom_norm", _dbl), ("n_per_batch", _dbl),
        ("n_rows", ctypes.c_int),
        ("d_rows", _vp), ("d_green", _vp), ("d_green64", _vp), ("d_ext", _vp), ("d_phi", _vp),
        ("d_ex", _vp), ("d_ey", _vp), ("d_wface", _vp),
        ("v_sub", _dbl), ("v_top", _dbl),
        ("top_dirichlet", ctypes.c_int),
        ("vscale", _dbl),
        ("d_hist", _vp),
        ("hist_cols", ctypes.c_int), ("max_batches", ctypes.c_int),
        ("n_probes", ctypes.c_int),
        ("d_probes", _vp), ("d_batch", _vp), ("d_counts", _vp), ("d_totals", _vp),
    ]


class InjectArgs(ctypes.Structure):
    """Mirror of ``tb_inject_args``."""
    _fields_ = [
        ("n_species", _i64),
        ("seed", ctypes.c_uint64), ("batch", ctypes.c_uint64),
        ("d_x", _vp), ("d_y", _vp), ("d_vx", _vp), ("d_vy", _vp), ("d_qm", _vp),
        ("d_spc", _vp),
        ("lx", _dbl), ("y0", _dbl),
        ("qm_ion", _dbl), ("qm_electron", _dbl),
        ("ion_mass", _dbl), ("e_charge", _dbl),
        ("electron_sigma", _dbl),
        ("ion_energy_eV", _dbl), ("ion_lateral_sigma", _dbl),
        ("d_energy_edges", _vp), ("d_energy_cdf", _vp),
        ("n_energy", ctypes.c_int),
        ("d_angle_edges", _vp), ("d_angle_cdf", _vp),
        ("n_angle", ctypes.c_int),
        ("angle_random_sign", ctypes.c_int),
        ("d_counter", _vp),
        ("d_bin_e", _vp), ("d_bin_a", _vp),
        ("d_clock", _vp), ("period", _dbl),
    ]


class TallyArgs(ctypes.Structure):
    """Mirror of ``tb_tally_args``."""
    _fields_ = [
        ("n_species", _i64),
        ("d_status", _vp), ("d_hit", _vp), ("d_bin_e", _vp), ("d_bin_a", _vp), ("d_slot", _vp),
        ("m", ctypes.c_int), ("n_energy", ctypes.c_int), ("n_angle", ctypes.c_int),
        ("d_table", _vp),
    ]


class AdjointArgs(ctypes.Structure):
    """Mirror of ``tb_adjoint_args``."""
    _fields_ = [
        ("n_batches", ctypes.c_int), ("n_energy", ctypes.c_int), ("n_angle", ctypes.c_int),
        ("d_tables", _vp), ("d_rE", _vp), ("d_rA", _vp), ("d_leak_MT", _vp),
        ("d_rho", _vp), ("d_scal", _vp), ("d_bottom", _vp),
        ("n_basis", ctypes.c_int),
        ("d_basis", _vp), ("d_resp_i", _vp), ("d_resp_e", _vp), ("d_resp_index", _vp),
    ]


SFLAG_COND, SFLAG_REGION, SFLAG_BOTTOM = 1, 2, 4

# Every symbol the header declares, with its ctypes signature.
SIGNATURES = {
    "tb_version": (ctypes.c_int, []),
    "tb_create": (ctypes.c_int, [ctypes.POINTER(_vp), ctypes.c_int, ctypes.c_int, ctypes.c_int, _dbl, _vp]),
    "tb_destroy": (ctypes.c_int, [_vp]),
    "tb_last_error": (ctypes.c_char_p, [_vp]),
    "tb_device_info": (ctypes.c_int, [_vp, ctypes.c_char_p, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]),
    "tb_set_fields": (ctypes.c_int, [_vp, _vp, _vp, _vp, _vp, _dbl, _vp]),
    "tb_set_rf_fields": (ctypes.c_int, [_vp, _vp, _vp, _vp, _vp, _vp, ctypes.c_int, _vp]),
    "tb_trace": (ctypes.c_int, [_vp, ctypes.POINTER(TraceArgs), ctypes.c_int, _vp]),
    "tb_check": (ctypes.c_int, [_vp, _vp]),
    "tb_set_tuning": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int]),
    "tb_set_claim_order": (ctypes.c_int, [_vp, ctypes.c_int]),
    "tb_reserve_claim_order": (ctypes.c_int, [_vp, ctypes.c_longlong]),
    "tb_poisson_setup": (ctypes.c_int, [_vp, _vp, _vp, _vp, _vp, ctypes.c_int]),
    "tb_poisson_levels": (ctypes.c_int, [_vp]),
    "tb_poisson_schedule": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    "tb_poisson_solve": (ctypes.c_int, [_vp, ctypes.c_int, _vp, _vp, _dbl, ctypes.c_int, ctypes.c_int,
                                        ctypes.POINTER(ctypes.c_int), ctypes.POINTER(_dbl), _vp]),
    "tb_step_charge": (ctypes.c_int, [_vp, ctypes.POINTER(StepDesc), _vp]),
    "tb_step_potential": (ctypes.c_int, [_vp, ctypes.POINTER(StepDesc), _vp]),
    "tb_step_monitors": (ctypes.c_int, [_vp, ctypes.POINTER(StepDesc), _vp, _vp, ctypes.c_int, _vp, _vp]),
    "tb_batch_reset": (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_longlong, _vp, ctypes.c_longlong, _vp, ctypes.c_int, _vp]),
    "tb_bench_smem": (ctypes.c_int, [_vp, ctypes.POINTER(_dbl)]),
    "tb_bench_l2_gather": (ctypes.c_int, [_vp, ctypes.c_longlong, ctypes.POINTER(_dbl)]),
    "tb_check_div_by": (ctypes.c_int, [_vp, ctypes.c_longlong, ctypes.c_ulonglong, ctypes.POINTER(ctypes.c_ulonglong)]),
    "tb_inject": (ctypes.c_int, [_vp, ctypes.POINTER(InjectArgs), _vp]),
    "tb_philox_fill": (ctypes.c_int, [_vp, ctypes.c_ulonglong, ctypes.c_ulonglong, ctypes.c_int, _vp, _vp]),
    "tb_pack_create": (ctypes.c_int, [ctypes.POINTER(_vp), ctypes.c_int, ctypes.POINTER(_vp)]),
    "tb_pack_destroy": (ctypes.c_int, [_vp]),
    "tb_pack_last_error": (ctypes.c_char_p, [_vp]),
    "tb_pack_set_args": (ctypes.c_int, [_vp, ctypes.POINTER(TraceArgs)]),
    "tb_pack_trace": (ctypes.c_int, [_vp, ctypes.c_int, _vp]),
    "tb_pack_check": (ctypes.c_int, [_vp, _vp]),
    "tb_pack_set_steps": (ctypes.c_int, [_vp, ctypes.POINTER(StepDesc)]),
    "tb_pack_step": (ctypes.c_int, [_vp, _vp]),
    "tb_tally": (ctypes.c_int, [_vp, ctypes.POINTER(TallyArgs), _vp]),
    "tb_adjoint_forward": (ctypes.c_int, [_vp, ctypes.POINTER(StepDesc), ctypes.POINTER(AdjointArgs), _vp]),
    "tb_adjoint_reverse": (ctypes.c_int, [_vp, ctypes.POINTER(StepDesc), ctypes.POINTER(AdjointArgs), _vp, _vp,
                                          _vp, _vp, _vp]),
    "tb_trace_f32_noalloc": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, _dbl, _vp, ctypes.POINTER(TraceArgs),
                                            _dbl, _vp]),
}

_lib = None


def lib():
    """Load the library once; raises RuntimeError if it is missing or incomplete."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH.name} is not built: run trench_b200.build.build() "
                               "(no CPU fallback exists)")
        h = ctypes.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(h, name)
            fn.restype = res
            fn.argtypes = args
        _lib = h
    return _lib


class TBError(RuntimeError):
    def __init__(self, code, message):
        super().__init__(message)
        self.code = code


def raise_for(code, ctx=None):
    """Map a TB status to the exception the reference raises for the same case."""
    if code == TB_OK:
        return
    msg = lib().tb_last_error(ctx).decode(errors="replace")
    if code == TB_ERR_ARG:
        raise ValueError(msg)
    raise TBError(code, msg)
