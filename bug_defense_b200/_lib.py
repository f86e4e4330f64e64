"""ctypes binding of libbugdef.so (the C ABI declared in include/bugdef.h).

The product path has no fallback: if the library or a CUDA device is missing, every
compute entry point raises RuntimeError (the reference raises RuntimeError for
engine='gpu' without a device, simulation/voxel_mc_3d.py:563-565).
"""
from __future__ import annotations

import ctypes
import os
from ctypes import (POINTER, Structure, c_char_p, c_double, c_float, c_int, c_int32, c_int64,
                    c_size_t, c_uint8, c_uint64, c_void_p)
from pathlib import Path

_HERE = Path(__file__).resolve().parent
LIB_PATH = _HERE / "_native" / "libbugdef.so"

BD_OK = 0
BD_ERR_INVALID_ARG = 1
BD_ERR_CUDA = 2
BD_ERR_OUT_OF_MEMORY = 3
BD_ERR_TIMEOUT = 4
BD_ERR_NO_DEVICE = 5
BD_ERR_STATE = 6

FLAG_ABLATED = 0x01
FLAG_DRY = 0x02
FLAG_VOID = 0x04

LEDGER_LAUNCHED = 0
LEDGER_SPECULAR = 1
LEDGER_DIFFUSE = 2
LEDGER_TRANSMITTED = 3
LEDGER_LATERAL = 4
LEDGER_ABSORBED = 5
LEDGER_ABSORBED_VOID = 6
LEDGER_ROULETTE_GAIN = 7
LEDGER_ROULETTE_LOSS = 8
LEDGER_TRUNCATED = 9
LEDGER_COLLISIONS = 10
LEDGER_CROSSINGS = 11
LEDGER_REFLECTIONS = 12
LEDGER_LEN = 16

BEAM_PROFILES = {'gaussian': 0, 'tophat': 1, 'kim_exp_disk': 2, 'kim_gauss_disk': 3}

MC_TALLY_FLUENCE = 0x1
MC_METAL_SEMANTICS = 0x2

BC_SERIES = 0
BC_METAL = 1

PLUME_DT_AS_GIVEN = 0
PLUME_DT_METAL = 1
PLUME_DT_SUBCYCLE = 2


class McParams(Structure):
    _fields_ = [
        ("nx", c_int32), ("ny", c_int32), ("nz", c_int32), ("launch_axis", c_int32),
        ("dx", c_float), ("dy", c_float), ("dz", c_float),
        ("lx", c_float), ("ly", c_float), ("lz", c_float),
        ("init_ux", c_float), ("init_uy", c_float), ("init_uz", c_float),
        ("cos_ph", c_float), ("sin_ph", c_float), ("cos_th_safe", c_float),
        ("x_center", c_float), ("y_center", c_float), ("z_center", c_float),
        ("sigma_axis", c_float), ("beam_radius", c_float), ("beam_profile", c_int32),
        ("n_ambient", c_float), ("r_max_sq", c_float), ("options", c_int32), ("_pad0", c_int32),
        ("n_photons", c_int64), ("photon_offset", c_int64), ("max_events", c_int64),
        ("seed", c_uint64),
    ]


class ThermalParams(Structure):
    _fields_ = [
        ("nx", c_int32), ("ny", c_int32), ("nz", c_int32), ("is_active", c_int32),
        ("dx", c_float), ("dy", c_float), ("dz", c_float), ("dt", c_float),
        ("h_eff", c_float), ("t_ambient", c_float), ("bc_mode", c_int32), ("q_scale", c_float),
    ]


class AblationParams(Structure):
    _fields_ = [
        ("nx", c_int32), ("ny", c_int32), ("nz", c_int32), ("is_active", c_int32),
        ("dx", c_float), ("dy", c_float), ("dz", c_float), ("dt", c_float),
        ("h_eff", c_float), ("t_ambient", c_float), ("t_abl", c_float), ("t_void", c_float),
        ("bc_mode", c_int32), ("has_arrhenius", c_int32), ("arr_A", c_float), ("arr_Ea_over_R", c_float),
        ("has_char", c_int32), ("char_A", c_float), ("char_Ea_over_R", c_float),
        ("q_scale", c_float), ("zero_src_in_ablated", c_int32),
    ]


class PlumeParams(Structure):
    _fields_ = [
        ("nx", c_int32), ("ny", c_int32), ("nz", c_int32), ("dt_policy", c_int32),
        ("dx", c_float), ("dy", c_float), ("dz", c_float), ("dt", c_float),
        ("D_xy", c_float), ("D_z", c_float), ("vz", c_float), ("tau_linger", c_float),
        ("n_sub", c_int32), ("_pad0", c_int32),
    ]


FLAG_NEWLY = 0x08
EPOCH_SKIP_MC = 0x1
EPOCH_NO_GRAPH = 0x2
EPOCH_SERIAL_PLUME = 0x4
EPOCH_EXTERNAL_PLUME = 0x8


class GridRef(Structure):
    _fields_ = [("ptr", c_void_p), ("value", c_float), ("_pad", c_int32)]


_F = c_void_p
_PHASE_FIELDS = [
    ("nx", c_int32), ("ny", c_int32), ("nz", c_int32), ("single_stage", c_int32), ("apply_removal", c_int32),
    ("has_char_state", c_int32), ("has_cs_mu_a", c_int32), ("has_cs_mu_s", c_int32), ("has_cs_k", c_int32),
    ("has_cs_rho_cp", c_int32), ("gap_k0", c_int32), ("gap_k1", c_int32), ("has_plume", c_int32),
    ("t_abl", c_float), ("alpha_max_stable", c_float), ("cs_chi_remove", c_float), ("k_void", c_float),
    ("rho_cp_void", c_float), ("t_void", c_float),
    ("plume_delta_mu", c_float), ("plume_mu_max", c_float), ("plume_ratio_a", c_float), ("plume_ratio_s", c_float),
    ("plume_g", c_float),
    ("T", _F), ("H_acc", _F), ("chi", _F), ("mu_a", _F), ("mu_s", _F), ("g", _F), ("n", _F), ("k", _F),
    ("rho_cp", _F), ("T_peak", _F), ("ablation_time", _F),
    ("h_lat", _F), ("wet_mu_a", _F), ("wet_k", _F), ("wet_rho_cp", _F),
    ("ds_mu_a", GridRef), ("ds_mu_s", GridRef), ("ds_g", GridRef), ("ds_n", GridRef), ("ds_k", GridRef),
    ("ds_rho_cp", GridRef), ("ds_t_remove", GridRef),
    ("cs_mu_a", GridRef), ("cs_mu_s", GridRef), ("cs_k", GridRef), ("cs_rho_cp", GridRef), ("cs_t_remove", GridRef),
    ("flags", _F), ("to_remove", _F), ("plume", _F), ("mu_ext", _F), ("props", _F),
]


class PhaseDesc(Structure):
    _fields_ = _PHASE_FIELDS


class EngineDesc(Structure):
    _fields_ = [
        ("phase", PhaseDesc), ("substep", AblationParams), ("n_substeps", c_int32),
        ("has_plume_transport", c_int32), ("plume", PlumeParams), ("mc", McParams),
        ("T_alt", _F), ("omega", _F), ("plume_alt", _F), ("A", _F), ("L", _F), ("lat_depth", _F),
        ("dt_epoch", c_double), ("voxel_volume", c_double),
    ]


class EpochDiag(Structure):
    _fields_ = [("ledger", c_double * 16), ("epoch", c_double), ("time_s", c_double), ("n_new", c_double),
                ("n_ablated", c_double), ("gap_open", c_double), ("plume_tau", c_double),
                ("plume_peak_mu_a", c_double), ("plume_ablated_sum", c_double), ("t_optical_ms", c_double),
                ("t_thermal_ms", c_double), ("t_epoch_end_ms", c_double), ("n_void", c_double),
                ("void_zlimit", c_double)]


class RecordSpec(Structure):
    _fields_ = [("y", c_int32), ("k_surface", c_int32), ("band_k0", c_int32 * 3), ("band_k1", c_int32 * 3),
                ("gap_k0", c_int32), ("gap_k1", c_int32), ("q_scale", c_float), ("plume_ratio_a", c_float)]


class RecordHead(Structure):
    _fields_ = [("time_s", c_double), ("epoch", c_double), ("plume_tau", c_double), ("n_new", c_double),
                ("n_void", c_double), ("absorbed_weight", c_double), ("peak_T", c_float * 3),
                ("depth_voxels", c_int32)]


TUNE_MC_BLOCKS_PER_SM = 0
TUNE_STENCIL_XC = 1
TUNE_PLUME_XC = 2
TUNE_PLUME_KERNEL = 3
TUNE_STENCIL_CAP = 4
PLUME_KERNEL_DIRECT = 4
PLUME_KERNEL_COMPACT = 6

CONV_FWD_RELU = 0
CONV_FWD_UPADD = 1
CONV_FWD_HEAD = 2
CONV_BWD_RAW = 3
CONV_BWD_MASK = 4
CONV_BWD_UPADD = 5


class ConvCall(Structure):
    _fields_ = [
        ("nx", c_int32), ("ny", c_int32), ("nz", c_int32), ("cin", c_int32), ("cout_total", c_int32),
        ("n_off", c_int32), ("n_slice", c_int32), ("taps", c_int32), ("mode", c_int32),
        ("input", _F), ("wimage", _F), ("bias", _F), ("out", _F), ("out_coarse", _F), ("aux", _F), ("aux2", _F),
        ("head", _F), ("a_noisy", _F), ("mask", _F), ("scale", c_float), ("loss_norm", c_float),
        ("pred", _F), ("target", _F), ("head_grad", _F), ("loss", _F), ("grad_out", _F),
    ]


# name -> (restype, argtypes); every entry point of include/bugdef.h
_SIGNATURES = {
    "bd_abi_version": (c_int, []),
    "bd_last_error": (c_int, [c_char_p, c_size_t]),
    "bd_device_count": (c_int, [POINTER(c_int)]),
    "bd_device_init": (c_int, [c_int]),
    "bd_stream_sync": (c_int, [c_void_p]),
    "bd_mc_pack_props": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
                                 c_float, c_float, c_float, c_int64, c_void_p, c_void_p]),
    "bd_mc_create": (c_int, [POINTER(c_void_p)]),
    "bd_mc_destroy": (c_int, [c_void_p]),
    "bd_mc_trace": (c_int, [c_void_p, POINTER(McParams), c_void_p, c_void_p, c_void_p, c_void_p,
                            c_void_p, c_void_p, c_void_p]),
    "bd_mc_trace_noalloc": (c_int, [POINTER(McParams), c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
                                    c_void_p, c_void_p]),
    "bd_fold_f32_to_f64": (c_int, [c_void_p, c_void_p, c_int64, c_void_p]),
    "bd_thermal_advance": (c_int, [POINTER(ThermalParams), c_void_p, c_void_p, c_int, c_void_p,
                                   c_void_p, c_void_p, c_void_p]),
    "bd_ablation_advance": (c_int, [POINTER(AblationParams), c_void_p, c_void_p, c_int, c_void_p,
                                    c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
    "bd_plume_advance": (c_int, [POINTER(PlumeParams), c_void_p, c_void_p, c_int, c_void_p,
                                 POINTER(c_int), c_void_p]),
    "bd_plume_steps_per_substep": (c_int, [POINTER(PlumeParams), POINTER(c_int), POINTER(c_float)]),
    "bd_pack_flags": (c_int, [c_void_p, c_void_p, c_void_p, c_int64, c_void_p, c_void_p]),
    "bd_engine_create": (c_int, [POINTER(EngineDesc), POINTER(c_void_p)]),
    "bd_engine_destroy": (c_int, [c_void_p]),
    "bd_engine_step_epoch": (c_int, [c_void_p, c_float, c_int, c_void_p]),
    "bd_engine_epoch_end": (c_int, [c_void_p, c_void_p]),
    "bd_engine_epoch_finish": (c_int, [c_void_p, c_void_p]),
    "bd_plume_batch_create": (c_int, [ctypes.POINTER(c_void_p), c_int, ctypes.POINTER(c_void_p)]),
    "bd_plume_batch_run": (c_int, [c_void_p, c_void_p]),
    "bd_plume_batch_destroy": (c_int, [c_void_p]),
    "bd_engine_read_diag": (c_int, [c_void_p, POINTER(EpochDiag), c_void_p]),
    "bd_engine_set_time": (c_int, [c_void_p, c_double, c_int64, c_void_p]),
    "bd_engine_set_mc": (c_int, [c_void_p, POINTER(McParams)]),
    "bd_engine_timing": (c_int, [c_void_p, c_int]),
    "bd_engine_timing_read": (c_int, [c_void_p, POINTER(c_double), POINTER(c_int64)]),
    "bd_engine_set_plume_optics": (c_int, [c_void_p, c_float, c_float, c_float, c_float]),
    "bd_engine_refresh_props": (c_int, [c_void_p, c_void_p]),
    "bd_record_slot_bytes": (c_int64, [c_int, c_int]),
    "bd_engine_record": (c_int, [c_void_p, POINTER(RecordSpec), c_void_p, c_void_p]),
    "bd_tune_set": (c_int, [c_int, c_int]),
    "bd_tune_get": (c_int, [c_int, POINTER(c_int)]),
    "bd_selftest_wait_timeout": (c_int, [c_int, c_int, c_void_p]),
    "bd_conv_plane_rows": (c_int64, [c_int, c_int, c_int]),
    "bd_conv_image_bytes": (c_int64, [c_int, c_int, c_int]),
    "bd_conv_pack_weights": (c_int, [c_int, c_int, c_int, c_int, c_int, c_int, c_void_p, c_void_p, c_void_p]),
    "bd_conv3d": (c_int, [POINTER(ConvCall), c_void_p]),
    "bd_conv3d_wgrad": (c_int, [c_int, c_int, c_int, c_int, c_int, c_int, c_void_p, c_void_p, c_void_p,
                                c_void_p]),
    "bd_unet_param_count": (c_int64, []),
    "bd_unet_create": (c_int, [c_int, c_int, c_int, c_int, POINTER(c_void_p)]),
    "bd_unet_destroy": (c_int, [c_void_p]),
    "bd_unet_set_params": (c_int, [c_void_p, c_void_p, c_void_p]),
    "bd_unet_get_params": (c_int, [c_void_p, c_void_p, c_void_p]),
    "bd_unet_forward": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_float, c_void_p, c_void_p]),
    "bd_unet_forward_backward": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_float, c_float,
                                         c_void_p, c_void_p]),
    "bd_unet_get_grads": (c_int, [c_void_p, c_void_p, c_void_p]),
    "bd_unet_adam": (c_int, [c_void_p, c_float, c_float, c_float, c_float, c_void_p]),
    "bd_unet_read_loss": (c_int, [c_void_p, POINTER(c_double), c_void_p]),
}

_lib = None


class BugdefError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[bd status {code}] {msg}")
        self.code = code


def load(path: str | os.PathLike | None = None) -> ctypes.CDLL:
    """Load libbugdef.so and bind every declared entry point (raises if a symbol is missing)."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    if path is None and os.environ.get("BUGDEF_LIB"):
        path = os.environ["BUGDEF_LIB"]  # another build of the same library (tuning variants)
    p = Path(path) if path is not None else LIB_PATH
    if not p.exists():
        raise RuntimeError(f"libbugdef.so not built ({p}); run `python -m bug_defense_b200.build`")
    lib = ctypes.CDLL(str(p))
    for name, (res, args) in _SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if _lib is None:
        _lib = lib
    return lib


def declared_symbols():
    return list(_SIGNATURES)


def last_error() -> str:
    buf = ctypes.create_string_buffer(512)
    load().bd_last_error(buf, 512)
    return buf.value.decode(errors="replace")


def check(code: int, what: str = "") -> None:
    if code == BD_OK:
        return
    msg = last_error()
    if what:
        msg = f"{what}: {msg}"
    if code == BD_ERR_INVALID_ARG:
        raise ValueError(msg)
    raise BugdefError(code, msg)


def call(name: str, *args):
    check(getattr(load(), name)(*args), name)


def device_count() -> int:
    n = c_int(0)
    check(load().bd_device_count(ctypes.byref(n)))
    return int(n.value)


def ptr(t) -> c_void_p:
    """Device (or host) address of a torch tensor / numpy array, or NULL for None."""
    if t is None:
        return c_void_p(None)
    if hasattr(t, "data_ptr"):
        return c_void_p(t.data_ptr())
    return c_void_p(t.ctypes.data)


def stream_ptr(stream=None) -> c_void_p:
    import torch
    s = stream if stream is not None else torch.cuda.current_stream()
    return c_void_p(s.cuda_stream)
