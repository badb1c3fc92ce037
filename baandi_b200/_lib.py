"""ctypes binding of libbaandi_b200.so (the C ABI of include/baandi_gpu.h).

The library is built in-tree by baandi_b200.build; importing this module never falls
back to a CPU implementation: a missing or unloadable library raises ImportError.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libbaandi_b200.so")

BG_OK = 0
BG_ESHAPE = 1
BG_ENONFINITE = 2
BG_EEPOCH = 3
BG_EDEVICE = 4
BG_ETIMEOUT = 5
BG_EINVAL = 6
BG_ENOMEM = 7
BG_PRECOND_SMOOTH, BG_PRECOND_TPA, BG_PRECOND_RITZ_SHIFT, BG_PRECOND_LEARNED = 0, 1, 2, 3
BG_LEARNED_PARAMS = 4609
BG_PTR_HOST = 0
BG_PTR_DEVICE = 1
BG_PREC_FP64, BG_PREC_FP32, BG_PREC_TENSOR = 0, 1, 2

CODE_NAMES = {
    BG_ESHAPE: "BG_ESHAPE", BG_ENONFINITE: "BG_ENONFINITE", BG_EEPOCH: "BG_EEPOCH",
    BG_EDEVICE: "BG_EDEVICE", BG_ETIMEOUT: "BG_ETIMEOUT", BG_EINVAL: "BG_EINVAL", BG_ENOMEM: "BG_ENOMEM",
}

# Every entry point include/baandi_gpu.h declares, with its ctypes signature.
_p = ctypes.c_void_p
_i32 = ctypes.c_int32
_i64 = ctypes.c_int64
_u64 = ctypes.c_uint64
_dbl = ctypes.c_double
_pp = ctypes.POINTER(ctypes.c_void_p)


class DeviceOpts(ctypes.Structure):
    _fields_ = [("device", _i32), ("reserved", _i32 * 7)]


class BasisDesc(ctypes.Structure):
    _fields_ = [("npw", _i64), ("miller", _p), ("kinetic", _p), ("dims", _i32 * 3), ("gamma", _i32)]


class Projectors(ctypes.Structure):
    _fields_ = [("nproj", _i32), ("table", _p), ("natoms", _i32), ("channels", _p), ("couplings", _p)]


class DavidsonOptions(ctypes.Structure):
    _fields_ = [("bands", _i64), ("threshold", _dbl), ("occupied", _i64), ("first_step", _i32), ("capacity", _i64),
                ("max_iterations", _i32), ("flags", _i32), ("preconditioner", _i32), ("apply_precision", _i32),
                ("reserved", _i32 * 1)]


class DavidsonStats(ctypes.Structure):
    _fields_ = [("iterations", _i32), ("reduced_solves", _i32), ("h_calls", _i64), ("h_columns", _i64),
                ("repairs", _i32), ("contractions", _i32), ("dropped", _i32), ("converged_count", _i32),
                ("fallbacks", _i32), ("tensor_iterations", _i32)]


class LearnedSamples(ctypes.Structure):
    _fields_ = [("n", _i64), ("ncols", _i32), ("feats", _p), ("base", _p), ("a", _p), ("z", _p), ("col", _p),
                ("ecol", _p)]


class MixerProfile(ctypes.Structure):
    _fields_ = [("beta", _dbl), ("history", _i32), ("thomas_fermi", _i32), ("reserved", _i32 * 4)]


class MixerDiagnostics(ctypes.Structure):
    _fields_ = [("iteration", _i32), ("occupancy", _i32), ("inserted_slot", _i32), ("reserved", _i32),
                ("gamma_l2", _dbl), ("gamma_max", _dbl), ("condition", _dbl)]


class SpeciesDesc(ctypes.Structure):
    _fields_ = [("z_valence", _dbl), ("mesh", _i32), ("r", _p), ("rab", _p), ("local", _p), ("nbeta", _i32),
                ("l", _p), ("beta_len", _p), ("beta", _p), ("dij", _p), ("natoms", _i32), ("positions", _p)]


SIGNATURES = {
    "bg_ctx_create": [ctypes.POINTER(DeviceOpts), _pp],
    "bg_ctx_destroy": [_p],
    "bg_last_error": [_p, ctypes.c_char_p, ctypes.c_size_t],
    "bg_op_create_complex": [_p, ctypes.POINTER(BasisDesc), ctypes.POINTER(Projectors), _i64, _pp],
    "bg_op_create_gamma_real": [_p, ctypes.POINTER(BasisDesc), ctypes.POINTER(Projectors), _i64, _pp],
    "bg_op_destroy": [_p],
    "bg_op_set_potential": [_p, _p, _u64],
    "bg_op_apply_block": [_p, _p, _p, _i64, _i64, _i32, _i32],
    "bg_op_diagonal": [_p, _p],
    "bg_op_rows": [_p, ctypes.POINTER(_i64)],
    "bg_op_capacity": [_p, ctypes.POINTER(_i64)],
    "bg_op_stream": [_p, _pp],
    "bg_op_set_stream": [_p, _p],
    "bg_op_sync": [_p],
    "bg_op_launches": [_p, ctypes.POINTER(_i64)],
    "bg_op_profile": [_p, _i32],
    "bg_op_stage_times": [_p, _p],
    "bg_op_set_potential_ptr": [_p, _p, _u64, _i32],
    "bg_op_add_local_change": [_p, _p, _p, _p, _i64, _i64, _i32],
    "bg_op_band_density_sum": [_p, _p, _i64, _i64, _p, _dbl, _p, _i32, _i32],
    "bg_fields_create": [_p, _p, _p, _pp],
    "bg_fields_destroy": [_p],
    "bg_fields_set_stream": [_p, _p],
    "bg_fields_volume": [_p, ctypes.POINTER(_dbl)],
    "bg_fields_lda_hartree": [_p, _p, _p, _p, _p, _i32],
    "bg_fields_set_sphere": [_p, _i64, _p],
    "bg_fields_sphere_forward": [_p, _p, _p, _i32],
    "bg_fields_sphere_inverse": [_p, _p, _p, _i32],
    "bg_mixer_create": [_p, ctypes.POINTER(MixerProfile), _i64, _p, _p, _dbl, _dbl, _dbl, _pp],
    "bg_mixer_destroy": [_p],
    "bg_mixer_set_stream": [_p, _p],
    "bg_mixer_update": [_p, _p, _p, _p, _i32, ctypes.POINTER(MixerDiagnostics)],
    "bg_mixer_gamma": [_p, _p, ctypes.POINTER(_i32)],
    "bg_mixer_reduced_residual": [_p, _p, _i32],
    "bg_mixer_metric": [_p, _p, _p, _p, _i32],
    "bg_kset_create": [_p, _i32, _p, _pp],
    "bg_kset_destroy": [_p],
    "bg_kset_apply": [_p, _p, _p, _p, _i32, _i32],
    "bg_kset_set_potential_ptr": [_p, _p, _u64, _i32],
    "bg_kset_band_density_sum": [_p, _p, _i64, _p, ctypes.c_double, _p, _i32, _i32],
    "bg_kset_sync": [_p],
    "bg_kset_stream": [_p, _pp],
    "bg_kset_set_stream": [_p, _p],
    "bg_kset_launches": [_p, ctypes.POINTER(_i64)],
    "bg_kset_profile": [_p, _i32],
    "bg_kset_stage_times": [_p, _p],
    "bg_davidson_solve": [_p, _p, _p, ctypes.POINTER(DavidsonOptions), _p, _p, _p, ctypes.POINTER(DavidsonStats)],
    "bg_kset_davidson_solve": [_p, _p, _p, ctypes.POINTER(DavidsonOptions), _i32, _p, _p, _p, _p],
    "bg_autotune_report": [ctypes.c_char_p, _i64],
    "bg_kset_davidson_solve_hx": [_p, _p, _p, _p, ctypes.POINTER(DavidsonOptions), _p, _p, _p, _p, _p],
    "bg_op_create_dense": [_p, _i64, _p, _i32, _i64, _pp],
    "bg_reduced_eigh": [_p, _i64, _i32, _p, _p, _p, _p, _p],
    "bg_zgemm_bf16x3": [_p, _i32, _i64, _i64, _i64, _p, _i64, _p, _i64, _p, _i64, _i32, _p],
    "bg_learned_set": [_p, _p],
    "bg_learned_clear": [_p],
    "bg_learned_samples_build": [_p, _i64, _i32, _i32, _p, _p, _p, _p, _p, _i32, _i64,
                                 ctypes.POINTER(LearnedSamples), _p],
    "bg_learned_loss_grad": [_p, ctypes.POINTER(LearnedSamples), _p, _p, _p, _p, _p],
    "bg_learned_adam": [_p, _p, _p, _p, _p, _p, _i32, ctypes.c_float, _p],
    "bg_local_apply_noalloc": [_p, _i64, _p, _p, _p, _p, _p, _i64, _p],
    "bg_setup_volume": [_p, ctypes.POINTER(_dbl)],
    "bg_setup_basis": [_p, _dbl, _p, _i64, ctypes.POINTER(_i64), _p, _p, _p],
    "bg_setup_grid": [_p, _dbl, _p, _p],
    "bg_setup_half_sphere": [_p, _i64, _p, _p],
    "bg_setup_projector_count": [_i32, ctypes.POINTER(SpeciesDesc), ctypes.POINTER(_i32), ctypes.POINTER(_i32)],
    "bg_setup_projectors": [_dbl, _i64, _p, _p, _i32, ctypes.POINTER(SpeciesDesc), _p, _p, _p],
    "bg_setup_local_form_factor": [ctypes.POINTER(SpeciesDesc), _dbl, _i64, _p, _p],
    "bg_setup_ewald": [_p, _i32, _p, _p, ctypes.POINTER(_dbl)],
    "bg_setup_atomic_charge": [_i64, _p, _p, _p, _dbl, _i64, _p, _p],
}

_lib = None


def load():
    """Load the in-tree library (ImportError if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -m baandi_b200.build` "
                          "(nvcc, sm_100a); there is no CPU fallback")
    lib = ctypes.CDLL(LIB_PATH)
    for name, args in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = ctypes.c_int
    _lib = lib
    return lib


class BaandiError(RuntimeError):
    """A non-zero status of the C ABI; `code` is the BG_E* value."""

    def __init__(self, code, message):
        super().__init__(f"{CODE_NAMES.get(code, code)}: {message}")
        self.code = code


def last_error(ctx=None) -> str:
    buf = ctypes.create_string_buffer(512)
    load().bg_last_error(ctx, buf, len(buf))
    return buf.value.decode(errors="replace")


def autotune_report() -> list:
    """The autotuner's decisions in this process (bg_autotune_report), parsed."""
    import json
    need = load().bg_autotune_report(None, 0)
    buf = ctypes.create_string_buffer(max(int(need), 3))
    load().bg_autotune_report(buf, len(buf))
    return json.loads(buf.value.decode())


def check(rc, ctx=None):
    if rc != BG_OK:
        raise BaandiError(rc, last_error(ctx))
