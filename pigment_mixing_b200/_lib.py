"""ctypes binding of the in-tree CUDA library (libpigment_mpm.so, C ABI in include/pigment_mpm.h).

There is no CPU fallback: if the library is missing or no sm_100 GPU is present, calls fail
with an exception.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libpigment_mpm.so")
_lib = None

PM_OK = 0
STATUS = {0: "PM_OK", 1: "PM_ERR_INVALID", 2: "PM_ERR_STATE", 3: "PM_ERR_CUDA", 4: "PM_ERR_IO",
          5: "PM_ERR_UNSUPPORTED", 6: "PM_ERR_CAPACITY"}

# Exported symbols with their ctypes signatures (argument types after the status return).
_vp, _dp, _fp, _up = C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_float), C.POINTER(C.c_uint32)
_u8p = C.POINTER(C.c_uint8)
SIGNATURES = {
    "pm_create": [C.c_int, C.POINTER(C.c_void_p)],
    "pm_destroy": [_vp],
    "pm_trim_memory": [C.c_int, C.c_uint64],
    "pm_initialize_basic": [_vp, C.c_char_p],
    "pm_set_param": [_vp, C.c_char_p, C.c_double],
    "pm_get_param": [_vp, C.c_char_p, _dp],
    "pm_set_param3": [_vp, C.c_char_p, _dp],
    "pm_load_pigment_config": [_vp, C.c_char_p],
    "pm_load_sim_config": [_vp, C.c_char_p],
    "pm_set_particles": [_vp, C.c_uint32, _fp, _fp, _fp],
    "pm_get_particles": [_vp, _fp, _fp, _fp, _fp, _u8p, _fp, _fp, _fp],
    "pm_get_particles_async": [_vp, _fp, _fp, _fp, _fp, _u8p],
    "pm_wait_particles": [_vp],
    "pm_add_plate": [_vp, C.c_double, C.c_int, C.c_int] + [C.c_double] * 8,
    "pm_add_spatula": [_vp, C.c_int, C.c_double, _fp, C.c_uint32],
    "pm_add_spatula_file": [_vp, C.c_int, C.c_double, C.c_char_p],
    "pm_add_box_knife": [_vp, C.c_int, C.c_double, _dp, _dp, C.c_uint32, C.c_double, _dp],
    "pm_add_ground": [_vp, C.c_int, C.c_double, C.c_double],
    "pm_add_curve": [_vp, C.c_int, C.c_double],
    "pm_setup_scene": [_vp, C.c_float, C.c_char_p, C.c_char_p, C.c_char_p],
    "pm_setup_scene_blobs": [_vp, C.c_float, _fp, _fp, C.c_uint32, C.c_char_p, C.c_char_p, C.c_char_p],
    "pm_prepare": [_vp],
    "pm_step": [_vp],
    "pm_advance": [_vp, C.c_uint32, _up],
    "pm_simulate": [_vp, C.c_uint32, _up],
    "pm_frame_finished": [_vp, C.POINTER(C.c_int)],
    "pm_is_finished": [_vp, C.POINTER(C.c_int)],
    "pm_get_grid_boundaries": [_vp, _dp, _dp],
    "pm_get_knife": [_vp, C.POINTER(C.c_int), _dp, _dp],
    "pm_get_error_flags": [_vp, _up, C.c_int],
    "pm_get_stats": [_vp, _dp, _dp, _dp, _up],
    "pm_get_grid": [_vp, _dp, _up, _fp, _fp, _fp, _fp, _fp, _fp],
    "pm_set_return_map": [_vp, C.c_int],
    "pm_get_stream": [_vp, C.POINTER(C.c_void_p)],
    "pm_profile_steps": [_vp, C.c_uint32, _fp, C.c_uint32],
    "pm_set_surrogate": [_vp, _fp],
    "pm_enable_sample_log": [_vp, C.c_uint32],
    "pm_get_samples": [_vp, _fp, _fp, C.c_uint32, _up],
    "pm_get_return_map_stats": [_vp, _up],
    "pm_mlp_train": [_fp, _fp, C.c_uint32, C.c_uint32, C.c_uint32, C.c_float, C.c_uint64, C.c_int, _fp, _fp, _up],
    "pm_mlp_loss_grad": [_fp, _fp, _fp, C.c_uint32, _fp, _fp],
    "pm_mlp_infer": [_fp, _fp, C.c_uint32, _fp],
    "pm_p2g_noalloc": [_vp] * 5 + [C.c_uint32, C.c_double, C.c_double, _dp, C.POINTER(C.c_int32)] + [_vp] * 5 + [_up],
    "pm_save_particle_data": [_vp, C.c_char_p, C.c_char_p],
    "pm_save_grid_data": [_vp, C.c_char_p, C.c_char_p],
    "pm_save_info": [_vp, C.c_char_p],
    "pm_save_checkpoint": [_vp, C.c_char_p],
    "pm_load_checkpoint": [_vp, C.c_char_p],
    "pm_splat_pigments": [_vp, _vp, C.c_int, C.c_float, C.c_float, _vp, _up, _dp, _dp],
    "pm_svd3_batch": [C.c_int, _vp, C.c_uint32, _vp, _vp, _vp],
    "pm_density_grid": [_vp, C.c_float, C.c_float, C.c_float, C.c_int, C.c_int, _vp, _vp, _vp, _vp, _vp, _vp, _up,
                        _dp, _dp, _up],
    "pm_anisotropy": [_vp, C.c_float, C.c_float, C.c_int, C.c_int, C.c_int, C.c_float, C.c_int, _vp, _vp, _vp, _vp,
                      _up],
    "pm_sample_latent_cylinder": [_vp, C.c_double, C.c_double, C.c_double, _dp, _up],
    "pm_sample_particles": [C.c_int, C.c_double, C.c_double, C.c_double, C.c_double, C.c_double, C.c_int, C.c_uint32,
                            C.c_uint32, C.c_uint32, _fp, C.c_uint32, _up, _dp, _dp],
    "pm_batch_create": [C.POINTER(C.c_void_p), C.c_uint32, C.POINTER(C.c_void_p)],
    "pm_batch_destroy": [_vp],
    "pm_batch_step": [_vp, C.c_uint32],
    "pm_batch_get_tuning": [_vp, _vp],
    "pm_batch_set_tuning": [_vp, _vp],
    "pm_batch_autotune": [_vp, C.c_uint32, _vp, _fp],
    "pm_batch_get_stream": [_vp, C.POINTER(C.c_void_p)],
    "pm_batch_profile": [_vp, C.c_uint32, _fp, C.c_uint32],
}


class BatchTuning(C.Structure):
    """pm_batch_tuning (include/pigment_mpm.h)."""
    _fields_ = [(n, C.c_int32) for n in ("flat_threads", "part_ctas_per_sm", "node_ctas_per_sm", "p2g_ctas_per_sm",
                                         "g2p_ctas_per_sm", "def_ctas_per_sm", "sur_ctas_per_sm", "chunk_rounds")]

    def as_dict(self) -> dict:
        return {n: int(getattr(self, n)) for n, _ in self._fields_}


class PMError(RuntimeError):
    """A pm_* call returned a non-zero status."""

    def __init__(self, fn: str, status: int, msg: str):
        super().__init__(f"{fn} -> {STATUS.get(status, status)}: {msg}")
        self.status = status


def lib() -> C.CDLL:
    """Load libpigment_mpm.so (fails loudly if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -m pigment_mixing_b200.build`")
    L = C.CDLL(LIB_PATH)
    for name, args in SIGNATURES.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = C.c_int
    L.pm_last_error_message.restype = C.c_char_p
    L.pm_last_error_message.argtypes = []
    L.pm_kernel_name.restype = C.c_char_p
    L.pm_kernel_name.argtypes = [C.c_void_p, C.c_int]
    L.pm_batch_kernel_name.restype = C.c_char_p
    L.pm_batch_kernel_name.argtypes = [C.c_void_p, C.c_int]
    L.pm_batch_kernels_per_round.restype = C.c_int32
    L.pm_batch_kernels_per_round.argtypes = [C.c_void_p]
    _lib = L
    return L


def call(name: str, *args) -> None:
    """Call pm_<name>, raising PMError on a non-zero status."""
    L = lib()
    rc = getattr(L, name)(*args)
    if rc != PM_OK:
        raise PMError(name, rc, (L.pm_last_error_message() or b"").decode())
