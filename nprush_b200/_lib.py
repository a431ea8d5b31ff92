"""ctypes binding of libnprush_cuda.so (the C ABI declared in include/nprush.h).

The product path has no CPU fallback: if the shared library is missing or no
sm_100 GPU is present, loading fails loudly with NpsError.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

HERE = Path(__file__).resolve().parent
LIB_PATH = Path(os.environ.get("NPRUSH_LIB", HERE / "libnprush_cuda.so"))

NPS_OK = 0
NPS_MEM_HOST, NPS_MEM_DEVICE, NPS_MEM_DEVICE_BORROW = 0, 1, 2
ERR_NAMES = {-1: "NPS_ERR_INVALID", -2: "NPS_ERR_CUDA", -3: "NPS_ERR_NOMEM", -4: "NPS_ERR_CAPACITY",
             -5: "NPS_ERR_TIMEOUT", -6: "NPS_ERR_STATE"}


class NpsError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERR_NAMES.get(code, code)}: {msg}")
        self.code = code


class nps_stats(ctypes.Structure):
    _fields_ = [("pairs", ctypes.c_uint64), ("pairs_capped", ctypes.c_uint64), ("max_tile_len", ctypes.c_uint32),
                ("adc_clones", ctypes.c_uint32), ("step_count", ctypes.c_uint32), ("reserved", ctypes.c_uint32 * 3)]


P = ctypes.c_void_p
U32 = ctypes.c_uint32
I32 = ctypes.c_int
F32 = ctypes.c_float
PP = ctypes.POINTER(ctypes.c_void_p)

# name -> argtypes (all return int status unless listed in _RET)
SIGNATURES = {
    "nps_create": [I32, PP],
    "nps_destroy": [P],
    "nps_sync": [P],
    "nps_set_stream": [P, P],
    "nps_sort_pairs": [P, P, P, U32, I32, U32, U32],
    "nps_splat_opt_create": [P, U32, PP],
    "nps_splat_opt_destroy": [P],
    "nps_splat_opt_write_params": [P, P, U32, U32, I32],
    "nps_splat_opt_write_state": [P, P, P, P, F32, P, I32],
    "nps_splat_opt_read_state": [P, P, P, P, P, P, P],
    "nps_splat_opt_write_vp": [P, P, P, U32, I32],
    "nps_splat_opt_set_target": [P, P, P, U32, U32, U32, I32],
    "nps_splat_opt_dispatch": [P],
    "nps_splat_opt_backward": [P, P],
    "nps_splat_opt_step": [P],
    "nps_splat_opt_adc": [P],
    "nps_splat_opt_render": [P, P, U32, U32, P, P],
    "nps_splat_opt_render_load": [P, P, U32, U32, P, P],
    "nps_splat_opt_buffers": [P, PP, PP, PP, PP, PP],
    "nps_splat_opt_stats": [P, ctypes.POINTER(nps_stats)],
    "nps_splat_opt_set_step_count": [P, U32],
    "nps_splat_adc_noalloc": [P, P, P, P, U32, F32, P, P],
    "nps_bezier_opt_create": [P, U32, PP],
    "nps_bezier_opt_destroy": [P],
    "nps_bezier_opt_write_params": [P, P, U32, U32, I32],
    "nps_bezier_opt_write_state": [P, P, P, P, F32, P, P, P, I32],
    "nps_bezier_opt_read_state": [P, P, P, P, P, P, P, P, P],
    "nps_bezier_opt_write_vp": [P, P, P, U32],
    "nps_bezier_opt_write_mode": [P, F32],
    "nps_bezier_opt_write_bg_penalty": [P, F32],
    "nps_bezier_opt_write_max_width": [P, F32],
    "nps_bezier_opt_write_kill_thresholds": [P, F32, F32],
    "nps_bezier_opt_set_adc_period": [P, U32],
    "nps_bezier_opt_write_no_kill": [P, I32],
    "nps_bezier_opt_set_target": [P, P, P, P, P, P, U32, U32, U32, I32],
    "nps_bezier_opt_dispatch": [P],
    "nps_bezier_opt_backward": [P, P],
    "nps_bezier_opt_step": [P],
    "nps_bezier_opt_adc": [P],
    "nps_bezier_opt_render": [P, P, U32, U32, P, P, U32, U32, P],
    "nps_bezier_opt_buffers": [P, PP, PP, PP, PP, PP, PP, PP],
    "nps_bezier_opt_stats": [P, ctypes.POINTER(nps_stats)],
    "nps_bezier_opt_set_step_count": [P, U32],
    "nps_gs_create": [P, U32, U32, PP],
    "nps_gs_destroy": [P],
    "nps_gs_write_params": [P, P, U32, U32, I32],
    "nps_gs_set_count": [P, U32],
    "nps_gs_write_state": [P, P, P, U32, I32],
    "nps_gs_read_state": [P, P, P, P, P, P, P],
    "nps_gs_set_lr": [P, P],
    "nps_gs_set_background": [P, F32, F32, F32],
    "nps_gs_set_targets": [P, P, U32, U32, U32, I32],
    "nps_gs_set_views": [P, P, P, P, U32],
    "nps_gs_set_image_size": [P, U32, U32],
    "nps_gs_forward": [P, P],
    "nps_gs_loss": [P, P],
    "nps_gs_set_loss": [P, I32, F32],
    "nps_gs_backward": [P, P],
    "nps_gs_backward_host": [P, P],
    "nps_gs_adam": [P],
    "nps_gs_train_step": [P, P],
    "nps_gs_set_graph": [P, I32],
    "nps_gs_read_image": [P, P, P],
    "nps_gs_adc": [P, F32, F32, F32, P],
    "nps_gs_set_accumulate": [P, I32, U32],
    "nps_gs_save": [P, ctypes.c_char_p],
    "nps_gs_load": [P, ctypes.c_char_p],
    "nps_gs_count": [P, P],
    "nps_gs_write_adc_stats": [P, P, P, I32],
    "nps_gs_psnr": [P, P],
    "nps_gs_buffers": [P, PP, PP, PP, PP, PP, PP],
    "nps_gs_stats": [P, ctypes.POINTER(nps_stats)],
    "nps_gs_set_timing": [P, I32],
    "nps_gs_stage_times": [P, P, P, U32, I32],
    "nps_gs_assign_ids": [P, U32],
    "nps_gs_set_policy_margin": [P, F32],
    "nps_gs_upload_targets": [P, P, P, U32, U32, U32],
    "nps_gs_read_loss": [P, P],
    "nps_gs_adc_buffers": [P, PP, PP],
    "nps_gs_set_deterministic": [P, I32],
    "nps_gs_set_variant": [P, I32, I32, I32, I32],
    "nps_gs_set_raster": [P, I32, I32, I32, I32, I32, I32],
    "nps_gs_set_tile": [P, U32],
    "nps_gs_get_raster": [P, P],
    "nps_gs_autotune_raster": [P, ctypes.c_char_p, P, P],
    "nps_splat_opt_set_wait_guard": [P, U32, U32],
    "nps_gs_set_sort_guard": [P, U32, U32],
    "nps_gs_autotune": [P, ctypes.c_char_p, P, P],
    "nps_gs_adc_features": [P, F32, F32, F32, F32, P, P, P],
    "nps_gs_adc_policy": [P, P, F32, F32, F32, F32, P, P],
    "nps_blur": [P, P, P, U32, U32, I32, I32, I32, U32, F32, I32],
    "nps_depth_aware_blur": [P, P, P, P, U32, U32, I32, I32],
    "nps_splat_edge": [P, P, P, U32, U32, F32, F32, I32],
    "nps_bvh_build": [P, U32, P, U32, P, P, P],
    "nps_pt_create": [P, P, U32, P, U32, PP],
    "nps_pt_destroy": [P],
    "nps_pt_bvh_size": [P, P, P],
    "nps_pt_read_bvh": [P, P, P],
    "nps_pt_set_env": [P, P, U32, U32],
    "nps_pt_trace": [P, P, U32, U32, P, U32, U32],
    "nps_pt_overflows": [P, P],
    "nps_pt_resolve": [P, P, P, U32, U32, I32],
    "nps_mesh_create": [P, P, U32, P, U32, PP],
    "nps_mesh_destroy": [P],
    "nps_mesh_set_matcap": [P, P, U32, U32],
    "nps_mesh_set_env": [P, P, U32, U32],
    "nps_mesh_set_pbr": [P, U32, P, U32, U32, I32, P, U32, U32],
    "nps_mesh_render": [P, P, P, P, U32, U32, I32, I32],
    "nps_mlp_num_params": [],
    "nps_mlp_create": [P, PP],
    "nps_mlp_destroy": [P],
    "nps_mlp_init": [P, ctypes.c_uint64],
    "nps_mlp_set_params": [P, P],
    "nps_mlp_get_params": [P, P],
    "nps_mlp_forward": [P, P, U32, P],
    "nps_mlp_grads": [P, P, P, U32, P, P, P],
    "nps_mlp_train": [P, P, P, U32, P, U32, U32, F32, ctypes.c_uint64, P, P],
}
_RET = {"nps_last_error": ctypes.c_char_p, "nps_version": ctypes.c_char_p}

_lib = None


def load():
    """Loads the shared library (raises NpsError if it is missing)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise NpsError(-6, f"{LIB_PATH} not built: run `python -m nprush_b200.build`")
    lib = ctypes.CDLL(str(LIB_PATH))
    for name, argt in SIGNATURES.items():
        fn = getattr(lib, name, None)
        if fn is None:
            continue  # symbol presence is checked by the tests against include/nprush.h
        fn.argtypes = argt
        fn.restype = ctypes.c_int
    for name, rt in _RET.items():
        getattr(lib, name).restype = rt
        getattr(lib, name).argtypes = []
    _lib = lib
    return lib


def check(rc: int):
    if rc != NPS_OK:
        msg = load().nps_last_error()
        raise NpsError(rc, msg.decode() if msg else "")


def call(name: str, *args):
    check(getattr(load(), name)(*args))


_contexts: dict = {}


def context(device: int = 0) -> int:
    """Shared nps_ctx for a device (one per process per device)."""
    if device not in _contexts:
        h = ctypes.c_void_p()
        call("nps_create", device, ctypes.byref(h))
        _contexts[device] = h.value
    return _contexts[device]
