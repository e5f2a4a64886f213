"""Loads libvortexlab_b200.so and declares the C ABI of include/vortexlab.h for ctypes.

There is no fallback: if the shared library is missing this module raises ImportError, and every
constructor of a device-resident sim raises VortexError when no CUDA device is present.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
# VORTEXLAB_B200_LIB selects another build of the same library (for example a profiling variant).
LIB_PATH = os.environ.get("VORTEXLAB_B200_LIB") or os.path.join(HERE, "libvortexlab_b200.so")

VL_OK, VL_EINVAL, VL_ECUDA, VL_EDIVERGED, VL_ENOMEM, VL_EUNSUPPORTED = 0, -1, -2, -3, -4, -5
VL_REC = 10
VL_MAX_FGROUPS = 4


class VortexError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{msg} (status {code})")
        self.code = code


class vl_velocity(C.Structure):
    _fields_ = [("kind", C.c_int), ("p", C.c_double * 4)]


class vl_wall(C.Structure):
    _fields_ = [("velocity", vl_velocity), ("vgroup", C.c_int), ("fgroup", C.c_int), ("shape", C.c_void_p)]


class vl_channel_spec(C.Structure):
    _fields_ = [
        ("nx", C.c_size_t), ("ny", C.c_size_t), ("inflow", C.c_int), ("u", C.c_double), ("nu", C.c_double),
        ("collision", C.c_int), ("magic", C.c_double), ("body", C.c_void_p), ("ramp_steps", C.c_uint64),
        ("has_kick", C.c_int), ("kick_cx", C.c_double), ("kick_cy", C.c_double), ("kick_omega", C.c_double),
        ("kick_start", C.c_uint64), ("kick_duration", C.c_uint64),
    ]


def _declare(L):
    d, i, u64, sz, vp, f = C.c_double, C.c_int, C.c_uint64, C.c_size_t, C.c_void_p, C.c_float
    P = C.POINTER
    sig = {
        "vl_last_error": (C.c_char_p, []),
        "vl_last_status": (i, []),
        "vl_abi_version": (i, []),
        "vl_device_count": (i, []),
        "vl_set_device": (i, [i]),
        "vl_pinned_alloc": (vp, [sz]),
        "vl_pinned_free": (None, [vp]),
        "vl_shape_circle": (vp, [d, d, d]),
        "vl_shape_polygon": (vp, [P(d), sz]),
        "vl_shape_rounded_square": (vp, [d, d, d, d]),
        "vl_shape_rotated": (vp, [vp, d, d, d]),
        "vl_shape_translated": (vp, [vp, d, d]),
        "vl_shape_section": (vp, [i, d, d, d, d, d]),
        "vl_shape_bitmap": (vp, [sz, sz, P(f), d, d, d]),
        "vl_shape_outside_band": (vp, [d, d]),
        "vl_shape_ellipse": (vp, [d, d, d, d]),
        "vl_shape_star": (vp, [d, d, P(d), sz, d]),
        "vl_shape_disks": (vp, [P(d), sz]),
        "vl_shape_free": (None, [vp]),
        "vl_shape_inside": (i, [vp, d, d]),
        "vl_cut_fraction": (d, [vp, d, d, d, d]),
        "vl_bounding_box": (i, [vp, d, d, P(d)]),
        "vl_builder_new": (vp, [sz, sz]),
        "vl_builder_free": (None, [vp]),
        "vl_builder_set_periodic": (i, [vp, i, i]),
        "vl_builder_set_tau": (i, [vp, d]),
        "vl_builder_set_collision": (i, [vp, i, d]),
        "vl_builder_set_accel": (i, [vp, d, d]),
        "vl_builder_add_wall": (i, [vp, P(vl_wall)]),
        "vl_builder_add_static_wall": (i, [vp]),
        "vl_builder_add_pressure": (i, [vp, d]),
        "vl_builder_add_radiating": (i, [vp, d]),
        "vl_builder_fill_rect": (i, [vp, sz, sz, sz, sz, i]),
        "vl_builder_fill_shape": (i, [vp, i]),
        "vl_builder_stage_split": (i, [vp, P(i), P(i), P(i), P(i)]),
        "vl_builder_link_table": (i, [vp, P(sz), P(sz), P(sz), P(C.c_uint8), P(C.c_int32), P(C.c_int32), P(d),
                                      P(C.c_int32)]),
        "vl_builder_build": (vp, [vp, i]),
        "vl_sim_free": (None, [vp]),
        "vl_sim_info": (i, [vp, P(sz), P(sz), P(sz), P(sz), P(sz), P(i), P(i)]),
        "vl_sim_init": (i, [vp, P(d), P(d), P(d), d, d, d]),
        "vl_sim_step": (i, [vp, u64]),
        "vl_sim_synchronize": (i, [vp]),
        "vl_sim_set_vscale": (i, [vp, i, d]),
        "vl_sim_get_vscale": (i, [vp, P(d)]),
        "vl_sim_set_outflow_target": (i, [vp, i, d]),
        "vl_sim_outlet_density_offset": (i, [vp, P(d)]),
        "vl_sim_t": (i, [vp, P(u64)]),
        "vl_sim_status": (i, [vp, P(i), P(u64)]),
        "vl_sim_force": (i, [vp, P(d)]),
        "vl_sim_download": (i, [vp, P(d)]),
        "vl_sim_upload": (i, [vp, P(d)]),
        "vl_sim_flags": (i, [vp, P(C.c_uint8)]),
        "vl_sim_macros_field": (i, [vp, P(d), P(d), P(d)]),
        "vl_sim_macros": (i, [vp, sz, sz, P(d)]),
        "vl_sim_total_mass": (i, [vp, P(d)]),
        "vl_sim_total_momentum": (i, [vp, P(d)]),
        "vl_sim_max_speed": (i, [vp, P(d)]),
        "vl_sim_vorticity": (i, [vp, P(f)]),
        "vl_sim_probe_density": (i, [vp, d, d, P(d)]),
        "vl_sim_probe_density_at_wall": (i, [vp, d, d, d, d, P(d)]),
        "vl_sim_state_hash": (i, [vp, P(u64)]),
        "vl_sim_record": (i, [vp, u64]),
        "vl_sim_history": (i, [vp, P(d), P(u64)]),
        "vl_sim_set_dp_probe": (i, [vp, d, d, d, d]),
        "vl_sim_last_step_ms": (i, [vp, P(f)]),
        "vl_sim_step_profiled": (i, [vp, u64, P(d), P(d), P(d)]),
        "vl_sim_set_prefetch_rows": (i, [vp, i]),
        "vl_sim_set_bulk_copies": (i, [vp, i]),
        "vl_sim_set_cells_per_thread": (i, [vp, i]),
        "vl_sim_set_schedule": (i, [vp, i]),
        "vl_sim_get_schedule": (i, [vp]),
        "vl_sim_autotune": (i, [vp, i, P(d)]),
        "vl_sim_launch_count": (i, [vp, P(u64)]),
        "vl_reduce_f64_static": (i, [vp, sz, vp, sz, d, d, vp, vp]),
        "vl_channel_new": (vp, [P(vl_channel_spec), i]),
        "vl_channel_free": (None, [vp]),
        "vl_channel_sim": (vp, [vp]),
        "vl_channel_set_absorbing": (i, [vp, i]),
        "vl_channel_step": (i, [vp, u64]),
        "vl_channel_coefficients": (i, [vp, d, P(d), P(d)]),
        "vl_channel_u_ref": (d, [vp]),
        "vl_batch_new": (vp, [i]),
        "vl_batch_free": (None, [vp]),
        "vl_batch_add_channel": (i, [vp, P(vl_channel_spec), u64]),
        "vl_batch_build": (i, [vp]),
        "vl_batch_size": (i, [vp]),
        "vl_batch_tunnel_info": (i, [vp, i, P(sz), P(sz), P(sz), P(u64)]),
        "vl_batch_run_async": (i, [vp, u64]),
        "vl_batch_wait": (i, [vp]),
        "vl_batch_history_copy": (i, [vp, i, P(i), P(u64), P(u64), P(d)]),
        "vl_batch_autotune_layouts": (i, [vp, i, P(d), i]),
        "vl_batch_hold": (i, [vp, i]),
        "vl_batch_start": (i, [vp, i, P(u64)]),
        "vl_batch_set_prefetch_tiles": (i, [vp, i]),
        "vl_batch_set_cells_per_thread": (i, [vp, i]),
        "vl_batch_set_tile": (i, [vp, i, i]),
        "vl_batch_get_tile": (i, [vp, P(i), P(i)]),
        "vl_batch_set_schedule": (i, [vp, i]),
        "vl_batch_autotune": (i, [vp, i, P(d)]),
        "vl_batch_run": (i, [vp, u64]),
        "vl_batch_last_run_ms": (i, [vp, P(f)]),
        "vl_batch_global_step": (i, [vp, P(u64)]),
        "vl_batch_launch_count": (i, [vp, P(u64)]),
        "vl_batch_status": (i, [vp, i, P(u64), P(i), P(d)]),
        "vl_batch_force_history_range": (i, [vp, i, u64, u64, P(d), P(u64)]),
        "vl_batch_force_history": (i, [vp, i, P(d), P(u64)]),
        "vl_batch_download": (i, [vp, i, P(d)]),
        "vl_batch_init": (i, [vp, i, P(d), P(d), P(d)]),
        "vl_batch_init_grid": (i, [vp, i, vp, i, i, i, d, d, d, d, d]),
        "vl_batch_set_steps": (i, [vp, i, C.c_uint64]),
        "vl_batch_macros_field": (i, [vp, i, P(d), P(d), P(d)]),
        "vl_batch_flags": (i, [vp, i, P(C.c_uint8)]),
        "vl_batch_state_hash": (i, [vp, i, P(u64)]),
        "vl_nn_gemm_bf16": (i, [vp, i, vp, i, i, i, i, vp, i, P(f), i, i, P(i), vp]),
        "vl_nn_im2col": (i, [vp, i, i, i, i, i, i, vp, vp]),
        "vl_nn_flip_weights": (i, [vp, i, i, i, i, vp, vp]),
        "vl_nn_col2im": (i, [vp, i, i, i, i, i, i, vp, i, vp]),
        "vl_nn_act_bwd": (i, [vp, vp, i, i, i, vp, vp, vp, vp]),
        "vl_nn_bias_grad": (i, [vp, i, i, vp, vp]),
        "vl_nn_transpose_bf16": (i, [vp, i, i, vp, vp]),
        "vl_nn_up2": (i, [vp, i, i, i, i, vp, i, i, vp]),
        "vl_nn_up2_bwd": (i, [vp, i, i, i, i, i, i, vp, i, vp]),
        "vl_nn_copy_channels": (i, [vp, C.c_longlong, i, vp, i, i, vp]),
        "vl_nn_slice_channels": (i, [vp, C.c_longlong, i, i, i, vp, i, vp]),
        "vl_nn_mse": (i, [vp, vp, vp, C.c_longlong, i, i, d, vp, vp, i, vp]),
        "vl_nn_adam": (i, [vp, vp, vp, vp, C.c_longlong, f, f, f, f, i, vp, vp]),
        "vl_nn_f32_to_bf16": (i, [vp, C.c_longlong, vp, vp]),
        "vl_fft": (i, [P(d), P(d), sz]),
        "vl_mean": (d, [P(d), sz]),
        "vl_rms": (d, [P(d), sz]),
        "vl_dominant_frequency": (i, [P(d), sz, d, P(d), P(d)]),
        "vl_peaks": (sz, [P(d), sz, P(d), P(d), sz]),
        "vl_crossing_frequency": (i, [P(d), sz, d, P(d)]),
        "vl_sample_at": (d, [P(d), sz, d]),
        "vl_ramp": (d, [u64, u64]),
        "vl_tau_for": (d, [d]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    return sig


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `python -m vortexlab_b200._build` "
            "(there is no CPU fallback for the step kernels)")
    L = C.CDLL(LIB_PATH)
    _declare(L)
    return L


lib = _load()
DECLARED = sorted(_declare(lib).keys())


def last_error() -> str:
    return lib.vl_last_error().decode()


def check(rc):
    if rc < 0:
        raise VortexError(rc, last_error())
    return rc


def nonnull(ptr):
    if not ptr:
        raise VortexError(lib.vl_last_status(), last_error())
    return ptr
