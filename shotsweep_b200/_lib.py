"""ctypes binding of libshotsweep.so (the C ABI declared in include/shotsweep.h).

The library is the only compute path: if it is missing or no CUDA device is
present, every call raises; there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import threading
from pathlib import Path

import torch

LIB_PATH = Path(__file__).resolve().parent / 'libshotsweep.so'
MAX_SHOTS = 16

OK, ERR_INVALID, ERR_UNSUPPORTED, ERR_CUDA, ERR_TIMEOUT, ERR_WORKSPACE, ERR_NONFINITE = 0, -1, -2, -3, -4, -5, -6
MODE_FORWARD, MODE_GRADIENT, MODE_IMAGES, MODE_SEGMENT = 0, 1, 2, 3


class Geometry(ctypes.Structure):
    """Mirror of ss_geometry."""
    _fields_ = [('nz', ctypes.c_int32), ('nx', ctypes.c_int32), ('nt', ctypes.c_int32), ('pad', ctypes.c_int32),
                ('n_shots', ctypes.c_int32), ('src_row', ctypes.c_int32),
                ('shot_cols', ctypes.c_int32 * MAX_SHOTS),
                ('dx', ctypes.c_double), ('dt', ctypes.c_double), ('r_coef', ctypes.c_double),
                ('vmax_damping', ctypes.c_double), ('amp_ref', ctypes.c_double)]


def make_geometry(nz, nx, nt, pad, shot_cols, src_row=1, dx=10.0, dt=1e-3, r_coef=1e-5,
                  vmax_damping=4500.0, amp_ref=2000.0):
    if not 1 <= len(shot_cols) <= MAX_SHOTS:
        raise ValueError(f'between 1 and {MAX_SHOTS} shots are supported')
    g = Geometry()
    g.nz, g.nx, g.nt, g.pad = int(nz), int(nx), int(nt), int(pad)
    g.n_shots, g.src_row = len(shot_cols), int(src_row)
    for i, c in enumerate(shot_cols):
        g.shot_cols[i] = int(c)
    g.dx, g.dt, g.r_coef, g.vmax_damping, g.amp_ref = float(dx), float(dt), float(r_coef), float(vmax_damping), float(amp_ref)
    return g


class BatchItem(ctypes.Structure):
    """Mirror of ss_batch_item."""
    _fields_ = [('nz', ctypes.c_int32), ('nx', ctypes.c_int32), ('nt', ctypes.c_int32), ('pad', ctypes.c_int32),
                ('n_shots', ctypes.c_int32), ('src_row', ctypes.c_int32),
                ('shot_cols', ctypes.c_int32 * MAX_SHOTS),
                ('vel_offset', ctypes.c_int64), ('obs_offset', ctypes.c_int64), ('out_offset', ctypes.c_int64),
                ('v_mute', ctypes.c_float), ('reserved', ctypes.c_int32)]


class Physics(ctypes.Structure):
    """Mirror of ss_physics."""
    _fields_ = [('dx', ctypes.c_double), ('dt', ctypes.c_double), ('r_coef', ctypes.c_double),
                ('vmax_damping', ctypes.c_double), ('amp_ref', ctypes.c_double)]


class BatchClassInfo(ctypes.Structure):
    """Mirror of ss_batch_class_info."""
    _fields_ = [('min_cluster', ctypes.c_int32), ('cluster', ctypes.c_int32), ('n_solves', ctypes.c_int32),
                ('threads', ctypes.c_int32), ('smem_bytes', ctypes.c_int32), ('slots', ctypes.c_int32),
                ('stream', ctypes.c_int32), ('rows_per_thread', ctypes.c_int32), ('cell_steps', ctypes.c_double)]


class SurfaceEstimate(ctypes.Structure):
    """Mirror of ss_surface_estimate."""
    _fields_ = [('velocity', ctypes.c_double), ('confidence', ctypes.c_double), ('fit_rmse_ms', ctypes.c_double),
                ('short_offset_curvature', ctypes.c_double), ('shot_slope_spread', ctypes.c_double),
                ('far_offset_velocity', ctypes.c_double), ('possible_refraction', ctypes.c_int32),
                ('status', ctypes.c_int32)]


EPI_F32, EPI_F32_ADD, EPI_BIAS_LRELU_BF16, EPI_BIAS_F32 = 0, 1, 2, 3
SURF_OK, SURF_NO_ONSETS, SURF_FEW_NEAR, SURF_SLOPE, SURF_FEW_SHOTS, SURF_UNRELIABLE, SURF_NONFINITE = range(7)
MAX_CLUSTER = 16

_P = ctypes.c_void_p
_SIGNATURES = {
    'ss_version': (ctypes.c_char_p, []),
    'ss_last_error': (ctypes.c_char_p, []),
    'ss_workspace_bytes': (ctypes.c_size_t, [ctypes.POINTER(Geometry), ctypes.c_int32, ctypes.c_int32]),
    'ss_set_rows_per_thread': (ctypes.c_int32, [ctypes.c_int32, ctypes.c_int32]),
    'ss_workspace_slots': (ctypes.c_int32, [ctypes.POINTER(Geometry), ctypes.c_int32, ctypes.c_size_t]),
    'ss_workspace_bytes_slots': (ctypes.c_size_t, [ctypes.POINTER(Geometry), ctypes.c_int32, ctypes.c_int32]),
    'ss_workspace_status': (ctypes.c_int32, [_P, _P]),
    'ss_plan_info': (ctypes.c_int32, [ctypes.POINTER(Geometry), ctypes.c_int32, ctypes.c_int32,
                                      ctypes.POINTER(ctypes.c_int64)]),
    'ss_forward': (ctypes.c_int32, [ctypes.POINTER(Geometry), ctypes.c_int32, _P, _P, _P, _P, ctypes.c_int32,
                                    _P, ctypes.c_size_t, _P]),
    'ss_gradient': (ctypes.c_int32, [ctypes.POINTER(Geometry), ctypes.c_int32, _P, _P, _P, _P, ctypes.c_float,
                                     _P, _P, _P, ctypes.c_size_t, _P]),
    'ss_images': (ctypes.c_int32, [ctypes.POINTER(Geometry), ctypes.c_int32, _P, _P, _P, _P, ctypes.c_float,
                                   ctypes.c_float, ctypes.c_int32, _P, _P, _P, _P, ctypes.c_size_t, _P]),
    'ss_forward_wavelets': (ctypes.c_int32, [ctypes.POINTER(Geometry), ctypes.c_int32, _P, _P, _P, _P,
                                             ctypes.c_size_t, _P]),
    'ss_gradient_wavelets': (ctypes.c_int32, [ctypes.POINTER(Geometry), ctypes.c_int32, _P, _P, _P, _P,
                                              ctypes.c_float, _P, _P, _P, ctypes.c_size_t, _P]),
    'ss_lap_f32': (ctypes.c_int32, [_P, _P, ctypes.c_int64, ctypes.c_int32, ctypes.c_int32, _P]),
    'ss_lap_f64': (ctypes.c_int32, [_P, _P, ctypes.c_int64, ctypes.c_int32, ctypes.c_int32, _P]),
    'ss_lap_adjoint_f32': (ctypes.c_int32, [_P, _P, ctypes.c_int64, ctypes.c_int32, ctypes.c_int32, _P]),
    'ss_lap_adjoint_f64': (ctypes.c_int32, [_P, _P, ctypes.c_int64, ctypes.c_int32, ctypes.c_int32, _P]),
    'ss_fold_edge_padding_f32': (ctypes.c_int32, [_P, _P, ctypes.c_int64, ctypes.c_int32, ctypes.c_int32,
                                                  ctypes.c_int32, _P]),
    'ss_fold_edge_padding_f64': (ctypes.c_int32, [_P, _P, ctypes.c_int64, ctypes.c_int32, ctypes.c_int32,
                                                  ctypes.c_int32, _P]),
    'ss_mute_weights': (ctypes.c_int32, [ctypes.POINTER(Geometry), ctypes.c_int32, _P, ctypes.c_float, _P, _P]),
    'ss_c2_field': (ctypes.c_int32, [ctypes.POINTER(Geometry), ctypes.c_int32, _P, _P, _P]),
    'ss_fp32_probe': (ctypes.c_int32, [_P, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                       ctypes.POINTER(ctypes.c_double), _P]),
    'ss_segment_workspace_bytes': (ctypes.c_size_t, [ctypes.POINTER(Geometry), ctypes.c_int32, ctypes.c_int32]),
    'ss_adjoint_segment': (ctypes.c_int32, [ctypes.POINTER(Geometry), ctypes.c_int32, _P, _P, _P, ctypes.c_int32,
                                            ctypes.c_int32, _P, _P, _P, _P, _P, _P, ctypes.c_size_t, _P]),
    'ss_gradient_finish': (ctypes.c_int32, [ctypes.POINTER(Geometry), ctypes.c_int32, _P, _P, _P, _P, _P, _P, _P]),
    'ss_batch_plan': (ctypes.c_int32, [ctypes.POINTER(Physics), ctypes.c_int32, ctypes.POINTER(BatchItem),
                                       ctypes.c_int32, ctypes.POINTER(ctypes.c_int32), ctypes.c_int32, _P,
                                       ctypes.POINTER(ctypes.c_size_t), ctypes.POINTER(ctypes.c_size_t)]),
    'ss_batch_min_cluster': (ctypes.c_int32, [ctypes.POINTER(BatchItem), ctypes.c_int32]),
    'ss_batch_min_cluster_rows': (ctypes.c_int32, [ctypes.POINTER(BatchItem), ctypes.c_int32, ctypes.c_int32]),
    'ss_batch_classes': (ctypes.c_int32, [_P, ctypes.POINTER(BatchClassInfo), ctypes.c_int32,
                                          ctypes.POINTER(ctypes.c_int32)]),
    'ss_batch_run': (ctypes.c_int32, [_P, _P, _P, _P, _P, ctypes.c_float, ctypes.c_float, ctypes.c_int32, _P, _P, _P,
                                      _P, _P, ctypes.c_size_t, _P]),
    'ss_surface_velocity': (ctypes.c_int32, [_P, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                             ctypes.POINTER(ctypes.c_double), ctypes.c_double, ctypes.c_double,
                                             ctypes.c_double, _P, _P]),
    'ss_backgrounds': (ctypes.c_int32, [_P, _P, _P, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                        _P, _P]),
    'ss_image_cache': (ctypes.c_int32, [_P, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                        ctypes.c_int32, ctypes.c_double, ctypes.c_float, _P, _P, _P, _P]),
    'ss_signed_log1p_f16': (ctypes.c_int32, [_P, ctypes.c_int64, _P, _P]),
    'ss_f16_scaled': (ctypes.c_int32, [_P, ctypes.c_int64, ctypes.c_float, _P, _P]),
    'ss_velocity_targets': (ctypes.c_int32, [_P, ctypes.c_int64, _P, _P, _P, ctypes.c_int32, ctypes.c_int32,
                                             ctypes.c_int32, _P, _P]),
    'ss_gemm_bf16': (ctypes.c_int32, [_P, ctypes.c_int64, _P, ctypes.c_int64, ctypes.c_int32, ctypes.c_int32,
                                      ctypes.c_int32, ctypes.c_int32, _P, ctypes.c_int64, _P, ctypes.c_float,
                                      ctypes.c_int32, _P, _P]),
    'ss_gemm_bf16_layout': (ctypes.c_int32, [_P, ctypes.c_int64, _P, ctypes.c_int64, ctypes.c_int32, ctypes.c_int32,
                                             ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, _P, ctypes.c_int64, _P,
                                             ctypes.c_float, ctypes.c_int32, _P, _P]),
    'ss_im2col_bf16': (ctypes.c_int32, [_P, _P, ctypes.c_int32, _P, _P]),
    'ss_col2im16_lrelu_bf16': (ctypes.c_int32, [_P, _P, ctypes.c_int32, _P, ctypes.c_float, _P, ctypes.c_int64, _P]),
    'ss_bias_grad_bf16': (ctypes.c_int32, [_P, ctypes.c_int64, ctypes.c_int64, ctypes.c_int32, _P, _P]),
    'ss_head_forward': (ctypes.c_int32, [_P, _P, _P, _P, _P, _P]),
    'ss_head_backward': (ctypes.c_int32, [_P, _P, _P, _P, ctypes.c_float, _P, _P, _P, _P]),
    'ss_l1_tanh_loss': (ctypes.c_int32, [_P, _P, ctypes.c_int64, _P, _P, _P]),
    'ss_adamw': (ctypes.c_int32, [_P, _P, _P, _P, ctypes.c_int64, _P, ctypes.c_float, ctypes.c_float, ctypes.c_float,
                                  ctypes.c_float, _P, _P, _P]),
    'ss_gather_rows_f32': (ctypes.c_int32, [_P, _P, ctypes.c_int32, ctypes.c_int64, _P, _P]),
    'ss_gathers_nhwc_bf16': (ctypes.c_int32, [_P, _P, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                              ctypes.c_float, _P, _P]),
    'ss_fwi_precondition': (ctypes.c_int32, [_P, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                             ctypes.c_float, _P, _P]),
    'ss_fwi_misfit': (ctypes.c_int32, [_P, _P, ctypes.c_int32, ctypes.c_int64, _P, _P]),
    'ss_lbfgs_direction': (ctypes.c_int32, [_P, _P, _P, _P, _P, _P, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                            ctypes.c_float, _P, _P, _P]),
    'ss_fwi_trial': (ctypes.c_int32, [_P, _P, _P, _P, ctypes.c_int32, ctypes.c_int32, ctypes.c_float, ctypes.c_float,
                                      _P, _P]),
    'ss_lbfgs_push': (ctypes.c_int32, [_P, _P, _P, _P, _P, _P, _P, _P, _P, ctypes.c_int32, ctypes.c_int32,
                                       ctypes.c_int32, _P]),
    'ss_wait_probe': (ctypes.c_int32, [_P, ctypes.c_double, _P]),
    'ss_images_noalloc': (ctypes.c_int32, [ctypes.POINTER(Geometry), ctypes.c_int32, _P, _P, _P, _P, ctypes.c_float,
                                           ctypes.c_float, ctypes.c_int32, _P, _P, _P, _P]),
}

_lock = threading.Lock()
_lib = None


def load(path=LIB_PATH):
    """Load the library once and declare every exported signature."""
    global _lib
    with _lock:
        if _lib is None:
            if not Path(path).exists():
                raise RuntimeError(f'libshotsweep is not built ({path}); run python -m shotsweep_b200.build')
            lib = ctypes.CDLL(str(path))
            for name, (res, args) in _SIGNATURES.items():
                fn = getattr(lib, name)
                fn.restype, fn.argtypes = res, args
            _lib = lib
        return _lib


def exported_symbols():
    return list(_SIGNATURES)


def check(rc, what):
    """Turn an ss_status into the reference's exception types."""
    if rc == OK:
        return
    msg = load().ss_last_error().decode() or 'unknown error'
    if rc in (ERR_INVALID, ERR_NONFINITE):
        raise ValueError(f'{what}: {msg}')
    raise RuntimeError(f'{what} failed ({rc}): {msg}')


def ptr(t):
    return ctypes.c_void_p(0 if t is None else t.data_ptr())


def stream_handle(device):
    return ctypes.c_void_p(torch.cuda.current_stream(device).cuda_stream)


def require_cuda(device):
    if device.type != 'cuda' or not torch.cuda.is_available():
        raise RuntimeError('shotsweep_b200 runs on a CUDA (sm_100a) device only; no CPU path exists')
