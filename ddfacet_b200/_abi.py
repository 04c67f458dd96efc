"""ctypes binding of libddfg.so (include/ddfg.h).

The structures below mirror the C header field for field.  ``lib()`` loads the in-tree library
(building it first if it is missing and nvcc is available) and raises if it cannot: there is no
fallback implementation behind this module.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

from . import build as _build

DDFG_OK = 0
DDFG_EINVAL = -1
DDFG_EUNSUPPORTED = -2
DDFG_ECUDA = -3
DDFG_EMAP = -4
DDFG_ESIZE = -5
DDFG_MAX_FACETS = 1024
DDFG_FACETS_PER_LAUNCH = 16
DDFG_TABLE_FACETS = 128

_i32 = C.c_int32
_i64 = C.c_int64
_f64 = C.c_double
_vp = C.c_void_p


class Facet(C.Structure):
    _fields_ = [
        ("grid", _vp),
        ("nband", _i32), ("npol", _i32), ("ny", _i32), ("nx", _i32),
        ("incr_x", _f64), ("incr_y", _f64),
        ("cu", _f64), ("cv", _f64), ("l0", _f64), ("m0", _f64),
        ("cf_data", _vp), ("cf_offset", _vp), ("cf_support", _vp),
        ("nw", _i32), ("overs", _i32),
        ("max_support", _i32),
        ("ref_wave", _f64), ("wmax", _f64),
        ("idir_kms", _i32), ("idir_beam", _i32),
        ("decorr_l", _f64), ("decorr_m", _f64),
        ("sumwt", _vp), ("sumjones", _vp), ("sumjones_chan", _vp),
        ("grid_acc", _vp),
    ]


class VisSet(C.Structure):
    _fields_ = [
        ("vis", _vp), ("uvw", _vp), ("flags", _vp), ("weights", _vp), ("freqs", _vp),
        ("freq_mean", _f64),
        ("recip_wvl", _vp),
        ("chan_map", _vp),
        ("nrow", _i64), ("nchan", _i32), ("ncorr", _i32),
        ("chan_equidistant", _i32),
        ("single_vis_blocks", _i32),
        ("bda_map", _vp), ("bda_len", _i64), ("block_start", _vp), ("nblocks", _i64),
        ("sparsification", _vp),
        ("uvw_dt", _vp), ("dt", _f64), ("dnu", _f64), ("do_tsmear", _i32), ("do_fsmear", _i32),
        ("large_blocks", _vp), ("nlarge", _i64), ("large_min_vis", _i64),
    ]


class Jones(C.Structure):
    _fields_ = [
        ("mode", _i32),
        ("kms", _vp), ("kms_dims", _i32 * 4), ("kms_tmap", _vp), ("kms_cmap", _vp),
        ("beam", _vp), ("beam_dims", _i32 * 4), ("beam_tmap", _vp), ("beam_cmap", _vp),
        ("a0", _vp), ("a1", _vp),
        ("interp_coefs", _vp), ("interp_mode", _i32),
        ("apply_amp", _i32), ("apply_phase", _i32), ("scale_jones", _i32),
        ("calib_error", _f64), ("wavelength_mean", _f64),
    ]


class Batch(C.Structure):
    _fields_ = [("workspace", _vp), ("workspace_bytes", C.c_size_t), ("facets_per_pack", _i32),
                ("stripes_per_item", _i32), ("ctas_per_sm", _i32), ("flags", _i32)]


class Pol(C.Structure):
    _fields_ = [("ncorr", _i32), ("npol", _i32), ("corr_ids", _i32 * 4), ("stokes_ids", _i32 * 4)]


# Entry points declared in include/ddfg.h, with their ctypes signatures.
SIGNATURES = {
    "ddfg_version": (C.c_int, []),
    "ddfg_last_error": (C.c_int, [C.c_char_p, C.c_int]),
    "ddfg_bda_plan_workspace_size": (C.c_size_t, [_i64]),
    "ddfg_bda_plan": (C.c_int, [_vp, _i64, _i64, _i64, _i32, _vp, _vp, C.c_size_t, _vp, C.POINTER(_i32)]),
    "ddfg_bda_plan_noalloc": (C.c_int, [_vp, _i64, _i64, _i64, _i32, _vp, _vp, C.POINTER(_i32)]),
    "ddfg_grid": (C.c_int, [C.POINTER(VisSet), C.POINTER(Jones), C.POINTER(Pol), C.POINTER(Facet), C.c_int,
                            C.c_int, _vp]),
    "ddfg_degrid": (C.c_int, [C.POINTER(VisSet), C.POINTER(Jones), C.POINTER(Pol), C.POINTER(Facet), C.c_int,
                              _vp]),
    "ddfg_degrid_adjoint": (C.c_int, [C.POINTER(VisSet), C.POINTER(Jones), C.POINTER(Pol), C.POINTER(Facet),
                                      C.c_int, _vp]),
    "ddfg_degrid_jones_grad": (C.c_int, [C.POINTER(VisSet), C.POINTER(Jones), C.POINTER(Pol), C.POINTER(Facet),
                                         C.c_int, _vp, _vp]),
    "ddfg_weights_uv_index": (C.c_int, [_vp, _i64, _vp, _i32, _vp, _vp, _i32, _f64, _i64, _i64, _i64, _vp, _vp]),
    "ddfg_weights_accumulate": (C.c_int, [_vp, _i64, _vp, _vp, _i64, _vp, _vp]),
    "ddfg_weights_robust": (C.c_int, [_vp, _i64, _i32, _f64, _vp, _vp]),
    "ddfg_weights_finalize": (C.c_int, [_vp, _vp, _i64, _vp, _i64, _vp]),
    "ddfg_bda_mode1_count": (C.c_int, [_vp, _vp, _vp, _i32, _i32, _vp, _f64, _f64, _f64, _f64, _vp, _vp, _vp]),
    "ddfg_bda_mode1_write": (C.c_int, [_vp, _vp, _vp, _i32, _i32, _vp, _f64, _f64, _f64, _f64, _vp, _vp, _vp, _vp,
                                       _vp]),
    "ddfg_bda_mode2_count": (C.c_int, [_vp, _vp, _vp, _i32, _i32, _vp, _f64, _f64, _f64, _f64, _vp, _vp, _vp]),
    "ddfg_bda_mode2_write": (C.c_int, [_vp, _vp, _vp, _i32, _i32, _vp, _f64, _f64, _f64, _f64, _vp, _vp, _vp, _vp,
                                       _vp]),
    "ddfg_batch_workspace_size": (C.c_size_t, []),
    "ddfg_grid_batched": (C.c_int, [C.POINTER(VisSet), C.POINTER(Jones), C.POINTER(Pol), C.POINTER(Facet), C.c_int,
                                    C.c_int, C.POINTER(Batch), _vp]),
    "ddfg_degrid_batched": (C.c_int, [C.POINTER(VisSet), C.POINTER(Jones), C.POINTER(Pol), C.POINTER(Facet),
                                      C.c_int, C.POINTER(Batch), _vp]),
    "ddfg_block_geometry": (C.c_int, [C.POINTER(VisSet), C.POINTER(Facet), C.c_int, _vp, _vp]),
    "ddfg_jones_time_map": (C.c_int, [_vp, _i64, _vp, _vp, _i32, _vp, _vp]),
    "ddfg_check_large_blocks_workspace_size": (C.c_size_t, [_i64]),
    "ddfg_check_large_blocks": (C.c_int, [C.POINTER(VisSet), _vp, C.c_size_t, _vp]),
    "ddfg_fft_plan_create": (C.c_int, [_i32, _i32, C.POINTER(_vp)]),
    "ddfg_fft_plan_destroy": (C.c_int, [_vp]),
    "ddfg_grid_to_image": (C.c_int, [_vp, _vp, _f64, _vp, _vp]),
    "ddfg_fft_centred": (C.c_int, [_vp, _vp, _i32, _f64, _vp, _vp]),
    "ddfg_stitch_facet": (C.c_int, [_vp, _i32, _i32, _i32, _vp, _vp, _vp, _vp, _vp, _i32, _i32, _i32, _vp]),
    "ddfg_image_normalise": (C.c_int, [_vp, _i32, _i32, _vp, _vp]),
    "ddfg_image_to_grid": (C.c_int, [_vp, _vp, _i32, _vp, _vp, _vp, _i32, _i32, _f64, _vp, _vp, _vp]),
    "ddfg_image_to_grid_adjoint": (C.c_int, [_vp, _vp, _i32, _vp, _vp, _vp, _i32, _i32, _f64, _vp, _vp, _vp]),
}

_lock = threading.Lock()
_lib = None


class DDFGError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"ddfg error {code}: {msg}")
        self.code = code
        self.msg = msg


def lib_path() -> str:
    return _build.LIB


def lib():
    """Load (building if needed) libddfg.so; raise if it cannot be loaded."""
    global _lib
    with _lock:
        if _lib is None:
            path = _build.LIB
            if not os.path.exists(path):
                _build.build()
            # torch first, so the library binds to the CUDA runtime torch already loaded.
            import torch  # noqa: F401
            h = C.CDLL(path, mode=C.RTLD_GLOBAL)
            for name, (res, args) in SIGNATURES.items():
                fn = getattr(h, name)
                fn.restype = res
                fn.argtypes = args
            _lib = h
    return _lib


def last_error() -> str:
    buf = C.create_string_buffer(512)
    lib().ddfg_last_error(buf, 512)
    return buf.value.decode(errors="replace")


def check(rc: int):
    if rc != DDFG_OK:
        msg = last_error()
        if rc == DDFG_EUNSUPPORTED:
            raise ValueError(msg)
        raise DDFGError(rc, msg)
    return rc
