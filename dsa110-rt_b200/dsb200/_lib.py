"""ctypes binding of ``libdsb200.so`` (the C ABI declared in include/dsb200.h).

The library is built in-tree (``__graft_entry__.build()``).  There is no CPU
fallback anywhere in this package: if the library is missing, or a tensor
is not on a CUDA device, calls raise.
"""

from __future__ import annotations

import ctypes
import os
from typing import Optional

import torch

_HERE = os.path.dirname(os.path.abspath(__file__))
# DSB200_CHECK=1 loads the bounds-checked build (table indices range-checked
# on the device, violations reported as DSB_E_BOUNDS in the status words)
CHECKED = os.environ.get("DSB200_CHECK", "") == "1"
SO_PATH = os.path.join(_HERE, "_native", "libdsb200_check.so" if CHECKED else "libdsb200.so")

DT_INT8, DT_F16, DT_F32 = 0, 1, 2

_c_int, _c_ll, _c_float, _vp = ctypes.c_int, ctypes.c_longlong, ctypes.c_float, ctypes.c_void_p

# name -> argtypes (all return c_int except those in _RESTYPES)
_SIGNATURES = {
    "dsb_version": [],
    "dsb_unpack_int4": [_vp, _c_int, _c_int, _c_int, _c_int, _c_float, _vp, _vp, _vp],
    "dsb_corr_split": [_vp, _vp, _c_int, _c_int, _c_int, _c_int, _c_int, _c_int, _c_int, _vp, _vp,
                       _vp],
    "dsb_corr_tc": [_vp, _c_ll, _c_int, _c_int, _c_int, _c_int, _c_int, _c_int, _c_int, _vp,
                    _c_ll, _c_ll, _c_ll, _c_ll, _c_int, _vp, _vp],
    "dsb_corr_tc_grid": [_vp, _c_ll, _c_int, _c_int, _c_int, _c_int, _c_int, _c_int, _vp, _vp,
                         _vp, _vp, _vp, _c_ll, _c_ll, _c_ll, _c_int, _vp, _vp, _vp],
    "dsb_uv_cells": [_vp, _vp, _c_int, _vp, _c_int, ctypes.c_double, _c_int, _vp, _vp, _vp],
    "dsb_grid_vis": [_vp, _c_int, _c_ll, _vp, _vp, _c_int, _vp, _vp],
    "dsb_dedisp_vis": [_vp, _vp, _c_int, _c_ll, _c_int, _vp, _vp, _vp, _c_int, _c_int, _c_int,
                       _vp, _vp],
    "dsb_static_sky": [_vp, _vp, _c_int, _c_int, _vp, _c_int, _c_int, _c_int, _c_int, _vp],
    "dsb_stage2_roll": [_vp, _c_int, _vp, _vp, _vp, _c_int, _c_int, _c_ll, _vp, _vp],
    "dsb_stage1_rows": [_vp, _c_ll, _c_ll, _c_int, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp,
                        _vp, _c_int, _vp, _vp, _vp, _c_ll, _c_int, _c_int, _c_int, _c_int,
                        _c_int, _vp, _c_int, _c_int, _c_int, _c_int, _vp, _vp],
    "dsb_stage1_block_size": [],
    "dsb_stage1_dm_group": [],
    "dsb_stage1_smem_bytes": [_c_int, _c_int, _c_int],
    "dsb_image_geometry": [_c_int, _vp],
    "dsb_graph_begin": [_vp],
    "dsb_graph_end_launch": [_vp, _vp],
    "dsb_graph_abort": [_vp],
    "dsb_graph_destroy": [_vp],
    "dsb_irfft2": [_vp, _c_int, _c_int, _vp, _vp, _vp],
    "dsb_image_fft": [_vp, _c_int, _vp, _vp, _vp, _vp, _vp, _vp, _c_int, _c_int, _c_int, _vp, _vp, _vp, _c_int, _vp, _vp, _vp, _c_int,
                      _c_int, _vp,
                      _vp, _c_int, _vp, _c_int, _vp, _vp, _vp, _vp, _vp, _c_int, _c_int, _c_int,
                      _c_int, _c_ll, _c_int, _c_int, _vp, _c_int, _vp, _vp],
    "dsb_combine_rows": [_vp, _c_int, _vp, _vp, _vp, _vp, _c_int, _vp, _vp, _vp, _vp, _vp, _vp, _c_int, _c_int,
                         _c_int, _c_int, _c_ll, _c_int, _c_int, _vp, _vp],
    "dsb_combine_dense": [_vp, _vp, _vp, _vp, _vp, _c_int, _vp, _c_int, _c_int, _c_int, _c_int,
                          _c_int, _c_int, _c_int, _c_int, _vp],
    "dsb_combine_sparse": [_vp, _vp, _vp, _vp, _vp, _vp, _c_int, _vp, _vp, _c_int, _c_int,
                           _c_int, _c_int, _c_int, _c_int, _c_int, _c_int, _c_int, _c_int,
                           _c_int, _c_int, _vp, _vp],
    "dsb_encode_rows": [_vp, _c_ll, _c_int, _c_int, _c_int, _vp, _vp, _vp],
    "dsb_cluster_mst": [_vp, _c_int, _c_int, _c_int, _vp, _vp],
    "dsb_cal_apply": [_vp, _vp, _vp, _vp, _c_int, _c_int, _c_int, _c_int, _c_int, _c_int, _c_int,
                      _vp, _vp, _vp],
    "dsb_ring_encode_cint8": [_vp, _vp, _c_int, _vp, _vp, _c_int, _c_int, _vp, _c_ll, _vp, _vp,
                              _vp, _vp, _vp, _vp, _vp],
    "dsb_rfi_zero_fill": [_vp, _c_int, _c_int, _c_int, _c_int, _vp, _vp, _c_int, _vp],
    "dsb_mask_to_cube": [_vp, _vp, _c_int, _c_int, _c_int, _c_int, _vp, _c_int, _c_int, _c_int,
                         _vp],
    "dsb_padded_cumsum": [_vp, _c_int, _c_int, _c_ll, _c_int, _vp, _vp],
    "dsb_multi_boxcar_argmax": [_vp, _c_ll, _vp, _vp, _vp, _c_int, _c_int, _c_int, _vp, _c_int,
                                _vp, _vp],
    "dsb_boxcar_from_cs": [_vp, _c_ll, _c_int, _c_int, _c_int, _vp, _vp],
    "dsb_boxcar_argmax_noalloc": [_vp, _c_int, _c_int, _c_ll, _c_int, _vp, _vp, _vp, _c_int,
                                  _c_int, _c_int, _vp, _c_int, _vp, _vp],
    "dsb_detect": [_vp, _c_int, _c_int, _c_int, _c_int, _c_ll, _c_ll, _vp, _c_ll, _vp, _c_int,
                   _vp, _c_int, _c_int, _c_float, _vp, _c_int, _c_int, _vp, _vp],
    "dsb_detect_sampled": [_vp, _c_int, _c_int, _c_int, _c_int, _c_ll, _c_ll, _vp, _c_ll, _vp,
                           _c_int, _vp, _c_int, _c_int, _c_float, _vp, _c_int, _c_int, _vp,
                           _vp, _vp, _vp, _c_int, _vp],
    "dsb_clipped_std": [_vp, _c_int, _c_int, _c_float, _c_int, _vp, _vp],
    "dsb_layer1_sigma": [_vp, _c_ll, _c_ll, _c_int, _vp, _c_int, _vp, _c_int, _c_float, _c_int,
                         _vp, _vp],
}

_RESTYPES = {"dsb_stage1_smem_bytes": _c_ll}

_lib: Optional[ctypes.CDLL] = None


class DsbError(RuntimeError):
    """A dsb200 C-ABI call returned an error code."""


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(SO_PATH):
            raise RuntimeError(
                f"dsb200 native library missing ({SO_PATH}); build it with "
                "`python -c 'import __graft_entry__ as g; g.build()'` (check=True for the "
                "bounds-checked one) — there is no CPU fallback")
        L = ctypes.CDLL(SO_PATH)
        for name, args in _SIGNATURES.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = _RESTYPES.get(name, _c_int)
        L.dsb_strerror.argtypes = [_c_int]
        L.dsb_strerror.restype = ctypes.c_char_p
        _lib = L
    return _lib


def declared_symbols():
    return list(_SIGNATURES) + ["dsb_strerror"]


def check(rc: int, what: str) -> None:
    if rc != 0:
        msg = lib().dsb_strerror(rc).decode()
        raise DsbError(f"{what}: {msg} (code {rc})")


def ptr(t: Optional[torch.Tensor]) -> ctypes.c_void_p:
    return ctypes.c_void_p(0 if t is None else t.data_ptr())


def stream_of(dev: torch.device) -> ctypes.c_void_p:
    return ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)


def require_cuda(t: torch.Tensor, name: str) -> None:
    if not isinstance(t, torch.Tensor):
        raise TypeError(f"{name} must be a torch.Tensor, got {type(t).__name__}")
    if t.device.type != "cuda":
        raise ValueError(f"{name} must be on a CUDA device (no CPU path), got {t.device}")
    if not t.is_contiguous():
        raise ValueError(f"{name} must be contiguous")


def cuda_device(device) -> torch.device:
    dev = torch.device(device)
    if dev.type != "cuda":
        raise ValueError(f"dsb200 runs on CUDA devices only (no CPU path); got {dev}")
    if dev.index is None:
        dev = torch.device("cuda", torch.cuda.current_device())
    return dev


def status_word(dev: torch.device) -> torch.Tensor:
    return torch.zeros(1, dtype=torch.int32, device=dev)


def check_status(status: torch.Tensor, what: str) -> None:
    code = int(status.item())
    if code != 0:
        msg = lib().dsb_strerror(code).decode()
        raise DsbError(f"{what}: device status {msg} (code {code})")
