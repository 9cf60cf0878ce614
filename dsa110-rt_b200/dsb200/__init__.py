"""dsb200 — B200 (sm_100a) implementation of dsa110-rt's fast FRB-search
hot path, behind the reference's own Python call surface.

Kernels live in ``libdsb200.so`` (C ABI: include/dsb200.h); this package is
the host side.  No CPU fallback: every op requires CUDA tensors and the
native library.
"""

from .constants import Band, DSA110_BAND, NANTS, NBASE, NCHAN_PER_CHGROUP  # noqa: F401

__all__ = ["Band", "DSA110_BAND", "NANTS", "NBASE", "NCHAN_PER_CHGROUP"]
