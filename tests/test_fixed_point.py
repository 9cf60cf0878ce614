"""The image kernel's fixed-point combine, restated on CPU: for every ring
form, the per-image power of two 2^k chosen from the bound keeps each part
below 2^(30 - ceil(log2 s_mult)) and every S sum below 2^30 (no int32
overflow), and rounds a part by at most 2^-(k+1); bf16 parts within 2^16 of
the bound are exact (for bounds above about 2^-72, where k is not clamped).  Worst cases: parts at the bound (bf16 rounded up),
int8 codes of -128, every contribution of an S entry at the bound."""

import numpy as np
import pytest

import dsb_oracle as O


def _ilogb(x):
    return int(np.frexp(np.float32(x))[1]) - 1


def _k(bound, s_mult, cint8):
    lmm = int(np.ceil(np.log2(s_mult))) if s_mult > 1 else 0
    return min(100, (22 if cint8 else 28) - _ilogb(bound) - lmm), lmm


@pytest.mark.parametrize("s_mult", [1, 2, 5, 16, 32])
def test_float_forms_stay_in_int32(s_mult):
    rng = np.random.default_rng(s_mult)
    for _ in range(200):
        B = np.float32(10.0 ** rng.uniform(-30, 30))
        k, lmm = _k(B, s_mult, cint8=False)
        # the largest parts the bound admits: B itself, and B rounded up to bf16
        worst = np.float32(max(float(B), float(O.round_bf16(np.float32([B]))[0])))
        part = np.rint(np.float64(worst) * 2.0 ** k)
        assert part < 2.0 ** (30 - lmm)
        assert s_mult * part < 2.0 ** 30
        # bf16 parts down to 2^-16 of the bound are exact on the 2^-k grid,
        # unless k is clamped at 100 (bounds below about 2^-72, where the
        # kernel keeps 2^-k x 0.5/N^2 a normal float)
        if k < 100:
            v = O.round_bf16((rng.uniform(2.0 ** -16, 1.0, 1000) * float(B)).astype(np.float32))
            scaled = v.astype(np.float64) * 2.0 ** k
            assert np.array_equal(scaled, np.rint(scaled))


@pytest.mark.parametrize("s_mult", [1, 3, 16, 32])
def test_cint8_form_stays_in_int32(s_mult):
    rng = np.random.default_rng(100 + s_mult)
    for _ in range(200):
        scales = (10.0 ** rng.uniform(-20, 20, 16)).astype(np.float32)
        k, lmm = _k(scales.max(), s_mult, cint8=True)
        # the part the kernel rounds: float32(scale * 2^k) * q, q = -128 worst
        f = (scales.astype(np.float64) * 2.0 ** k).astype(np.float32)
        part = np.abs(np.rint(f.astype(np.float64) * -128.0)).max()
        assert part < 2.0 ** (30 - lmm)
        assert s_mult * part < 2.0 ** 30
