"""The detector kernel bank (detector/kernels.py:191) against the
reference's own bank (fixture): ids, widths and (image, dm, time) order of
the default 128-kernel bank and of the production b1..b64 bank, and the
reference's validation errors."""

import os

import numpy as np
import pytest

from dsb200.kernels import build_kernel_bank

HERE = os.path.dirname(os.path.abspath(__file__))


def test_banks_equal_reference():
    z = np.load(os.path.join(HERE, "golden", "kernel_bank.npz"))
    for name, kw in (("full", {}), ("prod", dict(image_tokens=("unit",), dm_tokens=("d1",),
                                                 time_tokens=("b1", "b2", "b4", "b8", "b16",
                                                              "b32", "b64")))):
        bank = build_kernel_bank(**kw)
        assert [k.kernel_id for k in bank] == z[f"{name}_ids"].tolist()
        assert [[k.k_dm_width, k.k_time_width, k.image_kernel_size] for k in bank] == \
            z[f"{name}_w"].tolist()


@pytest.mark.parametrize("kw", [dict(image_tokens=("gauss",)), dict(dm_tokens=("d2",)),
                                dict(time_tokens=("b3",)), dict(time_tokens=("x4",))])
def test_bank_rejects_bad_tokens(kw):
    with pytest.raises(ValueError):
        build_kernel_bank(**kw)
