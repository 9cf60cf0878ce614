"""Slow correlator product (services/slow_corr_kernel.py:576-720).

* CPU: the oracle correlator over one full block, both pols, equals the
  reference's ``SlowCorrKernel`` on the same unpacked page (float32 integer
  codes, exact), by content hash and sampled values.
* GPU: ``dsb200.corr.SlowCorrKernel`` on int8 codes equals the oracle bit
  for bit.
"""

import os
import sys

import numpy as np
import pytest
import torch

import dsb_oracle as O

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
import make_golden as MG  # noqa: E402


@pytest.fixture(scope="module")
def oracle_vis():
    re, im = O.unpack_int4_gemm_layout(MG.unpack_raw(), 2048, 96, 384)
    vr, vi = O.corr_fast(re, im, t_int=4096, fuse_stokes_i=False)
    return (vr[0] + 1j * vi[0]).astype(np.complex64)


def test_oracle_full_block_matches_reference(golden_dir, oracle_vis):
    z = np.load(os.path.join(golden_dir, "slow_corr.npz"))
    assert tuple(oracle_vis.shape) == tuple(z["shape"])
    np.testing.assert_array_equal(oracle_vis.reshape(-1)[z["idx"]], z["samples"])
    assert MG.sha(np.ascontiguousarray(oracle_vis).view(np.float32)) == str(z["sha"])


@pytest.mark.gpu
def test_slow_corr_gpu_matches_oracle(oracle_vis):
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from dsb200.corr import SlowCorrKernel, unpack_int4_split
    dev = torch.device("cuda", 0)
    re, im = unpack_int4_split(MG.unpack_raw(), device=dev, out_dtype=torch.int8)
    vis = SlowCorrKernel(dev).compute_split(re, im).cpu().numpy()
    np.testing.assert_array_equal(vis, oracle_vis)
    with pytest.raises(ValueError):
        SlowCorrKernel(dev).compute_split(re[:, :, :, :8], im[:, :, :, :8])
