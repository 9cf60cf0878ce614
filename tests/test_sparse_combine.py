"""The compact-layout combine (combine_sparse_v4 + build_sparse_cell_csr,
image/tiled_combine_cuda.py:1092-1240).

* CPU: the CSR tables equal the reference's own build_sparse_cell_csr on
  seeded inverse LUTs (fixture made by running the reference), field by
  field, cell order and buckets included.
* GPU: the kernel equals the oracle (compact streams scattered back to dense
  grids, then combine_half) bit for bit, in fp16 pairs and complex64, with
  shifts that read outside the stream; and GpuImager.process_cube on the
  compact layout equals its dense path on the same streams.
"""

import os

import numpy as np
import pytest
import torch

import dsb_oracle as O
from dsb200.search import build_sparse_cell_csr

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.mark.parametrize("name", ["a", "b"])
def test_sparse_csr_equals_reference(name):
    z = np.load(os.path.join(HERE, "golden", "sparse_csr.npz"))
    csr = build_sparse_cell_csr(torch.from_numpy(z[f"{name}_lut"].astype(np.int64)),
                                n_grid=int(z[f"{name}_n_grid"]))
    for f in ("cell_uw", "cell_ptr", "ent_g", "ent_k", "ent_km"):
        np.testing.assert_array_equal(getattr(csr, f).numpy(), z[f"{name}_{f}"], err_msg=f)
    assert np.asarray(csr.buckets, np.int64).reshape(-1, 3).tolist() == \
        z[f"{name}_buckets"].tolist()


def _case(seed, n_sb=6, N=32, nfm=90, t_rows=40, t_pad=48):
    rng = np.random.default_rng(seed)
    lut = np.full((n_sb, N * N), -1, np.int64)
    for g in range(n_sb):
        cells = np.sort(rng.choice(N * N, nfm - 5 * g, replace=False))
        lut[g, cells] = rng.permutation(cells.size)
    dense = rng.integers(-128, 128, (n_sb, nfm, t_pad, 2)).astype(np.int8)
    return lut, dense, N, t_rows


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", [torch.complex32, torch.complex64])
def test_sparse_combine_matches_oracle(dtype):
    from dsb200.search import combine_sparse_v4
    dev = torch.device("cuda", 0)
    lut, dense, N, t_rows = _case(5)
    n_fdm, t_lo, t_out = 4, 3, 30
    rng = np.random.default_rng(6)
    shifts = rng.integers(-6, 12, (n_fdm, lut.shape[0])).astype(np.int32)
    csr = build_sparse_cell_csr(torch.from_numpy(lut).to(dev), n_grid=N)
    out = torch.zeros((n_fdm, t_out + 2, N, N // 2 + 1), dtype=dtype, device=dev)
    combine_sparse_v4(torch.from_numpy(dense).to(dev), csr, torch.from_numpy(shifts).to(dev),
                      t_rows=t_rows, t_out_len=t_out, t_lo=t_lo, out=out, out_row0=1,
                      shift_min=int(shifts.min()), shift_max=int(shifts.max()))
    torch.cuda.synchronize()
    want = O.combine_sparse(dense, lut, shifts, t_rows=t_rows, t_out_len=t_out, t_lo=t_lo)
    got = out.to(torch.complex64).cpu().numpy()
    if dtype == torch.complex32:
        want = (want.real.astype(np.float16).astype(np.float32)
                + 1j * want.imag.astype(np.float16).astype(np.float32))
    np.testing.assert_array_equal(got[:, 1:1 + t_out], want.astype(np.complex64))
    assert not got[:, 0].any() and not got[:, -1].any()      # rows outside untouched


@pytest.mark.gpu
def test_gpu_imager_compact_equals_dense():
    from dsb200.search import GpuImager, GpuImagerConfig
    dev = torch.device("cuda", 0)
    lut, dense, N, t_rows = _case(9, n_sb=4, N=64, nfm=300, t_rows=20, t_pad=24)
    G = lut.shape[0]
    # the same streams in the reference's dense layout [G, T, 2, N, N]
    full = np.zeros((G, t_rows, 2, N * N), np.int8)
    for g in range(G):
        cells = np.flatnonzero(lut[g] >= 0)
        full[g, :, :, cells] = dense[g, lut[g, cells], :t_rows]     # (cells, t, 2)
    full = full.reshape(G, t_rows, 2, N, N)
    cfg = GpuImagerConfig(n_grid=N, t_det=16, n_fdm=3, n_chgroup=G, kernel_support=1,
                          cube_dtype=torch.float32, device=dev)
    shifts = torch.tensor([[0, 1, 2, 3], [-1, 0, 2, 4], [3, 2, 1, 0]], dtype=torch.int32,
                          device=dev)
    a = GpuImager.build(cfg)
    got = a.process_cube(streams_cint8=torch.from_numpy(dense).to(dev), time_shifts_gpu=shifts,
                         compact_inv_lut=torch.from_numpy(lut).to(dev),
                         compact_t_stream=t_rows).clone()
    b = GpuImager.build(cfg)
    want = b.process_cube(streams_cint8=torch.from_numpy(full).to(dev), time_shifts_gpu=shifts)
    torch.cuda.synchronize()
    assert torch.equal(got, want)
