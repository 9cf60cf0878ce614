"""Tables of the detector's Layer-2 score samples (CPU).

The streaming detector (detector/forward.py:1425-1530) estimates each
kernel's noise from ``m`` score samples at flat indices over the cube's
interior ``[n_out, F, H, W]``, drawn per kernel k by ``torch.randint`` from a
generator seeded k, the cells outside the edge mask excluded.  The CUDA
detector finds its entries through ``Layer2Samples``: entries {cell, time,
k, slot} sorted by (cell, time) and the first entry of every 256-cell block.
These tests check those tables against the oracle's draw, and the oracle's
Layer-2 state against the library's (itself pinned to the reference).
"""

import numpy as np
import torch

import dsb_oracle as O
from dsb200.noise import Layer2State
from dsb200.search import Layer2Samples


def _tables(n_out=40, F=3, N=32, m=500, K=5):
    mask = O.edge_mask(N, kernel_support=1)
    l2 = Layer2Samples(n_kernels=K, m=m, n_out=n_out, n_fdm=F, npix=N * N,
                       active=mask.reshape(-1) != 0, device="cpu")
    return l2, mask, (n_out, F, N, m, K)


def test_entries_are_the_oracle_draw_inside_the_mask():
    l2, mask, (n_out, F, N, m, K) = _tables()
    idx = O.layer2_sample_index(K, m, n_out * F * N * N)
    fhw = F * N * N
    want = set()
    for k in range(K):
        for slot, i in enumerate(idx[k].tolist()):
            cell, t = i % fhw, i // fhw
            if mask.reshape(-1)[cell % (N * N)] != 0:
                want.add((cell, t, k, slot))
    got = {tuple(r) for r in l2.entries.tolist()}
    assert got == want
    # masked-out slots stay NaN for the clipped std to drop
    written = np.zeros((K, m), bool)
    written[l2.entries[:, 2], l2.entries[:, 3]] = True
    assert np.isnan(l2.samples.numpy()[~written]).all()
    assert written.sum() == len(want)


def test_entries_sorted_and_block_offsets():
    l2, mask, (n_out, F, N, m, K) = _tables()
    ent = l2.entries
    key = ent[:, 0] * (n_out + 1) + ent[:, 1]
    assert np.all(np.diff(key) >= 0)
    off = l2.d_off.numpy()
    assert off.size == F * N * N // 256 + 1 and off[0] == 0 and off[-1] == len(ent)
    for gb in range(off.size - 1):
        cells = ent[off[gb]:off[gb + 1], 0]
        assert np.all((cells >= 256 * gb) & (cells < 256 * (gb + 1)))
    assert l2.d_ent.dtype.itemsize == 4 and l2.d_ent.shape == (len(ent), 4)


def test_oracle_layer2_state_follows_the_library_state():
    """The oracle's float32 restatement of the default Layer-2 update (seed
    sqrt(width), zero keeps, Welford burn-in, then the EMA) against the
    library's state on a seeded sequence of estimates through both phases."""
    widths = [1, 2, 4, 8, 16]
    rng = np.random.default_rng(3)
    ora = O.Layer2State(widths, 0.5, tau_s=2.0, n_burnin=4)
    lib = Layer2State(len(widths), cube_cadence_s=0.5, tau_s=2.0, n_burnin=4)
    lib._s_k.copy_(torch.tensor([float(np.sqrt(w)) for w in widths], dtype=torch.float32))
    for i in range(12):
        sig = (np.sqrt(widths) * rng.uniform(0.8, 1.2, len(widths))).astype(np.float32)
        if i == 5:
            sig[2] = 0.0
        a = ora.update(sig)
        b, _ = lib.update_and_query(per_kernel_sigma=torch.from_numpy(sig))
        np.testing.assert_allclose(a, b.numpy(), rtol=2e-7)
