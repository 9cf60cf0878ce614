"""Wire encoding of dedispersed rows (transport/tx.py:825-873) and the
calibrated per-(chgroup, time) cint8 combine (fused_combine_cuda.py:431-505).

* CPU: the oracle's encoder equals the reference's ``_encode_rows`` on the
  seeded rows of ``tests/golden/make_golden.py`` (exact rounding ties, an
  all-zero tile, float16 overflow included), bit for bit.
* GPU: ``dsb_encode_rows`` equals the oracle bit for bit; the calibrated
  dense combine with per-tile scales equals the oracle's float32 fma
  restatement bit for bit, full grid and half spectrum.
"""

import os
import sys

import numpy as np
import pytest
import torch

import dsb_oracle as O

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
import make_golden as MG  # noqa: E402


def test_oracle_encode_rows_matches_reference(golden_dir):
    z = np.load(os.path.join(golden_dir, "transport.npz"))
    rows = MG.transport_rows()
    q16, s16 = O.encode_rows(rows, 16)
    assert np.array_equal(q16, z["q16"]) and np.array_equal(s16.view(np.uint32),
                                                            z["s16"].view(np.uint32))
    with np.errstate(over="ignore"):
        q32, s32 = O.encode_rows(rows, 32)
    assert np.array_equal(q32.view(np.uint16), z["q32"].view(np.uint16))
    assert np.array_equal(s32, z["s32"])
    # the tie tiles really exercise round-half-even
    assert np.any(rows[7].real % 1 == 0.5) and s16[7] == np.float32(1.0)


@pytest.mark.gpu
def test_encode_rows_gpu_matches_oracle():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from dsb200.transport import encode_rows
    dev = torch.device("cuda", 0)
    rng = np.random.default_rng(3)
    cases = [MG.transport_rows(),
             (rng.standard_normal((40, 2500)) * 50 + 1j * rng.standard_normal((40, 2500))
              ).astype(np.complex64),
             np.zeros((3, 0), np.complex64)]
    for rows in cases:
        for bits in (16, 32):
            with np.errstate(over="ignore"):
                wq, ws = O.encode_rows(rows, bits)
            gq, gs = encode_rows(torch.from_numpy(rows).to(dev), bits)
            gq, gs = gq.cpu().numpy(), gs.cpu().numpy()
            if bits == 16:
                assert np.array_equal(gq, wq)
            else:
                assert np.array_equal(gq.view(np.uint16), wq.view(np.uint16))
            assert np.array_equal(gs.view(np.uint32), ws.view(np.uint32))
    # a strided view (one tile of every other row) encodes as its copy
    rows = torch.from_numpy(cases[1]).to(dev)
    gq, gs = encode_rows(rows[::2], 16)
    wq, ws = O.encode_rows(cases[1][::2], 16)
    assert np.array_equal(gq.cpu().numpy(), wq)


@pytest.mark.gpu
@pytest.mark.parametrize("half", [False, True])
def test_per_tile_dequant_combine_matches_oracle(half):
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from dsb200.search import fused_dequant_combine_per_fdm, fused_dequant_combine_per_fdm_half
    dev = torch.device("cuda", 0)
    rng = np.random.default_rng(11)
    G, T, N, t_det, t_lo = 4, 10, 16, 9, 2
    q = rng.integers(-128, 128, (G, T, 2, N, N)).astype(np.int8)
    shifts = rng.integers(-2, 3, G).astype(np.int32)
    scales = (10.0 ** rng.uniform(-2, 2, (G, T))).astype(np.float32)
    scales[1, 3] = 0.0                      # a skipped (g, t) slot
    off_re = (rng.standard_normal((G, T)) * 0.1).astype(np.float32)
    off_im = (rng.standard_normal((G, T)) * 0.1).astype(np.float32)
    nw = N // 2 + 1 if half else N
    out = torch.zeros((t_det - t_lo, N, nw), dtype=torch.complex64, device=dev)
    d = lambda a: torch.from_numpy(a).to(dev)  # noqa: E731
    fn = fused_dequant_combine_per_fdm_half if half else fused_dequant_combine_per_fdm
    fn(d(q), d(shifts), out, scales=d(scales), offsets_re=d(off_re), offsets_im=d(off_im),
       t_lo=t_lo, fftshift=True)
    want = O.combine_dequant(q, shifts, scales, off_re, off_im, t_det, t_lo, half=half)
    np.testing.assert_array_equal(out.cpu().numpy(), want)
    # per-chgroup scales [G] take the same path with one value per chgroup
    out.zero_()
    fn(d(q), d(shifts), out, scales=d(scales[:, 0].copy()), offsets_re=d(off_re[:, 0].copy()),
       offsets_im=d(off_im[:, 0].copy()), t_lo=t_lo, fftshift=True)
    want = O.combine_dequant(q, shifts, scales[:, 0], off_re[:, 0], off_im[:, 0], t_det, t_lo,
                             half=half)
    np.testing.assert_array_equal(out.cpu().numpy(), want)


def test_oracle_decode_cint8_within_half_step():
    """Receiver side: float32(scale * q) is within half a quantisation step
    of every part (no part clips: |x| <= amax = 127 scale)."""
    rows = MG.transport_rows()
    q, s = O.encode_rows(rows, 16)
    back = O.decode_cint8(q, s)
    err = np.maximum(np.abs(back.real - rows.real), np.abs(back.imag - rows.imag))
    assert np.all(err <= 0.5 * s[:, None] * (1 + 1e-6))


@pytest.mark.gpu
def test_ring_encode_cint8_matches_oracle():
    """dsb_ring_encode_cint8 == the oracle encoder per (chgroup, coarse DM,
    time) row, bit for bit: payload at slot (t0 + t + shift2) mod depth, the
    pitch padding zeroed (and ignored in X), the row's scale beside it;
    all-zero and tie rows included."""
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from dsb200 import _lib
    dev = torch.device("cuda", 0)
    rng = np.random.default_rng(21)
    G, n_dm, n_t, t0 = 3, 2, 5, 17
    pitch = np.array([8, 12, 4], np.int32)
    nfill = np.array([7, 12, 3], np.int32)
    shift2 = rng.integers(0, 10, G * n_dm).astype(np.int32)
    depth = (shift2 + n_t + 3).astype(np.int32)
    gd_pitch = np.repeat(pitch, n_dm).astype(np.int64)
    x_base = np.concatenate([[0], np.cumsum(n_t * gd_pitch)]).astype(np.int64)
    seg_base = np.concatenate([[0], np.cumsum(depth * gd_pitch)]).astype(np.int64)
    sc_base = np.concatenate([[0], np.cumsum(depth)]).astype(np.int64)
    X = np.full(int(x_base[-1]), 1e6 + 1e6j, np.complex64)   # padding: must be ignored
    tie = MG.transport_rows()[7]
    rows = {}
    for gd in range(G * n_dm):
        g = gd // n_dm
        nf, pt = int(nfill[g]), int(pitch[g])
        for t in range(n_t):
            r = (rng.standard_normal(nf) * 30 + 1j * rng.standard_normal(nf) * 3).astype(
                np.complex64)
            if (gd, t) == (1, 2):
                r[:] = 0
            if (gd, t) == (2, 4):
                r = tie[:nf].copy()
            rows[gd, t] = r
            X[x_base[gd] + t * pt: x_base[gd] + t * pt + nf] = r
    D = torch.full((int(seg_base[-1]),), 0x5555, dtype=torch.int16, device=dev)
    scales = torch.full((int(sc_base[-1]),), -1.0, dtype=torch.float32, device=dev)
    st = _lib.status_word(dev)
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)  # noqa: E731
    keep = [d(X), d(x_base[:-1]), d(pitch), d(nfill), d(shift2), d(seg_base[:-1]), d(depth),
            d(sc_base[:-1])]
    _lib.check(_lib.lib().dsb_ring_encode_cint8(
        _lib.ptr(keep[0]), _lib.ptr(keep[1]), n_t, _lib.ptr(keep[2]), _lib.ptr(keep[3]), G, n_dm,
        _lib.ptr(keep[4]), t0, _lib.ptr(D), _lib.ptr(keep[5]), _lib.ptr(keep[6]),
        _lib.ptr(scales), _lib.ptr(keep[7]), _lib.ptr(st), _lib.stream_of(dev)), "ring encode")
    torch.cuda.synchronize()
    _lib.check_status(st, "ring encode")
    Dh = D.cpu().numpy().view(np.int8).reshape(-1, 2)
    sh = scales.cpu().numpy()
    for (gd, t), r in rows.items():
        g = gd // n_dm
        nf, pt = int(nfill[g]), int(pitch[g])
        wq, ws = O.encode_rows(r[None], 16)
        slot = (t0 + t + int(shift2[gd])) % int(depth[gd])
        e0 = int(seg_base[gd]) + slot * pt
        assert np.array_equal(Dh[e0:e0 + nf], wq[0])
        assert np.all(Dh[e0 + nf:e0 + pt] == 0)
        assert sh[int(sc_base[gd]) + slot].view(np.uint32) == ws[0].view(np.uint32)
