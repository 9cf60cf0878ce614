"""Tables of the fused combine + FFT image kernel (CPU).

The kernel's algorithm is restated here in numpy from the same tables it
reads; the result must equal the definition it replaces:

* the Hermitian half spectrum 0.5 (G[u, w] + conj G[-u, -w]), w in [0, N/2],
  with the fftshift checkerboard (-1)^(u+w)
  (image/fused_combine_cuda.py:560-620); then
* numpy.fft.irfft2 (image/imager_gpu.py:590).

So this test checks two things without a GPU: the table construction, and
the decimation-in-frequency fold with the packing of columns 0 and N/2.
"""

import types

import numpy as np
import pytest

import dsb_oracle as O
from dsb200.pipeline import build_image_tables


def _patterns(N, n_g, seed):
    """Seeded T-layout uv patterns of n_g chgroups on an N x N grid."""
    from dsb200 import synth
    band = O.Band(n_g, 32, 1.49875, 0.25 / 8192 * 16, 0)
    e, n = synth.t_layout(24, seed=seed)
    cell = O.top_of_band_cell_lambda(e, n, band, N)
    pats = []
    for g in range(n_g):
        r, c = O.build_pattern(e, n, band, g, n_grid=N, csf=4, cell_lambda=cell)
        pats.append(types.SimpleNamespace(ix_row=r, ix_col=c))
    return pats


def _meta_fields(T, m):
    """(column, n', q, last, rotation bits) of entry metadata m in the table's
    form: 16-bit w' | n' << 7 | q << 13 | last << 15 with the rotation bits in
    srot, or 32-bit w' | n' << 8 | q << 14 | last << 17 | rot << 18."""
    m = np.asarray(m, np.int64)
    if T.meta_bits == 16:
        return m & 127, (m >> 7) & 63, (m >> 13) & 3, (m >> 15) & 1, None
    return m & 255, (m >> 8) & 63, (m >> 14) & 7, (m >> 17) & 1, (m >> 18) & 3


def _emulate(T, slices, N, fftshift):
    """The kernel's steps, from its tables: combine into S, per-thread ranges
    with the static rotation, the per-pass fold into slots, dense columns
    transformed from their occupied slots only, constant columns broadcast,
    then the row transforms.  Slots no thread writes in a pass are NaN, so a
    read of one shows up in the result."""
    fold = T.fold
    LC, NC = N // fold, N // 2
    epv = T.gmeta.shape[2]
    S = np.zeros(T.n_s, np.complex128)
    for g, v in enumerate(slices):
        m = T.c_meta[T.cell_base[g]:T.cell_base[g] + v.size].astype(np.int64)
        vv = np.where((m >> 16) & 1, np.conj(v), v)
        np.add.at(S, m & 0xFFFF, vv)
    for kg, sc in T.c2.astype(np.int64):
        v = slices[(kg >> 16) & 63][kg & 0xFFFF]
        S[sc & 0xFFFF] += np.conj(v) if (sc >> 16) & 1 else v
    A = np.zeros((N, NC), np.complex128)
    twN = np.exp(2j * np.pi * np.arange(N) / N)
    wf = np.exp(2j * np.pi * np.arange(fold) / fold)      # W_FOLD^k
    n_thr = T.thr_b.size - 1
    compact = T.fold_code is not None
    for p in range(fold):
        # the column buffer with its row pitch NC + 2 (the compact tables of
        # the 32-bit form address it as n' * (NC + 2) + w')
        bufp = np.full((LC, NC + 2), np.nan, np.complex128)
        for t in range(n_thr):
            b, e = int(T.thr_b[t]), int(T.thr_b[t + 1])
            acc = 0j
            si = int(T.thr_slot[t]) if compact else 0
            for i in range(e - b):
                col, npr, q, last, rot = _meta_fields(T, int(T.gmeta[i // epv, t, i % epv]))
                if compact:   # the fold reads q and last from the nibble table
                    code = (int(T.fold_code[i // 8, t]) >> (4 * (i % 8))) & 15
                    q, last = code & 7, code >> 3
                if compact:   # the copy into TMEM reads the rotation table
                    rot = (int(T.fold_rot[t, i // 16]) >> (2 * (i % 16))) & 3
                sr = (int(T.srot[t]) >> (2 * i)) & 3 if rot is None else int(rot)
                stat = (1j) ** ((sr & 1) + (2 if (sr & 2) and fftshift else 0))
                acc += S[b + i] * stat * wf[(int(q) * p) % fold]
                if last:
                    if compact:
                        off = int(T.slot_off[si])
                        si += 1
                        bufp.reshape(-1)[off] = acc
                    else:
                        bufp[int(npr), int(col)] = acc
                    acc = 0j
            if compact:
                assert si == int(T.thr_slot[t + 1])
        buf = bufp[:, :NC]
        out = np.full((LC, NC), np.nan, np.complex128)
        for col, occ in zip(T.dcols.tolist(), T.dmask.tolist()):
            y = np.array([buf[n, col] if (occ >> n) & 1 else 0j for n in range(LC)])
            y = y * twN[(np.arange(LC) * p) % N]
            out[:, col] = np.fft.ifft(y) * LC          # sum_n' y W_LC^(+n' m)
        for kc in T.kcols.tolist():
            out[:, kc & 0xFFFF] = buf[0, kc & 0xFFFF] if kc >> 16 else 0j
        A[p::fold, :] = out
    img = np.zeros((N, N))
    for x in range(N):
        Y = np.zeros(N, np.complex128)
        Y[0] = A[x, 0].real
        Y[N // 2] = A[x, 0].imag
        Y[1:N // 2] = A[x, 1:N // 2]
        Y[N // 2 + 1:] = np.conj(A[x, 1:N // 2][::-1])
        img[x] = (np.fft.ifft(Y) * N).real
    return img * 0.5 / N ** 2


def _definition(pats, slices, N, fftshift):
    G = np.zeros((N, N), np.complex128)
    for p, v in zip(pats, slices):
        np.add.at(G, (p.ix_row.astype(np.int64), p.ix_col.astype(np.int64)), v)
    u = np.arange(N)[:, None]
    w = np.arange(N // 2 + 1)[None, :]
    H = 0.5 * (G[u, w] + np.conj(G[(N - u) % N, (N - w) % N]))
    if fftshift:
        H = H * np.where((u + w) % 2 == 1, -1.0, 1.0)
    return np.fft.irfft2(H, s=(N, N))


@pytest.mark.parametrize("N,n_g,fftshift", [(64, 3, True), (64, 2, False), (256, 4, True),
                                             (512, 4, True)])
def test_image_tables_restate_irfft2(N, n_g, fftshift):
    pats = _patterns(N, n_g, seed=7 + N)
    T = build_image_tables(pats, N)
    rng = np.random.default_rng(N + n_g)
    slices = [rng.standard_normal(p.ix_row.size) + 1j * rng.standard_normal(p.ix_row.size)
              for p in pats]
    got = _emulate(T, slices, N, fftshift)
    want = _definition(pats, slices, N, fftshift)
    assert np.abs(got - want).max() <= 1e-12 * max(1.0, np.abs(want).max())


@pytest.mark.parametrize("N", [256, 512])
def test_image_tables_layout(N):
    from dsb200.pipeline import image_geometry
    pats = _patterns(N, 3, seed=3)
    T = build_image_tables(pats, N)
    geo = image_geometry(N)
    assert T.fold == geo["fold"] and T.meta_bits == geo["meta_bits"]
    LC, NC = N // T.fold, N // 2
    n_thr, cap = geo["threads"], geo["max_entries"]
    epv = 8 if T.meta_bits == 16 else 4
    assert T.thr_b.size == n_thr + 1 and T.thr_b[0] == 0 and T.thr_b[-1] == T.n_s
    cnt = np.diff(T.thr_b)
    assert np.all(cnt >= 0) and cnt.max() <= cap
    assert T.gmeta.shape == (cap // epv, n_thr, epv)
    # entries in S order: slot (w', n') of each, and "last" on its final entry
    owner = np.repeat(np.arange(n_thr), cnt)
    idx = np.arange(T.n_s) - T.thr_b[owner]
    col, npr, q, last_bit, _ = _meta_fields(T, T.gmeta[idx // epv, owner, idx % epv])
    slot = col * LC + npr
    assert np.all(np.diff(slot) >= 0)                    # S is sorted by slot
    last = np.append(slot[1:] != slot[:-1], True)
    assert np.array_equal(last_bit.astype(bool), last)
    # every thread range ends on a slot boundary (whole slots per thread)
    ends = T.thr_b[1:][cnt > 0] - 1
    assert np.all(last_bit[ends] == 1)
    # columns: each packed column once; dense masks are the occupied n'
    cols = np.concatenate([T.dcols, T.kcols & 0xFFFF])
    assert sorted(cols.tolist()) == list(range(NC))
    occ = {}
    for sl in np.unique(slot).tolist():
        occ[sl // LC] = occ.get(sl // LC, 0) | (1 << (sl % LC))
    for c, msk in zip(T.dcols.tolist(), T.dmask.tolist()):
        assert msk == occ[c] and msk & ~1
    for kc in T.kcols.tolist():
        assert occ.get(kc & 0xFFFF, 0) == (1 if kc >> 16 else 0)
    assert T.cell_base[-1] == T.c_meta.size and np.all(T.cell_base % 64 == 0)
    if T.meta_bits == 32:
        # the fold's compact tables: nibbles q | last << 3, slots in S order
        code = (T.fold_code[idx // 8, owner].astype(np.int64) >> (4 * (idx % 8))) & 15
        assert np.array_equal(code & 7, q) and np.array_equal(code >> 3, last_bit)
        starts = np.flatnonzero(np.r_[True, slot[1:] != slot[:-1]])
        n_sl = starts.size
        assert T.thr_slot.size == n_thr + 1 and T.thr_slot[-1] == n_sl
        assert np.all(np.diff(T.thr_slot) >= 0)
        assert np.array_equal(T.thr_slot[:-1], np.searchsorted(starts, T.thr_b[:-1]))
        assert np.array_equal(T.slot_off[:n_sl], npr[starts] * (NC + 2) + col[starts])
        assert T.slot_off.size % 8 == 0 and n_sl <= LC * NC
        # device bytes: gmeta, nibbles, thr_slot padded to 16 bytes, slot_off
        nb = T.gmeta_device_bytes().size
        assert nb == (T.gmeta.nbytes + T.fold_code.nbytes + -(-(n_thr + 1) // 4) * 16 +
                      T.fold_rot.nbytes + T.slot_off.nbytes)
        _, _, _, _, rot = _meta_fields(T, T.gmeta[idx // epv, owner, idx % epv])
        rot_c = (T.fold_rot[owner, idx // 16].astype(np.int64) >> (2 * (idx % 16))) & 3
        assert np.array_equal(rot_c, rot)
    for g, p in enumerate(pats):                # padding after each chgroup's run
        assert np.all(T.c_meta[T.cell_base[g] + p.ix_row.size:T.cell_base[g + 1]] == 0xFFFFFFFF)
    assert T.n_s <= geo["s_capacity"]          # fits the kernel's shared S arrays
    # every S entry is hit by at least one pattern cell
    hit = np.zeros(T.n_s, bool)
    live = T.c_meta != 0xFFFFFFFF
    hit[T.c_meta[live] & 0xFFFF] = True
    hit[T.c2[:, 1] & 0xFFFF] = True
    assert hit.all()


def test_metric_configuration_tables_fit_and_restate_irfft2():
    """The 512^2 tables of the metric configuration's array (96 antennas on
    the bench's seeded T layout, 16 x 384 channels summed 16 to a subband)
    fit the kernel (S capacity, entries per thread, slots of the compact fold
    tables), and the kernel's steps restated from them give irfft2."""
    from dsb200 import synth
    from dsb200.pipeline import image_geometry
    N, csf = 512, 16
    e, n = synth.t_layout(96, seed=11)
    band = O.REFERENCE_BAND
    cell = O.top_of_band_cell_lambda(e, n, band, N)
    pats = []
    for g in range(band.n_chgroup):
        r, c = O.build_pattern(e, n, band, g, n_grid=N, csf=csf, cell_lambda=cell)
        pats.append(types.SimpleNamespace(ix_row=r, ix_col=c))
    T = build_image_tables(pats, N)
    geo = image_geometry(N)
    assert 20000 < T.n_s <= geo["s_capacity"]
    assert np.diff(T.thr_b).max() <= geo["max_entries"]
    assert int(T.thr_slot[-1]) <= (N // T.fold) * (N // 2)
    rng = np.random.default_rng(96)
    slices = [rng.standard_normal(p.ix_row.size) + 1j * rng.standard_normal(p.ix_row.size)
              for p in pats]
    got = _emulate(T, slices, N, True)
    want = _definition(pats, slices, N, True)
    assert np.abs(got - want).max() <= 1e-12 * max(1.0, np.abs(want).max())
