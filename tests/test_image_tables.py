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


def _emulate(T, slices, N, fftshift):
    fold = 4
    LC, NC = N // fold, N // 2
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
    q = (T.sq & 3).astype(np.int64)
    pk = ((T.sq >> 2) & 1).astype(np.int64)
    par = ((T.sq >> 3) & 1).astype(np.int64)
    C1 = int(round(np.sqrt(LC)))
    col = np.repeat(np.arange(NC * C1), np.diff(T.so)) // C1
    slot = col * LC + ((T.sq >> 4) & (LC - 1)).astype(np.int64)
    for p in range(fold):
        rot = q * p + pk + (2 * par if fftshift else 0)
        y = np.zeros(NC * LC, np.complex128)
        np.add.at(y, slot, S * (1j) ** (rot % 4))
        y = y.reshape(NC, LC).T                       # [n', col]
        y = y * twN[(np.arange(LC) * p) % N][:, None]
        X = np.fft.ifft(y, axis=0) * LC               # sum_n' y W_LC^(+n' m)
        A[p::fold, :] = X
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


@pytest.mark.parametrize("N,n_g,fftshift", [(64, 3, True), (64, 2, False), (256, 4, True)])
def test_image_tables_restate_irfft2(N, n_g, fftshift):
    pats = _patterns(N, n_g, seed=7 + N)
    T = build_image_tables(pats, N)
    rng = np.random.default_rng(N + n_g)
    slices = [rng.standard_normal(p.ix_row.size) + 1j * rng.standard_normal(p.ix_row.size)
              for p in pats]
    got = _emulate(T, slices, N, fftshift)
    want = _definition(pats, slices, N, fftshift)
    assert np.abs(got - want).max() <= 1e-12 * max(1.0, np.abs(want).max())


def test_image_tables_layout():
    N = 256
    pats = _patterns(N, 3, seed=3)
    T = build_image_tables(pats, N)
    LC = N // 4
    assert T.so[0] == 0 and T.so[-1] == T.n_s and np.all(np.diff(T.so) >= 0)
    C1 = 8
    assert T.so.size == N // 2 * C1 + 1
    assert sorted(T.corder.tolist()) == list(range(N // 2))
    # lane j = n' mod C1 of column w' owns exactly the entries of its run
    lane = np.repeat(np.arange(N // 2 * C1), np.diff(T.so)) % C1
    n1 = (T.sq >> 4) & (LC - 1)
    assert np.array_equal(n1 % C1, lane)
    # "last" marks the final entry of each (column, n') run of equal slots
    col = np.repeat(np.arange(N // 2 * C1), np.diff(T.so)) // C1
    slot = col * LC + n1
    last = np.append(slot[1:] != slot[:-1], True)
    assert np.array_equal(((T.sq >> 10) & 1).astype(bool), last)
    assert T.cell_base[-1] == T.c_meta.size and np.all(T.cell_base % 32 == 0)
    for g, p in enumerate(pats):                # padding after each chgroup's run
        assert np.all(T.c_meta[T.cell_base[g] + p.ix_row.size:T.cell_base[g + 1]] == 0xFFFFFFFF)
    assert T.n_s <= LC * (N // 2 + 2)          # fits the kernel's shared buffer
    # every S entry is hit by at least one pattern cell
    hit = np.zeros(T.n_s, bool)
    live = T.c_meta != 0xFFFFFFFF
    hit[T.c_meta[live] & 0xFFFF] = True
    hit[T.c2[:, 1] & 0xFFFF] = True
    assert hit.all()
