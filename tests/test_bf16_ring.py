"""BF16 storage form and cint8 wire form of the stage-2 ring (CPU).

* The oracle's bfloat16 rounding equals torch's float32 -> bfloat16
  conversion (nearest, ties to even), exact ties and large magnitudes
  included.
* Stated error of the precision form: images of the oracle pipeline with
  the BF16 ring against the same pipeline with the complex64 ring, on the
  same seeded raw pages.  The bound is 1e-2 of the image peak (the BF16
  path tolerance); the measured value is printed.
"""

import numpy as np
import torch

import dsb_oracle as O


def test_round_bf16_matches_torch():
    rng = np.random.default_rng(4)
    x = np.concatenate([
        rng.standard_normal(20000).astype(np.float32) * 1e3,
        rng.standard_normal(2000).astype(np.float32) * 1e30,
        np.float32([0.0, -0.0, 1.0, -1.0, 3.0e38, -3.0e38, np.inf, -np.inf]),
    ])
    # exact ties: the dropped 16 bits are 0x8000, kept lowest bit both 0 and 1
    hi = (rng.integers(0, 1 << 15, 4000, dtype=np.uint64) << np.uint64(17)) | \
        (rng.integers(0, 2, 4000, dtype=np.uint64) << np.uint64(16))
    ties = ((hi | np.uint64(0x8000)) & np.uint64(0x7F7FFFFF)).astype(np.uint32).view(np.float32)
    x = np.concatenate([x, ties, -ties])
    want = torch.from_numpy(x).to(torch.bfloat16).to(torch.float32).numpy()
    got = O.round_bf16(x)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    z = (x[:1000] + 1j * x[1000:2000]).astype(np.complex64)
    zr = O.round_bf16_complex(z)
    assert np.array_equal(zr.real, O.round_bf16(z.real)) and np.array_equal(
        zr.imag, O.round_bf16(z.imag))


def _small_setup(n_blocks=6):
    from dsb200 import synth
    from dsb200.constants import band_from_edges
    band = band_from_edges(2, 32, 1.49875, 1.31125)
    ob = O.Band(band.n_chgroup, band.nchan, band.f0_ghz, band.dnu_ghz, band.ch0)
    nant, npkt, N = 16, 256, 64
    e, n = synth.t_layout(nant, seed=5)
    cell = O.top_of_band_cell_lambda(e, n, ob, N)
    coarse = np.linspace(0, 30, 4)
    fine = np.repeat(coarse, 2) + np.tile([-1.875, 1.875], 4)
    fine = np.maximum(fine, 0)
    f2c = np.repeat(np.arange(4), 2)
    bursts = [synth.Burst(dm=20.0, t0_native=700, width_native=16, amp=1.0, dl=3, dm_pix=-5)]
    blocks = [synth.make_block(band=band, nant=nant, npkt=npkt, block_index=b, seed=9,
                               antpos_e=e, antpos_n=n, bursts=bursts, cell_lambda=cell, n_grid=N)
              for b in range(n_blocks)]
    kw = dict(nant=nant, npkt_block=npkt, t_int=8, csf=4, n_grid=N, coarse_dm=coarse,
              fine_dm=fine, fine_to_coarse=f2c, log_max_width=2, threshold=6.0)
    return ob, e, n, blocks, kw


def test_bf16_ring_image_error_against_complex64():
    ob, e, n, blocks, kw = _small_setup()
    k32, k16 = {}, {}
    O.run_pipeline(blocks, ob, e, n, chunk=32, sky_window=2, sky_warmup=1, keep=k32, **kw)
    O.run_pipeline(blocks, ob, e, n, chunk=32, sky_window=2, sky_warmup=1, keep=k16,
                   ring_dtype="bf16", **kw)
    # the BF16 streams are the complex64 ones rounded part by part
    for g in range(len(k32["D1"])):
        for d in range(len(k32["D1"][g])):
            a = k32["D1"][g][d].astype(np.complex64)
            np.testing.assert_array_equal(k16["D1"][g][d].astype(np.complex64),
                                          O.round_bf16_complex(a))
    assert len(k32["images"]) == len(k16["images"]) > 0
    err = max(np.abs(a - b).max() / np.abs(a).max()
              for a, b in zip(k32["images"], k16["images"]))
    print(f"BF16 ring: max image error {err:.3e} of the image peak")
    assert 0 < err <= 1e-2


def test_cint8_ring_image_error_against_complex64():
    """Stated error of the cint8 wire form on the same pages: every stream
    row is the complex64 row through the wire encoder and back, and the
    images stay within 2e-2 of the image peak of the complex64 ones (the
    measured value is printed)."""
    ob, e, n, blocks, kw = _small_setup()
    k32, k8 = {}, {}
    O.run_pipeline(blocks, ob, e, n, chunk=32, sky_window=2, sky_warmup=1, keep=k32, **kw)
    O.run_pipeline(blocks, ob, e, n, chunk=32, sky_window=2, sky_warmup=1, keep=k8,
                   ring_dtype="cint8", **kw)
    for g in range(len(k32["D1"])):
        for d in range(len(k32["D1"][g])):
            a = k32["D1"][g][d].astype(np.complex64)
            np.testing.assert_array_equal(k8["D1"][g][d].astype(np.complex64),
                                          O.decode_cint8(*O.encode_rows(a, 16)))
    assert len(k32["images"]) == len(k8["images"]) > 0
    err = max(np.abs(a - b).max() / np.abs(a).max()
              for a, b in zip(k32["images"], k8["images"]))
    print(f"cint8 ring: max image error {err:.3e} of the image peak")
    assert 0 < err <= 2e-2
