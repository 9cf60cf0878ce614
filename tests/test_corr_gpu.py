"""GPU parity: unpack and correlator kernels vs the CPU oracle (bit-exact
for integer codes; fp16 inputs within the reference's own 1e-3)."""

import numpy as np
import pytest
import torch

import dsb_oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dev():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda", 0)


def _raw(npkt, nant, nchan, seed, n_g=1):
    rng = np.random.default_rng(seed)
    return rng.integers(0, 256, n_g * npkt * nant * nchan * 4, dtype=np.uint8)


@pytest.mark.parametrize("dtype", [torch.int8, torch.float16, torch.float32])
def test_unpack_matches_oracle(dev, dtype):
    from dsb200.corr import unpack_int4_split
    npkt, nant, nchan = 24, 40, 72
    raw = _raw(npkt, nant, nchan, 3)
    re, im = unpack_int4_split(raw, device=dev, out_dtype=dtype, scale=0.05,
                               npkt=npkt, nant=nant, nchan=nchan)
    ore, oim = O.unpack_int4_gemm_layout(raw, npkt, nant, nchan)
    if dtype == torch.int8:
        np.testing.assert_array_equal(re.cpu().numpy(), ore)
        np.testing.assert_array_equal(im.cpu().numpy(), oim)
    else:
        want_re = torch.from_numpy(ore.astype(np.float32) * np.float32(0.05)).to(dtype)
        assert torch.equal(re.cpu(), want_re)
        want_im = torch.from_numpy(oim.astype(np.float32) * np.float32(0.05)).to(dtype)
        assert torch.equal(im.cpu(), want_im)


def test_unpack_rejects_wrong_size(dev):
    from dsb200.corr import unpack_int4_split
    with pytest.raises(ValueError, match="fada raw size"):
        unpack_int4_split(np.zeros(100, np.uint8), device=dev, npkt=2, nant=4, nchan=8)


@pytest.mark.parametrize("fuse,csf,nant", [(True, 4, 24), (True, 1, 24), (False, 1, 24),
                                           (True, 2, 21), (False, 1, 128), (True, 8, 128)])
def test_corr_split_int8_exact(dev, fuse, csf, nant):
    """The tensor-core split correlator (kind::f16 on int8 codes) equals
    the oracle's integer sums exactly, including antenna counts that are not
    a multiple of 8 (padded rows) and the largest supported (128)."""
    from dsb200.corr import FastCorrKernel, unpack_int4_split
    npkt, nchan, t_int = 16, 8, 8
    raw = _raw(npkt, nant, nchan, 5)
    re, im = unpack_int4_split(raw, device=dev, out_dtype=torch.int8, npkt=npkt, nant=nant,
                               nchan=nchan)
    k = FastCorrKernel(dev, t_int_fast_native=t_int, nants=nant, nchan=nchan)
    vis = k.compute_split(re, im, fuse_stokes_i=fuse, chan_sum_factor=csf).cpu().numpy()
    ore, oim = O.unpack_int4_gemm_layout(raw, npkt, nant, nchan)
    vr, vi = O.corr_fast(ore, oim, t_int=t_int, csf=csf, fuse_stokes_i=fuse)
    np.testing.assert_array_equal(vis.real.astype(np.int64), vr)
    np.testing.assert_array_equal(vis.imag.astype(np.int64), vi)


@pytest.mark.parametrize("fuse", [True, False])
def test_corr_split_fp32_on_tf32(dev, fuse):
    """float32 voltages run as kind::tf32: integer-valued voltages (the
    codes) correlate exactly; Gaussian voltages agree with the float64
    correlation within the tf32 rounding of the parts (2e-3 of the largest
    visibility)."""
    from dsb200.corr import FastCorrKernel, unpack_int4_split
    npkt, nant, nchan, t_int, csf = 32, 40, 8, 16, 2
    raw = _raw(npkt, nant, nchan, 9)
    re, im = unpack_int4_split(raw, device=dev, out_dtype=torch.float32, scale=1.0, npkt=npkt,
                               nant=nant, nchan=nchan)
    k = FastCorrKernel(dev, t_int_fast_native=t_int, nants=nant, nchan=nchan)
    c = csf if fuse else 1
    vis = k.compute_split(re, im, fuse_stokes_i=fuse, chan_sum_factor=c).cpu().numpy()
    k.check_status()
    ore, oim = O.unpack_int4_gemm_layout(raw, npkt, nant, nchan)
    vr, vi = O.corr_fast(ore, oim, t_int=t_int, csf=c, fuse_stokes_i=fuse)
    np.testing.assert_array_equal(vis.real.astype(np.int64), vr)
    np.testing.assert_array_equal(vis.imag.astype(np.int64), vi)
    rng = np.random.default_rng(4)
    gr = rng.standard_normal(ore.shape).astype(np.float32)
    gi = rng.standard_normal(ore.shape).astype(np.float32)
    vis = k.compute_split(torch.from_numpy(gr).to(dev), torch.from_numpy(gi).to(dev),
                          fuse_stokes_i=fuse, chan_sum_factor=c).cpu().numpy()
    E = (gr.astype(np.float64) + 1j * gi).reshape(nchan, 2, 2, npkt // (t_int // 2),
                                                   t_int // 2, nant)
    V = np.einsum("ctpfkb,ctpfka->fcpba", np.conj(E), E)    # (fv, ch, pol, b, a)
    a_idx, b_idx = O.upper_tri_indices(nant)
    want = V[:, :, :, b_idx, a_idx]                           # (fv, ch, pol, bls)
    if fuse:
        want = want.sum(axis=2).reshape(want.shape[0], nchan // c, c, -1).sum(axis=2)
        want = want.transpose(0, 2, 1)                        # (fv, bls, ch/csf)
    else:
        want = want.transpose(0, 3, 1, 2)                     # (fv, bls, ch, pol)
    assert np.abs(vis - want).max() <= 2e-3 * np.abs(want).max()


def test_corr_split_fp16_within_reference_tolerance(dev):
    from dsb200.corr import FastCorrKernel, unpack_int4_split
    npkt, nant, nchan, t_int, csf = 16, 32, 16, 8, 4
    raw = _raw(npkt, nant, nchan, 6)
    re, im = unpack_int4_split(raw, device=dev, out_dtype=torch.float16, npkt=npkt, nant=nant,
                               nchan=nchan)
    k = FastCorrKernel(dev, t_int_fast_native=t_int, nants=nant, nchan=nchan)
    vis = k.compute_split(re, im, fuse_stokes_i=True, chan_sum_factor=csf).cpu().numpy()
    ore, oim = O.unpack_int4_gemm_layout(raw, npkt, nant, nchan)
    vr, vi = O.corr_fast(ore, oim, t_int=t_int, csf=csf)
    want = (vr + 1j * vi) * 0.0025
    scale = np.abs(want).max()
    assert np.abs(vis - want).max() <= 1e-3 * scale


@pytest.mark.parametrize("nant,nchan,csf,t_int,npkt,n_g", [
    (96, 64, 16, 8, 16, 1),     # DSA-110 antennas, 24-channel-style summed groups
    (96, 32, 8, 8, 12, 2),      # two chgroup pages in one launch
    (16, 32, 1, 8, 32, 1),      # small array, no channel sum (scalar loader)
    (48, 16, 4, 16, 16, 1),     # sub-array, t_int 16
    (64, 24, 2, 8, 8, 1),       # csf not a multiple of 4 -> scalar loader
])
@pytest.mark.parametrize("layout", ["tbc", "bct"])
def test_corr_tc_matches_oracle(dev, nant, nchan, csf, t_int, npkt, n_g, layout):
    from dsb200.corr import FastCorrKernel
    raw = _raw(npkt, nant, nchan, 11 + nant, n_g)
    k = FastCorrKernel(dev, t_int_fast_native=t_int, nants=nant, nchan=nchan)
    r = torch.from_numpy(raw).to(dev)
    if n_g > 1:
        r = r.view(n_g, npkt, nant, nchan, 2, 2)
    out = k.compute_raw(r, chan_sum_factor=csf, layout=layout, max_ctas=7)
    torch.cuda.synchronize()
    assert int(k._last_status.item()) == 0
    got = out.cpu().numpy()
    if n_g == 1:
        got = got[None]
    page = npkt * nant * nchan * 4
    for g in range(n_g):
        vr, vi = O.corr_fast_from_raw(raw[g * page:(g + 1) * page], npkt=npkt, nant=nant,
                                      nchan=nchan, t_int=t_int, csf=csf)
        gg = got[g] if layout == "tbc" else got[g].transpose(2, 0, 1)
        np.testing.assert_array_equal(gg.real.astype(np.int64), vr)
        np.testing.assert_array_equal(gg.imag.astype(np.int64), vi)


def test_corr_tc_full_grid_of_ctas(dev):
    """Default grid (one CTA per SM) on a block with many more units than SMs."""
    from dsb200.corr import FastCorrKernel
    npkt, nant, nchan, csf, t_int = 64, 96, 96, 16, 8
    raw = _raw(npkt, nant, nchan, 77)
    k = FastCorrKernel(dev, t_int_fast_native=t_int, nants=nant, nchan=nchan)
    out = k.compute_raw(torch.from_numpy(raw).to(dev), chan_sum_factor=csf)
    torch.cuda.synchronize()
    vr, vi = O.corr_fast_from_raw(raw, npkt=npkt, nant=nant, nchan=nchan, t_int=t_int, csf=csf)
    got = out.cpu().numpy()
    np.testing.assert_array_equal(got.real.astype(np.int64), vr)
    np.testing.assert_array_equal(got.imag.astype(np.int64), vi)
