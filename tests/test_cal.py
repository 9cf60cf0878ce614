"""Per-antenna complex gains on split voltages (hot-path row a3):
apply_cal_split (services/slow_corr_kernel.py:417-528),
make_cal_broadcast_tensors (:531-569) and compute_dec_phase
(cal/cal_loader.py:209-290).

* CPU: the oracle equals the reference's eager float16 / float32 output,
  per-channel and broadcast gains, bit for bit; the DEC phase equals the
  reference's complex128 table bit for bit (hash); the host-side tensors
  and the argument checks of the drop-in.
* GPU: dsb_cal_apply equals the reference's output bit for bit, equals
  torch's own eager float16 ops on the full GEMM layout (384 x 2 x 2 x 2048
  x 96), takes the one-antenna path for odd antenna counts, and the
  correlator of calibrated voltages gives conj(G_i) G_j times the
  visibilities of the raw ones (float16 tolerance).
"""

import hashlib
import os
import sys

import numpy as np
import pytest
import torch

import dsb_oracle as O

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
import make_golden as MG  # noqa: E402


@pytest.fixture(scope="module")
def golden(golden_dir):
    return np.load(os.path.join(golden_dir, "cal.npz"))


def _sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


@pytest.mark.parametrize("name,dt", [("f16", np.float16), ("f32", np.float32)])
def test_oracle_apply_cal_matches_reference(golden, name, dt):
    re, im, gains, _ = MG.cal_inputs()
    g_re, g_im = O.make_cal_broadcast(gains, dt)
    assert np.array_equal(g_re, golden[f"g_re_{name}"]) and np.array_equal(
        g_im, golden[f"g_im_{name}"])
    r, i = re.astype(dt), im.astype(dt)
    o_re, o_im = O.apply_cal_split(r, i, g_re, g_im)
    assert np.array_equal(o_re.view(np.uint8), golden[f"out_re_{name}"].view(np.uint8))
    assert np.array_equal(o_im.view(np.uint8), golden[f"out_im_{name}"].view(np.uint8))
    b_re, b_im = O.apply_cal_split(r, i, g_re[5:6], g_im[5:6])
    assert np.array_equal(b_re.view(np.uint8), golden[f"bout_re_{name}"].view(np.uint8))
    assert np.array_equal(b_im.view(np.uint8), golden[f"bout_im_{name}"].view(np.uint8))


def test_dec_phase_matches_reference(golden):
    from dsb200.constants import DSA110_BAND, PHI_LAT_OVRO_RAD
    from dsb200.corr import compute_dec_phase
    _, _, _, antpos_n = MG.cal_inputs()
    for k, dec in enumerate((0.2, 1.3)):
        ph = compute_dec_phase(chgroup=5, obs_dec_rad=dec, antpos_n=antpos_n)
        assert ph.dtype == np.complex128 and ph.shape == (96, 384)
        assert _sha(ph.view(np.float64)) == str(golden[f"dec_phase_sha_{k}"])
        assert np.array_equal(ph[:, ::16], golden[f"dec_phase_cols_{k}"])
        oph = O.dec_phase(O.REFERENCE_BAND, 5, dec, antpos_n, PHI_LAT_OVRO_RAD)
        assert np.array_equal(oph, ph)
    with pytest.raises(ValueError):
        compute_dec_phase(chgroup=DSA110_BAND.n_chgroup, obs_dec_rad=0.1, antpos_n=antpos_n)


def test_broadcast_tensors_and_checks_on_host():
    from dsb200.corr import apply_cal_split, make_cal_broadcast_tensors
    _, _, gains, _ = MG.cal_inputs()
    for dt in (torch.float16, torch.float32):
        g_re, g_im = make_cal_broadcast_tensors(gains, device="cpu", dtype=dt)
        assert g_re.shape == (8, 1, 2, 1, 96) and g_re.dtype == dt
        w_re, w_im = O.make_cal_broadcast(gains, np.float16 if dt == torch.float16 else np.float32)
        assert np.array_equal(g_re.numpy(), w_re) and np.array_equal(g_im.numpy(), w_im)
    v = torch.zeros((8, 2, 2, 4, 96), dtype=torch.float16)
    g_re, g_im = make_cal_broadcast_tensors(gains, device="cpu", dtype=torch.float16)
    with pytest.raises(ValueError, match="shape"):
        apply_cal_split(v, v[:, :, :, :2], g_re, g_im)
    with pytest.raises(ValueError, match="dtype"):
        apply_cal_split(v, v.float(), g_re, g_im)
    with pytest.raises(ValueError, match="cal dtypes"):
        apply_cal_split(v, v, g_re.float(), g_im.float())
    with pytest.raises(ValueError, match="cal shape"):
        apply_cal_split(v, v, g_re[:, :, :, :, :5], g_im[:, :, :, :, :5])
    with pytest.raises(ValueError):            # no CPU path: CUDA tensors only
        apply_cal_split(v, v, g_re, g_im)
    with pytest.raises(ValueError):
        make_cal_broadcast_tensors(np.zeros((96, 8)), device="cpu")


# ---------------------------------------------------------------------------

gpu = pytest.mark.gpu


@pytest.fixture(scope="module")
def dev():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda", 0)


@gpu
@pytest.mark.parametrize("name,dt", [("f16", torch.float16), ("f32", torch.float32)])
def test_cal_apply_gpu_matches_reference(dev, golden, name, dt):
    from dsb200.corr import apply_cal_split
    re, im, _, _ = MG.cal_inputs()
    r = torch.from_numpy(re.astype(np.float32)).to(dev, dt)
    i = torch.from_numpy(im.astype(np.float32)).to(dev, dt)
    g_re = torch.from_numpy(golden[f"g_re_{name}"]).to(dev)
    g_im = torch.from_numpy(golden[f"g_im_{name}"]).to(dev)
    for sl, pre in ((slice(None), "out"), (slice(5, 6), "bout")):
        o_re, o_im = apply_cal_split(r, i, g_re[sl], g_im[sl])
        assert np.array_equal(o_re.cpu().numpy().view(np.uint8),
                              golden[f"{pre}_re_{name}"].view(np.uint8))
        assert np.array_equal(o_im.cpu().numpy().view(np.uint8),
                              golden[f"{pre}_im_{name}"].view(np.uint8))


@gpu
def test_cal_apply_full_layout_matches_torch_eager(dev):
    """The reference's own op on the GPU (torch eager float16) at the full
    GEMM layout, bit for bit."""
    from dsb200.corr import apply_cal_split
    g = torch.Generator(device=dev)
    g.manual_seed(7)
    shape = (384, 2, 2, 2048, 96)
    r = (torch.randint(-8, 8, shape, device=dev, generator=g) * 0.05).half()
    i = (torch.randint(-8, 8, shape, device=dev, generator=g) * 0.05).half()
    g_re = torch.randn((384, 1, 2, 1, 96), device=dev, generator=g).half()
    g_im = torch.randn((384, 1, 2, 1, 96), device=dev, generator=g).half()
    o_re, o_im = apply_cal_split(r, i, g_re, g_im)
    assert torch.equal(o_re, r * g_re - i * g_im)
    assert torch.equal(o_im, r * g_im + i * g_re)


@gpu
def test_cal_apply_odd_antenna_count(dev):
    from dsb200.corr import apply_cal_split
    rng = np.random.default_rng(3)
    shape = (3, 2, 2, 5, 7)
    re = rng.standard_normal(shape).astype(np.float16)
    im = rng.standard_normal(shape).astype(np.float16)
    g_re = rng.standard_normal((3, 1, 2, 1, 7)).astype(np.float16)
    g_im = rng.standard_normal((3, 1, 2, 1, 7)).astype(np.float16)
    o_re, o_im = apply_cal_split(*(torch.from_numpy(a).to(dev) for a in (re, im, g_re, g_im)))
    w_re, w_im = O.apply_cal_split(re, im, g_re, g_im)
    assert np.array_equal(o_re.cpu().numpy().view(np.uint16), w_re.view(np.uint16))
    assert np.array_equal(o_im.cpu().numpy().view(np.uint16), w_im.view(np.uint16))


@gpu
def test_calibrated_visibilities_carry_conj_gi_gj(dev):
    """Gains applied to the voltages reach the visibilities as
    conj(G_i) G_j (the identity the reference's cal path exists for)."""
    from dsb200.corr import (FastCorrKernel, apply_cal_split, make_cal_broadcast_tensors,
                             unpack_int4_split)
    npkt, nant, nchan, t_int = 16, 32, 16, 8
    rng = np.random.default_rng(12)
    raw = rng.integers(0, 256, npkt * nant * nchan * 4, dtype=np.uint8)
    re, im = unpack_int4_split(raw, device=dev, out_dtype=torch.float16, npkt=npkt, nant=nant,
                               nchan=nchan)
    # one gain per antenna, the same on every channel and pol
    ga = (0.5 + rng.uniform(0, 1, nant)) * np.exp(1j * rng.uniform(-np.pi, np.pi, nant))
    gains = np.broadcast_to(ga[:, None, None], (nant, nchan, 2))
    g_re, g_im = make_cal_broadcast_tensors(gains, device=dev, dtype=torch.float16)
    c_re, c_im = apply_cal_split(re, im, g_re, g_im)
    k = FastCorrKernel(dev, t_int_fast_native=t_int, nants=nant, nchan=nchan)
    v_raw = k.compute_split(re, im, fuse_stokes_i=True).cpu().numpy().astype(np.complex128)
    v_cal = k.compute_split(c_re, c_im, fuse_stokes_i=True).cpu().numpy().astype(np.complex128)
    # gains as the correlator saw them (float16 parts)
    gq = g_re[0, 0, 0, 0].float().cpu().numpy() + 1j * g_im[0, 0, 0, 0].float().cpu().numpy()
    a_idx, b_idx = O.upper_tri_indices(nant)     # bls = a(a+1)/2 + b, b <= a
    want = np.conj(gq[b_idx])[None, :, None] * gq[a_idx][None, :, None] * v_raw
    scale = np.abs(want).max()
    assert np.abs(v_cal - want).max() <= 2e-2 * scale
