"""DeterministicDetector (detector/forward.py:512, streaming production
form) on the fused detector kernel, against the oracle composition of the
same steps: padded cumsum, centred boxcars over the interior, S/N with the
previous cube's Layer-2 sigma_k, strict-'>' winner, top-k + merge radii,
then the Layer-2 update from each kernel's seeded samples.  Three cubes in a
row, so the second and third are decoded with learned sigma_k; a planted
dispersed-free burst must come out at its cell and width."""

import math

import numpy as np
import pytest
import torch

import dsb_oracle as O

pytestmark = pytest.mark.gpu


def test_deterministic_detector_matches_oracle_over_three_cubes():
    from dsb200.detector import DeterministicDetector
    from dsb200.kernels import build_kernel_bank
    dev = torch.device("cuda", 0)
    T, F, H, W = 96, 3, 16, 32
    widths = [1, 2, 4, 8, 16]
    det = DeterministicDetector(device=dev, threshold_sigma=6.0, merge_radius_t=4,
                                kernel_bank=build_kernel_bank(
                                    ("unit",), ("d1",), tuple(f"b{w}" for w in widths)),
                                cube_cadence_s=0.2, layer2_tau_s=2.0, layer2_n_burnin=2,
                                layer2_sigma_max_samples=2000)
    te = 8
    n_out = T - 2 * te
    offs = O.boxcar_offsets(widths, 16)
    l2 = O.Layer2State(widths, 0.2, tau_s=2.0, n_burnin=2)
    idx = O.layer2_sample_index(len(widths), 2000, n_out * F * H * W)
    rng = np.random.default_rng(4)
    for c in range(3):
        cube = rng.standard_normal((T, F, H, W)).astype(np.float32)
        cube[40 + c:44 + c, 1, 5, 7] += 4.0                  # a 4-sample burst
        got = det.forward(torch.from_numpy(cube).to(dev),
                          torch.ones((T, F), dtype=torch.bool, device=dev),
                          torch.ones(F, device=dev), event_specnum=1000 * c)
        # oracle
        sinv = (np.float32(1.0) / np.maximum(l2.s, np.float32(1e-30))).astype(np.float32)
        cs = O.padded_cumsum(cube, 16)
        score, win = O.multi_boxcar_argmax(cs, widths, offs, sinv, n_out, te)
        n_top = max(64, math.ceil(64 * T / n_out)) * len(widths)
        want = O.decode_topk(score, win, threshold=6.0, n_top=n_top, r_t=4, r_f=5, r_lm=3)
        csf = cs.reshape(cs.shape[0], -1)
        samp = np.empty(idx.shape, np.float32)
        for k, (w, off) in enumerate(zip(widths, offs)):
            t_in, cell = idx[k] // (F * H * W), idx[k] % (F * H * W)
            samp[k] = csf[t_in + te + off + w, cell] - csf[t_in + te + off, cell]
        l2.update(O.sigma_clipped_std_batched(samp))
        g = {(x.event_specnum - 1000 * c - te, int(x.dm_idx), int(x.l), int(x.m),
              x.width_samples): x.snr for x in got}
        w_ = {(x.t, x.f, x.l, x.m, widths[x.k]): x.snr for x in want}
        assert set(g) == set(w_), (c, sorted(set(g) ^ set(w_)))
        for k in g:
            assert abs(g[k] - w_[k]) <= 1e-5 * abs(w_[k]), (k, g[k], w_[k])
        assert any(k[1:4] == (1, 5, 7) and k[4] == 4 for k in g)
        np.testing.assert_allclose(det.layer2_state.s_k.cpu().numpy(), l2.s, rtol=2e-6)
    assert det.kernels() == tuple(f"unit:d1:b{w}" for w in widths)
