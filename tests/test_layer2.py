"""Layer-1 burn-in and Layer-2 per-kernel noise state (noise_norm/layer1.py:
342-600, noise_norm/layer2.py:113-452).  Layer-2: the
Welford burn-in, the EMA, zero estimates, invalid cubes, the clamp above
``sigma_max_ratio`` with its escape hatch, and scalar and per-kernel floors
equal the reference's state on CPU bit for bit over a seeded sequence of
per-kernel sigma estimates (tests/golden/make_golden.py)."""

import os
import sys

import numpy as np
import pytest
import torch

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
import make_golden as MG  # noqa: E402

from dsb200.noise import Layer2State  # noqa: E402


@pytest.mark.parametrize("ci", range(len(MG.LAYER2_CONFIGS)))
def test_layer2_state_matches_reference(golden_dir, ci):
    z = np.load(os.path.join(golden_dir, "layer2.npz"))
    sig, valid = MG.layer2_sequence()
    st = Layer2State(sig.shape[1], **MG.LAYER2_CONFIGS[ci])
    s_k, warm = [], []
    for c in range(sig.shape[0]):
        s, w = st.update_and_query(per_kernel_sigma=torch.from_numpy(sig[c]), valid=bool(valid[c]))
        s_k.append(s.numpy())
        warm.append(w)
    assert np.array_equal(np.asarray(s_k, np.float32).view(np.uint32), z[f"s_k_{ci}"].view(np.uint32))
    assert np.array_equal(np.asarray(warm), z[f"warm_{ci}"])
    assert [st.n_clamped_high, st.n_clamp_escapes, st.cube_count] == z[f"counters_{ci}"].tolist()
    assert np.array_equal(np.stack([st.per_kernel_clamped_high.numpy(),
                                    st.per_kernel_clamp_escapes.numpy(),
                                    st.per_kernel_clamp_streak.numpy()]), z[f"per_kernel_{ci}"])


def test_layer2_arguments_and_reset():
    with pytest.raises(ValueError):
        Layer2State(0)
    with pytest.raises(ValueError):
        Layer2State(3, sigma_floor=(0.1, 0.2))
    with pytest.raises(ValueError):
        Layer2State(3, tau_s=0.0)
    st = Layer2State(3, n_burnin=2)
    with pytest.raises(ValueError):
        st.update_and_query()
    with pytest.raises(ValueError):
        st.update_and_query(per_kernel_sigma=torch.ones(4))
    with pytest.raises(NotImplementedError):
        st.update_and_query(torch.zeros((3, 4, 1, 2, 2)))
    s, w = st.update_and_query(per_kernel_sigma=torch.tensor([2.0, 3.0, 4.0]))
    assert torch.equal(s, torch.tensor([2.0, 3.0, 4.0])) and w
    st.reset()
    assert st.cube_count == 0 and torch.equal(st.s_k, torch.ones(3))


@pytest.mark.parametrize("ci,kw", [(0, dict()), (1, dict(n_burnin_cubes=3, sigma_floor=0.97))])
def test_layer1_state_matches_reference(golden_dir, ci, kw):
    """Layer1State (noise_norm/layer1.py:342-600): burn-in medians, then the
    cube's own σ, and the floor, bit for bit."""
    from dsb200.noise import Layer1State
    z = np.load(os.path.join(golden_dir, "layer1_state.npz"))
    sig, _ = MG.layer2_sequence()
    st = Layer1State(sig.shape[1], **kw)
    got = np.asarray([st.update_and_query(per_fdm_sigma=torch.from_numpy(sig[c])).numpy()
                      for c in range(12)], np.float32)
    assert np.array_equal(got.view(np.uint32), z[f"l1_{ci}"].view(np.uint32))
    assert not st.is_warming_up and st.cube_count == 12
    with pytest.raises(ValueError):
        st.update_and_query(per_fdm_sigma=torch.ones(2))
