"""Per-cube clusterer (cluster/features.py, cluster/forward.py,
cluster/state.py), CPU.

* Features in both modes, the physical coordinates, and the DBSCAN
  backend's labels and records equal the reference's output on the seeded
  candidates of tests/golden/make_golden.py, bit for bit.
* HDBSCAN labels equal scikit-learn's HDBSCAN (min_samples + 1, as it
  counts the point itself) on the same weighted features: the reference's
  ``hdbscan`` package is not installed here.
* The reference's own unit cases: empty and single inputs, co-located and
  distant pairs, peak choice, counts, the fine-DM clamp, errors, and the
  asynchronous service.
"""

import os
import sys
from dataclasses import dataclass

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
import make_golden as MG  # noqa: E402

from dsb200 import cluster as CL  # noqa: E402


@dataclass(frozen=True)
class Cand:
    l: float
    m: float
    dm_fine: float
    event_specnum: int
    width_samples: int
    snr: float
    kernel_id: str = "unit:d1:b4"
    search_node_id: int = 2
    gpu_half: int = 1


def _golden_cands():
    l, m, dm, t, w, snr, node, half = MG.cluster_fields()
    return [Cand(float(l[i]), float(m[i]), float(dm[i]), int(t[i]), int(w[i]), float(snr[i]),
                 f"unit:d1:b{int(w[i])}", int(node[i]), int(half[i])) for i in range(len(l))]


@pytest.fixture(scope="module")
def golden(golden_dir):
    return np.load(os.path.join(golden_dir, "cluster.npz"))


def test_features_and_coords_match_reference(golden):
    geom = CL.CubeGeometry(**MG.cluster_geometry())
    cands = _golden_cands()
    np.testing.assert_array_equal(CL.candidates_to_features(cands, geom), golden["feat_int"])
    np.testing.assert_array_equal(
        CL.candidates_to_features(cands, geom, mode="real", weights=(1.0, 0.5, 2.0, 3e3, 3e3)),
        golden["feat_real"])
    np.testing.assert_array_equal(np.asarray(CL.candidates_to_real_coords(cands, geom)),
                                  golden["coords"])


@pytest.mark.parametrize("name,cfg", [
    ("db", CL.ClustererConfig(backend="dbscan")),
    ("dbreal", CL.ClustererConfig(backend="dbscan", feature_mode="real",
                                  weights=(1.0, 0.02, 20.0, 3e3, 3e3), dbscan_eps=2.5,
                                  dbscan_min_samples=3)),
])
def test_dbscan_labels_and_records_match_reference(golden, name, cfg):
    geom = CL.CubeGeometry(**MG.cluster_geometry())
    labels, recs = CL.cluster_candidates(_golden_cands(), geom, config=cfg)
    np.testing.assert_array_equal(labels, golden[name + "_labels"])
    got = np.asarray([[float(getattr(r, f)) for f in MG.RECORD_FIELDS] for r in recs])
    np.testing.assert_array_equal(got, golden[name + "_records"])
    assert len(set(labels.tolist()) - {-1}) >= 3


@pytest.mark.parametrize("feat", ["int", "real"])
def test_hdbscan_labels_match_scikit_learn(golden, feat):
    X = golden["feat_" + feat]
    got = CL.hdbscan_labels(X, min_cluster_size=2, min_samples=1, cluster_selection_epsilon=10.0,
                            allow_single_cluster=True)
    np.testing.assert_array_equal(got, golden["hdb_" + feat])
    # through the public entry with the reference's default config (INT mode)
    if feat == "int":
        geom = CL.CubeGeometry(**MG.cluster_geometry())
        labels, recs = CL.cluster_candidates(_golden_cands(), geom)
        np.testing.assert_array_equal(labels, golden["hdb_int"])
        n_cl = len(set(labels.tolist()) - {-1})
        assert [r.cluster_id for r in recs[:n_cl]] == list(range(n_cl))
        assert all(r.cluster_id == -1 and r.cntc == 1 for r in recs[n_cl:])
        assert sum(r.cntc for r in recs) == len(labels)


@pytest.mark.parametrize("seed", range(4))
def test_hdbscan_parameters_match_scikit_learn(seed):
    """Other minimum sizes, epsilons and the single-cluster switch on seeded
    blobs (tie-free and integer-valued)."""
    import warnings

    from sklearn.cluster import HDBSCAN
    rng = np.random.default_rng(seed)
    for trial in range(25):
        n = int(rng.integers(2, 70))
        centres = rng.uniform(0, 100, (int(rng.integers(1, 5)), 5))
        X = centres[rng.integers(0, centres.shape[0], n)] + rng.normal(0, 4.0, (n, 5))
        if trial % 2:
            X = np.round(X)
        mcs = int(rng.integers(2, 5))
        ms = int(min(rng.integers(1, 4), n - 1))
        eps = float(rng.choice([0.0, 5.0, 10.0, 30.0]))
        single = bool(rng.integers(0, 2))
        with warnings.catch_warnings():
            warnings.simplefilter("ignore")
            want = HDBSCAN(min_cluster_size=mcs, min_samples=ms + 1,
                           cluster_selection_epsilon=eps, metric="manhattan",
                           allow_single_cluster=single, copy=True).fit_predict(X)
        got = CL.hdbscan_labels(X, min_cluster_size=mcs, min_samples=ms,
                                cluster_selection_epsilon=eps, allow_single_cluster=single)
        np.testing.assert_array_equal(got, want, err_msg=f"seed {seed} trial {trial}")


def test_dbscan_matches_scikit_learn_on_blobs():
    from sklearn.cluster import DBSCAN
    rng = np.random.default_rng(9)
    for _ in range(40):
        X = np.round(rng.normal(0, 12, (int(rng.integers(1, 90)), 5)))
        eps, ms = float(rng.uniform(2, 20)), int(rng.integers(1, 5))
        np.testing.assert_array_equal(
            CL.dbscan_labels(X, eps=eps, min_samples=ms),
            DBSCAN(eps=eps, min_samples=ms, metric="cityblock").fit_predict(X))


# ---- the reference's unit cases -------------------------------------------


def _geom(**kw):
    base = dict(cube_id=0, specnum_start=1024, sample_period_specnum=16, t_det=256, n_grid=256,
                n_fdm_in_cube=8, sample_period_us=131.072, cell_l_rad=1.5e-4, cell_m_rad=1.5e-4,
                l0_rad=0.0, m0_rad=0.0, fine_dm_pc_cc=np.linspace(50.0, 800.0, 8),
                mjd_start=60942.1)
    base.update(kw)
    return CL.CubeGeometry(**base)


def _cand(l_pix=10, m_pix=20, fdm=2, t=64, snr=8.5, width=4):
    g = _geom()
    return Cand(float(l_pix), float(m_pix), float(g.fine_dm_pc_cc[fdm]),
                g.specnum_start + t, width, snr)


@pytest.mark.parametrize("backend", ["hdbscan", "dbscan"])
def test_empty_single_and_pairs(backend):
    cfg = CL.ClustererConfig(backend=backend)
    labels, recs = CL.cluster_candidates([], _geom(), config=cfg)
    assert labels.shape == (0,) and labels.dtype == np.int64 and recs == []
    labels, recs = CL.cluster_candidates([_cand(snr=20.0)], _geom(), config=cfg)
    assert labels.tolist() == [-1] and len(recs) == 1
    r = recs[0]
    assert (r.cluster_id, r.cntc, r.cntb_lm, r.cntb_dm, r.snr, r.peak_candidate_idx) == \
        (-1, 1, 1, 1, 20.0, 0)
    labels, recs = CL.cluster_candidates([_cand(snr=9.0), _cand(snr=15.0)], _geom(), config=cfg)
    assert labels.tolist() == [0, 0] and len(recs) == 1
    assert (recs[0].cntc, recs[0].cntb_lm, recs[0].cntb_dm, recs[0].peak_candidate_idx) == \
        (2, 1, 1, 1)
    far = [_cand(l_pix=10, m_pix=20, t=10), _cand(l_pix=200, m_pix=200, fdm=7, t=250)]
    labels, recs = CL.cluster_candidates(far, _geom(), config=cfg)
    assert labels.tolist() == [-1, -1] and [r.cluster_id for r in recs] == [-1, -1]


def test_peak_counts_and_units():
    cands = [_cand(l_pix=10, m_pix=20, snr=9.0), _cand(l_pix=10, m_pix=21, snr=22.7),
             _cand(l_pix=11, m_pix=20, fdm=3, snr=12.0), _cand(l_pix=10, m_pix=20, snr=8.0),
             _cand(l_pix=132, m_pix=230, fdm=4, t=64, snr=30.0),
             _cand(l_pix=132, m_pix=231, fdm=4, t=65, snr=7.0)]
    g = _geom(cell_l_rad=2.5e-4, cell_m_rad=2.5e-4)
    labels, recs = CL.cluster_candidates(cands, g, config=CL.ClustererConfig(backend="dbscan"))
    assert labels.tolist() == [0, 0, 0, 0, 1, 1]
    a, b = recs
    assert (a.cntc, a.cntb_lm, a.cntb_dm, a.snr, a.peak_candidate_idx) == (4, 3, 2, 22.7, 1)
    assert (a.l_pix, a.m_pix) == (10, 21)
    assert (b.l_pix, b.m_pix, b.fine_dm_idx, b.t_in_cube) == (132, 230, 4, 64)
    np.testing.assert_allclose(b.l_rad, (230 - 128) * 2.5e-4)
    np.testing.assert_allclose(b.m_rad, (132 - 128) * 2.5e-4)
    np.testing.assert_allclose(b.t_seconds, 64 * g.sample_period_us / 1e6)


def test_feature_errors_and_clamps():
    g = _geom()
    with pytest.raises(ValueError):
        CL.candidates_to_features([_cand()], g, mode="bogus")
    with pytest.raises(ValueError):
        CL.candidates_to_features([_cand()], g, weights=(1.0, 1.0))
    with pytest.raises(ValueError):
        CL.candidates_to_features([_cand(width=0)], g)
    with pytest.raises(ValueError):
        CL.cluster_candidates([_cand(), _cand()], g, config=CL.ClustererConfig(backend="x"))
    with pytest.raises(ValueError):
        CL.cluster_candidates([_cand(), _cand()], g, config=CL.ClustererConfig(metric="euclidean"))
    assert CL.candidates_to_features([], g).shape == (0, 5)
    lo = Cand(10.0, 20.0, 1.0, 1024, 4, 9.0)
    hi = Cand(10.0, 20.0, 9999.0, 1024, 4, 9.0)
    mid = Cand(10.0, 20.0, float(g.fine_dm_pc_cc[2] + 1.0), 1024, 4, 9.0)
    f = CL.candidates_to_features([lo, hi, mid], g)
    assert f[:, 1].tolist() == [0.0, 7.0, 2.0]
    assert CL.DEFAULT_WEIGHTS == (4.0, 1.0, 1.0, 1.0, 1.0)


def test_service_runs_cubes_and_counts():
    svc = CL.ClustererService(CL.ClustererConfig(backend="dbscan"))
    with pytest.raises(RuntimeError):
        svc.submit([_cand()], _geom())
    svc.start()
    with pytest.raises(RuntimeError):
        svc.start()
    try:
        futs = [svc.submit([_cand(snr=9.0), _cand(snr=15.0)], _geom(cube_id=k)) for k in range(3)]
        bad = svc.submit([_cand(width=0), _cand()], _geom(cube_id=9))
        res = [f.result(timeout=30) for f in futs]
        with pytest.raises(ValueError):
            bad.result(timeout=30)
    finally:
        svc.shutdown()
    assert [r.cube_id for r in res] == [0, 1, 2]
    assert all(r.labels.tolist() == [0, 0] and r.wall_ms >= 0 for r in res)
    assert (svc.n_submitted, svc.n_completed, svc.n_failed) == (4, 3, 1)
    with pytest.raises(ValueError):
        CL.ClustererService(max_workers=0)
