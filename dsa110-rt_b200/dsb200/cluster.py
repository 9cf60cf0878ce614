"""Per-cube candidate clusterer after the detector and the cross-kernel
merger: the reference's cluster/features.py, cluster/forward.py and
cluster/state.py.

Features (features.py:160-289).  One row per candidate, columns
``[log2 width, DM axis, time axis, l axis, m axis]``, each column scaled by
its weight (cityblock distance then weighs axis j by w_j):
* ``"int"`` mode: fine-DM index (the grid value closest to ``dm_fine``,
  left on a tie, clamped to the cube), ``t_in_cube = event_specnum -
  specnum_start``, and the rounded pixel indices ``l_pix``, ``m_pix``;
* ``"real"`` mode: ``dm_fine``, ``t_in_cube * sample_period_us / 1e6`` and
  sky radians with the axes swapped (cube row = sky m, column = sky l),
  pixels centred at ``n_grid // 2``.

Backends (forward.py:103-150), both written here on a dense cityblock
distance matrix (a cube carries at most a few thousand candidates):
* DBSCAN (``eps``, ``min_samples``, cityblock): clusters are the connected
  components of core points, numbered by their lowest core index; a border
  point joins the lowest-numbered cluster that reaches it (the labels of
  scikit-learn's DBSCAN, the reference's fallback backend);
* HDBSCAN (``min_cluster_size``, ``min_samples``,
  ``cluster_selection_epsilon``, ``allow_single_cluster``, manhattan): the
  algorithm of Campello, Moulavi and Sander (2013) as published in the
  ``hdbscan`` package (McInnes, Healy and Astels 2017) with the epsilon
  selection of Malzer and Baum (2019): core distances to the
  ``min_samples``-th other point, mutual reachability, minimum spanning tree,
  single-linkage hierarchy, condensed tree, excess-of-mass selection, then
  the epsilon search.

Records (forward.py:199-273): one per cluster id >= 0 in ascending order,
then one singleton (cluster id -1) per noise point in input order; each
carries its highest-SNR member's coordinates in both frames and the counts
``cntc`` (members), ``cntb_lm`` (distinct (l_pix, m_pix)), ``cntb_dm``
(distinct fine-DM indices).
"""

from __future__ import annotations

import logging
import math
import threading
import time
from concurrent.futures import Future, ThreadPoolExecutor
from dataclasses import dataclass
from typing import List, Optional, Sequence, Tuple

import numpy as np

_LOG = logging.getLogger(__name__)


class FeatureMode:
    INT: str = "int"
    REAL: str = "real"


class ClustererBackend:
    HDBSCAN: str = "hdbscan"
    DBSCAN: str = "dbscan"


# column weights [log2_width, dm, t, l, m] (the T2 cityblock convention)
DEFAULT_WEIGHTS: Tuple[float, float, float, float, float] = (4.0, 1.0, 1.0, 1.0, 1.0)


@dataclass(frozen=True)
class CubeGeometry:
    """Geometry of one search cube (the fields of the reference's
    ``CubeGeometry`` contract)."""

    cube_id: int
    specnum_start: int
    sample_period_specnum: int
    t_det: int
    n_grid: int
    n_fdm_in_cube: int
    sample_period_us: float
    cell_l_rad: float
    cell_m_rad: float
    l0_rad: float
    m0_rad: float
    fine_dm_pc_cc: np.ndarray
    mjd_start: float


@dataclass(frozen=True)
class ClusterRecord:
    """One cluster (or noise singleton) with its peak candidate (the fields
    of the reference's ``ClusterRecord`` contract)."""

    cluster_id: int
    cube_id: int
    cntc: int
    cntb_lm: int
    cntb_dm: int
    peak_candidate_idx: int
    l_rad: float
    m_rad: float
    l_pix: int
    m_pix: int
    dm_fine_pc_cc: float
    fine_dm_idx: int
    t_in_cube: int
    t_seconds: float
    width_samples: int
    snr: float
    kernel_id: str
    event_specnum: int
    search_node_id: int
    gpu_half: int


@dataclass(frozen=True)
class ClustererConfig:
    """Backend and hyper-parameters (forward.py:62-100 defaults)."""

    backend: str = ClustererBackend.HDBSCAN
    feature_mode: str = FeatureMode.INT
    weights: Tuple[float, float, float, float, float] = DEFAULT_WEIGHTS
    min_cluster_size: int = 2
    min_samples: int = 1
    cluster_selection_epsilon: float = 10.0
    dbscan_eps: Optional[float] = None
    dbscan_min_samples: int = 2
    metric: str = "manhattan"


# ---------------------------------------------------------------------------
# features
# ---------------------------------------------------------------------------


def centred_pix_offset(pix: float, n_grid: int) -> float:
    """``pix - n_grid // 2`` (the cube images are centred); ``pix`` itself
    when ``n_grid <= 0`` (features.py:58-87)."""
    n = int(n_grid)
    return float(pix) if n <= 0 else float(pix) - float(n // 2)


def _int_indices(cands: Sequence, geom) -> Tuple[np.ndarray, ...]:
    """(l_pix, m_pix, fine_dm_idx, t_in_cube) int64 arrays
    (features.py:90-140)."""
    l_pix = np.asarray([int(round(c.l)) for c in cands], np.int64)
    m_pix = np.asarray([int(round(c.m)) for c in cands], np.int64)
    grid = np.asarray(geom.fine_dm_pc_cc, np.float64)
    dm = np.asarray([c.dm_fine for c in cands], np.float64)
    nf = int(geom.n_fdm_in_cube)
    ins = np.searchsorted(grid, dm)
    safe = np.clip(ins, 1, max(1, grid.size - 1))
    left = np.abs(grid[safe - 1] - dm)
    right = np.abs(grid[np.minimum(safe, grid.size - 1)] - dm)
    fdm = np.where(left <= right, safe - 1, safe)
    fdm = np.where(ins <= 0, 0, np.where(ins >= nf, nf - 1, fdm)).astype(np.int64)
    t = np.asarray([int(c.event_specnum) - int(geom.specnum_start) for c in cands], np.int64)
    return l_pix, m_pix, fdm, t


def _log2_widths(cands: Sequence) -> np.ndarray:
    out = np.empty(len(cands), np.float64)
    for i, c in enumerate(cands):
        if c.width_samples <= 0:
            raise ValueError(f"width_samples={c.width_samples} must be > 0")
        out[i] = math.log2(float(c.width_samples))
    return out


def _sky(l_pix: np.ndarray, m_pix: np.ndarray, geom) -> Tuple[np.ndarray, np.ndarray]:
    """Sky (l, m) radians of cube (row, col) pixels: the row is the sky m
    axis and the column the sky l axis (features.py:262-273)."""
    n = int(geom.n_grid)
    c = 0.0 if n <= 0 else float(n // 2)
    l_rad = (m_pix.astype(np.float64) - c) * geom.cell_l_rad + geom.l0_rad
    m_rad = (l_pix.astype(np.float64) - c) * geom.cell_m_rad + geom.m0_rad
    return l_rad, m_rad


def candidates_to_features(cands: Sequence, geom, *, mode: str = FeatureMode.INT,
                           weights: Sequence[float] = DEFAULT_WEIGHTS) -> np.ndarray:
    """``(n, 5)`` float64 feature rows, weights applied (features.py:160-236)."""
    if mode not in (FeatureMode.INT, FeatureMode.REAL):
        raise ValueError(f"mode={mode!r}, expected one of {FeatureMode.INT!r}, "
                         f"{FeatureMode.REAL!r}")
    if len(weights) != 5:
        raise ValueError(f"weights must be length 5; got len={len(weights)}")
    if not cands:
        return np.zeros((0, 5), np.float64)
    l_pix, m_pix, fdm, t = _int_indices(cands, geom)
    out = np.empty((len(cands), 5), np.float64)
    out[:, 0] = _log2_widths(cands)
    if mode == FeatureMode.INT:
        out[:, 1], out[:, 2], out[:, 3], out[:, 4] = fdm, t, l_pix, m_pix
    else:
        out[:, 1] = [float(c.dm_fine) for c in cands]
        out[:, 2] = t.astype(np.float64) * geom.sample_period_us / 1e6
        out[:, 3], out[:, 4] = _sky(l_pix, m_pix, geom)
    out *= np.asarray(weights, np.float64)[None, :]
    return out


def candidates_to_real_coords(cands: Sequence, geom) -> List[tuple]:
    """Per candidate ``(l_rad, m_rad, dm_fine, t_seconds, l_pix, m_pix,
    fine_dm_idx, t_in_cube)`` (features.py:239-289)."""
    if not cands:
        return []
    l_pix, m_pix, fdm, t = _int_indices(cands, geom)
    l_rad, m_rad = _sky(l_pix, m_pix, geom)
    ts = t.astype(np.float64) * geom.sample_period_us / 1e6
    return [(float(l_rad[i]), float(m_rad[i]), float(c.dm_fine), float(ts[i]), int(l_pix[i]),
             int(m_pix[i]), int(fdm[i]), int(t[i])) for i, c in enumerate(cands)]


# ---------------------------------------------------------------------------
# backends
# ---------------------------------------------------------------------------


def cityblock_matrix(X: np.ndarray) -> np.ndarray:
    """Dense cityblock distances, summed over the columns in order."""
    X = np.asarray(X, np.float64)
    d = np.zeros((X.shape[0], X.shape[0]), np.float64)
    t = np.empty_like(d)
    for j in range(X.shape[1]):
        np.subtract.outer(X[:, j], X[:, j], out=t)
        np.abs(t, out=t)
        d += t
    return d


def dbscan_labels(X: np.ndarray, *, eps: float, min_samples: int) -> np.ndarray:
    """DBSCAN labels (-1 = noise) under cityblock distance; the neighbourhood
    of a point is every point within ``eps`` (itself included)."""
    n = X.shape[0]
    labels = np.full(n, -1, np.int64)
    if n == 0:
        return labels
    nb = cityblock_matrix(X) <= eps
    core = nb.sum(axis=1) >= min_samples
    nxt = 0
    for i in range(n):
        if labels[i] != -1 or not core[i]:
            continue
        # the core component of i, then every border point it reaches
        comp = np.zeros(n, bool)
        comp[i] = True
        front = comp.copy()
        while front.any():
            reach = nb[front].any(axis=0) & core & ~comp
            comp |= reach
            front = reach
        members = (nb[comp].any(axis=0) | comp) & (labels == -1)
        labels[members] = nxt
        nxt += 1
    return labels


def _bfs_hierarchy(Z: np.ndarray, root: int, n: int) -> List[int]:
    """Nodes under ``root`` of a single-linkage hierarchy, level by level,
    left child before right."""
    out, level = [], [root]
    while level:
        out.extend(level)
        level = [int(c) for x in level if x >= n for c in Z[x - n, :2]]
    return out


def mst_edges(X: np.ndarray, min_samples: int) -> np.ndarray:
    """Prim's minimum spanning tree over the mutual-reachability graph of the
    rows of X (cityblock distance, core distance to the ``min_samples``-th
    other point), from the library's host code (``dsb_cluster_mst``):
    ``(n - 1, 3)`` rows (source, point, distance) in the order added."""
    from . import _lib
    X = np.ascontiguousarray(X, np.float64)
    n = X.shape[0]
    core = np.empty(n, np.float64)
    edges = np.empty((n - 1, 3), np.float64)
    _lib.check(_lib.lib().dsb_cluster_mst(
        X.ctypes.data_as(_lib.ctypes.c_void_p), n, X.shape[1], int(min_samples),
        core.ctypes.data_as(_lib.ctypes.c_void_p), edges.ctypes.data_as(_lib.ctypes.c_void_p)),
        "dsb_cluster_mst")
    return edges


def _single_linkage(edges: np.ndarray, n: int) -> np.ndarray:
    """MST edges turned into a single-linkage hierarchy ``(n - 1, 4)``:
    left, right, distance, size; node n + i is row i.  Equal weights keep
    the order numpy's default argsort gives them (as scikit-learn's
    implementation does)."""
    edges = edges[np.argsort(edges[:, 2], kind="quicksort")]
    parent = np.arange(2 * n - 1)
    size = np.ones(2 * n - 1, np.int64)

    def find(x):
        r = x
        while parent[r] != r:
            r = parent[r]
        while parent[x] != r:
            parent[x], x = r, parent[x]
        return r

    Z = np.empty((n - 1, 4), np.float64)
    for k, (a, b, w) in enumerate(edges):
        ra, rb = find(int(a)), find(int(b))
        Z[k] = (ra, rb, w, size[ra] + size[rb])
        parent[ra] = parent[rb] = n + k
        size[n + k] = size[ra] + size[rb]
    return Z


def _condense(Z: np.ndarray, n: int, mcs: int) -> np.ndarray:
    """Condensed tree rows ``(parent, child, lambda, child_size)``: a split
    keeps both sides as new clusters only when both hold ``mcs`` points;
    otherwise the small side's points fall out at lambda = 1 / distance."""
    root = 2 * n - 2
    relabel = np.zeros(2 * n - 1, np.int64)
    relabel[root] = n
    nxt = n + 1
    ignore = np.zeros(2 * n - 1, bool)
    rows = []

    def count(x):
        return 1 if x < n else int(Z[x - n, 3])

    def drop(sub_root, into, lam):
        for s in _bfs_hierarchy(Z, sub_root, n):
            if s < n:
                rows.append((into, s, lam, 1))
            ignore[s] = True

    for node in _bfs_hierarchy(Z, root, n):
        if ignore[node] or node < n:
            continue
        left, right, dist = int(Z[node - n, 0]), int(Z[node - n, 1]), Z[node - n, 2]
        lam = 1.0 / dist if dist > 0.0 else np.inf
        lc, rc = count(left), count(right)
        p = relabel[node]
        if lc >= mcs and rc >= mcs:
            relabel[left] = nxt
            rows.append((p, nxt, lam, lc))
            relabel[right] = nxt + 1
            rows.append((p, nxt + 1, lam, rc))
            nxt += 2
        elif lc < mcs and rc < mcs:
            drop(left, p, lam)
            drop(right, p, lam)
        elif lc < mcs:
            relabel[right] = p
            drop(left, p, lam)
        else:
            relabel[left] = p
            drop(right, p, lam)
    return np.asarray(rows, np.float64).reshape(-1, 4)


def _subtree(ctree: np.ndarray, node: int) -> List[int]:
    """Clusters under ``node`` in the cluster part of a condensed tree."""
    out, level = [], [node]
    while level:
        out.extend(level)
        level = [int(c) for c in ctree[np.isin(ctree[:, 0], level), 1]]
    return out


def _epsilon_search(selected, ctree: np.ndarray, eps: float, allow_single: bool) -> set:
    root = int(ctree[:, 0].min())

    def birth_eps(c):
        return 1.0 / ctree[ctree[:, 1] == c, 2][0]

    def upwards(leaf):
        parent = int(ctree[ctree[:, 1] == leaf, 0][0])
        if parent == root:
            return parent if allow_single else leaf
        return parent if birth_eps(parent) > eps else upwards(parent)

    out, done = [], set()
    for leaf in selected:
        if birth_eps(leaf) < eps:
            if leaf not in done:
                top = upwards(leaf)
                out.append(top)
                done.update(s for s in _subtree(ctree, top) if s != top)
        else:
            out.append(leaf)
    return set(out)


def hdbscan_labels(X: np.ndarray, *, min_cluster_size: int = 2, min_samples: int = 1,
                   cluster_selection_epsilon: float = 0.0,
                   allow_single_cluster: bool = False) -> np.ndarray:
    """HDBSCAN labels (-1 = noise) under cityblock distance; see the module
    notes.  ``min_samples`` counts neighbours other than the point."""
    n = X.shape[0]
    if min_cluster_size < 2:
        raise ValueError(f"min_cluster_size={min_cluster_size}, expected >= 2")
    if n < 2:
        return np.full(n, -1, np.int64)
    Z = _single_linkage(mst_edges(X, min_samples), n)
    tree = _condense(Z, n, int(min_cluster_size))
    par, chi, lam, sz = tree[:, 0].astype(np.int64), tree[:, 1].astype(np.int64), tree[:, 2], \
        tree[:, 3].astype(np.int64)
    root = n
    n_nodes = int(max(chi.max(), par.max())) + 1
    birth = np.zeros(n_nodes)
    birth[chi] = lam
    birth[root] = 0.0
    clusters = sorted(set(par.tolist()))
    stab = {c: 0.0 for c in clusters}
    for p, lv, s in zip(par, lam, sz):
        stab[int(p)] += (lv - birth[p]) * s
    ctree = tree[sz > 1]
    nodes = sorted(stab, reverse=True)
    if not allow_single_cluster:
        nodes = nodes[:-1]
    is_cl = {c: True for c in nodes}
    for node in nodes:
        kids = ctree[ctree[:, 0] == node, 1].astype(np.int64)
        sub = float(np.sum([stab[int(c)] for c in kids]))
        if sub > stab[node]:
            is_cl[node] = False
            stab[node] = sub
        else:
            for s in _subtree(ctree, node):
                if s != node:
                    is_cl[s] = False
    if cluster_selection_epsilon != 0.0 and ctree.shape[0] > 0:
        eom = [c for c in is_cl if is_cl[c]]
        if len(eom) == 1 and eom[0] == int(ctree[:, 0].min()):
            chosen = set(eom) if allow_single_cluster else set()
        else:
            chosen = _epsilon_search(set(eom), ctree, cluster_selection_epsilon,
                                     allow_single_cluster)
        is_cl = {c: c in chosen for c in is_cl}
    selected = sorted(c for c in is_cl if is_cl[c])
    label_of = {c: i for i, c in enumerate(selected)}
    # each point belongs to the top of its chain of unselected clusters
    # (pointer doubling up the condensed tree)
    up = np.arange(n_nodes)
    free = ~np.isin(chi, selected)
    up[chi[free]] = par[free]
    while True:
        nxt = up[up]
        if np.array_equal(nxt, up):
            break
        up = nxt

    point_lam = np.zeros(n)
    m = chi < n
    point_lam[chi[m]] = lam[m]
    labels = np.full(n, -1, np.int64)
    root_kids_max = lam[par == root].max() if np.any(par == root) else 0.0
    for i in range(n):
        t = int(up[i])
        if t == root:
            if len(selected) == 1 and allow_single_cluster:
                thr = (1.0 / cluster_selection_epsilon if cluster_selection_epsilon != 0.0
                       else root_kids_max)
                labels[i] = label_of[root] if point_lam[i] >= thr else -1
        elif t in label_of:
            labels[i] = label_of[t]
    return labels


# ---------------------------------------------------------------------------
# public entry
# ---------------------------------------------------------------------------


def _record(cid: int, idx: np.ndarray, cands: Sequence, coords: List[tuple], geom) -> ClusterRecord:
    peak = int(idx[int(np.argmax([cands[i].snr for i in idx]))])
    c = cands[peak]
    l_rad, m_rad, dm, ts, l_pix, m_pix, fdm, t = coords[peak]
    return ClusterRecord(
        cluster_id=int(cid), cube_id=int(geom.cube_id), cntc=int(idx.size),
        cntb_lm=len({(coords[i][4], coords[i][5]) for i in idx}),
        cntb_dm=len({coords[i][6] for i in idx}), peak_candidate_idx=peak,
        l_rad=float(l_rad), m_rad=float(m_rad), l_pix=int(l_pix), m_pix=int(m_pix),
        dm_fine_pc_cc=float(dm), fine_dm_idx=int(fdm), t_in_cube=int(t), t_seconds=float(ts),
        width_samples=int(c.width_samples), snr=float(c.snr), kernel_id=c.kernel_id,
        event_specnum=int(c.event_specnum), search_node_id=int(c.search_node_id),
        gpu_half=int(c.gpu_half))


def cluster_candidates(cands: Sequence, geom, *, config: Optional[ClustererConfig] = None
                       ) -> Tuple[np.ndarray, List[ClusterRecord]]:
    """``(labels, records)`` of one cube's candidates (forward.py:153-238)."""
    cfg = config or ClustererConfig()
    if cfg.metric not in ("manhattan", "cityblock", "l1"):
        raise ValueError(f"metric={cfg.metric!r}: only the cityblock (manhattan) distance "
                         f"of the reference's configuration is implemented")
    if not cands:
        return np.zeros(0, np.int64), []
    X = candidates_to_features(cands, geom, mode=cfg.feature_mode, weights=cfg.weights)
    if len(cands) == 1:
        labels = np.full(1, -1, np.int64)
    elif cfg.backend == ClustererBackend.HDBSCAN:
        labels = hdbscan_labels(X, min_cluster_size=cfg.min_cluster_size,
                                min_samples=cfg.min_samples,
                                cluster_selection_epsilon=float(cfg.cluster_selection_epsilon),
                                allow_single_cluster=True)
    elif cfg.backend == ClustererBackend.DBSCAN:
        eps = float(cfg.dbscan_eps if cfg.dbscan_eps is not None
                    else cfg.cluster_selection_epsilon)
        labels = dbscan_labels(X, eps=eps, min_samples=int(cfg.dbscan_min_samples))
    else:
        raise ValueError(f"backend={cfg.backend!r}, expected one of "
                         f"{ClustererBackend.HDBSCAN!r}, {ClustererBackend.DBSCAN!r}")
    coords = candidates_to_real_coords(cands, geom)
    records = [_record(cid, np.nonzero(labels == cid)[0], cands, coords, geom)
               for cid in sorted({int(v) for v in labels.tolist() if v >= 0})]
    records += [_record(-1, np.asarray([i]), cands, coords, geom)
                for i in np.nonzero(labels == -1)[0]]
    return labels, records


# ---------------------------------------------------------------------------
# asynchronous service (state.py)
# ---------------------------------------------------------------------------


class ClustererServiceResult:
    """One cube's clustering: labels, records and the call's wall time."""

    __slots__ = ("cube_id", "labels", "records", "wall_ms")

    def __init__(self, cube_id: int, labels: np.ndarray, records: List[ClusterRecord],
                 wall_ms: float) -> None:
        self.cube_id = int(cube_id)
        self.labels = labels
        self.records = records
        self.wall_ms = float(wall_ms)


class ClustererService:
    """Clusters cubes on a worker thread (state.py:72-232): ``start``,
    ``submit(cands, geom) -> Future[ClustererServiceResult]``, ``shutdown``."""

    def __init__(self, config: Optional[ClustererConfig] = None, *, max_workers: int = 1):
        if max_workers <= 0:
            raise ValueError(f"max_workers={max_workers}, expected > 0")
        self._config = config or ClustererConfig()
        self._max_workers = max_workers
        self._executor: Optional[ThreadPoolExecutor] = None
        self._stopping = threading.Event()
        self._lock = threading.Lock()
        self._n = {"submitted": 0, "completed": 0, "failed": 0}

    def start(self) -> None:
        if self._executor is not None:
            raise RuntimeError("ClustererService.start() called twice")
        self._executor = ThreadPoolExecutor(max_workers=self._max_workers,
                                            thread_name_prefix="dsb-clusterer")

    def shutdown(self, *, wait: bool = True, timeout: Optional[float] = None) -> None:
        self._stopping.set()
        if self._executor is None:
            return
        self._executor.shutdown(wait=wait)
        self._executor = None

    def submit(self, cands: Sequence, geom) -> Future:
        if self._executor is None:
            raise RuntimeError("ClustererService.submit() requires start() first")
        with self._lock:
            self._n["submitted"] += 1
        return self._executor.submit(self._run_one, cands, geom)

    def _run_one(self, cands: Sequence, geom) -> ClustererServiceResult:
        t0 = time.perf_counter()
        try:
            labels, records = cluster_candidates(cands, geom, config=self._config)
        except Exception:
            with self._lock:
                self._n["failed"] += 1
            _LOG.exception("clustering failed for cube_id=%d (n_cands=%d)", geom.cube_id,
                           len(cands))
            raise
        wall_ms = (time.perf_counter() - t0) * 1e3
        with self._lock:
            self._n["completed"] += 1
        return ClustererServiceResult(geom.cube_id, labels, records, wall_ms)

    @property
    def n_submitted(self) -> int:
        with self._lock:
            return self._n["submitted"]

    @property
    def n_completed(self) -> int:
        with self._lock:
            return self._n["completed"]

    @property
    def n_failed(self) -> int:
        with self._lock:
            return self._n["failed"]

    @property
    def config(self) -> ClustererConfig:
        return self._config
