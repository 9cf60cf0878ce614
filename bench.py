"""Benchmark: real-time factor of the one-GPU fast search path.

A step is one voltage block (16 chgroup pages of 8192 packets x 96
antennas x 384 channels, 0.537 data-seconds) pushed through the streaming
pipeline: unpack + tensor-core correlator + per-subband gridding, stage-1
coarse dedispersion + static sky + stage-2 ring, and for every detector cube
the fine-DM combine, 2-D FFT imaging, Layer-1 noise, edge mask and the
boxcar detector.  ``value`` = data-seconds processed per wall-second (all
ranks), inputs resident in HBM; ``e2e`` is the same through the public API
from pinned host buffers (H2D inside the timed region).

``--impl reference`` times the CPU restatement of the reference algorithm
(the oracle) on the host cores on a bounded sample of the same workload.
"""

from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path[:0] = [os.path.join(ROOT, "dsa110-rt_b200"), os.path.join(ROOT, "oracle")]

METRIC = "real-time factor at 96-ant/6144-ch/2048-DM (data-seconds per second)"


def max_over_ranks(x: float, world: int, device) -> float:
    """x on this rank -> the largest x of all ranks (every rank calls it at
    the same point; one rank returns x itself)."""
    if world <= 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def agreed_status(code: int, world: int, device) -> int:
    """A device status code agreed on by every rank (the largest), so that
    all ranks raise together or none does."""
    return int(max_over_ranks(code, world, device))


def metric_for(cfg) -> str:
    """The metric's name with the workload's DM count (2048 for the default
    workload, the name above)."""
    return METRIC.replace("2048-DM", f"{cfg.fine_dm.size}-DM")


def workload_config(name: str):
    from dsb200.constants import DSA110_BAND
    from dsb200.pipeline import PipelineConfig
    if name == "dsa110-config5":
        # the metric configuration: 96 antennas / 6144 channels / 2048 DMs
        # over 0-3000 pc/cm^3, 512^2 images, boxcars 1..64, at the
        # reference's own search cadence (t_int 32 native samples = 1.049 ms
        # per tile, t_int_corr == t_int_search, configs/dsart_search_rt.yaml)
        return PipelineConfig(nant=96, band=DSA110_BAND, npkt_block=8192, t_int=32, csf=16,
                              n_grid=512, coarse_dm=np.linspace(0.0, 3000.0, 128),
                              fine_per_coarse=16, log_max_width=6, threshold=7.0,
                              chunk_tiles=512, fdm_batch=16)
    if name == "dsa110-2048dm-256":
        # the metric's 96 antennas / 6144 channels / 2048 DMs over its 0-3000
        # pc/cm^3, with the full DSA-110 shape's imaging: 256^2 grid,
        # boxcars 1..16, 262 us tiles (t_int 8)
        return PipelineConfig(nant=96, band=DSA110_BAND, npkt_block=8192, t_int=8, csf=16,
                              n_grid=256, coarse_dm=np.linspace(0.0, 3000.0, 128),
                              fine_per_coarse=16, log_max_width=4, threshold=7.0,
                              chunk_tiles=512, fdm_batch=32)
    if name == "dsa110-512dm":
        # the full DSA-110 shape as given: 512 DMs over 0-2000
        return PipelineConfig(nant=96, band=DSA110_BAND, npkt_block=8192, t_int=8, csf=16,
                              n_grid=256, coarse_dm=np.linspace(0.0, 2000.0, 32),
                              fine_per_coarse=16, log_max_width=4, threshold=7.0,
                              chunk_tiles=512, fdm_batch=8)
    if name == "medium5":
        # the per-image work of the metric configuration (96 antennas, 512^2,
        # boxcars 1..64, t_int 32) on 4 chgroups and short rings: a few GB on
        # the device, for profiling the per-image kernels
        from dsb200.constants import Band
        return PipelineConfig(nant=96, band=Band(n_chgroup=4), npkt_block=2048, t_int=32,
                              csf=16, n_grid=512, coarse_dm=np.linspace(0.0, 300.0, 8),
                              fine_per_coarse=4, log_max_width=6, threshold=7.0,
                              chunk_tiles=128, fdm_batch=8)
    if name == "medium":
        # the full per-image work (96 antennas, 16 chgroups, 256^2) on short
        # rings: a few GB on the device, for profiling the per-image kernels
        return PipelineConfig(nant=96, band=DSA110_BAND, npkt_block=512, t_int=8, csf=16,
                              n_grid=256, coarse_dm=np.linspace(0.0, 100.0, 8),
                              fine_per_coarse=4, log_max_width=4, threshold=7.0,
                              chunk_tiles=128, fdm_batch=8)
    if name == "small":
        from dsb200.constants import Band
        return PipelineConfig(nant=96, band=Band(n_chgroup=4), npkt_block=1024, t_int=8, csf=16,
                              n_grid=256, coarse_dm=np.linspace(0.0, 500.0, 8),
                              fine_per_coarse=4, log_max_width=4, threshold=7.0,
                              chunk_tiles=256, fdm_batch=8)
    raise SystemExit(f"unknown workload {name}")


def workload_desc(name, cfg):
    return {"workload": f"{name}: {cfg.nant} ant, {cfg.band.n_chgroup}x{cfg.band.nchan} ch "
                        f"(csf {cfg.csf} -> {cfg.band.n_chgroup * cfg.ceff} subbands), "
                        f"{cfg.npkt_block * 2}-sample blocks, t_int {cfg.t_int}, "
                        f"{cfg.n_grid}^2 grid, {cfg.fine_dm.size} DMs "
                        f"({cfg.coarse_dm.size} coarse x {cfg.fine_per_coarse} fine) "
                        f"0-{cfg.coarse_dm.max():.0f}, boxcars 1..{1 << cfg.log_max_width}",
            "t_img_us": cfg.t_int_us,
            "block_seconds": cfg.block_seconds, "l2": "inputs larger than L2 (19 GB/block)",
            "chunk_tiles": cfg.chunk_tiles, "fdm_batch": cfg.fdm_batch,
            "stage2_ring": {"c64": "complex64", "bf16": "bf16 re/im pairs (BF16 storage form)",
                            "cint8": "int8 re/im pairs with an amax/127 scale per row "
                                     "(cint8 wire form)"}[cfg.ring_dtype]}


class Clocks:
    """nvidia-smi clock/throttle sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        # the raw samples: DSB_CLOCKS_DIR when set, else the temp directory
        import tempfile
        self.path = os.path.join(os.environ.get("DSB_CLOCKS_DIR", tempfile.gettempdir()),
                                 f"clocks_{os.getpid()}.csv")

    def start(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}",
                                          f"--query-gpu={self.Q}", "--format=csv,noheader",
                                          "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:  # noqa: BLE001
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        self.proc.terminate()
        self.proc.wait()
        self.f.close()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            p = [x.strip() for x in line.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1].split()[0]))
                smax = float(p[2].split()[0])
            except ValueError:
                continue
            for n, v in zip(names, p[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        busy = [s for s in sm if smax and s > 0.3 * smax] or sm
        return {"sm_mhz": float(np.median(busy)) if busy else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# algorithmic work per launch (for the roofline of the dominant kernel)
# ---------------------------------------------------------------------------

# DRAM traffic of image_kernel<256, 1> (bf16 ring) measured by ncu (--set
# full, one launch) on the medium workload: 242.73 MB written for 1152
# images (the rest of the images still sat in L2 when the kernel ended),
# 49.53 MB read for 2 coarse DMs x 144 times
IMAGE_DRAM_WRITE_PER_IMAGE = 242.731776e6 / 1152
IMAGE_DRAM_READ_PER_SLICE_TIME = 49.525504e6 / (2 * 144)
# ring reads of the complex64 ring against the bf16 ring: ncu
# dram__bytes_read.sum of the same kernel on the medium workload, 99.22 MB
# (complex64) against 49.49 MB (bf16) per launch, in one paired capture
IMAGE_DRAM_READ_C64_RATIO = 99.225429e6 / 49.494272e6
# ---------------------------------------------------------------------------


def stage_work(pipe):
    cfg, T = pipe.cfg, pipe.tab
    C, N = cfg.chunk_tiles, cfg.n_grid
    nt = C + 2 * cfg.t_edge
    nb = cfg.fdm_batch
    nbase = cfg.nant * (cfg.nant + 1) // 2
    nchan = cfg.band.n_chgroup * cfg.band.nchan
    half = N * (N // 2 + 1)
    coarse_per_batch = max(1, nb // cfg.fine_per_coarse) if cfg.fine_per_coarse else nb
    esz = {"c64": 8, "bf16": 4, "cint8": 2}[cfg.ring_dtype]   # bytes per stage-2 ring cell
    # cint8: stage 1 writes complex64 rows that the quantiser reads back
    s1_out = 8 + 8 + 2 if cfg.ring_dtype == "cint8" else esz
    return {
        # tensor-core flops: 16 flops per (baseline, channel, native sample) (XX+YY complex MAC)
        "corr": ("tensor", 16.0 * nbase * nchan * C * cfg.t_int,
                 cfg.band.n_chgroup * C * cfg.t_int // 2 * cfg.nant * cfg.band.nchan * 4
                 + T.n_rows_y * C * 8),
        "stage1": ("hbm", None, T.n_rows_y * C * 8 + T.n_rows_d * C * s1_out),
        # fused combine + FFT: stage-2 ring slices of the batch's coarse DM(s)
        # read once, float32 images written once
        "image": ("hbm", None, int(T.n_filled.sum()) * coarse_per_batch * nt * esz
                  + nb * nt * N * N * 4),
        "detect": ("hbm", None, nb * nt * N * N * 4),
        "layer1": ("hbm", None, nb * cfg.l1_times * cfg.l1_pixels * 4),
    }


def measure_int8_peak(dev) -> float:
    """Dense int8 tensor throughput of this GPU (TOP/s): cuBLASLt's int8 GEMM
    (torch._int_mm) on 8192^3, best of 10 -- the denominator of the
    correlator's roofline (2 x 8192^3 ops per call)."""
    import torch
    n = 8192
    a = torch.randint(-8, 8, (n, n), dtype=torch.int8, device=dev)
    b = torch.randint(-8, 8, (n, n), dtype=torch.int8, device=dev)
    for _ in range(3):
        torch._int_mm(a, b)
    best = float("inf")
    for _ in range(10):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch._int_mm(a, b)
        e1.record()
        torch.cuda.synchronize(dev)
        best = min(best, e0.elapsed_time(e1) / 1e3)
    del a, b
    return 2.0 * n ** 3 / best / 1e12


# DRAM bytes per unit of work of the 512^2 kernels (bf16 ring), from the ncu
# captures of the medium5 workload (profiles/): image_kernel<512, 1> wrote
# 1558.412 MB for 1536 images and read 28.509 MB for 2 coarse DMs x 192
# times x 4 chgroups; detect_tma_kernel<6> read 1611.367 MB and wrote
# 16.182 MB (candidates, Layer-2 samples, register spills) for 1536 images
IMAGE512_DRAM_WRITE_PER_IMAGE = 1558.412e6 / 1536
IMAGE512_DRAM_READ_PER_SLICE_TIME_CHGROUP = 28.509e6 / (2 * 192 * 4)
DETECT64_DRAM_PER_IMAGE = (1611.367e6 + 16.182e6) / 1536


def stage_traffic(pipe) -> dict:
    """Measured DRAM bytes per launch (ncu, scaled from a capture of the same
    kernel on a smaller case by its units of work) where one was taken."""
    cfg = pipe.cfg
    out = {}
    nt = cfg.chunk_tiles + 2 * cfg.t_edge
    nb = cfg.fdm_batch
    if cfg.n_grid == 512 and cfg.ring_dtype == "bf16":
        cpb = max(1, nb // cfg.fine_per_coarse)
        out["image"] = (IMAGE512_DRAM_WRITE_PER_IMAGE * nb * nt +
                        IMAGE512_DRAM_READ_PER_SLICE_TIME_CHGROUP * cpb * nt * cfg.band.n_chgroup,
                        "ncu dram__bytes_read.sum + dram__bytes_write.sum of image_kernel<512> on "
                        "medium5 (1536 images), scaled by images written and ring slices read")
    if cfg.log_max_width == 6:
        out["detect"] = (DETECT64_DRAM_PER_IMAGE * nb * nt * (cfg.n_grid / 512) ** 2,
                         "ncu dram__bytes_read.sum + dram__bytes_write.sum of detect_tma_kernel<6> "
                         "on medium5 (1536 images of 512^2), scaled by image bytes read")
    if cfg.n_grid == 256 and cfg.ring_dtype != "cint8":
        cpb = max(1, nb // cfg.fine_per_coarse)
        rd = IMAGE_DRAM_READ_PER_SLICE_TIME * (IMAGE_DRAM_READ_C64_RATIO
                                                if cfg.ring_dtype == "c64" else 1.0)
        out["image"] = (IMAGE_DRAM_WRITE_PER_IMAGE * nb * nt + rd * cpb * nt,
                        "ncu dram bytes of image_kernel<256> on the medium workload (1152 "
                        "images), scaled to this launch")
    return out


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), float(d["bf16_tflops"]), "measured"
    return 6650.0, 1590.0, "fallback"


# ---------------------------------------------------------------------------
# CPU baseline: the oracle (restatement of the reference algorithm) on a
# bounded sample, extrapolated per data-second stage by stage
# ---------------------------------------------------------------------------


def cpu_baseline(cfg, threads: int, budget_s: float = 20.0):
    import dsb_oracle as O
    try:
        import threadpoolctl
        limiter = threadpoolctl.threadpool_limits(threads)
    except Exception:  # noqa: BLE001
        limiter = None
    rng = np.random.default_rng(0)
    G, C = cfg.band.n_chgroup, cfg.band.nchan
    tiles_per_s = 1e6 / cfg.t_int_us
    out = {}
    # correlator: one chgroup page, 8 tiles
    npkt = 8 * cfg.t_int // 2
    raw = rng.integers(0, 256, npkt * cfg.nant * C * 4, dtype=np.uint8)
    t0 = time.perf_counter()
    vr, vi = O.corr_fast_from_raw(raw, npkt=npkt, nant=cfg.nant, nchan=C, t_int=cfg.t_int,
                                  csf=cfg.csf)
    out["corr"] = (time.perf_counter() - t0) * G * tiles_per_s / 8
    # stage 1: one chgroup, one coarse DM, 64 tiles
    nbase = cfg.nant * (cfg.nant + 1) // 2
    ceff = C // cfg.csf
    n_filled = 2000
    cim = rng.integers(0, n_filled + 1, (nbase, ceff))
    vis = rng.integers(-50, 51, (64 + 32, nbase, ceff))
    sh = rng.integers(0, 32, (ceff, 1))
    t0 = time.perf_counter()
    O.stage1_dedisp(vis, sh, cim, n_filled, 64)
    out["stage1"] = (time.perf_counter() - t0) * 2 * G * cfg.coarse_dm.size * tiles_per_s / 64
    # search: one fine DM x 32 images: combine + FFT + boxcar detector
    N = cfg.n_grid
    streams = (rng.normal(size=(G, 32, N, N)) + 1j * rng.normal(size=(G, 32, N, N)))
    t0 = time.perf_counter()
    half = O.combine_half(streams, np.zeros(G, np.int64), 32, 0)
    img = O.image_from_half(half, N).astype(np.float32)
    mw = 1 << cfg.log_max_width
    cs = O.padded_cumsum(img[:, None], mw)
    widths = [1 << k for k in range(cfg.log_max_width + 1)]
    O.multi_boxcar_argmax(cs, widths, O.boxcar_offsets(widths, mw),
                          np.ones(len(widths), np.float32), 32 - mw, mw // 2)
    out["search"] = (time.perf_counter() - t0) * cfg.fine_dm.size * tiles_per_s / 32
    if limiter is not None:
        limiter.unregister() if hasattr(limiter, "unregister") else None
    sec_per_data_s = sum(out.values())
    return {"value": 1.0 / sec_per_data_s, "unit": "data-seconds/s", "cores": threads,
            "kind": "port",
            "sample": ("oracle (numpy restatement of the reference algorithm): correlator on one "
                       "chgroup page x 8 tiles, stage 1 on one chgroup x one coarse DM x 64 tiles, "
                       "combine+FFT+boxcars for one fine DM x 32 images; each stage's CPU seconds "
                       "scaled to one data-second of the full workload and summed"),
            "cpu_seconds_per_data_second": {k: round(v, 3) for k, v in out.items()}}


def _ref_import_path():
    """baseline/_ref: the unmodified reference, pip-installed (no deps)
    beside this file; it travels with the repository, the reference's own
    checkout does not."""
    p = os.path.join(ROOT, "baseline", "_ref")
    return p if os.path.isdir(os.path.join(p, "dsart")) else None


def cpu_model() -> str:
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


_REF_CACHE: dict = {}


def reference_cpu_chain(cfg, threads: int):
    """The reference's own CPU implementation of the path (the unmodified
    dsa110-rt from baseline/_ref, through its public functions), timed stage
    by stage on a bounded sample of the workload and scaled to one
    data-second; the stages are the ones the reference's CPU path runs:

      unpack_int4_split (slow_corr_kernel.py:220), one full 2048-packet page
      FastCorrKernel.compute_split, Stokes I + channel sum (corr_fast_kernel.py:364)
      Stage1MultiDMCoarseDM.dedisperse_from_vis on CPU = its
        _dedisperse_one_window_phase9_cpu (corr_fast_integration.py:647, :917)
      Stage2InterChgroupShiftFifo.push (stage2_chgroup_alignment.py:264)
      combine_chgroups (fine_dm/combiner.py:548)
      dirty_image_from_uv_grid + apply_edge_mask (image/imager.py:248, :304)
      precompute_padded_cumsum + boxcar_from_padded_cumsum per width, the
        strict-'>' max, decode_topk_argmax_lowmem (detector/forward.py:250,
        :339; detector/decoder.py:388)

    The reference runs only at its own geometry (96 antennas, 16 x 384
    channels), which is the workload's.  Its stage-1 plan is its synthetic
    summed plan (build_synthetic_summed_plan: the workload's coarse-DM count
    and range, zero shifts; the gather and scatter work is the same).
    Inputs and one-time set-up (pattern, gridder, plan) are built on the
    first call and kept: later calls time only the stages."""
    import torch
    ref = _ref_import_path()
    if ref is None:
        raise RuntimeError("baseline/_ref is not installed")
    if ref not in sys.path:
        sys.path.insert(0, ref)
    torch.set_num_threads(threads)
    from dsart.coarse_dm.stage2_chgroup_alignment import Stage2InterChgroupShiftFifo
    from dsart.coarse_dm.stage2_shifts import compute_stage2_shifts
    from dsart.coarse_dm.synthetic_plan import build_synthetic_summed_plan
    from dsart.detector.decoder import decode_topk_argmax_lowmem
    from dsart.detector.forward import boxcar_from_padded_cumsum, precompute_padded_cumsum
    from dsart.fine_dm.combiner import combine_chgroups
    from dsart.grid.kernel import FastVisGridder
    from dsart.grid.sparsity_pattern import build_pattern, compute_top_of_band_cell_lambda
    from dsart.image.imager import apply_edge_mask, compute_edge_mask, dirty_image_from_uv_grid
    from dsart.services.corr_fast_integration import Stage1MultiDMCoarseDM
    from dsart.services.corr_fast_kernel import FastCorrKernel
    from dsart.services.slow_corr_kernel import unpack_int4_split
    from dsb200 import synth

    if cfg.nant != 96 or cfg.band.nchan != 384 or cfg.band.n_chgroup != 16:
        raise RuntimeError("the reference runs only at 96 antennas / 16 x 384 channels")
    G, N = cfg.band.n_chgroup, cfg.n_grid
    tiles_per_s = 1e6 / cfg.t_int_us
    n_fine, n_coarse = cfg.fine_dm.size, cfg.coarse_dm.size
    rng = np.random.default_rng(0)
    sec = {}
    clock = time.perf_counter
    key = (N, cfg.t_int, cfg.csf, n_coarse, float(cfg.coarse_dm.max()))
    cache = _REF_CACHE.setdefault(key, {})
    # 1-2: one full page (2048 packets = 4096 samples) of one chgroup
    npkt = 2048
    if "raw" not in cache:
        cache["raw"] = rng.integers(0, 256, npkt * 96 * 384 * 4, dtype=np.uint8)
    raw = cache["raw"]
    pages_per_s = G * 1e6 / (2 * npkt * 32.768)
    t0 = clock()
    re, im = unpack_int4_split(raw, device="cpu", out_dtype=torch.float32)
    sec["unpack"] = (clock() - t0) * pages_per_s
    k = FastCorrKernel(device="cpu", t_int_fast_native=cfg.t_int, nants=96, nchan=384)
    t0 = clock()
    vis = k.compute_split(re, im, fuse_stokes_i=True, chan_sum_factor=cfg.csf)
    sec["corr"] = (clock() - t0) * pages_per_s
    del re, im
    n_fv = vis.shape[0]
    # 3: stage 1 of one chgroup's window over a subset of its coarse DMs
    g = G - 1
    if "grd" not in cache:
        e, n = synth.t_layout(96, seed=11)
        cell = compute_top_of_band_cell_lambda(e, n, n_grid=N)
        pat = build_pattern(e, n, chgroup=g, dec_deg=37.0, n_grid=N, chan_sum_factor=cfg.csf,
                            cell_lambda=cell)
        cache["grd"] = FastVisGridder.from_pattern(pat, e, n, device="cpu")
        cache["plan"] = build_synthetic_summed_plan(
            n_coarse=n_coarse, dm_max=float(cfg.coarse_dm.max()), chan_sum_factor=cfg.csf,
            t_int_fast_us=cfg.t_int_us)
    grd, plan = cache["grd"], cache["plan"]
    n_dm_s = min(8, n_coarse)
    st = Stage1MultiDMCoarseDM(plan=plan, gridder=grd, chgroup=g,
                               dm_indices=np.arange(n_dm_s), sliding_window=False)
    vis = vis.to(torch.complex64).contiguous()
    t0 = clock()
    dd = st.dedisperse_from_vis(vis, block_n=0)
    sec["stage1"] = (clock() - t0) * (n_coarse / n_dm_s) * G * tiles_per_s / n_fv
    # 4: the stage-2 FIFO of that chgroup (two pushes; the first seeds it)
    cd = cfg.coarse_dm[:n_dm_s]
    tab = compute_stage2_shifts(chgroup=g, coarse_dm_pc_cm3=cd, t_int_corr_us=cfg.t_int_us)
    fifo = Stage2InterChgroupShiftFifo(chgroup=g, coarse_dm_pc_cm3=cd, t_dedisp=dd.shape[1],
                                       t_int_corr_us=cfg.t_int_us, shift_table=tab)
    fifo.push(dd, block_n=0)
    t0 = clock()
    fifo.push(dd, block_n=1)
    sec["stage2_fifo"] = (clock() - t0) * (n_coarse / n_dm_s) * G * tiles_per_s / dd.shape[1]
    del vis, dd
    # 5-6: combine + image of one fine DM over 8 times
    nt = 8
    if "streams" not in cache:
        cache["streams"] = {gg: (rng.standard_normal((nt, N, N), np.float32)
                                 + 1j * rng.standard_normal((nt, N, N), np.float32)
                                 ).astype(np.complex64) for gg in range(G)}
    streams = cache["streams"]
    shifts = np.zeros(G, np.int32)
    t0 = clock()
    uv = combine_chgroups(per_chgroup_streams=streams, time_shift_per_chgroup=shifts,
                          t_window=(0, nt))
    sec["combine"] = (clock() - t0) * n_fine * tiles_per_s / nt
    mask = compute_edge_mask(n_grid=N, kernel_support=1)
    t0 = clock()
    img = apply_edge_mask(dirty_image_from_uv_grid(uv), mask)
    sec["image"] = (clock() - t0) * n_fine * tiles_per_s / nt
    del uv, img
    # 7: the detector on one fine DM's cube of up to 128 output times
    te, mw = cfg.t_edge, 1 << cfg.log_max_width
    n_out = min(cfg.chunk_tiles, 128)
    if "cube" not in cache:
        cache["cube"] = torch.from_numpy(
            rng.standard_normal((n_out + 2 * te, 1, N, N), np.float32))
    cube = cache["cube"]
    widths = [1 << i for i in range(cfg.log_max_width + 1)]
    sinv = [1.0 / np.sqrt(w) for w in widths]
    t0 = clock()
    cs = precompute_padded_cumsum(cube, axis=0, max_width=mw)
    best = win = None
    for kk, (w, si) in enumerate(zip(widths, sinv)):
        b = boxcar_from_padded_cumsum(cs, axis=0, width=w, max_width=mw, n_out=n_out,
                                      t_base=te) * si
        if best is None:
            best, win = b, torch.zeros(b.shape, dtype=torch.int16)
        else:
            better = b > best
            best = torch.where(better, b, best)
            win = torch.where(better, torch.full_like(win, kk), win)
    decode_topk_argmax_lowmem(best, win, threshold=cfg.threshold,
                              kernel_ids=[f"unit_d1_b{w}" for w in widths],
                              kernel_time_widths=widths, merge_radius_lm=cfg.merge_radius_lm,
                              merge_radius_fdm=cfg.merge_radius_fdm,
                              merge_radius_t=cfg.merge_radius_t, n_top=cfg.decoder_n_top)
    sec["detect"] = (clock() - t0) * n_fine * tiles_per_s / n_out
    total = sum(sec.values())
    return {"value": 1.0 / total, "unit": "data-seconds/s", "cores": threads,
            "kind": "reference",
            "torch_threads": torch.get_num_threads(), "os_cpu_count": os.cpu_count(),
            "cpu_model": cpu_model(),
            "sample": ("the unmodified reference (baseline/_ref) on the host cores: unpack + "
                       "correlator on one 2048-packet chgroup page, stage 1 + stage-2 FIFO on "
                       f"one chgroup x {n_dm_s} coarse DMs x {n_fv} tiles, combine + image of "
                       f"one fine DM x {nt} times, detector on one fine DM x {n_out} output "
                       "times; each stage's CPU seconds scaled to one data-second of the "
                       "workload and summed"),
            "cpu_seconds_per_data_second": {k_: round(v, 3) for k_, v in sec.items()}}


# ---------------------------------------------------------------------------


def serve_main(a, cfg):
    """Served streaming form: ``a.serve`` independent voltage streams on one
    GPU through ``dsb200.serve.StreamServer``.  Stream i delivers
    ``a.serve_blocks`` blocks of a seeded uneven length of 1-8 chunks
    (4096-32768 samples) with Poisson arrivals at (i mod 4 + 1) x real time;
    block copies are admitted under a device budget of two of the largest
    blocks, or what HBM holds beside the resident pipelines.  Bursts arrive
    in every stream at 0.5 per data-second (Poisson),
    DM uniform 50-2000, S/N uniform 7-40, 4 search samples wide, at seeded
    pixels; each block's bursts are drawn into its device copy before the
    search (the server's ``prepare`` hook), with amplitudes set from one
    reference burst measured first.  Reports the sustained real-time factor
    (data-seconds of all streams per wall-second, first arrival to last
    candidate), the p50/p99 arrival-to-candidate latency, and the fraction of
    bursts recovered."""
    import threading
    import torch
    from dsb200 import synth
    from dsb200.pipeline import SearchPipeline
    from dsb200.serve import StreamServer

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    S = a.serve
    e, n = synth.t_layout(cfg.nant, seed=11)
    ti = cfg.t_int
    # amplitude scale from one reference burst in a stream of its own
    noise = [synth.random_block_device(band=cfg.band, nant=cfg.nant, npkt=cfg.npkt_block,
                                       device=dev, seed=900 + i) for i in range(2)]
    ref = _reference_burst(cfg, e, n, noise, torch.empty_like(noise[0]), amp_ref=0.09)
    del noise
    torch.cuda.empty_cache()

    pipes = [SearchPipeline(cfg, e, n, device=dev) for _ in range(S)]
    for p in pipes:
        p.skip_warmup()
    k0 = pipes[0].chunk
    C = cfg.chunk_tiles
    per_chunk = C * cfg.t_int // 2                     # packets per chunk
    chunk_samp = 2 * per_chunk
    chunk_s = chunk_samp * 32.768e-6                   # data-seconds per chunk
    max_k = 8
    # one pinned host source of the largest block, shared (read-only) by all
    # streams; a k-chunk block is its contiguous prefix viewed as k-chunk pages
    src = synth.random_block_device(band=cfg.band, nant=cfg.nant, npkt=max_k * per_chunk,
                                    device=dev, seed=7).cpu().pin_memory().reshape(-1)
    page_shape = (cfg.nant, cfg.band.nchan, 2, 2)
    G = cfg.band.n_chgroup

    def block(k):
        npkt = k * per_chunk
        return src[:G * npkt * cfg.nant * cfg.band.nchan * 4].view(G, npkt, *page_shape)
    rng = np.random.default_rng(2024)
    plan = []                                          # (arrival s, stream, chunks)
    offsets = [[] for _ in range(S)]                   # first native sample of each block
    for i in range(S):
        rate = i % 4 + 1
        t, s0 = 0.0, 0
        for _ in range(a.serve_blocks):
            k = int(rng.integers(1, max_k + 1))
            t += rng.exponential(k * chunk_s / rate)
            plan.append((t, i, k))
            offsets[i].append(s0)
            s0 += k * chunk_samp
        offsets[i].append(s0)
    plan.sort()
    # bursts: Poisson at 0.5 per data-second of each stream, after the rings fill
    k_bot = _delay_per_dm(cfg.band)
    lat_chunks = pipes[0].depth1 + pipes[0].a + 2
    warm = int(k_bot * float(cfg.coarse_dm.max())) + chunk_samp
    bursts, grid = [], []
    for i in range(S):
        total = offsets[i][-1]
        tb = warm + rng.exponential(1.0 / 0.5) / 32.768e-6
        bi, gi = [], []
        while True:
            dm = float(rng.uniform(50.0, 2000.0))
            snr = float(rng.uniform(7.0, 40.0))
            w = 4 * ti
            end_chunk = (tb + k_bot * dm + w) / chunk_samp + lat_chunks
            if end_chunk >= total / chunk_samp:
                break
            dl, dmp = (int(v) for v in rng.integers(-(cfg.n_grid // 2 - 8), cfg.n_grid // 2 - 7, 2))
            amp = synth.amp_for_snr(snr, w, amp_ref=ref["amp"], snr_ref=ref["snr"],
                                    width_ref=ref["width_native"])
            bi.append(synth.Burst(dm=dm, t0_native=int(tb), width_native=w, amp=amp, dl=dl,
                                  dm_pix=dmp))
            gi.append((snr, w, dm, int(tb), dl, dmp))
            tb += rng.exponential(1.0 / 0.5) / 32.768e-6
        bursts.append(bi)
        grid.append(gi)

    def prepare(i, k, blk):
        s0 = offsets[i][k]
        n_samp = 2 * blk.shape[1]
        mine = [b for b in bursts[i] if b.t0_native < s0 + n_samp and
                b.t0_native + k_bot * b.dm + b.width_native + 8 > s0]
        if mine:
            synth.inject_bursts_device(blk, band=cfg.band, nant=cfg.nant, s0=s0, bursts=mine,
                                       antpos_e=e, antpos_n=n,
                                       cell_lambda=pipes[i].tab.cell_lambda, n_grid=cfg.n_grid,
                                       seed=31 + i)

    # two of the largest blocks, or what the device has left beside the
    # resident pipelines (less 8 GB of working room), at least one block
    free, _ = torch.cuda.mem_get_info(dev)
    budget = min(2 * src.numel(), free - (8 << 30))
    if budget < src.numel():
        raise SystemExit(f"serve: {free / 1e9:.1f} GB free cannot hold one "
                         f"{src.numel() / 1e9:.1f} GB block beside the pipelines")
    srv = StreamServer(pipes, budget, prepare=prepare).start()
    t0 = time.perf_counter()

    def feed():
        for t_arr, i, k in plan:
            dt = t0 + t_arr - time.perf_counter()
            if dt > 0:
                time.sleep(dt)
            srv.submit(i, block(k), t_arrival=time.perf_counter())
        srv.close()

    th = threading.Thread(target=feed)
    th.start()
    th.join()
    srv.join(3600)
    wall = max(r.t_done for rs in srv.results for r in rs) - t0
    for p in pipes:
        p.check_status()
    data_s = sum(k for _, _, k in plan) * chunk_s
    lat = np.asarray(srv.latencies_s()) * 1e3
    found = []
    for i in range(S):
        cands = [c for r in srv.results[i] for c in r.candidates]
        # the streams started in steady state (skip_warmup): their first
        # sample is search sample k0 * C of the pipeline's clock
        off = k0 * C * ti
        found += synth.match_bursts([(a_, w_, d_, t_ + off, l_, m_)
                                     for a_, w_, d_, t_, l_, m_ in grid[i]], cands,
                                    band=cfg.band, fine_dm=cfg.fine_dm, n_grid=cfg.n_grid, t_int=ti)
    print(json.dumps({
        "metric": "served streaming: sustained real-time factor (data-seconds of all streams "
                  "per wall-second) and arrival-to-candidate latency",
        "value": data_s / wall, "unit": "data-seconds/s", "n_gpus": 1, "streams": S,
        "higher_is_better": True, "blocks": len(plan), "data_seconds": data_s,
        "wall_s": wall, "latency_ms": {"p50": float(np.percentile(lat, 50)),
                                       "p99": float(np.percentile(lat, 99))},
        "offered_load_x_realtime": float(sum(i % 4 + 1 for i in range(S))),
        "device_budget_bytes": budget, "budget_peak_bytes": srv.budget.peak,
        "bursts": {"injected": len(found), "recovered": int(sum(q is not None for q in found)),
                   "reference_burst": ref},
        "config": dict(workload_desc(a.workload, cfg),
                       blocks="seeded 1-8 chunks (4096-32768 samples), Poisson arrivals at "
                              "1-4x real time per stream",
                       bursts="0.5 per data-second per stream, DM U(50, 2000), S/N U(7, 40), "
                              "4 search samples wide"),
        "data": "synthetic (seeded 4-bit Gaussian voltages, bursts drawn in on the device)"}))


def _delay_per_dm(band) -> float:
    """Native samples of dispersion delay per unit DM between the top and the
    bottom of the band."""
    nu = band.freq_table()
    return 4.148808 * (1.0 / float(nu.min()) ** 2 - 1.0 / float(nu[0, 0]) ** 2) * 1e3 / 32.768


def _injected_stream(cfg, e, n, noise, work, bursts, n_blocks, seed):
    """A fresh ``SearchPipeline`` over ``n_blocks`` blocks, block k a copy of
    ``noise[k % len(noise)]`` with the bursts that cover it drawn in
    (``inject_bursts_device``).  Returns (candidates, device ms in
    ``process_block``, fine DMs)."""
    import torch
    from dsb200 import synth
    from dsb200.pipeline import SearchPipeline
    dev = work.device
    blk = 2 * cfg.npkt_block
    k_bot = _delay_per_dm(cfg.band)
    pipe = SearchPipeline(cfg, e, n, device=dev)
    cell = pipe.tab.cell_lambda
    cands, dev_ms = [], 0.0
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    for k in range(n_blocks):
        s0 = k * blk
        work.copy_(noise[k % len(noise)])
        mine = [b for b in bursts if b.t0_native < s0 + blk and
                b.t0_native + k_bot * b.dm + b.width_native + 8 > s0]
        synth.inject_bursts_device(work, band=cfg.band, nant=cfg.nant, s0=s0, bursts=mine,
                                   antpos_e=e, antpos_n=n, cell_lambda=cell,
                                   n_grid=cfg.n_grid, seed=seed)
        ev0.record()
        got = pipe.process_block(work)
        ev1.record()
        torch.cuda.synchronize()
        dev_ms += ev0.elapsed_time(ev1)
        cands += got
    pipe.check_status()
    fine = pipe.cfg.fine_dm
    del pipe
    torch.cuda.empty_cache()
    return cands, dev_ms, fine


def _reference_burst(cfg, e, n, noise, work, amp_ref, dm=1000.0, width_search=4):
    """Measure the S/N of one burst of amplitude ``amp_ref`` (``width_search``
    search samples, DM ``dm``) in a stream of its own: the scale from which
    ``synth.amp_for_snr`` sets every injected burst's amplitude."""
    from dsb200 import synth
    blk = 2 * cfg.npkt_block
    ti = cfg.t_int
    warm = max(4 * blk, int(_delay_per_dm(cfg.band) * float(cfg.coarse_dm.max())) + blk)
    ref = (0.0, width_search * ti, float(dm), warm + blk // 3, 40 % (cfg.n_grid // 4),
           -(60 % (cfg.n_grid // 4)))
    rb = [synth.Burst(dm=ref[2], t0_native=ref[3], width_native=ref[1], amp=amp_ref,
                      dl=ref[4], dm_pix=ref[5])]
    n_blocks = int(np.ceil((ref[3] + _delay_per_dm(cfg.band) * dm + ref[1]) / blk)) + 3
    rc, _, fine = _injected_stream(cfg, e, n, noise, work, rb, n_blocks, seed=77)
    m = synth.match_bursts([ref], rc, band=cfg.band, fine_dm=fine, n_grid=cfg.n_grid, t_int=ti)
    if m[0] is None:
        raise SystemExit("the reference burst was not detected")
    return {"amp": amp_ref, "width_native": ref[1], "dm": float(dm), "snr": float(m[0].snr)}


def stress_main(a):
    """Stress/recovery sweep of the metric configuration: 200 bursts on an
    S/N grid 6-50 x width grid 1-32 search samples x DM grid 100-2900,
    arriving 0.3 s apart over a 60-data-second stream of seeded noise, at
    seeded random pixels.  The amplitude for each (S/N, width) follows from
    one reference burst measured first in a stream of its own
    (``dsb200.synth.amp_for_snr``: S/N ~ amp^2 sqrt(width)).  Blocks are
    replayed back to back (as fast as the GPU takes them); each is a copy of
    one of three resident noise blocks with the bursts that cover it drawn
    in (``inject_bursts_device``).  Reports the fraction of bursts
    recovered (a candidate at the burst's pixel +-2, DM +-10 % (at least 30)
    and time, ``match_bursts``), by S/N, width and DM, and the measured S/N
    against the injected.  The candidate lists of a reduced sweep are checked
    against the oracle on the same seeds in the test suite; at this size
    the oracle does not run.  Prints its own JSON line."""
    import torch
    from dsb200 import synth

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    cfg = workload_config(a.workload)
    cfg.ring_dtype = a.ring
    e, n = synth.t_layout(cfg.nant, seed=11)
    npkt = cfg.npkt_block
    blk = 2 * npkt                                       # native samples per block
    noise = [synth.random_block_device(band=cfg.band, nant=cfg.nant, npkt=npkt, device=dev,
                                       seed=900 + i) for i in range(3)]
    work = torch.empty_like(noise[0])
    k_bot = _delay_per_dm(cfg.band)
    warm = 4 * blk                                       # rings full before the first burst

    def blocks_for(t_last, dm_max, w_max):
        return int(np.ceil((t_last + k_bot * dm_max + w_max) / blk)) + 3

    ti = cfg.t_int
    ref = _reference_burst(cfg, e, n, noise, work, amp_ref=0.06)

    snrs = [6, 7, 8, 10, 12, 15, 20, 30, 40, 50]
    widths = [1, 4, 16, 32]                              # search samples
    dms = [100.0, 800.0, 1500.0, 2200.0, 2900.0]
    spacing = int(round(0.3 / (32.768e-6)))
    grid = synth.burst_grid(snrs=snrs, widths=[w * ti for w in widths], dms=dms,
                            t_first_native=warm, spacing_native=spacing, n_grid=cfg.n_grid,
                            seed=2024)
    amps = [synth.amp_for_snr(s, w, amp_ref=ref["amp"], snr_ref=ref["snr"],
                              width_ref=ref["width_native"]) for s, w, *_ in grid]
    bursts = [synth.Burst(dm=d, t0_native=t0, width_native=w, amp=am, dl=dl, dm_pix=dp)
              for (s, w, d, t0, dl, dp), am in zip(grid, amps)]
    n_blocks = blocks_for(max(g[3] for g in grid), max(dms),
                          max(widths) * ti)
    cands, dev_ms, fine = _injected_stream(cfg, e, n, noise, work, bursts, n_blocks, seed=2024)
    got = synth.match_bursts(grid, cands, band=cfg.band, fine_dm=fine, n_grid=cfg.n_grid,
                             t_int=ti)

    def frac(sel):
        idx = [i for i, g in enumerate(grid) if sel(g)]
        return {"n": len(idx), "recovered": float(np.mean([got[i] is not None for i in idx]))}
    ratio = [float(q.snr) / g[0] for g, q in zip(grid, got) if q is not None]
    data_s = n_blocks * cfg.block_seconds
    # a cube decodes its top cells before merging them (the reference's
    # decoder), so a bright burst can take every decoded cell of a cube that
    # a fainter one shares: count the misses that share a cube with a
    # stronger burst
    cube = [int((g[3] + k_bot * g[2]) / ti // cfg.chunk_tiles) for g in grid]
    shaded = [any(cube[j] == cube[i] and grid[j][0] > grid[i][0] for j in range(len(grid)))
              for i in range(len(grid))]
    crowded = sum(1 for i, q in enumerate(got) if q is None and shaded[i])
    alone = [i for i in range(len(grid)) if not shaded[i]]
    print(json.dumps({
        "metric": "stress/recovery sweep: fraction of injected bursts recovered",
        "value": float(np.mean([q is not None for q in got])), "unit": "fraction",
        "higher_is_better": True, "n_gpus": 1, "n_bursts": len(grid),
        "recovered_at_or_above_snr_8": frac(lambda g: g[0] >= 8)["recovered"],
        "by_snr": {str(s): frac(lambda g, s=s: g[0] == s) for s in snrs},
        "by_width_search_samples": {str(w): frac(lambda g, w=w: g[1] == w * ti) for w in widths},
        "by_dm": {str(d): frac(lambda g, d=d: g[2] == d) for d in dms},
        "measured_over_injected_snr": {"median": float(np.median(ratio)),
                                       "p10": float(np.percentile(ratio, 10)),
                                       "p90": float(np.percentile(ratio, 90))},
        "reference_burst": ref,
        "missed": int(sum(q is None for q in got)),
        "missed_sharing_a_cube_with_a_stronger_burst": int(crowded),
        "without_a_stronger_burst_in_their_cube": {
            "n": len(alone),
            "recovered": float(np.mean([got[i] is not None for i in alone])) if alone else None,
            "recovered_at_or_above_snr_8": float(np.mean(
                [got[i] is not None for i in alone if grid[i][0] >= 8])) if alone else None},
        "decoder_n_top": cfg.decoder_n_top,
        "candidates": len(cands), "blocks": n_blocks, "data_seconds": data_s,
        "device_seconds": dev_ms / 1e3, "real_time_factor": data_s / (dev_ms / 1e3),
        "config": dict(workload_desc(a.workload, cfg),
                       sweep="S/N {6..50} x width {1,4,16,32} search samples x DM {100..2900}, "
                             "200 bursts 0.3 s apart, seeded pixels; blocks replayed back to "
                             "back"),
        "data": "synthetic (seeded 4-bit Gaussian noise blocks, sigma 3, bursts drawn in)"}))


def batched_main(a):
    """Batched form: six channel groups of uneven size (512-1536 channels),
    sub-arrays of 96, 64 and 48 antennas and DM plans of 128-1024 trials
    (``dsb200.batched.config3_groups``) advanced together, one CUDA graph of
    every group's launches per 16384-sample block.  With ``--autotune`` each
    group's tile shapes are chosen by ``dsb200.batched.autotune`` first.
    Times K blocks with the graph and K without (the same launches issued
    one by one), and an end-to-end pass with every group's block copied
    from pinned host memory inside the timed region.  Prints its own JSON
    line."""
    import torch
    from dsb200 import synth
    from dsb200.batched import BatchedSearch, autotune, config3_groups

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    groups = config3_groups()
    tuned = []
    if a.autotune:
        new = []
        for cfg, e, n in groups:
            best, table = autotune(cfg, e, n, device=dev, blocks=2)
            tuned.append({"fdm_batch": best.fdm_batch, "stage1_dm_group": best.stage1_dm_group,
                          "ms_per_block": {f"{k[0]}x{k[1]}": v for k, v in table.items()}})
            new.append((best, e, n))
        groups = new
    blocks = [synth.random_block_device(band=c.band, nant=c.nant, npkt=c.npkt_block, device=dev,
                                        seed=100 + i) for i, (c, _, _) in enumerate(groups)]
    block_s = groups[0][0].block_seconds
    out = {}
    for graph in (True, False):
        bs = BatchedSearch(groups, device=dev, use_graph=graph)
        bs.skip_warmup()
        for _ in range(a.warmup):
            bs.process_block(blocks)
        torch.cuda.synchronize()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        ev0.record()
        for _ in range(a.steps):
            bs.process_block(blocks)
        ev1.record()
        torch.cuda.synchronize()
        bs.check_status()
        out[graph] = ev0.elapsed_time(ev1) / a.steps
        launches = sum(p.launches for p in bs.pipes)
        if graph:
            n_launch = launches // (a.warmup + a.steps)
            host = [torch.empty(b.shape, dtype=torch.uint8, pin_memory=True).copy_(b)
                    for b in blocks]
            dbuf = blocks
            ev0.record()
            for _ in range(a.steps):
                for h, d in zip(host, dbuf):
                    d.copy_(h, non_blocking=True)
                bs.process_block(dbuf)
            ev1.record()
            torch.cuda.synchronize()
            bs.check_status()
            ms_e2e = ev0.elapsed_time(ev1) / a.steps
            h2d = sum(b.numel() for b in blocks)
            d2h = sum(p.last_d2h_bytes for p in bs.pipes)
            del host
        bs.close()
        del bs
        torch.cuda.empty_cache()
    print(json.dumps({
        "metric": "batched form: real-time factor (data-seconds of the whole band per "
                  "device-second)", "value": block_s / (out[True] / 1e3),
        "unit": "data-seconds/s", "n_gpus": 1, "steps": a.steps, "warmup": a.warmup,
        "ms_per_step": out[True], "ms_per_step_without_graph": out[False],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "gpu_launches": n_launch, "graph_launches_per_step": 1,
        "e2e": {"value": block_s / (ms_e2e / 1e3), "unit": "data-seconds/s",
                "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h)},
        "autotune": tuned or None,
        "config": {"workload": "batched: 6 channel groups (512, 768, 1024, 1024, 1280, 1536 ch "
                               "as 256-channel chgroups, csf 16), sub-arrays 96/96/64/64/48/48 "
                               "ant, DM plans 128/256/512/512/768/1024 trials to 500-3000, "
                               "16384-sample blocks, t_int 8, 256^2 grid, boxcars 1..16",
                   "groups": [{"nant": c.nant, "chans": c.band.n_chgroup * c.band.nchan,
                               "n_dm": int(c.fine_dm.size), "max_dm": float(c.coarse_dm.max()),
                               "fdm_batch": c.fdm_batch, "stage1_dm_group": c.stage1_dm_group}
                              for c, _, _ in groups],
                   "l2": "inputs larger than L2 (every group's block resident, "
                         f"{sum(b.numel() for b in blocks) / 1e9:.1f} GB)"},
        "dtype": "int8 (correlator) / bf16 ring, f32 accumulate",
        "data": "synthetic (seeded 4-bit Gaussian voltages, sigma 3, T-layout antennas)"}))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=6)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="dsa110-config5")
    ap.add_argument("--ring", default="bf16", choices=["c64", "bf16", "cint8"],
                    help="stage-2 ring element: the BF16 storage form (bf16 re/im, float32 "
                         "accumulation; the precision form of the full DSA-110 shape), "
                         "complex64, or the cint8 wire form (int8 re/im, a scale per row)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--stage-times", action="store_true", help="print per-stage device times")
    ap.add_argument("--serve", type=int, default=0, metavar="S",
                    help="served streaming form instead: S voltage streams, seeded uneven "
                         "blocks, Poisson arrivals; prints its own JSON line")
    ap.add_argument("--serve-blocks", type=int, default=12, help="blocks per served stream")
    ap.add_argument("--batched", action="store_true",
                    help="batched form instead: six uneven channel groups with their own "
                         "sub-arrays and DM plans, one CUDA graph per block; prints its own "
                         "JSON line")
    ap.add_argument("--stress", action="store_true",
                    help="stress/recovery sweep of the workload instead: 200 bursts on an "
                         "S/N x width x DM grid over 60 data-seconds; prints its own JSON line")
    ap.add_argument("--autotune", action="store_true",
                    help="with --batched: choose each group's tile shapes by timing first")
    a = ap.parse_args()
    a.warmup = max(3, a.warmup)

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    cfg = workload_config(a.workload)
    cfg.ring_dtype = a.ring

    if a.serve:
        if rank == 0:
            serve_main(a, cfg)
        return
    if a.batched:
        if rank == 0:
            batched_main(a)
        return
    if a.stress:
        if rank == 0:
            stress_main(a)
        return

    if a.impl == "reference":
        if rank != 0:
            return
        threads = os.cpu_count() or 1
        # the reference's own CPU chain (baseline/_ref); the oracle port only
        # where the reference is not installed
        timed = reference_cpu_chain if _ref_import_path() else cpu_baseline
        for _ in range(a.warmup):
            timed(cfg, threads)
        res, walls = [], []
        for _ in range(max(1, a.steps)):
            t0 = time.perf_counter()
            res.append(timed(cfg, threads))
            walls.append(time.perf_counter() - t0)
        v = float(np.median([r["value"] for r in res]))
        cb = dict(res[0])
        cb["value"] = v
        cb["values_per_step"] = [r["value"] for r in res]
        line = {"metric": metric_for(cfg), "value": v, "unit": "data-seconds/s", "n_gpus": a.gpus,
                "steps": a.steps, "warmup": a.warmup,
                "ms_per_step": float(np.mean(walls)) * 1e3,
                "ms_per_step_note": "host wall time of one step, i.e. one bounded sample of the "
                                    "chain; value is that sample's CPU seconds per stage scaled "
                                    "to one data-second of the workload",
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f32" if cb.get("kind") == "reference" else "f64",
                "data": "synthetic", "config": workload_desc(a.workload, cfg), "impl": "reference",
                "cpu_baseline": cb,
                "e2e": {"value": v, "unit": "data-seconds/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return

    import torch
    import torch.distributed as dist
    from dsb200 import synth
    from dsb200.pipeline import SearchPipeline

    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    e, n = synth.t_layout(cfg.nant, seed=11)
    pipe = SearchPipeline(cfg, e, n, device=dev)
    resident_bytes = torch.cuda.memory_allocated(dev)
    pipe.skip_warmup()
    # one device-resident block (19.3 GB, larger than L2) for the timed run
    blocks = [synth.random_block_device(band=cfg.band, nant=cfg.nant, npkt=cfg.npkt_block,
                                        device=dev, seed=1000 * rank)]
    block_bytes = blocks[0].numel()

    def barrier():
        if world > 1:
            dist.barrier()

    def run(k, timing=False):
        pipe.timing = timing
        for i in range(k):
            pipe.process_block(blocks[i % len(blocks)])
        pipe.timing = False

    def check_all(p):
        """The device status word, agreed on by every rank before any raises."""
        code = agreed_status(int(p.status.item()), world, dev)
        if code:
            from dsb200 import _lib
            raise _lib.DsbError(f"pipeline: {_lib.lib().dsb_strerror(code).decode()} "
                                f"(code {code})")

    # warm-up
    run(a.warmup)
    torch.cuda.synchronize()
    pipe.events = {}
    launches0 = pipe.launches
    clocks = Clocks(torch.cuda.current_device())
    barrier()
    torch.cuda.synchronize()
    clocks.start()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record()
    run(a.steps, timing=True)
    ev1.record()
    torch.cuda.synchronize()
    clk = clocks.stop()
    barrier()
    ms = ev0.elapsed_time(ev1)
    # a kernel that flagged an error (capacity, bound, bounded wait) makes the
    # run fail here rather than report a number (on every rank alike)
    check_all(pipe)
    launches = (pipe.launches - launches0) // max(1, a.steps)
    stages = pipe.stage_times_ms()
    ms = max_over_ranks(ms, world, dev)
    ms_step = ms / a.steps
    value = world * cfg.block_seconds * a.steps / (ms / 1e3)

    # e2e: blocks in pinned host memory through the public streaming API
    # (SearchPipeline.process_blocks): every step's H2D copy is inside the
    # timed region, overlapped with the previous block's compute
    e2e = None
    if not a.no_e2e:
        host = torch.empty(blocks[0].shape, dtype=torch.uint8, pin_memory=True)
        host.copy_(blocks[0])
        # the streaming loop keeps two device buffers of its own
        del blocks[:]
        torch.cuda.empty_cache()
        for _ in pipe.process_blocks([host]):
            pass
        torch.cuda.synchronize()
        barrier()
        t0 = time.perf_counter()
        ev0.record()
        for _ in pipe.process_blocks([host] * a.steps):
            pass
        ev1.record()
        torch.cuda.synchronize()
        check_all(pipe)
        ms_e = ev0.elapsed_time(ev1)
        ms_e = max_over_ranks(ms_e, world, dev)
        lat = np.asarray(pipe.block_latency_s) * 1e3
        e2e = {"value": world * cfg.block_seconds * a.steps / (ms_e / 1e3),
               "unit": "data-seconds/s", "h2d_bytes_per_step": int(block_bytes),
               "d2h_bytes_per_step": int(pipe.last_d2h_bytes), "wall_s": time.perf_counter() - t0,
               "block_to_candidate_latency_ms": {"p50": float(np.percentile(lat, 50)),
                                                 "p99": float(np.percentile(lat, 99)),
                                                 "blocks": int(lat.size),
                                                 "block_ms": cfg.block_seconds * 1e3}}
        del host

    # roofline of every kernel (stage), the dominant one as "roofline"
    hbm, bf16, peak_src = load_peaks()
    i8 = measure_int8_peak(dev)
    work = stage_work(pipe)
    traffic = stage_traffic(pipe)
    roofs = {}
    for st, tm in stages.items():
        if st not in work:
            continue
        kind, flops, nbytes = work[st]
        mean_s = tm["mean_ms"] / 1e3
        if kind == "tensor":
            achieved = flops / mean_s / 1e12
            r = {"bound": "tensor", "achieved": achieved, "peak": i8, "unit": "TOP/s",
                 "frac": achieved / i8, "algorithmic_ops_per_launch": flops,
                 "peak_note": "dense int8 (cuBLASLt torch._int_mm 8192^3, best of 10, measured "
                              "in this run)",
                 "raw_input_gbs": nbytes / mean_s / 1e9}
        else:
            achieved = nbytes / mean_s / 1e9
            r = {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                 "frac": achieved / hbm, "algorithmic_bytes_per_launch": nbytes,
                 "peak_note": f"{peak_src} copy bandwidth"}
        r["mean_launch_ms"] = tm["mean_ms"]
        r["traffic"], r["traffic_note"] = traffic.get(st, (None, None))
        roofs[st] = r
    dom = max((k for k in stages if k in roofs), key=lambda k: stages[k]["total_ms"])
    roof = dict(roofs[dom], kernel=dom)

    if rank == 0:
        cb = None
        if not a.no_cpu:
            threads = os.cpu_count() or 1
            cb = (reference_cpu_chain(cfg, threads) if _ref_import_path()
                  else cpu_baseline(cfg, threads=threads))
        line = {"metric": metric_for(cfg), "value": value, "unit": "data-seconds/s", "n_gpus": world,
                "steps": a.steps, "warmup": a.warmup, "ms_per_step": ms_step,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": ("int8 (correlator) / bf16 ring, f32 accumulate" if a.ring == "bf16"
                          else "int8 (correlator) / f32"), "data": "synthetic (seeded 4-bit Gaussian "
                "voltages, sigma 3, T-layout antennas)", "config": workload_desc(a.workload, cfg),
                "clocks": clk, "e2e": e2e, "gpu_launches": launches, "roofline": roof,
                "pipeline_resident_bytes": int(resident_bytes),
                "rooflines_per_kernel": roofs,
                "cpu_baseline": cb,
                "stages_ms_per_step": {k: round(v["total_ms"] / a.steps, 3)
                                       for k, v in stages.items()}}
        print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
