"""Benchmark of the B200 intra encoder: the AVIF encode through mt_encode_rgb8.

Default workload: the 1920x1080 generator image (seed 3: sinusoids, rectangles,
noise sigma 4, the 64-px texture band and the gradient quadrant), 4:2:0,
quality 60 (qindex 70, QM level 6).  One step is one whole encode: colour
conversion and padding, the 8x8 decisions over the dependency wavefront of
the frame (every 8x8 luma block x 13 intra modes x 7 transform types, each
candidate predicted, transformed, quantised with the QM, trellised,
reconstructed, priced by SATD distortion and coefficient rate; chroma UV DC),
coefficient token emission, block syntax, deblocking, the CDEF decision, range
coding with the cdef_idx literals, headers and the AVIF container.  The
decisions are this library's 8x8 rule, not the reference's decode_sb, and the
file is byte for byte the oracle encode's (oracle/oracle_avif.py), which is
checked in every default run.

  value  MPix/s with the RGB already in device memory (mt_encode_rgb8_device),
         the whole call between CUDA events on its stream, L2 flushed before
         each step
  e2e    MPix/s through mt_encode_rgb8 with host RGB (pinned), the copies of the
         call inside the timed region; the bytes both ways are the library's
         count of its own copies

The roofline is the dominant kernel's (encode_blocks_kernel: the persistent
decision kernel): its algorithmic integer/FP32 operations over its device time
against the SMs' issue rate, and the dependency view that bounds it (levels of
the 8x8 dependency graph and the time per level).

The line also carries the earlier kernel-level measurements of the same frame
as secondary entries: ``level8`` (one batched 8x8 RDO level over a
reconstruction snapshot, the oracle's results asserted equal), ``level4`` /
``level16``, ``split16``, ``leaf8`` and ``frame_filters``.

``--impl reference`` times the oracle encode (the CPU restatement of the same
encode; the Rust reference cannot be built here) on all host cores, one whole
encode per step; it never loads the CUDA library.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

W, H, SEED, QUALITY, SUB = 1920, 1080, 3, 60, 2  # the 1080p 4:2:0 quality-60 frame
MODES = list(range(13))
MPIX = W * H / 1e6
METRIC = "MPix/s (AVIF encode, mt_encode_rgb8 1920x1080 4:2:0 quality 60)"
LEVEL_METRIC = "MPix/s (8x8 RDO level, 1080p luma)"
SMS, LANES_PER_SM = 148, 128  # B200: SMs x INT32/FP32 lanes per SM
# DRAM bytes of one level8_kernel launch on this workload, dram__bytes_read.sum
# + dram__bytes_write.sum of the ncu capture in profiles/level8_kernel_1080p_q60.md
NCU_DRAM_BYTES_PER_LAUNCH = 198_752_000 + 1_367_270_000

# Algorithmic integer / FP32 operations of one 8x8 candidate chain, counted on
# the oracle's scalar restatement (oracle/oracle_chain.cpp; one add, sub, mul,
# shift, min, max, compare, select, convert or float op each; a clamp is two):
#   prediction per mode (DC 40, V/H 0, directional 600 with the edge filter,
#   SMOOTH 512, SMOOTH_V/H 256, PAETH 640), residual 64,
#   forward 2-D (dct1d_8 = 62 ops, the Q12 ADST8 = 144 per 1-D pass; IDTX 256),
#   quantisation + f32 targets 11 per coefficient (704), the QM re-rounding 8 per
#   coefficient (512) on the 2-D types, dequantisation 192,
#   inverse 2-D (inv_dct8 = 98, inv_adst8 = 140 per 1-D pass, plus the 256-op
#   intermediate clip and the 128-op final rounding; IDTX 512),
#   SATD bridge 770 (reconstruction difference 256, 8x8 Hadamard 384 + |.| and
#   sum 127, scaling), RD cost 20,
#   and per coefficient up to the end of block 22 (trellis round-down and EOB
#   trim) + 12 (the rate walk's context and token costs).
PRED_OPS = {0: 40, 1: 0, 2: 0, 9: 512, 10: 256, 11: 256, 12: 640}  # directional modes 3..8: 600
FWD_OPS = {0: 256, 1: 992, 4: 2304, 5: 1648, 6: 1648}
INV_OPS = {0: 512, 1: 1952, 4: 2624, 5: 2288, 6: 2288}
QUANT_OPS, QM_OPS, DEQUANT_OPS, RESID_OPS, SATD_OPS, RD_OPS, PER_COEF_OPS = 704, 512, 192, 64, 770, 20, 34


def chain_ops(combos, results, nblocks, qm_on):
    """Algorithmic operations of every candidate of a level (combo-major
    results): the fixed part by (mode, type) plus the per-coefficient part up to
    each candidate's own end of block."""
    fixed = np.array([PRED_OPS.get(int(m), 600) + RESID_OPS + FWD_OPS[int(t)] + QUANT_OPS
                      + (QM_OPS if qm_on and int(t) != 0 else 0) + DEQUANT_OPS + INV_OPS[int(t)] + SATD_OPS + RD_OPS
                      for m, t in zip(combos["mode"], combos["tx_type"])], np.int64)
    eob = results["eob"].astype(np.int64).reshape(len(combos), nblocks)
    coefs = np.where((eob >= 0) & (eob < 64), eob + 1, 0).sum(axis=1)
    return int((fixed * nblocks).sum() + PER_COEF_OPS * coefs.sum())


def config_line():
    """The config object both arms print."""
    return {"workload": "encode_rgb8 1920x1080 4:2:0 quality 60 (qindex 70, QM 6), generator image seed 3: every "
                        "64x64 superblock split to 8x8 blocks, each luma block the lowest RD cost of 13 intra modes x "
                        "7 transform types (91 candidates), chroma UV_DC_PRED + DCT_DCT, deblocking, CDEF decision, "
                        "range coding, AVIF container",
            "decisions": "the library's 8x8 rule (not the reference's decode_sb search)",
            "config": "EncodeConfig defaults (Slow: CDEF on, updating CDFs, sRGB-YCbCr CICP) with quality 60",
            "blocks": (W // 8) * ((H + 7) // 8), "candidates_per_block": 91,
            "l2": "256 MB buffer written before each timed step"}


def level_config(nb, nc):
    """The config of the secondary 8x8-level measurement."""
    return {"workload": "rdo-level-8x8 1920x1080 4:2:0 quality 60 (qindex 70, QM 6), seed 3: every 8x8 luma block "
                        "x 13 intra modes x 5 transform types (IDTX, DCT_DCT, ADST_ADST, ADST_DCT, DCT_ADST)",
            "cdfs": "default decision snapshot Cdfs::new(qctx 2)", "lambdas": "shipped Slow laws at qindex 70 4:2:0",
            "candidates": nb * nc, "blocks": nb, "combos": nc, "l2": "inputs re-read after an L2 flush per step"}


def encode_rgb():
    from maroontree_b200 import synth

    return synth.generate_rgb(W, H, SEED, sigma=4.0, variant="1080p")


def oracle_encode(rgb, threads):
    """The oracle encode of the frame on `threads` host cores: (bytes, seconds)."""
    from oracle import oracle_avif as oa

    t0 = time.perf_counter()
    avif = oa.encode_rgb8(rgb, QUALITY, 0, threads=threads)
    return avif, time.perf_counter() - t0


# Algorithmic operations of one block's decision (the roofline's work unit),
# from the per-stage table above with every coefficient up to the end of block
# counted (an upper bound of the per-coefficient part): the 13 predictions, and
# per (mode, type) the rest of the chain (V_DCT / H_DCT counted as DCT_DCT, an
# upper bound: one 1-D pass each); chroma adds two DC_PRED + DCT_DCT chains (8x8
# in 4:4:4; in 4:2:0 a 4x4 chain, counted as a quarter of the 8x8 one).
def block_ops(sub):
    per_type = (0, 1, 1, 1, 4, 5, 6)  # IDTX, DCT_DCT, V_DCT, H_DCT, ADST_ADST, ADST_DCT, DCT_ADST
    chain = sum(RESID_OPS + FWD_OPS[t] + QUANT_OPS + (QM_OPS if t != 0 else 0) + DEQUANT_OPS + INV_OPS[t] + SATD_OPS
                + RD_OPS + 64 * PER_COEF_OPS for t in per_type)
    luma = len(MODES) * chain + sum(PRED_OPS.get(m, 600) for m in MODES)
    chroma = PRED_OPS[0] + RESID_OPS + FWD_OPS[1] + QUANT_OPS + QM_OPS + DEQUANT_OPS + INV_OPS[1] + SATD_OPS + RD_OPS + \
        64 * PER_COEF_OPS
    return luma + (2 * chroma if sub == 0 else chroma // 2)


def make_workload():
    """The workload of the secondary kernel-level measurements: the frame's
    luma, a seeded reconstruction snapshot (source plus +-3 coding error), the
    8x8 level's blocks and (mode, type) combos, and the frame laws' quantiser,
    QM row, lambdas and default CDF slice from the library's C ABI."""
    import maroontree_b200 as mt
    from maroontree_b200 import abi, synth

    qidx = mt.quality_to_q(QUALITY)
    qm_level = mt.qm_levels(qidx, SUB)[0]
    q = mt.quant_new(qidx, 8, qm_level)
    qm = mt.qm_row(qm_level, 0, 8)
    lam = mt.rd_lambdas(qidx, q.dc_q, SUB)
    cdfs = mt.coef_cdfs_default(mt.qcat(qidx), 8, 8, 0)
    rgb = synth.generate_rgb(W, H, SEED, sigma=4.0, variant="1080p")
    src = synth.rgb_to_luma(rgb)
    rec = synth.synthetic_recon(src, SEED + 1000)
    blocks = synth.level_blocks(W, H, seed=SEED)
    combos = synth.level_combos(MODES, abi.TX_2D_SCAN_TYPES)
    cands = synth.candidates_of_level(blocks, combos)
    prm = mt.chain_params(W, H, trellis_lambda0=lam.trellis_lambda0, mode_lambda=lam.mode_lambda,
                          satd_scale=lam.satd_scale, satd_bridge=lam.satd_bridge)
    return dict(src=src, rec=rec, blocks=blocks, combos=combos, cands=cands, cdfs=cdfs, q=q, qm=qm, prm=prm, rgb=rgb,
                qidx=qidx, qm_level=qm_level, lam=lam)


class ClockSampler:
    """Samples nvidia-smi clocks and throttle reasons while the timed region runs."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index=0):
        self.index = index
        self.samples = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.FIELDS,
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=5)
                if out.returncode == 0 and out.stdout.strip():
                    self.samples.append([v.strip() for v in out.stdout.strip().split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if len(s) > 4 + i and s[4 + i] == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


class Replicas:
    """One process per GPU, each encoding its own frame (replicas: the path has
    no exchange step, so nothing crosses ranks on the data path).  The process
    group carries only the barriers around the timed region and the max-over-
    ranks reduction of the step time; only rank 0 prints the JSON line."""

    def __init__(self, backend="nccl", timeout_s=120):
        self.world, self.rank, self.local = dist_env()
        self.dist = None
        if self.world > 1:
            import datetime

            import torch.distributed as dist

            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
            self.dist = dist

    def barrier(self):
        if self.dist is not None:
            self.dist.barrier()

    def max(self, value, device="cpu"):
        """The maximum of a per-rank float over all ranks."""
        if self.dist is None:
            return float(value)
        import torch

        t = torch.tensor([float(value)], dtype=torch.float64, device=device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def job_value(self, step_ms, units_per_rank=MPIX):
        """Whole-job throughput: the units every rank processed over the slowest rank's step."""
        return self.world * units_per_rank / (step_ms / 1e3)

    def emit(self, line):
        if self.rank == 0:
            print(json.dumps(line), flush=True)

    def close(self):
        if self.dist is not None:
            self.dist.barrier()
            self.dist.destroy_process_group()
            self.dist = None


def cpu_level(wl, threads):
    """The oracle over every candidate of the level on `threads` host cores:
    (results, seconds)."""
    from oracle import pyoracle as po

    t0 = time.perf_counter()
    res, _, _ = po.candidate_chain(wl["src"], wl["rec"], wl["prm"], wl["q"], wl["qm"], wl["cdfs"], wl["cands"],
                                   threads=threads)
    return res, time.perf_counter() - t0


def run_reference(args):
    """The reference arm: the oracle encode (the CPU restatement of the same
    encode; the Rust reference cannot be built here), one whole encode per
    step on all host cores.  Its inputs come from the oracle and the shared
    image generator alone; the CUDA library is never loaded."""
    world, rank, _ = dist_env()
    if rank != 0:
        return 0
    from oracle import build as obuild

    obuild.build()
    rgb = encode_rgb()
    threads = os.cpu_count() or 1
    for _ in range(args.warmup):
        oracle_encode(rgb, threads)
    times = [oracle_encode(rgb, threads)[1] for _ in range(args.steps)]
    step_s = float(np.mean(times))
    value = MPIX / step_s
    line = {
        "impl": "reference", "metric": METRIC, "value": round(value, 4),
        "unit": "MPix/s", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(step_s * 1e3, 3), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "int32+f32", "data": "synthetic", "config": config_line(),
        "cpu_baseline": {"value": round(value, 4), "unit": "MPix/s", "cores": threads, "kind": "port",
                         "sample": "one whole 1920x1080 encode per step (the oracle's restatement, all host cores)"},
        "e2e": {"value": round(value, 4), "unit": "MPix/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def measure_small_level(dev, wl, n, reps=5, cpu=True):
    """The batched 4x4 or 16x16 level over the same 1080p luma: 4x4 -- 129,600
    blocks x 13 modes x the SPLIT4 trial types DCT, ADST, IDTX-without-trellis,
    ADST_DCT, DCT_ADST; 16x16 -- 8,040 blocks x 13 modes x the 16x16 proxy's
    types DCT, ADST, IDTX.  Device time with CUDA events after an L2 flush, and
    the oracle on all host cores over the same candidates."""
    import ctypes as C

    import torch
    import maroontree_b200 as mt
    from maroontree_b200 import abi, synth

    q = wl["q"]
    qm = mt.qm_row(wl["qm_level"], 0, n)
    blocks = synth.level_blocks(W, H, n=n, seed=SEED)
    if n == 4:
        combos = synth.level_combos(MODES, (abi.TX_DCT_DCT, abi.TX_ADST_ADST, abi.TX_IDTX, abi.TX_ADST_DCT,
                                            abi.TX_DCT_ADST), no_trellis_types=(abi.TX_IDTX,))
        cdfs = mt.coef_cdfs_default(mt.qcat(wl["qidx"]), 4, 4, 0)
        entry, scratch_fn = "mt_rdo_level4_device", "mt_rdo_level4_scratch_bytes"
        what = "rdo-level-4x4 1920x1080 luma, qindex 70, QM 6, 13 modes x 5 types (IDTX without trellis)"
    else:
        combos = synth.level_combos(MODES, (abi.TX_DCT_DCT, abi.TX_ADST_ADST, abi.TX_IDTX))
        cdfs = mt.coef_cdfs_default(mt.qcat(wl["qidx"]), 16, 16, 0)
        entry, scratch_fn = "mt_rdo_level16_device", "mt_rdo_level16_scratch_bytes"
        what = "rdo-level-16x16 1920x1080 luma, qindex 70, QM 6, 13 modes x 3 types (DCT, ADST, IDTX)"
    costs = mt.coef_costs(cdfs)
    prm = mt.chain_params(W, H, tx_size=n, trellis_lambda0=wl["lam"].trellis_lambda0, mode_lambda=wl["prm"].mode_lambda,
                          satd_scale=wl["prm"].satd_scale, satd_bridge=wl["prm"].satd_bridge)
    nb, nc = len(blocks), len(combos)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a).view(np.uint8).copy()).to(dev)
    d = [t(wl["src"]), t(wl["rec"]), t(qm), t(np.frombuffer(bytes(costs), np.uint8)), t(blocks), t(combos)]
    d_best = torch.empty(nb * abi.BEST_DTYPE.itemsize, dtype=torch.uint8, device=dev)
    d_res = torch.empty(nb * nc * abi.RESULT_DTYPE.itemsize, dtype=torch.uint8, device=dev)
    d_keys = torch.empty(getattr(mt.load(), scratch_fn)(nb, nc), dtype=torch.uint8, device=dev)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=dev)
    fn = getattr(mt.load(), entry)

    def launch():
        rc = fn(d[0].data_ptr(), d[1].data_ptr(), C.byref(prm), C.byref(q), d[2].data_ptr(), d[3].data_ptr(),
                d[4].data_ptr(), nb, d[5].data_ptr(), nc, d_best.data_ptr(), d_res.data_ptr(), d_keys.data_ptr(), None)
        assert rc == 0, rc

    for _ in range(3):
        launch()
    ms = []
    for _ in range(reps):
        flush.zero_()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        a.record()
        launch()
        b.record()
        torch.cuda.synchronize()
        ms.append(a.elapsed_time(b))
    step = float(np.median(ms))
    out = {"ms": round(step, 4), "mpix_s": round(MPIX / (step / 1e3), 2), "candidates": nb * nc, "workload": what}
    if cpu:
        from oracle import pyoracle as po

        cands = synth.candidates_of_level(blocks, combos)
        threads = os.cpu_count() or 1
        t0 = time.perf_counter()
        po.candidate_chain(wl["src"], wl["rec"], prm, q, qm, cdfs, cands, threads=threads)
        dt = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": round(MPIX / dt, 4), "unit": "MPix/s", "cores": threads, "kind": "port",
                               "sample": f"the whole level, {len(cands)} candidates ({dt:.2f} s)"}
    return out


def measure_split16(dev, wl, search, reps=5, cpu=True, depth2=False):
    """The 16x16 leaf's TX_8X8 split trial over the same 1080p luma: 8,040
    blocks x 13 modes = 104,520 jobs of four quadrants each (DCT_DCT with
    trellis_optimize_ctx, and with `search` the 4:4:4 type trials).  Device time
    with CUDA events after an L2 flush; the oracle on all host cores over the
    same jobs.  depth2: the depth-2 trial instead (sixteen TX_4X4 per job, five
    types each)."""
    import ctypes as C

    import torch
    import maroontree_b200 as mt
    from maroontree_b200 import abi, synth

    q = wl["q"]
    qm = mt.qm_row(wl["qm_level"], 0, 4 if depth2 else 8)
    cdfs = mt.coef_cdfs_default(mt.qcat(wl["qidx"]), 4 if depth2 else 8, 4 if depth2 else 8, 0)
    costs = mt.coef_costs(cdfs)
    jobs = synth.split16_jobs(W, H, MODES, seed=SEED)
    n = len(jobs)
    prm = mt.split16_params(W, H, trellis_lambda0=wl["lam"].trellis_lambda0, rd_lambda=wl["lam"].lambda_d, band_tilt=1.9,
                            tx_search=search, tx_guard_shift=5 if search else 4)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a).view(np.uint8).copy()).to(dev)
    d_src, d_rec, d_qm, d_costs, d_jobs = (t(wl["src"]), t(wl["rec"]), t(qm), t(np.frombuffer(bytes(costs), np.uint8)),
                                           t(jobs))
    rdt = abi.SPLIT16_D2_RESULT_DTYPE if depth2 else abi.SPLIT16_RESULT_DTYPE
    d_res = torch.empty(n * rdt.itemsize, dtype=torch.uint8, device=dev)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=dev)
    lib = mt.load()
    entry = lib.mt_split16_depth2_device if depth2 else lib.mt_split16_luma_device

    def launch():
        rc = entry(d_src.data_ptr(), d_rec.data_ptr(), C.byref(prm), C.byref(q),
                                        d_qm.data_ptr(), d_costs.data_ptr(), d_jobs.data_ptr(), n,
                                        d_res.data_ptr(), None, None, None)
        assert rc == 0, rc

    for _ in range(3):
        launch()
    ms = []
    for _ in range(reps):
        flush.zero_()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        torch.cuda._sleep(200_000)
        a.record()
        launch()
        b.record()
        torch.cuda.synchronize()
        ms.append(a.elapsed_time(b))
    step = float(np.median(ms))
    what = (f"split16 leaf trial 1920x1080 luma, qindex 70, QM 6, 8,040 blocks x 13 modes, "
            f"{'4:4:4 type search (7 types per quadrant)' if search else '4:2:0 (DCT_DCT per quadrant)'}")
    if depth2:
        what = ("split16 depth-2 trial 1920x1080 luma, qindex 70, QM 6, 8,040 blocks x 13 modes, sixteen TX_4X4 "
                "per job, 5 types each")
    out = {"ms": round(step, 4), "mpix_s": round(MPIX / (step / 1e3), 2), "jobs": n,
           "jobs_per_s": round(n / (step / 1e3)), "workload": what}
    if cpu:
        from oracle import pyoracle as po

        threads = os.cpu_count() or 1
        t0 = time.perf_counter()
        (po.split16_depth2 if depth2 else po.split16_luma)(wl["src"], wl["rec"], prm, q, qm, cdfs, jobs,
                                                           threads=threads)
        dt = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": round(MPIX / dt, 4), "unit": "MPix/s", "cores": threads, "kind": "port",
                               "sample": f"all {n} jobs ({dt:.2f} s)"}
    return out


def measure_leaf8(dev, wl, refine, reps=5, cpu=True, n16=False, n32=False):
    """The 8x8 leaf's luma search over the same 1080p luma: the mode loop's
    candidates (32,400 blocks x 13 modes, DCT_DCT with trellis_optimize_ctx and
    sse_recon) or the winners' transform-type refinement (32,400 blocks, seven
    types, 4:4:4 form).  Device time with CUDA events after an L2 flush; the
    oracle on all host cores over the same jobs.  n16: the 16x16 leaf's
    mode-loop candidates (8,040 blocks x 13 modes, trellis_optimize_ctx at
    TX_16X16) or its winners' refinement (8,040 blocks, five types).  n32: the
    32x32 leaf's mode-loop candidates (1,980 blocks x 13 modes, TX_32X32
    DCT_DCT with trellis_optimize_ctx)."""
    import ctypes as C

    import torch
    import maroontree_b200 as mt
    from maroontree_b200 import abi, synth

    q = wl["q"]
    size = 32 if n32 else (16 if n16 else 8)
    qm = mt.qm_row(wl["qm_level"], 0, size)
    cdfs = mt.coef_cdfs_default(mt.qcat(wl["qidx"]), size, size, 0)
    costs = mt.coef_costs(cdfs)
    jobs = synth.leaf8_jobs(W, H, [abi.PAETH_PRED] if refine else MODES, seed=SEED, n=size)
    n = len(jobs)
    prm = mt.split16_params(W, H, trellis_lambda0=wl["lam"].trellis_lambda0, rd_lambda=wl["lam"].lambda_d, band_tilt=1.9,
                            tx_search=refine, tx_guard_shift=5)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a).view(np.uint8).copy()).to(dev)
    d_src, d_rec, d_qm, d_costs, d_jobs = (t(wl["src"]), t(wl["rec"]), t(qm), t(np.frombuffer(bytes(costs), np.uint8)),
                                           t(jobs))
    d_res = torch.empty(n * abi.LEAF8_RESULT_DTYPE.itemsize, dtype=torch.uint8, device=dev)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=dev)
    lib = mt.load()
    if n32:
        entry = lib.mt_leaf32_luma_device
    elif n16:
        entry = lib.mt_leaf16_tx_refine_device if refine else lib.mt_leaf16_luma_device
    else:
        entry = lib.mt_leaf8_tx_refine_device if refine else lib.mt_leaf8_luma_device

    def launch():
        rc = entry(d_src.data_ptr(), d_rec.data_ptr(), C.byref(prm), C.byref(q), d_qm.data_ptr(), d_costs.data_ptr(),
                   d_jobs.data_ptr(), n, d_res.data_ptr(), None, None, None)
        assert rc == 0, rc

    for _ in range(3):
        launch()
    ms = []
    for _ in range(reps):
        flush.zero_()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        torch.cuda._sleep(200_000)
        a.record()
        launch()
        b.record()
        torch.cuda.synchronize()
        ms.append(a.elapsed_time(b))
    step = float(np.median(ms))
    what = ("leaf8 winners' transform-type refinement 1920x1080 luma, 32,400 blocks, 7 types" if refine else
            "leaf8 mode-loop candidates 1920x1080 luma, 32,400 blocks x 13 modes (DCT_DCT + trellis_optimize_ctx)")
    if n16:
        what = ("leaf16 winners' transform-type refinement 1920x1080 luma, 8,040 blocks, 5 types" if refine else
                "leaf16 mode-loop candidates 1920x1080 luma, 8,040 blocks x 13 modes (DCT_DCT + trellis_optimize_ctx)")
    if n32:
        what = "leaf32 mode-loop candidates 1920x1080 luma, 1,980 blocks x 13 modes (TX_32X32 DCT_DCT + " \
               "trellis_optimize_ctx)"
    out = {"ms": round(step, 4), "mpix_s": round(MPIX / (step / 1e3), 2), "jobs": n, "workload": what}
    if cpu:
        from oracle import pyoracle as po

        threads = os.cpu_count() or 1
        t0 = time.perf_counter()
        if n32:
            po.leaf32(wl["src"], wl["rec"], prm, q, qm, cdfs, jobs, threads=threads)
        elif n16:
            po.leaf16(wl["src"], wl["rec"], prm, q, qm, cdfs, jobs, refine=refine, threads=threads)
        else:
            po.leaf8(wl["src"], wl["rec"], prm, q, qm, cdfs, jobs, refine=refine, threads=threads)
        dt = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": round(MPIX / dt, 4), "unit": "MPix/s", "cores": threads, "kind": "port",
                               "sample": f"all {n} jobs ({dt:.2f} s)"}
    return out


def measure_leaf64(dev, wl, grid, reps=5, cpu=True):
    """The 64x64 leaf's luma legs over the same 1080p luma: the four-TX_32X32
    candidate leg (480 blocks x 13 modes, four TX_32X32 with
    trellis_optimize_ctx each) or the sixteen-TX_16X16 tx_depth-2 leg on one
    mode per block (480 blocks, sixteen TX_16X16 each, the modes spread over
    the blocks).  Device time with CUDA events after an L2 flush; the oracle on
    all host cores over the same jobs."""
    import ctypes as C

    import torch
    import maroontree_b200 as mt
    from maroontree_b200 import abi, synth

    q = wl["q"]
    size = 16 if grid else 32
    qm = mt.qm_row(wl["qm_level"], 0, size)
    cdfs = mt.coef_cdfs_default(mt.qcat(wl["qidx"]), size, size, 0)
    costs = mt.coef_costs(cdfs)
    jobs = synth.leaf64_jobs(W, H, MODES, seed=SEED, grid=grid)
    if grid:  # one (winning) mode per block
        nb = len(jobs) // len(MODES)
        jobs = jobs[np.arange(nb) + nb * (np.arange(nb) % len(MODES))]
    n = len(jobs)
    prm = mt.split16_params(W, H, trellis_lambda0=wl["lam"].trellis_lambda0, rd_lambda=wl["lam"].lambda_d,
                            band_tilt=1.9, wsse_scale=1.0)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a).view(np.uint8).copy()).to(dev)
    d_src, d_rec, d_qm, d_costs, d_jobs = (t(wl["src"]), t(wl["rec"]), t(qm), t(np.frombuffer(bytes(costs), np.uint8)),
                                           t(jobs))
    rdt = abi.GRID16_RESULT_DTYPE if grid else abi.QUAD32_RESULT_DTYPE
    d_res = torch.empty(n * rdt.itemsize, dtype=torch.uint8, device=dev)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=dev)
    lib = mt.load()

    def launch():
        args = [d_src.data_ptr(), d_rec.data_ptr(), C.byref(prm), C.byref(q), d_qm.data_ptr(), d_costs.data_ptr(),
                d_jobs.data_ptr(), n, d_res.data_ptr()]
        rc = lib.mt_grid16_luma_device(*args, None, None) if grid else lib.mt_quad32_luma_device(*args, None)
        assert rc == 0, rc

    for _ in range(3):
        launch()
    ms = []
    for _ in range(reps):
        flush.zero_()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        torch.cuda._sleep(200_000)
        a.record()
        launch()
        b.record()
        torch.cuda.synchronize()
        ms.append(a.elapsed_time(b))
    step = float(np.median(ms))
    what = ("leaf64 tx_depth-2 leg 1920x1080 luma, 480 blocks x 1 mode (sixteen TX_16X16)" if grid else
            "leaf64 four-TX_32X32 leg 1920x1080 luma, 480 blocks x 13 modes")
    out = {"ms": round(step, 4), "mpix_s": round(MPIX / (step / 1e3), 2), "jobs": n, "workload": what}
    if cpu:
        from oracle import pyoracle as po

        threads = os.cpu_count() or 1
        t0 = time.perf_counter()
        if grid:
            po.grid16_luma(wl["src"], wl["rec"], prm, q, qm, cdfs, jobs, threads=threads)
        else:
            po.quad32_luma(wl["src"], wl["rec"], prm, q, qm, cdfs, jobs, threads=threads)
        dt = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": round(MPIX / dt, 4), "unit": "MPix/s", "cores": threads, "kind": "port",
                               "sample": f"all {n} jobs ({dt:.2f} s)"}
    return out


def measure_uv16(dev, wl, reps=5, cpu=True, form="420"):
    """The 16x16 leaf's 4:2:0 chroma search (pick_uv16_420) over every 16x16
    leaf of the 1080p frame (8,040 leaves: DC, CfL, 60 shortlist predictions
    per plane, the 4 best priced in full) with the frame's chroma quantiser
    and QM, the default chroma TX_8X8 and mode CDFs.  Device time with CUDA
    events after an L2 flush; the oracle on all host cores over the same
    leaves."""
    import ctypes as C

    import torch
    import maroontree_b200 as mt
    from maroontree_b200 import abi, synth

    # form: "420" pick_uv16_420, "444" pick_uv16_444, "420_32" pick_uv32_420, "444_32" pick_uv32_444
    qidx = wl["qidx"]
    sub = 0 if form.startswith("444") else SUB
    tx = 32 if form.endswith("_32") else (16 if form == "444" else 8)
    qm_uv = mt.qm_levels(qidx, sub)[1]
    q = mt.quant_new_chroma(qidx, 0, 0, 8, qm_uv)
    qm = mt.qm_row(qm_uv, 1, tx) if qm_uv < 15 else None
    cdfs = mt.coef_cdfs_default(mt.qcat(qidx), tx, tx, 1)
    costs = mt.coef_costs(cdfs)
    mcdfs = mt.uv_mode_cdfs_default()
    mcost = mt.uv_mode_costs(mcdfs)
    if sub:
        src, rec = synth.planes420(wl["rgb"], SEED)
    else:
        src, rec = synth.planes444(wl["rgb"], SEED)
    cw, ch = src[1].shape[1], src[1].shape[0]
    prm = mt.split16_params(cw, ch, trellis_lambda0=wl["lam"].trellis_lambda0, rd_lambda=wl["lam"].mode_lambda,
                            wsse_scale=1.0, vis=(W >> (1 if sub else 0), H >> (1 if sub else 0)))
    uvp = mt.uv16_params(src[0].shape[1], joint_k=4, angle_deltas=True, dir_lambda=wl["lam"].lambda_d)
    entry, po_entry, jobs, what = {
        "420": ("mt_pick_uv16_420_device", "pick_uv16_420", synth.uv16_jobs(W, H, SEED),
                "pick_uv16_420 1920x1080 4:2:0, 8,040 16x16 leaves (DC, CfL, 60-entry SATD shortlist, 4 priced)"),
        "444": ("mt_pick_uv16_444_device", "pick_uv16_444", synth.uv16_444_jobs(W, H, SEED),
                "pick_uv16_444 1920x1080 4:4:4, 8,040 16x16 leaves (DC, CfL, SATD top-3, zone-2 deltas)"),
        "420_32": ("mt_pick_uv32_420_device", "pick_uv32_420", synth.uv16_444_jobs(W, H, SEED, leaf=32),
                   "pick_uv32_420 1920x1080 4:2:0, 1,980 32x32 leaves (16x16 chroma: DC, CfL, SATD top-3, deltas)"),
        "444_32": ("mt_pick_uv32_444_device", "pick_uv32_444", synth.uv32_444_jobs(W, H, SEED),
                   "pick_uv32_444 1920x1080 4:4:4, 1,980 32x32 leaves (32x32 chroma: DC, CfL, SATD top-3, deltas)"),
    }[form]
    n = len(jobs)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a).view(np.uint8).copy()).to(dev)
    d_p = [t(a) for a in (src[1], src[2], rec[1], rec[2], rec[0])]
    d_qm = t(qm) if qm is not None else None
    d_costs, d_mc, d_jobs = t(np.frombuffer(bytes(costs), np.uint8)), t(np.frombuffer(bytes(mcost), np.uint8)), t(jobs)
    d_res = torch.empty(n * abi.UV16_RESULT_DTYPE.itemsize, dtype=torch.uint8, device=dev)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=dev)
    lib = mt.load()

    def launch():
        rc = getattr(lib, entry)(*[a.data_ptr() for a in d_p], C.byref(prm), C.byref(uvp), C.byref(q),
                                         None if d_qm is None else d_qm.data_ptr(), d_costs.data_ptr(),
                                         d_mc.data_ptr(), d_jobs.data_ptr(), n, d_res.data_ptr(), None, None, None)
        assert rc == 0, rc

    for _ in range(3):
        launch()
    ms = []
    for _ in range(reps):
        flush.zero_()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        torch.cuda._sleep(200_000)
        a.record()
        launch()
        b.record()
        torch.cuda.synchronize()
        ms.append(a.elapsed_time(b))
    step = float(np.median(ms))
    out = {"ms": round(step, 4), "mpix_s": round(MPIX / (step / 1e3), 2), "jobs": n,
           "workload": what + ", frame chroma quantiser and QM"}
    if cpu:
        from oracle import pyoracle as po

        threads = os.cpu_count() or 1
        t0 = time.perf_counter()
        getattr(po, po_entry)(src[1], src[2], rec[1], rec[2], rec[0], prm, uvp, q, qm,
                              po.default_cdfs(mt.qcat(qidx), tx, plane=1), po.uv_mode_cdfs(), jobs, threads=threads)
        dt = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": round(MPIX / dt, 4), "unit": "MPix/s", "cores": threads, "kind": "port",
                               "sample": f"all {n} leaves ({dt:.2f} s)"}
    return out


def measure_filters(dev, wl, hbm_peak, reps=5):
    """Device time of the frame-wide kernels on the 1080p 4:2:0 frame."""
    import ctypes as C

    import torch
    import maroontree_b200 as mt
    from maroontree_b200 import abi, synth

    lib = mt.load()
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=dev)
    t16 = lambda a: torch.from_numpy(np.ascontiguousarray(a).astype(np.int16)).to(dev)
    t8 = lambda a: torch.from_numpy(np.ascontiguousarray(a, np.uint8)).to(dev)

    def timed(fn, reset=None):
        # The GPU is kept busy (L2 flush, then a ~100 us spin) while the host
        # enqueues the start event, the call's launches and the end event, so
        # the events bracket device time, not the host's launch latency.
        ms = []
        for i in range(reps + 2):
            if reset:
                reset()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            flush.zero_()
            torch.cuda._sleep(200_000)
            a.record()
            rc = fn()
            b.record()
            torch.cuda.synchronize()
            assert rc == 0, rc
            if i >= 2:
                ms.append(a.elapsed_time(b))
        return float(np.median(ms))

    def entry(ms, nbytes, what):
        gbs = nbytes / (ms / 1e3) / 1e9
        return {"ms": round(ms, 4), "alg_bytes": int(nbytes), "achieved_gbs": round(gbs, 1),
                "frac_hbm": round(gbs / hbm_peak, 4), "bytes": what}

    out = {}
    # colour conversion + padding (RGB -> padded Y / Cb / Cr)
    pw, ph, pcw, pch = mt.padded_plane_dims(W, H, 2)
    d_rgb = t8(wl["rgb"])
    y = torch.empty((ph, pw), dtype=torch.int16, device=dev)
    cb = torch.empty((pch, pcw), dtype=torch.int16, device=dev)
    cr = torch.empty_like(cb)
    ms = timed(lambda: lib.mt_csc_rgb8_device(d_rgb.data_ptr(), W, H, 2, y.data_ptr(), cb.data_ptr(), cr.data_ptr(),
                                              None))
    out["csc"] = entry(ms, W * H * 3 + (pw * ph + 2 * pcw * pch) * 2, "3 B/px in + 2 B per output sample")
    # adaptive-quantisation grid over the padded luma the conversion produced
    nsb = ((pw + 63) // 64) * ((ph + 63) // 64)
    cells = torch.empty(nsb * 4, dtype=torch.uint8, device=dev)
    refs = torch.empty(2 * 64, dtype=torch.float32, device=dev)
    for tag, q in (("aq_grid", wl["qidx"]), ("aq_grid_q116", 116)):
        ap = mt.aq_params(pw, ph, q)
        ascr = torch.empty(lib.mt_aq_grid_scratch_bytes(C.byref(ap)), dtype=torch.uint8, device=dev)
        ms = timed(lambda: lib.mt_aq_grid_device(y.data_ptr(), C.byref(ap), cells.data_ptr(), refs.data_ptr(),
                                                 ascr.data_ptr(), None))
        out[tag] = entry(ms, pw * ph * 2, "2 B luma read per sample")
        out[tag]["bound"] = "launch / per-tile serial means (two kernels; dark protection from qindex 90)"
    # screen-content gate: the photo frame stops at the block pass; a mixed
    # text / UI / photo frame of the same size runs the copy stage too
    for tag, lum in (("screen_gate_photo", y), ("screen_gate_mixed",
                     torch.from_numpy(synth.screen_luma(pw, ph, 5, photo_frac=0.3).view(np.int16)).to(dev))):
        sp = mt.screen_gate_params(pw, ph, 1, 1, wl["qidx"])
        sscr = torch.empty(lib.mt_screen_gate_scratch_bytes(C.byref(sp)), dtype=torch.uint8, device=dev)
        sres = abi.ScreenGateResult()
        ms = timed(lambda: lib.mt_screen_gate_device(lum.data_ptr(), C.byref(sp), sscr.data_ptr(), C.byref(sres),
                                                     None))
        out[tag] = entry(ms, pw * ph * 2, "2 B luma read per sample (block pass; the copy stage re-reads windows)")
        out[tag]["verdict"] = {"copy_stage": sres.copy_stage, "ibc_pays": sres.ibc_pays,
                               "few_colour": sres.few_colour}
        out[tag]["bound"] = "host synchronisation after the block pass (and after the copy stage)"
    # chroma-from-luma alpha of every 8x8 chroma block (4:2:0), from the
    # converted luma and chroma planes
    cfl = np.zeros((pch // 8) * (pcw // 8), abi.CFL_BLOCK_DTYPE)
    cys, cxs = np.meshgrid(np.arange(0, pch - 7, 8), np.arange(0, pcw - 7, 8), indexing="ij")
    cfl["cx"], cfl["cy"], cfl["dc"] = cxs.ravel(), cys.ravel(), 128
    d_cfl = torch.from_numpy(cfl.view(np.uint8).copy()).to(dev)
    d_alpha = torch.empty(2 * len(cfl), dtype=torch.int8, device=dev)
    ms = timed(lambda: lib.mt_cfl_alpha_device(y.data_ptr(), pw, cb.data_ptr(), cr.data_ptr(), pcw, 1, 1, 8, 8, 0, 0, 8,
                                               d_cfl.data_ptr(), len(cfl), d_alpha.data_ptr(), None, None))
    out["cfl_alpha"] = entry(ms, len(cfl) * 64 * (4 * 2 + 2 * 2), "4 luma + 2 chroma samples (2 B) per chroma sample")
    out["cfl_alpha"]["blocks"] = len(cfl)
    # the filter-intra shortlist of every 16x16 luma block (five modes each)
    fys, fxs = np.meshgrid(np.arange(0, H - 15, 16), np.arange(0, W - 15, 16), indexing="ij")
    fpos = np.stack([fxs.ravel(), fys.ravel()], axis=1).astype(np.uint16)
    d_fpos = torch.from_numpy(fpos.view(np.uint8).copy()).to(dev)
    d_fsrc, d_frec = t16(wl["src"]), t16(wl["rec"])
    d_fsc = torch.empty(len(fpos) * 5 * 8, dtype=torch.uint8, device=dev)
    d_fmd = torch.empty(len(fpos) * 5, dtype=torch.uint8, device=dev)
    ms = timed(lambda: lib.mt_filter_intra_beam_device(d_fsrc.data_ptr(), d_frec.data_ptr(), W, W, H, 0, 0, 8, 16, 16,
                                                       d_fpos.data_ptr(), len(fpos), d_fsc.data_ptr(),
                                                       d_fmd.data_ptr(), None, None))
    out["filter_intra_beam16"] = entry(ms, len(fpos) * 5 * (256 * 2 + 33 * 2),
                                       "per (block, mode): the 16x16 source (2 B / sample) and the 33 edge samples")
    out["filter_intra_beam16"]["blocks"] = len(fpos)
    # the lossy luma palette candidates of every 16x16 block of a 1080p
    # screen-content luma plane: histogram gate, 14 centre sets, Viterbi maps
    # (the shipped screen-frame map, lambda = 0.35 x the mode lambda), index bits
    scr = synth.screen_luma(W, H, 7)
    d_scr = t16(scr)
    popts = mt.palette_opts(viterbi_lambda=0.35 * wl["prm"].mode_lambda,
                            color_costs=np.random.default_rng(5).uniform(0.15, 7.0, (7, 5, 8)))
    d_pc = torch.empty(len(fpos) * abi.PALETTE_SLOTS * abi.PALETTE_CAND_DTYPE.itemsize, dtype=torch.uint8, device=dev)
    d_pm = torch.empty(len(fpos) * abi.PALETTE_SLOTS * 256, dtype=torch.uint8, device=dev)
    ms = timed(lambda: lib.mt_luma_palette_device(d_scr.data_ptr(), W, W, H, 8, 16, 16, d_fpos.data_ptr(), len(fpos),
                                                  C.byref(popts), d_pc.data_ptr(), d_pm.data_ptr(), None))
    out["luma_palette16"] = entry(ms, len(fpos) * (256 * 2 + abi.PALETTE_SLOTS * (256 + 24)),
                                  "per block: the 16x16 source (2 B / sample), 14 maps (1 B / sample) and candidates")
    out["luma_palette16"]["blocks"] = len(fpos)
    out["luma_palette16"]["palette_blocks"] = None  # filled below from the candidates
    pc = np.frombuffer(d_pc.cpu().numpy().tobytes(), abi.PALETTE_CAND_DTYPE).reshape(len(fpos), abi.PALETTE_SLOTS)
    out["luma_palette16"]["palette_blocks"] = int((pc["hist_len"][:, 0] > 0).sum())
    # the UV palette candidates of every 16x16 block of 1080p 4:4:4
    # screen-content chroma planes: exact palette or the four lossy candidates,
    # Viterbi UV maps at the same lambda
    d_su, d_sv = t16(synth.screen_luma(W, H, 11)), t16(synth.screen_luma(W, H, 12))
    d_uc = torch.empty(len(fpos) * abi.UV_PALETTE_SLOTS * abi.UV_PALETTE_CAND_DTYPE.itemsize, dtype=torch.uint8,
                       device=dev)
    d_um = torch.empty(len(fpos) * abi.UV_PALETTE_SLOTS * 256, dtype=torch.uint8, device=dev)
    ms = timed(lambda: lib.mt_uv_palette_device(d_su.data_ptr(), d_sv.data_ptr(), W, 16, 16, d_fpos.data_ptr(),
                                                len(fpos), C.byref(popts), d_uc.data_ptr(), d_um.data_ptr(), None))
    out["uv_palette16"] = entry(ms, len(fpos) * (256 * 2 * 2 + abi.UV_PALETTE_SLOTS * (256 + 36)),
                                "per block: the 16x16 U and V source (2 B / sample), 4 maps (1 B / sample), candidates")
    out["uv_palette16"]["blocks"] = len(fpos)
    uc = np.frombuffer(d_uc.cpu().numpy().tobytes(), abi.UV_PALETTE_CAND_DTYPE).reshape(len(fpos), -1)
    out["uv_palette16"]["exact_blocks"] = int((uc["exact"][:, 0] == 1).sum())
    out["uv_palette16"]["lossy_blocks"] = int(((uc["exact"][:, 0] == 0) & (uc["n_colors"].max(1) > 0)).sum())
    # deblocking of the three planes (frame_deblock at the shipped levels)
    pwm, phm, _, _, bid = synth.partition_maps(pw // 4, ph // 4, 7)
    tx = synth.transform_maps(pwm, phm, bid, 8)
    planes = [synth.blocky_plane(pw, ph, bid, 7), synth.blocky_plane(pcw, pch, bid[::2, ::2], 8),
              synth.blocky_plane(pcw, pch, bid[::2, ::2], 9)]
    d0 = [t16(p) for p in planes]
    dp = [p.clone() for p in d0]
    maps = [t8(m) for m in list(tx) + [pwm, phm]]
    g = abi.DeblockFrameParams()
    g.w8, g.h8, g.disp_w, g.disp_h, g.sub_x, g.sub_y, g.mono, g.bd = pw, ph, W, H, 1, 1, 0, 8
    scr = torch.empty(max(1, lib.mt_deblock_frame_scratch_bytes(C.byref(g))), dtype=torch.uint8, device=dev)
    ly, luv, _ = mt.loop_filter_levels(wl["qidx"], 1, 1)

    def reset_db():
        for a, b in zip(dp, d0):
            a.copy_(b)

    ms = timed(lambda: lib.mt_deblock_frame_device(*[p.data_ptr() for p in dp], *[m.data_ptr() for m in maps],
                                                   C.byref(g), ly, luv, luv, scr.data_ptr(), None), reset_db)
    samples = pw * ph + 2 * pcw * pch
    out["deblock"] = entry(ms, 4 * samples, "2 B read + 2 B write per sample (3 planes, both edge directions)")
    out["deblock"]["levels"] = [ly, luv, luv]
    # CDEF: the table pass alone (device events) and the whole frame (host search inside)
    src, rec, skip = synth.cdef_inputs(W, H, 1, 1, False, 3)
    prm = mt.cdef_params(W, H, 1, 1, wl["qidx"])
    r0 = [t16(p) for p in rec]
    rr = [p.clone() for p in r0]
    ss = [t16(p) for p in src]
    sk = t8(skip)
    nb, nu = skip.size, ((prm.w8 + 63) // 64) * ((prm.h8 + 63) // 64)
    dirs = torch.empty(nb, dtype=torch.uint8, device=dev)
    vars_ = torch.empty(nb, dtype=torch.int32, device=dev)
    tabs = [torch.empty((nu, 12), dtype=torch.int64, device=dev) for _ in range(3)]
    ms_tab = timed(lambda: lib.mt_cdef_tables_device(*[p.data_ptr() for p in rr], *[p.data_ptr() for p in ss],
                                                     sk.data_ptr(), C.byref(prm), dirs.data_ptr(), vars_.data_ptr(),
                                                     *[t.data_ptr() for t in tabs], None))
    cscr = torch.empty(lib.mt_cdef_scratch_bytes(C.byref(prm)), dtype=torch.uint8, device=dev)
    dec = abi.CdefDecision()

    def reset_cdef():
        for a, b in zip(rr, r0):
            a.copy_(b)

    ms_frame = timed(lambda: lib.mt_cdef_frame_device(*[p.data_ptr() for p in rr], *[p.data_ptr() for p in ss],
                                                      sk.data_ptr(), C.byref(prm), cscr.data_ptr(), C.byref(dec), None,
                                                      None), reset_cdef)
    out["cdef_tables"] = entry(ms_tab, 4 * samples, "2 B recon + 2 B source read per sample")
    out["cdef_tables"]["bound"] = "issue (12 candidate filters + weighted SSE per sample)"
    out["cdef_frame"] = entry(ms_frame, 6 * samples, "tables + apply: 2 B recon + 2 B source + 2 B write")
    out["cdef_frame"]["cdef_bits"] = dec.bits
    out["workload"] = "1920x1080 4:2:0, qindex 70; L2 flushed before each timed call"
    return out


def measure_level8(dev, wl, steps, warmup, op_peak, hbm_peak, cpu):
    """The batched 8x8 RDO level over a reconstruction snapshot of the frame
    (every block x 13 modes x 5 types): device time after an L2 flush, the
    host ABI call, the integer-op roofline, and the oracle over the same
    candidates on all host cores with its results asserted equal."""
    import torch
    import maroontree_b200 as mt
    from maroontree_b200 import abi

    blocks, combos = wl["blocks"], wl["combos"]
    nb, nc = len(blocks), len(combos)
    n = nb * nc
    costs = mt.coef_costs(wl["cdfs"])
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a).view(np.uint8).copy()).to(dev)
    d_src, d_rec, d_qm = t(wl["src"]), t(wl["rec"]), t(wl["qm"])
    d_costs = t(np.frombuffer(bytes(costs), np.uint8))
    d_blocks, d_combos = t(blocks), t(combos)
    d_best = torch.empty(nb * abi.BEST_DTYPE.itemsize, dtype=torch.uint8, device=dev)
    d_res = torch.empty(n * abi.RESULT_DTYPE.itemsize, dtype=torch.uint8, device=dev)
    d_keys = torch.empty(mt.rdo_level8_scratch_bytes(nb, nc), dtype=torch.uint8, device=dev)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev)

    def launch():
        mt.rdo_level8_device(d_src, d_rec, wl["prm"], wl["q"], d_qm, d_costs, d_blocks, nb, d_combos, nc, d_best,
                             d_res, d_keys, stream=stream.cuda_stream)

    for _ in range(max(warmup, 3)):
        launch()
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    for i in range(steps):
        flush.zero_()
        ev[i][0].record(stream)
        launch()
        ev[i][1].record(stream)
    torch.cuda.synchronize()
    step_ms = float(np.mean([a.elapsed_time(b) for a, b in ev]))
    src, rec = wl["src"], wl["rec"]
    e2e = []
    for _ in range(max(1, steps)):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        mt.rdo_level8(src, rec, wl["prm"], wl["q"], wl["qm"], costs, blocks, combos)
        e2e.append(time.perf_counter() - t0)
    res_gpu = d_res.cpu().numpy().view(abi.RESULT_DTYPE)
    ops = chain_ops(combos, res_gpu, nb, wl["qm"] is not None)
    achieved = ops / (step_ms / 1e3)
    alg_bytes = n * (32 + 128 + 66) + nb * 60
    out = {"metric": LEVEL_METRIC, "value": round(MPIX / (step_ms / 1e3), 3), "ms": round(step_ms, 4),
           "e2e_mpix_s": round(MPIX / float(np.median(e2e)), 3), "config": level_config(nb, nc),
           "roofline": {"bound": "int32/fp32 issue", "achieved_tops": round(achieved / 1e12, 3),
                        "peak_tops": round(op_peak / 1e12, 3), "frac": round(achieved / op_peak, 4),
                        "traffic": NCU_DRAM_BYTES_PER_LAUNCH, "ops_per_launch": ops,
                        "hbm_frac": round(alg_bytes / (step_ms / 1e3) / 1e9 / hbm_peak, 4)},
           "gpu_launches": 4 * steps}
    if cpu:
        threads = os.cpu_count() or 1
        ref, dt = cpu_level(wl, threads)
        out["cpu_baseline"] = {"value": round(MPIX / dt, 4), "unit": "MPix/s", "cores": threads, "kind": "port",
                               "sample": f"the whole level, {n} candidates ({dt:.2f} s)"}
        out["results_equal_oracle"] = res_gpu.tobytes() == ref.tobytes()
        if not out["results_equal_oracle"]:
            raise SystemExit("bench: the GPU level's results differ from the oracle's")
    return out


BATCH = 8  # 1080p frames of the batched measurement (seeds SEED .. SEED + 7)


def measure_batch(steps, avif_alone, reps=3):
    """mt_encode_rgb8_batch over BATCH different 1920x1080 4:2:0 quality-60
    frames (the headline's frame and seven more seeds of the generator): all
    their 8x8 decisions in one persistent launch, their host work on threads
    of their own.  Wall time of the call (host RGB in, AVIF bytes out), the
    aggregate MPix/s, and each file checked against the single-image call."""
    from maroontree_b200 import abi, synth
    from maroontree_b200 import encoder as enc

    imgs = [synth.generate_rgb(W, H, SEED + k, sigma=4.0, variant="1080p") for k in range(BATCH)]
    cfg = enc.config(quality=QUALITY, chroma=0)
    out = enc.encode_rgb8_batch(imgs, cfg)  # warm-up (buffers for every image)
    times = []
    for _ in range(max(reps, 1)):
        t0 = time.perf_counter()
        out = enc.encode_rgb8_batch(imgs, cfg)
        times.append(time.perf_counter() - t0)
    dt = float(np.median(times))
    same = out[0] == avif_alone and all(o == enc.encode_rgb8(im, cfg) for o, im in zip(out[1:3], imgs[1:3]))
    if not same:
        raise SystemExit("bench: a batched file differs from the image encoded alone")
    return {"images": BATCH, "ms": round(dt * 1e3, 2), "mpix_s": round(BATCH * MPIX / dt, 2),
            "ms_per_image": round(dt * 1e3 / BATCH, 2), "bytes_equal_alone": same,
            "workload": f"mt_encode_rgb8_batch of {BATCH} 1920x1080 4:2:0 quality 60 frames (generator seeds "
                        f"{SEED}..{SEED + BATCH - 1}), host RGB in, AVIF bytes out, wall time of the call"}


C3_W = C3_H = 4096  # the 4096x4096 4:4:4 quality-60 frame: two tiles


def measure_c3(dev, hbm_peak, steps, reps=5, encode=True):
    """The 4096x4096 frame (generator seed 5, sigma 8 noise on the left half,
    piecewise-constant cells on the right), 4:4:4 quality 60: the whole encode
    through mt_encode_rgb8 (host RGB in, AVIF out; two tiles), and the frame
    filters at that size against the HBM roofline -- deblocking of the three
    planes with the encoder's uniform 8x8 geometry and with random AV1-shaped
    geometry, the CDEF tables and the whole frame CDEF (tables, strength
    search, apply) -- each timed with CUDA events after an L2 flush."""
    import ctypes as C

    import torch
    import maroontree_b200 as mt
    from maroontree_b200 import abi, synth
    from maroontree_b200 import encoder as enc

    lib = mt.load()
    rgb = synth.generate_rgb(C3_W, C3_H, 5, sigma=8.0, variant="large")
    res = {}
    if encode:
        cfg = enc.config(quality=60, chroma=2)
        first = enc.encode_rgb8(rgb, cfg)  # warm-up (buffers, module)
        times, st = [], abi.EncodeStats()
        for _ in range(max(steps, 3)):
            t0 = time.perf_counter()
            out = enc.encode_rgb8(rgb, cfg, stats=st)
            times.append(time.perf_counter() - t0)
            if out != first:
                raise SystemExit("bench: the 4096x4096 encode is not repeatable")
        dt = float(np.median(times))
        res = {"workload": "mt_encode_rgb8 of the 4096x4096 4:4:4 quality-60 frame (two tiles), host RGB in, AVIF "
                           "out, median wall time",
               "ms": round(dt * 1e3, 2), "mpix_s": round(C3_W * C3_H / dt / 1e6, 2), "avif_bytes": len(first),
               "blocks_kernel_ms": round(st.blocks_ms, 3), "levels": int(st.levels), "blocks": int(st.blocks),
               "tokens": int(st.tokens)}
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=dev)
    t16 = lambda a: torch.from_numpy(np.ascontiguousarray(a).astype(np.int16)).to(dev)
    t8 = lambda a: torch.from_numpy(np.ascontiguousarray(a, np.uint8)).to(dev)

    def timed(fn, reset):
        ms = []
        for i in range(reps + 2):
            reset()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            flush.zero_()
            torch.cuda._sleep(200_000)
            a.record()
            rc = fn()
            b.record()
            torch.cuda.synchronize()
            assert rc == 0, rc
            if i >= 2:
                ms.append(a.elapsed_time(b))
        return float(np.median(ms))

    def entry(ms, nbytes, what):
        gbs = nbytes / (ms / 1e3) / 1e9
        return {"ms": round(ms, 4), "alg_bytes": int(nbytes), "achieved_gbs": round(gbs, 1),
                "frac_hbm": round(gbs / hbm_peak, 4), "bytes": what}

    src, rec, skip = synth.cdef_inputs(C3_W, C3_H, 0, 0, False, 5, rgb=rgb)
    samples = 3 * C3_W * C3_H
    r0 = [t16(p) for p in rec]
    rr = [p.clone() for p in r0]
    ss = [t16(p) for p in src]

    def reset():
        for a, b in zip(rr, r0):
            a.copy_(b)

    g = abi.DeblockFrameParams()
    g.w8, g.h8, g.disp_w, g.disp_h, g.sub_x, g.sub_y, g.mono, g.bd = C3_W, C3_H, C3_W, C3_H, 0, 0, 0, 8
    scr = torch.empty(max(1, lib.mt_deblock_frame_scratch_bytes(C.byref(g))), dtype=torch.uint8, device=dev)
    ly, luv, _ = mt.loop_filter_levels(70, 0, 0)
    n4r, n4c = C3_H // 4, C3_W // 4
    two = np.full((n4r, n4c), 2, np.uint8)
    uniform = [two, two, np.tile((np.arange(n4c) % 2 == 0).astype(np.uint8), (n4r, 1)),
               np.tile((np.arange(n4r) % 2 == 0).astype(np.uint8)[:, None], (1, n4c)), two, two]
    pwm, phm, _, _, bid = synth.partition_maps(n4c, n4r, 7)
    random_maps = list(synth.transform_maps(pwm, phm, bid, 8)) + [pwm, phm]
    outp = [torch.empty_like(p) for p in rr]
    for tag, mp in (("deblock_uniform8", uniform), ("deblock_random", random_maps)):
        maps = [t8(m) for m in mp]
        # the encoder's entry: unfiltered planes in, filtered planes out
        ms = timed(lambda: lib.mt_deblock_frame_device_to(*[p.data_ptr() for p in rr], *[p.data_ptr() for p in outp],
                                                          *[m.data_ptr() for m in maps], C.byref(g), ly, luv, luv,
                                                          scr.data_ptr(), None), reset)
        res[tag] = entry(ms, 4 * samples, "2 B read + 2 B write per sample (3 planes, both edge directions)")
        # the in-place entry (a snapshot copy of the planes first)
        ms = timed(lambda: lib.mt_deblock_frame_device(*[p.data_ptr() for p in rr], *[m.data_ptr() for m in maps],
                                                       C.byref(g), ly, luv, luv, scr.data_ptr(), None), reset)
        res[tag]["in_place_ms"] = round(ms, 4)
    prm = mt.cdef_params(C3_W, C3_H, 0, 0, 70)
    sk = t8(skip)
    nu = (C3_W // 64) * (C3_H // 64)
    dirs = torch.empty(skip.size, dtype=torch.uint8, device=dev)
    vars_ = torch.empty(skip.size, dtype=torch.int32, device=dev)
    tabs = [torch.empty((nu, 12), dtype=torch.int64, device=dev) for _ in range(3)]
    ms = timed(lambda: lib.mt_cdef_tables_device(*[p.data_ptr() for p in rr], *[p.data_ptr() for p in ss],
                                                 sk.data_ptr(), C.byref(prm), dirs.data_ptr(), vars_.data_ptr(),
                                                 *[t.data_ptr() for t in tabs], None), reset)
    res["cdef_tables"] = entry(ms, 4 * samples, "2 B recon + 2 B source read per sample")
    res["cdef_tables"]["bound"] = "issue (12 candidate filters + weighted SSE per sample)"
    cscr = torch.empty(lib.mt_cdef_scratch_bytes(C.byref(prm)), dtype=torch.uint8, device=dev)
    dec = abi.CdefDecision()
    ms = timed(lambda: lib.mt_cdef_frame_device(*[p.data_ptr() for p in rr], *[p.data_ptr() for p in ss],
                                                sk.data_ptr(), C.byref(prm), cscr.data_ptr(), C.byref(dec), None,
                                                None), reset)
    res["cdef_frame"] = entry(ms, 6 * samples, "tables + apply: 2 B recon + 2 B source + 2 B write per sample")
    res["cdef_frame"]["cdef_bits"] = dec.bits
    res["filters_workload"] = ("4096x4096 4:4:4 planes of the same frame (luma, contrast-reduced chroma copies) with "
                               "seeded per-unit coding error; qindex 70; L2 flushed before each timed call")
    return res


def run_ours(args):
    import torch
    import maroontree_b200 as mt
    from maroontree_b200 import abi
    from maroontree_b200 import encoder as enc

    _, _, local = dist_env()
    torch.cuda.set_device(local)
    ranks = Replicas("nccl")
    world, rank = ranks.world, ranks.rank
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    mt.load()
    rgb = encode_rgb()
    cfg = enc.config(quality=QUALITY, chroma=0)  # MT_CHROMA_420
    # replicas: every rank encodes its own copy of the frame, no collective on the data path
    d_rgb = torch.from_numpy(np.ascontiguousarray(rgb).reshape(-1)).to(dev)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev)  # the legacy default stream, the library's stream

    def step(stats=None):
        return enc.encode_rgb8_device(d_rgb.data_ptr(), W, H, cfg, stats=stats)

    for _ in range(max(args.warmup, 3)):
        avif = step()
    torch.cuda.synchronize()
    ranks.barrier()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    stats = [abi.EncodeStats() for _ in range(args.steps)]
    with ClockSampler(local) as clk:
        torch.cuda.synchronize()
        for i in range(args.steps):
            flush.zero_()  # L2 flush between timed steps (outside the events)
            ev[i][0].record(stream)
            avif = step(stats[i])
            ev[i][1].record(stream)
        torch.cuda.synchronize()
    step_ms = ranks.max(float(np.mean([a.elapsed_time(b) for a, b in ev])), device=dev)
    value = ranks.job_value(step_ms)

    # e2e through mt_encode_rgb8: host RGB (pinned) in, AVIF bytes out
    pinned = torch.empty(rgb.nbytes, dtype=torch.uint8, pin_memory=True)
    pinned.numpy()[:] = np.ascontiguousarray(rgb).reshape(-1)
    host_rgb = pinned.numpy().reshape(rgb.shape)
    e2e_times, e2e_stats = [], abi.EncodeStats()
    ranks.barrier()
    for _ in range(max(1, args.steps)):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        avif_e2e = enc.encode_rgb8(host_rgb, cfg, stats=e2e_stats)
        e2e_times.append(time.perf_counter() - t0)
    e2e_s = ranks.max(float(np.median(e2e_times)), device=dev)
    if avif_e2e != avif:
        raise SystemExit("bench: the host and device entry points gave different files")

    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    hbm_peak = peaks.get("hbm_gbs", 6650.0)
    clocks = clk.summary()
    clk_mhz = clocks.get("sm_mhz") or 1965.0
    op_peak = SMS * LANES_PER_SM * clk_mhz * 1e6  # thread operations per second at the sampled SM clock
    blocks_ms = float(np.mean([st.blocks_ms for st in stats]))
    nblocks, nlevels = stats[0].blocks, stats[0].levels
    ops = nblocks * block_ops(SUB)
    achieved = ops / (blocks_ms / 1e3)

    secondary = {}
    cpu = parity = None
    if rank == 0:
        secondary["batch"] = measure_batch(args.steps, avif)
        secondary["c3"] = measure_c3(dev, hbm_peak, args.steps)
    nocpu = world > 1 or args.no_cpu
    if rank == 0 and not args.headline_only:
        wl = make_workload()
        secondary["level8"] = measure_level8(dev, wl, args.steps, args.warmup, op_peak, hbm_peak, not nocpu)
        secondary["frame_filters"] = measure_filters(dev, wl, hbm_peak)
        secondary["level4"] = measure_small_level(dev, wl, 4, cpu=not nocpu)
        secondary["level16"] = measure_small_level(dev, wl, 16, cpu=not nocpu)
        split16 = {k: measure_split16(dev, wl, k == "search", cpu=not nocpu) for k in ("dct", "search")}
        split16["depth2"] = measure_split16(dev, wl, False, cpu=not nocpu, depth2=True)
        secondary["split16"] = split16
        leaf8 = {k: measure_leaf8(dev, wl, k == "refine", cpu=not nocpu) for k in ("luma", "refine")}
        leaf8["luma16"] = measure_leaf8(dev, wl, False, cpu=not nocpu, n16=True)
        leaf8["refine16"] = measure_leaf8(dev, wl, True, cpu=not nocpu, n16=True)
        leaf8["luma32"] = measure_leaf8(dev, wl, False, cpu=not nocpu, n32=True)
        leaf8["quad32_64"] = measure_leaf64(dev, wl, False, cpu=not nocpu)
        leaf8["grid16_64"] = measure_leaf64(dev, wl, True, cpu=not nocpu)
        secondary["uv16_420"] = measure_uv16(dev, wl, cpu=not nocpu)
        secondary["uv_search"] = {f: measure_uv16(dev, wl, cpu=not nocpu, form=f) for f in ("444", "420_32", "444_32")}
        secondary["leaf8"] = leaf8
    if rank == 0 and not nocpu:
        from oracle import build as obuild

        obuild.build()
        threads = os.cpu_count() or 1
        want, dt = oracle_encode(rgb, threads)
        cpu = {"value": round(MPIX / dt, 4), "unit": "MPix/s", "cores": threads, "kind": "port",
               "sample": f"one whole 1920x1080 encode by the oracle ({dt:.2f} s)"}
        # the timed encode's file must be the oracle encode's, byte for byte
        parity = {"avif_bytes_equal_oracle": avif == want, "bytes": len(avif)}
        if avif != want:
            raise SystemExit("bench: the GPU encode's file differs from the oracle encode's")

    line = {
        "metric": METRIC, "value": round(value, 3), "unit": "MPix/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(step_ms, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32+f32",
        "data": "synthetic", "config": config_line(),
        "parallelism": f"replicas x{world}",
        "e2e": {"value": round(ranks.job_value(e2e_s * 1e3), 3), "unit": "MPix/s",
                "h2d_bytes_per_step": int(e2e_stats.h2d_bytes), "d2h_bytes_per_step": int(e2e_stats.d2h_bytes)},
        "roofline": {"bound": "int32/fp32 issue", "achieved": round(achieved / 1e12, 4),
                     "peak": round(op_peak / 1e12, 3), "unit": "Tops/s", "frac": round(achieved / op_peak, 4),
                     "traffic": None, "kernel": "encode_blocks_kernel",
                     "ops_per_launch": int(ops), "kernel_ms": round(blocks_ms, 4),
                     "ops_basis": "per 8x8 block: 13 predictions + 91 (mode, type) chains with every coefficient "
                                  "counted + two chroma chains, by the per-stage operation table of the oracle",
                     "peak_basis": f"{SMS} SMs x {LANES_PER_SM} INT32/FP32 lanes x the sampled SM clock "
                                   f"({clk_mhz:.0f} MHz); no measured integer peak exists",
                     "dependency": {"levels": int(nlevels), "blocks": int(nblocks),
                                    "us_per_level": round(blocks_ms * 1e3 / max(nlevels, 1), 3),
                                    "note": "the kernel is bound by its chain of dependent 8x8 blocks (a block "
                                            "needs its left, top, top-left and, where its edges use them, "
                                            "top-right and bottom-left neighbours), not by issue or HBM"}},
        "host": {"call_ms": round(float(np.mean([st.call_ms for st in stats])), 4),
                 "blocks_kernel_ms": round(blocks_ms, 4), "tokens": int(stats[0].tokens),
                 "avif_bytes": len(avif)},
        "parity": parity,
        "gpu_launches": int(sum(st.kernel_launches for st in stats)),
        "clocks": clocks,
        "cpu_baseline": cpu,
    }
    line.update(secondary)
    ranks.emit(line)
    ranks.close()
    return 0


# The single measurements of --only: name -> (what it runs).
ONLY = {
    "uv16": "pick_uv16_420 over the 8,040 16x16 leaves of the 1080p frame (uv16_420_kernel)",
    "quad32": "the 64x64 leaf's four-TX_32X32 leg, 480 blocks x 13 modes (quad32_kernel)",
    "grid16": "the 64x64 leaf's sixteen-TX_16X16 leg, 480 blocks (grid16_kernel)",
    "leaf32": "the 32x32 leaf's mode-loop candidates, 1,980 blocks x 13 modes (leaf_kernel<32>)",
    "c3_filters": "the 4096x4096 4:4:4 frame filters: deblocking and CDEF (lf_fused_kernel, the CDEF search)",
    "uv444": "pick_uv16_444 over the 8,040 16x16 leaves of the 1080p frame at 4:4:4 (uv444_kernel<16>)",
    "uv32_420": "pick_uv32_420 over the 1,980 32x32 leaves of the 1080p frame (uv32_420_kernel)",
    "uv32_444": "pick_uv32_444 over the 1,980 32x32 leaves of the 1080p frame at 4:4:4 (uv444_kernel<32>)",
}


def run_only(args):
    import torch
    import maroontree_b200 as mt

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    mt.load()
    if args.only == "c3_filters":
        try:
            peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        except (OSError, ValueError):
            peaks = {}
        out = measure_c3(dev, peaks.get("hbm_gbs", 6650.0), 1, reps=1, encode=False)
    else:
        wl = make_workload()
        run = {"uv16": lambda: measure_uv16(dev, wl, reps=1, cpu=False),
               "uv444": lambda: measure_uv16(dev, wl, reps=1, cpu=False, form="444"),
               "uv32_420": lambda: measure_uv16(dev, wl, reps=1, cpu=False, form="420_32"),
               "uv32_444": lambda: measure_uv16(dev, wl, reps=1, cpu=False, form="444_32"),
               "quad32": lambda: measure_leaf64(dev, wl, False, reps=1, cpu=False),
               "grid16": lambda: measure_leaf64(dev, wl, True, reps=1, cpu=False),
               "leaf32": lambda: measure_leaf8(dev, wl, False, reps=1, cpu=False, n32=True)}[args.only]
        out = run()
    print(json.dumps({"only": args.only, "what": ONLY[args.only], **out}))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--headline-only", action="store_true", help="skip the secondary kernel-level measurements")
    ap.add_argument("--only", choices=sorted(ONLY),
                    help="run one secondary measurement alone (one timed call after the warm-up calls, no CPU leg) "
                         "and print its JSON; the kernel profiles are taken on these runs")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    if args.only:
        return run_only(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
