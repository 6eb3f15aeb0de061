#!/usr/bin/env python
"""Benchmark: Taylor-FFA acceleration search (f, fdot) + boxcar S/N + candidate
compaction on one B200 per rank.

Workload (one "step" = one pass of the hot path over one time series):
  2^22 float32 samples at 64 us (268 s), seed 7, N(0,1) noise plus 4 injected
  accelerated pulsars; search f in [5, 50] Hz, accel in [-200, 200] m/s^2,
  nbins 64, eta 2, boxcar widths {1,2,3,4,6,8,12,16}; scores of all
  1,932,740 final (accel, freq) cells x 8 widths, compacted at S/N >= 7.
Metric: param-trials/s = final coordinates x widths per second (whole job).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun every rank runs an independent replica (the FFA of one series
does not shard: "replicas only"); value = trials of all ranks / max step time.
The reference arm times the reference's own CPU code (oracle/_ref, built from
the reference sources with its Release flags) on the host cores.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "param-trials/s (FFA+S/N)"
UNIT = "param-trials/s"
SNR_MIN = 7.0
FLUSH_BYTES = 256 << 20  # > 126 MB L2: written between timed steps


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--storage", default="fp32", choices=["fp32", "bf16"])
    ap.add_argument("--basis", default="taylor", choices=["taylor", "chebyshev"],
                    help="polynomial basis of the pruning workload")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-parity", action="store_true",
                    help="skip the comparison of the candidates with the reference's CPU code")
    ap.add_argument("--no-autotune", action="store_true",
                    help="keep the default launch shapes instead of timing the candidates first")
    ap.add_argument("--tuning", default=None,
                    help="apply these launch shapes (JSON of FFACUDA.tuning) instead of autotuning")
    ap.add_argument("--no-mixed-batched", action="store_true",
                    help="skip the BF16-storage + batched measurement beside the plain FP32 line")
    ap.add_argument("--no-reference-gpu", action="store_true",
                    help="skip timing the reference's own GPU path (oracle/_ref/libloki_ref_cuda.so)")
    ap.add_argument("--no-configs", action="store_true",
                    help="skip the short runs of the other workloads summarised under `configs`")
    ap.add_argument("--reference-gpu-child", default=None, help=argparse.SUPPRESS)
    ap.add_argument("--pipeline-execs", type=int, default=2,
                    help="executors (own compute streams) the end-to-end search pipeline alternates between")
    ap.add_argument("--workload", default="taylor_accel",
                    choices=["taylor_accel", "freq_sweep", "prune_jerk", "mc_cascade", "multi_series",
                             "octave_sweep", "beam_scheme", "fourier_accel"],
                    help="taylor_accel (default): Taylor (f, fdot) FFA + S/N; freq_sweep: plain period "
                         "sweep; prune_jerk: FFA to 32 segments + one pruning run; mc_cascade: 8-stage "
                         "Monte-Carlo threshold cascade; multi_series: 512 series of uneven length, "
                         "batched with CUDA graphs; octave_sweep: the frequency sweep over octave "
                         "regions (FFAFreqSweep) on the freq_sweep series; beam_scheme: the "
                         "DynamicThresholdScheme beam search (16 stages, reference default sizes); "
                         "fourier_accel: the default search through the Fourier-domain FFA")
    return ap.parse_args()


def workload():
    from loki_b200.synthetic import taylor_accel_workload

    return taylor_accel_workload(seed=7)


def config_dict(params, extra=None):
    d = {
        "workload": "taylor_ffa_accel_2^22x64us_nbins64_eta2",
        "nsamps": params["nsamps"],
        "tsamp": params["tsamp"],
        "nbins": params["nbins"],
        "eta": params["eta"],
        "param_limits": params["param_limits"],
        "score_widths": params["score_widths"],
        "snr_min": SNR_MIN,
        "l2": f"flushed: {FLUSH_BYTES >> 20} MiB written between timed steps",
        "parallelism": "replicas",
    }
    if extra:
        d.update(extra)
    return d


# ---- clocks -----------------------------------------------------------------

class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "50"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
            # Wait (up to 5 s) for the first sample, so that the timed region
            # that follows is covered by samples.
            t_end = time.time() + 5.0
            while time.time() < t_end and os.path.getsize(self.path) == 0:
                time.sleep(0.02)
        except (OSError, FileNotFoundError):
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        with open(self.path) as fh:
            for line in fh:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


# ---- peaks / ncu data ---------------------------------------------------------

def hbm_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as fh:
            return float(json.load(fh)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def tensor_peak():
    """Dense BF16/FP16 tensor-core peak (TFLOP/s): the measured burst figure if
    present, else the fallback measured earlier on these GPUs."""
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as fh:
            return float(json.load(fh)["bf16_tflops"]), "measured"
    except (OSError, KeyError, ValueError):
        return 1590.0, "fallback"


def ncu_traffic(stage: str):
    """Per-launch DRAM bytes of a stage from the committed ncu summary, if any."""
    p = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    try:
        with open(p) as fh:
            return json.load(fh).get(stage)
    except (OSError, ValueError):
        return None


def smem_peak_gbs(device_index, clk):
    """Nominal shared-memory bandwidth: 128 B/clock/SM x SMs x max SM clock."""
    import torch

    props = torch.cuda.get_device_properties(device_index)
    mhz = (clk or {}).get("sm_max_mhz") or 1965.0
    return 128 * props.multi_processor_count * mhz * 1e6 / 1e9


def stage_roofline(stage_ms, stage_bytes, steps, clk, device_index, brute_adds):
    """Roofline object of the dominant stage.

    HBM-bound stages (merges, merge+score, compaction) report algorithmic HBM
    bytes per launch / average launch time against the measured copy peak.
    The level-0 brute fold reads little HBM data: its bound is shared memory
    (one 4-byte read per sample x level-0 frequency x row from the staged
    series tile, brute_adds = those reads), so it is reported as "smem"
    against the nominal shared-memory bandwidth, with its HBM fraction kept as
    a second field. Every merge level's HBM fraction is listed too."""
    dom = max(stage_ms, key=stage_ms.get)
    dom_ms = stage_ms[dom] / steps
    peak, peak_kind = hbm_peak()
    hbm_ach = stage_bytes[dom] / (dom_ms / 1e3) / 1e9
    levels = {k: (stage_bytes[k] / (stage_ms[k] / steps / 1e3) / 1e9) / peak
              for k in sorted(stage_ms) if k.startswith("merge")}
    hbm = {"achieved": hbm_ach, "peak": peak, "peak_source": peak_kind, "unit": "GB/s", "frac": hbm_ach / peak,
           "algorithmic_bytes": stage_bytes[dom]}
    if dom.startswith("brute_fold"):
        smem_bytes = 4 * brute_adds
        speak = smem_peak_gbs(device_index, clk)
        sach = smem_bytes / (dom_ms / 1e3) / 1e9
        return {"bound": "smem", "kernel": dom, "achieved": sach, "peak": speak, "unit": "GB/s",
                "frac": sach / speak, "peak_source": "nominal 128 B/clock/SM x SMs at the max SM clock",
                "algorithmic_bytes": smem_bytes, "adds": brute_adds, "avg_ms": dom_ms,
                "traffic": ncu_traffic(dom), "hbm": hbm, "merge_hbm_frac": levels}
    return {"bound": "hbm", "kernel": dom, "achieved": hbm_ach, "peak": peak, "peak_source": peak_kind,
            "unit": "GB/s", "frac": hbm_ach / peak, "traffic": ncu_traffic(dom),
            "algorithmic_bytes": stage_bytes[dom], "avg_ms": dom_ms, "merge_hbm_frac": levels}


# ---- reference CPU path -------------------------------------------------------

def reference_runner(params, kind="timing"):
    from oracle import ref

    nthreads = os.cpu_count() or 1
    cfg = ref.make_cfg(params["nsamps"], params["tsamp"], params["nbins"], params["eta"], params["param_limits"],
                       nthreads=nthreads)
    ffa = ref.RefFFA(cfg, kind=kind)
    widths = np.array(params["score_widths"], dtype=np.uint64)
    ntrials = int(ffa.ncoords[-1]) * widths.size

    def step(ts_e, ts_v):
        fold = ffa.execute(ts_e, ts_v)
        scores = ref.snr_boxcar_3d(fold, widths, params["nbins"], nthreads=nthreads, kind=kind).ravel()
        idx = np.flatnonzero(scores >= SNR_MIN)  # FFAFreqSweep compaction (>=, flat order)
        return idx, scores[idx]

    return step, ntrials, nthreads


def cpu_baseline(params, ts_e, ts_v, budget_s=20.0):
    from oracle import ref

    if not ref.available("timing"):
        return None
    step, ntrials, nthreads = reference_runner(params)
    step(ts_e, ts_v)  # warm-up
    times = []
    t_end = time.perf_counter() + budget_s
    while len(times) < 5 and (not times or time.perf_counter() + times[-1] < t_end):
        t0 = time.perf_counter()
        step(ts_e, ts_v)
        times.append(time.perf_counter() - t0)
    med = statistics.median(times)
    return {"value": ntrials / med, "unit": UNIT, "cores": nthreads, "kind": "reference",
            "sample": f"full workload, median of {len(times)} runs of FFA::execute + snr_boxcar_3d + "
                      f"compaction ({med:.3f} s each), reference CPU code built with its Release flags"}


def candidate_parity(params, ts_e, ts_v, idx, snr):
    """Compares a search's candidates (flat cell x width indices in increasing
    order, S/N) with the reference's own CPU code on the same series: the IEEE
    build of the reference (FFA<float>::execute + snr_boxcar_3d, then the
    FFAFreqSweep compaction score >= snr_min in flat order)."""
    from oracle import ref

    if not ref.available("parity"):
        return {"checked": False, "why": "oracle/_ref was not built"}
    step, _, nthreads = reference_runner(params, kind="parity")
    t0 = time.perf_counter()
    r_idx, r_snr = step(ts_e, ts_v)
    secs = time.perf_counter() - t0
    idx = np.asarray(idx, dtype=np.int64)
    snr = np.asarray(snr, dtype=np.float32)
    same_idx = idx.shape == r_idx.shape and bool(np.array_equal(idx, r_idx))
    same_bits = same_idx and bool(np.array_equal(snr.view(np.uint32), r_snr.astype(np.float32).view(np.uint32)))
    max_diff = float(np.max(np.abs(snr - r_snr))) if same_idx and snr.size else None
    return {"checked": True, "candidates_equal": same_idx, "snr_bits_equal": same_bits,
            "candidates_match": same_idx and (max_diff is None or max_diff <= 1e-4),
            "snr_max_abs_diff": max_diff, "n": int(idx.size), "n_ref": int(r_idx.size),
            "vs": "oracle/_ref/libloki_ref_parity.so (the reference's CPU code, IEEE build)",
            "ref_threads": nthreads, "ref_seconds": secs}


# ---- the reference's own GPU path ---------------------------------------------

def _reference_gpu_child(args):
    """Child process: time the reference's GPU FFA + scorer (FFACUDA::execute on
    device spans, snr_boxcar_3d_cuda_d; lib/*_cuda.cu with its Release flags) on
    the workload's series, as this library's line times its own (CUDA events,
    L2 flushed between steps); write the timing as JSON to OUT.json and the
    last step's scores to OUT.npy."""
    import torch

    from oracle import ref

    if args.workload != "taylor_accel":
        raise SystemExit(f"the reference's GPU path is timed on taylor_accel only, not {args.workload}")
    ts_e, ts_v, params, _ = workload()
    torch.cuda.set_device(0)
    cfg = ref.make_cfg(params["nsamps"], params["tsamp"], params["nbins"], params["eta"], params["param_limits"])
    R = ref.RefGPU(cfg, device=0, use_fourier=False)
    widths = np.asarray(params["score_widths"], np.uint32)
    e = torch.from_numpy(ts_e).cuda()
    v = torch.from_numpy(ts_v).cuda()
    fold = torch.empty(R.fold_len, dtype=torch.float32, device="cuda")
    w = torch.from_numpy(widths.view(np.int32)).cuda()
    scores = torch.empty(R.ncoords_final * widths.size, dtype=torch.float32, device="cuda")
    flush = torch.empty(FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")
    sp = torch.cuda.current_stream().cuda_stream

    def step():
        R.scores(e.data_ptr(), v.data_ptr(), params["nsamps"], fold.data_ptr(), w.data_ptr(), widths.size,
                 scores.data_ptr(), sp)

    for _ in range(max(args.warmup, 3)):
        step()
    torch.cuda.synchronize()
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    stops = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    for k in range(args.steps):
        flush.zero_()
        starts[k].record()
        step()
        stops[k].record()
    torch.cuda.synchronize()
    ms = sum(a.elapsed_time(b) for a, b in zip(starts, stops)) / args.steps
    np.save(args.reference_gpu_child + ".npy", scores.cpu().numpy())
    with open(args.reference_gpu_child + ".json", "w") as fh:
        json.dump({"ms_per_step": ms, "ntrials": int(R.ncoords_final * widths.size)}, fh)
    return 0


# At this workload's sizes (segments of 16384 samples) the reference's GPU
# Fourier brute fold launches kernel_fold_complex_unified<false> (lib/kernels_cuda.cu)
# with 256 threads for 33 harmonics: threads 33..255 return before the block's
# DC reduction, whose warp shuffles then name lanes that have exited and whose
# second stage reads per-warp sums that were never written. Its scores come out
# wrong by up to 4e6 in S/N; the code has undefined behaviour, so it is not run.
REF_GPU_FOURIER_WHY = ("not run: the reference's GPU Fourier brute fold takes kernel_fold_complex_unified<false> "
                       "here (2 x 16384 x 4 B > 48 KB shared), whose block reduction follows an early return of "
                       "threads >= nbins_f (undefined behaviour, wrong DC terms)")


def reference_gpu(args, ours_ms, ours_scores):
    """The reference's GPU path timed in a child process (so that a failure
    there cannot take this run with it), compared with this library's scores
    of the same series."""
    import subprocess
    import tempfile

    from oracle import ref

    if args.workload == "fourier_accel":
        return {"checked": False, "why": REF_GPU_FOURIER_WHY}
    if not ref.gpu_available():
        return {"checked": False, "why": "oracle/_ref/libloki_ref_cuda.so was not built"}
    with tempfile.TemporaryDirectory() as td:
        out = os.path.join(td, "refgpu")
        cmd = [sys.executable, os.path.join(ROOT, "bench.py"), "--workload", args.workload, "--steps",
               str(args.steps), "--warmup", str(args.warmup), "--reference-gpu-child", out]
        try:
            r = subprocess.run(cmd, capture_output=True, text=True, timeout=900)
        except subprocess.TimeoutExpired:
            return {"checked": False, "why": "the reference's GPU path did not finish within 900 s"}
        if r.returncode != 0 or not os.path.exists(out + ".json"):
            return {"checked": False, "why": f"the reference's GPU path failed (exit {r.returncode}): "
                                             f"{(r.stderr or '').strip().splitlines()[-1:]}"}
        with open(out + ".json") as fh:
            t = json.load(fh)
        rs = np.load(out + ".npy")
    d = np.abs(rs.astype(np.float64) - np.asarray(ours_scores, np.float64))
    return {"checked": True, "what": "FFACUDA::execute (device spans) + snr_boxcar_3d_cuda_d, the reference's "
                                     "lib/*_cuda.cu built with its Release flags (-O3 -use_fast_math), same "
                                     "series on the same GPU, L2 flushed between steps",
            "ms_per_step": t["ms_per_step"], "value": t["ntrials"] / (t["ms_per_step"] / 1e3), "unit": UNIT,
            "ours_ms_per_step": ours_ms, "speedup": t["ms_per_step"] / ours_ms,
            "scores_max_abs_diff": float(d.max()), "scores_mean_abs_diff": float(d.mean())}


def mixed_batched(args, cfg, ffa, e, v, plain_ms, want_idx, want_snr, nbatch=4):
    """The two systems patterns together on the same series: BF16 fold storage
    and nbatch series per launch (one executor, max_batch = nbatch), ms per
    series against the plain FP32 single-series step, and the first series'
    candidates against the plain ones. FP32 batched is timed beside it."""
    import torch

    from loki_b200.ffa import FFACUDA

    eb = e.reshape(1, -1).repeat(nbatch, 1).contiguous()
    vb = v.reshape(1, -1).repeat(nbatch, 1).contiguous()
    flush = torch.empty(FLUSH_BYTES // 4, dtype=torch.float32, device=e.device)
    cap = 1 << 22
    out = {"nbatch": nbatch, "plain_fp32_ms_per_series": plain_ms}
    for storage in ("bf16", "fp32"):
        fb = FFACUDA(cfg, device_id=e.device.index or 0, fold_storage=storage, max_batch=nbatch)
        fb.set_tuning(ffa.tuning)
        idx = torch.empty(cap, dtype=torch.int32, device=e.device)
        snr = torch.empty(cap, dtype=torch.float32, device=e.device)
        cnt = torch.zeros(1, dtype=torch.int64, device=e.device)
        for _ in range(max(args.warmup, 3)):
            fb.search_batch(eb, vb, SNR_MIN, idx, snr, cnt)
        torch.cuda.synchronize()
        starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
        stops = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
        for k in range(args.steps):
            flush.zero_()
            starts[k].record()
            fb.search_batch(eb, vb, SNR_MIN, idx, snr, cnt)
            stops[k].record()
        torch.cuda.synchronize()
        ms = sum(a.elapsed_time(b) for a, b in zip(starts, stops)) / args.steps / nbatch
        n = int(cnt.item())
        got = idx[:n].cpu().numpy().view(np.uint32)
        per = int(fb.plan.ncoords[-1]) * cfg.n_scoring_widths
        first = got < per
        same = bool(np.array_equal(got[first], want_idx) and
                    np.array_equal(snr[:n].cpu().numpy()[first].view(np.uint32), want_snr.view(np.uint32)))
        out[f"{storage}_batched_ms_per_series"] = ms
        out[f"{storage}_batched_candidates_equal_plain"] = same
        del fb
    out["ratio_mixed_batched_vs_plain"] = plain_ms / out["bf16_batched_ms_per_series"]
    return out


def run_reference(args, rank):
    if rank != 0:
        return 0
    from oracle import ref

    ts_e, ts_v, params, _ = workload()
    if not ref.available("timing"):
        emit({"impl": "reference", "unavailable": "oracle/_ref was not built (make -C oracle ref)"})
        return 0
    step, ntrials, nthreads = reference_runner(params)
    for _ in range(max(args.warmup, 1)):
        step(ts_e, ts_v)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        step(ts_e, ts_v)
        times.append(time.perf_counter() - t0)
    total = sum(times)
    value = ntrials * args.steps / total
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic", "config": config_dict(params, {"cpu_threads": nthreads}),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": nthreads, "kind": "reference",
                         "sample": f"full workload per step, {args.steps} steps"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    emit(line)
    return 0


# ---- our path -------------------------------------------------------------------

def job_throughput(units_per_rank, local_ms, dist=None, device=None):
    """Whole-job throughput of N replicas (one process per GPU): every rank
    processed units_per_rank in local_ms (its own device time); the job took
    the slowest rank's time, so value = units over all ranks / max time.
    Returns (value per second, max ms)."""
    import torch

    t = torch.tensor([float(local_ms)], dtype=torch.float64, device=device)
    world = 1
    if dist is not None:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        world = dist.get_world_size()
    ms_max = float(t.item())
    return units_per_rank * world / (ms_max / 1e3), ms_max


def run_ours(args, rank, world, local_rank):
    import torch

    from loki_b200 import _capi as C
    from loki_b200.configs import PulsarSearchConfig
    from loki_b200.ffa import FFACUDA

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device(f"cuda:{local_rank}"))

    status = 0
    ts_e, ts_v, params, _ = workload()
    cfg = PulsarSearchConfig(params["nsamps"], params["tsamp"], params["nbins"], params["eta"],
                             np.array(params["param_limits"]), use_fourier=False,
                             score_widths=params["score_widths"], snr_min=SNR_MIN)
    ffa = FFACUDA(cfg, device_id=local_rank, fold_storage=args.storage)
    nc = int(ffa.plan.ncoords[-1])
    nw = cfg.n_scoring_widths
    ntrials = nc * nw
    cap = 1 << 20
    dev = f"cuda:{local_rank}"
    e = torch.from_numpy(ts_e).to(dev)
    v = torch.from_numpy(ts_v).to(dev)
    idx = torch.empty(cap, dtype=torch.int32, device=dev)
    snr = torch.empty(cap, dtype=torch.float32, device=dev)
    cnt = torch.zeros(1, dtype=torch.int64, device=dev)
    flush = torch.empty(FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream()
    sp = stream.cuda_stream
    L = C.lib()

    def step():
        C.check(L.lk_ffa_search(ffa._h, e.data_ptr(), v.data_ptr(), SNR_MIN, idx.data_ptr(), snr.data_ptr(),
                                cap, cnt.data_ptr(), sp))

    tuning = None
    if args.tuning:
        ffa.set_tuning(json.loads(args.tuning))
        tuning = ffa.tuning
    elif not args.no_autotune:
        # launch shapes timed on this series before the warm-up (not timed)
        tuning = ffa.autotune(e, v, reps=3)
    for _ in range(max(args.warmup, 3)):
        step()
    torch.cuda.synchronize()
    if ffa.status() != 0:
        raise RuntimeError("device status word set during warm-up")

    ffa.set_profiling(True)
    stage_ms: dict[str, float] = {}
    stage_bytes: dict[str, int] = {}
    stage_launches: dict[str, int] = {}
    launches = 0
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    stops = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    clocks = ClockSampler(local_rank)
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    wall0 = time.perf_counter()
    for k in range(args.steps):
        flush.zero_()
        starts[k].record(stream)
        step()
        stops[k].record(stream)
        for st in ffa.profile():  # synchronises the stream
            key = st["stage"] if st["level"] < 0 else f'{st["stage"]}_l{st["level"]}'
            stage_ms[key] = stage_ms.get(key, 0.0) + st["ms"]
            stage_bytes[key] = st["bytes"]
            stage_launches[key] = st["launches"]
            launches += st["launches"]
    torch.cuda.synchronize()
    wall = time.perf_counter() - wall0
    clk = clocks.stop()
    ffa.set_profiling(False)
    step_ms = sum(a.elapsed_time(b) for a, b in zip(starts, stops)) / args.steps
    value, step_ms_max = job_throughput(ntrials, step_ms, dist, dev)
    ncand = int(cnt.item())
    rescored = ffa.rescored_cells() if args.storage == "bf16" else 0

    # roofline of the dominant stage
    roofline = stage_roofline(stage_ms, stage_bytes, args.steps, clk, local_rank,
                              2 * params["nsamps"] * int(ffa.plan.param_counts[0][-1]))
    stages = {k: {"avg_ms": stage_ms[k] / args.steps, "bytes": stage_bytes[k],
                  "gbs": stage_bytes[k] / (stage_ms[k] / args.steps / 1e3) / 1e9}
              for k in sorted(stage_ms, key=stage_ms.get, reverse=True)}

    # end to end through the public API with host buffers: every step copies
    # its series from pinned host memory and reads its candidates back; the
    # pipeline overlaps step k + 1's copy and step k - 1's read-back with step
    # k's search, and alternates consecutive steps between two executors on
    # their own compute streams (one step's brute fold beside the previous
    # step's merges and scoring)
    e2e = None
    if not args.no_e2e:
        from loki_b200.pipeline import SearchPipeline

        he = torch.from_numpy(ts_e).pin_memory()
        hv = torch.from_numpy(ts_v).pin_memory()
        pipe = SearchPipeline(ffa, SNR_MIN, max_cands=cap, n_exec=args.pipeline_execs)
        for _ in pipe.run([(he, hv)] * args.warmup):
            pass
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        pipe.h2d_bytes = pipe.d2h_bytes = 0
        t0 = time.perf_counter()
        for _ in pipe.run([(he, hv)] * args.steps):
            pass
        e2e_s = time.perf_counter() - t0
        t = torch.tensor([e2e_s], dtype=torch.float64, device=dev)
        if dist is not None:
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e = {"value": ntrials * world * args.steps / float(t.item()), "unit": UNIT,
               "h2d_bytes_per_step": pipe.h2d_bytes // args.steps, "d2h_bytes_per_step": pipe.d2h_bytes // args.steps,
               "api": "loki_b200.pipeline.SearchPipeline over FFACUDA (lk_ffa_search): pinned host series in, "
                      "candidates out, copies overlapped with the previous/next search, "
                      f"{args.pipeline_execs} executors on their own compute streams"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(params, ts_e, ts_v)
    parity = None
    if rank == 0 and not args.no_parity:
        # the last timed step's candidates against the reference's, full size
        parity = candidate_parity(params, ts_e, ts_v, idx[:ncand].cpu().numpy(), snr[:ncand].cpu().numpy())
    mb = None
    if rank == 0 and world == 1 and not args.no_mixed_batched:
        mb = mixed_batched(args, cfg, ffa, e, v, step_ms_max, idx[:ncand].cpu().numpy().view(np.uint32),
                           snr[:ncand].cpu().numpy())
    ref_gpu = None
    if rank == 0 and world == 1 and not args.no_reference_gpu:
        ref_gpu = reference_gpu(args, step_ms_max, ffa.scores(e, v).cpu().numpy())

    others = None
    if rank == 0 and world == 1 and not args.no_configs:
        others = other_configs()

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": step_ms_max, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": config_dict(params, {"fold_storage": args.storage, "final_coords": nc, "n_widths": nw,
                                           "candidates": ncand, "rescored_cells": rescored,
                                           "rescore_margin": list(ffa.rescore_margin),
                                           "tuning": tuning}),
            "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches,
            "clocks": clk, "stages": stages, "wall_s": wall, "parity": parity, "reference_gpu": ref_gpu,
            "mixed_batched": mb, "configs": others,
        }
        emit(line)
        if parity is not None and parity.get("checked") and not parity["candidates_match"]:
            print("bench: the search's candidates differ from the reference's", file=sys.stderr)
            status = 1
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return status


# The other benchmark workloads, each run once in its own process after the
# headline's timed region (steps, warm-up): the plain period sweep (2^21
# samples, nbins 128), the jerk pruning run (2^23 samples, 31 levels), 512
# series of uneven length, the 8-stage Monte-Carlo cascade, the octave sweep,
# the beam search and the Fourier-domain search.
OTHER_CONFIGS = (("freq_sweep", 5, 3), ("prune_jerk", 5, 3), ("multi_series", 1, 3), ("mc_cascade", 5, 3),
                 ("octave_sweep", 3, 3), ("beam_scheme", 3, 3), ("fourier_accel", 5, 3))
OTHER_TIMEOUT_S = 300


def other_configs():
    """Runs each workload of OTHER_CONFIGS as `bench.py --workload W` (no CPU
    baseline) and keeps the parts of its line that describe it: value,
    step time, end-to-end rate, clocks and its full-size parity fields."""
    out = {}
    for name, steps, warmup in OTHER_CONFIGS:
        cmd = [sys.executable, os.path.abspath(__file__), "--workload", name, "--steps", str(steps),
               "--warmup", str(warmup), "--no-cpu-baseline"]
        t0 = time.perf_counter()
        try:
            r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True,
                               timeout=OTHER_TIMEOUT_S, cwd=ROOT)
        except subprocess.TimeoutExpired:
            out[name] = {"rc": None, "error": f"timed out after {OTHER_TIMEOUT_S} s"}
            continue
        rec = {"rc": r.returncode, "wall_s": round(time.perf_counter() - t0, 1)}
        line = None
        for ln in r.stdout.splitlines():
            if ln.startswith('{"metric"'):
                line = json.loads(ln)
        if line is None:
            tail = r.stderr.strip().splitlines()[-1:] or [""]
            rec["error"] = tail[0][-300:]
        else:
            e2e = line.get("e2e")
            cfg = line.get("config") or {}
            rec.update({
                "workload": cfg.get("workload"), "metric": line.get("metric"), "value": line.get("value"),
                "unit": line.get("unit"), "ms_per_step": line.get("ms_per_step"), "steps": line.get("steps"),
                "warmup": line.get("warmup"), "dtype": line.get("dtype"),
                "e2e": e2e.get("value") if isinstance(e2e, dict) else None,
                "parity": line.get("parity"),
                "clocks": line.get("clocks"),
            })
        out[name] = rec
    return out


_JSON_OUT = None


def _reserve_stdout():
    """Keep the process's stdout for the JSON line alone: the reference's
    native CPU code writes progress-bar control sequences to stdout, so fd 1
    is pointed at stderr and the JSON line goes to a saved copy of it."""
    global _JSON_OUT
    sys.stdout.flush()
    _JSON_OUT = os.fdopen(os.dup(1), "w")
    os.dup2(2, 1)


def emit(obj):
    """Print one JSON line on the real stdout."""
    out = _JSON_OUT if _JSON_OUT is not None else sys.stdout
    out.write(json.dumps(obj) + "\n")
    out.flush()


def main():
    # bench_workloads imports this file as `bench`; share this instance (and
    # its saved stdout) instead of loading a second copy.
    sys.modules.setdefault("bench", sys.modules[__name__])
    _reserve_stdout()
    args = parse()
    if args.reference_gpu_child is not None:
        return _reference_gpu_child(args)
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.workload != "taylor_accel":
        import bench_workloads

        return bench_workloads.run(args, rank, world, local_rank)
    if args.impl == "reference":
        return run_reference(args, rank)
    return run_ours(args, rank, world, local_rank)


if __name__ == "__main__":
    sys.exit(main())
