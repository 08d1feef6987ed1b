"""Benchmark: body-steps/s of the Barnes-Hut step on B200.

Default workload: two colliding exponential discs, N = 4,194,304, theta = 0.5,
FP64 state, softening 0.01, dt = 1e-4 (seeded synthetic input; no dataset).
One "step" is the whole reference step: bounding box, Morton sort, tree,
moments, force + kick, drift.  `value` is device-timed (CUDA events on the
library's stream around K graph-launched steps) with the bodies resident in
HBM; `e2e` times the same steps through the C ABI with host buffers: every
step uploads the bodies from pinned host memory and downloads positions and
velocities back, which is the reference's own per-step contract
(BarnesHutCuda.cu:632-646) plus an upload.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--mode fp64|split] [--n N]

--impl reference times the reference's CPU Barnes-Hut (compiled from the
reference sources into oracle/_ref when available, else the CPU oracle's
restatement of the GPU step) on the host cores, on a bounded sample.
Under torchrun each rank runs an independent replica ("replicas only": the
step does not shard); rank 0 prints one JSON line.
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import os
import pathlib
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parent
PKG = ROOT / "n-body-2d_b200"

FLOPS_PER_INTERACTION = 14  # dx,dy,d2,+eps,r^-3 (3 mul),m*,2 fma: FP64/FP32 flops, rsqrt as 1
FALLBACK_PEAKS = {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}
# Algorithmic HBM bytes per body for each memory-bound phase (FP64 state,
# u64 codes, u32 payload): bbox 16 + Morton 16 in / 12 out; the sort's
# histogram read (8) and P radix passes of 12 in + 12 out (P = 8 here;
# sort_bytes() gives the bytes of a sort that took fewer passes); gather 44 in
# + 44 out; tree build about 8 x 3 reads + 32 writes per cell at 1.72 cells per
# body (96); moments 24 per body + 24 per cell (65); drift 32 in + 16 out (FP64
# mode only: SPLIT fuses it into the force kernel, and the learned step's last
# phase is the correction kernel).
PHASE_BYTES_PER_BODY = {"bbox+morton": 16 + 28, "sort": 8 + 8 * 24, "gather": 88, "tree": 96,
                        "moments": 65, "drift": 48}


def phase_bytes(passes: int, mono_prefix: bool) -> dict:
    """Algorithmic bytes per body of each HBM phase.  SPLIT monopoles take the
    prefix sums in their own phase before the tree (24 bytes read and 32
    written per body) and the cell records in the linking pass (about 24
    bytes per body: 40 per cell at 0.6 cells per body), so the moments phase
    is empty."""
    out = dict(PHASE_BYTES_PER_BODY, sort=sort_bytes(passes))
    if mono_prefix:
        out.pop("moments")
        out["prefix"] = 56
        out["tree"] += 24
    return out


def sort_bytes(passes: int) -> int:
    """Bytes per body of a sort over the top `passes` key bytes: histogram read,
    the passes, and the tie pass's read of the sorted keys when passes < 8."""
    return 8 + 24 * passes + (8 if passes < 8 else 0)


def _package():
    if "nbody_b200" in sys.modules:
        return sys.modules["nbody_b200"]
    spec = importlib.util.spec_from_file_location(
        "nbody_b200", PKG / "__init__.py", submodule_search_locations=[str(PKG)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["nbody_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


# DRAM bytes one launch of the SPLIT monopole force kernel moves per body:
# ncu dram__bytes_read.sum + dram__bytes_write.sum of one force_split launch
# on the 1,048,576-body collision (77.5 MB + 6.6 MB = 84.1 MB, --clock-control
# none).  Bodies and cells both grow linearly with N, so the figure scales by
# N; it is a property of the kernel's access pattern, re-measured when the
# kernel changes.
FORCE_TRAFFIC_BYTES_PER_BODY = 84.1e6 / 1048576


def _peaks() -> tuple[dict, str]:
    f = ROOT / "MEASURED_PEAKS.json"
    if f.exists():
        return json.loads(f.read_text()), "measured"
    return dict(FALLBACK_PEAKS), "fallback"


class ClockSampler:
    """SM clock and clock-event reasons of the benchmarked GPU, sampled from
    before the timed region to after it; samples are kept when their timestamp
    falls inside the region widened by one interval.  NVML (read-only queries,
    the device found by its UUID) is polled every 2 ms from a thread, so even a
    region of a few tens of ms gets a dozen samples; nvidia-smi at 20 ms is the
    fallback when NVML cannot be loaded."""

    FIELDS = ("timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    REASON_BITS = (("hw_slowdown", 0x8), ("hw_thermal_slowdown", 0x40),
                   ("sw_thermal_slowdown", 0x20), ("sw_power_cap", 0x4))
    NVML_INTERVAL_MS = 2
    SMI_INTERVAL_MS = 20

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.nvml = None
        self.thread = None
        self.stop = None
        self.t0 = self.t1 = None
        self.samples: list[tuple] = []   # (time, sm MHz, max sm MHz, reason names)
        self.interval_ms = self.SMI_INTERVAL_MS

    def _nvml_handle(self):
        import pynvml
        import torch

        pynvml.nvmlInit()
        try:
            uuid = str(torch.cuda.get_device_properties(self.device).uuid)
            return pynvml, pynvml.nvmlDeviceGetHandleByUUID(
                uuid if uuid.startswith("GPU-") else "GPU-" + uuid)
        except Exception:
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.device)

    def _poll(self, pynvml, h):
        reasons_of = getattr(pynvml, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
            pynvml.nvmlDeviceGetCurrentClocksThrottleReasons
        smax = pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM)
        while not self.stop.is_set():
            try:
                clk = pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM)
                bits = reasons_of(h)
            except Exception:
                break
            self.samples.append((time.time(), float(clk), float(smax),
                                 [name for name, bit in self.REASON_BITS if bits & bit]))
            self.stop.wait(self.NVML_INTERVAL_MS / 1000.0)

    def __enter__(self):
        import threading

        try:
            pynvml, h = self._nvml_handle()
            self.nvml = pynvml
            self.interval_ms = self.NVML_INTERVAL_MS
            self.stop = threading.Event()
            self.thread = threading.Thread(target=self._poll, args=(pynvml, h), daemon=True)
            self.thread.start()
            time.sleep(0.05)
            return self
        except Exception:
            self.nvml = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", str(self.SMI_INTERVAL_MS), "-i", str(self.device)],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            time.sleep(0.5)  # let the sampler start before the region opens
        except OSError:
            self.proc = None
        return self

    def mark_start(self):
        self.t0 = time.time()

    def mark_end(self):
        self.t1 = time.time()
        time.sleep(2.5 * self.interval_ms / 1000.0)

    def __exit__(self, *exc):
        if self.thread is not None:
            self.stop.set()
            self.thread.join(timeout=5)
            try:
                self.nvml.nvmlShutdown()
            except Exception:
                pass
        if self.proc is not None:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.samples = self._parse_smi([ln for ln in out.splitlines() if ln.strip()])

    @staticmethod
    def _parse_smi(lines):
        import datetime

        def stamp(text):
            for fmt in ("%Y/%m/%d %H:%M:%S.%f", "%Y/%m/%d %H:%M:%S", "%Y-%m-%d %H:%M:%S.%f"):
                try:
                    return datetime.datetime.strptime(text, fmt).timestamp()
                except ValueError:
                    pass
            return None

        names = [name for name, _ in ClockSampler.REASON_BITS]
        out = []
        for ln in lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 10:
                continue
            try:
                clk, clk_max = float(parts[2]), float(parts[3])
            except ValueError:
                continue
            out.append((stamp(parts[0]), clk, clk_max,
                        [n for n, val in zip(names, parts[6:10]) if val.lower() == "active"]))
        return out

    def summary(self) -> dict:
        pad = self.interval_ms / 1000.0
        windowed = self.t0 is not None and any(ts is not None for ts, *_ in self.samples)
        sm, smax, reasons = [], [], set()
        for ts, clk, clk_max, names in self.samples:
            if windowed and (ts is None or not (self.t0 - pad <= ts <= self.t1 + pad)):
                continue
            sm.append(clk)
            smax.append(clk_max)
            reasons.update(names)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0,
                    "source": "nvml" if self.nvml else "nvidia-smi"}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax),
                "reasons": sorted(reasons), "samples": len(sm),
                "interval_ms": self.interval_ms, "windowed": windowed,
                "source": "nvml" if self.nvml else "nvidia-smi"}


def _dist():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


# the pipelined loop's first upload and last download overlap nothing; enough
# steps keep that fill and drain a small share of the e2e time
E2E_MIN_STEPS = 40
E2E_HOW = ("per step: nb_upload_async of mass/pos/vel from pinned memory (upload stream), nb_step, "
           "nb_download_async of pos/vel (copy stream); the copies overlap the neighbouring steps; "
           "wall clock over at least 40 steps, one untimed round first")


def e2e_loop(ctx, hm, hp, hv, op, ov, steps: int) -> None:
    """steps x (upload, step, download) through the C ABI with pinned host
    buffers.  Step k's upload runs on the upload stream while step k-1
    computes, and its download on the copy stream while step k+1 computes;
    the results alternate between two host buffers."""
    for k in range(steps):
        ctx.upload_async(hm, hp, hv)
        ctx.step(1, sync=False)
        ctx.download_async(op[k & 1], ov[k & 1])
    ctx.download_wait()
    ctx.sync()


def max_over_ranks(value: float) -> float:
    """Largest value over the ranks of the default process group (the job's
    time is its slowest replica's); the value itself without one."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return value
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([value], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def _workload(kind: str, n: int, seed: int = 0):
    nb = _package()
    return nb.universes.make(kind, n, seed)


def cpu_baseline(n: int, theta: float, mass, pos, vel) -> dict:
    """Bounded CPU sample: one full step of the whole workload on all host
    cores, with the reference's CPU Barnes-Hut when it was built from the
    reference sources, else with the CPU oracle's restatement of the GPU step."""
    ref = ROOT / "oracle" / "_ref"
    cores = os.cpu_count() or 1
    if str(ROOT) not in sys.path:
        sys.path.insert(0, str(ROOT))
    runner = ref / "ref_cpu_bh"
    if runner.exists():
        from oracle import refcpu  # drives the reference CPU backend binary

        t = refcpu.time_steps(mass, pos, vel, theta=theta, steps=1, threads=cores)
        # the reference CPU walk differs from the GPU one: diagonal opening test
        # and |a| = G M / (d^2 + eps^2) (BarnesHut.cpp:115, 131-134)
        return {"value": n / t, "unit": "body-steps/s", "cores": cores, "kind": "reference",
                "sample": f"1 step of the full N={n} workload, reference BarnesHut (CPU), "
                          f"{cores} threads"}
    import oracle

    st = oracle.RefState(mass, pos, vel)
    t0 = time.perf_counter()
    st.step(theta=theta, eps2=1e-4, dt=1e-4, G=1.0, nthreads=cores)
    t = time.perf_counter() - t0
    return {"value": n / t, "unit": "body-steps/s", "cores": cores, "kind": "port",
            "sample": f"1 step of the full N={n} workload, CPU restatement of the reference "
                      f"GPU step, {cores} OpenMP threads"}


def gpu_baseline(nb, device: int) -> dict:
    """The reference's own GPU step on the same B200 beside this library's, on
    the one workload the reference kernel runs safely (its 32-entry traversal
    stack, CU:400, overflows on the discs: the oracle's replay needs 43
    entries at 4M bodies).  Both are timed on the jittered 262,144-body grid:
    the reference by the harness driver's host clock, this library by CUDA
    events (FP64 parity walk and SPLIT)."""
    if str(ROOT) not in sys.path:
        sys.path.insert(0, str(ROOT))
    m, p, v = nb.universes.make("grid", 262144, 0)
    ref = _ref_gpu_record(_ref_gpu_timed(m, p, v, 0.5, 5), 262144)
    mk = lambda mode: nb.SimConfig(timestep=1e-4, theta=0.5, epsilon_squared=1e-4, G=1.0,
                                   mode=mode, device=device)
    fp64 = _timed_context(nb, mk(nb.NB_MODE_FP64), m, p, v, 3, 20, accuracy=False)
    split = _timed_context(nb, mk(nb.NB_MODE_SPLIT), m, p, v, 3, 20, accuracy=False)
    rec = {"case": GRID_CASE, "reference": ref,
           "ours_fp64": {k: fp64[k] for k in ("value", "ms_per_step", "phases_ms")},
           "ours_split": {k: split[k] for k in ("value", "ms_per_step", "phases_ms")}}
    if "value" in ref:
        rec["ratio_fp64_vs_reference"] = fp64["value"] / ref["value"]
        rec["ratio_split_vs_reference"] = split["value"] / ref["value"]
    # the reference's own step ends with a download of every body (CU:632-646):
    # both sides again with that copy in every step, on the host clock
    ref_dl = _ref_gpu_record(_ref_gpu_timed(m, p, v, 0.5, 5, download=True), 262144,
                             how="the reference's CUDA kernels (BarnesHutCuda.cu, unmodified) under "
                                 "the harness driver, each step ending with the scatter to original "
                                 "order and the copy of all positions and velocities to host memory "
                                 "(CU:498-506, 632-646); host clock over K steps")
    dl = {"reference": ref_dl,
          "ours_fp64": _stepped_with_download(nb, mk(nb.NB_MODE_FP64), m, p, v, 3, 20),
          "ours_split": _stepped_with_download(nb, mk(nb.NB_MODE_SPLIT), m, p, v, 3, 20)}
    if "value" in ref_dl:
        dl["ratio_fp64_vs_reference"] = dl["ours_fp64"]["value"] / ref_dl["value"]
        dl["ratio_split_vs_reference"] = dl["ours_split"]["value"] / ref_dl["value"]
    rec["with_download_every_step"] = dl
    return rec


def _stepped_with_download(nb, cfg, m, p, v, warmup: int, steps: int) -> dict:
    """Steps of one context each followed by nb_download of every body into
    host arrays (the reference's per-step copy), host clock over K steps."""
    hp, hv = np.empty((m.shape[0], 2)), np.empty((m.shape[0], 2))
    with nb.NbContext(cfg, m, p, v) as ctx:
        # the download is stream-ordered after the step and waits for its copies
        for _ in range(warmup):
            ctx.step(1, sync=False)
            ctx.download(hp, hv)
        t0 = time.perf_counter()
        for _ in range(steps):
            ctx.step(1, sync=False)
            ctx.download(hp, hv)
        dt = (time.perf_counter() - t0) / steps
    return {"value": m.shape[0] / dt, "unit": "body-steps/s", "ms_per_step": dt * 1e3,
            "how": "nb_step(1) then nb_download of all positions and velocities into host "
                   "arrays, each step; host clock"}


def run_reference(args) -> None:
    """The reference arm: the reference's own CPU Barnes-Hut on the host cores,
    W untimed then K timed steps of the full workload in one process."""
    world, rank, _ = _dist()
    if rank != 0:
        return
    if str(ROOT) not in sys.path:
        sys.path.insert(0, str(ROOT))
    cores = os.cpu_count() or 1
    from oracle import refcpu

    if args.kind == "ensemble":
        run_reference_ensemble(args, refcpu, cores, world)
        return
    m, p, v = _workload(args.kind, args.n)
    if refcpu.available():
        t = refcpu.time_steps(m, p, v, theta=args.theta, steps=args.steps, warmup=args.warmup,
                              threads=cores)
        kind = "reference"
        sample = (f"{args.steps} timed steps (after {args.warmup} untimed) of the full "
                  f"N={args.n} workload, reference BarnesHut CPU backend, {cores} threads")
    else:
        import oracle

        st = oracle.RefState(m, p, v)
        for _ in range(args.warmup):
            st.step(theta=args.theta, eps2=1e-4, dt=1e-4, G=1.0, nthreads=cores)
        t0 = time.perf_counter()
        for _ in range(args.steps):
            st.step(theta=args.theta, eps2=1e-4, dt=1e-4, G=1.0, nthreads=cores)
        t = (time.perf_counter() - t0) / args.steps
        kind = "port"
        sample = (f"{args.steps} timed steps of the full N={args.n} workload, CPU restatement "
                  f"of the reference GPU step, {cores} OpenMP threads")
    value = args.n / t
    ref_gpu = reference_gpu_records(args, m, p, v)
    line = {
        "impl": "reference", "metric": "body-steps/s", "value": value, "unit": "body-steps/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": t * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": _config(args),
        "cpu_baseline": {"value": value, "unit": "body-steps/s", "cores": cores, "kind": kind,
                         "sample": sample},
        "e2e": {"value": value, "unit": "body-steps/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    if ref_gpu is not None:
        line["reference_gpu"] = ref_gpu
    print(json.dumps(line), flush=True)


REF_GPU_HOW = ("the reference's CUDA kernels (BarnesHutCuda.cu, unmodified) under the harness "
               "driver, host clock over K steps after one untimed step (the reference's step "
               "synchronises with the host at every tree level), without the per-step download "
               "of the bodies")
GRID_CASE = ("jittered grid, 512 x 512 = 262,144 bodies, seed 0, theta 0.5: the CPU oracle's "
             "replay finds at most 28 of the reference kernel's 32 traversal-stack entries in use")


def _ref_gpu_timed(m, p, v, theta: float, steps: int, download: bool = False) -> dict:
    """refgpu.time_steps, with any failure of the harness reported, not raised."""
    from oracle import refgpu

    try:
        return refgpu.time_steps(m, p, v, theta=theta, steps=steps, download=download)
    except Exception as e:  # the record says why; the arm's own line still prints
        return {"unavailable": f"reference GPU harness failed: {type(e).__name__}: {e}"[:300]}


def _ref_gpu_record(r: dict, n: int, how: str = REF_GPU_HOW) -> dict:
    if "seconds_per_step" not in r:
        return r
    return {"value": n / r["seconds_per_step"], "unit": "body-steps/s",
            "ms_per_step": r["seconds_per_step"] * 1e3, "max_stack": r["max_stack"],
            "how": how}


def reference_gpu_records(args, m, p, v) -> dict:
    """The reference's own GPU path, where its 32-entry stack (CU:400) holds:
    the benchmark workload when the oracle's replay certifies it (else the
    refusal, with the stack depth the replay found), and always the jittered
    262,144-body grid, which it certifies."""
    out = {}
    steps = max(1, min(args.steps, 5))
    if args.kind != "grid":
        out[args.workload] = _ref_gpu_record(_ref_gpu_timed(m, p, v, args.theta, steps), args.n)
    nb = _package()
    gm, gp, gv = nb.universes.make("grid", 262144, 0)
    rec = _ref_gpu_record(_ref_gpu_timed(gm, gp, gv, 0.5, steps), 262144)
    rec["case"] = GRID_CASE
    out["grid256k"] = rec
    return out


def run_reference_ensemble(args, refcpu, cores: int, world: int) -> None:
    """Reference arm of the ensemble: the reference CPU backend holds one
    universe per process, so it steps the universes one after another.  A
    bounded sample: the first universes of the ensemble up to about one
    million bodies, each for W untimed and K timed steps."""
    nb = _package()
    m, p, v, counts = nb.universes.ensemble_batch(args.universes, seed=0)
    off = np.concatenate([[0], np.cumsum(counts.astype(np.int64))])
    bodies, seconds, used = 0, 0.0, 0
    for u in range(len(counts)):
        sl = slice(off[u], off[u + 1])
        if refcpu.available():
            t = refcpu.time_steps(m[sl], p[sl], v[sl], theta=args.theta, steps=args.steps,
                                  warmup=args.warmup, threads=cores)
            kind = "reference"
        else:
            import oracle

            st = oracle.RefState(m[sl], p[sl], v[sl])
            for _ in range(args.warmup):
                st.step(theta=args.theta, eps2=1e-4, dt=1e-4, G=1.0, nthreads=cores)
            t0 = time.perf_counter()
            for _ in range(args.steps):
                st.step(theta=args.theta, eps2=1e-4, dt=1e-4, G=1.0, nthreads=cores)
            t = (time.perf_counter() - t0) / args.steps
            kind = "port"
        bodies += int(counts[u])
        seconds += t
        used += 1
        if bodies >= 1_000_000:
            break
    value = bodies / seconds
    sample = (f"universes 0..{used - 1} of the {len(counts)}-universe ensemble ({bodies} bodies), "
              f"each {args.steps} timed steps after {args.warmup} untimed, one after another, "
              f"{cores} threads")
    line = {
        "impl": "reference", "metric": "body-steps/s", "value": value, "unit": "body-steps/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": seconds * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": args.workload, "universes": int(len(counts)),
                   "n": int(m.shape[0]), "theta": args.theta},
        "cpu_baseline": {"value": value, "unit": "body-steps/s", "cores": cores, "kind": kind,
                         "sample": sample},
        "e2e": {"value": value, "unit": "body-steps/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def _config(args) -> dict:
    return {"workload": args.workload, "n": args.n, "theta": args.theta, "mode": args.mode,
            "quadrupole": bool(getattr(args, "quad", False)), "leaf_size": getattr(args, "leaf", 0),
            "learned": bool(getattr(args, "learned", False)), "bmax_ratio": getattr(args, "bmax", 0.0),
            "softening": 0.01, "dt": 1e-4, "G": 1.0, "state": "f64",
            "l2": "inputs larger than L2 (state + tree > 126 MB at this N)"}


def run_ours(args) -> None:
    world, rank, local = _dist()
    nb = _package()
    import torch

    torch.cuda.set_device(local)
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    m, p, v = _workload(args.kind, args.n, seed=rank)
    mode = {"split": nb.NB_MODE_SPLIT, "fp64": nb.NB_MODE_FP64,
            "allpairs": nb.NB_MODE_ALLPAIRS}[args.mode]
    weights = None
    if args.learned:
        weights, args.bmax = _learned_weights()
    cfg = nb.SimConfig(timestep=1e-4, theta=args.theta, epsilon_squared=1e-4, G=1.0, mode=mode,
                       device=local, quadrupole=args.quad, leaf_size=args.leaf,
                       learned=args.learned, bmax_ratio=args.bmax)
    ctx = nb.NbContext(cfg, m, p, v)
    if weights is not None:
        ctx.set_mlp_weights(weights)
    ctx.step(args.warmup)

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            import torch.distributed as dist

            dist.barrier()
            torch.cuda.synchronize()

    barrier()
    with ClockSampler(local) as clocks:
        clocks.mark_start()
        ctx.step(args.steps, sync=False)
        ctx.sync()
        clocks.mark_end()
    barrier()
    st = ctx.stats()
    ms = st.ms_last_step
    phases = ctx.phase_times()
    passes = ctx.debug_sort_passes() if args.mode != "allpairs" else 0
    ms = max_over_ranks(ms)
    value = world * args.n / (ms * 1e-3)

    # e2e through the C ABI: host buffers, copies inside the timed region
    pin = lambda shape: torch.empty(shape, dtype=torch.float64, pin_memory=True).numpy()
    hm, hp, hv = pin((args.n,)), pin((args.n, 2)), pin((args.n, 2))
    hm[:], hp[:], hv[:] = m, p, v
    # double-buffered results; uploads and downloads overlap the steps (e2e_loop)
    op, ov = [pin((args.n, 2)) for _ in range(2)], [pin((args.n, 2)) for _ in range(2)]
    e2e_steps = max(args.steps, E2E_MIN_STEPS)
    e2e_loop(ctx, hm, hp, hv, op, ov, 1)  # untimed: sets up the upload staging area
    barrier()
    t0 = time.perf_counter()
    e2e_loop(ctx, hm, hp, hv, op, ov, e2e_steps)
    e2e_t = max_over_ranks((time.perf_counter() - t0) / e2e_steps)

    accuracy = None
    if not args.no_accuracy:
        from nbody_b200 import accuracy as acc_mod

        acc_now = ctx.accelerations()
        pos_now, _ = ctx.download()
        accuracy = acc_mod.force_errors(acc_now, m, pos_now, 1e-4, k=args.error_sample,
                                        device=local)
        accuracy["oracle"] = "FP64 all-pairs (GPU kernel), same Plummer law"

    peaks, peak_kind = _peaks()
    clk = clocks.summary()
    sm_mhz = clk["sm_mhz"] or peaks.get("sm_max_mhz", 1965.0)
    interactions = st.cell_interactions + st.body_interactions
    force_ms = phases.get("force", ms)
    # FP64: 64 FMA lanes per SM per clock on B200 (37 TF at 1.965 GHz); FP32: 128.
    lanes = 128 if args.mode == "split" else 64
    fp_peak = 148 * lanes * 2 * sm_mhz * 1e6 / 1e12
    achieved = FLOPS_PER_INTERACTION * interactions / (force_ms * 1e-3) / 1e12
    hbm = peaks.get("hbm_gbs", FALLBACK_PEAKS["hbm_gbs"])
    rooflines = {}
    mono = args.mode == "split" and not args.quad
    for name, bpb in phase_bytes(passes or 8, mono).items():
        if name == "drift" and args.mode != "fp64":
            continue
        if args.mode == "allpairs" and name != "force":
            continue  # the all-pairs step has no sort, tree or drift phase
        if phases.get(name, 0) > 0:
            gbs = bpb * args.n / (phases[name] * 1e-3) / 1e9
            rooflines[name] = {"bound": "hbm", "achieved": round(gbs, 1), "peak": hbm,
                               "unit": "GB/s", "frac": round(gbs / hbm, 4),
                               "ms": round(phases[name], 4)}
    line = {
        "metric": "body-steps/s", "value": value, "unit": "body-steps/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32+f64" if args.mode == "split" else "f64", "data": "synthetic",
        "config": _config(args),
        "roofline": {"kernel": "force", "bound": "fp32" if args.mode == "split" else "fp64",
                     "achieved": round(achieved, 3), "peak": round(fp_peak, 2),
                     "unit": "TFLOP/s", "frac": round(achieved / fp_peak, 4),
                     "traffic": (FORCE_TRAFFIC_BYTES_PER_BODY * args.n
                                 if args.mode == "split" and not args.quad and not args.learned
                                 else None),
                     "traffic_source": "ncu dram__bytes_read+write of one force_split launch at "
                                       "1M bodies (FORCE_TRAFFIC_BYTES_PER_BODY), scaled by n",
                     "peak_source": f"nominal {lanes} FMA/clk/SM x 148 SMs at the sampled "
                                    f"median SM clock {sm_mhz} MHz",
                     "interactions_per_s": interactions / (force_ms * 1e-3),
                     "interactions_per_body": interactions / args.n,
                     "flops_per_interaction": FLOPS_PER_INTERACTION,
                     # one 1/sqrt per interaction on the SFU: 16 per clock per SM
                     "sfu_frac": round(interactions / (force_ms * 1e-3)
                                       / (148 * 16 * sm_mhz * 1e6), 4),
                     "sfu_peak_source": f"nominal 16 MUFU ops/clk/SM x 148 SMs at {sm_mhz} MHz"},
        "rooflines_hbm": rooflines, "hbm_peak_source": f"{peak_kind} MEASURED_PEAKS.json hbm_gbs"
        if peak_kind == "measured" else "fallback 6.65 TB/s",
        "phases_ms": {k: round(v, 4) for k, v in phases.items()},
        "sort_passes": passes,
        "e2e": {"value": world * args.n / e2e_t, "unit": "body-steps/s",
                "h2d_bytes_per_step": 40 * args.n, "d2h_bytes_per_step": 32 * args.n,
                "steps": e2e_steps,
                "how": E2E_HOW},
        "gpu_launches": int(st.kernels_per_step) * args.steps,
        "clocks": clk,
        "accuracy": accuracy,
    }
    ctx.close()
    if rank == 0 and args.variants:
        line["variants"] = run_variants(args, nb, m, p, v, local, value, accuracy)
    elif (rank == 0 and accuracy and not args.no_learned_comparison and args.workload == "collision4m"
          and args.mode == "split" and not args.learned and not args.quad and not args.bmax):
        # the headline comparison: the learned theta = 1.0 step against this plain step
        lv = run_variants(args, nb, m, p, v, local, value, accuracy,
                          only=("learned_theta1.0",)).get("learned_theta1.0")
        if lv:
            line["learned_vs_plain"] = {
                "learned_value": lv["value"], "learned_ms_per_step": lv["ms_per_step"],
                "ratio": lv["speedup_vs_plain"], "learned_p50": lv["p50"], "learned_p99": lv["p99"],
                "plain_p99": accuracy["p99"], "fallback_rule": lv["fallback_rule"],
                "target_ratio": 2.0}
    # the extra records run on one GPU only: under torchrun the other ranks
    # would wait at the closing barrier longer than the process group allows
    if (world == 1 and not args.no_learned_comparison and args.workload == "collision4m"
            and args.mode == "split" and not args.learned and not args.quad and not args.bmax):
        line["at_accuracy_bar"] = at_accuracy_bar(args, nb, m, p, v, local)
    if rank == 0 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(args.n, args.theta, m, p, v)
        if world == 1:
            line["gpu_baseline"] = gpu_baseline(nb, local)
    if world == 1 and args.workload == "collision4m" and not args.no_sub_configs:
        line["configs"] = sub_configs(args, nb, local)
    if world > 1:
        import torch.distributed as dist

        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


def _hbm_rooflines(phases: dict, n: int, fp64: bool, passes: int = 8,
                   mono_prefix: bool = False) -> dict:
    peaks, kind = _peaks()
    hbm = peaks.get("hbm_gbs", FALLBACK_PEAKS["hbm_gbs"])
    out = {}
    for name, bpb in phase_bytes(passes, mono_prefix).items():
        if name == "drift" and not fp64:
            continue
        if phases.get(name, 0) > 0:
            gbs = bpb * n / (phases[name] * 1e-3) / 1e9
            out[name] = {"achieved_gbs": round(gbs, 1), "frac": round(gbs / hbm, 4),
                         "ms": round(phases[name], 4)}
    out["peak_gbs"] = hbm
    out["peak_source"] = f"{kind} hbm_gbs"
    return out


def _timed_context(nb, cfg, m, p, v, warmup: int, steps: int, counts=None, error_sample=65536,
                   accuracy=True, autotune=False, weights=None) -> dict:
    """W + K graph-launched steps of one context, device-timed, with the phase
    times and (optionally) the p50/p99 force error of the state after them."""
    from nbody_b200 import accuracy as acc_mod

    with nb.NbContext(cfg, m, p, v, counts=counts) as ctx:
        if weights is not None:
            ctx.set_mlp_weights(weights)
        tuned = ctx.autotune(2) if autotune else None
        ctx.step(warmup)
        ctx.step(steps, sync=False)
        ctx.sync()
        st = ctx.stats()
        phases = ctx.phase_times()
        passes = ctx.debug_sort_passes()
        rec = {"ms_per_step": st.ms_last_step, "sort_passes": passes, "value": m.shape[0] / (st.ms_last_step * 1e-3),
               "unit": "body-steps/s", "steps": steps, "warmup": warmup,
               "phases_ms": {k: round(x, 4) for k, x in phases.items()},
               "interactions_per_body": (st.cell_interactions + st.body_interactions)
               / m.shape[0]}
        if tuned:
            rec["autotuned"] = {"leaf_size": tuned[0], "bodies_per_lane": tuned[1]}
        if accuracy:
            acc_now = ctx.accelerations()
            pos_now, _ = ctx.download()
            if counts is None:
                err = acc_mod.force_errors(acc_now, m, pos_now, cfg.epsilon_squared,
                                           k=error_sample, device=cfg.device)
            else:
                err = acc_mod.ensemble_force_errors(acc_now, m, pos_now, counts,
                                                    cfg.epsilon_squared, k=error_sample,
                                                    device=cfg.device)
            rec["p50"], rec["p99"] = err["p50"], err["p99"]
    rec["rooflines_hbm"] = _hbm_rooflines(phases, m.shape[0], cfg.mode == nb.NB_MODE_FP64, passes,
                                          cfg.mode == nb.NB_MODE_SPLIT and not cfg.quadrupole)
    return rec


def sub_configs(args, nb, device: int) -> dict:
    """The other benchmark configurations, each bounded to a few seconds, so
    the default run carries them: the 16,384-body disc (SPLIT and the FP64
    parity walk), the 16,777,216-body Plummer disc (SPLIT next to all-FP64),
    and the 512-universe ensemble (one batched context against one context
    per universe launched in turn).  Errors against FP64 all-pairs on 65,536
    targets (per universe for the ensemble)."""
    out = {}
    mk = lambda mode, **kw: nb.SimConfig(timestep=1e-4, theta=0.5, epsilon_squared=1e-4, G=1.0,
                                         mode=mode, device=device, **kw)
    m, p, v = nb.universes.make("disc", 16384, 0)
    out["disc16k"] = {
        "split": _timed_context(nb, mk(nb.NB_MODE_SPLIT), m, p, v, 3, 200),
        "fp64": _timed_context(nb, mk(nb.NB_MODE_FP64), m, p, v, 3, 200),
        "config": "one exponential disc, N=16,384, seed 0, theta=0.5"}
    m, p, v = nb.universes.make("plummer", 16777216, 0)
    out["plummer16m"] = {
        "split": _timed_context(nb, mk(nb.NB_MODE_SPLIT), m, p, v, 3, 5),
        "fp64": _timed_context(nb, mk(nb.NB_MODE_FP64), m, p, v, 3, 3),
        "config": "projected Plummer disc, N=16,777,216, seed 0, theta=0.5; SPLIT (FP32 "
                  "traversal, FP64 box/COM/integrator) next to the all-FP64 walk"}
    del m, p, v
    m, p, v, counts = nb.universes.ensemble_batch(512, seed=0)
    batched = _timed_context(nb, mk(nb.NB_MODE_SPLIT), m, p, v, 3, 5, counts=counts,
                             autotune=True)
    off = np.concatenate([[0], np.cumsum(counts.astype(np.int64))])
    tuned = batched.get("autotuned", {}).get("leaf_size", 0)
    import torch

    ctxs = [nb.NbContext(mk(nb.NB_MODE_SPLIT, leaf_size=tuned), m[off[u]:off[u + 1]],
                         p[off[u]:off[u + 1]], v[off[u]:off[u + 1]]) for u in range(len(counts))]
    try:
        for c in ctxs:
            c.step(2)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        lsteps = 3
        for _ in range(lsteps):
            for c in ctxs:
                c.step(1, sync=False)
        for c in ctxs:
            c.sync()
        lt = (time.perf_counter() - t0) / lsteps
    finally:
        for c in ctxs:
            c.close()
    n = int(m.shape[0])
    out["ensemble512"] = {
        "batched": batched,
        "looped": {"value": n / lt, "unit": "body-steps/s", "ms_per_step_wall": lt * 1e3,
                   "steps": lsteps,
                   "how": "one context per universe, each step launched universe after "
                          "universe; wall clock from the first launch to the last sync"},
        "speedup_batched_vs_looped": batched["value"] / (n / lt),
        "config": f"512 exponential discs, {n} bodies, sizes {int(counts.min())}.."
                  f"{int(counts.max())}, theta=0.5"}
    return out


def run_ensemble(args) -> None:
    """Batched ensemble: 512 exponential discs of 1,024..262,144 bodies
    (log-uniform), advanced together by one batched context (one graph per
    step, one persistent traversal launch) after the autotuner picked the leaf
    and group sizes.  The same universes are then stepped as one context each,
    launched one after another every step, for the comparison."""
    world, rank, local = _dist()
    nb = _package()
    import torch

    torch.cuda.set_device(local)
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    m, p, v, counts = nb.universes.ensemble_batch(args.universes, seed=rank)
    n = int(m.shape[0])
    args.n = n
    cfg = nb.SimConfig(timestep=1e-4, theta=args.theta, epsilon_squared=1e-4, G=1.0,
                       mode=nb.NB_MODE_SPLIT, device=local, quadrupole=args.quad,
                       leaf_size=args.leaf)
    ctx = nb.NbContext(cfg, m, p, v, counts=counts)
    leaf, bpl = ctx.autotune(2) if not args.leaf else (args.leaf, 2)
    ctx.step(args.warmup)

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            import torch.distributed as dist

            dist.barrier()
            torch.cuda.synchronize()

    barrier()
    with ClockSampler(local) as clocks:
        clocks.mark_start()
        t0 = time.perf_counter()
        ctx.step(args.steps, sync=False)
        ctx.sync()
        wall = (time.perf_counter() - t0) / args.steps
        clocks.mark_end()
    barrier()
    st = ctx.stats()
    ms = max_over_ranks(st.ms_last_step)
    phases = ctx.phase_times()
    value = world * n / (ms * 1e-3)

    pin = lambda shape: torch.empty(shape, dtype=torch.float64, pin_memory=True).numpy()
    hm, hp, hv = pin((n,)), pin((n, 2)), pin((n, 2))
    hm[:], hp[:], hv[:] = m, p, v
    op, ov = [pin((n, 2)) for _ in range(2)], [pin((n, 2)) for _ in range(2)]
    e2e_steps = max(args.steps, E2E_MIN_STEPS)
    e2e_loop(ctx, hm, hp, hv, op, ov, 1)  # untimed: sets up the upload staging area
    barrier()
    t0 = time.perf_counter()
    e2e_loop(ctx, hm, hp, hv, op, ov, e2e_steps)
    e2e_t = max_over_ranks((time.perf_counter() - t0) / e2e_steps)

    accuracy = None
    if not args.no_accuracy:
        from nbody_b200 import accuracy as acc_mod

        acc_now = ctx.accelerations()
        pos_now, _ = ctx.download()
        accuracy = acc_mod.ensemble_force_errors(acc_now, m, pos_now, counts, 1e-4,
                                                 k=args.error_sample, device=local)
        accuracy["oracle"] = "FP64 all-pairs within each universe (GPU kernel)"
    ctx.close()

    # one context per universe, each step launched universe after universe
    looped = None
    if rank == 0:
        off = np.concatenate([[0], np.cumsum(counts.astype(np.int64))])
        cfg1 = nb.SimConfig(timestep=1e-4, theta=args.theta, epsilon_squared=1e-4, G=1.0,
                            mode=nb.NB_MODE_SPLIT, device=local, quadrupole=args.quad,
                            leaf_size=leaf)
        ctxs = [nb.NbContext(cfg1, m[off[u]:off[u + 1]], p[off[u]:off[u + 1]],
                             v[off[u]:off[u + 1]]) for u in range(len(counts))]
        for c in ctxs:
            c.step(args.warmup)
        torch.cuda.synchronize()
        lsteps = max(1, min(args.steps, 5))
        t0 = time.perf_counter()
        for _ in range(lsteps):
            for c in ctxs:
                c.step(1, sync=False)
        for c in ctxs:
            c.sync()
        lt = (time.perf_counter() - t0) / lsteps
        dev_ms = sum(c.stats().ms_last_step for c in ctxs)
        for c in ctxs:
            c.close()
        looped = {"value": n / lt, "unit": "body-steps/s", "ms_per_step_wall": lt * 1e3,
                  "sum_of_device_ms": dev_ms, "steps": lsteps,
                  "batched_wall_ms_per_step": wall * 1e3,
                  "speedup_batched_vs_looped": (n / wall) / (n / lt),
                  "how": f"{len(counts)} contexts (one graph each, own streams), every step "
                         "launches them one after another; wall clock from the first launch "
                         "to the last sync"}

    peaks, peak_kind = _peaks()
    clk = clocks.summary()
    sm_mhz = clk["sm_mhz"] or peaks.get("sm_max_mhz", 1965.0)
    interactions = st.cell_interactions + st.body_interactions
    force_ms = phases.get("force", ms)
    fp_peak = 148 * 128 * 2 * sm_mhz * 1e6 / 1e12
    achieved = FLOPS_PER_INTERACTION * interactions / (force_ms * 1e-3) / 1e12
    line = {
        "metric": "body-steps/s", "value": value, "unit": "body-steps/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32+f64", "data": "synthetic",
        "config": {"workload": args.workload, "universes": int(len(counts)), "n": n,
                   "n_min": int(counts.min()), "n_max": int(counts.max()), "theta": args.theta,
                   "mode": "split", "leaf_size": leaf, "bodies_per_lane": bpl,
                   "autotuned": not args.leaf, "softening": 0.01, "dt": 1e-4, "G": 1.0,
                   "l2": "inputs larger than L2"},
        "roofline": {"kernel": "force", "bound": "fp32", "achieved": round(achieved, 3),
                     "peak": round(fp_peak, 2), "unit": "TFLOP/s",
                     "frac": round(achieved / fp_peak, 4), "traffic": None,
                     "peak_source": f"nominal 128 FMA/clk/SM x 148 SMs at the sampled median "
                                    f"SM clock {sm_mhz} MHz",
                     "interactions_per_body": interactions / n,
                     "flops_per_interaction": FLOPS_PER_INTERACTION},
        "phases_ms": {k: round(v, 4) for k, v in phases.items()},
        "e2e": {"value": world * n / e2e_t, "unit": "body-steps/s",
                "h2d_bytes_per_step": 40 * n, "d2h_bytes_per_step": 32 * n, "steps": e2e_steps,
                "how": E2E_HOW},
        "gpu_launches": int(st.kernels_per_step) * args.steps,
        "clocks": clk, "accuracy": accuracy, "looped_single_universe": looped,
    }
    if world > 1:
        import torch.distributed as dist

        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


def _learned_weights():
    """The trained correction and the b_max ratio of the walk it was trained on."""
    weights = PKG / "weights" / "correction_theta1.npy"
    record = weights.with_suffix(".json")
    bmax = json.loads(record.read_text()).get("bmax_ratio", 0.0) if record.exists() else 0.0
    return np.load(weights), bmax


# The comparison at the accuracy bar (p99 relative force error <= 1e-3
# against FP64 all-pairs): neither walk of the literal comparison reaches it
# on the colliding discs (plain theta = 0.5 has p99 ~2e-2), so the bar is met
# by the analytic quadrupole walk at a smaller angle.  PLAIN_AT_BAR is the
# fastest plain walk measured to meet it on this workload; LEARNED_AT_BAR
# walks at a larger angle and lets the network (trained on the quadrupole
# walk's residuals, band = cells PLAIN_AT_BAR would open) supply the rest.
PLAIN_AT_BAR = dict(theta=0.4, quadrupole=True)
LEARNED_AT_BAR = dict(theta=0.5, quadrupole=True, learned=True, band_theta=0.4)
LEARNED_AT_BAR_WEIGHTS = "correction_quad_theta0.5"
ACCURACY_BAR = 1e-3


def at_accuracy_bar(args, nb, m, p, v, device) -> dict:
    """Plain and learned steps at the accuracy bar, timed like the main line
    (W + K graph-launched steps, CUDA events), each with its p50/p99 against
    FP64 all-pairs on 65,536 targets; the learned step falls back to the
    plain one when its p99 misses the bar."""
    out = {"bar_p99": ACCURACY_BAR}
    mk = lambda **kw: nb.SimConfig(timestep=1e-4, epsilon_squared=1e-4, G=1.0,
                                   mode=nb.NB_MODE_SPLIT, device=device, **kw)
    plain = _timed_context(nb, mk(**PLAIN_AT_BAR), m, p, v, args.warmup, args.steps,
                           error_sample=args.error_sample)
    out["plain"] = dict(config=PLAIN_AT_BAR, **plain)
    wfile = PKG / "weights" / f"{LEARNED_AT_BAR_WEIGHTS}.npy"
    if not wfile.exists():
        out["learned"] = {"unavailable": f"no trained weights {wfile.name}"}
        return out
    learned = _timed_context(nb, mk(**LEARNED_AT_BAR), m, p, v, args.warmup, args.steps,
                             error_sample=args.error_sample, weights=np.load(wfile))
    out["learned"] = dict(config=LEARNED_AT_BAR, weights=wfile.name, **learned)
    out["ratio"] = learned["value"] / plain["value"]
    out["plain_meets_bar"] = plain["p99"] <= ACCURACY_BAR
    out["learned_meets_bar"] = learned["p99"] <= ACCURACY_BAR
    out["fallback_rule"] = ("kept" if learned["p99"] <= ACCURACY_BAR
                            else "falls back to the plain step (learned p99 above the bar)")
    out["target_ratio"] = 2.0
    return out


def run_variants(args, nb, m, p, v, device, plain_value, plain_accuracy, only=None) -> dict:
    """The learned theta = 1.0 step next to the plain theta = 0.5 one (same
    workload, same timing method), plus the analytic-quadrupole and plain
    theta = 1.0 walks, each with its p50/p99 force error against FP64
    all-pairs.  The learned step falls back to plain theta = 0.5 when its p99
    is worse than the plain step's (the learned mode's fallback rule)."""
    from nbody_b200 import accuracy as acc_mod

    weights = PKG / "weights" / "correction_theta1.npy"
    record = weights.with_suffix(".json")
    out = {}
    specs = [("mono_theta1.0", dict(theta=1.0)),
             ("mono_theta1.0_bmax0.75", dict(theta=1.0, bmax_ratio=0.75)),
             ("quad_theta0.7", dict(theta=0.7, quadrupole=True)),
             ("quad_theta0.8_bmax0.75", dict(theta=0.8, quadrupole=True, bmax_ratio=0.75)),
             ("quad_theta1.0", dict(theta=1.0, quadrupole=True)),
             ("quad_theta1.0_bmax0.75", dict(theta=1.0, quadrupole=True, bmax_ratio=0.75))]
    if weights.exists():
        # the walk the network was trained on (the b_max ratio of its record)
        bmax = json.loads(record.read_text()).get("bmax_ratio", 0.0) if record.exists() else 0.0
        specs.insert(0, ("learned_theta1.0", dict(theta=1.0, learned=True, bmax_ratio=bmax)))
    if only is not None:
        specs = [(name, kw) for name, kw in specs if name in only]
    for name, kw in specs:
        cfg = nb.SimConfig(timestep=1e-4, epsilon_squared=1e-4, G=1.0, mode=nb.NB_MODE_SPLIT,
                           device=device, **kw)
        with nb.NbContext(cfg, m, p, v) as ctx:
            if kw.get("learned"):
                ctx.set_mlp_weights(np.load(weights))
            ctx.step(args.warmup)
            ctx.step(args.steps, sync=False)
            ctx.sync()
            ms = ctx.stats().ms_last_step
            phases = ctx.phase_times()
            acc_now = ctx.accelerations()
            pos_now, _ = ctx.download()
        err = acc_mod.force_errors(acc_now, m, pos_now, 1e-4, k=args.error_sample, device=device)
        val = args.n / (ms * 1e-3)
        out[name] = {"value": val, "ms_per_step": ms, "speedup_vs_plain": val / plain_value,
                     "p50": err["p50"], "p99": err["p99"],
                     "force_ms": round(phases.get("force", 0.0), 4),
                     "correction_ms": round(phases.get("drift", 0.0), 4)}
    if "learned_theta1.0" in out and plain_accuracy:
        lv = out["learned_theta1.0"]
        lv["fallback_rule"] = ("kept" if lv["p99"] <= plain_accuracy["p99"]
                               else "falls back to plain theta=0.5 (p99 above the plain step's)")
    return out


WORKLOADS = {
    "collision4m": ("collision", 4194304, 0.5),
    "disc16k": ("disc", 16384, 0.5),
    "plummer16m": ("plummer", 16777216, 0.5),
    "ensemble512": ("ensemble", 0, 0.5),
    "grid256k": ("grid", 262144, 0.5),
}


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--mode", choices=["fp64", "split", "allpairs"], default="split",
                    help="allpairs: the reference's AllPairsSim on the GPU (FP64, no tree)")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="collision4m")
    ap.add_argument("--n", type=int, default=None, help="override the body count")
    ap.add_argument("--theta", type=float, default=None)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--quad", action="store_true", help="SPLIT: add quadrupole terms")
    ap.add_argument("--leaf", type=int, default=0, help="SPLIT: direct-sum cell size (0=default)")
    ap.add_argument("--no-accuracy", action="store_true")
    ap.add_argument("--no-sub-configs", action="store_true",
                    help="skip the bounded 16K-disc / 16.7M-Plummer / 512-universe records "
                         "of the default run")
    ap.add_argument("--error-sample", type=int, default=65536)
    ap.add_argument("--no-learned-comparison", action="store_true",
                    help="skip the learned theta=1.0 step timed next to the default plain step")
    ap.add_argument("--variants", action="store_true",
                    help="also time the learned, quadrupole and plain theta=1.0 walks")
    ap.add_argument("--universes", type=int, default=512, help="ensemble512: universe count")
    ap.add_argument("--bmax", type=float, default=0.0,
                    help="SPLIT: b_max acceptance ratio (nb_params.bmax_ratio; 0 = off)")
    ap.add_argument("--learned", action="store_true",
                    help="SPLIT with the learned far-field correction (weights/correction_theta1; "
                         "its b_max ratio)")
    args = ap.parse_args(argv)
    kind, n, theta = WORKLOADS[args.workload]
    args.kind = kind
    args.n = args.n or n
    if args.learned and args.theta is None:
        theta = 1.0  # the learned correction's walk
    args.theta = theta if args.theta is None else args.theta
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    elif kind == "ensemble":
        run_ensemble(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
