#!/usr/bin/env python3
"""Throughput of the SU(2) pure-gauge hot path on B200 -- one JSON line on rank 0.

Headline (the reference's own update, in its precision): a 48^4 SU(2) lattice at beta = 3.09,
Haar-random (hot) start from Philox, FP64 links.  One step = one checkerboard heatbath sweep over
all 4V links followed by the plaquette (the reference's qcd.c:54-60 loop: gaugefieldUpdate, then
plaquette).  `value` is heatbath link updates per second over all GPUs (4V per step per GPU);
`e2e` is the same step through the C ABI with the field uploaded from pinned host memory each step.
`extras` holds the FP32 figures (1 heatbath + 4 overrelaxation sweeps, APE, W, Q), their ratio to
FP64, the error of FP32 against FP64 on a thermalised field, the batched replicas, the graph loop,
one configuration's measurement and the 96^4 lattice.

Multi-GPU: independent replicas (one lattice per GPU, different seed), no data-path collective;
the job aggregate is the sum of per-GPU work divided by the slowest rank's time.

--impl reference times the reference's own C code (compiled from source into oracle/_ref by
oracle/build_ref.sh) on the host cores: one independent process per core running the reference's
localHeatbathUpdate over a bounded slice of the same 48^4 lattice each step.
"""
import argparse
import json
import math
import os
import subprocess
import sys
import tempfile
import time

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

METRIC = "link updates/s & APE steps/s at 48^4, FP32 vs FP64 GPU, % HBM roofline"
UNIT = "link-updates/s"
BETA = 3.09
N_OR = 4
FALLBACK_HBM_GBS = 6650.0


# ------------------------------------------------------------------ helpers ---

R9 = [r for r in range(1, 10) for t in range(1, 10)]
T9 = [t for r in range(1, 10) for t in range(1, 10)]
APE_SEQ = 10   # smearing steps per timed call
# one call of each kernel family on a lattice L (the --kernel mode)
KERNELS = {
    "heatbath": lambda L: L.sweep(1, 1, 0),
    "overrelax": lambda L: L.sweep(1, 0, 1),
    "plaquette": lambda L: L.plaquette(),
    "ape_all": lambda L: L.ape(1, 0.5, "all"),
    "ape_spatial": lambda L: L.ape(1, 0.5, "spatial"),
    "wilson": lambda L: L.wilson(R9, T9),
    "qtop": lambda L: L.qtop(),
}

def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--dims", default="48,48,48,48")
    ap.add_argument("--no-extras", action="store_true", help="headline only")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--kernel", choices=sorted(KERNELS), default=None,
                    help="time one kernel family alone on the workload lattice (for profiling): "
                         "--steps calls after --warmup calls, one JSON line")
    ap.add_argument("--precision", default="fp32", choices=["fp32", "fp64"], help="precision for --kernel")
    return ap.parse_args()


class Dist:
    """Rank plumbing when launched by torchrun: torch.distributed over NCCL on GPUs (gloo where no GPU
    is visible, e.g. the CPU tests of the multi-rank path); nothing for a single process.  The ranks
    run independent replicas and exchange only timings."""

    def __init__(self):
        self.rank = int(os.environ.get("RANK", "0"))
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.torch = None
        if self.world > 1:
            import datetime
            import torch
            import torch.distributed as dist
            self.gpu = torch.cuda.is_available()
            if self.gpu:
                torch.cuda.set_device(self.local)
            dist.init_process_group("nccl" if self.gpu else "gloo", timeout=datetime.timedelta(seconds=300))
            self.torch = torch
            self.dist = dist

    def barrier(self):
        if self.torch:
            if self.gpu:
                self.dist.barrier(device_ids=[self.local])
            else:
                self.dist.barrier()

    def _reduce(self, x, op):
        if not self.torch:
            return x
        t = self.torch.tensor([float(x)], device="cuda" if self.gpu else "cpu", dtype=self.torch.float64)
        self.dist.all_reduce(t, op=op)
        return float(t.item())

    def max(self, x):
        return self._reduce(x, self.dist.ReduceOp.MAX) if self.torch else x

    def sum(self, x):
        return self._reduce(x, self.dist.ReduceOp.SUM) if self.torch else x

    def close(self):
        if self.torch:
            self.dist.destroy_process_group()


class NvmlClocks:
    """SM clock and clock-event reasons read through NVML every 5 ms from a thread, strictly between
    start() and stop() (the timed region is tens of milliseconds, shorter than nvidia-smi's sampling
    period).  Reads only; changes no setting."""

    def __init__(self, device):
        import pynvml
        self.nv = pynvml
        pynvml.nvmlInit()
        self.h = pynvml.nvmlDeviceGetHandleByIndex(device)
        self.smax = pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM)
        get = getattr(pynvml, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
            pynvml.nvmlDeviceGetCurrentClocksThrottleReasons
        self.reasons_of = lambda: get(self.h)
        self.bits = {"hw_slowdown": 0x8, "hw_thermal_slowdown": 0x40, "sw_thermal_slowdown": 0x20, "sw_power_cap": 0x4}
        self.rows, self.thread, self.stop_flag = [], None, None

    def _run(self):
        while not self.stop_flag.is_set():
            self.rows.append((self.nv.nvmlDeviceGetClockInfo(self.h, self.nv.NVML_CLOCK_SM), self.reasons_of()))
            self.stop_flag.wait(0.005)

    def start(self):
        import threading
        self.rows, self.stop_flag = [], threading.Event()
        self.thread = threading.Thread(target=self._run, daemon=True)
        self.thread.start()

    def stop(self):
        self.stop_flag.set()
        self.thread.join()
        if not self.rows:
            return None
        sm = sorted(r[0] for r in self.rows)
        reasons = sorted({k for _, m in self.rows for k, b in self.bits.items() if m & b})
        return {"sm_mhz": float(sm[len(sm) // 2]), "sm_max_mhz": float(self.smax), "reasons": reasons,
                "samples": len(self.rows), "source": "NVML every 5 ms inside the timed passes"}


def clock_sampler(device):
    try:
        return NvmlClocks(device)
    except Exception:   # no NVML binding or no device: nvidia-smi's 200 ms samples
        return Clocks(device)


class Clocks:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.f = None

    def start(self):
        try:
            self.f = tempfile.NamedTemporaryFile("w+", delete=False, suffix=".csv")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None

    def stop(self):
        if not self.proc:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.f.close()
        rows = []
        for line in open(self.f.name):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.f.name)
        if not rows:
            return None
        sm = sorted(float(r[1]) for r in rows if r[1].replace(".", "").isdigit())
        smax = max((float(r[2]) for r in rows if r[2].replace(".", "").isdigit()), default=None)
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        med = sm[len(sm) // 2] if sm else None
        return {"sm_mhz": med, "sm_max_mhz": smax, "reasons": reasons, "samples": len(rows)}


def measured_peak():
    p = os.path.join(REPO, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return FALLBACK_HBM_GBS, "fallback"


def dram_traffic(key):
    """Per-launch DRAM bytes of a kernel from the committed ncu summary (profiles/dram_traffic.json)."""
    try:
        with open(os.path.join(REPO, "profiles", "dram_traffic.json")) as f:
            v = json.load(f).get(key)
        return None if v is None else float(v["bytes_per_launch"])
    except (OSError, ValueError, KeyError, TypeError):
        return None


def cpu_info():
    model = "unknown"
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                model = line.split(":", 1)[1].strip()
                break
    except OSError:
        pass
    return model, os.cpu_count() or 1


def mem_available_gb():
    try:
        for line in open("/proc/meminfo"):
            if line.startswith("MemAvailable"):
                return int(line.split()[1]) / 1e6
    except OSError:
        pass
    return 16.0


# ---------------------------------------------------- reference CPU baseline ---

def ref_harness(dims):
    p = os.path.join(REPO, "oracle", "_ref", "x".join(map(str, dims)), "harness")
    return p if os.path.exists(p) else None


def cpu_reference_rate(dims, reps, warm, sites, procs=None):
    """Run `procs` independent reference processes, each heatbath-updating `sites` sites x 4 dirs
    per rep with the reference's localHeatbathUpdate; returns per-rep aggregate rates."""
    exe = ref_harness(dims)
    model, ncpu = cpu_info()
    vol = math.prod(dims)
    per_proc_gb = vol * 4 * 32 * 2.2 / 1e9 + vol * 64 / 1e9 + 0.2
    if procs is None:
        procs = max(1, min(ncpu, int(mem_available_gb() * 0.6 / per_proc_gb)))
    if exe:
        kind = "reference"
        cmds = [[exe, "bench_hb", "1", str(1 + i), str(BETA), str(sites), str(warm + reps)] for i in range(procs)]
    else:
        kind = "port"
        cmds = [[sys.executable, os.path.join(REPO, "oracle", "port_bench.py"), ",".join(map(str, dims)),
                 str(1 + i), str(BETA), str(sites), str(warm + reps)] for i in range(procs)]
    ps = [subprocess.Popen(c, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True) for c in cmds]
    per_rep = [0.0] * (warm + reps)
    for p in ps:
        out, _ = p.communicate()
        if p.returncode != 0:
            raise RuntimeError(f"CPU baseline process failed: {p.args}")
        for line in out.splitlines():
            f = line.split()
            if len(f) >= 5 and f[0] == "RESULT" and f[1] == "hb_s":
                r, n, t = int(f[2]), int(f[3]), float(f[4])
                per_rep[r] += n / t
    timed = per_rep[warm:]
    return {
        "rates": timed, "kind": kind, "cores": procs, "model": model, "nproc": ncpu,
        "sample": f"{procs} independent processes x {sites} sites x 4 dirs of localHeatbathUpdate per step "
                  f"on a hot {'x'.join(map(str, dims))} lattice (beta={BETA}), heatbath only "
                  f"(the reference has no overrelaxation)",
    }


def cpu_reference_kernels(gpu, dims, small=(24, 24, 24, 24)):
    """The reference's own APE_all and spatial APE steps and its Q, timed on the workload's lattice,
    and its W(R<=9, T<=9) set timed at `small` and scaled by the site count (at 48^4 the set takes
    ~160 s on one core); one process each on one core, run concurrently, timed by the reference's
    getTime.  Beside them, the GPU figures of the same run."""
    exe, exe_small = ref_harness(dims), ref_harness(small)
    if not exe or not exe_small:
        return None
    jobs = {"ape_all": (exe, ["bench_ape", "all", "0.5", "2"], dims),
            "ape_spatial": (exe, ["bench_ape", "spatial", "0.5", "2"], dims),
            "qtop": (exe, ["bench_qtop", "1"], dims),
            "wilson_R9T9": (exe_small, ["bench_wil", "9", "9", "1"], small)}
    # the harness writes the reference's log file into its working directory: a private temporary one
    tmp = tempfile.TemporaryDirectory(prefix="su2ref_")
    ps = {k: (subprocess.Popen([e] + a, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True, cwd=tmp.name), d)
          for k, (e, a, d) in jobs.items()}
    out = {"dims": list(dims), "note": f"single-core reference time per unit; W timed at {'x'.join(map(str, small))} "
                                       "and scaled by the site count, the others timed at dims; GPU rates from this run"}
    gpu_rate = {"ape_all": "ape_all_steps_per_s", "ape_spatial": "ape_spatial_steps_per_s",
                "wilson_R9T9": "wilson_R9T9_sweeps_per_s", "qtop": "qtop_per_s"}
    for k, (p, d) in ps.items():
        txt, _ = p.communicate()
        ts = [float(line.split()[3]) for line in txt.splitlines() if line.startswith("RESULT") and line.split()[1]
              .endswith("_s")]
        if p.returncode != 0 or not ts:
            continue
        t_ref = min(ts) * math.prod(dims) / math.prod(d)
        e = {"cpu_ref_s_per_unit": t_ref, "timed_at": list(d)}
        for prec in ("fp64", "fp32"):
            r = gpu.get(f"{prec}_{gpu_rate[k]}")
            if r:
                e[f"gpu_{prec}_s_per_unit"] = 1.0 / r
                e[f"speedup_{prec}_vs_1_core"] = t_ref * r
        out[k] = e
    tmp.cleanup()
    return out


def run_reference(args, dist, dims):
    # under torchrun rank 0 alone times the reference on the host's cores; the others do nothing
    dist.barrier()
    if dist.rank != 0:
        return
    K, W = args.steps, args.warmup
    sites = 200_000 if math.prod(dims) > 200_000 else math.prod(dims)
    t0 = time.time()
    res = cpu_reference_rate(dims, K, W, sites)
    wall = time.time() - t0
    val = sum(res["rates"]) / len(res["rates"])
    line = {
        "impl": "reference", "metric": METRIC, "value": val, "unit": UNIT, "n_gpus": args.gpus, "steps": K,
        "warmup": W, "ms_per_step": 1e3 * (4 * sites) / (val / res["cores"]), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (RANLUX hot start of the reference)",
        "config": {"workload": f"{'x'.join(map(str, dims))} SU(2) beta={BETA} hot start, heatbath link updates "
                               f"(reference CPU code, one process per core)", "dims": dims},
        "cpu_baseline": {"value": val, "unit": UNIT, "cores": res["cores"], "kind": res["kind"],
                         "sample": res["sample"], "cpu_model": res["model"], "nproc": res["nproc"]},
        "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "wall_s": wall,
    }
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ our arm ---

def time_steps(lat, K, fn):
    lat.synchronize()
    lat.timer_begin()
    for _ in range(K):
        fn()
    return lat.timer_end()


def batch_figures(dist, sweeps=1000, seq_sweeps=20):
    """Batched replicas: (a) 64 lattices 16 x 8^4, 16 x 10^4, 16 x 12^4, 16 x 16^4, beta ~ U[2.2, 3.2],
    distinct seeds, alternating hot/cold, `sweeps` sweeps of 1 HB + 4 OR with the plaquette of every
    replica every sweep, one CUDA-graph replay per sweep; (b) the same for 64 x 12^4 against 64 single
    handles swept one after another (no graph)."""
    import random
    from masterarbeit_b200.su2g import Batch, Lattice

    rng = random.Random(2024 + dist.rank)
    out = {}

    def specs(sizes):
        return [{"dims": (L, L, L, L), "beta": rng.uniform(2.2, 3.2), "seed": 7000 + 97 * dist.rank + i,
                 "replica": i, "start": "haar" if i % 2 else "cold"} for i, L in enumerate(sizes)]

    for name, sizes in (("mixed_64", [8] * 16 + [10] * 16 + [12] * 16 + [16] * 16), ("uniform_64x12", [12] * 64)):
        reps = specs(sizes)
        upd = (1 + N_OR) * 4 * sum(L ** 4 for L in sizes)
        B = Batch(reps, precision="fp32", device=dist.local)
        block = B.autotune(1, N_OR)
        mode, _ = B.config()
        B.run(10, 1, N_OR, 1)
        trace, ms = B.run(sweeps, 1, N_OR, 1)
        # each form at each of its CTA widths, 200 sweeps (the autotuner's choice is the timed run above)
        forms = {}
        for fm, fb in (("graph", 64), ("graph", 128), ("graph", 256), ("persistent", 128), ("persistent", 256)):
            B.configure(fm, fb)
            B.run(5, 1, N_OR, 1)
            _, fms = B.run(200, 1, N_OR, 1)
            forms[f"{fm}_{fb}"] = upd / (fms / 200 / 1e3)
        B.close()
        ms_sweep_batch = ms / sweeps
        Ls = [Lattice(r["dims"], precision="fp32", beta=r["beta"], seed=r["seed"], start=r["start"],
                      replica=r["replica"], device=dist.local) for r in reps]
        for L in Ls:
            L.sweep_plaquette(1, 1, N_OR)
        t0 = time.perf_counter()
        for _ in range(seq_sweeps):
            for L in Ls:
                L.sweep_plaquette(1, 1, N_OR)
        ms_sweep_seq = (time.perf_counter() - t0) * 1e3 / seq_sweeps
        for L in Ls:
            L.close()
        out[name] = {"replicas": len(sizes), "sites": sum(L ** 4 for L in sizes), "autotuned_block": block,
                     "autotuned_form": mode, "link_updates_per_s_by_form": forms,
                     "sweeps": sweeps, "batched_ms_per_sweep": ms_sweep_batch,
                     "batched_link_updates_per_s": upd / (ms_sweep_batch / 1e3),
                     "sequential_ms_per_sweep": ms_sweep_seq, "speedup_vs_sequential": ms_sweep_seq / ms_sweep_batch,
                     "plaquette_trace_finite": bool(trace is not None and all(map(math.isfinite, trace.ravel())))}
    return out


def graph_figures(dist, sweeps=200):
    """The small-lattice chain of the reference's own test run (8^4, beta 3.09, cold start, seed 1,
    `sweeps` x (1 HB + N_OR OR) with the plaquette after every sweep), issued call by call against
    one replayed CUDA graph per sweep (su2g_graph_run)."""
    from masterarbeit_b200.su2g import Lattice

    out = {}
    for prec in ("fp64", "fp32"):
        a = Lattice((8, 8, 8, 8), precision=prec, beta=3.09, seed=1, start="cold", device=dist.local)
        b = Lattice((8, 8, 8, 8), precision=prec, beta=3.09, seed=1, start="cold", device=dist.local)
        for _ in range(5):
            a.sweep_plaquette(1, 1, N_OR)
        b.graph_run(5, 1, 1, N_OR)
        t0 = time.perf_counter()
        for _ in range(sweeps):
            p_last = a.sweep_plaquette(1, 1, N_OR)
        plain = time.perf_counter() - t0
        t0 = time.perf_counter()
        trace, _ = b.graph_run(sweeps, 1, 1, N_OR)
        graph = time.perf_counter() - t0
        out[f"{prec}_8x8x8x8"] = {"sweeps": sweeps, "plain_sweeps_per_s": sweeps / plain,
                                  "graph_sweeps_per_s": sweeps / graph, "speedup": plain / graph,
                                  "identical_to_plain": bool(trace[-1] == p_last)}
        a.close()
        b.close()
    return out


def kernel_rate(L, K, fn, cls, units, bytes_per_unit, peak):
    """Plain-call rate of `fn` (K calls) and the CUDA-event duration of its `cls` launches (a second
    pass with every launch bracketed by events): (units per second, GB/s, fraction of peak)."""
    ms = time_steps(L, K, fn)
    L.profile(True)
    time_steps(L, K, fn)
    n, tms = L.profile_read()[cls]
    L.profile(False)
    gbs = units * bytes_per_unit / (tms / n / 1e3) / 1e9
    return K / (ms / 1e3), gbs, gbs / peak


def precision_figures(L, prec, dims, K, W, peak, clk, extras):
    """Throughput of every kernel of the path on lattice L of precision `prec`: the 1 HB + 4 OR step,
    the heatbath-only sweep, APE all / spatial, W(R<=9, T<=9) and Q."""
    vol = math.prod(dims)
    lb = 16 if prec == "fp32" else 32
    step = lambda: L.sweep_plaquette(1, 1, N_OR)
    for _ in range(W):
        step()
    ms = time_steps(L, K, step)
    extras[f"{prec}_1hb{N_OR}or_link_updates_per_s"] = (1 + N_OR) * 4 * vol * K / (ms / 1e3)
    L.profile(True)
    time_steps(L, K, step)
    prof = L.profile_read()
    L.profile(False)
    for cls, transfers in (("overrelax", 9), ("heatbath", 8)):
        n, tms = prof[cls]
        gbs = (vol // 2) * transfers * lb / (tms / n / 1e3) / 1e9
        extras[f"{prec}_{cls}_pass_gbs"] = gbs
        extras[f"{prec}_{cls}_pass_frac_of_peak"] = gbs / peak
    hb = lambda: L.sweep_plaquette(1, 1, 0)
    ms = time_steps(L, K, hb)
    extras[f"{prec}_heatbath_link_updates_per_s"] = 4 * vol * K / (ms / 1e3)
    # smearing runs in sequences (15 / 30 APE_all steps before Q, 100-400 spatial before W): each
    # figure is per step within sequences of APE_SEQ steps
    for mode, per_site in (("all", 8), ("spatial", 6)):
        L.ape(APE_SEQ, 0.5, mode)
        rate, gbs, frac = kernel_rate(L, K, lambda: L.ape(APE_SEQ, 0.5, mode), "ape", vol, per_site * lb, peak)
        extras[f"{prec}_ape_{mode}_steps_per_s"] = rate * APE_SEQ
        extras[f"{prec}_ape_{mode}_gbs"] = gbs
        extras[f"{prec}_ape_{mode}_frac_of_peak"] = frac
    R = [r for r in range(1, 10) for t in range(1, 10)]
    T = [t for r in range(1, 10) for t in range(1, 10)]
    # ALU-bound rows: algorithmic flops (line method: 765 quaternion products per site for R, T <= 9;
    # clover charge: 576 products per site; 28 flop a product) against the nominal FP32 / FP64 rate of
    # 148 SMs x 128 / 64 lanes x 2 flop at the SM clock sampled in the headline's timed region
    f_mhz = (clk or {}).get("sm_mhz") or 1965.0
    alu_peak = 148 * (128 if prec == "fp32" else 64) * 2 * f_mhz * 1e6
    extras[f"{prec}_alu_peak_tflops_nominal"] = alu_peak / 1e12
    L.wilson([1], [1])
    ms_w = time_steps(L, 3, lambda: L.wilson(R, T)) / 3
    extras[f"{prec}_wilson_R9T9_sweeps_per_s"] = 1e3 / ms_w
    extras[f"{prec}_wilson_R9T9_frac_of_alu_peak"] = vol * 765 * 28 / (ms_w / 1e3) / alu_peak
    L.qtop()
    ms_q = time_steps(L, 3, L.qtop) / 3
    extras[f"{prec}_qtop_per_s"] = 1e3 / ms_q
    extras[f"{prec}_qtop_frac_of_alu_peak"] = vol * 576 * 28 / (ms_q / 1e3) / alu_peak


def fp32_error_table(dims, device, seed):
    """Error of the FP32 path against FP64 on one thermalised field (200 sweeps of 1 HB + 4 OR in FP64
    from a Haar start, uploaded into both precisions): the plaquette, W(R <= 10, T <= 16) after 100 /
    200 / 400 spatial APE steps and Q after 15 / 30 APE_all steps (alpha 0.5)."""
    from masterarbeit_b200.su2g import Lattice
    L64 = Lattice(dims, precision="fp64", beta=BETA, seed=seed, start="haar", device=device)
    L64.sweep(200, 1, N_OR)
    U = L64.download()
    L32 = Lattice(dims, precision="fp32", beta=BETA, device=device)
    L32.upload(U)
    p32, p64 = L32.plaquette(), L64.plaquette()
    out = {"field": f"{'x'.join(map(str, dims))} FP64 field after 200 sweeps of 1 HB + {N_OR} OR (Haar start), "
                    "rounded to FP32 for the FP32 path", "plaquette_rel": abs(p32 - p64) / abs(p64)}
    R = [r for r in range(1, 11) for t in range(1, 17)]
    T = [t for r in range(1, 11) for t in range(1, 17)]
    for n in (100, 200, 400):
        w32 = L32.measure(R=R, T=T, ns_s=n, alpha_s=0.5)[1]
        w64 = L64.measure(R=R, T=T, ns_s=n, alpha_s=0.5)[1]
        d = abs(w32 - w64)
        big = abs(w64) >= 1e-2
        out[f"wilson_after_{n}_spatial_ape"] = {
            "max_rel_where_W_ge_1e-2": float((d[big] / abs(w64[big])).max()), "loops_W_ge_1e-2": int(big.sum()),
            "max_abs": float(d.max()), "max_rel_all": float((d / abs(w64)).max()),
            "W10_16_fp64": float(w64[-1]), "W10_16_rel": float(d[-1] / abs(w64[-1]))}
    q32 = L32.measure(q_ape=[15, 30], alpha_q=0.5)[0]
    q64 = L64.measure(q_ape=[15, 30], alpha_q=0.5)[0]
    for i, n in enumerate((15, 30)):
        L64.upload(U)
        L64.ape(n, 0.5, "all")
        sabs = L64.qtop(with_abs=True)[1]
        out[f"qtop_after_{n}_ape_all"] = {"q_fp64": float(q64[i]), "abs": float(abs(q32[i] - q64[i])),
                                          "abs_over_sum_abs_q": float(abs(q32[i] - q64[i]) / sabs),
                                          "rel": float(abs(q32[i] - q64[i]) / max(abs(q64[i]), 1e-300))}
    out["meets_1e-6_relative"] = {
        "plaquette": out["plaquette_rel"] <= 1e-6,
        "wilson_W_ge_1e-2": all(out[f"wilson_after_{n}_spatial_ape"]["max_rel_where_W_ge_1e-2"] <= 1e-6
                                for n in (100, 200, 400)),
        "wilson_all": all(out[f"wilson_after_{n}_spatial_ape"]["max_rel_all"] <= 1e-6 for n in (100, 200, 400)),
        "qtop": all(out[f"qtop_after_{n}_ape_all"]["rel"] <= 1e-6 for n in (15, 30))}
    L32.close()
    L64.close()
    return out


def big_lattice_figures(device, seed, K=3):
    """96^4 (84.9 M sites): the sweeps and APE steps in both precisions, and one configuration of the
    thesis' 96^4 measurement (400 spatial APE steps, then W(R <= 12, T <= 20)) in FP32, beside the
    reference's logged time for it (measurements/96x96x96x96_SU2_b3.09_NAPE_400.meas)."""
    from masterarbeit_b200.su2g import Lattice
    dims = (96, 96, 96, 96)
    vol = math.prod(dims)
    out = {"dims": list(dims)}
    for prec in ("fp32", "fp64"):
        L = Lattice(dims, precision=prec, beta=BETA, seed=seed, start="haar", device=device)
        L.sweep(1, 1, N_OR)
        ms = time_steps(L, K, lambda: L.sweep(1, 1, 0))
        out[f"{prec}_heatbath_link_updates_per_s"] = 4 * vol * K / (ms / 1e3)
        ms = time_steps(L, K, lambda: L.sweep(1, 1, N_OR))
        out[f"{prec}_1hb{N_OR}or_link_updates_per_s"] = (1 + N_OR) * 4 * vol * K / (ms / 1e3)
        for mode in ("all", "spatial"):
            L.ape(APE_SEQ, 0.5, mode)
            ms = time_steps(L, K, lambda: L.ape(APE_SEQ, 0.5, mode))
            out[f"{prec}_ape_{mode}_steps_per_s"] = APE_SEQ * K / (ms / 1e3)
        if prec == "fp32":
            R = [r for r in range(1, 13) for t in range(1, 21)]
            T = [t for r in range(1, 13) for t in range(1, 21)]
            spec = dict(R=R, T=T, ns_s=400, alpha_s=0.5)
            L.measure(**spec)
            L.synchronize()
            t0 = time.perf_counter()
            L.measure(**spec)
            out["fp32_measurement_s_per_configuration"] = time.perf_counter() - t0
            out["measurement_spec"] = "400 spatial APE steps (alpha 0.5), then W(R <= 12, T <= 20)"
            out["reference_logged_s_per_configuration"] = 56715.0
            out["reference_logged_source"] = ("measurements/96x96x96x96_SU2_b3.09_NAPE_400.meas (thesis cluster, one "
                                              "core; 400 spatial APE + W(R <= 12, T <= 20) per configuration)")
            L.measure_release()
        L.close()
    return out


def run_ours(args, dist, dims):
    from masterarbeit_b200.su2g import Lattice, PinnedArray

    K, W = args.steps, args.warmup
    vol = math.prod(dims)
    rank = dist.rank
    peak, peak_kind = measured_peak()
    # the headline: the reference's own update in the reference's precision -- one FP64 checkerboard
    # heatbath sweep of all 4V links, then the plaquette (qcd.c:54-60: gaugefieldUpdate, plaquette)
    lat = Lattice(dims, precision="fp64", beta=BETA, seed=1000 + rank, start="haar", replica=rank, device=dist.local)

    def step():   # su2g_sweep_plaquette: the plaquette is summed inside the sweep's last update passes
        lat.sweep_plaquette(1, 1, 0)

    for _ in range(W):
        step()
    clocks = clock_sampler(dist.local)
    dist.barrier()
    lat.synchronize()
    clocks.start()
    ms = time_steps(lat, K, step)   # the headline: plain calls, as a user makes them
    # the same K steps again, twice, with every launch bracketed by CUDA events: the per-kernel
    # durations of the roofline (the events add a few microseconds between launches, so not the
    # headline).  The pass with the shorter heatbath launches is used; both are reported.
    passes = []
    for _ in range(2):
        lat.profile(True)
        ms_i = time_steps(lat, K, step)
        passes.append((ms_i, lat.profile_read()))
        lat.profile(False)
    clk = clocks.stop()   # sampled over all timed passes
    ms_instr, prof = min(passes, key=lambda p: p[1]["heatbath"][1] / max(1, p[1]["heatbath"][0]))
    dist.barrier()
    ms_max = dist.max(ms)
    upd_per_step = 4 * vol
    value = upd_per_step * K * dist.world / (ms_max / 1e3)
    launches = sum(n for n, _ in prof.values())
    link64 = 32
    n_hb, t_hb = prof["heatbath"]
    avg = t_hb / n_hb
    alg = (vol // 2) * 8 * link64
    achieved = alg / (avg / 1e3) / 1e9
    traffic = dram_traffic("heatbath_fp64_" + "x".join(map(str, dims)))
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": dist.world, "steps": K, "warmup": W,
        "ms_per_step": ms_max / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic: Philox Haar-random hot start (no checkpoints or datasets)",
        "config": {"workload": f"{'x'.join(map(str, dims))} SU(2) beta={BETA} hot start; step = 1 checkerboard "
                               "heatbath sweep (heatbath only, as the reference) + plaquette (summed inside "
                               "the sweep's last update passes)",
                   "dims": list(dims), "precision": "fp64 links and arithmetic, as the reference",
                   "l2": f"inputs larger than L2 (field {4 * vol * link64 / 1e6:.0f} MB > 126 MB)",
                   "parallelism": f"replicas x{dist.world}"},
        "roofline": {"bound": "hbm", "kernel": "FP64 heatbath pass k_update<double, mu, 0> (the 8 update "
                                              "launches of a step; 3 of them also sum the plaquette)",
                     "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak, "traffic": traffic,
                     "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured"
                     else "fallback 6650 GB/s",
                     "alg_bytes_per_launch": alg,
                     "alg_bytes_note": "Vh = V/2 links updated; per update 8 links of 32 B move (the 6 staple "
                                       "links of the three other directions, read, counted once per site over both "
                                       "parity passes: 3V links; U_mu of the other parity: V/2; the update "
                                       "written: V/2)",
                     "avg_launch_ms": avg, "launches": n_hb,
                     "timing": "per-kernel CUDA-event durations from two more passes of the same K steps with "
                               "every launch bracketed by events (the one with the shorter heatbath launches); "
                               "value and ms_per_step from the plain pass",
                     "ms_per_step_with_events": ms_instr / K,
                     "avg_launch_ms_each_event_pass": [p[1]["heatbath"][1] / max(1, p[1]["heatbath"][0])
                                                       for p in passes]},
        "gpu_launches": launches,
        "clocks": clk,
    }

    extras = {}
    if not args.no_extras:
        for prec in ("fp32", "fp64"):
            L = lat if prec == "fp64" else Lattice(dims, precision="fp32", beta=BETA, seed=1000 + rank,
                                                    start="haar", replica=rank, device=dist.local)
            precision_figures(L, prec, dims, K, W, peak, clk, extras)
            if prec == "fp32":
                L.close()
        for k in ("1hb4or_link_updates_per_s", "heatbath_link_updates_per_s", "ape_all_steps_per_s",
                  "ape_spatial_steps_per_s", "wilson_R9T9_sweeps_per_s", "qtop_per_s"):
            extras[f"fp32_over_fp64_{k}"] = extras[f"fp32_{k}"] / extras[f"fp64_{k}"]
        extras["fp32_error_vs_fp64"] = fp32_error_table(dims, dist.local, 3000 + rank)
        extras["batch"] = batch_figures(dist)
        extras["graph_loop"] = graph_figures(dist)
        # one configuration's measurement (the 48^4 flows of the thesis: 400 spatial APE steps then
        # W(R<=9, T<=9); Q after 30 APE_all steps), one CUDA graph per configuration
        L = Lattice(dims, precision="fp32", beta=BETA, seed=1000 + rank, start="haar", replica=rank, device=dist.local)
        L.sweep(2, 1, N_OR)
        R9 = [r for r in range(1, 10) for t in range(1, 10)]
        T9 = [t for r in range(1, 10) for t in range(1, 10)]
        spec = dict(q_ape=[30], alpha_q=0.5, R=R9, T=T9, ns_t=0, alpha_t=0.0, ns_s=400, alpha_s=0.5)
        L.measure(**spec)
        reps = 3
        L.synchronize()
        t0 = time.perf_counter()
        for _ in range(reps):
            L.measure(**spec)
        extras["measurement_fp32_ms_per_configuration"] = (time.perf_counter() - t0) * 1e3 / reps
        extras["measurement_spec"] = "Q after 30 APE_all (alpha 0.5); W(R<=9, T<=9) after 400 spatial APE (alpha 0.5)"
        L.measure_release()
        L.close()
        extras["lattice_96x96x96x96"] = big_lattice_figures(dist.local, 4000 + rank)
    line["extras"] = extras

    # end to end through the C ABI with host buffers: upload the configuration from pinned host
    # memory (the reference's pu block, FP64 AoS), one heatbath sweep with its acceptance, read back
    # the plaquette
    host = PinnedArray((vol, 4, 4))
    lat.download(host.array)

    def e2e_step():
        lat.upload(host.array)
        lat.sweep_plaquette(1, 1, 0, acc=True)

    e2e_step()
    dist.barrier()
    t0 = time.perf_counter()
    ms_e2e = time_steps(lat, K, e2e_step)
    wall_e2e = time.perf_counter() - t0
    ms_e2e = dist.max(ms_e2e)
    line["e2e"] = {"value": upd_per_step * K * dist.world / (ms_e2e / 1e3), "unit": UNIT,
                   "h2d_bytes_per_step": vol * 16 * 8, "d2h_bytes_per_step": 8 + 8,
                   "host_wall_s": wall_e2e,
                   "what": "su2g_upload_aos_f64 (pinned host FP64 field, the reference's pu block) + "
                           "su2g_sweep_plaquette(1 heatbath sweep; plaquette and acceptance read back)"}
    host.free()

    if rank == 0 and dist.world == 1 and not args.no_cpu:
        res = cpu_reference_rate(dims, 1, 0, 200_000)
        line["cpu_baseline"] = {"value": res["rates"][0], "unit": UNIT, "cores": res["cores"], "kind": res["kind"],
                                "sample": res["sample"], "cpu_model": res["model"], "nproc": res["nproc"]}
        if not args.no_extras:
            # the reference's other kernels, timed beside the GPU figures of this run (CPU-baseline leg)
            ck = cpu_reference_kernels(extras, dims)
            if ck:
                line["cpu_baseline"]["per_kernel"] = ck
    lat.close()
    if rank == 0:
        print(json.dumps(line), flush=True)


def run_kernel(args, dims):
    """One kernel family alone: a Haar-start lattice after 2 sweeps of 1 HB + 4 OR, --warmup calls,
    then --steps calls timed with CUDA events on the lattice's stream (a profiling target)."""
    from masterarbeit_b200.su2g import Lattice
    L = Lattice(dims, precision=args.precision, beta=BETA, seed=1000, start="haar")
    L.sweep(2, 1, N_OR)
    fn = KERNELS[args.kernel]
    for _ in range(args.warmup):
        fn(L)
    ms = time_steps(L, max(1, args.steps), lambda: fn(L))
    L.close()
    print(json.dumps({"kernel": args.kernel, "precision": args.precision, "dims": dims, "calls": args.steps,
                      "ms_per_call": ms / max(1, args.steps)}), flush=True)


def main():
    args = parse()
    dims = [int(x) for x in args.dims.split(",")]
    if args.kernel:
        run_kernel(args, dims)
        return
    dist = Dist()
    try:
        if args.impl == "reference":
            run_reference(args, dist, dims)
        else:
            run_ours(args, dist, dims)
    finally:
        dist.close()


if __name__ == "__main__":
    main()
