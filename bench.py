"""Benchmark of the VecGeom hot path on B200: Mpoints/s per shape op.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl vgb|reference]
                    [--workload shapes|heavy|box|baskets|nav] [--only]
                    [--precision fp64|fp32r]

One step = every (shape, op) pair of the workload run once over its whole
point batch through libvgb.  Workloads (seeded synthetic inputs):
  shapes  tube (rmin 5, rmax 20, dz 30, phi 0-270 deg), cone (0/10, 5/20,
          dz 25) and sphere (rmin 10, rmax 30, theta 0-90 deg), 2^22 points each,
          1/3 inside, 1/3 outside in a 1.5x box, 1/3 within 1e-6 mm of the
          surface, isotropic directions; Inside, Contains, SafetyToIn,
          DistanceToIn on all points, SafetyToOut and DistanceToOut on the
          points Contains() accepts.
  heavy   torus, polycone, polyhedron and box minus tube, the same mix and ops.
  box     box (10, 20, 30) mm, 2^20 points uniform in 1.5x the box; the same
          ops (DistanceToOut/SafetyToOut on the inside subset).
  baskets 4,096 mixed baskets of eight jittered shape kinds at random
          placements, DistanceToIn + SafetyToIn, one captured graph launch.
  nav     served navigation in a layered detector: Poisson-arriving requests of
          straight tracks, steps/s with p50/p99 request latency.
The default run is the shapes workload, with the others and the FP32+refine
form as extra keys (--only: just the named workload).
value = point-ops / device time (inputs resident in HBM, L2 flushed before
every op, CUDA events around each launch); e2e = the same ops through the
public API with pinned host buffers (copies inside the timed region): per
shape one vgb_batch_fused call over all points (DistanceToOut and SafetyToOut
where Contains() holds), so each point crosses PCIe once, with the PCIe floor
of the same bytes beside it; e2e_per_op = the same with one vgb_batch call per
op.  Rank 0 prints one JSON line.
"""
from __future__ import annotations

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

# algorithmic bytes per point through the FP64 SOA API
BYTES = {"contains": 25, "inside": 28, "safety_to_in": 32, "safety_to_out": 32,
         "distance_to_in": 64, "distance_to_out": 64}
OPS = ("inside", "contains", "safety_to_in", "safety_to_out", "distance_to_in",
       "distance_to_out")
LOCAL_OPS = ("safety_to_out", "distance_to_out")   # run on the Contains() subset


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="vgb", choices=["vgb", "reference"])
    ap.add_argument("--workload", default="shapes",
                    choices=["shapes", "heavy", "box", "baskets", "nav"])
    ap.add_argument("--baskets", type=int, default=4096, help="baskets of the basket workload")
    ap.add_argument("--requests", type=int, default=300, help="requests of the nav workload")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "fp32r"])
    ap.add_argument("--n", type=int, default=0, help="points per shape (0 = workload default)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--shapes", default="", help="comma list restricting the workload's shapes")
    ap.add_argument("--only", action="store_true",
                    help="only the named workload (the default run adds the other "
                         "configurations and the other precision as extra keys)")
    return ap.parse_args()


# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) per point of the
# dominant kernels, each from one ncu capture of a 2^22-point launch; the
# profiles/ summaries give the command and the raw figures.
NCU_TRAFFIC_PER_POINT = {
    # profiles/sphere_distance_to_in_fp64_2p22.md, current build
    ("sphere", "distance_to_in", "fp64"): (202.023424e6 + 24.235776e6) / 4194304,
}


def workload_shapes(name: str):
    from vecgeom_b200 import workloads as W
    return W.bench_config(name)


L2_POLICY = "flushed (256 MB read sweep) before every op, outside the events"


def workload_desc(name, n, precision):
    d = _workload_desc(name, n, precision)
    d["l2"] = L2_POLICY
    return d


def _workload_desc(name, n, precision):
    if name == "heavy":
        return {"workload": "torus/polycone/polyhedron/box-minus-tube, 2^22 mixed points each",
                "shapes": ["torus(0,5,50)", "polycone(10 planes, phi 0-300deg)",
                           "polyhedron(8 sides, 6 planes, 10/40)", "box(30,30,30)-tube(15,dz 40)"],
                "points_per_shape": n, "ops": list(OPS), "precision": precision}
    if name == "box":
        return {"workload": "box (10,20,30) mm fp64, 2^20 uniform points in 1.5x box",
                "points_per_shape": n, "ops": list(OPS), "precision": precision}
    return {"workload": "tube/cone/sphere, 2^22 mixed points each (1/3 in, 1/3 out, "
                        "1/3 within 1e-6 mm of the surface)",
            "shapes": ["tube(5,20,30,0-270deg)", "cone(0,10,5,20,25)", "sphere(10,30,th 0-90deg)"],
            "points_per_shape": n, "ops": list(OPS), "precision": precision}


# ---------------------------------------------------------------------------
# clocks
# ---------------------------------------------------------------------------

class ClockSampler:
    """Samples SM clock and clock-event (throttle) reasons through NVML every
    few milliseconds while running (reads only; changes no GPU setting)."""

    REASONS = {"hw_slowdown": "nvmlClocksEventReasonHwSlowdown",
               "hw_thermal_slowdown": "nvmlClocksEventReasonHwThermalSlowdown",
               "sw_thermal_slowdown": "nvmlClocksEventReasonSwThermalSlowdown",
               "sw_power_cap": "nvmlClocksEventReasonSwPowerCap",
               "hw_power_brake": "nvmlClocksEventReasonHwPowerBrakeSlowdown"}

    def __init__(self, index: int, period_s: float = 0.001):
        self.index = index
        self.period = period_s
        self.samples = []
        self.reasons = set()
        self.max_mhz = None
        self._stop = threading.Event()
        self._thread = None
        self.err = None

    def _handle(self, N):
        """NVML handle of this process's GPU: by index, else by the UUID CUDA
        reports (NVML's numbering can differ from CUDA's in a container)."""
        try:
            return N.nvmlDeviceGetHandleByIndex(self.index)
        except Exception:  # noqa: BLE001
            import torch
            uuid = str(torch.cuda.get_device_properties(self.index).uuid)
            return N.nvmlDeviceGetHandleByUUID(uuid if uuid.startswith("GPU-") else "GPU-" + uuid)

    def _smi_loop(self, err):
        """Fallback: nvidia-smi's query loop (reads only)."""
        import torch
        uuid = str(torch.cuda.get_device_properties(self.index).uuid)
        uuid = uuid if uuid.startswith("GPU-") else "GPU-" + uuid
        cmd = ["nvidia-smi", "-i", uuid, "--query-gpu=clocks.sm,clocks.max.sm,"
               "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
               "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
               "--format=csv,noheader,nounits", "-lms", "50"]
        try:
            proc = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError as e:
            self.err = f"{err}; nvidia-smi unavailable: {e}"
            return

        def loop():
            names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
            for line in proc.stdout:
                if self._stop.is_set():
                    break
                f = [v.strip() for v in line.split(",")]
                try:
                    self.samples.append(float(f[0]))
                    self.max_mhz = float(f[1])
                except (ValueError, IndexError):
                    continue
                for name, v in zip(names, f[2:]):
                    if v.lower() == "active":
                        self.reasons.add(name)
            proc.terminate()
        self._proc = proc
        self._thread = threading.Thread(target=loop, daemon=True)
        self._thread.start()

    def start(self):
        try:
            import pynvml as N
            N.nvmlInit()
            h = self._handle(N)
            self.max_mhz = float(N.nvmlDeviceGetMaxClockInfo(h, N.NVML_CLOCK_SM))
        except Exception as e:  # noqa: BLE001
            self._smi_loop(f"nvml unavailable: {e}")
            return

        def loop():
            while not self._stop.is_set():
                try:
                    self.samples.append(float(N.nvmlDeviceGetClockInfo(h, N.NVML_CLOCK_SM)))
                    r = N.nvmlDeviceGetCurrentClocksEventReasons(h)
                    for name, attr in self.REASONS.items():
                        if r & getattr(N, attr, 0):
                            self.reasons.add(name)
                except Exception as e:  # noqa: BLE001
                    self.err = str(e)
                    return
                time.sleep(self.period)
        self._thread = threading.Thread(target=loop, daemon=True)
        self._thread.start()

    def stop(self) -> dict:
        self._stop.set()
        proc = getattr(self, "_proc", None)
        if proc is not None:
            proc.terminate()
            try:
                proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                proc.kill()
        if self._thread is not None:
            self._thread.join(timeout=2)
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz,
                    "reasons": [self.err or "no samples"], "samples": 0}
        return {"sm_mhz": float(np.median(self.samples)), "sm_max_mhz": self.max_mhz,
                "reasons": sorted(self.reasons), "samples": len(self.samples)}


# ---------------------------------------------------------------------------
# CPU baseline: the reference Scalar backend (oracle/_ref) or the C oracle
# ---------------------------------------------------------------------------

def cpu_rate(workloads: dict, budget_s: float = 12.0, sample: int = 1 << 18) -> dict:
    """Point-ops/s of the reference on this host's cores, all threads, on a
    bounded sample: the first `sample` points of each shape's arrays of the very
    workload the GPU arm times (same seeds, same mix).  Each op repeats for
    about budget_s / (shapes x ops) seconds."""
    import oracle
    from oracle import oracle_unplaced, ref_unplaced
    threads = os.cpu_count() or 1
    use_ref = oracle.RefLib.available()
    kind = "reference" if use_ref else "port"
    per = budget_s / (len(workloads) * len(OPS))
    tot_pts, tot_t = 0, 0.0
    if use_ref:
        ref = oracle.RefLib()
    else:
        orc = oracle.Oracle()
        threads = 1
    for name, wl in workloads.items():
        spec = wl.spec
        m0 = min(sample, wl.n)
        # the points on which the reference's own result is defined (its
        # polyhedron reads past its segment array within 1e-9 mm of an end plane)
        keep = oracle.reference_defined(spec, wl.z[:m0])
        pts = tuple(np.ascontiguousarray(a[:m0][keep]) for a in (wl.x, wl.y, wl.z))
        dirs = tuple(np.ascontiguousarray(a[:m0][keep]) for a in (wl.dx, wl.dy, wl.dz))
        if use_ref:
            pv = ref.placed(ref_unplaced(ref, spec))
            tr = ref.last_transform

            def run(op, p, d, s, pv=pv, tr=tr, spec=spec):
                if spec.kind == "sphere" and op == oracle.DISTANCE_TO_IN:
                    # the reference's sphere DistanceToIn is a stub; time USolids'
                    return ref.usphere_distance_to_in(spec.params, tr, p, d, nthreads=threads)
                return ref.batch(pv, op, p, d, s, nthreads=threads)
        else:
            sh = oracle_unplaced(orc, spec)
            xf = orc.xform()
            run = lambda op, p, d, s: orc.batch(sh, xf, op, p, d, s)  # noqa
        inside = run(oracle.CONTAINS, pts, None, None).astype(bool)
        sub = tuple(np.ascontiguousarray(a[inside]) for a in pts)
        subd = tuple(np.ascontiguousarray(a[inside]) for a in dirs)
        for opname in OPS:
            op = getattr(oracle, opname.upper())
            p, d = (sub, subd) if opname in LOCAL_OPS else (pts, dirs)
            use_dir = opname.startswith("distance")
            m = len(p[0])
            st = np.full(m, 1e30)
            reps, t0 = 0, time.perf_counter()
            while True:
                run(op, p, d if use_dir else None, st if use_dir else None)
                reps += 1
                el = time.perf_counter() - t0
                if el >= per:
                    break
            tot_pts += reps * m
            tot_t += el
    m0 = min(sample, min(wl.n for wl in workloads.values()))
    return {"value": tot_pts / tot_t / 1e6, "unit": "Mpoints/s", "cores": threads, "kind": kind,
            "sample": f"the first {m0} points of each shape's arrays of the timed workload (same "
                      f"seeds and mix; for the polyhedron without the points within 4e-9 mm of "
                      f"an end plane, where the reference reads past its segment array), the same "
                      f"ops (DistanceToOut/SafetyToOut on the Contains() subset); each op repeated "
                      f"for ~{per:.2f} s, {threads} threads"}


def generate(workload: str, n: int = 0, rank: int = 0) -> dict:
    """The seeded arrays of a shape workload, shape name -> ShapeWorkload,
    drawn in spawned worker processes."""
    from vecgeom_b200 import workloads as W
    shapes, n0, mix = W.bench_config(workload)
    n = n or n0
    jobs = [(workload, name, n, W.bench_seed(si, rank), mix) for si, name in enumerate(shapes)]
    return dict(zip(shapes, W.bench_workloads(jobs)))


def run_reference_arm(args):
    """The reference's own CPU implementation of the path (oracle/_ref, the
    reference compiled from its sources) on this host's cores, on the GPU arm's
    workload, metric and config.  A step is a bounded sample of the workload."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    wls = generate(args.workload, args.n)
    n = next(iter(wls.values())).n
    step_budget = max(2.0, 60.0 / max(1, args.steps))
    for _ in range(args.warmup):
        cpu_rate(wls, budget_s=0.5, sample=1 << 14)
    times = []
    cb = None
    for _ in range(max(1, args.steps)):
        cb = cpu_rate(wls, budget_s=step_budget)
        times.append(cb["value"])
    v = float(np.median(times))
    line = {"impl": "reference", "metric": "Mpoints/s per shape op (fp64)", "value": v,
            "unit": "Mpoints/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
            "config": workload_desc(args.workload, n, "fp64"),
            "cpu_baseline": {"value": v, "unit": "Mpoints/s", "cores": cb["cores"],
                             "kind": cb["kind"], "sample": cb["sample"]},
            "e2e": {"value": v, "unit": "Mpoints/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# mixed baskets: one persistent launch (CUDA graph) over many shape instances
# ---------------------------------------------------------------------------

def run_baskets(args):
    """4096 baskets (lognormal sizes, median 1024, clipped 16..65536), one
    jittered shape instance of the eight benchmark kinds each at a random
    placement; DistanceToIn + SafetyToIn per point.  One step = one replay of
    the captured persistent launch.  Inputs (~7 M points, ~400 MB) exceed L2."""
    import torch
    import vecgeom_b200 as V
    from vecgeom_b200 import workloads as W
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    rank = int(os.environ.get("RANK", "0"))
    bs = W.config4_baskets(args.baskets, seed=W.SEED_BASE + 4 + 1000 * rank)
    g = V.Geometry()
    placed, offsets, pts, dirs, step = W.build_baskets(g, bs)
    g.CloseGeometry()
    n = len(pts[0])
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    P = V.SOA3D(*(dev(a) for a in pts))
    D = V.SOA3D(*(dev(a) for a in dirs))
    S = dev(step)
    DTI, STI = 1 << 2, 1 << 4
    outs = {2: torch.empty(n, dtype=torch.float64, device="cuda"),
            4: torch.empty(n, dtype=torch.float64, device="cuda")}
    plan = V.BasketPlan(g, [(pv, o, b.n) for pv, o, b in zip(placed, offsets, bs)], DTI | STI)
    stream = torch.cuda.current_stream()
    block, tile, tune_ms = plan.tune(P, D, S, outs, reps=3, stream=stream)
    plan.capture(P, D, S, outs)
    for _ in range(max(3, args.warmup)):
        plan.replay(stream)
    torch.cuda.synchronize()
    V.lib().vgb_launch_count_reset()
    clk = ClockSampler(torch.cuda.current_device())
    clk.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        plan.replay(stream)
    e1.record(stream)
    torch.cuda.synchronize()
    clocks = clk.stop()
    launches = int(V.lib().vgb_launch_count())
    ms = e0.elapsed_time(e1) / args.steps
    value = 2 * n / (ms * 1e-3) / 1e6
    # the same work as one fused call per basket (the unbatched form)
    ref = {k: torch.empty_like(v) for k, v in outs.items()}

    def unbatched():
        for pv, off, b in zip(placed, offsets, bs):
            if b.n:
                sl = slice(off, off + b.n)
                pv.fused(DTI | STI, V.SOA3D(P.x[sl], P.y[sl], P.z[sl]),
                         {k: v[sl] for k, v in ref.items()},
                         dirs=V.SOA3D(D.x[sl], D.y[sl], D.z[sl]), step_max=S[sl])
    unbatched()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    unbatched()
    torch.cuda.synchronize()
    unb_ms = (time.perf_counter() - t0) * 1e3
    same = all(bool(((outs[k] == ref[k]) | (outs[k].isnan() & ref[k].isnan())).all())
               for k in outs)
    # end to end: pinned host inputs in, results out, every step
    hp = [torch.from_numpy(np.ascontiguousarray(a)).pin_memory() for a in (*pts, *dirs, step)]
    ho = {k: torch.empty(n, dtype=torch.float64).pin_memory() for k in outs}
    dv = [P.x, P.y, P.z, D.x, D.y, D.z, S]
    for _ in range(2):
        for a, b in zip(dv, hp):
            a.copy_(b, non_blocking=True)
        plan.replay(stream)
        for k in outs:
            ho[k].copy_(outs[k], non_blocking=True)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    e2e_steps = max(1, min(args.steps, 5))
    for _ in range(e2e_steps):
        for a, b in zip(dv, hp):
            a.copy_(b, non_blocking=True)
        plan.replay(stream)
        for k in outs:
            ho[k].copy_(outs[k], non_blocking=True)
    torch.cuda.synchronize()
    e2e_s = (time.perf_counter() - t0) / e2e_steps
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        pass
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    bpp = 24 + 24 + 8 + 8 + 8  # x,y,z + direction + step_max in, two doubles out
    achieved = bpp * n / (ms * 1e-3) / 1e9
    kinds = {k: sum(b.n for b in bs if b.spec.kind == k) for k in W.BASKET_KINDS}
    line = {"metric": "Mpoints/s per shape op (fp64, mixed baskets in one persistent launch)",
            "value": round(value, 2), "unit": "Mpoints/s", "n_gpus": 1, "steps": args.steps,
            "warmup": max(3, args.warmup), "ms_per_step": round(ms, 4),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded)",
            "config": {"workload": f"{len(bs)} baskets, lognormal sizes (median 1024, sigma 1, "
                                   "clipped 16-65536), 8 shape kinds jittered +-20%, random "
                                   "placements; DistanceToIn + SafetyToIn",
                       "points": n, "points_per_kind": kinds,
                       "l2": "inputs (~%d MB) exceed L2" % (bpp * n >> 20),
                       "autotuned": {"block": block, "tile": tile, "ms": round(tune_ms, 4)}},
            "unbatched": {"ms": round(unb_ms, 3), "mpoints_s": round(2 * n / unb_ms / 1e3, 2),
                          "launches": sum(1 for b in bs if b.n),
                          "results_identical": same},
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": hbm,
                         "unit": "GB/s", "frac": round(achieved / hbm, 4), "traffic": None,
                         "kernel": "k_baskets", "bytes_per_point": bpp,
                         "peak_source": "measured" if "hbm_gbs" in peaks else "fallback"},
            "e2e": {"value": round(2 * n / e2e_s / 1e6, 2), "unit": "Mpoints/s",
                    "h2d_bytes_per_step": 56 * n, "d2h_bytes_per_step": 16 * n},
            "gpu_launches": launches, "clocks": clocks}
    return line


# ---------------------------------------------------------------------------
# served navigation: continuous batching of Poisson-arriving track baskets
# ---------------------------------------------------------------------------

def nav_cpu_baseline(pts, dirs, max_steps, n_simple=16384, n_abbox=4096):
    """The reference's navigators on the host cores over the first tracks of
    the trace workload (oracle/_ref, the reference built from its sources):
    SimpleNavigator on every core (one navigator and state pair per thread),
    ABBoxNavigator on one (its ABBoxManager shares one hit list)."""
    import oracle
    from vecgeom_b200 import workloads as W
    if not oracle.RefLib.available():
        return None
    ref = oracle.RefLib()
    W.build_detector(oracle.RefBuilder(ref))
    threads = os.cpu_count() or 1
    sub = lambda a, k: tuple(np.ascontiguousarray(v[:k]) for v in a)  # noqa: E731
    t0 = time.perf_counter()
    _, _, _, nst = oracle.ref_nav_trace(ref, sub(pts, n_simple), sub(dirs, n_simple), 1e30,
                                        max_steps, threads)
    simple = float(nst.sum()) / (time.perf_counter() - t0)
    t0 = time.perf_counter()
    _, _, _, nst_ab = oracle.ref_abbox_nav_trace(ref, sub(pts, n_abbox), sub(dirs, n_abbox), 1e30,
                                                 max_steps)
    abbox = float(nst_ab.sum()) / (time.perf_counter() - t0)
    return {"value": round(simple, 1), "unit": "steps/s", "cores": threads, "kind": "reference",
            "sample": f"first {n_simple} trace tracks, SimpleNavigator, {threads} threads",
            "abbox_single_thread": {"value": round(abbox, 1), "unit": "steps/s",
                                    "sample": f"first {n_abbox} trace tracks, ABBoxNavigator, "
                                              "1 thread"}}


def run_nav(args):
    """Layered detector (14,011 placed volumes).  Requests of 1-16384 tracks
    (log-uniform sizes) from the origin, isotropic, arrive as a Poisson stream
    at ~80% of the measured saturated throughput; each track steps (safety +
    FindNextBoundaryAndStep) until it leaves the world or 64 steps.  The served
    run uses --precision; the other form is served with the same arrivals for
    comparison, and the raw trace throughput of both forms and of
    ABBoxNavigator is reported."""
    import torch
    import vecgeom_b200 as V
    from vecgeom_b200 import workloads as W
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    g = V.Geometry()
    W.build_detector(W.VgbBuilder(g))
    max_steps, spl = 64, 8
    rng = np.random.default_rng(W.SEED_BASE + 5)
    nreq = args.requests
    sizes = np.clip(np.round(np.exp(rng.uniform(0., np.log(16384.), nreq))), 1, 16384).astype(int)
    reqs = [W.isotropic_tracks(int(m), W.SEED_BASE + 500 + k) for k, m in enumerate(sizes)]
    prec_main = V.PREC_FP64 if args.precision == "fp64" else V.PREC_FP32_REFINE

    def drain(srv, arrivals=None):
        """Serves every request; request k is submitted when the wall clock
        passes arrivals[k] (None: all at once).  Returns latencies (s), total
        steps and wall time."""
        t0 = time.perf_counter()
        pending = list(range(nreq))
        lat, steps, done_n = {}, 0, 0
        rid_of, sub = {}, {}
        while done_n < nreq:
            now = time.perf_counter() - t0
            while pending and (arrivals is None or arrivals[pending[0]] <= now):
                k = pending.pop(0)
                sub[k] = t0 + (arrivals[k] if arrivals is not None else now)
                rid_of[srv.submit(*reqs[k])] = k
            done, live, queued = srv.step()
            tdone = time.perf_counter()
            for rid in done:
                k = rid_of.pop(rid)
                r = srv.result(rid)
                steps += int(r["nsteps"].sum())
                lat[k] = tdone - sub[k]
                done_n += 1
            if not done and not live and not queued and pending and arrivals is not None:
                time.sleep(max(0., min(0.002, arrivals[pending[0]] - now)))
        return lat, steps, time.perf_counter() - t0

    def serve(precision, arrivals, spl_=None):
        srv = V.NavServer(g, max_tracks=1 << 18, steps_per_launch=spl_ or spl,
                          max_steps=max_steps, precision=precision)
        drain(srv)  # warm-up
        if arrivals is None:
            _, st, wall = drain(srv)
            return st, wall, None
        lat, st, wall = drain(srv, arrivals)
        L = np.array([lat[k] for k in range(nreq)]) * 1e3
        return st, wall, {"p50": round(float(np.percentile(L, 50)), 3),
                          "p99": round(float(np.percentile(L, 99)), 3),
                          "max": round(float(L.max()), 3)}

    # steps per launch: the saturated FP64 throughput picks it (fewer, longer
    # launches amortise the per-iteration admission and retirement)
    sweep = {}
    for cand in (4, 8, 16, 32, 64):
        st_, wall_, _ = serve(V.PREC_FP64, None, cand)
        sweep[cand] = st_ / wall_
    spl = max(sweep, key=sweep.get)
    # saturated throughput of the FP64 form sets one arrival stream for both forms
    sat_steps, sat_s, _ = serve(V.PREC_FP64, None)
    rate = 0.8 * (sat_steps / sat_s) / (sat_steps / nreq)      # requests per second
    arrivals = np.cumsum(rng.exponential(1. / rate, nreq))
    other = V.PREC_FP32_REFINE if prec_main == V.PREC_FP64 else V.PREC_FP64
    o_steps, o_wall, o_lat = serve(other, arrivals)
    clk = ClockSampler(torch.cuda.current_device())
    V.lib().vgb_launch_count_reset()
    clk.start()
    steps, wall, lat = serve(prec_main, arrivals)
    clocks = clk.stop()
    launches = int(V.lib().vgb_launch_count())
    sat32_steps, sat32_s, _ = serve(V.PREC_FP32_REFINE, None)
    # raw trace throughput (one launch, 2^17 tracks, device events)
    n = 1 << 17
    pts, dirs = W.isotropic_tracks(n, W.SEED_BASE + 7)
    dev = lambda a: torch.from_numpy(a).cuda()  # noqa: E731
    P, D = V.SOA3D(*(dev(a) for a in pts)), V.SOA3D(*(dev(a) for a in dirs))
    nst = torch.zeros(n, dtype=torch.int32, device="cuda")
    nav = V.SimpleNavigator(g)
    abnav = V.ABBoxNavigator(g)
    trace = {}
    for name, pr in (("fp64", V.PREC_FP64), ("fp32r", V.PREC_FP32_REFINE), ("abbox", None)):
        def run():
            if pr is None:
                abnav.Trace(P, D, 1e30, max_steps, nst)
            else:
                nav.Trace(P, D, 1e30, max_steps, nst, precision=pr)
        for _ in range(2):
            run()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        run()
        e1.record()
        torch.cuda.synchronize()
        trace[name] = round(int(nst.sum()) / (e0.elapsed_time(e1) * 1e-3), 1)
    cpu = nav_cpu_baseline(pts, dirs, max_steps)
    tag = "fp64" if prec_main == V.PREC_FP64 else "fp32+refine"
    line = {"metric": f"nav steps/s ({tag}, served) with p50/p99 request latency",
            "value": round(steps / wall, 1), "unit": "steps/s", "n_gpus": 1,
            "steps": nreq, "warmup": 1, "ms_per_step": round(wall / nreq * 1e3, 4),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if prec_main == V.PREC_FP64 else "f32+f64",
            "data": "synthetic (seeded)",
            "config": {"workload": "layered detector, 14011 placed volumes, 4 levels; "
                                   f"{nreq} requests of 1-16384 tracks (log-uniform) from the "
                                   "origin, Poisson arrivals at 80% of the FP64 saturated "
                                   "throughput",
                       "max_steps": max_steps, "steps_per_launch": spl,
                       "steps_per_launch_sweep": {str(k): round(v, 1) for k, v in sweep.items()},
                       "tracks": int(sizes.sum()),
                       "saturated_steps_per_s": {"fp64": round(sat_steps / sat_s, 1),
                                                 "fp32r": round(sat32_steps / sat32_s, 1)},
                       "arrival_rate_per_s": round(rate, 2)},
            "latency_ms": lat,
            "other_precision": {"precision": "fp32+refine" if other else "fp64",
                                "steps_per_s": round(o_steps / o_wall, 1), "latency_ms": o_lat},
            "trace_steps_per_s": trace,
            "cpu_baseline": cpu,
            "e2e": {"value": round(steps / wall, 1), "unit": "steps/s",
                    "h2d_bytes_per_step": int(48 * sizes.sum() / nreq),
                    "d2h_bytes_per_step": int(36 * sizes.sum() / nreq)},
            "gpu_launches": launches, "clocks": clocks}
    return line


# ---------------------------------------------------------------------------
# peaks and rooflines
# ---------------------------------------------------------------------------

def load_peaks() -> dict:
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        return {}


def load_op_costs() -> dict:
    """Algorithmic flops per point of every (workload, shape, op), from
    bench/op_costs.json (bench/make_op_costs.py)."""
    try:
        return json.load(open(os.path.join(ROOT, "bench", "op_costs.json")))["workloads"]
    except (OSError, ValueError, KeyError):
        return {}


def measure_fma_peaks(stream) -> dict:
    """FP64 and FP32 FMA throughput of this GPU (vgb_measure_fma_peak: one
    launch of independent FMA chains on every SM, CUDA events; best of 5 after
    2 warm-up launches), in GFLOP/s with an FMA counted as 2 flops."""
    import ctypes
    import vecgeom_b200 as V
    L = V.lib()
    out = {}
    for name, fp32, iters in (("fp64", 0, 2048), ("fp32", 1, 4096)):
        best = 0.0
        for k in range(7):
            fl, ms = ctypes.c_double(), ctypes.c_float()
            V.check(L.vgb_measure_fma_peak(fp32, iters, ctypes.c_void_p(stream.cuda_stream),
                                           ctypes.byref(fl), ctypes.byref(ms)))
            if k >= 2:
                best = max(best, fl.value / (ms.value * 1e-3) / 1e9)
        out[f"{name}_gflops"] = round(best, 1)
    out["method"] = ("vgb_measure_fma_peak: 8 independent FMA chains per thread, every SM "
                     "filled, CUDA events; best of 5")
    return out


def pcie_floor(h2d_bytes: int, d2h_bytes: int, reps: int = 3) -> dict:
    """The end-to-end floor of a step that moves h2d_bytes in and d2h_bytes out:
    both copies between pinned host buffers and the device at once, on two
    streams (a B200's copy engines run the two directions together, each a
    little slower than alone), timed like the end-to-end calls (wall clock
    around synchronised repetitions, after one untimed)."""
    import torch
    hi = torch.empty(h2d_bytes, dtype=torch.uint8).pin_memory()
    ho = torch.empty(d2h_bytes, dtype=torch.uint8).pin_memory()
    di = torch.empty(h2d_bytes, dtype=torch.uint8, device="cuda")
    do = torch.empty(d2h_bytes, dtype=torch.uint8, device="cuda")
    s_in, s_out = torch.cuda.Stream(), torch.cuda.Stream()

    def timed(copy_in: bool, copy_out: bool) -> float:
        def once():
            if copy_in:
                with torch.cuda.stream(s_in):
                    di.copy_(hi, non_blocking=True)
            if copy_out:
                with torch.cuda.stream(s_out):
                    ho.copy_(do, non_blocking=True)
        once()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(reps):
            once()
        torch.cuda.synchronize()
        return (time.perf_counter() - t0) / reps
    t_in, t_out, t_both = timed(True, False), timed(False, True), timed(True, True)
    del hi, ho, di, do
    return {"both_ms": round(t_both * 1e3, 3), "h2d_gbs": round(h2d_bytes / t_in / 1e9, 1),
            "d2h_gbs": round(d2h_bytes / t_out / 1e9, 1),
            "method": "the step's bytes copied in and out at once (pinned host memory, two "
                      "streams), wall clock like the end-to-end calls"}


def replica_rate(points: int, step_ms: float, world: int, dist=None, device: str = "cuda"):
    """Replicas: every rank processes its own batch of `points` per step.  The
    job's step time is the slowest rank's (an all-reduce MAX over the ranks) and
    the whole-job rate is world x points over it, in Mpoint-ops/s.  Returns
    (step ms, rate)."""
    if world > 1:
        import torch
        t = torch.tensor([step_ms], dtype=torch.float64, device=device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        step_ms = float(t.item())
    return step_ms, world * points / (step_ms * 1e-3) / 1e6


def op_roofline(opname: str, points: int, seconds: float, flops_per_point, hbm_gbs: float,
                fp64_gflops) -> dict:
    """Where one op sits: its algorithmic bytes (and flops, when counted) per
    point over its event-timed duration, against measured HBM bandwidth and
    FP64 FMA throughput; the bound is the resource its arithmetic intensity
    (flops per byte) saturates first."""
    gbs = BYTES[opname] * points / seconds / 1e9
    r = {"gbs": round(gbs, 1), "frac_hbm": round(gbs / hbm_gbs, 4), "bound": "hbm"}
    if flops_per_point is not None and fp64_gflops:
        gfl = flops_per_point * points / seconds / 1e9
        ai = flops_per_point / BYTES[opname]
        r.update({"gflops": round(gfl, 1), "frac_fp64": round(gfl / fp64_gflops, 4),
                  "flops_per_byte": round(ai, 3)})
        if ai > fp64_gflops / hbm_gbs:
            r["bound"] = "fp64"
    return r


# ---------------------------------------------------------------------------
# shape workloads on the GPU
# ---------------------------------------------------------------------------

def run_shapes(args, workload: str, wls: dict, precision: str, peaks: dict, fma: dict,
               with_e2e: bool = True, with_cpu: bool = True, world: int = 1, rank: int = 0,
               dist=None) -> dict:
    """One step = every (shape, op) of the workload once over its whole batch
    (inputs resident in HBM, L2 flushed before every op, CUDA events around
    each launch).  Returns the JSON line."""
    import torch

    import vecgeom_b200 as V
    from vecgeom_b200 import workloads as W

    L = V.lib()
    prec = V.PREC_FP64 if precision == "fp64" else V.PREC_FP32_REFINE
    shapes = {k: w.spec for k, w in wls.items()}
    if args.shapes:
        keep = set(args.shapes.split(","))
        shapes = {k: v for k, v in shapes.items() if k in keep}
    n = next(iter(wls.values())).n
    stream = torch.cuda.current_stream()
    local = torch.cuda.current_device()

    # --- geometry + inputs resident in HBM --------------------------------
    g = V.Geometry()
    placed = {}
    for name, spec in shapes.items():
        lv = g.LogicalVolume(name, W.build_unplaced(g, spec))
        placed[name] = lv.Place(g.Transformation3D())
    g.CloseGeometry()

    def dev(a):
        return torch.from_numpy(np.ascontiguousarray(a)).cuda()

    tasks = []   # (shape, opname, n, callable on device, callable on host)
    fused_calls = []  # end-to-end: one fused host-buffer call per point set
    fused_h2d = fused_d2h = 0
    checks = []  # (shape, opname, output, FP64 output, FP64 call) for the error report
    h2d_bytes = d2h_bytes = 0
    for si, (name, spec) in enumerate(shapes.items()):
        wl = wls[name]
        pv = placed[name]
        P = V.SOA3D(dev(wl.x), dev(wl.y), dev(wl.z))
        D = V.SOA3D(dev(wl.dx), dev(wl.dy), dev(wl.dz))
        S = dev(wl.step)
        c = torch.empty(n, dtype=torch.uint8, device="cuda")
        pv.Contains(P, c, precision=prec)
        torch.cuda.synchronize()
        sel = c.bool()
        PS = V.SOA3D(P.x[sel].contiguous(), P.y[sel].contiguous(), P.z[sel].contiguous())
        DS = V.SOA3D(D.x[sel].contiguous(), D.y[sel].contiguous(), D.z[sel].contiguous())
        SS = S[sel].contiguous()
        ns = int(sel.sum().item())
        # pinned host copies for the end-to-end leg
        pin = lambda t: t.cpu().pin_memory()  # noqa: E731
        if with_e2e:
            HP = V.SOA3D(pin(P.x), pin(P.y), pin(P.z))
            HD = V.SOA3D(pin(D.x), pin(D.y), pin(D.z))
            HS = pin(S)
            HPS = V.SOA3D(pin(PS.x), pin(PS.y), pin(PS.z))
            HDS = V.SOA3D(pin(DS.x), pin(DS.y), pin(DS.z))
            HSS = pin(SS)
        for opname in OPS:
            local_op = opname in LOCAL_OPS
            m = ns if local_op else n
            dt = {"contains": torch.uint8, "inside": torch.int32}.get(opname, torch.float64)
            out_d = torch.empty(m, dtype=dt, device="cuda")
            pts_d, dirs_d, st_d = (PS, DS, SS) if local_op else (P, D, S)
            meth = {"contains": "Contains", "inside": "Inside", "safety_to_in": "SafetyToIn",
                    "safety_to_out": "SafetyToOut", "distance_to_in": "DistanceToIn",
                    "distance_to_out": "DistanceToOut"}[opname]
            fn = getattr(pv, meth)
            out64 = torch.empty_like(out_d)
            if opname.startswith("distance"):
                run64 = (lambda fn=fn, a=pts_d, b=dirs_d, s=st_d, o=out64:
                         fn(a, b, s, o, precision=V.PREC_FP64))
                run_d = (lambda fn=fn, a=pts_d, b=dirs_d, s=st_d, o=out_d:
                         fn(a, b, s, o, precision=prec))
            else:
                run64 = lambda fn=fn, a=pts_d, o=out64: fn(a, o, precision=V.PREC_FP64)  # noqa
                run_d = lambda fn=fn, a=pts_d, o=out_d: fn(a, o, precision=prec)  # noqa: E731
            checks.append((name, opname, out_d, out64, run64))
            run_h = None
            if with_e2e:
                out_h = torch.empty(m, dtype=dt).pin_memory()
                pts_h, dirs_h, st_h = (HPS, HDS, HSS) if local_op else (HP, HD, HS)
                if opname.startswith("distance"):
                    run_h = (lambda fn=fn, a=pts_h, b=dirs_h, s=st_h, o=out_h:
                             fn(a, b, s, o, precision=prec))
                    h2d_bytes += m * 56
                else:
                    run_h = lambda fn=fn, a=pts_h, o=out_h: fn(a, o, precision=prec)  # noqa
                    h2d_bytes += m * 24
                d2h_bytes += m * out_d.element_size()
            tasks.append((name, opname, m, run_d, run_h))
        if with_e2e and precision == "fp64":
            # the fused end-to-end form: one call per shape over all points, every
            # op, DistanceToOut and SafetyToOut evaluated where Contains() holds
            # (VGB_FUSED_LOCAL_INSIDE_ONLY): each point crosses PCIe once; the
            # point-ops are the device step's.  vgb_batch_fused computes in FP64
            # only, so the FP32+refine form's end-to-end number is the per-op one
            code = {"contains": 0, "inside": 1, "distance_to_in": 2, "distance_to_out": 3,
                    "safety_to_in": 4, "safety_to_out": 5}
            outs = {code[o]: torch.empty(n, dtype={"contains": torch.uint8,
                                                   "inside": torch.int32}
                                         .get(o, torch.float64)).pin_memory() for o in OPS}
            fused_calls.append(lambda pv=pv, hp=HP, hd=HD, hs=HS, outs=outs:
                               pv.fused(0x3f, hp, outs, hd, hs, local_inside_only=True))
            fused_h2d += n * 56
            fused_d2h += sum(v.element_size() * n for v in outs.values())

    # L2 flush: a read sweep over 256 MB (> 126 MB L2); reading leaves clean lines,
    # so the next kernel pays no write-back for the flush itself
    flush = torch.ones(64 << 20, dtype=torch.float32, device="cuda")
    flush_sink = torch.empty((), dtype=torch.float32, device="cuda")
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in tasks]

    def one_step(timed: bool):
        for k, t in enumerate(tasks):
            torch.sum(flush, dim=0, out=flush_sink)
            if timed:
                ev[k][0].record(stream)
            t[3]()
            if timed:
                ev[k][1].record(stream)

    warm = max(3, args.warmup)
    for _ in range(warm):
        one_step(False)
    torch.cuda.synchronize()

    per_task_ms = np.zeros(len(tasks))
    clocks = ClockSampler(local)
    clocks.start()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    L.vgb_launch_count_reset()
    for _ in range(args.steps):
        one_step(True)
        torch.cuda.synchronize()
        per_task_ms += np.array([a.elapsed_time(b) for a, b in ev])
    launches = int(L.vgb_launch_count())
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clk = clocks.stop()

    pts_per_step = sum(t[2] for t in tasks)
    step_ms, value = replica_rate(pts_per_step, float(per_task_ms.sum()) / args.steps, world,
                                  dist)

    # rooflines: every op, and the dominant one (largest share of the step)
    hbm_peak = float(peaks.get("hbm_gbs", 6650.0))
    fp64_peak = fma.get("fp64_gflops")
    costs = load_op_costs().get(workload, {})
    per_op, per_op_roof = {}, {}
    for i, (name, opname, m, _, _) in enumerate(tasks):
        sec = per_task_ms[i] / args.steps * 1e-3
        per_op[f"{name}:{opname}"] = round(m / sec / 1e6, 1)
        c = costs.get(name, {})
        fl = c.get(opname, {}).get("flops_per_point") if isinstance(c, dict) else None
        per_op_roof[f"{name}:{opname}"] = op_roofline(opname, m, sec, fl, hbm_peak, fp64_peak)
    k = int(np.argmax(per_task_ms))
    name, opname, m, _, _ = tasks[k]
    dom = per_op_roof[f"{name}:{opname}"]
    traffic = None
    tp = NCU_TRAFFIC_PER_POINT.get((name, opname, precision))
    if tp is not None:
        traffic = int(round(tp * m))
    if dom["bound"] == "fp64":
        roof = {"bound": "fp64", "achieved": dom["gflops"], "peak": fp64_peak, "unit": "GFLOP/s",
                "frac": dom["frac_fp64"]}
    else:
        roof = {"bound": "hbm", "achieved": dom["gbs"], "peak": hbm_peak, "unit": "GB/s",
                "frac": dom["frac_hbm"]}
    roof.update({"traffic": traffic, "kernel": f"{name} {opname}",
                 "bytes_per_point": BYTES[opname],
                 "flops_per_point": (costs.get(name, {}) or {}).get(opname, {}).get(
                     "flops_per_point") if isinstance(costs.get(name), dict) else None,
                 "frac_hbm": dom["frac_hbm"], "frac_fp64": dom.get("frac_fp64"),
                 "peak_source": ("hbm: measured (MEASURED_PEAKS.json)" if "hbm_gbs" in peaks
                                 else "hbm: fallback") + "; fp64: measured (vgb_measure_fma_peak)"})

    # end-to-end through the public API with pinned host buffers
    e2e = e2e_per_op = None
    if with_e2e:
        def timed_wall(calls):
            for _ in range(2):
                for c in calls:
                    c()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            reps = max(1, min(args.steps, 3))
            for _ in range(reps):
                for c in calls:
                    c()
            sec = (time.perf_counter() - t0) / reps
            if world > 1:
                tt = torch.tensor([sec], device="cuda")
                dist.all_reduce(tt, op=dist.ReduceOp.MAX)
                sec = float(tt.item())
            return sec
        e2e_s = timed_wall([t[4] for t in tasks])
        e2e_per_op = {"value": round(world * pts_per_step / e2e_s / 1e6, 2),
                      "unit": "Mpoints/s", "h2d_bytes_per_step": int(h2d_bytes),
                      "d2h_bytes_per_step": int(d2h_bytes),
                      "api": "vgb_batch, host buffers, 1 call per op"}
        if fused_calls:
            e2e_s = timed_wall(fused_calls)
            e2e = {"value": round(world * pts_per_step / e2e_s / 1e6, 2), "unit": "Mpoints/s",
                   "h2d_bytes_per_step": int(fused_h2d), "d2h_bytes_per_step": int(fused_d2h),
                   "api": "vgb_batch_fused, host buffers, 1 call per shape (local ops where "
                          "Contains() holds)",
                   "ms_per_step": round(e2e_s * 1e3, 3)}
            # the PCIe floor of the same bytes: the end-to-end step's bound
            floor = pcie_floor(int(fused_h2d), int(fused_d2h))
            floor["frac"] = round(floor["both_ms"] / (e2e_s * 1e3), 4)
            e2e["pcie_floor"] = floor
        else:
            e2e = e2e_per_op

    # FP32+refine: error of every op against the FP64 form on the same points
    err = None
    if precision != "fp64":
        err = {}
        for t, (name, opname, o, o64, run64) in zip(tasks, checks):
            t[3]()
            run64()
            torch.cuda.synchronize()
            a, b = o.double(), o64.double()
            both = torch.isfinite(a) & torch.isfinite(b)
            dif = torch.where(both, (a - b).abs(), torch.zeros_like(a))
            bad = ~(both | ((a == b) | (a.isnan() & b.isnan())))
            err[f"{name}:{opname}"] = {
                "max_mm": float(dif.max().item()) if dif.numel() else 0.,
                "p99_mm": float(torch.quantile(dif[:1 << 24].float(), .99).item())
                if dif.numel() else 0.,
                "class_mismatches": int(bad.sum().item())}
    line = {"metric": "Mpoints/s per shape op" + (" (fp64)" if precision == "fp64"
                                                  else " (fp32+refine)"),
            "value": round(value, 2), "unit": "Mpoints/s", "n_gpus": world,
            "steps": args.steps, "warmup": warm, "ms_per_step": round(step_ms, 4),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if precision == "fp64" else "f32+f64",
            "data": "synthetic (seeded)",
            "config": workload_desc(workload, n, precision),
            "per_op_mpoints_s": per_op, "roofline": roof, "roofline_per_op": per_op_roof,
            "e2e": e2e, "e2e_per_op": e2e_per_op, "error_vs_fp64": err,
            "gpu_launches": launches, "clocks": clk}
    if with_cpu and rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_rate({k: wls[k] for k in shapes})
    return line


def summary(line: dict) -> dict:
    """The keys of a sub-benchmark line kept under the default line's configs."""
    keep = ("metric", "value", "unit", "ms_per_step", "config", "per_op_mpoints_s", "roofline",
            "roofline_per_op", "e2e", "error_vs_fp64", "gpu_launches", "clocks", "cpu_baseline")
    return {k: line[k] for k in keep if k in line}


# ---------------------------------------------------------------------------
# the GPU arm
# ---------------------------------------------------------------------------

def main():
    args = parse()
    if args.impl == "reference":
        run_reference_arm(args)
        return
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    extra = (args.workload == "shapes" and world == 1 and not args.only)
    # seeded inputs are drawn before CUDA starts, in spawned worker processes
    wls = {}
    if args.workload in ("shapes", "heavy", "box"):
        wls[args.workload] = generate(args.workload, args.n, rank)
    if extra:
        wls["box"] = generate("box")
        wls["heavy"] = generate("heavy")
    import torch
    import torch.distributed as dist

    torch.cuda.set_device(local)
    if args.workload == "baskets":
        print(json.dumps(run_baskets(args)), flush=True)
        return
    if args.workload == "nav":
        print(json.dumps(run_nav(args)), flush=True)
        return
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    peaks = load_peaks()
    fma = measure_fma_peaks(torch.cuda.current_stream())
    line = run_shapes(args, args.workload, wls[args.workload], args.precision, peaks, fma,
                      with_e2e=not args.no_e2e, world=world, rank=rank,
                      dist=dist if world > 1 else None)
    line["fma_peaks"] = fma
    if extra:
        other = "fp32r" if args.precision == "fp64" else "fp64"
        line["other_precision"] = summary(run_shapes(args, "shapes", wls["shapes"], other, peaks,
                                                     fma, with_e2e=not args.no_e2e,
                                                     with_cpu=False))
        line["configs"] = {
            "box": summary(run_shapes(args, "box", wls["box"], "fp64", peaks, fma,
                                      with_e2e=False)),
            "heavy": summary(run_shapes(args, "heavy", wls["heavy"], "fp64", peaks, fma,
                                        with_e2e=False)),
            "baskets": run_baskets(args),
            "nav": run_nav(args),
        }
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
