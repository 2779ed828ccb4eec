#!/usr/bin/env python
"""Benchmark of the OpenCFD-EC per-iteration hot path on B200.

Workload (the headline configuration): the FP64 RANS-SA swept wing, 8 uneven blocks, ~2.1 M
cells, WENO5 + Roe, LU-SGS, M 0.8, AoA 3 deg, Re 1e7 per chord (analytic O-H mesh; synthetic,
seeded - no external mesh or dataset).  A step is one NS_Time_advance (residual + LU-SGS +
update + limiter + BC + halo); the metric is cell-updates/s = cells x steps / device time.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--precision fp64|mixed] [--impl ours|reference] [--shard]

With N > 1 (torchrun) every rank solves its own copy of the case (independent solves at
different angles of attack, no collective on the data path: "weak" scaling); the timed region is
bracketed by barriers and the slowest rank's device time is used.  --shard instead splits one
config 3 wing-body solve (24 blocks) over the ranks by whole blocks, with the packed interface
halos crossing by NCCL send/recv every step ("strong" scaling).  --impl reference times the CPU
restatement of the reference algorithm (oracle/) on the host cores instead (rank 0 only).
One JSON line is printed by rank 0.
"""
import argparse
import json
import os
import statistics
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "opencfd-ec_b200"))

# algorithmic bytes per cell-update (per-kernel data model: unique inputs + outputs once)
#   residual: reads U + metrics, writes Res, dt, Lc, Lv;  LU-SGS lower: Res,U,dt,vol,Lc,Lv,S,n -> DU*;
#   upper + update: DU*,U,dt,vol,Lc,Lv,S,n -> U
BYTES = {
    ("fp64", 5): {"residual": 248, "lusgs_lower": 256, "lusgs_upper": 256},
    ("fp64", 6): {"residual": 584, "lusgs_lower": 304, "lusgs_upper": 304},
    ("fp64", 7): {"residual": 600, "lusgs_lower": 328, "lusgs_upper": 328},
    ("mixed", 5): {"residual": 148, "lusgs_lower": 176, "lusgs_upper": 176},
    ("mixed", 6): {"residual": 356, "lusgs_lower": 192, "lusgs_upper": 192},
    ("mixed", 7): {"residual": 364, "lusgs_lower": 216, "lusgs_upper": 216},
}


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """Samples SM clock / throttle reasons through NVML while the timed region runs."""

    def __init__(self, dev_index, period=0.01):
        self.samples, self.reasons, self.max_mhz = [], set(), None
        self.period, self.stop_flag, self.th, self.h = period, False, None, None
        try:
            import pynvml
            pynvml.nvmlInit()
            import torch
            uuid = str(torch.cuda.get_device_properties(dev_index).uuid)
            n = pynvml.nvmlDeviceGetCount()
            for q in range(n):
                hq = pynvml.nvmlDeviceGetHandleByIndex(q)
                u = pynvml.nvmlDeviceGetUUID(hq)
                u = u.decode() if isinstance(u, bytes) else u
                if uuid in u or u.replace("GPU-", "") in uuid:
                    self.h = hq
            if self.h is None and n == 1:
                self.h = pynvml.nvmlDeviceGetHandleByIndex(0)
            self.nv = pynvml
            if self.h is not None:
                self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM)
        except Exception:
            self.h = None

    def _run(self):
        nv = self.nv
        names = {
            "hw_slowdown": getattr(nv, "nvmlClocksEventReasonHwSlowdown", 0x8),
            "sw_thermal_slowdown": getattr(nv, "nvmlClocksEventReasonSwThermalSlowdown", 0x20),
            "hw_thermal_slowdown": getattr(nv, "nvmlClocksEventReasonHwThermalSlowdown", 0x40),
            "sw_power_cap": getattr(nv, "nvmlClocksEventReasonSwPowerCap", 0x4),
        }
        while not self.stop_flag:
            try:
                self.samples.append(nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM))
                r = nv.nvmlDeviceGetCurrentClocksEventReasons(self.h) if hasattr(nv, "nvmlDeviceGetCurrentClocksEventReasons") else nv.nvmlDeviceGetCurrentClocksThrottleReasons(self.h)
                for k, bit in names.items():
                    if r & bit:
                        self.reasons.add(k)
            except Exception:
                pass
            time.sleep(self.period)

    def __enter__(self):
        if self.h is not None:
            self.th = threading.Thread(target=self._run, daemon=True)
            self.th.start()
        return self

    def __exit__(self, *a):
        self.stop_flag = True
        if self.th:
            self.th.join()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": sorted(self.reasons), "samples": 0}
        return {"sm_mhz": statistics.median(self.samples), "sm_max_mhz": self.max_mhz, "reasons": sorted(self.reasons),
                "samples": len(self.samples)}


def rank_aoa(rank):
    """Independent replica solves: the angle of attack (deg) of each rank's copy of the case."""
    return 3.0 + 0.25 * rank


WORKLOADS = ("config2", "config2_medium", "config1", "config4")


class BatchItems:
    """The 64 config-4 airfoils as one workload (one batch handle)."""

    def __init__(self, items):
        self.items = items
        self.name = "config4_64_naca_airfoils"
        self.dims = [d for _, c in items for d in c.dims]
        self.ncells = sum(c.ncells for _, c in items)


def make_case(args, rank):
    from ocfd_b200 import cases
    prec = 1 if args.precision == "mixed" else 0
    if args.workload == "config4":
        items = cases.config4_batch(n=64, precision=prec)
        return items[0][0], BatchItems(items)
    return getattr(cases, args.workload)(precision=prec, aoa=rank_aoa(rank))


def open_solver(p, case):
    from ocfd_b200 import capi
    return capi.Batch(case.items) if isinstance(case, BatchItems) else capi.Solver(p, case)


def describe(p, case):
    turb = {0: "Euler" if not p.if_viscous else "laminar", 2: "RANS-SA", 3: "RANS-SST"}[int(p.iflag_turbulence_model)]
    scheme = {5: "MUSCL3", 7: "WENO5", 9: "WENO7"}.get(int(p.iflag_scheme), "scheme%d" % p.iflag_scheme)
    flux = {1: "SW", 2: "HLL", 3: "HLLC", 4: "Roe", 5: "VanLeer", 6: "AUSMPW"}[int(p.iflag_flux)]
    tm = "LU-SGS" if p.time_method == 0 else "RK3"
    return "%s %s %s+%s %s" % (case.name, turb, scheme, flux, tm)


def max_over_ranks(value, dist=None, device="cpu"):
    """The slowest rank's time: every rank takes part, every rank gets the maximum."""
    if dist is None:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_rate(world, units_per_rank, ms):
    """Whole-job throughput: the units all ranks processed / the slowest rank's time."""
    return world * units_per_rank / (ms * 1e-3)


def cpu_sample(args, min_seconds=10.0, max_steps=50):
    """Times the CPU oracle (restatement of the reference algorithm, all host threads) on the same
    workload: full mesh, one warm-up step, then steps until min_seconds of CPU work (at most
    max_steps), and one more step on a single host thread.  Returns (cell-updates/s, threads,
    description, the single-thread sample or None)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle_py
    p, case = make_case(args, 0)
    o = oracle_py.OracleCase(p, case)
    o.advance(1)
    n, t0 = 0, time.time()
    while True:
        o.advance(1)
        n += 1
        el = time.time() - t0
        if el >= min_seconds or n >= max_steps:
            break
    threads = oracle_py.threads()
    # one more step of the same (warm) case on a single host thread
    single = None
    if threads > 1:
        oracle_py.set_threads(1)
        t1 = time.time()
        o.advance(1)
        e1 = time.time() - t1
        oracle_py.set_threads(threads)
        single = {"value": case.ncells / e1, "unit": "cell-updates/s", "cores": 1,
                  "sample": "%s, 1 LU-SGS step on 1 host thread after the %d above, %.1f s" % (case.name, n + 1, e1)}
    o.close()
    return case.ncells * n / el, threads, "%s, %d LU-SGS step(s) after 1 warm-up, %.1f s on %d host threads" % (case.name, n, el, threads), single


def event_ms(s, nsteps):
    """Device time (ms) of nsteps steps of handle s, CUDA events on the handle's stream."""
    import torch
    st = torch.cuda.ExternalStream(s.stream())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    s.advance(nsteps)
    e1.record(st)
    e1.synchronize()
    return e0.elapsed_time(e1)


def mixed_leg(args, rank, cl64, cd64):
    """The same workload in mixed precision (FP32 reconstruction / fluxes / sources / metrics, FP64
    state, LU-SGS diagonal, norms, forces): rate and CL / CD error against the FP64 run after the
    same number of steps (1 count = 1e-4)."""
    from ocfd_b200 import capi, cases
    p, case = getattr(cases, args.workload)(precision=1, aoa=rank_aoa(rank))
    s = capi.Solver(p, case)
    s.advance(args.warmup)
    s.synchronize()
    ms = event_ms(s, args.steps)
    _, cl, cd, _ = s.forces()
    s.close()
    return {"value": case.ncells * args.steps / (ms * 1e-3), "unit": "cell-updates/s", "ms_per_step": ms / args.steps,
            "dCL_counts": abs(cl - cl64) * 1e4, "dCD_counts": abs(cd - cd64) * 1e4, "steps": args.warmup + args.steps}


def batch_leg(args, nsteps=100):
    """Config 4: 64 independent 2-D-extruded airfoil solves (O-meshes 129x33 .. 385x97, SA,
    AUSMPW + MUSCL3, mixed precision) in one handle: one step graph covers all 64."""
    from ocfd_b200 import capi, cases
    items = cases.config4_batch(n=64)
    cells = sum(c.ncells for _, c in items)
    b = capi.Batch(items)
    b.advance(args.warmup)
    b.synchronize()
    n = min(args.steps, nsteps)
    ms = event_ms(b, n)
    launches = b.launches_per_step()
    phases = {k: v / 3 for k, v in b.profile(3).items()}   # ms per step, CUDA events on the handle's stream
    lu = (b.lu_kernel_version(), b.lu_tile_width())
    one_launch = b.lu_one_launch()
    b.close()
    # roofline per phase: the phase's algorithmic bytes per cell (mixed, NV = 6) x cells / its time;
    # when both LU-SGS sweeps run as one launch, profile() reports their joint time as the lower one
    peak, peak_kind = peaks()
    bm = dict(BYTES[("mixed", 6)])
    keys = ("residual", "lusgs_lower", "lusgs_upper")
    if one_launch:
        bm["lusgs_both"] = bm["lusgs_lower"] + bm["lusgs_upper"]
        phases = dict(phases)
        phases["lusgs_both"] = phases.pop("lusgs_lower")
        phases.pop("lusgs_upper", None)
        keys = ("residual", "lusgs_both")
    roof = {}
    for k in keys:
        if phases.get(k, 0.0) > 0.0:
            gbs = bm[k] * cells / (phases[k] * 1e-3) / 1e9
            roof[k] = {"bytes_per_cell": bm[k], "achieved_GBps": gbs, "frac": gbs / peak}
    return {"workload": "config4: 64 NACA 4-digit O-mesh airfoils (k=3), SA, AUSMPW+MUSCL3, mixed, seed 1234",
            "cells": cells, "value": cells * n / (ms * 1e-3), "unit": "cell-updates/s", "ms_per_step": ms / n,
            "steps": n, "launches_per_step": launches, "phase_ms_per_step": phases,
            "phase_roofline": roof, "peak_GBps": peak, "peak_kind": peak_kind,
            "lu_kernel": {"version": lu[0], "tile_columns": lu[1], "both_sweeps_one_launch": one_launch}}


def sweep_serving_leg(max_iters=3000, rate=4.0, seed=99):
    """Serving a design sweep: 24 requests, 8 Mach / AoA points (seeded, M in U[0.3, 0.75], AoA in
    U[-2, 6] deg) on each of 3 airfoil meshes (129x33, 257x65, 385x97; SA, AUSMPW + MUSCL3, mixed),
    Poisson arrivals at rate/s, run to the convergence tests of serving_leg.  Two arms: one handle
    per request (Server, up to 32 in flight) and slots of one batch handle per mesh (SlotServer,
    8 slots; a request enters a running batch through ocfd_reset_solve)."""
    import numpy as np
    from ocfd_b200 import cases, serve
    rng = np.random.default_rng(seed)
    items = []
    for ni, nj, m, t in ((129, 33, 0.02, 0.12), (257, 65, 0.0, 0.10), (385, 97, 0.04, 0.14)):
        for _ in range(8):
            items.append(cases.airfoil(ni=ni, nj=nj, m=m, p=0.4, t=t, ma=float(rng.uniform(0.3, 0.75)),
                                       aoa=float(rng.uniform(-2.0, 6.0)), re=6.0e6, scheme=5, flux=6, turb=2, precision=1))
    order = rng.permutation(len(items))
    items = [items[q] for q in order]
    out = {}
    for name, srv in (("handle_per_request", serve.Server(max_active=32, chunk=50)), ("slots_per_mesh", serve.SlotServer(slots=8, chunk=50))):
        reqs = serve.poisson_requests(items, rate=rate, seed=seed, max_iters=max_iters)
        t0 = time.perf_counter()
        res = srv.run(reqs)
        out[name] = serve.summarize(res, time.perf_counter() - t0)
    out["workload"] = "24 requests (8 Mach/AoA points on each of 3 airfoil meshes), Poisson %.1f/s, max %d iterations, mixed" % (rate, max_iters)
    return out


def diverges_at(p, case, max_steps):
    """First iteration whose residual norm is NaN (the solver reports OCFD_ERR_NAN), or None."""
    from ocfd_b200 import capi
    s = capi.Solver(p, case)
    try:
        for it in range(max_steps):
            s.advance(1)
            try:
                s.residual()
            except FloatingPointError:
                return it + 1
        return None
    finally:
        s.close()


def config3_leg(args, nsteps=20):
    """Config 3 (SST wing-body: the swept wing with an ellipsoidal fuselage, 24 uneven blocks,
    ~7.8 M cells, MUSCL3): the stand-in (Roe; LU-SGS CFL 1 in FP64 and mixed, RK3 mixed at CFL 0.5)
    timed over the same steps with the CL / CD error of mixed against FP64 in counts, and the case
    as stated (HLLC + LU-SGS; RK3 at CFL 1.5) run until its residual turns NaN."""
    from ocfd_b200 import capi, cases
    out, forces = {}, {}
    for name, over in (("fp64", dict(precision=0)), ("mixed", dict(precision=1)), ("rk3_mixed", dict(precision=1, time_method=3, cfl=0.5))):
        p, case = cases.config3(**over)
        s = capi.Solver(p, case)
        s.advance(args.warmup)
        s.synchronize()
        ms = event_ms(s, nsteps)
        _, cl, cd, _ = s.forces()
        forces[name] = (cl, cd)
        out[name] = {"value": case.ncells * nsteps / (ms * 1e-3), "unit": "cell-updates/s", "ms_per_step": ms / nsteps}
        s.close()
    out["workload"] = "%s RANS-SST MUSCL3+Roe (stand-in), %d blocks, %d cells, %d steps after %d warm-up" % (
        case.name, len(case.dims), case.ncells, nsteps, args.warmup)
    out["mixed"]["dCL_counts"] = abs(forces["mixed"][0] - forces["fp64"][0]) * 1e4
    out["mixed"]["dCD_counts"] = abs(forces["mixed"][1] - forces["fp64"][1]) * 1e4
    out["mixed"]["speedup_vs_fp64"] = out["fp64"]["ms_per_step"] / out["mixed"]["ms_per_step"]
    p, case = cases.config3_as_specified(precision=0)
    q, case_r = cases.config3_as_specified(rk3=True, precision=0)
    out["as_specified"] = {
        "hllc_lusgs_fp64": {"diverged_at_step": diverges_at(p, case, 30), "of_steps": 30},
        "rk3_cfl1.5_hllc_fp64": {"diverged_at_step": diverges_at(q, case_r, 5), "of_steps": 5},
        "note": "the reference algorithm (HLLC with its v-for-w right star state; explicit RK3 with SST) diverges on this "
                "wing-body in the CPU restatement as well (tests/test_oracle_config3.py); the rates above are the Roe stand-in"}
    return out


def serving_leg(max_iters=5000, n=14, rate=2.0):
    """Continuous batching: Poisson arrivals (rate/s) of seeded airfoil solves (config 4 sizes) and
    reduced swept wings, run to a 1e-6 residual drop or |dCL| < 1e-4 over 200 iterations (at most
    max_iters).  Four arms over the same requests: mixed and FP64, each with up to 32 solves in
    flight and one at a time.  Per arm: p50 / p99 time from arrival to the end of the solve, the
    same over the converged requests only, how many reached the cap, throughput; between the
    precisions (concurrent arms): per-request CL / CD difference over the requests both converged."""
    import numpy as np
    from ocfd_b200 import cases, serve
    def items(precision):
        its = cases.config4_batch(n=n - 2, seed=77, precision=precision)
        its.append(cases.config2_medium(precision=precision, aoa=2.0))
        its.append(cases.config2_small(precision=precision, aoa=4.0))
        return its
    out, res_of = {}, {}
    for name, prec, max_active in (("mixed_concurrent", 1, 32), ("fp64_concurrent", 0, 32),
                                   ("mixed_one_at_a_time", 1, 1), ("fp64_one_at_a_time", 0, 1)):
        reqs = serve.poisson_requests(items(prec), rate=rate, seed=2024, max_iters=max_iters)
        t0 = time.perf_counter()
        res = serve.Server(max_active=max_active, chunk=50).run(reqs)
        out[name] = serve.summarize(res, time.perf_counter() - t0)
        conv = [r.latency for r in res if r.converged in ("residual", "cl")]
        out[name]["converged_p50_s"] = float(np.percentile(conv, 50)) if conv else None
        out[name]["converged_p99_s"] = float(np.percentile(conv, 99)) if conv else None
        res_of[name] = {r.rid: r for r in res}
    both = [q for q in res_of["mixed_concurrent"] if res_of["mixed_concurrent"][q].converged in ("residual", "cl")
            and res_of["fp64_concurrent"][q].converged in ("residual", "cl")]
    dcl = [abs(res_of["mixed_concurrent"][q].cl - res_of["fp64_concurrent"][q].cl) * 1e4 for q in both]
    dcd = [abs(res_of["mixed_concurrent"][q].cd - res_of["fp64_concurrent"][q].cd) * 1e4 for q in both]
    out["mixed_vs_fp64"] = {"requests_converged_in_both": len(both),
                            "dCL_counts_max": max(dcl) if dcl else None, "dCL_counts_median": float(np.median(dcl)) if dcl else None,
                            "dCD_counts_max": max(dcd) if dcd else None,
                            "note": "each arm stops a solve at its own convergence test, so the differences include where each stopped"}
    out["workload"] = "%d requests, Poisson %.1f/s: %d config-4 airfoils + config2_medium + config2_small wings, max %d iterations" % (
        n, rate, n - 2, max_iters)
    return out


def bench_config(p, case, prec, world):
    """The `config` object of the JSON line, the same for both arms of one workload."""
    return {"workload": describe(p, case), "cells": case.ncells, "blocks": len(case.dims), "precision": prec,
            "parallelism": "replicas x%d (independent solves, no collective)" % world,
            "l2": "working set %.1f GB > 126 MB L2 (no flush needed)" % (case.ncells * 1200 / 1e9)}



def converged_leg(args):
    """CL / CD / final-residual error of the mixed form against FP64 at convergence, per
    configuration (1 count = 1e-4), and config 1's FP64 history against the oracle's.
    config 2: both precisions over the configuration's 5000 iterations; config 4: the 64 airfoils
    over 8000 iterations, errors over those whose FP64 CL moved < 0.1 count in the last 400;
    config 3 (stand-in): 1000 iterations; config 1: the FP64 GPU run of 2000 iterations against
    the committed history of the CPU restatement (tests/golden/history_config1.npz)."""
    import numpy as np
    from ocfd_b200 import capi, cases
    out = {}

    def final(p, case, n, chunk=500):
        s = capi.Solver(p, case)
        for _ in range(n // chunk):
            s.advance(chunk)
        _, cl, cd, _ = s.forces()
        rms = s.residual()[1][0]
        s.close()
        return cl, cd, rms

    for name, mk, n in (("config2", cases.config2, 5000), ("config3", cases.config3, 1000)):
        a = final(*mk(precision=0), n)
        b = final(*mk(precision=1), n)
        out[name] = {"iterations": n, "cl_fp64": a[0], "cd_fp64": a[1], "dCL_counts": abs(b[0] - a[0]) * 1e4,
                     "dCD_counts": abs(b[1] - a[1]) * 1e4, "rms_rho_fp64": a[2], "rms_rho_mixed": b[2],
                     "rms_rel_err": abs(b[2] - a[2]) / a[2]}
    hist = {}
    for prec in (0, 1):
        bt = capi.Batch(cases.config4_batch(n=64, precision=prec))
        cl = []
        for _ in range(40):
            bt.advance(200)
            cl.append(bt.forces_all())
        bt.close()
        hist[prec] = cl
    cl64 = np.array([h[1] for h in hist[0]])
    cd64 = np.array([h[2] for h in hist[0]])
    cl32, cd32 = hist[1][-1][1], hist[1][-1][2]
    settled = np.abs(cl64[-1] - cl64[-3]) < 1e-5
    dcl, dcd = np.abs(cl32 - cl64[-1]) * 1e4, np.abs(cd32 - cd64[-1]) * 1e4
    out["config4"] = {"iterations": 8000, "solves": 64, "settled": int(settled.sum()),
                      "dCL_counts_settled_max": float(dcl[settled].max()) if settled.any() else None,
                      "dCD_counts_settled_max": float(dcd[settled].max()) if settled.any() else None,
                      "dCL_counts_all_median": float(np.median(dcl)), "dCL_counts_all_max": float(dcl.max()),
                      "dCD_counts_all_max": float(dcd.max())}
    gd = np.load(os.path.join(ROOT, "tests", "golden", "history_config1.npz"))
    p, case = cases.config1()
    s = capi.Solver(p, case)
    rms, mx, co = [], [], []
    for _ in range(int(gd["steps"])):
        s.advance(1)
        a, b = s.residual()
        rms.append(b[:5])
        mx.append(a[:5])
        co.append(s.forces()[1:3])
    s.close()
    d_rms = np.abs(np.array(rms) - gd["res_rms"][:, :5]) / np.abs(gd["res_rms"][:, :5])
    d_max = np.abs(np.array(mx) - gd["res_max"][:, :5]) / np.abs(gd["res_max"][:, :5])
    d_co = np.abs(np.array(co) - gd["clcdcs"][:, :2])
    bad = np.any(d_rms > 1e-10, axis=1) | np.any(d_max > 1e-10, axis=1)
    out["config1_fp64_vs_oracle"] = {"iterations": int(gd["steps"]), "res_rms_max_rel": float(d_rms.max()),
                                     "res_max_max_rel": float(d_max.max()), "clcd_max_abs": float(d_co.max()),
                                     "first_iteration_beyond_1e-10": int(np.argmax(bad)) + 1 if bad.any() else None}
    return out



def run_reference(args, budget_s=150.0):
    """The reference arm: the CPU restatement of the reference algorithm (oracle/, FP64, all host
    threads) on the same workload, rank 0 only.  Times args.steps full steps, or as many as fit
    in budget_s seconds, after args.warmup warm-up steps."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle_py
    oracle_py.build()
    p, case = make_case(args, 0)
    o = oracle_py.OracleCase(p, case)
    o.advance(args.warmup)
    n, t0 = 0, time.time()
    while n < args.steps:
        o.advance(1)
        n += 1
        if time.time() - t0 > budget_s:
            break
    el = time.time() - t0
    o.close()
    threads = oracle_py.threads()
    v = case.ncells * n / el
    line = {
        "impl": "reference", "metric": "cell-updates/s", "value": v, "unit": "cell-updates/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": el / n * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic (analytic mesh, seeded)",
        "config": bench_config(p, case, "fp64", int(os.environ.get("WORLD_SIZE", "1"))),
        "cpu_baseline": {"value": v, "unit": "cell-updates/s", "cores": threads, "kind": "port",
                         "sample": "full workload, %d of %d steps (%.0f s budget) after %d warm-up on the CPU "
                                   "restatement of the reference (oracle/), %d threads" % (n, args.steps, budget_s, args.warmup, threads)},
        "e2e": {"value": v, "unit": "cell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def shard_main(args):
    """--shard: one config 3 wing-body solve (24 blocks) split over the ranks by whole blocks (the
    reference's automatic partition), each rank's blocks on its GPU, the packed interface halos
    crossing by NCCL send/recv on the handle's stream every step and the norms and forces
    all-reduced (ocfd_create_part).  The total work is fixed: strong scaling.  One rank runs the
    same code path with no peers."""
    import datetime
    import torch
    import torch.distributed as dist
    from ocfd_b200 import build, capi, cases
    from ocfd_b200.shard import ShardedSolver, ThreadComm, TorchComm, partition

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if not os.path.exists(capi.LIB_PATH):
        build.build()
    if world > 1:
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=torch.device("cuda", local))
        comm, d = TorchComm(), dist
    else:
        comm, d = ThreadComm(1).comm(0), None
    prec = args.precision
    p, case = cases.config3(precision=1 if prec == "mixed" else 0)
    owner = partition(case.dims, world)
    s = ShardedSolver(p, case, owner, rank, comm)
    stream = torch.cuda.ExternalStream(s.stream())
    s.advance(args.warmup)
    s.residual()

    def barrier():
        torch.cuda.synchronize()
        if d is not None:
            d.barrier()

    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    with ClockSampler(local) as clk:
        ev0.record(stream)
        s.advance(args.steps)
        ev1.record(stream)
        ev1.synchronize()
    barrier()
    ms = max_over_ranks(ev0.elapsed_time(ev1), d, "cuda")
    value = case.ncells * args.steps / (ms * 1e-3)
    ph = s.profile(3)
    phases = {k: max_over_ranks(v / 3.0, d, "cuda") for k, v in ph.items()}
    rmax, rrms = s.residual()
    _, cl, cd, _ = s.forces()
    # end to end: this rank's blocks' state from pinned host memory, every step advance + norms +
    # forces read back, the state back to the host at the end
    host = [torch.empty(s.state_shape(b), dtype=torch.float64, pin_memory=True).numpy() for b in range(s.nblk)]
    for b in range(s.nblk):
        s.get_state(b, out=host[b])
    e2e_steps = min(args.steps, 50)
    barrier()
    t0 = time.perf_counter()
    for b in range(s.nblk):
        s.set_state(b, host[b])
    for _ in range(e2e_steps):
        s.advance(1)
        s.residual()
        s.forces()
    for b in range(s.nblk):
        s.get_state(b, out=host[b])
    t_e2e = max_over_ranks(time.perf_counter() - t0, d, "cuda")
    state_bytes = sum(h.nbytes for h in host)
    nb = s.nblk
    launches = s.launches_per_step() * args.steps
    s.close()
    if d is not None:
        d.barrier()
        d.destroy_process_group()
    if rank == 0:
        peak, peak_kind = peaks()
        bmodel = BYTES[(prec, int(p.nvar))]
        line = {
            "metric": "cell-updates/s", "value": value, "unit": "cell-updates/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": "f64" if prec == "fp64" else "f32/f64", "data": "synthetic (analytic mesh, seeded)",
            "config": {"workload": describe(p, case) + " block-sharded", "cells": case.ncells, "blocks": len(case.dims),
                       "precision": prec, "blocks_on_rank0": nb,
                       "parallelism": "blocks sharded over %d ranks (packed halos by NCCL send/recv each step; "
                                      "norms and forces all-reduced)" % world,
                       "l2": "working set %.1f GB > 126 MB L2 (no flush needed)" % (case.ncells * 1200 / 1e9)},
            "roofline": {"bound": "hbm", "kernel": "residual phase (slowest rank)", "peak": peak, "peak_kind": peak_kind,
                         "unit": "GB/s", "traffic": None,
                         "achieved": bmodel["residual"] * case.ncells / world / (phases["residual"] * 1e-3) / 1e9,
                         "frac": bmodel["residual"] * case.ncells / world / (phases["residual"] * 1e-3) / 1e9 / peak,
                         "phase_ms_per_step": phases},
            "cpu_baseline": None,
            "e2e": {"value": case.ncells * e2e_steps / t_e2e, "unit": "cell-updates/s", "steps": e2e_steps,
                    "h2d_bytes_per_step": state_bytes / e2e_steps, "d2h_bytes_per_step": state_bytes / e2e_steps + (14 + 9) * 8},
            "gpu_launches": launches, "clocks": clk.summary(), "residual_rms": rrms[: int(p.nvar)].tolist(), "cl": cl, "cd": cd,
        }
        print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--precision", choices=["fp64", "mixed"], default="fp64")
    ap.add_argument("--workload", choices=WORKLOADS, default="config2",
                    help="config2 (the headline case); the others are for profiler captures (config4: the "
                         "64-airfoil batch in one handle)")
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU-baseline sample")
    ap.add_argument("--no-extra", action="store_true", help="skip the mixed-precision, batch and serving legs")
    ap.add_argument("--no-converged", action="store_true", help="skip the runs to convergence (mixed vs FP64 error per config)")
    ap.add_argument("--shard", action="store_true",
                    help="one config 3 wing-body solve split over the ranks by blocks (NCCL halo exchange, strong scaling) "
                         "instead of one replica of the workload per rank")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    if args.shard:
        return shard_main(args)

    import numpy as np
    import torch
    from ocfd_b200 import build, capi

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=torch.device("cuda", local))
    if not os.path.exists(capi.LIB_PATH):
        build.build()

    p, case = make_case(args, rank)
    s = open_solver(p, case)
    stream = torch.cuda.ExternalStream(s.stream())
    s.advance(args.warmup)
    s.residual()
    torch.cuda.synchronize()

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    with ClockSampler(local) as clk:
        ev0.record(stream)
        s.advance(args.steps)
        ev1.record(stream)
        ev1.synchronize()
    barrier()
    ms = max_over_ranks(ev0.elapsed_time(ev1), dist, "cuda")
    rmax, rrms = s.residual()
    _, cl64, cd64, _ = s.forces()
    ncell = case.ncells
    value = aggregate_rate(world, ncell * args.steps, ms)

    # roofline of the dominant kernel.  The LU-SGS sweeps are one launch each (k_lusgs_wave), the
    # residual phase is ~15 launches; the single longest launch is the one reported, timed with
    # CUDA events on the handle's stream over 3 profiled steps.
    ph = s.profile(3)
    peak, peak_kind = peaks()
    prec = args.precision
    bmodel = BYTES[(prec, s.nvar)]
    single = [k for k in ("lusgs_lower", "lusgs_upper") if ph[k] > 0.0]
    dom = max(single, key=lambda k: ph[k]) if single else "residual"
    luv, lutc = s.lu_kernel_version(), s.lu_tile_width()
    one_launch = s.lu_one_launch()
    kernel_name = {"lusgs_lower": "k_lusgs_wave%d<lower, %d columns>" % (luv, lutc),
                   "lusgs_upper": "k_lusgs_wave%d<upper, %d columns>" % (luv, lutc),
                   "residual": "residual phase (all flux/source kernels)"}[dom]
    dom_bytes = bmodel[dom]
    if one_launch and dom == "lusgs_lower":  # both sweeps in one launch: their joint bytes and time
        kernel_name = "k_lusgs_wave4_ul<both sweeps, %d columns>" % lutc
        dom_bytes = bmodel["lusgs_lower"] + bmodel["lusgs_upper"]
    t_dom = ph[dom] / 3.0 * 1e-3
    achieved = dom_bytes * ncell / t_dom / 1e9
    traffic = None
    tfile = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tfile):
        try:
            with open(tfile) as f:
                tj = json.load(f)
            key = "%s/%s" % (prec, dom)
            if one_launch and dom == "lusgs_lower":
                traffic = sum(tj["%s/%s" % (prec, k)]["bytes_per_cell"] for k in ("lusgs_lower", "lusgs_upper")) * ncell
            elif key in tj:
                traffic = tj[key]["bytes_per_cell"] * ncell
        except Exception:
            traffic = None
    roofline = {"bound": "hbm", "kernel": kernel_name, "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_kind": peak_kind, "traffic": traffic, "bytes_per_cell": dom_bytes,
                "launch_ms": t_dom * 1e3, "phase_ms_per_step": {k: v / 3.0 for k, v in ph.items()},
                "residual_phase_GBps": bmodel["residual"] * ncell / (ph["residual"] / 3.0 * 1e-3) / 1e9}

    # end to end through the C-ABI with host buffers: state H2D from pinned memory, then every
    # step advance + residual norms + forces read back (the driver loop with Kstep_show = 1),
    # state D2H at the end
    host = [torch.empty(s.state_shape(b), dtype=torch.float64, pin_memory=True).numpy() for b in range(s.nblk)]
    for b in range(s.nblk):
        s.get_state(b, out=host[b])
    e2e_steps = min(args.steps, 50)
    barrier()
    t0 = time.perf_counter()
    for b in range(s.nblk):
        s.set_state(b, host[b])
    for _ in range(e2e_steps):
        s.advance(1)
        s.residual()
        s.forces()
    for b in range(s.nblk):
        s.get_state(b, out=host[b])
    t_e2e = max_over_ranks((time.perf_counter() - t0) * 1e3, dist, "cuda") * 1e-3
    state_bytes = sum(h.nbytes for h in host)
    e2e = {"value": aggregate_rate(world, ncell * e2e_steps, t_e2e * 1e3), "unit": "cell-updates/s", "steps": e2e_steps,
           "h2d_bytes_per_step": state_bytes / e2e_steps, "d2h_bytes_per_step": state_bytes / e2e_steps + (14 + 9) * 8}
    launches = s.launches_per_step() * args.steps
    s.close()

    extra = {}
    if not args.no_extra and args.precision == "fp64":
        def leg(name, fn, *a):
            # an extra leg that fails is reported in its own key; the headline line still prints
            try:
                extra[name] = fn(*a)
            except Exception as e:  # noqa: BLE001
                extra[name] = {"failed": "%s: %s" % (type(e).__name__, e)}
        leg("mixed", mixed_leg, args, rank, cl64, cd64)
        if "ms_per_step" in extra["mixed"]:
            extra["mixed"]["speedup_vs_fp64"] = (ms / args.steps) / extra["mixed"]["ms_per_step"]
        if world == 1:
            leg("batch", batch_leg, args)
            if "value" in extra["batch"]:  # the mixed batch against the FP64 single-solve rate (target 3x)
                extra["batch"]["vs_fp64_config2"] = extra["batch"]["value"] / value
            leg("config3", config3_leg, args)
            leg("serving", serving_leg)
            leg("sweep_serving", sweep_serving_leg)
            if not args.no_converged:
                leg("converged", converged_leg, args)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        try:
            v, cores, desc, single = cpu_sample(args)
            cpu = {"value": v, "unit": "cell-updates/s", "cores": cores, "kind": "port", "sample": desc}
            if single:
                cpu["single_thread"] = single
        except Exception as e:  # the baseline is reported, never required
            cpu = {"value": None, "unit": "cell-updates/s", "cores": 0, "kind": "port", "sample": "failed: %s" % e}

    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        line = {
            "metric": "cell-updates/s", "value": value, "unit": "cell-updates/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64" if prec == "fp64" else "f32/f64",
            "data": "synthetic (analytic mesh, seeded)",
            "config": bench_config(p, case, prec, world),
            "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches,
            "clocks": clk.summary(), "residual_rms": rrms[: s.nvar].tolist(), "cl": cl64, "cd": cd64,
        }
        line.update(extra)
        print(json.dumps(line), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
