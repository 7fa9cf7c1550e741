"""Benchmark of the fused MR-LBM collide-stream step on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Workload (one "step" = one lattice update of the whole domain): the periodic
Taylor-Green vortex, D3Q27, 256^3 nodes, FP32 moments, Re = 1600, u0 = 0.04,
L = N / 2pi, tau = 1/2 + 3 u0 L / Re (src/cases/taylorGreen/constants.inc,
flow_initialization.inc).  Synthetic: the initial field is the analytic vortex.

Multi-GPU: the path does not shard (one domain per GPU), so N > 1 runs N
independent replicas ("scaling": "weak"); value = all ranks' lattice updates /
the max over ranks of the device time.

--impl reference times the CPU implementation of the same step on the host
cores: the FP64 OpenMP oracle (the reference has no CPU path of its own), on a
bounded sample of the workload.  At N = 1 it also runs the reference's own
CUDA program for this workload once (its sources built for sm_100) and reports
the MLUPS that program prints as the side field `reference_gpu_program`.

Timing: W warm-up steps, then regions of exactly K device-timed steps,
repeated until 0.5 s of timed work has run (so the clock sampler sees it);
ms_per_step is the median region's.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "mr-lbm_b200"))

N = 256
LATTICE = 27
U0 = 0.04
RE = 1600.0
L_TG = N / (2 * np.pi)
TAU = 0.5 + 3.0 * U0 * L_TG / RE
E2E_STEPS = 1000          # the workload's run length
REPORT_EVERY = 100        # kinetic-energy report cadence (taylorGreen/output.inc REPORT_SAVE)
B_ALG = 2 * 10 * 4        # algorithmic bytes per lattice update: 10 FP32 moments read + written
METRIC = "MLUPS (fused MR-LBM step)"
MIN_TIMED_S = 0.5         # timed regions repeat until this much device time has run
MAX_REGIONS = 1000


def workload_config():
    return {"workload": "taylor_green_256^3_d3q%d_fp32" % LATTICE, "grid": [N, N, N], "lattice": "D3Q%d" % LATTICE,
            "storage": "fp32", "re": RE, "u0": U0, "tau": round(TAU, 8), "steps_per_e2e_run": E2E_STEPS,
            "l2": "inputs larger than L2 (2 x 671 MB ping-pong moment buffers)", "parallelism": "replicas"}


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            j = json.load(f)
        return float(j["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profiled_traffic():
    """DRAM bytes per launch of the step kernel from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", "zmarch_step_d3q%d_f32_tgv.md" % LATTICE)
    try:
        for line in open(path):
            if line.startswith("traffic_bytes_per_launch_256:"):
                return float(line.split(":")[1])
    except OSError:
        pass
    return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.samples = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.FIELDS, "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.samples.append([v.strip() for v in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm = [float(s[1]) for s in self.samples if len(s) > 2 and s[1].replace(".", "").isdigit()]
        smax = [float(s[2]) for s in self.samples if len(s) > 2 and s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for s in self.samples:
            for k, nm in enumerate(names):
                if len(s) > 5 + k and s[5 + k].strip().lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(self.samples)}


def dist_setup(gpus):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=120))
        pg = dist
    return world, rank, local, pg


def barrier(pg):
    if pg is not None:
        pg.barrier()


def max_over_ranks(pg, v):
    if pg is None:
        return v
    import torch
    t = torch.tensor([v], dtype=torch.float64)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(pg, v):
    if pg is None:
        return v
    import torch
    t = torch.tensor([v], dtype=torch.float64)
    pg.all_reduce(t, op=pg.ReduceOp.SUM)
    return float(t.item())


def cpu_oracle_mlups(budget_s, n=96, steps_max=40):
    """FP64 OpenMP oracle on an n^3 Taylor-Green sample, same lattice and tau."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_ffi

    z, y, x = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    L = n / (2 * np.pi)
    rho = 1 + (1 / (16 / 3)) * U0 * U0 * (np.cos(2 * x / L) + np.cos(2 * y / L)) * (np.cos(2 * z / L) + 2)
    ux = U0 * np.sin(x / L) * np.cos(y / L) * np.cos(z / L)
    uy = -U0 * np.cos(x / L) * np.sin(y / L) * np.cos(z / L)
    d = oracle_ffi.make_desc(n, n, n, q=LATTICE, tau=TAU)
    o = oracle_ffi.OracleDomain(d)
    o.init_from_macro(rho, ux, uy, np.zeros_like(ux))
    o.step(1)  # warm-up (page faults, thread start)
    t0 = time.perf_counter()
    steps = 0
    while steps < steps_max and (time.perf_counter() - t0) < budget_s:
        o.step(1)
        steps += 1
    dt = time.perf_counter() - t0
    threads = oracle_ffi.lib().orc_threads()
    return steps * n ** 3 / dt / 1e6, threads, "%d^3 D3Q%d Taylor-Green, %d steps, FP64" % (n, LATTICE, steps)


def reference_gpu_program(timeout_s=600):
    """The reference's own CUDA program for this workload (taylorGreen on
    D3Q27 at 256^3, Re 1600, u0 0.04, 1000 steps, KE every 100 steps), built
    for sm_100 from the reference's sources by oracle/build_ref_cuda.sh, run
    once in a scratch folder; its printed MLUPS (src/main.cuh:44-67: CUDA
    events around its whole step loop, report steps included)."""
    import re
    import tempfile

    exe = os.path.join(ROOT, "oracle", "_ref", "refsim_tgv256_q27")
    if not os.path.exists(exe):
        return {"unavailable": "oracle/_ref/refsim_tgv256_q27 not built"}
    with tempfile.TemporaryDirectory(prefix="refsim_") as wd:
        t0 = time.perf_counter()
        try:
            r = subprocess.run([exe], cwd=wd, capture_output=True, text=True, timeout=timeout_s)
        except subprocess.TimeoutExpired:
            return {"unavailable": "timed out after %d s" % timeout_s}
        wall = time.perf_counter() - t0
    m = re.search(r"MLUPS:\s*([0-9.]+)", r.stdout)
    if r.returncode != 0 or not m:
        return {"unavailable": "exit %d, no MLUPS line" % r.returncode}
    return {"value": float(m.group(1)), "unit": "MLUPS", "wall_s": round(wall, 2),
            "what": "the reference's CUDA program (its src/ built for sm_100, taylorGreen D3Q27 256^3, "
                    "1000 steps, KE report every 100), its own MLUPS timer"}


def run_reference_arm(args):
    world, rank, local, pg = dist_setup(args.gpus)
    if rank != 0:
        return 0
    # each of W+K steps is one step of a bounded sample; budget keeps the run to a few minutes
    n = 128
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_ffi
    z, y, x = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    L = n / (2 * np.pi)
    rho = 1 + (1 / (16 / 3)) * U0 * U0 * (np.cos(2 * x / L) + np.cos(2 * y / L)) * (np.cos(2 * z / L) + 2)
    ux = U0 * np.sin(x / L) * np.cos(y / L) * np.cos(z / L)
    uy = -U0 * np.cos(x / L) * np.sin(y / L) * np.cos(z / L)
    o = oracle_ffi.OracleDomain(oracle_ffi.make_desc(n, n, n, q=LATTICE, tau=TAU))
    o.init_from_macro(rho, ux, uy, np.zeros_like(ux))
    o.step(max(args.warmup, 1))
    t0 = time.perf_counter()
    o.step(args.steps)
    dt = time.perf_counter() - t0
    mlups = args.steps * n ** 3 / dt / 1e6
    threads = oracle_ffi.lib().orc_threads()
    sample = "%d^3 D3Q%d Taylor-Green per step (bounded sample of the 256^3 workload), FP64 OpenMP" % (n, LATTICE)
    line = {"impl": "reference", "metric": METRIC, "value": round(mlups, 3), "unit": "MLUPS", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(1e3 * dt / args.steps, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload_config(),
            "cpu_baseline": {"value": round(mlups, 3), "unit": "MLUPS", "cores": threads, "kind": "port",
                             "sample": sample},
            "e2e": {"value": round(mlups, 3), "unit": "MLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    if world == 1 and not args.no_ref_gpu:
        line["reference_gpu_program"] = reference_gpu_program()
    print(json.dumps(line), flush=True)
    return 0


def run_gpu_arm(args):
    import mrlbm

    world, rank, local, pg = dist_setup(args.gpus)
    mrlbm.set_device(local)
    nodes = N ** 3
    d = mrlbm.make_desc(N, N, N, lattice=LATTICE, storage=mrlbm.F32, periodic=(1, 1, 1), tau=TAU)
    dom = mrlbm.Domain(d)
    dom.set_tile_order(bool(args.tile_order))
    dom.init_taylor_green(U0, L_TG)
    # warm-up
    dom.step(max(args.warmup, 3))
    dom.synchronize()
    # device-timed regions of exactly K steps each (CUDA events on the
    # domain's stream), repeated until MIN_TIMED_S of timed work has run so
    # the clock sampler sees the region; ms_per_step is the median region's.
    # Every rank runs the same number of regions (the count is agreed on
    # after the first region).
    reps = []
    with ClockSampler(local) as clk:
        while True:
            barrier(pg)
            dom.synchronize()
            reps.append(dom.time_steps(args.steps))
            dom.synchronize()
            if len(reps) == 1:
                first = max_over_ranks(pg, reps[0])
                nrep = max(1, min(MAX_REGIONS, int(np.ceil(args.min_timed_s * 1e3 / max(first, 1e-6)))))
            if len(reps) >= nrep:
                break
    barrier(pg)
    ms = float(statistics.median(reps))
    ms_max = max_over_ranks(pg, ms)
    total_lups = sum_over_ranks(pg, float(args.steps * nodes))
    value = total_lups / (ms_max * 1e-3) / 1e6
    per_gpu_mlups = args.steps * nodes / (ms * 1e-3) / 1e6

    # roofline of the dominant kernel (the step is the only kernel in the timed region)
    peak, peak_kind = measured_peaks()
    achieved = per_gpu_mlups * 1e6 * B_ALG / 1e9
    traffic = profiled_traffic()

    # end to end through the C ABI with pinned host buffers: upload the initial
    # moments (reference idxMom layout), run the workload's 1000 steps with the
    # kinetic-energy report every 100 steps, download the final moments.
    nm = dom.nm
    host_in = mrlbm.PinnedArray((nm * nodes,))
    host_out = mrlbm.PinnedArray((nm * nodes,))
    host_in.array[:] = dom.moments_ref_layout()
    reports = 0
    barrier(pg)
    dom.synchronize()
    t0 = time.perf_counter()
    dom.set_moments_ref_layout(host_in.array)
    for s in range(0, E2E_STEPS, REPORT_EVERY):
        dom.step(REPORT_EVERY)
        dom.sums()          # FP64 reduction + D2H of the report
        reports += 1
    dom.L.mrlbm_get_moments_ref_layout(dom.h, mrlbm._fp(host_out.array))
    dom.synchronize()
    t_e2e = time.perf_counter() - t0
    barrier(pg)
    t_e2e_max = max_over_ranks(pg, t_e2e)
    e2e_value = sum_over_ranks(pg, float(E2E_STEPS * nodes)) / t_e2e_max / 1e6
    field_bytes = nm * nodes * 4
    h2d = field_bytes / E2E_STEPS
    d2h = (field_bytes + reports * 64) / E2E_STEPS

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        mlups_cpu, threads, sample = cpu_oracle_mlups(budget_s=args.cpu_budget)
        cpu = {"value": round(mlups_cpu, 3), "unit": "MLUPS", "cores": threads, "kind": "port", "sample": sample}

    sums = dom.sums()
    ok = sums["nonfinite"] == 0 and sums["max_speed"] < 0.3
    dom.close()
    host_in.free()
    host_out.free()
    if rank == 0:
        line = {
            "metric": METRIC, "value": round(value, 1), "unit": "MLUPS", "n_gpus": world,
            "steps": args.steps, "warmup": max(args.warmup, 3), "ms_per_step": round(ms_max / args.steps, 5),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (analytic Taylor-Green initial field)", "config": workload_config(),
            "hbm_gbs_algorithmic": round(achieved, 1),
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 4), "peak_kind": peak_kind,
                         "traffic": traffic, "bytes_per_lup_algorithmic": B_ALG,
                         "frac_of_8tbs_nominal": round(achieved / 8000.0, 4)},
            "cpu_baseline": cpu,
            "e2e": {"value": round(e2e_value, 1), "unit": "MLUPS", "h2d_bytes_per_step": round(h2d, 1),
                    "d2h_bytes_per_step": round(d2h, 1), "steps": E2E_STEPS,
                    "what": "H2D initial moments + 1000 steps + FP64 KE report every 100 + D2H final moments"},
            "gpu_launches": args.steps,
            "timed_regions": {"count": len(reps), "steps_each": args.steps,
                              "ms_min": round(min(reps), 4), "ms_median": round(ms, 4), "ms_max": round(max(reps), 4),
                              "what": "each region times exactly K steps; value uses the median region"},
            "clocks": clk.summary(),
            "health": {"finite": bool(sums["nonfinite"] == 0), "max_speed": sums["max_speed"], "ok": bool(ok)},
        }
        print(json.dumps(line), flush=True)
    if pg is not None:
        pg.destroy_process_group()
    return 0


def run_batch_workload(args):
    """256 lid cavities, edges U{24..96} per axis, Re U[50, 1000], lid 0.05,
    advanced together by the persistent batched kernel (graph replay, chunk
    autotuner), against the same cavities solved one at a time with plain
    single-domain launches.  Each member's arithmetic is identical in both
    (bit-identical results, tests/test_gpu_batch.py), so accuracy is equal."""
    import mrlbm

    mrlbm.set_device(0)
    rng = np.random.default_rng(20261203)
    ndom = args.domains
    sizes = rng.integers(24, 97, size=(ndom, 3))
    res = rng.uniform(50.0, 1000.0, size=ndom)
    steps = args.batch_steps
    out = []
    for storage, sname in ((mrlbm.F16, "fp16"), (mrlbm.F32, "fp32")):
        b = mrlbm.Batch(mrlbm.D3Q19, storage)
        mem = []
        for k in range(ndom):
            nx, ny, nz = (int(v) for v in sizes[k])
            d = mrlbm.lid_cavity_desc(nx, re=float(res[k]), lid_u=0.05, storage=storage, ny=ny, nz=nz)
            m = b.add(d)
            m.set_node_types(mrlbm.lid_cavity_node_types(nx, ny, nz, 1))
            m.init_uniform()
            mem.append(m)
        t0 = time.perf_counter()
        b.autotune()
        rows = b.rows()
        t_tune = time.perf_counter() - t0
        for m in mem:
            m.init_uniform()
        info = b.info()
        b.step(16)
        b.synchronize()
        ms = b.time_steps(steps)
        nodes = info["nodes"]
        healthy = all(m.sums()["nonfinite"] == 0 for m in mem)
        # one at a time: each cavity alone, plain launches, per-step time
        # measured over `alone_steps` steps and scaled to the run length
        t_alone = 0.0
        for k in range(ndom):
            nx, ny, nz = (int(v) for v in sizes[k])
            d = mrlbm.lid_cavity_desc(nx, re=float(res[k]), lid_u=0.05, storage=storage, ny=ny, nz=nz)
            dom = mrlbm.Domain(d)
            dom.set_node_types(mrlbm.lid_cavity_node_types(nx, ny, nz, 1))
            dom.init_uniform()
            dom.step(3)
            t_alone += dom.time_steps(args.alone_steps) / args.alone_steps * steps
            dom.close()
        b.close()
        out.append({"storage": sname, "solves_per_s": ndom / (ms * 1e-3), "mlups": nodes * steps / (ms * 1e-3) / 1e6,
                    "ms": ms, "alone_solves_per_s": ndom / (t_alone * 1e-3), "speedup_vs_alone": t_alone / ms,
                    "items": info["items"], "nodes": nodes, "autotune_s": round(t_tune, 2),
                    "tile_rows": rows, "finite": healthy})
    line = {"metric": "batched solves/s (256 lid cavities, %d steps each)" % steps, "value": round(out[0]["solves_per_s"], 3),
            "unit": "solves/s", "n_gpus": 1, "steps": steps, "higher_is_better": True, "dtype": "f16 storage, f32 arithmetic",
            "data": "synthetic (seed 20261203)",
            "config": {"workload": "batched_cavities_256_d3q19", "edges": "U{24..96} per axis", "re": "U[50,1000]",
                       "lid": 0.05, "alone_steps_timed": args.alone_steps},
            "variants": out}
    print(json.dumps(line), flush=True)
    return 0


def serve_requests(rng, count, rate):
    """`count` requests with Poisson arrivals (mean `rate`/s), 50/50 lid
    cavities (Re U[50, 1000]) and power-law ducts (n U[0.6, 1.2], 5 % voxel
    obstacles), edges U{32..192}."""
    import mrlbm

    arrivals = np.cumsum(rng.exponential(1.0 / rate, size=count))
    reqs = []
    for k in range(count):
        n = int(rng.integers(32, 193))
        if rng.random() < 0.5:
            reqs.append(mrlbm.make_request(mrlbm.REQ_LID_CAVITY, n, re=float(rng.uniform(50, 1000))))
        else:
            reqs.append(mrlbm.make_request(mrlbm.REQ_DUCT, n, nnf_n=float(rng.uniform(0.6, 1.2)), solid_fraction=0.05,
                                           seed=int(rng.integers(1 << 62))))
    return reqs, arrivals


def serve_phase(args, reqs, arrivals, storage):
    """The requests through the continuous-batching server, then one at a
    time with plain single-domain launches (a request's latency includes
    building its domain in both); returns the phase's record and the served
    results (steps, final moments)."""
    import mrlbm

    srv = mrlbm.Server(storage=storage, hbm_budget=150e9, max_active=args.max_active, steps_per_tick=100,
                       residual_tol=1e-6, max_steps=args.max_steps, keep_results=True,
                       capacity_nodes=args.serve_capacity)
    t0 = srv.now()
    ids = []
    for r, a in zip(reqs, arrivals):
        r.arrival = t0 + float(a)
        ids.append(srv.submit(r))
    wall0 = time.perf_counter()
    while True:
        active = srv.tick()
        st = srv.stats()
        if active == 0 and st["queued"] == 0:
            break
        if active == 0:
            time.sleep(0.001)  # waiting for the next arrival
    wall = time.perf_counter() - wall0
    stats = srv.stats()
    served = []
    for i, r in zip(ids, reqs):
        res = srv.result(i)
        nm = 11 if r.kind == mrlbm.REQ_DUCT else 10
        served.append((res, srv.moments(i, r.n, nm) if res["status"] == 0 else None))
        srv.release(i)
    srv.close()
    t_alone = 0.0
    lat_alone = []
    clock = 0.0
    for r, a in zip(reqs, arrivals):
        t1 = time.perf_counter()
        dom = mrlbm.request_domain(r, storage)
        dom.residual()
        steps = 0
        while steps < args.max_steps:
            dom.step(100)
            steps += 100
            if dom.residual() <= 1e-6:
                break
        dom.synchronize()
        dt = time.perf_counter() - t1
        dom.close()
        t_alone += dt
        clock = max(clock, float(a)) + dt
        lat_alone.append(clock - float(a))
    steps_done = [res["steps"] for res, _ in served]
    resid = [res["residual"] for res, _ in served]
    rec = {"rate_per_s": None, "requests": len(reqs), "solves_per_s": round(stats["solves_per_s"], 4),
           "p50_latency_s": stats["p50_latency"], "p99_latency_s": stats["p99_latency"],
           "mean_latency_s": stats["mean_latency"], "done": stats["done"], "failed": stats["failed"],
           "wall_s": round(wall, 3), "mlups": stats["lattice_updates"] / wall / 1e6,
           "alone": {"solves_per_s": len(reqs) / t_alone, "p50_latency_s": float(np.percentile(lat_alone, 50)),
                     "p99_latency_s": float(np.percentile(lat_alone, 99))},
           "speedup_vs_alone": (stats["solves_per_s"] / (len(reqs) / t_alone)) if t_alone > 0 else None,
           "steps_per_request": {"min": int(min(steps_done)), "max": int(max(steps_done))},
           "final_residual": {"min": float(min(resid)), "max": float(max(resid))},
           "retired_on_residual": int(sum(1 for s in steps_done if s < args.max_steps))}
    return rec, served


def serve_errors(reqs, served, sample):
    """Relative L2 error of each sampled served velocity field against an FP32
    solve of the same request for the same number of steps (fluid nodes)."""
    import mrlbm

    out = {"lid_cavity": [], "duct": []}
    for k, (r, (res, m)) in enumerate(zip(reqs, served)):
        if m is None or k >= sample:
            continue
        ref = mrlbm.request_domain(r, mrlbm.F32)
        ref.step(res["steps"])
        mr = ref.moments()
        ref.close()
        _, nt = mrlbm.request_describe(r, mrlbm.F32)
        fluid = nt != mrlbm.NODE_SOLID
        du = (m[1:4] - mr[1:4])[:, fluid].astype(np.float64)
        e = float(np.sqrt(np.sum(du * du) / np.sum(mr[1:4][:, fluid].astype(np.float64) ** 2)))
        out["lid_cavity" if r.kind == mrlbm.REQ_LID_CAVITY else "duct"].append(e)
    return {t: {"sampled": len(v), "u_rel_l2_max": max(v) if v else None, "u_rel_l2_mean": float(np.mean(v)) if v else None}
            for t, v in out.items()}


def run_serve_workload(args):
    """Serving (continuous batching) of D3Q19 solves: Poisson arrivals,
    50/50 lid cavities and power-law ducts with 5 % voxel obstacles, edges
    U{32..192}, each until residual <= 1e-6 or --max-steps, HBM budget 150 GB,
    at two loads: the saturating rate (--rate, 200/s by default: offered work
    far above what one GPU does) and a rate below capacity (--rate-low), each
    against the same requests solved one at a time with plain single-domain
    launches.  --serve-capacity limits the nodes running together (0, the
    default: none; 8e6, about one 200^3 domain: large solves run in arrival
    order, small ones share a batch).  Storage --serve-storage
    (split-velocity fp16 by default); the
    accuracy columns compare sampled served velocity fields with FP32 solves
    of the same requests for the same step counts."""
    import mrlbm

    mrlbm.set_device(0)
    storage = {"f16": mrlbm.F16, "f16u": mrlbm.F16U, "f32": mrlbm.F32}[args.serve_storage]
    phases = {}
    for name, rate, count in (("saturated", args.rate, args.requests), ("below_capacity", args.rate_low,
                                                                        args.requests_low)):
        rng = np.random.default_rng(20261203)
        reqs, arrivals = serve_requests(rng, count, rate)
        rec, served = serve_phase(args, reqs, arrivals, storage)
        rec["rate_per_s"] = rate
        rec["accuracy_vs_fp32"] = serve_errors(reqs, served, args.error_sample)
        phases[name] = rec
        del served
    sat = phases["saturated"]
    line = {"metric": "serving solves/s and latency (continuous batching)", "value": sat["solves_per_s"],
            "unit": "solves/s", "n_gpus": 1, "higher_is_better": True,
            "dtype": "%s storage, f32 arithmetic" % args.serve_storage, "data": "synthetic (seed 20261203)",
            "config": {"workload": "serving_poisson_d3q19", "edges": "U{32..192}",
                       "mix": "50/50 lid cavity / power-law duct (5% obstacles)", "residual_tol": 1e-6,
                       "max_steps": args.max_steps, "hbm_budget_gb": 150, "storage": args.serve_storage,
                       "capacity_nodes": args.serve_capacity},
            "phases": phases}
    print(json.dumps(line), flush=True)
    return 0


def moment_errors(a, b, rho0=1.0):
    """Per-moment relative L2 / Linf of a against b (both [moment][...]),
    each normalised by its moment group (rho - rho0 by rho, u components by
    |u|, second moments by the second-moment group), and the relative L2
    error of the velocity vector."""
    groups = {0: [0], 1: [1, 2, 3], 4: [4, 5, 6, 7, 8, 9]}
    gid = {0: 0, 1: 1, 2: 1, 3: 1, 4: 4, 5: 4, 6: 4, 7: 4, 8: 4, 9: 4}
    norms = {}
    for g, ks in groups.items():
        ref = [b[k].astype(np.float64) + (rho0 if k == 0 else 0.0) for k in ks]
        norms[g] = (np.sqrt(sum(float(np.sum(r * r)) for r in ref) / len(ks)),
                    max(float(np.max(np.abs(r))) for r in ref))
    out = {}
    for k in range(10):
        d = a[k].astype(np.float64) - b[k].astype(np.float64)
        n2, ninf = norms[gid[k]]
        out[k] = (float(np.sqrt(np.sum(d * d))) / n2, float(np.max(np.abs(d))) / ninf)
    du = sum(float(np.sum((a[k].astype(np.float64) - b[k].astype(np.float64)) ** 2)) for k in (1, 2, 3))
    uu = sum(float(np.sum(b[k].astype(np.float64) ** 2)) for k in (1, 2, 3))
    return out, float(np.sqrt(du / uu))


def run_thermal_workload(args):
    """Thermal scalar (D3Q19 flow + D3G19 scalar, FP32): the Rayleigh-Benard
    cell of src/cases/rayleighBenard_Periodic scaled to N^3 (hot / cold walls
    in x with the neighbour-flux rule, gravity along x, periodic y and z, Pr 10,
    Ra 1e5), device-timed like the step benchmark, next to the same walled
    flow without the scalar."""
    import mrlbm

    mrlbm.set_device(0)
    n = 256
    tau = 0.55
    nu = (tau - 0.5) / 3
    alpha = nu / 10.0
    gb = 1e5 * alpha * nu / n ** 3
    t = np.zeros((n, n, n), dtype=np.uint32)
    rule = mrlbm.THERMAL_RULE(mrlbm.THERMAL_DIRICHLET_FLUX)
    t[:, :, 0] = mrlbm.WEST | rule | mrlbm.THERMAL_INDEX(0)
    t[:, :, -1] = mrlbm.EAST | rule | mrlbm.THERMAL_INDEX(1)
    out = {}
    for th in (True, False):
        kw = dict(thermal=dict(diffusivity=alpha, reference=1.0, gravity_beta=(gb, 0, 0), wall=(1.5, 0.5))) if th else {}
        d = mrlbm.make_desc(n, n, n, lattice=19, periodic=(0, 1, 1), tau=tau, **kw)
        dom = mrlbm.Domain(d)
        dom.set_node_types(t)
        dom.init_uniform()
        dom.step(max(args.warmup, 3))
        dom.synchronize()
        ms = dom.time_steps(args.steps)
        sums = dom.sums()
        dom.close()
        out["thermal" if th else "flow"] = {"mlups": round(args.steps * n ** 3 / (ms * 1e-3) / 1e6, 1),
                                            "ms_per_step": round(ms / args.steps, 5),
                                            "finite": bool(sums["nonfinite"] == 0)}
    b_alg = 2 * 14 * 4 + 1
    line = {"metric": "MLUPS (fused step with the thermal scalar)", "value": out["thermal"]["mlups"], "unit": "MLUPS",
            "n_gpus": 1, "steps": args.steps, "warmup": max(args.warmup, 3), "higher_is_better": True,
            "dtype": "f32", "data": "synthetic (rest state, hot and cold walls)",
            "config": {"workload": "rayleigh_benard_%d^3_d3q19_d3g19_fp32" % n, "pr": 10, "ra": 1e5,
                       "bytes_per_lup_algorithmic": b_alg},
            "hbm_gbs_algorithmic": round(out["thermal"]["mlups"] * 1e6 * b_alg / 1e9, 1),
            "same_walls_without_scalar": out["flow"], "thermal": out["thermal"]}
    print(json.dumps(line), flush=True)
    return 0


def run_cavity_workload(args):
    """Walled domain: the lid-driven cavity of src/cases/lidDrivenCavity_3D
    (wall classes on all six faces, the lid moving at 0.05, Re 100) at
    --cavity-n^3, D3Q19 by default (--cavity-lattice), FP32, device-timed like
    the step benchmark from the rest state."""
    import mrlbm

    mrlbm.set_device(0)
    n, q = args.cavity_n, args.cavity_lattice
    d = mrlbm.lid_cavity_desc(n, re=100.0, lid_u=0.05, lattice=q)
    dom = mrlbm.Domain(d)
    dom.set_tile_order(bool(args.tile_order))
    dom.set_node_types(mrlbm.lid_cavity_node_types(n, n, n, 1))
    dom.init_uniform()
    dom.step(max(args.warmup, 3))
    dom.synchronize()
    with ClockSampler(0) as clk:
        ms = dom.time_steps(args.steps)
    sums = dom.sums()
    dom.close()
    mlups = args.steps * n ** 3 / (ms * 1e-3) / 1e6
    b_alg = 2 * 10 * 4 + 1  # moments read and written, node class read
    line = {"metric": "MLUPS (fused step, walled domain)", "value": round(mlups, 1), "unit": "MLUPS", "n_gpus": 1,
            "steps": args.steps, "warmup": max(args.warmup, 3), "ms_per_step": round(ms / args.steps, 5),
            "higher_is_better": True, "dtype": "f32", "data": "synthetic (rest state, moving lid)",
            "config": {"workload": "lid_cavity_%d^3_d3q%d_fp32" % (n, q), "re": 100.0, "lid_u": 0.05,
                       "bytes_per_lup_algorithmic": b_alg},
            "hbm_gbs_algorithmic": round(mlups * 1e6 * b_alg / 1e9, 1), "clocks": clk.summary(),
            "finite": bool(sums["nonfinite"] == 0)}
    print(json.dumps(line), flush=True)
    return 0


def run_zslab_workload(args):
    """Z-slab decomposition on one GPU: the benchmark vortex (D3Q27, 256^3,
    FP32) cut into 2 and 4 slabs, each a library domain on its own stream with
    the plane exchange (device copies) after every step, device-timed next to
    the undivided domain.  On one GPU the slabs share the SMs, so this measures
    what the cut and the exchange cost, not multi-GPU scaling; the moments
    after the timed steps are checked equal to the undivided run's."""
    import torch

    import mrlbm
    import zslab

    mrlbm.set_device(0)
    torch.cuda.set_device(0)
    n = 256
    L = n / (2 * np.pi)
    tau = 0.5 + 3.0 * 0.04 * L / 1600.0
    d = mrlbm.make_desc(n, n, n, lattice=27, tau=tau)
    warm = max(args.warmup, 3)
    mono = mrlbm.Domain(d)
    mono.init_taylor_green(0.04, L)
    m0 = mono.moments()
    mono.step(warm)
    mono.synchronize()
    ms = mono.time_steps(args.steps)
    want = mono.moments()
    mono.close()
    out = {"undivided": {"mlups": round(args.steps * n ** 3 / (ms * 1e-3) / 1e6, 1),
                         "ms_per_step": round(ms / args.steps, 5)}}
    for parts in (2, 4):
        zs = zslab.ZSlabDomain.local(d, parts)
        zs.set_moments(m0)
        zs.step(warm)
        zs.synchronize()
        streams = [torch.cuda.ExternalStream(s.dom.get_stream()) for s in zs.slabs]
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(streams[0])
        for st in streams[1:]:
            st.wait_event(e0)
        zs.step(args.steps)
        for st in streams[1:]:
            ev = torch.cuda.Event()
            ev.record(st)
            streams[0].wait_event(ev)
        e1.record(streams[0])
        e1.synchronize()
        ms = e0.elapsed_time(e1)
        p = zs.slabs[0].dom.zplane(mrlbm.ZPLANE_FIRST)
        equal = bool(np.array_equal(zs.moments(), want))
        zs.close()
        out["slabs_%d" % parts] = {"mlups": round(args.steps * n ** 3 / (ms * 1e-3) / 1e6, 1),
                                   "ms_per_step": round(ms / args.steps, 5),
                                   "exchange_bytes_per_step": 2 * parts * p["npairs"] * p["bytes"],
                                   "equal_to_undivided": equal}
    line = {"metric": "MLUPS (z-slab decomposition on one GPU)", "value": out["slabs_4"]["mlups"], "unit": "MLUPS",
            "n_gpus": 1, "steps": args.steps, "warmup": warm, "higher_is_better": True, "dtype": "f32",
            "data": "synthetic (analytic Taylor-Green initial field)",
            "config": {"workload": "taylor_green_256^3_d3q27_fp32_zslabs", "slabs": [2, 4],
                       "l2": "inputs larger than L2"},
            **out}
    print(json.dumps(line), flush=True)
    return 0 if all(v.get("equal_to_undivided", True) for v in out.values()) else 1


def run_precision_workload(args):
    """Storage precision study: the Taylor-Green vortex, D3Q27, n^3 (512 by
    default), Re 1600 (--precision-re), u0 0.04, 1000 steps, with the moments
    stored as FP32, FP16, FP16 with split velocity (F16U) and BF16 (FP32
    arithmetic throughout).  Reports device-timed MLUPS of
    each, and per-moment relative L2 / Linf errors of FP16 / BF16 against FP32
    over the whole field; with --reference (a file written by
    oracle/tgv_reference.py) also every storage against the FP64 oracle on the
    z planes that file holds."""
    import mrlbm

    mrlbm.set_device(0)
    n, steps, re = args.n, args.precision_steps, args.precision_re
    L = n / (2 * np.pi)
    tau = 0.5 + 3.0 * U0 * L / re
    ref = None
    if args.reference:
        ref = np.load(args.reference)
        if int(ref["n"]) != n or int(ref["steps"]) != steps:
            raise SystemExit("reference file is for n=%d, %d steps" % (int(ref["n"]), int(ref["steps"])))
    planes = [int(p) for p in ref["planes"]] if ref is not None else []
    res = {}
    full32 = None
    words = {mrlbm.F32: (10, 4), mrlbm.F16: (10, 2), mrlbm.F16U: (13, 2), mrlbm.BF16: (10, 2)}
    for storage, name in ((mrlbm.F32, "fp32"), (mrlbm.F16, "fp16"), (mrlbm.F16U, "fp16u"), (mrlbm.BF16, "bf16")):
        d = mrlbm.make_desc(n, n, n, lattice=27, storage=storage, tau=tau)
        dom = mrlbm.Domain(d)
        dom.init_taylor_green(U0, L)
        # 3 warm-up steps, then the timed run restarts from the initial state
        m0 = dom.moments()
        dom.step(3)
        dom.set_moments(m0)
        del m0
        with ClockSampler(0) as clk:
            ms = dom.time_steps(steps)
        m = dom.moments()
        r = {"mlups": round(steps * n ** 3 / (ms * 1e-3) / 1e6, 1), "ms": round(ms, 2),
             "bytes_per_lup": 2 * words[storage][0] * words[storage][1], "clocks": clk.summary()}
        if ref is not None:
            o = np.moveaxis(ref["moments"].astype(np.float64), -1, 0)  # [m][planes][y][x]
            e, ue = moment_errors(m[:, planes], o)
            r["vs_fp64_planes"] = {"u_rel_l2": ue, "per_moment": {str(k): [v[0], v[1]] for k, v in e.items()}}
        if storage == mrlbm.F32:
            full32 = m
        else:
            e, ue = moment_errors(m, full32)
            r["vs_fp32_full"] = {"u_rel_l2": ue, "per_moment": {str(k): [v[0], v[1]] for k, v in e.items()}}
        s = dom.sums()
        r["finite"] = bool(s["nonfinite"] == 0)
        del m
        dom.close()
        res[name] = r
    line = {"metric": "storage precision: MLUPS and error vs FP64 (TGV D3Q27)", "value": res["fp16"]["mlups"],
            "unit": "MLUPS", "n_gpus": 1, "steps": steps, "higher_is_better": True,
            "dtype": "fp16/bf16 storage, f32 arithmetic", "data": "synthetic (analytic Taylor-Green initial field)",
            "config": {"workload": "taylor_green_%d^3_d3q27_precision" % n, "re": re, "u0": U0, "tau": tau,
                       "reference": ("FP64 oracle, z planes %s" % planes) if ref is not None else None},
            "fp16_over_fp32": round(res["fp16"]["mlups"] / res["fp32"]["mlups"], 3),
            "bf16_over_fp32": round(res["bf16"]["mlups"] / res["fp32"]["mlups"], 3),
            "fp16u_over_fp32": round(res["fp16u"]["mlups"] / res["fp32"]["mlups"], 3),
            "storages": res}
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000, help="timed steps (2000 at 256^3: about 0.8 s, long enough for several clock samples)")
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--min-timed-s", type=float, default=MIN_TIMED_S,
                    help="repeat the K-step timed region until this much device time has run (0: one region)")
    ap.add_argument("--no-ref-gpu", action="store_true",
                    help="reference arm: skip the side run of the reference's own CUDA program")
    ap.add_argument("--cpu-budget", type=float, default=15.0)
    ap.add_argument("--workload", default="tgv",
                    choices=["tgv", "batch", "serve", "precision", "thermal", "zslab", "cavity"],
                    help="tgv: the headline step benchmark (default); batch / serve / precision / thermal / zslab / "
                         "cavity: the batched-cavity, serving, storage-precision, thermal-scalar, z-slab and "
                         "walled-cavity workloads (run on their own)")
    ap.add_argument("--lattice", type=int, default=27, choices=[19, 27],
                    help="tgv workload: velocity set (D3Q27 is the benchmark's; D3Q19 for comparison)")
    ap.add_argument("--n", type=int, default=512, help="precision workload: grid edge")
    ap.add_argument("--precision-steps", type=int, default=1000)
    ap.add_argument("--precision-re", type=float, default=RE)
    ap.add_argument("--reference", default=None, help="precision workload: FP64 planes from oracle/tgv_reference.py")
    ap.add_argument("--cavity-n", type=int, default=128, help="cavity workload: grid edge")
    ap.add_argument("--tile-order", type=int, default=1, choices=[0, 1],
                    help="vortex and cavity workloads: overlapped tile-ordered steps (1) or whole-launch order (0)")
    ap.add_argument("--cavity-lattice", type=int, default=19, choices=[19, 27])
    ap.add_argument("--domains", type=int, default=256)
    ap.add_argument("--batch-steps", type=int, default=5000)
    ap.add_argument("--alone-steps", type=int, default=200)
    ap.add_argument("--requests", type=int, default=32)
    ap.add_argument("--rate", type=float, default=200.0)
    ap.add_argument("--rate-low", type=float, default=0.1, help="serving: the below-capacity arrival rate")
    ap.add_argument("--requests-low", type=int, default=12)
    ap.add_argument("--serve-storage", default="f16u", choices=["f16", "f16u", "f32"])
    ap.add_argument("--error-sample", type=int, default=8, help="serving: requests compared with an FP32 solve")
    ap.add_argument("--serve-capacity", type=float, default=0.0,
                    help="serving: lattice nodes the running solves may hold together (0, the default: every "
                         "arrived request shares the GPU; 8e6: large solves in arrival order)")
    ap.add_argument("--max-active", type=int, default=512)
    ap.add_argument("--max-steps", type=int, default=20000)
    args = ap.parse_args()
    global LATTICE
    LATTICE = args.lattice
    if args.impl == "reference":
        return run_reference_arm(args)
    if args.workload == "batch":
        return run_batch_workload(args)
    if args.workload == "serve":
        return run_serve_workload(args)
    if args.workload == "precision":
        return run_precision_workload(args)
    if args.workload == "thermal":
        return run_thermal_workload(args)
    if args.workload == "zslab":
        return run_zslab_workload(args)
    if args.workload == "cavity":
        return run_cavity_workload(args)
    return run_gpu_arm(args)


if __name__ == "__main__":
    sys.exit(main())
