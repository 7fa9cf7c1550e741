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
bounded sample of the workload.
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


def workload_config():
    return {"workload": "taylor_green_256^3_d3q27_fp32", "grid": [N, N, N], "lattice": "D3Q27",
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
    path = os.path.join(ROOT, "profiles", "zmarch_step_d3q27_f32_tgv.md")
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
    return steps * n ** 3 / dt / 1e6, threads, "%d^3 D3Q27 Taylor-Green, %d steps, FP64" % (n, steps)


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
    sample = "%d^3 D3Q27 Taylor-Green per step (bounded sample of the 256^3 workload), FP64 OpenMP" % n
    line = {"impl": "reference", "metric": METRIC, "value": round(mlups, 3), "unit": "MLUPS", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(1e3 * dt / args.steps, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload_config(),
            "cpu_baseline": {"value": round(mlups, 3), "unit": "MLUPS", "cores": threads, "kind": "port",
                             "sample": sample},
            "e2e": {"value": round(mlups, 3), "unit": "MLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def run_gpu_arm(args):
    import mrlbm

    world, rank, local, pg = dist_setup(args.gpus)
    mrlbm.set_device(local)
    nodes = N ** 3
    d = mrlbm.make_desc(N, N, N, lattice=LATTICE, storage=mrlbm.F32, periodic=(1, 1, 1), tau=TAU)
    dom = mrlbm.Domain(d)
    dom.init_taylor_green(U0, L_TG)
    # warm-up
    dom.step(max(args.warmup, 3))
    dom.synchronize()
    # device-timed K steps (CUDA events on the domain's stream)
    barrier(pg)
    dom.synchronize()
    with ClockSampler(local) as clk:
        ms = dom.time_steps(args.steps)
    dom.synchronize()
    barrier(pg)
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
            "clocks": clk.summary(),
            "health": {"finite": bool(sums["nonfinite"] == 0), "max_speed": sums["max_speed"], "ok": bool(ok)},
        }
        print(json.dumps(line), flush=True)
    if pg is not None:
        pg.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-budget", type=float, default=15.0)
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference_arm(args)
    return run_gpu_arm(args)


if __name__ == "__main__":
    sys.exit(main())
