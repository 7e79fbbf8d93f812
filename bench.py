"""Benchmark: particle-updates/s of the full SPH + gravity KDK step, Evrard
collapse N = 1,048,576 on one B200, mixed FP32/FP64 vs plain FP64.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One step = kick + drift, Morton sort + octree, h search (N_ngb = 64 +- 5),
density + EOS, Barnes-Hut gravity (theta = 0.5, eps = 0.01), hydro
acceleration + du/dt, kick + u update + FP64 energy sums -- the loop body of
the reference's serial driver (sph_code/sph_serial.py:142-193).  Inputs are
seeded synthetic Evrard ICs (the reference's IC files are not available).

Multi-GPU: the path runs independent replicas (one Evrard system per rank);
value = total particles x steps / max over ranks of the timed region.

--impl reference times the reference's CPU algorithm (the C restatement of
sph_code/libsx.py in oracle/, all host threads) on a bounded row sample of
the same workload; rank 0 only.

--clouds K replaces the single cloud by a batched ensemble of K independent
Evrard clouds (N log-uniform in [2048, 65536]) stepped by one launch
sequence.  The roofline of the dominant kernel (the gravity walk, FP32-pipe
bound) is taken against the FP32 rate measured on the same GPU in the same
run (sph3_probe_fp32_rate).
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_DEFAULT = 1048576
DT = 1e-3


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--n", type=int, default=N_DEFAULT)
    p.add_argument("--no-fp64", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-cpu", action="store_true")
    p.add_argument("--leaf", type=int, default=0)
    p.add_argument("--clouds", type=int, default=0,
                   help="batched ensemble instead of one cloud: this many independent Evrard clouds, N "
                        "log-uniform in [2048, 65536], M and R uniform in [0.5, 2] (--n is ignored; no CPU "
                        "baseline)")
    p.add_argument("--set", action="append", default=[], metavar="KEY=VALUE",
                   help="override a Config field of the timed context (repeatable), e.g. --set stack_cap=1024")
    return p.parse_args()


# ------------------------------------------------------------ clocks
class Clocks:
    """nvidia-smi samples (200 ms) while the timed region runs."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for k, nm in enumerate(names):
                if f[5 + k].lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------------ CPU baseline
def cpu_rows_time(ic, rows, n_ngb=64):
    """Wall time of the reference CPU algorithm (oracle C restatement, all
    threads) for the given rows: h search, density, direct gravity,
    hydro acceleration and du/dt, each an all-N loop per row."""
    import oracle as oc
    pos, m = ic["pos"], ic["m"]
    n = pos.shape[0]
    eps = np.full(n, 0.01)
    h = ic["h"]
    u = ic["u"]
    gama = 5.0 / 3.0
    t0 = time.perf_counter()
    oc.h_smooth_rows(pos, h, rows, n_ngb=n_ngb, tol=5, max_iter=2000)
    oc.density_rows(pos, m, h, rows)
    oc.grav_direct_rows(pos, m, 1.0, eps, rows)
    rho = ic["rho"]
    P = (gama - 1.0) * rho * u
    c = np.sqrt(gama * (gama - 1.0) * u)
    oc.hydro_rows(pos, ic["vel"], rho, P, c, h, m, 0, 1.0, 2.0, 0.1, rows=rows, want_dudt=False)
    oc.hydro_rows(pos, ic["vel"], rho, P, c, h, m, 0, 1.0, 2.0, 0.1, rows=rows, want_acc=False)
    return time.perf_counter() - t0


def rows_for(ic, target_s, rng, threads):
    """Rows whose CPU pass takes about target_s: a call has a fixed cost
    (O(N) set-up of the derived arrays, thread start) of a few tenths of a
    second, so the per-row cost is measured twice, the second time on a
    sample large enough for that cost to be small."""
    n = ic["pos"].shape[0]
    k = min(n, max(4 * threads, 64))
    t = cpu_rows_time(ic, rng.choice(n, k, replace=False))
    k2 = int(min(n, max(k, 0.25 * target_s * k / max(t, 1e-9))))
    if k2 > k:
        t2 = cpu_rows_time(ic, rng.choice(n, k2, replace=False))
        per_row = max(t2 - t * 0.5, 0.5 * t2) / k2  # discount part of the fixed cost
    else:
        per_row = t / k
    return int(min(n, max(k, target_s / max(per_row, 1e-9))))


def cpu_baseline(ic, target_s=12.0):
    import oracle as oc
    oc.build()
    threads = oc.num_threads()
    rng = np.random.default_rng(123)
    n = ic["pos"].shape[0]
    nrows = rows_for(ic, target_s, rng, threads)
    rows = rng.choice(n, nrows, replace=False)
    t = cpu_rows_time(ic, rows)
    return {"value": nrows / t, "unit": "particle-updates/s", "cores": threads, "kind": "port",
            "sample": "%d random rows x all %d particles of the N=%d Evrard step (h search, density, "
                      "direct gravity, hydro accel, du/dt), %.1f s wall; extrapolated per particle" %
                      (nrows, n, n, t)}


# ------------------------------------------------------------ GPU arm
# DRAM bytes per particle of one gravity launch, from the ncu capture
# summarised in profiles/k_gravity_f32_evrard262k.md (14.07 MB at N=262144)
GRAV_DRAM_BYTES_PER_PARTICLE = 14.07e6 / 262144


def make_ic(n, seed, clouds=0):
    from sph_3_b200.ic import evrard, evrard_batch
    if clouds:
        return evrard_batch(ncloud=clouds, seed=seed, n_min=2048, n_max=65536)
    return evrard(n, seed=seed)


def run_ours(args, rank, world, local_rank):
    import torch
    from sph_3_b200 import Config, Context, costs

    torch.cuda.set_device(local_rank)
    # a real stream: torch's legacy default stream has handle 0, which the C
    # ABI reads as "the context's own stream"
    bench_stream = torch.cuda.Stream()
    torch.cuda.set_stream(bench_stream)
    dist = world > 1
    if dist:
        import torch.distributed as td
    ic = make_ic(args.n, seed=rank, clouds=args.clouds)
    n = len(ic["m"])
    counts = ic.get("counts")
    eps = np.full(n, 0.01)

    def setup(prec, timing=False):
        cfg = Config(precision=prec, timing=timing)
        if args.leaf:
            cfg = cfg.replace(leaf_size=args.leaf)
        for kv in args.set:
            k, v = kv.split("=", 1)
            cur = getattr(cfg, k)
            cfg = cfg.replace(**{k: type(cur)(v) if not isinstance(cur, bool) else v.lower() in ("1", "true")})
        ctx = Context(cfg, device=local_rank)
        if counts is not None:
            ctx.set_clouds(counts)
        ctx.set_particles(ic["pos"], ic["m"], vel=ic["vel"], u=ic["u"], eps=eps)
        ctx.first_step(DT)
        return ctx

    def timed(ctx, steps, warmup):
        stream = torch.cuda.current_stream()
        sp = stream.cuda_stream
        ctx.step(DT, warmup, stream=sp)
        torch.cuda.synchronize()
        if dist:
            td.barrier()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        ctx.step(DT, steps, stream=sp)
        e1.record(stream)
        torch.cuda.synchronize()
        if dist:
            td.barrier()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        if dist:
            t = torch.tensor([ms], device="cuda")
            td.all_reduce(t, op=td.ReduceOp.MAX)
            ms = float(t.item())
        return ms

    # ---- mixed (headline)
    ctx = setup("mixed")
    free_b, total_b = torch.cuda.mem_get_info()
    clocks = Clocks(local_rank)
    e_start = ctx.energy()
    clocks.start()
    ms = timed(ctx, args.steps, args.warmup)
    ck = clocks.stop()
    kernels_per_step = ctx.kernels_per_step()
    e_end = ctx.energy()
    status = ctx.status_names()
    ctx.counters(clear=True)
    ms_step = ms / args.steps
    value = world * n * args.steps / (ms / 1e3)

    # ---- per-phase times and counters (events between phases, no graph)
    ctx.set_config(ctx.config.replace(timing=True))
    ctx.phase_times(clear=True)
    ctx.counters(clear=True)
    kphase = max(3, min(args.steps, 8))
    ctx.step(DT, kphase)
    ph = {k: v / kphase for k, v in ctx.phase_times().items()}
    raw = ctx.counters()
    # tree sizes are set by the last build and the walk maxima are maxima, not sums
    cnt = {k: (v if k in ("tree_nodes", "walk_max_iter") else v / kphase) for k, v in raw.items()
           if k != "walk_max_where"}
    cnt["mean_group_size"] = n / max(cnt.get("grav_groups", 0), 1)
    ctx.set_config(ctx.config.replace(timing=False))

    # ---- e2e through host buffers (pinned), C ABI per step
    e2e = None
    if not args.no_e2e:
        fields = ["pos", "vel", "u", "h", "acc", "dudt_prev"]
        host = {f: torch.from_numpy(ctx.get_field(f)).pin_memory() for f in fields}
        outs = {f: torch.empty_like(host[f]).pin_memory() for f in fields}
        bytes_in = sum(host[f].numel() * 8 for f in fields)
        k_e2e = max(2, min(args.steps, 5))

        def e2e_step():
            for f in fields:
                ctx.set_field(f, host[f])
            ctx.step(DT, 1)
            for f in fields:
                ctx.get_field(f, out=outs[f])

        e2e_step()
        torch.cuda.synchronize()
        if dist:
            td.barrier()
        t0 = time.perf_counter()
        for _ in range(k_e2e):
            e2e_step()
        torch.cuda.synchronize()
        dt_e2e = time.perf_counter() - t0
        if dist:
            t = torch.tensor([dt_e2e], device="cuda")
            td.all_reduce(t, op=td.ReduceOp.MAX)
            dt_e2e = float(t.item())
        e2e = {"value": world * n * k_e2e / dt_e2e, "unit": "particle-updates/s",
               "h2d_bytes_per_step": int(bytes_in), "d2h_bytes_per_step": int(bytes_in),
               "ms_per_step": 1e3 * dt_e2e / k_e2e,
               "path": "sph3_set_field x6 (pinned host) -> sph3_step -> sph3_get_field x6"}
    ctx.close()

    # ---- FP64 path, same code
    fp64 = None
    if not args.no_fp64:
        c64 = setup("fp64")
        ms64 = timed(c64, max(3, args.steps // 2), max(2, args.warmup // 2))
        k64 = max(3, args.steps // 2)
        fp64 = {"value": world * n * k64 / (ms64 / 1e3), "ms_per_step": ms64 / k64,
                "status": c64.status_names()}
        c64.close()

    # ---- roofline of the dominant kernel
    g_flops = (cnt.get("grav_node", 0) * costs.GRAV_NODE_QUAD + cnt.get("grav_part", 0) * costs.GRAV_PART)
    kernels = {}
    peaks = {}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            peaks = json.load(fh)
    except OSError:
        pass
    hbm_peak = float(peaks.get("hbm_gbs", 6650.0))
    hbm_src = "measured (MEASURED_PEAKS.json hbm_gbs)" if "hbm_gbs" in peaks else "fallback 6650 GB/s"
    sm_mhz = ck.get("sm_mhz") or 1965.0
    fp32_nominal = 148 * 128 * 2 * sm_mhz * 1e6 / 1e12
    try:  # measured on this GPU: packed-FP32 FMA chains on every SM
        from sph_3_b200 import _lib
        fp32_peak = _lib.probe_fp32_rate(local_rank, ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
        fp32_src = ("measured on this GPU: %.1f TFLOP/s of packed FP32 FMA chains (sph3_probe_fp32_rate); "
                    "nominal at the sampled %.0f MHz: %.1f" % (fp32_peak, sm_mhz, fp32_nominal))
    except Exception as exc:  # noqa: BLE001 - report the nominal rate instead
        fp32_peak = fp32_nominal
        fp32_src = ("nominal FP32 issue rate 148 SM x 128 lanes x 2 at the sampled median SM clock (%.0f MHz); "
                    "the probe failed: %s" % (sm_mhz, exc))
    for k, msv in ph.items():
        bytes_alg = costs.BYTES.get(k, 0) * n
        kernels[k] = {"ms": msv, "share": msv / max(sum(ph.values()), 1e-9),
                      "algorithmic_GBps": bytes_alg / (msv / 1e3) / 1e9 if msv > 0 else None}
    dom = max(ph, key=lambda k: ph[k])
    if dom == "gravity":
        ach = g_flops / (ph["gravity"] / 1e3) / 1e12
        roof = {"kernel": "k_gravity_f32<QUAD>", "bound": "fp32", "achieved": ach, "peak": fp32_peak,
                "unit": "TFLOP/s", "frac": ach / fp32_peak,
                "traffic": GRAV_DRAM_BYTES_PER_PARTICLE * n,
                "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one N=262144 launch "
                                  "(14.07 MB), scaled per particle to this N "
                                  "(profiles/k_gravity_f32_evrard262k.md)",
                "peak_source": fp32_src + "; MEASURED_PEAKS.json has no CUDA-core FP32 figure",
                "work": "%.3g node + %.3g particle interactions per launch" % (cnt.get("grav_node", 0),
                                                                               cnt.get("grav_part", 0))}
    else:
        bytes_alg = costs.BYTES.get(dom, 0) * n
        ach = bytes_alg / (ph[dom] / 1e3) / 1e9
        roof = {"kernel": dom, "bound": "hbm", "achieved": ach, "peak": hbm_peak, "unit": "GB/s",
                "frac": ach / hbm_peak, "traffic": None, "peak_source": hbm_src}

    cpu = None
    if rank == 0 and not args.no_cpu and not args.clouds:
        # CPU reference needs rho for the hydro rows: use the GPU's FP64 state
        icb = dict(ic)
        c2 = Context(Config(precision="fp64", gravity=False), device=local_rank)
        c2.set_particles(ic["pos"], ic["m"], vel=ic["vel"], u=ic["u"])
        c2.compute("boot_h", "h", "density")
        icb["h"] = c2.get_field("h")
        icb["rho"] = c2.get_field("rho")
        c2.close()
        cpu = cpu_baseline(icb)

    drift = abs((e_end["E"] - e_start["E"]) / e_start["E"]) if e_start["E"] != 0 else None
    line = {
        "metric": ("particle-updates/sec per SPH+gravity step at N=1M (mixed FP32/FP64)" if not args.clouds else
                   "particle-updates/sec per SPH+gravity step, batched Evrard ensemble (mixed FP32/FP64)"),
        "value": value,
        "unit": "particle-updates/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms_step,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32 pair arithmetic, f64 state/accumulators",
        "data": "synthetic seeded Evrard ICs (r = sqrt(U), isotropic, equal mass)",
        "config": {"workload": ("Evrard collapse N=%d, N_ngb=64, theta=0.5, eps=0.01, dt=1e-3, one full "
                                "KDK step per update" % n) if not args.clouds else
                               ("batched ensemble of %d independent Evrard clouds (N=%d in total, each N "
                                "log-uniform in [2048, 65536]), N_ngb=64, theta=0.5, eps=0.01, dt=1e-3, one "
                                "full KDK step of every cloud per update, one launch sequence" % (args.clouds, n)),
                   "n_per_gpu": n, "parallelism": "replicas",
                   "l2": "working set ~0.5 GB per GPU > 126 MB L2 (no flush needed)",
                   "cuda_graph": True, "overrides": list(args.set)},
        "fp64": fp64,
        "mixed_over_fp64": (value / fp64["value"]) if fp64 else None,
        "energy_drift_timed_region": drift,
        "status": status,
        "e2e": e2e,
        "roofline": roof,
        "kernels": kernels,
        "counters_per_step": cnt,
        "clocks": ck,
        "gpu_launches": kernels_per_step * args.steps if kernels_per_step > 0 else None,
        "gpu_launches_per_step": kernels_per_step,
        "device_bytes_in_use": int(total_b - free_b),
        "cpu_baseline": cpu,
    }
    return line


def run_reference(args, rank, world):
    if rank != 0:
        return None
    n = args.n
    ic = make_ic(n, seed=0)
    import oracle as oc
    oc.build()
    threads = oc.num_threads()
    rng = np.random.default_rng(7)
    # h from a kd-free bootstrap on a subsample is not needed: the CPU loop
    # cost does not depend on the h values beyond the iteration count
    ic["h"] = np.full(n, 0.5 * (64.0 / n) ** (1.0 / 3.0) * 1.2)
    ic["rho"] = np.full(n, 1.0)
    rows_per_step = rows_for(ic, 4.0, rng, threads)
    for _ in range(args.warmup):
        cpu_rows_time(ic, rng.choice(n, max(threads, rows_per_step // 8), replace=False))
    t_tot = 0.0
    rows_tot = 0
    for _ in range(args.steps):
        rows = rng.choice(n, rows_per_step, replace=False)
        t_tot += cpu_rows_time(ic, rows)
        rows_tot += rows.size
    value = rows_tot / t_tot
    return {
        "impl": "reference",
        "metric": "particle-updates/sec per SPH+gravity step at N=1M (mixed FP32/FP64)",
        "value": value, "unit": "particle-updates/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * n / value, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic seeded Evrard ICs",
        "config": {"workload": "Evrard collapse N=%d, N_ngb=64, one full step per update" % n},
        "cpu_baseline": {"value": value, "unit": "particle-updates/s", "cores": threads, "kind": "port",
                         "sample": "%d random rows x all %d particles per step (h search, density, direct "
                                   "gravity, hydro accel, du/dt), extrapolated per particle" %
                                   (rows_per_step, n)},
        "e2e": {"value": value, "unit": "particle-updates/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1 and args.impl == "ours":
        import datetime

        import torch
        import torch.distributed as td
        torch.cuda.set_device(local_rank)
        td.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    if args.impl == "reference":
        line = run_reference(args, rank, world)
    else:
        line = run_ours(args, rank, world, local_rank)
    if rank == 0 and line is not None:
        print(json.dumps(line), flush=True)
    if world > 1 and args.impl == "ours":
        import torch.distributed as td
        td.destroy_process_group()


if __name__ == "__main__":
    main()
