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
    p.add_argument("--steps", type=int, default=50)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--n", type=int, default=N_DEFAULT)
    p.add_argument("--no-fp64", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-cpu", action="store_true")
    p.add_argument("--no-errors", action="store_true")
    p.add_argument("--no-ensemble", action="store_true")
    p.add_argument("--no-cooling", action="store_true")
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
    """SM clock and throttle-reason samples while the timed region runs: NVML
    every 10 ms from a thread (nvidia-smi at 200 ms if NVML is missing)."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    NAMES = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")

    def __init__(self, index, period_s=0.01):
        self.index = index
        self.period = period_s
        self.proc = None
        self.nvml = None
        self.samples = []  # (sm_mhz, sm_max_mhz, set of reason names)
        self.lines = []
        self._stop = threading.Event()

    def start(self):
        try:
            import pynvml
            pynvml.nvmlInit()
            self.nvml = pynvml
            self.h = pynvml.nvmlDeviceGetHandleByIndex(self.index)
            self.smax = float(pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM))
            self.bits = {"hw_slowdown": pynvml.nvmlClocksEventReasonHwSlowdown,
                         "hw_thermal_slowdown": pynvml.nvmlClocksEventReasonHwThermalSlowdown,
                         "sw_thermal_slowdown": pynvml.nvmlClocksEventReasonSwThermalSlowdown,
                         "sw_power_cap": pynvml.nvmlClocksEventReasonSwPowerCap}
            self.t = threading.Thread(target=self._poll, daemon=True)
            self.t.start()
            return
        except Exception:  # noqa: BLE001 - fall back to nvidia-smi
            self.nvml = None
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _poll(self):
        pn = self.nvml
        while not self._stop.is_set():
            try:
                sm = float(pn.nvmlDeviceGetClockInfo(self.h, pn.NVML_CLOCK_SM))
                r = int(pn.nvmlDeviceGetCurrentClocksEventReasons(self.h))
                self.samples.append((sm, self.smax, {k for k, b in self.bits.items() if r & b}))
            except Exception:  # noqa: BLE001
                pass
            self._stop.wait(self.period)

    def _read(self):
        for line in self.proc.stdout:
            f = [x.strip() for x in line.strip().split(",")]
            if len(f) < 9:
                continue
            try:
                self.samples.append((float(f[1]), float(f[2]),
                                     {nm for k, nm in enumerate(self.NAMES) if f[5 + k].lower().startswith("active")}))
            except ValueError:
                continue

    def stop(self):
        self._stop.set()
        if self.nvml is not None:
            self.t.join(timeout=2)
            src = "nvml, %d ms" % round(self.period * 1e3)
        elif self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            src = "nvidia-smi, 200 ms"
        else:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no clock source"], "samples": 0}
        sm = [x[0] for x in self.samples]
        reasons = set()
        for x in self.samples:
            reasons |= x[2]
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_min_mhz": float(np.min(sm)) if sm else None,
                "sm_max_mhz": self.samples[-1][1] if self.samples else None,
                "reasons": sorted(reasons), "samples": len(sm), "source": src}


# ------------------------------------------------------------ CPU baseline
WORKLOAD = ("Evrard collapse N=%d, N_ngb=64, theta=0.5, eps=0.01, dt=1e-3, one full KDK step per update")


def cpu_state(n, seed=0, n_ngb=64):
    """The CPU measurements' shared, untimed set-up (both arms use it): the
    Evrard ICs and, since an O(N^2) h search over all N particles is out of
    reach on the host, h and rho from the profile's expected number density
    n(r) = N / (2 pi r) (M = R = 1): h = 0.5 (3 N_ngb / (4 pi n(r)))^(1/3),
    rho = n(r) / N.  The per-row cost of the reference's loops does not depend
    on these values except through the h search's iteration count, which
    cpu_rows_time settles before timing."""
    from sph_3_b200.ic import evrard
    ic = evrard(n, seed=seed)
    r = np.maximum(np.linalg.norm(ic["pos"], axis=1), 1e-6)
    nd = n / (2.0 * np.pi * r)
    ic["h"] = 0.5 * (3.0 * n_ngb / (4.0 * np.pi * nd)) ** (1.0 / 3.0)
    ic["rho"] = nd / n
    return ic


def cpu_rows_time(ic, rows, n_ngb=64):
    """Wall time of the reference CPU algorithm (oracle C restatement, all
    threads) for the given rows: h search, density, direct gravity,
    hydro acceleration and du/dt, each an all-N loop per row.  Before the
    clock starts, the rows' h is brought into the window (untimed), as the
    driver's loop calls the h search with the previous step's h."""
    import oracle as oc
    pos, m = ic["pos"], ic["m"]
    n = pos.shape[0]
    eps = np.full(n, 0.01)
    h = ic["h"].copy()
    h[rows] = oc.h_smooth_rows(pos, h, rows, n_ngb=n_ngb, tol=5, max_iter=2000)[0]
    u = ic["u"]
    gama = 5.0 / 3.0
    rho = ic["rho"]
    P = (gama - 1.0) * rho * u
    c = np.sqrt(gama * (gama - 1.0) * u)
    t0 = time.perf_counter()
    oc.h_smooth_rows(pos, h, rows, n_ngb=n_ngb, tol=5, max_iter=2000)
    oc.density_rows(pos, m, h, rows)
    oc.grav_direct_rows(pos, m, 1.0, eps, rows)
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


def cpu_sample_desc(nrows, n, secs):
    return ("%d random rows x all %d particles of the N=%d Evrard step (h search from an in-window h, density, "
            "direct gravity, hydro accel, du/dt), %.1f s wall; rows / time = particle-updates/s" %
            (nrows, n, n, secs))


def cpu_baseline(n, target_s=12.0):
    import oracle as oc
    oc.build()
    threads = oc.num_threads()
    ic = cpu_state(n)
    rng = np.random.default_rng(123)
    nrows = rows_for(ic, target_s, rng, threads)
    rows = rng.choice(n, nrows, replace=False)
    t = cpu_rows_time(ic, rows)
    return {"value": nrows / t, "unit": "particle-updates/s", "cores": threads, "kind": "port",
            "sample": cpu_sample_desc(nrows, n, t)}


# ------------------------------------------------------------ GPU arm
# DRAM bytes per particle of one gravity launch, from an ncu capture of the
# step's gravity walk at N=524288 (dram__bytes_read.sum + dram__bytes_write.sum
# = 31.12 + 1.79 MB)
GRAV_DRAM_BYTES_PER_PARTICLE = 32.78e6 / 524288


def make_ic(n, seed, clouds=0):
    from sph_3_b200.ic import evrard, evrard_batch
    if clouds:
        return evrard_batch(ncloud=clouds, seed=seed, n_min=2048, n_max=65536)
    return evrard(n, seed=seed)


def stated_errors(ctx, n, grav_rows=4096, sph_rows=256):
    """Errors of the mixed path stated beside the throughput, measured on the
    benchmark's own state after the timed steps (outside the timed region):
    Barnes-Hut gravity against the FP64 direct sum (GPU, sph3_gravity_direct_rows)
    on grav_rows random particles; density, hydro acceleration and du/dt
    recomputed at the current state against the oracle (the reference's FP64
    formulas on the host) on sph_rows random particles, with the GPU's own h,
    and for the hydro terms its own rho, P, c."""
    import oracle as oc
    rng = np.random.default_rng(99)
    rows = rng.choice(n, grav_rows, replace=False)
    acc = ctx.get_field("acc_g")[rows]
    ref, _ = ctx.gravity_direct_rows(rows)
    eg = np.linalg.norm(acc - ref, axis=1) / np.linalg.norm(ref, axis=1)
    ctx.compute("density", "acc_sph", "dudt")
    f = {k: ctx.get_field(k) for k in ("pos", "vel", "m", "h", "rho", "P", "c", "acc_sph", "dudt")}
    r2 = rng.choice(n, sph_rows, replace=False)
    rho = oc.density_rows(f["pos"], f["m"], f["h"], r2)
    erho = np.abs(f["rho"][r2] - rho) / rho
    a, du = oc.hydro_rows(f["pos"], f["vel"], f["rho"], f["P"], f["c"], f["h"], f["m"], rows=r2)
    ea = np.linalg.norm(f["acc_sph"][r2] - a, axis=1) / np.linalg.norm(a, axis=1)
    edu = np.abs(f["dudt"][r2] - du) / np.maximum(np.abs(du), 1e-6 * np.sqrt(np.mean(du ** 2)))

    def stats(e):
        return {"median": float(np.median(e)), "p95": float(np.percentile(e, 95)),
                "p99": float(np.percentile(e, 99)), "max": float(np.max(e))}

    return {"gravity_bh_theta0.5_vs_fp64_direct": dict(stats(eg), rows=int(grav_rows), bound_median=1e-3),
            "density_vs_oracle": dict(stats(erho), rows=int(sph_rows), bound_max=1e-5),
            "hydro_accel_vs_oracle": dict(stats(ea), rows=int(sph_rows)),
            "dudt_vs_oracle": dict(stats(edu), rows=int(sph_rows)),
            "how": "after the timed steps, outside the timed region; relative errors per particle "
                   "(vector norm for accelerations)"}


def run_ensemble(args, local_rank, timed, world, ncloud=256):
    """The batched-ensemble workload: ncloud Evrard clouds, N log-uniform in
    [2048, 65536], M and R in [0.5, 2], one launch sequence per pass, walk
    parameters from the autotuner (cached per workload shape), mixed and
    FP64 step times."""
    from sph_3_b200 import Config, Context, autotune
    from sph_3_b200.ic import evrard_batch
    b = evrard_batch(ncloud=ncloud, seed=0, n_min=2048, n_max=65536)
    nt = int(b["counts"].sum())
    out = {"workload": "%d independent Evrard clouds, N log-uniform in [2048, 65536] (N=%d in total), "
                       "M, R uniform in [0.5, 2], one full KDK step of every cloud per update" % (ncloud, nt),
           "n_total": nt}
    for prec in ("mixed", "fp64"):
        ctx = Context(Config(precision=prec), device=local_rank)
        ctx.set_clouds(b["counts"])
        ctx.set_particles(b["pos"], b["m"], vel=b["vel"], u=b["u"])
        ctx.first_step(DT)
        if prec == "mixed":
            best, times = autotune.autotune(ctx, steps=3, warmup=2,
                                            grid={"leaf_size": (8, 12, 16, 24), "walk_warps": (2, 4, 8),
                                                  "stack_cap": (768,)})
            out["autotuned"] = best
        k = 10 if prec == "mixed" else 4
        ms = timed(ctx, k, 3)
        out[prec] = {"ms_per_step": ms / k, "value": world * nt * k / (ms / 1e3), "status": ctx.status_names()}
        ctx.close()
    out["mixed_over_fp64"] = out["mixed"]["value"] / out["fp64"]["value"]
    return out


def run_cooling(local_rank, n=4194304, k=20):
    """The heating/cooling step (hcoolingZ) on n float particles resident on
    the GPU (inputs of 76 B per particle, 319 MB at the default n: larger than
    L2), with a seeded table of the reference's layout: ms per launch and the
    algorithmic bytes per particle (typ, u, rho, x, y, z read; u and N_M ion
    fractions written) against the HBM peak."""
    import torch
    from sph_3_b200 import cooling
    dev = torch.device("cuda", local_rank)
    tab = cooling.seeded_table(seed=0)
    t = cooling.CoolTable(tab, device=local_rank)
    units = cooling.Units(unit_density_cgs=1e-24, unit_time_s=3e13, unit_u_cgs=1e12, unit_length_cm=3.086e21)
    g = torch.Generator(device=dev).manual_seed(1)
    xyz = tuple(torch.rand(n, device=dev, generator=g) * 4 - 2 for _ in range(3))
    rho = 10.0 ** (torch.rand(n, device=dev, generator=g) * 8 - 4)
    u0 = 10.0 ** (torch.rand(n, device=dev, generator=g) * 6 - 3)
    typ = torch.zeros(n, dtype=torch.int32, device=dev)
    u = u0.clone()
    for _ in range(3):
        u.copy_(u0)
        cooling.hcooling(t, units, DT, u, rho, xyz, typ=typ)
    torch.cuda.synchronize()
    # each launch cools fresh energies (the copy is outside the timed events)
    ms = 0.0
    st = torch.cuda.current_stream()
    for _ in range(k):
        u.copy_(u0)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(st)
        cooling.hcooling(t, units, DT, u, rho, xyz, typ=typ)
        e1.record(st)
        torch.cuda.synchronize()
        ms += e0.elapsed_time(e1)
    ms /= k
    nm = int(tab["dims"][4])
    per = 4 * 6 + 4 + 4 * nm
    t.close()
    return {"workload": "hcoolingZ over %d gas particles (float), seeded table dims %s (N_kpc, N_T, N_nH, N_Z, "
                        "N_M, N_t)" % (n, list(int(d) for d in tab["dims"])),
            "ms_per_launch": ms, "particles_per_s": n / (ms / 1e3),
            "algorithmic_bytes_per_particle": per, "algorithmic_GBps": per * n / (ms / 1e3) / 1e9}


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
        # the reference loop's state (sph_serial.py:142-193 keeps r, v, acc, h,
        # u, ut_previous as host arrays): in from and out to page-locked host
        # buffers every step, through the one C-ABI call that overlaps the
        # transfers with the step (sph3_step_io)
        fields = ["pos", "vel", "u", "h", "acc", "dudt_prev"]
        host = {f: torch.from_numpy(ctx.get_field(f)).pin_memory() for f in fields}
        outs = {f: torch.empty_like(host[f]).pin_memory() for f in fields}
        bytes_in = sum(host[f].numel() * 8 for f in fields)
        k_e2e = max(3, min(args.steps, 10))

        def e2e_step():
            ctx.step_io(DT, host, outs)

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
               "path": "sph3_step_io: 6 fields in from page-locked host buffers, one KDK step, 6 fields out, "
                       "transfers on two copy streams overlapping the step"}
    errors = None
    if not args.no_errors and rank == 0:
        errors = stated_errors(ctx, n)
    ctx.close()

    # ---- FP64 path, same code
    fp64 = None
    if not args.no_fp64:
        c64 = setup("fp64")
        k64 = max(3, args.steps // 4)
        ms64 = timed(c64, k64, max(3, args.warmup // 2))
        fp64 = {"value": world * n * k64 / (ms64 / 1e3), "ms_per_step": ms64 / k64,
                "status": c64.status_names()}
        # per-phase FP64 times (events between phases, no graph), as for the mixed path
        c64.set_config(c64.config.replace(timing=True))
        c64.phase_times(clear=True)
        c64.step(DT, 3)
        fp64["kernels_ms"] = {k: v / 3 for k, v in c64.phase_times().items()}
        c64.close()

    # ---- batched ensemble (256 clouds), autotuned, in the same process
    ensemble = None
    if not args.no_ensemble and not args.clouds:
        ensemble = run_ensemble(args, local_rank, timed, world)

    # ---- the heating/cooling step on its own (not part of the Evrard step)
    cool = None
    if not args.no_cooling and not args.clouds:
        cool = run_cooling(local_rank)

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
    if cool is not None:
        cool["frac_of_hbm_peak"] = cool["algorithmic_GBps"] / hbm_peak
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
        roof = {"kernel": "k_gravity_f32<QUAD, no potential>", "bound": "fp32", "achieved": ach, "peak": fp32_peak,
                "unit": "TFLOP/s", "frac": ach / fp32_peak,
                "traffic": GRAV_DRAM_BYTES_PER_PARTICLE * n,
                "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one N=524288 launch "
                                  "(32.78 MB), scaled per particle to this N",
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
        cpu = cpu_baseline(n)

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
        "config": {"workload": (WORKLOAD % n) if not args.clouds else
                               ("batched ensemble of %d independent Evrard clouds (N=%d in total, each N "
                                "log-uniform in [2048, 65536]), N_ngb=64, theta=0.5, eps=0.01, dt=1e-3, one "
                                "full KDK step of every cloud per update, one launch sequence" % (args.clouds, n)),
                   "n_per_gpu": n, "parallelism": "replicas",
                   "l2": "working set ~0.5 GB per GPU > 126 MB L2 (no flush needed)"},
        "run": {"cuda_graph": True, "overrides": list(args.set)},
        "fp64": fp64,
        "mixed_over_fp64": (value / fp64["value"]) if fp64 else None,
        "mixed_over_fp64_per_phase": ({k: fp64["kernels_ms"][k] / v for k, v in ph.items() if v > 0}
                                      if fp64 else None),
        "errors": errors,
        "ensemble": ensemble,
        "cooling": cool,
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
    """The reference's CPU algorithm (the oracle's C restatement of
    sph_code/libsx.py, all host threads) on the same workload: each step is a
    bounded sample of rows of the N = 1M step, timed whole; value = rows
    processed / time."""
    if rank != 0:
        return None
    n = args.n
    import oracle as oc
    oc.build()
    threads = oc.num_threads()
    ic = cpu_state(n)
    rng = np.random.default_rng(7)
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
        "warmup": args.warmup, "ms_per_step": 1e3 * t_tot / args.steps,
        "ms_per_full_step_extrapolated": 1e3 * n / value, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic seeded Evrard ICs (r = sqrt(U), isotropic, equal mass)",
        "config": {"workload": WORKLOAD % n, "n_per_gpu": n, "parallelism": "replicas",
                   "l2": "working set ~0.5 GB per GPU > 126 MB L2 (no flush needed)"},
        "cpu_baseline": {"value": value, "unit": "particle-updates/s", "cores": threads, "kind": "port",
                         "sample": "each step: " + cpu_sample_desc(rows_per_step, n, t_tot / args.steps)},
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
