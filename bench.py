"""Benchmark of the B200 lattice update (multiphaseLB per-timestep path).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload NAME]

Default workload: the thermal van der Waals column, D2Q9, 128 x 512 nodes,
liMRT flow + liTempMRT heat, bounce-back / fixedT walls, FP64, on the fused
box path.  One step = one time step of the whole lattice.  The lattice state
(~21 MB) fits in L2, so a 256 MiB buffer is written between timed steps and
each step is timed alone with CUDA events on the library's stream.  The
other named workloads (D3Q15 bubble 192^3, D2Q9 bubble 256^2) follow under
"extra", device-timed the same way, FP64 and FP32-deviation.  On one GPU,
"time_to_equilibrium" compares the plain FP64 path with the batched
FP32-deviation + warm-start + filter form on a seeded bubble ensemble.

For N > 1 (torchrun, one process per GPU) every rank advances its own
replica of the workload (weak scaling; the path has no exchange step on one
domain), and the time is the max over ranks.

Prints one JSON line (rank 0).
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
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "GLUPS on 1 B200 (FP64 vs FP32-dev); time-to-equilibrium w/ warm start"

# Algorithmic bytes per lattice-node update: every population read once and
# written once, plus per-node state that cannot be rebuilt from the
# populations (the heat-source history S: read + write, kept FP64).
# bytes_per_lup: FP64 storage; bytes_per_lup32: FP32-deviation storage.
WORKLOADS = {
    "column_d2q9_128x512": dict(bytes_per_lup=304, bytes_per_lup32=160,
                                desc="thermal VdW column, D2Q9, f+g, bounceBack+fixedT walls, periodic x",
                                eos="van der Waals a=9/392, b=2/21, R=1, T0=0.85 Tc, fixedT walls 0.86/0.84 Tc, "
                                    "g=-1e-5: the stated a=9/49 makes psi NaN at 0.85 Tc (p - rho/3 > 0 in the "
                                    "vapour; the reference's own solver gives NaN); a=9/392 keeps T/Tc, rho_c and "
                                    "the coexistence densities",
                                build=lambda c: c.column_case(128, 512)),
    "bubble_d2q9_256": dict(bytes_per_lup=144, bytes_per_lup32=72, desc="static bubble, D2Q9 liMRT, fully periodic",
                            eos="Carnahan-Starling a=1, b=4, R=1, T=0.8 Tc, G=-1, vapour disc R=40, tanh width 5",
                            build=lambda c: c.bubble_case(0, 256, 40.0, 5.0, 0.8)),
    "bubble_d3q15_192": dict(bytes_per_lup=240, bytes_per_lup32=120, desc="static bubble, D3Q15 xuMRT, fully periodic",
                             eos="Carnahan-Starling a=1, b=4, R=1, T=0.75 Tc, G=-1, vapour sphere R=48, tanh width 5",
                             build=lambda c: c.bubble_case(1, 192, 48.0, 5.0, 0.75)),
}
# timed after the named workload in a default run (device time, FP64 and FP32-deviation)
EXTRA_WORKLOADS = ("bubble_d3q15_192", "bubble_d2q9_256")
PROFILE_TRAFFIC = {  # (workload, kernel) -> ncu summary under profiles/ holding the per-launch DRAM bytes
    ("column_d2q9_128x512", "k_fused_d2q9"): "k_fused_d2q9_column_128x512.txt",
    ("bubble_d2q9_256", "k_fused_d2q9"): "k_fused_d2q9_bubble_256.txt",
    ("bubble_d3q15_192", "k_fused_d3q15"): "k_fused_d3q15_bubble.txt",
    ("bubble_d3q15_192", "k_fused_d3q15_tma"): "k_fused_d3q15_tma_bubble_192.txt",
}
FALLBACK_HBM_GBS = 6650.0


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def profiled_traffic(workload, kernel, tile_config=-1):
    """DRAM bytes per launch of the step kernel from the committed ncu summary:
    the line for this tile candidate (dram_bytes_per_full_launch_cfgN) where
    the summary has one, else its only figure."""
    name = PROFILE_TRAFFIC.get((workload, kernel))
    if not name:
        return None
    path = os.path.join(ROOT, "profiles", name)
    found = {}
    try:
        for line in open(path):
            if line.startswith("dram_bytes_per_full_launch"):
                key, val = line.split(":", 1)
                found[key.strip()] = float(val.split()[0])
    except OSError:
        return None
    return found.get(f"dram_bytes_per_full_launch_cfg{tile_config}", found.get("dram_bytes_per_full_launch"))


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                self.rows.append(parts)

    def mark(self):
        return len(self.rows)

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self, start=0):
        rows = self.rows[start:] or self.rows
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch.distributed as dist
        import datetime
        backend = "nccl" if os.environ.get("MPLB_BENCH_BACKEND", "nccl") == "nccl" else "gloo"
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return world, rank, local


def max_over_ranks(x, world, device):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world, device):
    if world > 1:
        import torch.distributed as dist
        dist.barrier(device_ids=[device.index] if device.type == "cuda" else None)


# --------------------------------------------------------------- CPU baseline
def _cpu_worker(args):
    """One single-core reference run of `steps` steps on the workload (spawned process)."""
    workload, steps, kind = args
    sys.path.insert(0, ROOT)
    from multiphaselb_b200 import cases
    from oracle.oracle import Checker
    case = WORKLOADS[workload]["build"](cases)
    k = Checker(kind, case)
    k.upload_case()
    k.initialize()
    t0 = time.perf_counter()
    k.step(steps)
    dt = time.perf_counter() - t0
    return case.n * steps, dt


def cpu_baseline(workload, steps, procs):
    """Reference CPU solver (oracle/_ref, single-threaded like the reference)
    on `procs` host cores, each running an independent copy for `steps` steps."""
    from oracle import oracle as orc
    kind = "ref" if orc.available("ref") else "port"
    if not orc.available(kind):
        orc.build(kind)
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    t0 = time.perf_counter()
    if procs == 1:
        res = [_cpu_worker((workload, steps, kind))]
    else:
        with ctx.Pool(procs) as pool:
            res = pool.map(_cpu_worker, [(workload, steps, kind)] * procs)
    wall = time.perf_counter() - t0
    lups = sum(r[0] for r in res)
    slowest = max(r[1] for r in res)
    return dict(value=lups / slowest / 1e9, unit="GLUPS", cores=procs, step_ms=slowest / max(steps, 1) * 1e3,
                kind="reference" if kind == "ref" else "port",
                sample=f"{steps} steps of the full {WORKLOADS[workload]['desc']} lattice per core, "
                       f"{procs} independent single-threaded copies (the reference has no threads; its "
                       f"parallelism is MPI ranks, absent here); wall {wall:.1f}s")


# -------------------------------------------------------------------- our arm
def measure(case, path, precision, steps, warmup, local, stream, flush, world, dev):
    """Warm-up, then `steps` steps each timed alone after an L2 flush (CUDA
    events on the library's stream, clocks sampled meanwhile); then the same
    steps back to back (informational)."""
    import torch
    from multiphaselb_b200 import Lattice
    with torch.cuda.stream(stream):
        lat = Lattice(case, path=path, device=local, stream=stream.cuda_stream, precision=precision)
        lat.upload_case()
        lat.initialize()
        info0 = lat.info()
        for _ in range(warmup):
            lat.step(1)
        torch.cuda.synchronize()
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        barrier(world, dev)
        torch.cuda.synchronize()
        with ClockSampler(local) as clk:
            time.sleep(0.3)
            mark = clk.mark()
            launches0 = lat.info()["kernel_launches"]
            for i in range(steps):
                flush.zero_()
                ev[i][0].record(stream)
                lat.step(1)
                ev[i][1].record(stream)
            torch.cuda.synchronize()
            launches = lat.info()["kernel_launches"] - launches0
            time.sleep(0.25)
            clocks = clk.summary(mark)
        s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s0.record(stream)
        lat.step(steps)
        s1.record(stream)
        torch.cuda.synchronize()
        steady_ms = s0.elapsed_time(s1) / steps
        barrier(world, dev)
        step_ms = [st.elapsed_time(en) for st, en in ev]
        info = lat.info()
        lat.close()
    return dict(step_ms=step_ms, steady_ms=steady_ms, launches=launches, clocks=clocks, info=info, info0=info0)


def kernel_name(case, precision, tile_config=-1):
    """The step kernel the autotuner picked (3D candidates 6 to 9 are the TMA-staged kernel)."""
    from multiphaselb_b200 import abi
    if precision == abi.FP32_DEV:
        return "k_fused32_d2q9" if case.lattice == abi.D2Q9 else "k_fused32_d3q15"
    if case.lattice == abi.D2Q9:
        return "k_fused_d2q9"
    return "k_fused_d3q15_tma" if tile_config in (6, 7, 8, 9) else "k_fused_d3q15"


def time_to_equilibrium(ncases):
    """Seeded static-bubble ensemble (D2Q9 CS, L in 64..512, T/Tc in [0.6, 0.95],
    R in [8, 0.3 L]) to max |drho/dt| < 1e-9 over 1000 steps: the plain FP64
    path (lone handles one after another) against the accelerated form
    (FP32-deviation lattices in one batch, learned warm start, time-averaging
    filter windows of two sound crossing times).  Wall seconds of the stepping
    on the host clock around device-synchronised runs, set-up excluded."""
    from multiphaselb_b200 import abi, ensemble, warmstart
    specs = ensemble.draw(ncases)
    plain = ensemble.run_plain(specs, 1000, 1e-9, 400000)
    init = warmstart.initializer(abi.D2Q9)
    filt = (2.0, 2000, 4000)
    acc = ensemble.run_batched(specs, 1000, 1e-9, 400000, init, filt=filt)
    c = ensemble.compare(acc, plain)
    return {"cases": ncases, "tol": 1e-9, "check_interval": 1000,
            "plain_fp64_s": round(c["plain_wall_s"], 3), "accelerated_s": round(c["batched_wall_s"], 3),
            "ratio": round(c["speedup"], 3), "target_ratio": 5.0,
            "plain_steps": c["plain_steps"], "accelerated_steps": c["batched_steps"],
            "converged": f"{acc['converged']}/{ncases}", "warm_started": acc["warm_started"],
            "max_rel_coexistence": c["max_rel_coexistence"], "within_1e-3": f"{c['within_1e3']}/{c['compared']}",
            "accelerated_form": "batched FP32-deviation + learned warm start (tcgen05 inference) + "
                                f"time-averaging filter (scale {filt[0]}, first {filt[1]}, every {filt[2]})",
            "data": f"ensemble.draw({ncases}), seeded; plain = FP64 fused path, tanh/Maxwell start"}


def run_ours(a):
    import torch
    from multiphaselb_b200 import PATH_AUTO, PATH_FUSED, PATH_OPERATORS, Lattice, abi, cases
    world, rank, local = dist_setup()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    path = {"auto": PATH_AUTO, "fused": PATH_FUSED, "operators": PATH_OPERATORS}[a.path]
    stream = torch.cuda.Stream(device=dev)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)  # 256 MiB > 126 MB L2
    peak, peak_kind = peaks()
    peak_source = f"{peak_kind} MEASURED_PEAKS hbm_gbs" if peak_kind == "measured" else "fallback 6.65 TB/s"

    def device_line(name, steps):
        """FP64 and FP32-deviation device timings of one workload."""
        wl = WORKLOADS[name]
        case = wl["build"](cases)
        r64 = measure(case, path, abi.FP64, steps, a.warmup, local, stream, flush, world, dev)
        total_ms = max_over_ranks(sum(r64["step_ms"]), world, dev)
        kernel_ms = sum(r64["step_ms"]) / len(r64["step_ms"])  # one fused launch per step
        achieved = wl["bytes_per_lup"] * case.n / (kernel_ms * 1e-3) / 1e9
        kname = kernel_name(case, abi.FP64, r64["info"]["tile_config"])
        out = {
            "case": case, "r64": r64, "total_ms": total_ms,
            "value": round(case.n * steps * world / (total_ms * 1e-3) / 1e9, 4),
            "ms_per_step": round(total_ms / steps, 6),
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 4), "peak_source": peak_source,
                         "traffic": profiled_traffic(name, kname, r64["info"]["tile_config"]), "kernel": kname,
                         "kernel_ms": round(kernel_ms, 6)},
        }
        if not a.no_fp32:
            r32 = measure(case, path, abi.FP32_DEV, steps, a.warmup, local, stream, flush, world, dev)
            ms32 = max_over_ranks(sum(r32["step_ms"]), world, dev) / steps
            ach32 = wl["bytes_per_lup32"] * case.n / (sum(r32["step_ms"]) / steps * 1e-3) / 1e9
            out["fp32_dev"] = {"value": round(case.n * world / (ms32 * 1e-3) / 1e9, 4), "unit": "GLUPS",
                               "ms_per_step": round(ms32, 6), "bytes_per_lup": wl["bytes_per_lup32"],
                               "roofline_frac": round(ach32 / peak, 4), "kernel": kernel_name(case, abi.FP32_DEV),
                               "steady_state_glups": round(case.n / (r32["steady_ms"] * 1e-3) / 1e9, 4),
                               "launches": int(r32["launches"]),
                               "note": "same workload, FP32-deviation storage (not bit-identical to FP64; "
                                       "its error against FP64 is measured by multiphaselb_b200.accuracy)"}
        return out

    head = device_line(a.workload, a.steps)
    case, wl, r64 = head["case"], WORKLOADS[a.workload], head["r64"]
    info, info0 = r64["info"], r64["info0"]
    launches = {"fp64_timed_steps": int(r64["launches"]), "fp32_dev_timed_steps": int(head.get("fp32_dev", {}).get("launches", 0))}

    # end to end through the C-ABI: pinned host fields -> device, steps, all fields back
    n, Q = case.n, case.Q
    pin = lambda shape: torch.empty(shape, dtype=torch.float64, pin_memory=True).numpy()  # noqa: E731
    h_rho, h_U, h_T = pin((n,)), pin((n, 3)), pin((n,))
    h_rho[:], h_U[:], h_T[:] = case.rho, case.U, case.T
    out = dict(rho=pin((n,)), U=pin((n, 3)), T=pin((n,)), Fi=pin((n, 3)), Ft=pin((n, 3)), S=pin((n,)),
               f=pin((n, Q)), g=pin((n, Q)))
    e2e_steps = a.steps
    with torch.cuda.stream(stream):
        lat = Lattice(case, path=path, device=local, stream=stream.cuda_stream)
        lat.upload(rho=h_rho, U=h_U, T=h_T)
        lat.initialize()
        lat.step(a.warmup)
        lat.download(out)
        barrier(world, dev)
        torch.cuda.synchronize()
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        k0 = lat.info()["kernel_launches"]
        t0.record(stream)
        lat.upload(rho=h_rho, U=h_U, T=h_T)
        lat.initialize()
        lat.step(e2e_steps)
        lat.download(out)
        t1.record(stream)
        torch.cuda.synchronize()
        launches["e2e"] = int(lat.info()["kernel_launches"] - k0)
        e2e_ms = max_over_ranks(t0.elapsed_time(t1), world, dev)
        lat.close()
    h2d = n * (1 + 3 + 1) * 8
    d2h = n * (1 + 3 + 1 + 3 + 3 + 1 + Q + (Q if case.g is not None else Q)) * 8

    # the same run from nothing: handle creation (mesh tables to the device)
    # and the tile autotuner at the first step included (host wall clock;
    # informational, what a drop-in driver's first run of a lattice pays)
    torch.cuda.synchronize()
    w0 = time.perf_counter()
    with torch.cuda.stream(stream):
        lat = Lattice(case, path=path, device=local, stream=stream.cuda_stream)
        lat.upload(rho=h_rho, U=h_U, T=h_T)
        lat.initialize()
        lat.step(e2e_steps)
        lat.download(out)
        lat.close()
    torch.cuda.synchronize()
    cold_s = time.perf_counter() - w0

    line = {
        "metric": METRIC, "value": head["value"], "unit": "GLUPS", "n_gpus": world,
        "steps": a.steps, "warmup": a.warmup, "ms_per_step": head["ms_per_step"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded lattice of the named shape; no dataset)",
        "config": {"workload": a.workload, "desc": wl["desc"], "eos": wl["eos"], "nodes_per_gpu": n,
                   "path": {0: "auto", 1: "operators", 2: "fused"}[path] + f" -> {['', 'operators', 'fused'][info0['path']]}",
                   "l2": "256 MiB buffer written between timed steps; each step timed alone",
                   "parallelism": f"replicas x{world}", "bytes_per_lup": wl["bytes_per_lup"]},
        "roofline": head["roofline"],
        "e2e": {"value": round(n * e2e_steps * world / (e2e_ms * 1e-3) / 1e9, 4), "unit": "GLUPS",
                "h2d_bytes_per_step": round(h2d / e2e_steps, 1), "d2h_bytes_per_step": round(d2h / e2e_steps, 1),
                "timed": f"upload rho/U/T from pinned host memory, initialize, {e2e_steps} steps, download every field"},
        "e2e_cold": {"value": round(n * e2e_steps / cold_s / 1e9, 4), "unit": "GLUPS", "wall_ms": round(cold_s * 1e3, 3),
                     "note": "the e2e run including handle creation and the tile autotuner's first-step timing "
                             "(host wall clock, informational)"},
        "steady_state": {"ms_per_step": round(r64["steady_ms"], 6), "value": round(n / (r64["steady_ms"] * 1e-3) / 1e9, 4),
                         "unit": "GLUPS", "note": "no L2 flush between steps (informational, not the headline)"},
        "tile_config": info["tile_config"],
        "tile_ms": [round(t, 5) for t in info["tile_ms"] if t != 0.0],
        "clocks": r64["clocks"],
    }
    if "fp32_dev" in head:
        line["fp32_dev"] = {k: v for k, v in head["fp32_dev"].items() if k != "launches"}
    # the other named workloads, device-timed the same way (FP64 and FP32-deviation)
    extra = {}
    for name in ([] if a.no_extra else [w for w in EXTRA_WORKLOADS if w != a.workload]):
        x = device_line(name, a.extra_steps or a.steps)
        launches[name] = int(x["r64"]["launches"] + x.get("fp32_dev", {}).get("launches", 0))
        extra[name] = {"desc": WORKLOADS[name]["desc"], "eos": WORKLOADS[name]["eos"], "nodes": x["case"].n,
                       "steps": a.extra_steps or a.steps, "value": x["value"], "unit": "GLUPS",
                       "ms_per_step": x["ms_per_step"], "roofline": x["roofline"],
                       "tile_config": x["r64"]["info"]["tile_config"], "clocks": x["r64"]["clocks"]}
        if "fp32_dev" in x:
            extra[name]["fp32_dev"] = {k: v for k, v in x["fp32_dev"].items() if k != "launches"}
    if extra:
        line["extra"] = extra
    line["gpu_launches"] = launches["fp64_timed_steps"]  # the headline's timed region
    line["gpu_launches_by_region"] = launches
    if rank == 0 and world == 1 and not a.no_cpu:
        line["cpu_baseline"] = cpu_baseline(a.workload, a.cpu_steps, 1)
    if world == 1 and a.tte_cases > 0:
        line["time_to_equilibrium"] = time_to_equilibrium(a.tte_cases)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


def cpu_ranks(workload, steps, procs):
    """The reference's own multi-rank step (oracle/_ref: its collisions,
    streaming, boundaries and its sendPdfField / recvPdfField / sync*
    exchanges, multiPhasePP.c:122-240) on `procs` host threads, one rank per
    thread, over the reference partitioner's standard decomposition of the
    full lattice.  Messages pass through an in-process mailbox instead of an
    MPI library."""
    from multiphaselb_b200 import cases, slabs
    from oracle import oracle as orc
    if not orc.available("ref"):
        orc.build("ref")
    case = WORKLOADS[workload]["build"](cases)
    parts = slabs.partition(case, slabs.standard_owner(case.n, procs))
    ranks = orc.RefRanks(parts)
    ranks.initialize()
    t0 = time.perf_counter()
    ranks.step(steps)
    dt = time.perf_counter() - t0
    ghosts = sum(len(p.gidx) - len(p.own) for p in parts)
    return dict(value=case.n * steps / dt / 1e9, unit="GLUPS", cores=procs, step_ms=dt / max(steps, 1) * 1e3,
                kind="reference",
                sample=f"{steps} steps of the full {WORKLOADS[workload]['desc']} lattice as {procs} ranks "
                       f"(standard decomposition, {ghosts} ghost nodes), one thread per rank, exchanging "
                       f"through the reference's own send/recv/sync code over an in-process mailbox; "
                       f"wall {dt:.1f}s")


def run_reference(a):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    procs = a.cpu_procs or max(1, (os.cpu_count() or 1))
    procs = min(procs, 64)
    # one step = one time step of the full lattice on every core; K is capped
    # so that the run stays within minutes (a reference step of the column
    # takes about 25 ms on one core)
    steps = max(1, min(a.steps, a.ref_max_steps))
    samples = []
    leg = cpu_ranks if a.ref_mode == "ranks" else cpu_baseline
    leg(a.workload, max(1, min(a.warmup, 20)), procs)  # warm-up: process start, page-in
    t0 = time.perf_counter()
    for _ in range(max(1, a.ref_repeats)):
        samples.append(leg(a.workload, steps, procs))
    wall = time.perf_counter() - t0
    best = samples[-1]
    v = statistics.median(s["value"] for s in samples)
    line = {
        "metric": METRIC, "value": round(v, 6), "unit": "GLUPS", "n_gpus": world, "steps": steps,
        "warmup": a.warmup, "ms_per_step": round(best["step_ms"], 4), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded lattice of the named shape)",
        "impl": "reference",
        "config": {"workload": a.workload, "desc": WORKLOADS[a.workload]["desc"],
                   "parallelism": (f"{procs} reference ranks, one thread each, standard decomposition"
                                   if a.ref_mode == "ranks" else
                                   f"{procs} independent single-threaded reference processes")},
        "cpu_baseline": {"value": round(v, 6), "unit": "GLUPS", "cores": procs, "kind": best["kind"],
                         "sample": best["sample"]},
        "e2e": {"value": round(v, 6), "unit": "GLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "wall_s": round(wall, 2),
    }
    if steps != a.steps:
        line["steps_requested"] = a.steps
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="column_d2q9_128x512", choices=list(WORKLOADS))
    ap.add_argument("--path", default="auto", choices=["auto", "fused", "operators"])
    ap.add_argument("--cpu-steps", type=int, default=150)
    ap.add_argument("--cpu-procs", type=int, default=0)
    ap.add_argument("--ref-repeats", type=int, default=1)
    ap.add_argument("--ref-max-steps", type=int, default=3000,
                    help="reference arm: at most this many steps per core (keeps the run within minutes)")
    ap.add_argument("--ref-mode", default="copies", choices=["copies", "ranks"],
                    help="reference arm: independent single-rank copies of the lattice, one per core (an upper "
                         "bound on the reference's MPI scaling), or the lattice split into ranks that run the "
                         "reference's own exchange code, one thread each")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-fp32", action="store_true")
    ap.add_argument("--no-extra", action="store_true", help="time the named workload only")
    ap.add_argument("--extra-steps", type=int, default=0, help="timed steps of each extra workload (default --steps)")
    ap.add_argument("--tte-cases", type=int, default=24,
                    help="bubbles of the time-to-equilibrium comparison (1 GPU only; 0 = skip)")
    a = ap.parse_args()
    if a.warmup < 3:
        ap.error("--warmup must be >= 3")
    if a.impl == "reference":
        run_reference(a)
    else:
        run_ours(a)


if __name__ == "__main__":
    main()
