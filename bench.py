"""Benchmark: grid-point RK4 updates per second on the stratified-shell workload.

Workload (N = 1): 6 x 128^3 stratified spherical shell (r in [0.7, 1]; c = 0.1 + 0.9 s^0.5,
rho0 = (s + 0.01)^1.5, s = (1-r)/0.3; outer-5% sponge; one Gaussian pulse).  A "step" is
one call of the reference's RK4 (timestep.f90:41-86): five 2N-storage stages (edge
exchange + fused RHS/BC/sponge/update) and the explicit filter.  The unit of work is one
grid point advanced one full step.

* value       FP32 fused path (4 fields; rho is write-only with g0 = 0), device-resident,
              CUDA events on the library stream, K steps after W warm-up steps.
* fp64        the plain FP64 path (5 fields) on the same workload, for the FP32-vs-FP64
              comparison; fp32_rel_err_vs_fp64 is the per-field relative L2 after the run.
* e2e         the same metric through the C-ABI with host buffers: state uploaded from
              pinned host memory, K steps of RK4 each followed by the reference's per-step
              norm (cube.f90:77; solar_gpu_rk4_norms, read back once after the last step),
              final state downloaded.  fp64.e2e is the same for the FP64 path.
* fp32_err_c2_1000  FP32 (4 fields) against FP64 (5 fields) after 1000 steps of the
              workload: per-field relative L2 and max |difference| / max |FP64|.
* roofline    the dominant kernel (the fused stage kernel): algorithmic bytes per launch
              (q and qw read, q and qw written; 3F words in stage 1, 4F in stages 2-5)
              over its mean launch time from per-launch CUDA events.
* cpu_baseline the FP64 C++ restatement of the reference (the oracle), all host cores.

N > 1: one process per GPU (torchrun), each GPU runs its own replica of the workload
(weak scaling; the runs are independent, no collective on the data path); value is the
total over ranks with the time taken as the max over ranks.
``--impl reference`` times the reference's CPU path (the oracle port) instead.
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

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402


def stage_traffic(cfg, tile):
    """DRAM bytes per stage launch (mean over the five stages of a step) from the committed
    ncu launch-list summary, when it covers this workload; else None."""
    import re
    if cfg.name != "c2" or cfg.nx != 128:
        return None
    try:
        txt = open(os.path.join(ROOT, "profiles", "launch_list_c2_6x128cubed.md")).read()
        m = re.search(r"traffic_stage_fp32_mean_bytes_per_launch = (\d+)", txt)
        return float(m.group(1)) if m else None
    except Exception:
        return None


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms during a region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        rows = []
        try:
            for line in open(self.path):
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        except Exception:
            pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"], "samples": 0}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": reasons, "samples": len(rows)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=torch.device("cuda", local))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def cpu_baseline(cfg, nsteps: int):
    import oracle
    threads = os.cpu_count() or 1
    oracle.set_threads(threads)
    o = oracle.Oracle(cfg)
    q = o.initial_state()
    t0 = time.perf_counter()
    q = o.rk4(q, nsteps)
    dt = time.perf_counter() - t0
    return {"value": cfg.points * nsteps / dt, "unit": "grid-pt RK4 updates/s", "cores": threads,
            "kind": "port",
            "sample": f"{nsteps} full RK4 step(s) of the 6x{cfg.nx}^3 workload, FP64 C++ restatement "
                      f"of the reference (OpenMP, {threads} threads), {dt:.2f} s"}


def run_reference(args, world, rank):
    """The reference's CPU path (the oracle port) on the bench workload, rank 0 only."""
    if rank != 0:
        return
    from solar_b200 import configs
    import oracle
    cfg = configs.get(args.config)
    threads = os.cpu_count() or 1
    oracle.set_threads(threads)
    o = oracle.Oracle(cfg)
    q = o.initial_state()
    q = o.rk4(q, args.warmup)
    t0 = time.perf_counter()
    q = o.rk4(q, args.steps)
    dt = time.perf_counter() - t0
    value = cfg.points * args.steps / dt
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "grid-pt RK4 updates/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt * 1e3 / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": run_config(cfg, args.gpus), "fields": 5,
        "cpu_baseline": {"value": value, "unit": "grid-pt RK4 updates/s", "cores": threads, "kind": "port",
                         "sample": f"{args.steps} full RK4 steps after {args.warmup} warm-up, FP64 C++ restatement "
                                   f"of the reference, OpenMP {threads} threads"},
        "e2e": {"value": value, "unit": "grid-pt RK4 updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


METRIC = "grid-pt RK4 updates/s"


def run_config(cfg, world):
    """The workload description both arms print (same keys, same values)."""
    return {"workload": workload_name(cfg), "nx": cfg.nx, "nr": cfg.nr, "points": cfg.points,
            "parallelism": f"replica x{world}",
            "l2": "inputs larger than L2: three state buffers of %.0f MB each" % (
                6 * 4 * cfg.nr * (cfg.nx + 6) * (cfg.nx + 16) * 4 / 1e6)}


def workload_name(cfg):
    return (f"{cfg.name}: 6 x {cfg.nx}^2 x {cfg.nr} stratified spherical shell, CFL 0.5 dt={cfg.dt:.4g}, "
            f"sponge {cfg.sponge.length} outer points")


def rel_errors(a, b, fields):
    names = ("rho", "v_xi", "v_eta", "v_r", "p")
    return {names[m]: float(np.linalg.norm(a[:, m] - b[:, m]) / max(np.linalg.norm(b[:, m]), 1e-300)) for m in fields}


def adjoint_block(device: int, nsteps: int, k: int, nfd: int):
    """Misfit gradient dJ/dc on the adjoint workload (6 x 96^3 stratified shell, 32 receivers
    at r = 0.98, data from a model with eight sound-speed anomalies), timed on the device in
    FP32 (4 fields) and FP64 (5 fields).  The FP32 gradient is checked against the FP64 one
    (relative L2), and both against central finite differences of the GPU FP64 misfit along
    nfd directions (half random per point, half smooth blobs near the anomalies)."""
    import numpy as np
    from solar_b200 import configs, receivers
    from solar_b200.solver import Solver

    cfg = configs.c4(nsteps=nsteps)
    loc = receivers.locate(cfg, cfg.receivers)
    c0 = receivers.sound_speed(cfg)
    c_true = receivers.sound_speed(cfg, cfg.dc_blobs)
    with Solver(cfg, device=device) as s:
        s.init_sources()
        q0 = s.get_state()

    def traces(c):
        with Solver(cfg, device=device, c2_3d=c ** 2) as s:
            s.set_state(q0)
            s.set_receivers(loc)
            return s.record(nsteps)

    def gradient(prec, nf):
        with Solver(cfg, precision=prec, nfields=nf, device=device, c2_3d=c0 ** 2) as s:
            s.set_state(q0)
            s.set_receivers(loc)
            s.misfit_gradient(min(k, nsteps), k, data[:min(k, nsteps)])      # warm-up, allocates
            return s.misfit_gradient(nsteps, k, data)

    data = traces(c_true)
    res64 = gradient("fp64", 5)
    res32 = gradient("fp32", 4)
    g64, g32 = res64["grad_c"], res32["grad_c"]
    rng = np.random.default_rng(44)
    errs64, errs32 = [], []
    for m in range(nfd):
        if m % 2 == 0:
            d = rng.standard_normal(c0.shape) * c0
        else:      # four blobs around the anomalies, where the receivers are sensitive
            centres = np.array([cfg.dc_blobs[i][0] for i in rng.choice(len(cfg.dc_blobs), 4, replace=False)])
            centres = centres + rng.uniform(-0.05, 0.05, centres.shape)
            d = receivers.sound_speed(cfg, [(tuple(x), 0.06, 1.0) for x in centres]) - c0
        d[:, 0] = 0.0
        d[:, -1] = 0.0
        eps = 1e-6 / np.abs(d / c0).max()
        jp = 0.5 * float(((traces(c0 + eps * d) - data) ** 2).sum())
        jm = 0.5 * float(((traces(c0 - eps * d) - data) ** 2).sum())
        fd = (jp - jm) / (2 * eps)
        for g, errs in ((g64, errs64), (g32, errs32)):
            ad = float(np.vdot(g.ravel(), d.ravel()))
            errs.append(abs(fd - ad) / abs(fd))
    pts = cfg.points

    def timing(res):
        total_ms = res["forward_ms"] + res["recompute_ms"] + res["adjoint_ms"]
        return {"misfit": res["misfit"], "gradient_ms": total_ms, "forward_ms": res["forward_ms"],
                "recompute_ms": res["recompute_ms"], "adjoint_ms": res["adjoint_ms"],
                "adjoint_pt_steps_per_s": pts * nsteps / (res["adjoint_ms"] / 1e3),
                "gradient_cost_in_forward_runs": total_ms / res["forward_ms"]}

    out = {"workload": "c4: 6 x %d^3 stratified shell, %d steps, %d receivers, checkpoint every %d steps" % (
        cfg.nx, nsteps, len(loc), k)}
    out["fp32"] = timing(res32)
    out["fp32"]["fields"] = 4
    out["fp32"]["grad_rel_l2_vs_fp64"] = float(np.linalg.norm(g32 - g64) / np.linalg.norm(g64))
    out["fp32"]["fd_rel_err_max"] = max(errs32) if errs32 else None
    out["fp32"]["fd_rel_errs"] = errs32
    out["fp64"] = timing(res64)
    out["fp64"]["fields"] = 5
    out["fp64"]["fd_rel_err_max"] = max(errs64) if errs64 else None
    out["fp64"]["fd_rel_errs"] = errs64
    out["fd_directions"] = nfd
    out["fd_reference"] = "central differences of the GPU FP64 misfit, eps = 1e-6 relative"
    out["fd_tolerance"] = 1e-4
    return out


def fp32_error_block(cfg, device: int, nsteps: int):
    """FP32 (4 fields) against FP64 (5 fields) on the benchmark workload after nsteps steps:
    per-field relative L2 and max |FP32 - FP64| / max |FP64|."""
    from solar_b200.solver import Solver

    states = {}
    for prec, nf in (("fp64", 5), ("fp32", 4)):
        with Solver(cfg, precision=prec, nfields=nf, device=device) as s:
            s.init_sources()
            s.rk4(nsteps)
            states[prec] = s.get_state()
    a, b = states["fp32"], states["fp64"]
    names = ("rho", "v_xi", "v_eta", "v_r", "p")
    out = {"steps": nsteps}
    for m in (1, 2, 3, 4):
        out[names[m]] = {"rel_l2": float(np.linalg.norm(a[:, m] - b[:, m]) / np.linalg.norm(b[:, m])),
                         "max_abs_over_max_ref": float(np.abs(a[:, m] - b[:, m]).max() / np.abs(b[:, m]).max())}
    out["max_rel_l2"] = max(out[names[m]]["rel_l2"] for m in (1, 2, 3, 4))
    out["tolerance"] = 1e-5
    return out


def e2e_block(cfg, precision: str, nfields: int, args, world: int, local: int):
    """End to end through the C-ABI with host buffers: the six-zone FP64 state comes in from
    pinned host memory, K steps run with the per-step norm of v_r (cube.f90:74-78), the
    norms and the final state come back to pinned host memory.  Host wall clock around the
    whole job; max over ranks."""
    import torch
    from solar_b200.solver import Solver

    # the stored fields cross PCIe as FP64 (rho is not stored with 4 fields: not copied)
    state_bytes = 6 * nfields * cfg.nr * cfg.nx * cfg.nx * 8
    host = torch.empty(6 * 5 * cfg.nr * cfg.nx * cfg.nx, dtype=torch.float64, pin_memory=True).numpy()
    out = torch.empty_like(torch.from_numpy(host)).pin_memory().numpy()
    norms = torch.empty(args.steps, dtype=torch.float64, pin_memory=True).numpy()
    with Solver(cfg, precision=precision, nfields=nfields, device=local) as se:
        se.init_sources()
        se.get_state(out=host.reshape(se.state_shape))
        se.rk4_norms(args.warmup, out=norms[:args.warmup] if args.warmup <= args.steps else None)
        barrier(world)
        t0 = time.perf_counter()
        se.set_state(host.reshape(se.state_shape))
        se.rk4_norms(args.steps, out=norms)
        se.get_state(out=out.reshape(se.state_shape))
        te = time.perf_counter() - t0
    te = max_over_ranks(te, world)
    return {"value": cfg.points * args.steps * world / te, "unit": "grid-pt RK4 updates/s",
            "h2d_bytes_per_step": state_bytes / args.steps,
            "d2h_bytes_per_step": (state_bytes + 8 * args.steps) / args.steps,
            "ms_per_step": te * 1e3 / args.steps, "norm_vr_last": float(norms[-1]),
            "note": "state in from pinned host memory once per job (the stored fields, FP64; an FP32 "
                    "context rounds them to float on host threads and copies half those bytes), K RK4 "
                    "steps each followed by norm(v_r) (cube.f90:74-78) kept on the device and read "
                    "back once, state out at the end (FP64); host wall clock of the whole job"}


def batch_block(device: int):
    """The batched-sources workload: 64 independent runs of 6 x 64^3 (stratified shell,
    per-run seeded source), uneven step counts 200..1000, FP32, all runs in the same
    launches (one captured graph per step, finished runs masked off on the device)."""
    from solar_b200 import configs
    from solar_b200.solver import Solver

    cfg = configs.c3()
    R = len(cfg.runs)
    with Solver(cfg, precision="fp32", nfields=4, nruns=R, device=device) as s:
        for r in range(R):
            s.init_sources(cfg.runs[r], run=r)
        s.rk4_runs([3] * R)                                   # warm-up (graph capture)
        ms = s.time_rk4_runs(cfg.run_steps)
        tile = list(s.tile) if s.tile else "default"
    work = cfg.points * sum(cfg.run_steps)
    with Solver(cfg, precision="fp32", nfields=4, nruns=1, device=device) as s1:
        s1.init_sources(cfg.runs[0])
        s1.rk4(3)
        one = s1.time_rk4(200)["total_ms"]
    single = cfg.points * 200 / (one / 1e3)
    return {"workload": "c3: %d runs of 6 x %d^3, steps %d..%d (sum %d), FP32 F=4" % (
                R, cfg.nx, min(cfg.run_steps), max(cfg.run_steps), sum(cfg.run_steps)),
            "value": work / (ms / 1e3), "unit": "grid-pt RK4 updates/s", "ms": ms,
            "graph_replays": max(cfg.run_steps), "tile": tile,
            "single_run_value": single, "batch_speedup_vs_one_run_at_a_time": (work / (ms / 1e3)) / single}


def large_block(device: int, nsteps: int):
    """The large-grid workload: 6 x 384^3 stratified shell, 16 sources, FP32 F=4 and FP64
    F=5 on the same grid (state 5.7 GB / 14.4 GB per buffer)."""
    from solar_b200 import configs
    from solar_b200.solver import Solver

    cfg = configs.c5(nsteps=nsteps)
    out = {"workload": "c5: 6 x %d^3, %d steps" % (cfg.nx, nsteps)}
    for prec, nf in (("fp32", 4), ("fp64", 5)):
        t0 = time.perf_counter()
        s = Solver(cfg, precision=prec, nfields=nf, device=device)
        init_s = time.perf_counter() - t0
        with s:
            s.init_sources()
            s.rk4(3)
            t = s.time_rk4(nsteps)
            out[prec] = {"value": cfg.points * nsteps / (t["total_ms"] / 1e3), "ms_per_step": t["total_ms"] / nsteps,
                         "fields": nf, "norm_vr": s.norm(4),
                         "init_s": init_s}    # solar_gpu_init: host tables, uploads, state buffers
    out["fp32_speedup"] = out["fp32"]["value"] / out["fp64"]["value"]
    return out


def split_block(cfg, args, world, local):
    """The sphere split across the job's processes (strong scaling of one six-zone run):
    gcd(world, 6) zone groups x radial slabs; each rank exchanges edge lines and boundary
    planes with its neighbours every phase over torch.distributed (NCCL).  Timed with CUDA
    events on the library's stream, max over ranks."""
    import torch

    import torch.distributed as dist

    from solar_b200 import distributed as D

    own_group = not dist.is_initialized()
    if own_group:                             # one process: a one-rank group
        import socket
        with socket.socket() as sk:
            sk.bind(("127.0.0.1", 0))
            port = sk.getsockname()[1]
        dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1)
    zs = D.ZoneSplitSolver(cfg, precision="fp32", nfields=4, device=local)
    zs.solver.init_sources()
    zs.rk4(args.warmup)
    barrier(world)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(zs.stream)
    zs.rk4(args.steps)
    e1.record(zs.stream)
    e1.synchronize()
    ms = max_over_ranks(e0.elapsed_time(e1), world)
    norm = zs.norm(4)
    zs.close()
    if own_group:
        dist.destroy_process_group()
    ngroups, nslabs = D.layout(world)
    return {"value": cfg.points * args.steps / (ms / 1e3), "unit": "grid-pt RK4 updates/s", "scaling": "strong",
            "ms_per_step": ms / args.steps, "zone_groups": ngroups, "radial_slabs": nslabs, "norm_vr": norm}


def large_adjoint_block(device: int, nsteps: int, outer: int, inner: int):
    """Misfit gradient on the large grid (6 x 384^3 stratified shell, 16 sources, FP32 4
    fields, one receiver 0.02 above each source, zero data so J = 1/2 sum p^2): two
    checkpoint levels keep it inside one GPU's memory."""
    import numpy as np
    import torch

    from solar_b200 import configs, receivers
    from solar_b200.solver import Solver

    cfg = configs.c5(nsteps=nsteps)
    pts = [np.asarray(s.x0) / np.linalg.norm(s.x0) * 0.97 for s in cfg.sources]
    loc = receivers.locate(cfg, pts)
    with Solver(cfg, precision="fp32", nfields=4, device=device) as s:
        s.init_sources()
        s.set_receivers(loc)
        res = s.misfit_gradient(nsteps, outer, np.zeros((nsteps, len(loc))), inner_every=inner)
        free, total = torch.cuda.mem_get_info(device)
    g = res["grad_c"]
    total_ms = res["forward_ms"] + res["recompute_ms"] + res["adjoint_ms"]
    return {"workload": "c5: 6 x %d^3 stratified shell, %d steps, %d receivers, FP32 F=4, checkpoints every %d "
                        "steps with inner checkpoints every %d" % (cfg.nx, nsteps, len(loc), outer, inner),
            "misfit": res["misfit"], "gradient_ms": total_ms, "forward_ms": res["forward_ms"],
            "recompute_ms": res["recompute_ms"], "adjoint_ms": res["adjoint_ms"],
            "adjoint_pt_steps_per_s": cfg.points * nsteps / (res["adjoint_ms"] / 1e3),
            "gradient_cost_in_forward_runs": total_ms / res["forward_ms"],
            "device_memory_in_use_gb": (total - free) / 1e9, "grad_finite": bool(np.isfinite(g).all()),
            "grad_norm": float(np.linalg.norm(g))}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="solar", choices=["solar", "reference"])
    ap.add_argument("--config", default="c2")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--adjoint-steps", type=int, default=500)
    ap.add_argument("--adjoint-checkpoint", type=int, default=50)
    ap.add_argument("--adjoint-fd", type=int, default=16)
    ap.add_argument("--err-steps", type=int, default=1000,
                    help="steps of the FP32-vs-FP64 error check on the workload (0 = skip)")
    ap.add_argument("--split", action="store_true",
                    help="also run the sphere split across the job's processes (zone groups x radial slabs)")
    ap.add_argument("--no-batch", action="store_true")
    ap.add_argument("--no-large", action="store_true")
    ap.add_argument("--large-steps", type=int, default=200)
    ap.add_argument("--no-large-adjoint", action="store_true",
                    help="skip the misfit gradient on the 6 x 384^3 grid")
    ap.add_argument("--large-adjoint-steps", type=int, default=20,
                    help="steps of the 6 x 384^3 misfit gradient (200 = the workload's full run, ~160 GB)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    world, rank, local = dist_setup()
    if args.impl == "reference":
        run_reference(args, world, rank)
        return

    from solar_b200 import configs
    from solar_b200.solver import Solver

    cfg = configs.get(args.config)
    pts = cfg.points
    peak, peak_kind = load_peaks()

    # ---------------------------------------------------------------- FP32 fused path
    s32 = Solver(cfg, precision="fp32", nfields=4, device=local)
    tile32 = list(s32.tile) if s32.tile else "default"
    s32.init_sources()
    s32.rk4(args.warmup)
    barrier(world)
    s32.synchronize()
    with ClockSampler(local) as clk:
        t = s32.time_rk4(args.steps)
    barrier(world)
    ms32 = max_over_ranks(t["total_ms"], world)
    value = pts * args.steps * world / (ms32 / 1e3)
    q32 = s32.get_state()

    # per-kernel launch times (graph off) for the roofline of the dominant kernel
    kt = s32.time_rk4(max(4, min(args.steps, 20)), per_kernel=True)
    F, w = 4, 4
    stage_bytes = (3 * F + 4 * 4 * F) / 5.0 * w * pts          # mean algorithmic bytes per stage launch
    filter_bytes = 2 * F * w * pts
    stage_gbs = stage_bytes / (kt["stage_ms"] / 1e3) / 1e9
    filter_gbs = filter_bytes / (kt["filter_ms"] / 1e3) / 1e9
    step_bytes = 21 * F * w * pts
    s32.close()

    # ---------------------------------------------------------------- FP64 plain path
    s64 = Solver(cfg, precision="fp64", nfields=5, device=local)
    s64.init_sources()
    s64.rk4(args.warmup)
    barrier(world)
    t64 = s64.time_rk4(args.steps)
    barrier(world)
    ms64 = max_over_ranks(t64["total_ms"], world)
    value64 = pts * args.steps * world / (ms64 / 1e3)
    q64 = s64.get_state()
    kt64 = s64.time_rk4(4, per_kernel=True)
    s64.close()
    err = rel_errors(q32, q64, (1, 2, 3, 4))

    # ---------------------------------------------------------------- end to end (C-ABI, host buffers)
    e2e = e2e64 = None
    if not args.no_e2e:
        e2e = e2e_block(cfg, "fp32", 4, args, world, local)
        e2e64 = e2e_block(cfg, "fp64", 5, args, world, local)

    split = split_block(cfg, args, world, local) if args.split else None
    if rank != 0:
        return
    adjoint = batch = large = None
    if world == 1 and not args.no_adjoint:
        adjoint = adjoint_block(local, args.adjoint_steps, args.adjoint_checkpoint, args.adjoint_fd)
    if world == 1 and not args.no_batch:
        batch = batch_block(local)
    if world == 1 and not args.no_large:
        large = large_block(local, args.large_steps)
    large_adj = None
    if world == 1 and not args.no_large_adjoint:
        large_adj = large_adjoint_block(local, args.large_adjoint_steps, 20, 4)
    err1000 = None
    if world == 1 and args.err_steps > 0:
        err1000 = fp32_error_block(cfg, local, args.err_steps)
    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(cfg, 2)
    clocks = clk.summary()
    line = {
        "metric": METRIC,
        "value": value, "unit": "grid-pt RK4 updates/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms32 / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": run_config(cfg, world), "fields": 4,
        "path": "FP32 fused path, 4 fields; the FP64 plain path (5 fields) is reported under fp64",
        "fp64": {"value": value64, "ms_per_step": ms64 / args.steps, "fields": 5,
                 "fp32_speedup": value / value64, "e2e": e2e64,
                 "stage_ms": kt64["stage_ms"], "filter_ms": kt64["filter_ms"], "edge_ms": kt64["edge_ms"]},
        "fp32_rel_err_vs_fp64": err,
        "fp32_err_c2_1000": err1000,
        "roofline": {"bound": "hbm", "achieved": stage_gbs, "peak": peak, "unit": "GB/s",
                     "frac": stage_gbs / peak, "traffic": stage_traffic(cfg, tile32), "peak_kind": peak_kind,
                     "traffic_source": "dram__bytes_read.sum + dram__bytes_write.sum per stage launch, mean of "
                                       "the five stages, from the committed ncu launch list of this workload "
                                       "(profiles/launch_list_c2_6x128cubed.md), not measured in this run",
                     "timing": "mean per-launch CUDA-event time of launches made without the step graph",
                     "kernel": "stage_kernel<float> (tile x, tile y, planes per CTA = %s)" % (tile32,),
                     "algorithmic_bytes_per_launch": stage_bytes,
                     "mean_launch_ms": kt["stage_ms"],
                     "filter": {"achieved": filter_gbs, "frac": filter_gbs / peak, "mean_launch_ms": kt["filter_ms"]},
                     "edge_mean_launch_ms": kt["edge_ms"],
                     "step_roofline_pt_steps_per_s": peak * 1e9 / (21 * F * w),
                     "step_frac": (value / world) * (21 * F * w) / (peak * 1e9)},
        "gpu_launches": 12 * args.steps,
        "clocks": clocks,
        "e2e": e2e,
        "cpu_baseline": cpu,
        "adjoint": adjoint,
        "batched_sources": batch,
        "large_grid": large,
        "large_grid_adjoint": large_adj,
        "zone_split": split,
    }
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
