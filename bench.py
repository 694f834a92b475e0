"""Benchmark of the FR residual + SSP-RK3 hot path: DOF-RHS evaluations/s.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload: the Taylor-Green configuration -- 256x256 jittered (seed 1,
+-0.15h) Q1 quads on [0,pi]^2 with slip walls, P3 (65 536 elements, 1 048 576
DOF per variable), u = sin x cos y, v = -cos x sin y, M = 0.3, compressible
Navier-Stokes with Re = 5000, Pr = 0.72, Roe flux, HU correction.  One bench
step = one SSP-RK3 time step = three residual evaluations over the whole
mesh; DOF-RHS/s = E * n_sp * 3 * K / t.

The headline `value` is the precision form (FP32 volume, face, gradient and
operator work; FP64 state, RK accumulation and reductions); the same case in
FP64 is the `fp64` object with `speedup_vs_fp64`; `precision_errors` gives
the L2 / Linf error of rho, rho u, rho v, rho E after 1000 steps at CFL 0.5
against the FP64 path (which matches the FP64 oracle to 1e-12 per residual)
with the FP64 conditioning floor beside it.  The same mesh and state in the
reference's residual semantics (compat: Rusanov, inviscid, clamps, FP64) is
the `compat` object.  `p5_precision` is the precision form of the same flow
at P5 on 512x512 quads; `mixed_elements` the shear layer on 384x384 quads
with 30% split into triangles (P2-P4, SD and GA, precision form against
FP64).

ours:      the CUDA path, timed with CUDA events on the solver's stream, max
           over ranks; N > 1 runs one independent replica per GPU (the path
           has no exchange on one GPU; weak scaling).
reference: the oracle (the CPU restatement of the residual; the reference has
           no CPU path) on the same workload, FP64, with every host thread,
           rank 0.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "DOF-RHS evals/s, FP32-split vs FP64 GPU at stated L2 err; adjoint/fwd ratio"
UNIT = "DOF-RHS/s"
GAMMA, MACH = 1.4, 0.3
NX = 256
P = 3
DT = 2.0e-4


MODES = {
    "ns": dict(compat=False, viscous=True, riemann="Roe", flux_type="HU", Re=5000.0, Pr=0.72),
    "ns32": dict(compat=False, viscous=True, riemann="Roe", flux_type="HU", Re=5000.0, Pr=0.72,
                 precision="mixed"),
    "compat": dict(compat=True, viscous=False, riemann="Rusanov", flux_type="HU"),
}


def workload_name(mode="ns"):
    if mode == "ns":
        return (f"TGV {NX}x{NX} jittered Q1 quads on [0,pi]^2, slip walls, P{P}, Navier-Stokes "
                f"Re 5000 Pr 0.72, Roe, HU, SSP-RK3")
    return (f"TGV {NX}x{NX} jittered Q1 quads on [0,pi]^2, slip walls, P{P}, reference residual "
            f"semantics (Rusanov, inviscid, clamps), SSP-RK3")


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def algorithmic_bytes_per_element(p, w_s=8, w_g=8, w_t=8, viscous=False):
    """Bytes one element moves per residual evaluation with the fused RK stage:
    w_s*12*n_sp (stage state, base state, output) + w_g*5*n_sp (J and four
    metric terms) + w_t*32*n_f (own trace write + neighbour trace read)
    [+ w_t*64*n_f for the gradient traces of Navier-Stokes]."""
    nsp, nf = (p + 1) ** 2, p + 1
    b = w_s * 12 * nsp + w_g * 5 * nsp + w_t * 32 * nf
    if viscous:
        b += w_t * 64 * nf
    return b


def mode_bytes_per_element(mode, p=P):
    """Algorithmic bytes per element and residual of a bench mode: FP64
    everywhere, or (mixed) FP64 state with FP32 metrics and traces."""
    w = 4 if MODES[mode].get("precision") == "mixed" else 8
    return algorithmic_bytes_per_element(p, 8, w, w, viscous=MODES[mode].get("viscous", False))


def traffic_from_profile(kernel_key):
    """Per-launch DRAM bytes of the dominant kernel from the committed ncu
    summary (profiles/traffic.json), or None."""
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
            return json.load(f).get(kernel_key)
    except Exception:
        return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
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
        except Exception:
            self.proc.kill()
        self.t.join(timeout=2)
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
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def build_case():
    from zhijian_b200 import meshgen as M
    mesh = M.tgv_mesh(NX, seed=1)
    return mesh


def make_params_for(mode="ns"):
    from zhijian_b200.solver import make_params
    return make_params(poly_order=P, gamma=GAMMA, rho_inf=1.0, p_inf=1.0 / (GAMMA * MACH * MACH),
                       Mach=MACH, bcs=[(1, "slipwall")], **MODES[mode])


def make_solver(mesh, mode="ns"):
    from zhijian_b200.solver import FRSolver
    return FRSolver(mesh, make_params_for(mode))


def make_oracle(mesh, mode, threads):
    from oracle import oracle as O
    orc = O.Oracle(mesh, P, GAMMA, 1.0, 1.0 / (GAMMA * MACH * MACH), MACH, 0.0, threads=threads)
    m = MODES[mode]
    step = orc.step
    if not m["compat"]:
        orc.set_physics(2, 1, m["viscous"], m.get("Re", 1000.0), m.get("Pr", 0.72))
        step = orc.step_phys
    return orc, step


def cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def oracle_rate(mesh, mode, warmup=1, runs=5, run_seconds=2.0, min_steps=1):
    """The oracle (FP64, all host threads) on the full benchmark mesh: `warmup`
    untimed SSP-RK3 steps, then `runs` timed runs of at least `min_steps`
    steps and `run_seconds` seconds each; returns the median DOF-RHS/s, the
    per-run rates, the median ms per step, the steps timed and the threads."""
    from zhijian_b200 import meshgen as M
    threads = os.cpu_count() or 1
    orc, step = make_oracle(mesh, mode, threads)
    U = M.taylor_green(orc.sp_coords())
    for _ in range(max(1, warmup)):
        U, _ = step(U, DT, 1)
    dof = mesh.n_elem * (P + 1) ** 2
    rates, ms, steps = [], [], 0
    for _ in range(runs):
        n, t0 = 0, time.perf_counter()
        while True:
            U, _ = step(U, DT, 1)
            n += 1
            el = time.perf_counter() - t0
            if n >= min_steps and el >= run_seconds:
                break
        rates.append(dof * 3 * n / el)
        ms.append(1e3 * el / n)
        steps += n
    return statistics.median(rates), rates, statistics.median(ms), steps, threads


def cpu_baseline(mesh, seconds=10.0, mode="ns"):
    """The oracle (FP64 Navier-Stokes, the benchmark's scheme) on the host
    cores over the full benchmark mesh: median of five runs of about
    seconds/5 each after a warm-up step, with the spread and the CPU model;
    beside it the same for the reference's residual semantics (compat)."""
    v, rates, _, steps, threads = oracle_rate(mesh, mode, run_seconds=seconds / 5)
    vc, _, _, steps_c, _ = oracle_rate(mesh, "compat", run_seconds=seconds / 10)
    return {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"median of 5 runs ({steps} SSP-RK3 steps in all) on the full mesh; "
                      f"spread {min(rates):.3g}-{max(rates):.3g}",
            "cpu": cpu_model(), "compat_value": vc}


def run_reference(args):
    """--impl reference: the oracle port (the reference has no CPU path) with
    all host threads on the benchmark's workload, rank 0 only: W warm-up
    steps, then the median of five timed runs of at least max(K/5, 1) steps
    and 2 s each."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return None
    mesh = build_case()
    v, rates, ms, steps, threads = oracle_rate(mesh, "ns", warmup=args.warmup,
                                               run_seconds=getattr(args, "run_seconds", 2.0),
                                               min_steps=max(1, args.steps // 5))
    return {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "impl": "reference",
            "config": {"workload": workload_name("ns"), "precision": "fp64",
                       "elements": mesh.n_elem, "dof_per_var": mesh.n_elem * (P + 1) ** 2},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": f"median of 5 runs ({steps} SSP-RK3 steps in all) on the full "
                                       f"mesh; spread {min(rates):.3g}-{max(rates):.3g}"},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


KERNELS = {"ns": "k_ns_grad_lines<3,double> + k_ns_stage<3,Roe,double> (one residual)",
           "ns32": "k_ns_grad_lines<3,float> + k_ns_stage<3,Roe,float> (one residual)",
           "compat": "k_compat_stage<3>"}
LAUNCHES_PER_RHS = {"ns": 2, "ns32": 2, "compat": 1}
# handles of the streamed end-to-end loop: 2 reach 3.6e9 DOF-RHS/s, 3 and 4
# both 4.2e9 (the host copies, 67 MB per step, bound it at 3)
E2E_HANDLES = 3


class Ranks:
    """One process per GPU (torchrun): rank and world from the environment, a
    process group with a short timeout when world > 1, a barrier and the
    maximum of a per-rank number (the timing rule: the job takes as long as
    its slowest rank).  backend "nccl" with a CUDA device in the bench; the
    tests run the same code with "gloo" on the CPU."""

    def __init__(self, backend="nccl", device=None, timeout_s=120):
        import torch
        import torch.distributed as dist
        self.dist = dist
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.device = device if device is not None else torch.device("cpu")
        self.backend = backend
        if self.world > 1:
            import datetime
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))

    def barrier(self):
        if self.world > 1:
            if self.backend == "nccl":
                self.dist.barrier(device_ids=[self.local])
            else:
                self.dist.barrier()

    def max(self, x):
        if self.world == 1:
            return x
        import torch
        t = torch.tensor([x], dtype=torch.float64, device=self.device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.world > 1:
            self.dist.destroy_process_group()


def whole_job_rate(units_per_rank, world, ms):
    """Units all ranks processed per second over the slowest rank's time
    (replicas: every rank processes the same units)."""
    return world * units_per_rank / (ms * 1e-3)


def run_ours(args):
    import torch
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    ranks = Ranks("nccl", dev)
    world, rank = ranks.world, ranks.rank

    def barrier_sync():
        torch.cuda.synchronize()
        ranks.barrier()
        torch.cuda.synchronize()

    max_over_ranks = ranks.max

    from zhijian_b200 import meshgen as M
    mesh = build_case()
    stream = torch.cuda.Stream(dev)        # a real stream: events and kernels share it
    peak, peak_kind = load_peaks()
    sampler = ClockSampler(local)   # sampled from warm-up through the timed regions
    sampler.start()
    time.sleep(0.2)

    def timed(mode):
        s = make_solver(mesh, mode)
        s.set_stream(stream.cuda_stream)
        U0 = M.taylor_green(s.solution_point_coords())
        s.copyToDevice(U0)
        s.advance(DT, args.warmup)
        barrier_sync()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        barrier_sync()
        e0.record(stream)
        s.advance(DT, args.steps, sync=False)
        e1.record(stream)
        barrier_sync()
        ms = max_over_ranks(e0.elapsed_time(e1))
        s.check_state()
        dof = s.n_elem * s.n_sp
        per_rhs = ms * 1e-3 / (3 * args.steps)
        nbytes = mode_bytes_per_element(mode) * s.n_elem
        achieved = nbytes / per_rhs / 1e9
        roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": traffic_from_profile(f"{mode}|tgv{NX}"),
                "peak_kind": peak_kind, "kernel": KERNELS[mode],
                "algorithmic_bytes_per_launch": nbytes,
                "algorithmic_bytes_per_element": mode_bytes_per_element(mode),
                "launches_per_residual": LAUNCHES_PER_RHS[mode]}
        return s, U0, dof, ms, roof

    head = "ns32"
    s, U0, dof, ms, roofline = timed(head)
    value = whole_job_rate(dof * 3 * args.steps, world, ms)
    launches = 3 * args.steps * LAUNCHES_PER_RHS[head]

    # end to end through the C-ABI with host buffers: per step a state goes
    # H2D from pinned memory, one SSP-RK3 step runs, the new state comes back
    # D2H.  Serial: one handle, blocking copies.  Streamed (the headline): the
    # steps' inputs are independent states, dealt round-robin over
    # E2E_HANDLES handles on as many streams with queued copies, so the
    # handles' uploads, steps and downloads overlap (one copy engine per
    # direction).
    n_e2e = max(4, min(args.steps, 50))
    host = torch.from_numpy(U0.copy()).pin_memory()
    hnp = host.numpy()
    s.copyToDevice(hnp)
    s.advance(DT, 1)
    barrier_sync()
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    for _ in range(n_e2e):
        s.copyToDevice(hnp)
        s.advance(DT, 1, sync=False)
        s.copyToHost(out=hnp)
    f1.record(stream)
    barrier_sync()
    ems_serial = max_over_ranks(f0.elapsed_time(f1))
    pairs = [(s, stream)]
    for _ in range(E2E_HANDLES - 1):
        st = torch.cuda.Stream(dev)
        h = make_solver(mesh, head)
        h.set_stream(st.cuda_stream)
        pairs.append((h, st))
    nh = len(pairs)
    hin = [torch.from_numpy(U0.copy()).pin_memory().numpy() for _ in range(nh)]
    hout = [torch.empty(U0.shape, dtype=torch.float64).pin_memory().numpy() for _ in range(nh)]

    def streamed(n):
        for i in range(n):
            h = pairs[i % nh][0]
            h.copyToDeviceAsync(hin[i % nh])
            h.advance(DT, 1, sync=False)
            h.copyToHostAsync(hout[i % nh])
    streamed(2 * nh)
    barrier_sync()
    g0 = torch.cuda.Event(enable_timing=True)
    g0.record(stream)
    for _, st in pairs[1:]:
        st.wait_event(g0)
    streamed(n_e2e)
    ends = []
    for _, st in pairs:
        ev = torch.cuda.Event(enable_timing=True)
        ev.record(st)
        ends.append(ev)
    barrier_sync()
    ems = max_over_ranks(max(g0.elapsed_time(ev) for ev in ends))
    e2e = {"value": whole_job_rate(dof * 3 * n_e2e, world, ems), "unit": UNIT,
           "h2d_bytes_per_step": int(U0.nbytes), "d2h_bytes_per_step": int(U0.nbytes),
           "steps": n_e2e,
           "mode": f"independent states over {nh} handles on {nh} streams, queued copies from pinned memory",
           "serial": {"value": whole_job_rate(dof * 3 * n_e2e, world, ems_serial),
                      "mode": "one handle, blocking copies"}}
    for h, _ in pairs:
        h.close()

    s64, _, _, ms64, roof64 = timed("ns")
    s64.close()
    fp64 = {"workload": workload_name("ns") + ", FP64", "value": whole_job_rate(dof * 3 * args.steps, world, ms64),
            "ms_per_step": ms64 / args.steps, "roofline": roof64,
            "gpu_launches": 3 * args.steps * LAUNCHES_PER_RHS["ns"]}
    clocks = sampler.stop()

    sc, _, dofc, msc, roofc = timed("compat")
    sc.close()
    compat = {"workload": workload_name("compat"), "value": whole_job_rate(dofc * 3 * args.steps, world, msc),
              "ms_per_step": msc / args.steps, "roofline": roofc,
              "gpu_launches": 3 * args.steps}

    precision = precision_errors(mesh, stream) if not args.no_error_run else None
    adjoint = adjoint_run(stream) if not args.no_adjoint else None
    p5 = p5_precision_case(stream, args) if not args.no_p5 else None
    shear = shear_layer_sweep(stream, args) if not args.no_mixed else None
    parts = partition_case(mesh, args) if (world == 1 and not args.no_parts) else None

    out = None
    if rank == 0:
        detail = {"fp64": fp64, "compat": compat, "precision_errors": precision, "adjoint": adjoint,
                  "p5_precision": p5, "mixed_elements": shear, "partitioned": parts, "e2e": e2e,
                  "roofline": roofline}
        out = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
               "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
               "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
               "dtype": "f32", "data": "synthetic",
               "config": {"workload": workload_name("ns") + ", precision form", "elements": mesh.n_elem,
                          "dof_per_var": dof, "rhs_per_step": 3,
                          "precision": "FP32 volume/face/gradient/operator work; FP64 state, RK, norms",
                          "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                          "l2": "no flush: each stage streams > 200 MB > 126 MB L2"},
               "roofline": {k: roofline[k] for k in ("bound", "achieved", "peak", "unit", "frac", "traffic",
                                                     "peak_kind", "kernel")},
               "e2e": {k: e2e[k] for k in ("value", "unit", "h2d_bytes_per_step", "d2h_bytes_per_step")},
               "e2e_serial": e2e["serial"]["value"],
               "gpu_launches": launches, "clocks": clocks,
               "fp64_value": fp64["value"], "fp64_frac": roof64["frac"],
               "speedup_vs_fp64": value / fp64["value"],
               "compat_value": compat["value"], "compat_frac": roofc["frac"]}
        if precision:
            out["l2_err_1000"] = precision["l2"]
            out["linf_err_1000"] = precision["linf"]
        if adjoint:
            out["adjoint_forward_ratio"] = adjoint["ratio"]
            out["adjoint_fd_err"] = adjoint["fd_check"]["max_rel_err"]
        if p5:
            out["p5_value"] = p5["mixed"]["value"]
            out["p5_speedup_vs_fp64"] = p5["speedup_vs_fp64"]
            out["p5_split_bf16_value"] = p5["split_bf16"]["value"]
            out["p5_split_bf16_speedup_vs_fp64"] = p5["split_bf16"]["speedup_vs_fp64"]
            if "errors" in p5:
                out["p5_l2_err_1000"] = p5["errors"]["l2"]
                out["p5_split_bf16_l2_err_1000"] = p5["errors"]["split_bf16_l2"]
        if parts:
            parts["vs_whole"] = parts["value"] / value
            out["parts4_vs_whole"] = parts["vs_whole"]
        if shear:
            out["mixed_mesh_speedups"] = [round(c["speedup_vs_fp64"], 3) for c in shear["cases"]]
        if world == 1 and not args.no_cpu_baseline:
            out["cpu_baseline"] = cpu_baseline(mesh, args.cpu_seconds, "ns")
        if args.detail:
            with open(args.detail, "w") as f:
                json.dump(dict(out, detail=detail), f, indent=1)
    ranks.close()
    return out


def p5_precision_case(stream, args, n=512, steps_err=1000):
    """The precision form of the Taylor-Green case on 512x512 jittered quads
    (seed 2) at P5 (36 solution points, 9.4 M DOF per variable), Navier-Stokes
    Re 5000, Roe, HU: DOF-RHS/s of the precision form, of its split-BF16
    variant (tensor-core operator products) and of the FP64 path
    (CUDA events over min(args.steps, 100) steps after args.warmup), and the
    L2 / Linf error of the precision form against the FP64 path after 1000
    steps, with the FP64 conditioning floor (FP64 from the initial state
    rounded once to FP32).  Both at CFL 0.3: at 512x512 and P5 the explicit
    viscous limit is below the convective step at CFL 0.5 (the FP64 path
    diverges within 50 steps there; inviscid, or at 256x256, CFL 0.5 is
    stable)."""
    import torch
    from zhijian_b200 import meshgen as M
    from zhijian_b200.norms import state_errors
    from zhijian_b200.solver import FRSolver, make_params
    mesh = M.tgv_mesh(n, seed=2)

    def solver(prec):
        prm = make_params(poly_order=5, gamma=GAMMA, rho_inf=1.0, p_inf=1.0 / (GAMMA * MACH * MACH),
                          Mach=MACH, riemann="Roe", flux_type="HU", compat=False, viscous=True,
                          Re=5000.0, Pr=0.72, CFL=0.3, bcs=[(1, "slipwall")], precision=prec)
        sv = FRSolver(mesh, prm)
        sv.set_stream(stream.cuda_stream)
        return sv
    out = {"workload": f"TGV {n}x{n} jittered (seed 2) Q1 quads, P5, Navier-Stokes Re 5000, Roe, HU, SSP-RK3"}
    U0 = dt = None
    steps = min(args.steps, 100)
    for prec in ("fp64", "mixed", "split_bf16"):
        sv = solver(prec)
        if U0 is None:
            U0 = M.taylor_green(sv.solution_point_coords())
        sv.copyToDevice(U0)
        if dt is None:
            dt = sv.computeTimeStep()
        sv.advance(dt, args.warmup)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        sv.advance(dt, steps, sync=False)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / steps
        out[prec] = {"ms_per_step": ms, "value": sv.n_elem * sv.n_sp * 3 / (ms * 1e-3), "steps": steps}
        sv.close()
    out["speedup_vs_fp64"] = out["mixed"]["value"] / out["fp64"]["value"]
    out["split_bf16"]["speedup_vs_fp64"] = out["split_bf16"]["value"] / out["fp64"]["value"]
    if not args.no_error_run:
        s64, s32, sbf, sfl = solver("fp64"), solver("mixed"), solver("split_bf16"), solver("fp64")
        for sv, U in ((s64, U0), (s32, U0), (sbf, U0), (sfl, U0.astype(np.float32).astype(np.float64))):
            sv.copyToDevice(U)
            sv.advance(dt, steps_err)
        U64, U32, Ubf, Ufl = s64.copyToHost(), s32.copyToHost(), sbf.copyToHost(), sfl.copyToHost()
        for sv in (s64, s32, sbf, sfl):
            sv.close()
        e, eb, fl = state_errors(U32, U64), state_errors(Ubf, U64), state_errors(Ufl, U64)
        out["errors"] = {"steps": steps_err, "dt": dt, "cfl": 0.3, "vars": ["rho", "rhou", "rhov", "rhoE"],
                         "l2": e["l2"], "linf": e["linf"], "fp64_floor_l2": fl["l2"],
                         "split_bf16_l2": eb["l2"], "split_bf16_linf": eb["linf"]}
    return out


# CFL per order for the shear layer: the reference's convective time step,
# kept under the explicit viscous limit of the 384x384 mesh (P3 at CFL 0.5
# diverges within 20 steps on quads alone; the SD correction at P4 needs the
# smallest value).
SHEAR_CFL = {2: 0.2, 3: 0.1, 4: 0.02}


def shear_layer_sweep(stream, args, n=384, steps_err=200):
    """The mixed-element case: 384x384 quads on [0,1]^2 with a seeded (seed 3)
    30% split into two triangles each, the Navier-Stokes shear layer (Re 2000,
    M 0.3), HLLC, slip walls at y = 0, 1 and a far field at rest at x = 0, 1
    (meshgen.SHEAR_LAYER_PARAMS); P2, P3, P4
    with the SD and GA corrections.  Per case: DOF-RHS/s of the precision form
    and of the FP64 path (CUDA events, min(args.steps, 50) steps after
    args.warmup), and the L2 / Linf error of the precision form against the
    FP64 path after `steps_err` steps at SHEAR_CFL[P], over the solution
    points in use (triangles hold (P+1)(P+2)/2 of their (P+1)^2 slots).  The
    layer is Kelvin-Helmholtz unstable: the FP32 rounding seeds a physical
    instability, so the difference grows with time (after 1000 steps it is
    1e-5 to 1e-3 in rho u, and P4 with SD diverges between 600 and 1000
    steps); 200 steps keep every case inside its stable window."""
    import torch
    from zhijian_b200 import meshgen as M
    from zhijian_b200.norms import state_errors
    from zhijian_b200.solver import FRSolver, make_params
    mesh = M.shear_layer_mesh(n)
    kinds = None
    cases = []
    for P in (2, 3, 4):
        for flux in ("SD", "GA"):
            def solver(prec):
                prm = make_params(poly_order=P, flux_type=flux, CFL=SHEAR_CFL[P], precision=prec,
                                  **M.SHEAR_LAYER_PARAMS)
                sv = FRSolver(mesh, prm)
                sv.set_stream(stream.cuda_stream)
                return sv
            case = {"P": P, "flux_type": flux, "cfl": SHEAR_CFL[P]}
            U0 = dt = None
            steps = min(args.steps, 50)
            for prec in ("fp64", "mixed"):
                sv = solver(prec)
                if U0 is None:
                    U0 = M.shear_layer(sv.solution_point_coords())
                    kinds = sv.element_kinds()
                    mask = sv.slot_mask()
                    case["dof_per_var"] = int(mask.sum())
                sv.copyToDevice(U0)
                if dt is None:
                    dt = sv.computeTimeStep()
                sv.advance(dt, args.warmup)
                torch.cuda.synchronize()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                sv.advance(dt, steps, sync=False)
                e1.record(stream)
                torch.cuda.synchronize()
                ms = e0.elapsed_time(e1) / steps
                case[prec] = {"ms_per_step": ms, "value": case["dof_per_var"] * 3 / (ms * 1e-3), "steps": steps}
                sv.close()
            case["speedup_vs_fp64"] = case["mixed"]["value"] / case["fp64"]["value"]
            if not args.no_error_run:
                s64, s32 = solver("fp64"), solver("mixed")
                for sv in (s64, s32):
                    sv.copyToDevice(U0)
                    sv.advance(dt, steps_err)
                U64, U32 = s64.copyToHost()[mask], s32.copyToHost()[mask]
                for sv in (s64, s32):
                    sv.close()
                e = state_errors(U32, U64)
                case["errors"] = {"steps": steps_err, "dt": dt, "finite": bool(np.isfinite(U64).all()),
                                  "l2": e["l2"], "linf": e["linf"]}
            cases.append(case)
    return {"workload": f"shear layer {n}x{n} quads, seeded 30% split into triangles "
                        f"({int((kinds == 0).sum())} triangles, {int((kinds == 1).sum())} quads), "
                        "Navier-Stokes Re 2000 M 0.3, far field at rest, HLLC, SSP-RK3",
            "unit": UNIT, "vars": ["rho", "rhou", "rhov", "rhoE"], "cases": cases}


def adjoint_run(stream, steps=200, k_ckpt=20, n_fd=4):
    """Discrete adjoint of the Taylor-Green case on 128x128 jittered quads
    (seed 4), P3, Roe, Re 5000, 200 SSP-RK3 steps at CFL 0.5, checkpoints
    every 20 steps; J = domain integral of the kinetic energy at the final
    time.  Device times of the checkpointed forward sweep and of the backward
    sweep (recomputation included), the device memory of the checkpoints and
    segment states, and central differences (h = 1e-6) on n_fd smooth seeded
    directions as a spot check (the 64-direction check is in tests/)."""
    import math
    import torch
    from zhijian_b200 import meshgen as M
    from zhijian_b200.objectives import kinetic_energy, quadrature_weights
    from zhijian_b200.solver import FRSolver, make_params
    mesh = M.tgv_mesh(128, seed=4)
    prm = make_params(poly_order=P, gamma=GAMMA, rho_inf=1.0, p_inf=1.0 / (GAMMA * MACH * MACH), Mach=MACH,
                      riemann="Roe", flux_type="HU", compat=False, viscous=True, Re=5000.0, Pr=0.72,
                      bcs=[(1, "slipwall")])
    s = FRSolver(mesh, prm)
    s.set_stream(stream.cuda_stream)
    U0 = M.taylor_green(s.solution_point_coords())
    s.copyToDevice(U0)
    dt = s.computeTimeStep()
    wq = quadrature_weights(mesh, P)

    def J_of(U):
        s.copyToDevice(U)
        s.advance(dt, steps)
        return kinetic_energy(s.copyToHost(), wq)
    _, Gf = J_of(U0)
    runs = []
    for _ in range(2):                       # the first call also builds the buffers
        s.copyToDevice(U0)
        G = torch.from_numpy(Gf.copy()).cuda()
        torch.cuda.synchronize()
        info = s.adjoint_run(dt, steps, k_ckpt, G.data_ptr())
        runs.append(info)
    g = G.cpu().numpy()
    info = runs[-1]
    n = 128
    errs = []
    for d in range(n_fd):
        c = M.uniform01(5 + d, 64).reshape(4, 4, 4) * 2.0 - 1.0
        ii, jj = np.meshgrid(np.arange(n), np.arange(n))
        x = (ii.ravel() + 0.5) / n * math.pi
        y = (jj.ravel() + 0.5) / n * math.pi
        V = np.zeros_like(U0)
        for v in range(4):
            f = sum(c[v, a, b] * np.sin((a + 1) * x) * np.sin((b + 1) * y) for a in range(4) for b in range(4))
            V[..., v] = f[:, None]
        V *= np.abs(U0).max(axis=(0, 1))
        h = 1e-6
        fd = (J_of(U0 + h * V)[0] - J_of(U0 - h * V)[0]) / (2 * h)
        errs.append(abs(float(np.sum(g * V)) - fd) / abs(fd))
    s.close()
    return {"workload": "TGV 128x128 jittered (seed 4) Q1 quads, P3, Roe, HU, Navier-Stokes Re 5000, "
                        f"{steps} SSP-RK3 steps at CFL 0.5, checkpoints every {k_ckpt} steps, "
                        "J = integral of 1/2 rho |u|^2 at the final time",
            "ms_forward": info["ms_forward"], "ms_adjoint": info["ms_adjoint"],
            "ratio": info["ms_adjoint"] / info["ms_forward"],
            "device_bytes": info["bytes"], "dJ_dRe": info["dRe"],
            "fd_check": {"h": 1e-6, "directions": n_fd, "max_rel_err": max(errs)}}


def partition_case(mesh, args, nparts=4, mode="ns32"):
    """The headline workload split into `nparts` RCB parts on this one GPU and
    stepped by the multi-part driver (each part on its own stream; after each
    launch that writes traces the cut-face rows are gathered, copied into the
    neighbours' buffers and scattered into their ghost rows; one captured
    graph per step once the first call has run): DOF-RHS/s and its ratio to
    the whole-mesh handle on the same GPU.  It measures the cost of the
    exchange machinery, not a link: every copy stays on one device."""
    import torch
    from zhijian_b200 import meshgen as M
    from zhijian_b200.partition import PartitionedSolver
    parts = PartitionedSolver(mesh, make_params_for(mode), nparts)
    streams = [torch.cuda.Stream() for _ in range(nparts)]
    for p, st in zip(parts.parts, streams):
        p.set_stream(st.cuda_stream)
    parts.copyToDevice(M.taylor_green(parts.solution_point_coords()))
    parts.advance(DT, max(args.warmup, 3))
    torch.cuda.synchronize()
    steps = max(args.steps, 20)
    e0 = torch.cuda.Event(enable_timing=True)
    e0.record(streams[0])
    for st in streams[1:]:
        st.wait_event(e0)
    parts.advance(DT, steps, sync=False)
    ends = []
    for st in streams:
        ev = torch.cuda.Event(enable_timing=True)
        ev.record(st)
        ends.append(ev)
    torch.cuda.synchronize()
    ms = max(e0.elapsed_time(ev) for ev in ends)
    for p in parts.parts:
        p.check_state()
    parts.close()
    dof = mesh.n_elem * (P + 1) ** 2
    return {"workload": workload_name(mode) + f", precision form, {nparts} RCB parts on one GPU",
            "value": dof * 3 * steps / (ms * 1e-3), "ms_per_step": ms / steps, "steps": steps}


def precision_errors(mesh, stream, steps=1000):
    """L2 / Linf error of the precision form against the FP64 path after
    `steps` SSP-RK3 steps at CFL 0.5 from the Taylor-Green state (the FP64 GPU
    path matches the FP64 oracle to 1e-12 per residual, tests/), with the FP64
    conditioning floor: the FP64 path from the initial state rounded once to
    FP32."""
    from zhijian_b200 import meshgen as M
    from zhijian_b200.norms import state_errors
    s64, s32, sfl = make_solver(mesh, "ns"), make_solver(mesh, "ns32"), make_solver(mesh, "ns")
    U0 = M.taylor_green(s64.solution_point_coords())
    s64.copyToDevice(U0)
    dt = s64.computeTimeStep()
    for s, U in ((s64, U0), (s32, U0), (sfl, U0.astype(np.float32).astype(np.float64))):
        s.set_stream(stream.cuda_stream)
        s.copyToDevice(U)
        s.advance(dt, steps)
    U64, U32, Ufl = s64.copyToHost(), s32.copyToHost(), sfl.copyToHost()
    for s in (s64, s32, sfl):
        s.close()
    e, fl = state_errors(U32, U64), state_errors(Ufl, U64)
    return {"steps": steps, "dt": dt, "cfl": 0.5, "vars": ["rho", "rhou", "rhov", "rhoE"],
            "against": "FP64 GPU path (= FP64 oracle to 1e-12 per residual)",
            "l2": e["l2"], "linf": e["linf"], "l2_abs": e["l2_abs"], "linf_abs": e["linf_abs"],
            "fp64_floor_l2": fl["l2"],
            "fp64_floor": "FP64 run from the initial state rounded once to FP32"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--no-error-run", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--no-p5", action="store_true")
    ap.add_argument("--no-mixed", action="store_true")
    ap.add_argument("--no-parts", action="store_true")
    ap.add_argument("--detail", default=None, help="also write every sub-result to this JSON file")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        out = run_reference(args)
    else:
        from zhijian_b200 import build
        build.build()
        out = run_ours(args)
    if out is not None:
        print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
