"""Benchmark of the matrix-free operators.

Headline workload (config 2, `--workload heat`): unit cube, 64^3 hexahedra with
interior vertices displaced by U[-0.1h, 0.1h] (PCG64 seed 2), FE_Q(4)
(16,974,593 DoFs), heat operator M/dt + div(k(T) grad) with
k(T) = k0 (1 + 1e-3 T), k0 = 1, rho c_p = 1, dt = 1e-3, T ~ U[300, 3000]
(seed 3), Dirichlet T = 0 on all faces.  A step is one FP64 operator apply
(vmult) with all data resident in HBM; value = DoFs x steps / time (whole job:
N GPUs run independent replicas).  After the timed steps the same operator is
solved with CG + Chebyshev(5)/Jacobi to a relative residual of 1e-10 in the
plain FP64 form and in the FP32-inner / FP64-defect-correction form (solves/s,
p50/p99 latency over repeated solves, and each form's true relative residual
under the oracle's FP64 operator).

With no --workload flag (N = 1) the line also carries, as extra keys, the
other configurations measured in the same run:
  c1  16^3 Q2 heat (35,937 DoFs): vmult (launch-latency bound), CG + Jacobi;
  c3  128^3 Q2 advection-diffusion, vortex velocity, theta = 0.5, D = 1e-3:
      vmult FP64 / FP32, one theta-scheme step of phi0 = tanh(d / 0.01)
      solved with GMRES(30) + Jacobi in both forms;
  c4  256 independent heat solves advanced together (batch_problems), against
      the plain FP64 GPU form of the same problems;
  c5  the Poisson request stream of serve_requests (20,000 requests at
      200 req/s) served by the continuous-batching loop, plus a stream below
      the device's capacity (engine latency without queueing), against the
      plain FP64 GPU form.

`--impl reference` times the tuned CPU port of the reference's operator
(oracle/cpu_port.cpp: compile-time degree, SIMD over cell batches, OpenMP over
colour-ordered batches, geometry and k(T_q) precomputed, -march=native): the
reference itself needs deal.II/Trilinos/p4est/MPI, which this image does not
have.  Each step is one full apply with all host threads.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "mat-free DoFs/s & solves/s, FP32+FP64-refined vs FP64 at 1e-10; p50/p99 latency"
DT, K0, K_ALPHA = 1e-3, 1.0, 1e-3
THETA, DIFFUSIVITY = 0.5, 1e-3
# the current single-operator workload: name ("heat" = config 2, "advdiff" =
# config 3, "c1" = config 1), cells per direction and degree
WL = {"name": "heat", "nc": [64, 64, 64], "degree": 4}

# dram__bytes_read.sum + dram__bytes_write.sum of the FP64 warp apply kernel
# (default schedule: CTA cell groups), per apply (8 colour launches): the heat
# workload's 48^3 capture of profiles/warp_apply_q4_general_48c.md (286.9 MB
# over two colour launches, 1,147.6 MB per apply of 110,592 cells) scaled by
# the cells of a 64^3 apply (262,144 / 110,592), as traffic grows with the
# cells processed; the level-set workload's capture is at full size
# (profiles/warp_apply_q2_uniform_128c.md: 381.4 MB over two launches).  The
# lane apply (one thread per Q2 cell, the level-set workload's default) was
# captured at full size over all 8 colour launches of an apply with the cache
# left warm between launches (profiles/lane_apply_q2_uniform_128c.md: 481.8 MB
# read, 298.4 MB written).
MEASURED_TRAFFIC_BYTES = {("heat", 64, "warp"): 2.720e9, ("advdiff", 128, "warp"): 1.526e9,
                         ("advdiff", 128, "lane"): 0.780e9}


def set_workload(name, cells=0):
    WL["name"] = name
    if name == "advdiff":
        WL["degree"], WL["nc"] = 2, [cells or 128] * 3
    elif name == "c1":
        WL["degree"], WL["nc"] = 2, [cells or 16] * 3
    else:
        WL["degree"], WL["nc"] = 4, [cells or 64] * 3


def n_dofs_of():
    return int(np.prod([n * WL["degree"] + 1 for n in WL["nc"]]))


def algorithmic_bytes(n_dofs, n_cells, degree, real_bytes):
    """Algorithmic bytes of one apply (the accounting of the hot-path scope
    table): s (N_src + N_dst) + s N_aux + s G + 4 E, with N_aux = N (the
    temperature read for k(T)) and G = 10 geometry values per quadrature point
    (J^-T and JxW) on the perturbed heat mesh, and N_aux = G = 0 on the uniform
    meshes; 4 E = one cell index per cell."""
    nq = (degree + 1) ** 3
    if WL["name"] in ("advdiff", "c1"):
        return real_bytes * 2 * n_dofs + 4 * n_cells
    return real_bytes * (3 * n_dofs) + real_bytes * 10 * nq * n_cells + 4 * n_cells


def streamed_bytes(n_dofs, n_cells, degree, real_bytes):
    """Bytes this implementation must stream per apply: src read, dst write and,
    on the perturbed mesh, the merged coefficient stream (c_mass JxW and the 6
    entries of c_diff k(T_q) JxW J^-1 J^-T per quadrature point, which folds the
    temperature and the geometry into 7 values)."""
    nq = (degree + 1) ** 3
    if WL["name"] in ("advdiff", "c1"):
        return real_bytes * 2 * n_dofs
    return real_bytes * (2 * n_dofs) + real_bytes * 7 * nq * n_cells


def algorithmic_flops(n_cells, degree):
    """Algorithmic flops of one apply (the hot-path scope table's secondary
    roofline): E (24 n^4 + c_q n^3), c_q = 20 on Cartesian heat cells, 45 on
    general geometry (the J^-T transforms), 60 with the analytic velocity."""
    n = degree + 1
    c_q = {"advdiff": 60, "c1": 20}.get(WL["name"], 45)
    return n_cells * (24 * n ** 4 + c_q * n ** 3)


def apply_kernel_name(op, p, geom):
    """The FP64 apply kernel the operator's schedule runs."""
    sc = op.schedule("fp64")
    if sc["lane_cells"] and geom == "UNIFORM" and p <= 2:
        return f"lane_apply_kernel<{p},double> x {4 if WL['nc'][0] <= 32 else 8} colour launches"
    return f"warp_apply_kernel<{p},double,{geom}> x 8 colour launches"


def fma_peaks(M):
    """Measured FMA throughput (GFLOP/s) in FP64 and FP32 (mpdg_fma_peak)."""
    import ctypes as C
    g64, g32 = C.c_double(0.0), C.c_double(0.0)
    M._capi.check(M._capi.lib().mpdg_fma_peak(C.byref(g64), C.byref(g32)), "fma_peak")
    return g64.value, g32.value


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu):
        self.gpu = gpu
        self.proc = None
        self.path = os.path.join("/tmp", f"mpdg_clocks_{os.getpid()}_{id(self)}.csv")

    def __enter__(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "50"], stdout=self.f,
                stderr=subprocess.DEVNULL)
            # wait for the first sample so the timed region is covered
            t0 = time.time()
            while time.time() - t0 < 5.0 and os.path.getsize(self.path) == 0:
                time.sleep(0.05)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self):
        if self.proc is None or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def job_seconds(t_local, world):
    """The job's time: the maximum of the ranks' device-timed regions (one
    all-reduce; on NCCL through a CUDA tensor, on gloo through a CPU one)."""
    if world <= 1:
        return t_local
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    tt = torch.tensor([t_local], dtype=torch.float64, device=dev)
    dist.all_reduce(tt, op=dist.ReduceOp.MAX)
    return float(tt)


def replica_throughput(units_per_rank, world, t_job):
    """Whole-job throughput of N independent replicas (weak scaling, no exchange
    step): all ranks' units over the slowest rank's time."""
    return units_per_rank * world / t_job


def percentiles(lat_s):
    lat = np.sort(np.asarray(lat_s, dtype=np.float64))
    return {"p50_ms": 1e3 * float(np.percentile(lat, 50)), "p99_ms": 1e3 * float(np.percentile(lat, 99)),
            "max_ms": 1e3 * float(lat[-1]), "samples": int(lat.size)}


# ------------------------------------------------------------ problem set-up
def mesh_inputs():
    """(vertices, Dirichlet mask or None, temperature or None) of the workload."""
    from meltpooldg_b200.operators import box_vertices, boundary_mask
    nc, p = WL["nc"], WL["degree"]
    if WL["name"] == "advdiff":
        return box_vertices(nc), None, None
    if WL["name"] == "c1":
        return box_vertices(nc), boundary_mask(nc, p), None
    V = box_vertices(nc, perturb=0.1, seed=2)
    T = np.random.Generator(np.random.PCG64(3)).uniform(300.0, 3000.0, n_dofs_of())
    return V, boundary_mask(nc, p), T


def make_operator(M, mesh, T):
    import torch
    if WL["name"] == "advdiff":
        return M.AdvectionDiffusionOperator(mesh, DT, theta=THETA, diffusivity=DIFFUSIVITY,
                                            velocity="vortex", precisions=("fp64", "fp32")), None
    if WL["name"] == "c1":
        return M.HeatDiffuseOperator(mesh, DT, rho_cp=1.0, k0=1.0, precisions=("fp64", "fp32")), None
    op = M.HeatDiffuseOperator(mesh, DT, rho_cp=1.0, k0=K0, k_alpha=K_ALPHA, precisions=("fp64", "fp32"))
    Td = torch.tensor(T, device="cuda")
    op.set_temperature(Td)
    return op, Td


def workload_config():
    N, E = n_dofs_of(), int(np.prod(WL["nc"]))
    name = {"advdiff": "advection-diffusion operator apply, Q2, 128^3 uniform hex cells, vortex velocity, "
                       "theta=0.5, D=1e-3",
            "c1": "heat operator apply, Q2, 16^3 uniform hex cells, k=1, dt=1e-3, Dirichlet faces",
            }.get(WL["name"], "heat operator apply, Q4, 64^3 perturbed hex cells, k(T)=k0(1+1e-3T)")
    return {"workload": name, "n_dofs": N, "cells": E, "degree": WL["degree"]}


# ------------------------------------------------------------ CPU legs (port and oracle)
def port_operator():
    """The tuned CPU port of the workload's operator (oracle/cpu_port.cpp)."""
    from oracle import cpu_port as P
    V, mask, T = mesh_inputs()
    nc, p = WL["nc"], WL["degree"]
    if WL["name"] == "advdiff":
        return P.PortOperator(V, nc, p, None, uniform=True, kind=1, dt=DT, theta=THETA, diffusivity=DIFFUSIVITY,
                              velocity="vortex")
    if WL["name"] == "c1":
        return P.PortOperator(V, nc, p, mask, uniform=True, kind=0, dt=DT, rho_cp=1.0, k0=1.0)
    return P.PortOperator(V, nc, p, mask, uniform=False, kind=0, dt=DT, rho_cp=1.0, k0=K0, k_alpha=K_ALPHA,
                          temperature=T)


def cpu_apply_rate(seconds=5.0, port=None):
    """The port's full applies on all host threads for about `seconds` (after 3
    warm-up applies); returns the cpu_baseline dict."""
    from oracle import cpu_port as P
    own = port is None
    port = port or port_operator()
    N = port.n_dofs
    src = np.random.Generator(np.random.PCG64(0)).uniform(-1.0, 1.0, N)
    dst = np.zeros(N)
    for _ in range(3):
        port.vmult(dst, src)
    reps, t0 = 0, time.perf_counter()
    while True:
        port.vmult(dst, src)
        reps += 1
        dt = time.perf_counter() - t0
        if dt > seconds:
            break
    if own:
        port.close()
    return {"value": N * reps / dt, "unit": "DoFs/s", "cores": P.threads(), "kind": "port",
            "sample": f"{reps} full applies of the workload in {dt:.2f} s (after 3 untimed), "
                      "tuned C++ port (oracle/cpu_port.cpp, -O3 -march=native, OpenMP)"}


def oracle_true_residual(b_host, x_host):
    """|b - A x| / |b| with A the oracle's FP64 operator of the workload: the
    error of a device solve stated against the oracle."""
    from oracle import oracle as O
    V, mask, T = mesh_inputs()
    om = O.Mesh(3, WL["degree"], WL["nc"], V)
    if WL["name"] == "advdiff":
        oop = O.Operator(O.ADVDIFF, DT, theta=THETA, diffusivity=DIFFUSIVITY, vel_kind=O.VEL_VORTEX)
    elif WL["name"] == "c1":
        oop = O.Operator(O.HEAT, DT, rho_cp=1.0, k0=1.0, dirichlet=mask)
    else:
        oop = O.Operator(O.HEAT, DT, rho_cp=1.0, k0=K0, k_alpha=K_ALPHA, temperature=T, dirichlet=mask)
    r = b_host - O.vmult(om, oop, x_host)
    return float(np.linalg.norm(r) / np.linalg.norm(b_host))


# ------------------------------------------------------------ reference arm
def run_reference(args, rank, world):
    """The reference's CPU path, restated as the tuned port, on the headline
    workload: each step one full apply with all host threads."""
    if rank != 0:
        return
    from oracle import cpu_port as P
    port = port_operator()
    N = port.n_dofs
    src = np.random.Generator(np.random.PCG64(0)).uniform(-1.0, 1.0, N)
    dst = np.zeros(N)
    for _ in range(max(args.warmup, 3)):
        port.vmult(dst, src)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        port.vmult(dst, src)
        times.append(time.perf_counter() - t0)
    port.close()
    tot = sum(times)
    value = N * args.steps / tot
    cores = P.threads()
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "DoFs/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": dict(workload_config(), parallelism=f"OpenMP x{cores}"),
        "cpu_baseline": {"value": value, "unit": "DoFs/s", "cores": cores, "kind": "port",
                         "sample": f"{args.steps} full applies of the workload (one per step)"},
        "e2e": {"value": value, "unit": "DoFs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "tuned C++ port of the reference's operator (oracle/cpu_port.cpp: compile-time degree, "
                "SIMD batches of 8 cells, OpenMP over colour-ordered batches, geometry and k(T_q) "
                "precomputed, -O3 -march=native); the reference needs deal.II + Trilinos + p4est + MPI, "
                "absent from this image",
    }
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------ single-operator workloads
def solve_inputs(op, mask, N):
    """The workload's linear system: (b, exact solution or None, solver, preconditioner)."""
    import torch
    nc, p = WL["nc"], WL["degree"]
    if WL["name"] == "advdiff":
        # one theta-scheme step of the tanh level set
        X = [np.linspace(0.0, 1.0, n * p + 1) for n in nc]  # Q2 Gauss-Lobatto nodes are uniform
        Z, Y, Xg = np.meshgrid(X[2], X[1], X[0], indexing="ij")
        d = 0.25 - np.sqrt((Xg - 0.5) ** 2 + (Y - 0.75) ** 2 + (Z - 0.5) ** 2)
        phi0 = torch.tensor(np.tanh(d / 0.01).reshape(-1), device="cuda")
        b = torch.zeros_like(phi0)
        op.create_rhs(b, phi0)
        return b, None, "GMRES", "Diagonal"
    seed = 1 if WL["name"] == "c1" else 5
    xs = torch.tensor(np.random.Generator(np.random.PCG64(seed)).uniform(-1, 1, N), device="cuda")
    xs[torch.tensor(mask.astype(bool), device="cuda")] = 0.0
    b = torch.empty_like(xs)
    op.vmult(b, xs)
    return b, xs, "CG", ("Diagonal" if WL["name"] == "c1" else "Chebyshev")


def run_profile_solve(args):
    """One solve of the workload's system in the given form after an untimed
    warm-up solve, inside a cudaProfilerStart/Stop range (for
    `ncu --profile-from-start off`); prints the solve's report."""
    import torch
    import meltpooldg_b200 as M
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
    V, mask, T = mesh_inputs()
    mesh = M.Mesh(V, WL["nc"], WL["degree"], mask)
    op, Td = make_operator(M, mesh, T)
    b, _, solver_type, prec = solve_inputs(op, mask, mesh.n_dofs)
    data = M.LinearSolverData(solver_type=solver_type, preconditioner_type=prec, rel_tolerance=1e-10,
                              abs_tolerance=1e-20, mixed_precision=args.profile_solve == "fp32_refined")
    x = torch.zeros_like(b)
    M.LinearSolver.solve(op, x, b, data)
    torch.cuda.synchronize()
    x.zero_()
    torch.cuda.cudart().cudaProfilerStart()
    M.LinearSolver.solve(op, x, b, data)
    torch.cuda.synchronize()
    torch.cuda.cudart().cudaProfilerStop()
    print(json.dumps({"profile_solve": args.profile_solve, "workload": WL["name"],
                      "report": dict(M.LinearSolver.last_report)}), flush=True)


def run_operator_workload(args, rank, world, headline):
    """One apply workload (config 2, 3 or 1): timed FP64 applies, FP32 applies,
    the multi-vector pass, the host-buffer e2e apply, the solves, the CPU
    baseline.  Returns the line's dict (printed by the caller)."""
    import torch
    import torch.distributed as dist
    import meltpooldg_b200 as M
    local = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(local)
    V, mask, T = mesh_inputs()
    nc, p = WL["nc"], WL["degree"]
    mesh = M.Mesh(V, nc, p, mask)
    N = mesh.n_dofs
    op, Td = make_operator(M, mesh, T)
    # the library's autotuner picks the apply schedule per precision (untimed);
    # --no-autotune keeps the operator's default schedule (profiling runs)
    tuned = {} if args.no_autotune else {prec: op.autotune(prec, reps=10)[:2] for prec in ("fp64", "fp32")}
    rng = np.random.Generator(np.random.PCG64(0))
    src = torch.tensor(rng.uniform(-1.0, 1.0, N), device="cuda")
    dst = torch.empty_like(src)
    src32, dst32 = src.float(), torch.empty(N, dtype=torch.float32, device="cuda")
    steps = args.steps if headline else max(20, min(args.steps, 200))

    def barrier():
        if world > 1:
            dist.barrier()

    for _ in range(max(args.warmup, 3)):
        op.vmult(dst, src)
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    launches0 = M.kernel_launches()
    stream = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        e0.record(stream)
        for _ in range(steps):
            op.vmult(dst, src)
        e1.record(stream)
        torch.cuda.synchronize()
    launches = M.kernel_launches() - launches0
    barrier()
    t = e0.elapsed_time(e1) / 1e3
    t_max = job_seconds(t, world)
    value = replica_throughput(N * steps, world, t_max)
    apply_s = t / steps

    # FP32 apply
    for _ in range(3):
        op.vmult(dst32, src32)
    e0.record(stream)
    for _ in range(steps):
        op.vmult(dst32, src32)
    e1.record(stream)
    torch.cuda.synchronize()
    apply32_s = e0.elapsed_time(e1) / 1e3 / steps

    multi = None
    if headline:
        # multi-vector apply: 4 operands per pass share one read of the
        # coefficients (the images of the least-squares predictor, mpdg_vmult_multi)
        srcs = [src] + [torch.roll(src, 7 * v) for v in range(1, 4)]
        dsts = [dst] + [torch.empty_like(src) for _ in range(3)]
        for _ in range(3):
            op.vmult_multi(dsts, srcs)
        multi_steps = max(3, steps // 4)
        e0.record(stream)
        for _ in range(multi_steps):
            op.vmult_multi(dsts, srcs)
        e1.record(stream)
        torch.cuda.synchronize()
        multi_s = e0.elapsed_time(e1) / 1e3 / multi_steps
        multi = {"vectors": 4, "ms_per_pass": 1e3 * multi_s, "value": 4 * N / multi_s, "unit": "DoFs/s",
                 "speedup_vs_4_single_applies": 4 * apply_s / multi_s}
        del srcs, dsts

    # end to end through the host-buffer C-ABI call (pinned host buffers)
    e2e_s = float("nan")
    if not args.no_e2e:
        hsrc = torch.empty(N, dtype=torch.float64).pin_memory()
        hdst = torch.empty(N, dtype=torch.float64).pin_memory()
        hsrc.copy_(src.cpu())
        hs, hd = hsrc.numpy(), hdst.numpy()
        op.vmult_host(hd, hs)
        e2e_steps = max(3, min(50, steps // 2))
        t0 = time.perf_counter()
        for _ in range(e2e_steps):
            op.vmult_host(hd, hs)
        e2e_s = (time.perf_counter() - t0) / e2e_steps

    peak, peak_kind = load_peaks()
    E = int(np.prod(nc))
    f64_peak, f32_peak = fma_peaks(M)
    flops = algorithmic_flops(E, p)
    geom = "UNIFORM" if WL["name"] in ("advdiff", "c1") else "GENERAL"
    b64, b32 = algorithmic_bytes(N, E, p, 8), algorithmic_bytes(N, E, p, 4)
    st64, st32 = streamed_bytes(N, E, p, 8), streamed_bytes(N, E, p, 4)
    kernel_kind = "lane" if apply_kernel_name(op, p, geom).startswith("lane") else "warp"
    traffic = MEASURED_TRAFFIC_BYTES.get((WL["name"], nc[0], kernel_kind))
    roof = {"bound": "hbm", "achieved": b64 / apply_s / 1e9, "peak": peak, "unit": "GB/s",
            "frac": b64 / apply_s / 1e9 / peak, "traffic": traffic,
            "traffic_note": None if traffic is None else
            ("ncu dram read+write per apply (8 launches), 48^3 capture scaled by cells" if WL["name"] == "heat"
             else f"ncu dram read+write per apply (8 {kernel_kind} apply launches), full-size capture"),
            "algorithmic_bytes": b64, "kernel": apply_kernel_name(op, p, geom),
            "peak_source": f"MEASURED_PEAKS.json hbm_gbs ({peak_kind})",
            "streamed": {"bytes": st64, "achieved": st64 / apply_s / 1e9, "frac": st64 / apply_s / 1e9 / peak},
            "fp32": {"achieved": b32 / apply32_s / 1e9, "frac": b32 / apply32_s / 1e9 / peak,
                     "algorithmic_bytes": b32, "streamed_bytes": st32,
                     "streamed_frac": st32 / apply32_s / 1e9 / peak},
            "flops": {"per_apply": flops, "unit": "GFLOP/s",
                      "fp64": {"achieved": flops / apply_s / 1e9, "peak": f64_peak,
                               "frac": flops / apply_s / 1e9 / f64_peak},
                      "fp32": {"achieved": flops / apply32_s / 1e9, "peak": f32_peak,
                               "frac": flops / apply32_s / 1e9 / f32_peak},
                      "peak_source": "mpdg_fma_peak: FMA chains measured on this GPU (8 per thread, 8 CTAs per SM)"}}

    # solves to 1e-10 in the plain FP64 form and the FP32-inner / FP64-refined form
    solves, solve_io = None, None
    if not args.no_solve:
        b, xs, solver_type, prec = solve_inputs(op, mask, N)
        solves = {"solver": f"{solver_type} + {prec}",
                  "timing": f"wall clock per solve, {args.solve_reps} solves after one untimed warm-up solve"}
        solve_io = {"b": b.cpu().numpy(), "x": {}}
        ref_x = None
        for form, mixed in (("fp64", False), ("fp32_refined", True)):
            data = M.LinearSolverData(solver_type=solver_type, preconditioner_type=prec,
                                      rel_tolerance=1e-10, abs_tolerance=1e-20, mixed_precision=mixed)
            lat = []
            rep = None
            for r in range(args.solve_reps + 1):
                x = torch.zeros_like(b)
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                M.LinearSolver.solve(op, x, b, data)
                torch.cuda.synchronize()
                if r > 0:
                    lat.append(time.perf_counter() - t0)
                rep = dict(M.LinearSolver.last_report)
            if ref_x is None:
                ref_x = x.clone()
            solve_io["x"][form] = x.cpu().numpy()
            err = float((x - ref_x).abs().max() / ref_x.abs().max())
            solves[form] = dict(
                percentiles(lat), solves_per_s=world / statistics.median(lat),
                iterations=rep["iterations"], outer_iterations=rep["outer_iterations"],
                operator_applies=rep["operator_applies"],
                relative_residual=rep["final_residual"] / rep["initial_residual"],
                lambda_max=rep["lambda_max"] or None,
                max_rel_error_vs_fp64_solution=err,
                max_rel_error_vs_exact=None if xs is None else float((x - xs).abs().max() / xs.abs().max()))
        solves["speedup_fp32_refined_vs_fp64"] = (solves["fp32_refined"]["solves_per_s"] /
                                                  solves["fp64"]["solves_per_s"])
    sched64, sched32 = op.schedule("fp64"), op.schedule("fp32")
    op.close()
    mesh.close()
    del src, dst, src32, dst32, Td
    torch.cuda.empty_cache()

    cpu = None
    if rank == 0 and not args.no_cpu:
        cpu = cpu_apply_rate(args.cpu_seconds)
        if solve_io is not None:
            # the CPU checker's view of every device solve: the true relative
            # residual under the oracle's FP64 operator
            for form, xh in solve_io["x"].items():
                solves[form]["true_relative_residual_vs_oracle"] = oracle_true_residual(solve_io["b"], xh)

    return {
        "metric": METRIC, "value": value, "unit": "DoFs/s", "n_gpus": world, "steps": steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * t_max / steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": dict(workload_config(), parallelism=f"replicas x{world}",
                       l2={"advdiff": "inputs larger than L2: src/dst 2 x 136 MB",
                           "c1": "inputs smaller than L2 (0.6 MB): launch-latency bound, L2 not flushed",
                           }.get(WL["name"], "inputs larger than L2: coefficient stream 1.8 GB per apply"),
                       schedule={"fp64": sched64, "fp32": sched32,
                                 "autotuned_ms": {k: v[1] for k, v in tuned.items()},
                                 "picked_by": "default schedule" if args.no_autotune else
                                 "mpdg_op_autotune (10 applies per candidate)"}),
        "roofline": roof,
        "cpu_baseline": cpu,
        "e2e": None if args.no_e2e else {
            "value": N / e2e_s, "unit": "DoFs/s", "h2d_bytes_per_step": 8 * N,
            "d2h_bytes_per_step": 8 * N, "call": "mpdg_vmult_host (pinned host buffers)"},
        "fp32_apply": {"value": N / apply32_s, "unit": "DoFs/s", "ms_per_apply": 1e3 * apply32_s},
        "multi_apply": multi,
        "solves": solves,
        "gpu_launches": launches,
        "clocks": clk.summary(),
    }


# ----------------------------------------------------------------- batched solves
BATCH_SIZE = 256


def batch_problems(n=BATCH_SIZE):
    """256 heat problems: n^3 cells with n ~ U{8..48}, degree ~ U{2,3,4},
    k0 log-uniform in [1, 100], rho c_p = 1, dt = 1e-3, Dirichlet on all faces,
    seeded right-hand sides (seed 100 + i); PCG64 seed 4 draws the shapes."""
    from meltpooldg_b200 import batch as B
    rng = np.random.Generator(np.random.PCG64(4))
    out = []
    for i in range(n):
        nc = int(rng.integers(8, 49))
        p = int(rng.choice([2, 3, 4]))
        k0 = float(np.exp(rng.uniform(0.0, np.log(100.0))))
        out.append(B.Problem(kind=B.OP_HEAT, degree=p, nc=nc, k0=k0, dt=1e-3, rho_cp=1.0,
                             rel_tolerance=1e-10, rhs_seed=100 + i))
    return out


def serve_requests(n_req, rate=200.0, seed=7):
    """Poisson arrivals (mean rate req/s, PCG64 seed 7): cells n^3 with
    n = min(96, round(LogNormal(ln 24, 0.5))), degree ~ U{2,3,4}, half heat
    (k0 = 1, rho c_p = 1) and half advection-diffusion (vortex velocity,
    theta = 0.5, D = 1e-3), dt = 1e-3, tolerance 1e-10, seeds 1000 + i."""
    from meltpooldg_b200 import batch as B
    rng = np.random.Generator(np.random.PCG64(seed))
    arr = np.cumsum(rng.exponential(1.0 / rate, size=n_req))
    out = []
    for i in range(n_req):
        nc = int(min(96, max(2, round(float(rng.lognormal(np.log(24.0), 0.5))))))
        p = int(rng.choice([2, 3, 4]))
        kind = B.OP_HEAT if rng.uniform() < 0.5 else B.OP_ADVDIFF
        out.append(B.Problem(kind=kind, degree=p, nc=nc, dt=1e-3, k0=1.0, rho_cp=1.0, theta=0.5,
                             diffusivity=1e-3, rel_tolerance=1e-10, rhs_seed=1000 + i))
    return out, arr


def single_fp64_solve(M, prob, b_host):
    """The plain FP64 GPU form of one problem: its own mesh and operator, CG
    (heat) or GMRES(30) (advection-diffusion) with Jacobi to 1e-10; returns
    (x on host, iterations)."""
    import torch
    nc = (prob.nc,) * 3
    mesh = M.Mesh(M.box_vertices(nc), nc, prob.degree, M.boundary_mask(nc, prob.degree))
    if prob.kind == 0:
        op = M.HeatDiffuseOperator(mesh, prob.dt, rho_cp=prob.rho_cp, k0=prob.k0)
        data = M.LinearSolverData(solver_type="CG", rel_tolerance=1e-10, abs_tolerance=0.0)
    else:
        op = M.AdvectionDiffusionOperator(mesh, prob.dt, theta=prob.theta, diffusivity=prob.diffusivity,
                                          velocity="vortex")
        data = M.LinearSolverData(solver_type="GMRES", rel_tolerance=1e-10, abs_tolerance=0.0)
    b = torch.from_numpy(b_host).to("cuda")
    x = torch.zeros_like(b)
    its = M.LinearSolver.solve(op, x, b, data)
    xh = x.cpu().numpy()
    op.close()
    mesh.close()
    return xh, its


def run_batch(args, rank, world):
    """Config 4: 256 independent heat solves advanced together, one graph launch
    per Krylov step.  A step is one whole batch: admission of the 256 problems
    (device right-hand sides), the solve of all to 1e-10, release."""
    import torch
    import meltpooldg_b200 as M
    from meltpooldg_b200 import batch as B
    local = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(local)
    probs = batch_problems(args.problems)
    n_dofs = [p.n_dofs for p in probs]
    N_total = int(sum(n_dofs))
    budget = 150 * 10**9
    steps = args.batch_steps

    def one_batch(e2e=False, tune=False, keep=False):
        rhs = [p.rhs() for p in probs] if e2e else None
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        with B.Batch(budget, capacity=len(probs)) as bt:
            ts = [bt.submit(p, rhs=rhs[i] if e2e else None) for i, p in enumerate(probs)]
            tune_res = (bt.autotune(), bt.shape()) if tune else None
            gsteps, _ = bt.run(poll_steps=16)
            res = [bt.take(t, p.n_dofs if (e2e or keep) else None) for t, p in zip(ts, probs)]
        t1 = time.perf_counter()
        return t1 - t0, gsteps, res, tune_res

    # warm-up (also the autotuner's pass over this membership)
    _, _, _, tune_res = one_batch(tune=True)
    (cap, apply_ms), shape = tune_res
    for _ in range(max(0, args.warmup - 1)):
        one_batch()
    launches0 = M.kernel_launches()
    times, graph_steps = [], []
    with ClockSampler(local) as clk:
        for _ in range(steps):
            dt, st, res, _ = one_batch()
            times.append(dt)
            graph_steps.append(st)
    launches = M.kernel_launches() - launches0
    reps = [r for _, r in res]
    t_step = float(np.mean(times))
    value = len(probs) * world / t_step

    # end to end: host right-hand sides in, host solutions out
    e2e_t, _, res_e2e, _ = one_batch(e2e=True)

    # the plain FP64 GPU form of the same problems, one after another
    t0 = time.perf_counter()
    errs, its64 = [], []
    for p, (xb, rb) in zip(probs, res_e2e):
        x64, it = single_fp64_solve(M, p, p.rhs())
        its64.append(it)
        errs.append(float(np.linalg.norm(xb - x64) / max(np.linalg.norm(x64), 1e-300)))
    t64 = time.perf_counter() - t0

    peak, peak_kind = load_peaks()
    E_total = int(sum(p.nc ** 3 for p in probs))
    b_apply = 2 * 4 * N_total + 4 * E_total  # FP32 src read + dst write and a cell index, every problem
    roof = {"bound": "hbm", "achieved": b_apply / (apply_ms * 1e-3) / 1e9, "peak": peak, "unit": "GB/s",
            "frac": b_apply / (apply_ms * 1e-3) / 1e9 / peak, "traffic": None,
            "algorithmic_bytes": b_apply,
            "kernel": f"batch_apply_kernel<float> x 8 colour launches over all {len(probs)} problems",
            "apply_ms": apply_ms, "autotuned_shape": shape,
            "peak_source": f"MEASURED_PEAKS.json hbm_gbs ({peak_kind})"}
    # box cells move ~8 bytes per DoF: the apply is bound by its arithmetic
    # (Cartesian heat cells: E (24 n^4 + 20 n^3) per problem), as the
    # single-problem applies of the same degrees are
    _, f32_peak = fma_peaks(M)
    f_apply = float(sum(p.nc ** 3 * (24 * (p.degree + 1) ** 4 + 20 * (p.degree + 1) ** 3) for p in probs))
    roof["flops"] = {"per_apply": f_apply, "unit": "GFLOP/s",
                     "fp32": {"achieved": f_apply / (apply_ms * 1e-3) / 1e9, "peak": f32_peak,
                              "frac": f_apply / (apply_ms * 1e-3) / 1e9 / f32_peak},
                     "dofs_per_s": N_total / (apply_ms * 1e-3),
                     "peak_source": "mpdg_fma_peak: FMA chains measured on this GPU (8 per thread, 8 CTAs per SM)"}
    cpu = None
    if rank == 0 and not args.no_cpu:
        cpu = cpu_batch_rate(probs, its64, args.cpu_seconds)
    iters = [r["iterations"] for r in reps]
    return {
        "metric": "batched heat solves/s at 1e-10 (FP32 apply, FP64 residuals)", "value": value,
        "unit": "solves/s", "n_gpus": world, "steps": steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * t_step, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 apply / f64 residuals", "data": "synthetic",
        "config": {"workload": f"{len(probs)} heat solves, n^3 cells n~U{{8..48}}, Q2/Q3/Q4, k0 log-uniform [1,100], "
                               "dt=1e-3, seeded rhs, CG + Jacobi to 1e-10",
                   "n_dofs_total": N_total, "problems": len(probs),
                   "l2": f"inputs larger than L2: {N_total * 44 / 1e9:.1f} GB resident",
                   "timing": "host clock around synchronous batch calls (admission to release)"},
        "roofline": roof, "cpu_baseline": cpu,
        "e2e": {"value": len(probs) / e2e_t, "unit": "solves/s", "h2d_bytes_per_step": 8 * N_total,
                "d2h_bytes_per_step": 8 * N_total,
                "call": "mpdg_batch_submit (host rhs) / mpdg_batch_run / mpdg_batch_take (host x)"},
        "fp64_plain": {"solves_per_s": len(probs) / t64, "seconds": t64,
                       "iterations_mean": float(np.mean(its64)),
                       "speedup_batched_vs_fp64": value / (len(probs) / t64)},
        "batched": {"graph_steps": graph_steps[-1], "iterations_mean": float(np.mean(iters)),
                    "iterations_max": int(max(iters)),
                    "all_converged": all(r["status"] == 0 for r in reps),
                    "max_rel_residual": max(r["final_residual"] / r["initial_residual"] for r in reps),
                    "max_rel_error_vs_fp64_solution": max(errs),
                    "iteration_diff_vs_fp64_max": int(max(abs(a - b) for a, b in zip(iters, its64)))},
        "gpu_launches": launches,
        "clocks": clk.summary(),
    }


def cpu_batch_rate(probs, its64, seconds):
    """The tuned CPU port's FP64 CG + Jacobi solves (diagonal by unit vectors
    per cell, as deal.II's compute_diagonal) of the smallest problems of the
    batch until about `seconds`; the rate per DoF-iteration scales to the whole
    batch (sum of n_dofs x FP64 iterations)."""
    from oracle import cpu_port as P
    from meltpooldg_b200 import box_vertices, boundary_mask
    order = np.argsort([p.n_dofs for p in probs])
    spent, work, done = 0.0, 0.0, 0
    for i in order:
        p = probs[i]
        nc = (p.nc,) * 3
        port = P.PortOperator(box_vertices(nc), nc, p.degree, boundary_mask(nc, p.degree), uniform=True, kind=0,
                              dt=p.dt, rho_cp=p.rho_cp, k0=p.k0)
        b = p.rhs()
        t0 = time.perf_counter()
        _, it, _ = port.cg_jacobi(b, rel_tol=1e-10, abs_tol=0.0)
        spent += time.perf_counter() - t0
        port.close()
        work += p.n_dofs * max(it, 1)
        done += 1
        if spent > seconds:
            break
    total_work = float(sum(p.n_dofs * max(it, 1) for p, it in zip(probs, its64)))
    rate = len(probs) / (spent * total_work / work)
    return {"value": rate, "unit": "solves/s", "cores": P.threads(), "kind": "port",
            "sample": f"port CG+Jacobi of the {done} smallest problems ({spent:.1f} s), scaled by "
                      f"n_dofs x iterations to all {len(probs)}"}


def serve_work(probs, reps, wall):
    """Iterations per kind and the operator applies the stream needed:
    DoF-applies = sum of n_dofs x applies (CG: 1 per iteration, BiCGStab: 2)."""
    out = {}
    total = 0.0
    for kind, name in ((0, "heat"), (1, "advdiff")):
        its = [r["iterations"] for p, r in zip(probs, reps) if p.kind == kind]
        work = sum(p.n_dofs * r["operator_applies"] for p, r in zip(probs, reps) if p.kind == kind)
        total += work
        if its:
            out[name] = {"requests": len(its), "iterations_mean": float(np.mean(its)),
                         "iterations_max": int(max(its)), "dof_applies": float(work)}
    out["dof_applies_per_s"] = total / wall
    return out


def run_serve(args, rank, world):
    """Config 5: Poisson stream of heat / advection-diffusion requests served by
    the library's loop (continuous batching, 150 GB admission budget), against
    the plain FP64 GPU form serving the same stream one request at a time; and
    the same kind of stream below the device's capacity, whose latencies are the
    engine's own rather than queueing."""
    import torch
    import meltpooldg_b200 as M
    from meltpooldg_b200 import batch as B
    local = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(local)
    n_req = args.requests
    probs, arr = serve_requests(n_req)
    budget = 150 * 10**9
    # warm-up: a short stream
    wp, wa = serve_requests(max(8, args.warmup * 4))
    with B.Batch(budget, capacity=4096) as bt:
        bt.serve(wp, wa * 0.0, poll_steps=4)
    keep = list(range(0, n_req, max(1, n_req // 32)))
    launches0 = M.kernel_launches()
    with ClockSampler(local) as clk:
        with B.Batch(budget, capacity=4096) as bt:
            out = bt.serve(probs, arr, poll_steps=args.poll_steps, keep_solutions=keep)
    launches = M.kernel_launches() - launches0
    reps = out["reports"]
    value = n_req / out["wall_s"]

    # below capacity: the same distribution of requests at a lower arrival rate
    low = None
    if args.low_rate > 0 and args.low_requests > 0:
        lp, la = serve_requests(args.low_requests, rate=args.low_rate, seed=8)
        with B.Batch(budget, capacity=4096) as bt:
            lo = bt.serve(lp, la, poll_steps=args.poll_steps)
        low = dict(percentiles(lo["latency_s"]), requests=args.low_requests, rate_req_per_s=args.low_rate,
                   solves_per_s=args.low_requests / lo["wall_s"],
                   all_converged=all(r["status"] == 0 for r in lo["reports"]))

    # plain FP64 GPU form on the same stream: one request at a time, FIFO
    fp64 = None
    if not args.no_fp64_arm:
        n64 = min(n_req, args.fp64_requests)
        lat64, errs = [], []
        t0 = time.perf_counter()
        for i in range(n64):
            now = time.perf_counter() - t0
            if arr[i] > now:
                time.sleep(arr[i] - now)
            x64, _ = single_fp64_solve(M, probs[i], probs[i].rhs())
            lat64.append(time.perf_counter() - t0 - arr[i])
            if out["solutions"] is not None and out["solutions"][i] is not None:
                xb = out["solutions"][i]
                errs.append(float(np.linalg.norm(xb - x64) / max(np.linalg.norm(x64), 1e-300)))
        wall64 = time.perf_counter() - t0
        fp64 = dict(percentiles(lat64), requests=n64, solves_per_s=n64 / wall64,
                    max_rel_error_batched_vs_fp64=max(errs) if errs else None, compared_solutions=len(errs))
    n_dofs = np.array([p.n_dofs for p in probs])
    return {
        "metric": "served solves/s at 1e-10 with p50/p99 latency (continuous batching)",
        "value": value, "unit": "solves/s", "n_gpus": world, "steps": 1, "warmup": args.warmup,
        "ms_per_step": 1e3 * out["wall_s"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 apply / f64 residuals", "data": "synthetic",
        "config": {"workload": f"Poisson stream, 200 req/s, {n_req} requests, n=min(96, LogNormal(ln 24, 0.5)), "
                               "Q2/Q3/Q4, 50% heat (CG) / 50% advection-diffusion (BiCGStab in the batch; "
                               "the reference and the single-problem path use GMRES), 150 GB budget",
                   "n_dofs_mean": float(n_dofs.mean()), "n_dofs_max": int(n_dofs.max()),
                   "poll_steps": args.poll_steps,
                   "timing": "host clock (request arrival to solution on the host)"},
        "latency": percentiles(out["latency_s"]),
        "below_capacity": low,
        "loop": out["stats"],
        "work": serve_work(probs, reps, out["wall_s"]),
        "all_converged": all(r["status"] == 0 for r in reps),
        "max_rel_residual": max(r["final_residual"] / max(r["initial_residual"], 1e-300) for r in reps),
        "fp64_plain": fp64,
        "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": int(8 * n_dofs.sum()),
                "call": "mpdg_serve (device right-hand sides, solutions copied to the host)"},
        "gpu_launches": launches,
        "clocks": clk.summary(),
    }


def run_extras(args, rank, world):
    """The other configurations, measured in the same run as the headline."""
    extras = {}
    for name in ("c1", "advdiff"):
        set_workload(name)
        line = run_operator_workload(args, rank, world, headline=False)
        extras["c3" if name == "advdiff" else "c1"] = line
    set_workload("heat")
    extras["c4"] = run_batch(args, rank, world)
    extras["c5"] = run_serve(args, rank, world)
    return extras


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=400)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--solve-reps", type=int, default=20, help="timed solves per form (after one warm-up solve)")
    ap.add_argument("--no-solve", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=5.0)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-extras", action="store_true", help="headline workload only")
    ap.add_argument("--no-autotune", action="store_true", help="keep the default apply schedule")
    ap.add_argument("--cells", type=int, default=0,
                    help="cells per direction (default: the workload's; smaller sizes for profiling)")
    ap.add_argument("--workload", default=None, choices=["heat", "advdiff", "c1", "batch", "serve"],
                    help="one workload only (default: the headline plus the others as extra keys)")
    ap.add_argument("--problems", type=int, default=BATCH_SIZE,
                    help="batch: problems in the batch (the first of the seeded sequence)")
    ap.add_argument("--batch-steps", type=int, default=2, help="batch: timed whole batches")
    ap.add_argument("--requests", type=int, default=20000, help="serve: requests in the stream")
    ap.add_argument("--poll-steps", type=int, default=4, help="serve: graph steps between checks")
    ap.add_argument("--low-rate", type=float, default=40.0, help="serve: arrival rate of the below-capacity stream")
    ap.add_argument("--low-requests", type=int, default=1000, help="serve: requests of the below-capacity stream")
    ap.add_argument("--no-fp64-arm", action="store_true", help="serve: skip the plain FP64 arm")
    ap.add_argument("--profile-solve", default=None, choices=["fp64", "fp32_refined"],
                    help="one solve of the workload's system inside a profiler range (ncu --profile-from-start off)")
    ap.add_argument("--fp64-requests", type=int, default=500,
                    help="serve: requests of the stream the plain FP64 arm serves")
    args = ap.parse_args()
    set_workload(args.workload if args.workload in ("heat", "advdiff", "c1") else "heat", args.cells)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if world > 1 and args.impl == "ours":
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    try:
        if args.profile_solve:
            run_profile_solve(args)
        elif args.impl == "reference":
            run_reference(args, rank, world)
        elif args.workload == "batch":
            line = run_batch(args, rank, world)
            if rank == 0:
                print(json.dumps(line), flush=True)
        elif args.workload == "serve":
            line = run_serve(args, rank, world)
            if rank == 0:
                print(json.dumps(line), flush=True)
        else:
            line = run_operator_workload(args, rank, world, headline=True)
            if args.workload is None and not args.no_extras and world == 1:
                line["extra"] = run_extras(args, rank, world)
            if rank == 0:
                print(json.dumps(line), flush=True)
    finally:
        if world > 1 and args.impl == "ours":
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
