#!/usr/bin/env python3
"""Benchmark of the B200 assembly engine.

Default workload (N=1): vector P2 linear elasticity on UnitCubeMesh(48,48,48)
(663,552 tetrahedra, 2,738,019 dofs, 231,797,385 CSR non-zeros), interior
vertices jittered by a seeded uniform +-0.15h, E = 1, nu = 0.3, body force
(0,0,-1).  One step = SystemAssembler-style assembly of A and b in one pass
(FP64), inputs resident in HBM.  Also measured on the same data: the
FP32-contraction path (max relative error vs the FP64 result) and the
matrix-free action y = A x.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload NAME] [--impl reference]

Prints ONE JSON line (rank 0).  Multi-GPU (torchrun): every rank assembles
its own independently seeded mesh (weak scaling, no collective on the data
path); the time is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Assembly Mcells/s, FP32/batched vs plain FP64 GPU at <=1e-6 rel err; %HBM peak"

WORKLOADS = {
    # name: (kind, n, degree, description)
    "elasticity_p2_48": ("elasticity", 48, 2, "vector P2 elasticity, UnitCubeMesh(48) jittered 0.15h, A+b"),
    "poisson_p1_32": ("poisson", 32, 1, "P1 Poisson kappa P1 + load f P1, UnitCubeMesh(32), A+b"),
    "poisson_p2_96": ("poisson", 96, 2, "P2 Poisson kappa P1 + load f P1, UnitCubeMesh(96), A+b"),
    "poisson_p1_64": ("poisson", 64, 1, "P1 Poisson kappa=exp(g) g~N(0,0.25) + load kappa*f (f P1), "
                      "UnitCubeMesh(64), A+b; adjoint dL/dkappa timed beside it"),
    "poisson_p1_96": ("poisson", 96, 1, "P1 Poisson kappa=exp(g) g~N(0,0.25) + load kappa*f (f P1), "
                      "UnitCubeMesh(96), A+b; adjoint dL/dkappa timed beside it"),
    "batched_512": ("batched", 512, 0, "512 UnitSquareMesh(n), n log-uniform [8,256], jitter 0.2h, "
                    "P1/P2 kappa*grad.grad, one graph-captured persistent launch"),
}


# What the numbers' correctness rests on (the full-size entry-wise parity
# tests compare these configurations with the oracle).
PARITY_NOTE = ("oracle-pinned: entry-wise vs the CPU restatement of DOLFIN's assembly at full size "
               "(P1 values also pinned by the reference's known answers; P2 and vector-P2 values by "
               "the oracle's independent quadrature only)")

# the adjoint workloads: kappa = exp(g), g ~ N(0, 0.5^2) per vertex
LOGNORMAL_KAPPA = {"poisson_p1_64", "poisson_p1_96"}


def run_batched(args, rank, world):
    """512 independent triangle meshes in one persistent, graph-captured launch
    vs a per-mesh launch loop (the batched workload)."""
    import torch
    from dolfin_b200 import _capi, synthetic
    from dolfin_b200.batch import BatchAssembler, autotune
    t0 = time.perf_counter()
    specs = synthetic.batched_square_meshes(512, 2024 + rank)
    built = [synthetic.build_batch_member(sp) for sp in specs]
    members = [(V, k) for (_, V, k, _, _) in built]
    for V, _ in members:
        V.pattern()
    setup_s = time.perf_counter() - t0
    best, timings = autotune(members, precision="fp64", cache_path=None)
    B = BatchAssembler(members, *best)
    cells = B.ncells
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")
    for _ in range(args.warmup):
        B.assemble()
        B.assemble_loop()
        B.assemble("fp32")  # its graph is captured on first use
    torch.cuda.synchronize()
    with ClockSampler(int(os.environ.get("LOCAL_RANK", "0"))) as clk:
        sustain(lambda: B.assemble(), 0.6)
        l0 = _capi.kernel_launches()
        ms = float(np.mean(time_steps(lambda: B.assemble(), args.steps, flush)))
        launches = _capi.kernel_launches() - l0
        sustain(lambda: B.assemble(), 0.4)
    ms_loop = float(np.mean(time_steps(lambda: B.assemble_loop(), args.steps, flush)))
    ms32 = float(np.mean(time_steps(lambda: B.assemble("fp32"), args.steps, flush)))
    vals64 = [A.values_tensor().clone() for A in B.assemble()]
    torch.cuda.synchronize()
    v32 = [A.values_tensor().clone() for A in B.assemble("fp32")]
    torch.cuda.synchronize()
    err32 = max(float((a - b).abs().max() / a.abs().max()) for a, b in zip(vals64, v32))
    nnz = sum(A.nnz() for A in B.matrices)
    nv = sum(V.mesh().num_vertices() for V, _ in members)
    Bytes = sum(csr_bytes(A.nnz(), V.dim(), V.mesh().num_cells(), 6 if V.degree() == 2 else 3,
                          2, V.mesh().num_vertices(), V.mesh().num_vertices(), False)
                for A, (V, _) in zip(B.matrices, members))
    peak, peak_kind = load_peaks()
    achieved = Bytes / (ms * 1e-3) / 1e9
    # e2e: kappa fields H2D from pinned host memory, matrices D2H
    h_k = [torch.from_numpy(np.ascontiguousarray(kv)).pin_memory() for (_, _, _, _, kv) in built]
    h_v = [torch.empty(A.nnz(), dtype=torch.float64, pin_memory=True) for A in B.matrices]

    def e2e():
        for (V, k), hk in zip(members, h_k):
            k.tensor().copy_(hk, non_blocking=True)
        B.assemble()
        for A, hv in zip(B.matrices, h_v):
            hv.copy_(A.values_tensor(), non_blocking=True)
        torch.cuda.current_stream().synchronize()

    e2e()
    te = time.perf_counter()
    for _ in range(3):
        e2e()
    e2e_ms = (time.perf_counter() - te) / 3 * 1e3
    if rank == 0:
        line = {
            "metric": METRIC, "value": round(cells * world / (ms * 1e-3) / 1e6, 3), "unit": "Mcells/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 4),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded batch of jittered unit-square meshes)",
            "config": {"workload": "batched_512", "meshes": 512, "cells": cells, "nnz": nnz,
                       "tuned": {"tile_threads": best[0], "seg_cap_bytes": best[1], "ctas_per_sm": best[2]},
                       "tuning_ms": timings, "setup_s": round(setup_s, 2),
                       "l2": "flushed between steps (256 MiB write)"},
            "loop": {"ms_per_step": round(ms_loop, 4), "mcells_s": round(cells / (ms_loop * 1e-3) / 1e6, 3),
                     "persistent_speedup": round(ms_loop / ms, 3)},
            "fp32_contract": {"ms_per_step": round(ms32, 4), "speedup_vs_fp64": round(ms / ms32, 3),
                              "max_rel_err_vs_fp64": err32},
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 4), "traffic": None, "peak_source": peak_kind,
                         "algorithmic_bytes": Bytes},
            "e2e": {"value": round(cells / (e2e_ms * 1e-3) / 1e6, 3), "unit": "Mcells/s",
                    "ms_per_step": round(e2e_ms, 3), "h2d_bytes_per_step": 8 * nv,
                    "d2h_bytes_per_step": 8 * nnz},
            "gpu_launches": int(launches), "clocks": clk.summary(),
        }
        print(json.dumps(line), flush=True)


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock/throttle sampling during the timed region."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = f"/tmp/db2_clocks_{os.getpid()}.csv"

    def __enter__(self):
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}",
                 "--query-gpu=clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.fh, stderr=subprocess.DEVNULL)
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
            self.fh.close()

    def summary(self):
        if self.proc is None or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as fh:
            for line in fh:
                f = [x.strip() for x in line.split(",")]
                if len(f) < 8:
                    continue
                try:
                    sm.append(float(f[0]))
                    smax = float(f[1])
                except ValueError:
                    continue
                for nm, val in zip(names, f[4:8]):
                    if val.lower() == "active":
                        reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def setup_workload(name, seed, device, n_override=None):
    import torch
    import dolfin_b200 as d2
    from dolfin_b200 import synthetic
    kind, n, deg, _ = WORKLOADS[name]
    n = n_override or n
    t0 = time.perf_counter()
    mesh = d2.UnitCubeMesh(n, n, n)
    x0 = mesh.coordinates()
    if kind == "elasticity":
        x = synthetic.jitter_interior(x0, n, 0.15, seed)
        mesh.set_coordinates(x)
        V = d2.VectorFunctionSpace(mesh, "Lagrange", deg)
        u, v = d2.TrialFunction(V), d2.TestFunction(V)
        E, nu = 1.0, 0.3
        mu = d2.Constant(E / (2 * (1 + nu)))
        lmbda = d2.Constant(E * nu / ((1 + nu) * (1 - 2 * nu)))
        eps = lambda w: d2.sym(d2.grad(w))
        sigma = lambda w: 2 * mu * eps(w) + lmbda * d2.tr(eps(w)) * d2.Identity(3)
        a = d2.inner(sigma(u), eps(v)) * d2.dx
        L = d2.inner(d2.Constant((0.0, 0.0, -1.0)), v) * d2.dx
        fields, funcs = {}, ()
    else:
        x = x0
        V = d2.FunctionSpace(mesh, "Lagrange", deg)
        W = d2.FunctionSpace(mesh, "Lagrange", 1)
        if name in LOGNORMAL_KAPPA:
            kv = synthetic.lognormal_field(mesh.num_vertices(), 0.5, seed)
        else:
            kv = synthetic.uniform_field(mesh.num_vertices(), 0.5, 2.0, seed)
        fv = synthetic.uniform_field(mesh.num_vertices(), -1.0, 1.0, seed + 1)
        kappa, f = d2.Function(W, kv), d2.Function(W, fv)
        u, v = d2.TrialFunction(V), d2.TestFunction(V)
        a = kappa * d2.inner(d2.grad(u), d2.grad(v)) * d2.dx
        # the adjoint workloads differentiate A and b: b = kappa*f*v*dx
        L = (kappa * f * v * d2.dx) if name in LOGNORMAL_KAPPA else (f * v * d2.dx)
        fields = {"kappa": kv, "f": fv}
        funcs = (kappa, f)
    S = d2.SystemAssembler(a, L)
    A, b = d2.Matrix(), d2.Vector(n=V.dim())
    S.assemble(A, b)  # builds the pattern and the plan, first assembly
    torch.cuda.synchronize()
    setup_s = time.perf_counter() - t0
    return dict(mesh=mesh, V=V, a=a, L=L, S=S, A=A, b=b, x=x, fields=fields, kind=kind, n=n,
                deg=deg, setup_s=setup_s, name=name, funcs=funcs)


def csr_bytes(nnz, N, C, k_node, gdim, Nv, coeff_dofs, with_b):
    """Algorithmic bytes of one CSR assembly, inputs read once and outputs
    written once: 4 k C (cell->node map) + 8 gdim Nv (coordinates) + 8 per
    coefficient dof + 12 nnz (8 B value write + 4 B column index) + 4 (N+1)
    (row pointers) + 8 N (the vector, when b is assembled too)."""
    return (4 * k_node * C + 8 * gdim * Nv + 8 * coeff_dofs + 12 * nnz + 4 * (N + 1)
            + (8 * N if with_b else 0))


def algorithmic_bytes(w):
    mesh, V, A = w["mesh"], w["V"], w["A"]
    C, Nv = mesh.num_cells(), mesh.num_vertices()
    k_node = 10 if w["deg"] == 2 else 4
    return csr_bytes(A.nnz(), V.dim(), C, k_node, 3, Nv, Nv * len(w["fields"]), True)


def profiled_traffic(workload):
    """(DRAM bytes read + written per A+b step of the assembly kernels,
    source): from the committed ncu launch list of this workload under
    profiles/ -- a separate one-pass capture, not measured by this run, so
    the source names the file and the kernel revision it was captured on."""
    name = f"k_assemble_launches_{workload}.txt"
    path = os.path.join(ROOT, "profiles", name)
    traffic, rev = None, None
    try:
        with open(path) as fh:
            for line in fh:
                if line.startswith("traffic_bytes_per_step:"):
                    traffic = int(line.split(":")[1])
                if line.startswith("kernel_revision:"):
                    rev = line.split(":", 1)[1].strip()
    except OSError:
        return None, None
    if traffic is None:
        return None, None
    return traffic, f"profiles/{name} (ncu capture at {rev or 'an earlier revision'}; not measured in this run)"


def sustain(fn, seconds):
    """Run fn() back to back for about `seconds` (clock sampling window)."""
    import torch
    t0 = time.perf_counter()
    while time.perf_counter() - t0 < seconds:
        for _ in range(8):
            fn()
        torch.cuda.synchronize()


def time_steps(fn, steps, flush=None):
    """Per-step CUDA-event device time (ms) of fn() on the current stream."""
    import torch
    evs = []
    for _ in range(steps):
        if flush is not None:
            flush.zero_()
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        fn()
        e.record()
        evs.append((s, e))
    torch.cuda.synchronize()
    return [s.elapsed_time(e) for s, e in evs]


def cpu_baseline_sample(w, target_s=10.0, threads=1):
    """The oracle (CPU restatement of DOLFIN's serial assemble_cells loop with
    coeffRef-style CSR insertion) on the first cells of the same mesh."""
    from oracle import oracle as orc
    mesh = w["mesh"]
    om = orc.Mesh(3, np.ascontiguousarray(w["x"]), mesh.cells())
    deg = w["deg"]
    vs = 3 if w["kind"] == "elasticity" else 1
    od, N = orc.dofmap(om, deg, vs)
    S = 2048 if w["kind"] == "elasticity" else (8192 if deg == 2 else 65536)
    sub = orc.Mesh(3, om.coords, om.cells[:S])
    dsub = np.ascontiguousarray(od[:S])
    rp, cols = orc.sparsity(N, N, dsub, dsub)
    if w["kind"] == "elasticity":
        fa = orc.form(orc.ELASTICITY, 3, deg, 3, mu=1 / 2.6, lmbda=0.3 / (1.3 * 0.4))
        fl = orc.form(orc.LOAD, 3, deg, 3, coeff=orc.COEFF_CONST, c=(0, 0, -1))
        wa = wl = wl2 = None
    else:
        fa = orc.form(orc.DIFFUSION, 3, deg, 1, coeff=orc.COEFF_P1)
        wa, wl = w["fields"]["kappa"], w["fields"]["f"]
        if w["name"] in LOGNORMAL_KAPPA:
            fl = orc.form(orc.LOAD, 3, deg, 1, coeff=orc.COEFF_P1_TIMES_P1)
            wl, wl2 = wa, wl
        else:
            fl = orc.form(orc.LOAD, 3, deg, 1, coeff=orc.COEFF_P1)
            wl2 = None
    reps, t = 0, 0.0
    while t < target_s:
        t0 = time.perf_counter()
        orc.assemble_matrix(fa, sub, dsub, dsub, rp, cols, w=wa)
        orc.assemble_vector(fl, sub, dsub, N, w=wl, w2=wl2)
        t += time.perf_counter() - t0
        reps += 1
    return {"value": S * reps / t / 1e6, "unit": "Mcells/s", "cores": threads, "kind": "port",
            "sample": (f"first {S} cells of the workload mesh, A+b, {reps} passes, {t:.1f} s; the oracle "
                       "(CPU restatement of DOLFIN's serial cell loop, element tensors by quadrature), "
                       "not DOLFIN's own speed")}


# ---------------------------------------------------------------------------
# Reference arm: the reference's algorithm on the host cores.  DOLFIN itself
# cannot be built here (it needs FFC/UFL, Boost, Eigen, MPI); its serial
# assembly path is restated in oracle/ (C++) and run on every host core, one
# process per core over disjoint cell ranges of the same workload.
# ---------------------------------------------------------------------------
_REF = {}


def _ref_init(workload, rank, ncells, ncores):
    """Oracle inputs of one reference worker: `ncells` consecutive cells of the
    workload mesh (3D workloads), or whole member meshes of the batched
    workload taken round-robin until about `ncells` cells."""
    from oracle import oracle as orc
    from dolfin_b200 import synthetic
    kind, n, deg, _ = WORKLOADS[workload]
    if kind == "batched":
        jobs, done = [], 0
        specs = synthetic.batched_square_meshes(512, 2024)
        for sp in specs[rank::ncores]:
            m = sp["n"]
            om = orc.unit_square_mesh(m, m)
            om.coords = synthetic.jitter_interior(om.coords, m, sp["jitter"], sp["seed"])
            kv = synthetic.uniform_field(om.nv, 0.5, 2.0, sp["seed"] + 1)
            od, N = orc.dofmap(om, sp["degree"], 1)
            rp, cols = orc.sparsity(N, N, od, od)
            fa = orc.form(orc.DIFFUSION, 2, sp["degree"], 1, coeff=orc.COEFF_P1)
            jobs.append((fa, om, od, rp, cols, kv))
            done += om.nc
            if done >= ncells:
                break
        _REF.update(orc=orc, jobs=jobs, ncells=done)
        return
    om = orc.unit_cube_mesh(n, n, n)
    vs = 3 if kind == "elasticity" else 1
    if kind == "elasticity":
        om.coords = synthetic.jitter_interior(om.coords, n, 0.15, 1000)
        fa = orc.form(orc.ELASTICITY, 3, deg, 3, mu=1 / 2.6, lmbda=0.3 / (1.3 * 0.4))
        fl = orc.form(orc.LOAD, 3, deg, 3, coeff=orc.COEFF_CONST, c=(0, 0, -1))
        wa = wl = wl2 = None
    else:
        fa = orc.form(orc.DIFFUSION, 3, deg, 1, coeff=orc.COEFF_P1)
        wa = (synthetic.lognormal_field(om.nv, 0.5, 1000) if workload in LOGNORMAL_KAPPA
              else synthetic.uniform_field(om.nv, 0.5, 2.0, 1000))
        wl = synthetic.uniform_field(om.nv, -1.0, 1.0, 1001)
        if workload in LOGNORMAL_KAPPA:  # b = kappa*f*v*dx
            fl = orc.form(orc.LOAD, 3, deg, 1, coeff=orc.COEFF_P1_TIMES_P1)
            wl2, wl = wl, wa
        else:
            fl = orc.form(orc.LOAD, 3, deg, 1, coeff=orc.COEFF_P1)
            wl2 = None
    od, N = orc.dofmap(om, deg, vs)
    lo = (rank * ncells) % om.nc
    sub = orc.Mesh(3, om.coords, np.ascontiguousarray(om.cells[lo:lo + ncells]))
    dsub = np.ascontiguousarray(od[lo:lo + ncells])
    rp, cols = orc.sparsity(N, N, dsub, dsub)
    _REF.update(orc=orc, sub=sub, dsub=dsub, rp=rp, cols=cols, fa=fa, fl=fl, wa=wa, wl=wl, wl2=wl2, N=N,
                jobs=None, ncells=sub.nc)


def _ref_work(_):
    r = _REF
    t0 = time.perf_counter()
    if r["jobs"] is not None:
        for fa, om, od, rp, cols, kv in r["jobs"]:
            r["orc"].assemble_matrix(fa, om, od, od, rp, cols, w=kv)
    else:
        r["orc"].assemble_matrix(r["fa"], r["sub"], r["dsub"], r["dsub"], r["rp"], r["cols"], w=r["wa"])
        r["orc"].assemble_vector(r["fl"], r["sub"], r["dsub"], r["N"], w=r["wl"], w2=r["wl2"])
    return time.perf_counter() - t0


def _ref_worker_main(workload, rank, ncells, ncores, q_in, q_out):
    _ref_init(workload, rank, ncells, ncores)
    q_out.put(("ready", _REF["ncells"]))
    while True:
        msg = q_in.get()
        if msg is None:
            return
        q_out.put(_ref_work(None))


def run_reference(args, rank, world):
    if rank != 0:
        return
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    kind, n, deg, desc = WORKLOADS[args.workload]
    total_cells = 6 * n ** 3 if kind != "batched" else None
    ncores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
    per = {"elasticity": 512, "poisson": 32768 if deg == 1 else 4096, "batched": 16384}[kind]
    procs, qin, qout = [], [], []
    for r in range(ncores):
        qi, qo = ctx.Queue(), ctx.Queue()
        p = ctx.Process(target=_ref_worker_main, args=(args.workload, r, per, ncores, qi, qo))
        p.start()
        procs.append(p)
        qin.append(qi)
        qout.append(qo)
    cells_per_step = 0
    for qo in qout:
        tag, nc = qo.get(timeout=900)
        assert tag == "ready"
        cells_per_step += nc

    def step():
        t0 = time.perf_counter()
        for qi in qin:
            qi.put(1)
        for qo in qout:
            qo.get(timeout=900)
        return time.perf_counter() - t0

    for _ in range(args.warmup):
        step()
    times = [step() for _ in range(args.steps)]
    for qi in qin:
        qi.put(None)
    for p in procs:
        p.join(timeout=60)
    t = float(np.mean(times))
    value = cells_per_step / t / 1e6
    line = {
        "metric": METRIC, "impl": "reference", "value": round(value, 4), "unit": "Mcells/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(t * 1e3, 3), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded; same mesh and fields)",
        "config": {"workload": args.workload, "description": desc},
        "cpu_baseline": {"value": round(value, 4), "unit": "Mcells/s", "cores": ncores, "kind": "port",
                         "sample": (f"{cells_per_step} cells per step over {ncores} cores "
                                    + ("(whole member meshes, round-robin)" if kind == "batched"
                                       else f"(disjoint cell ranges, {100.0 * cells_per_step / total_cells:.1f} % "
                                            f"of the {total_cells} cells)")
                                    + "; the oracle: a CPU restatement of DOLFIN's serial assemble_cells + "
                                      "EigenMatrix::add whose element tensors come from Gauss-Jacobi "
                                      "quadrature (slower than FFC's generated tabulate_tensor), so this "
                                      "is not DOLFIN's own speed")},
        "e2e": {"value": round(value, 4), "unit": "Mcells/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


DEFAULT_WORKLOAD = "elasticity_p2_48"
# B200 FP64 peak, nominal (no measured FP64 figure exists on this pool):
# context for the matrix-free action's arithmetic rate only.
NOMINAL_FP64_TFLOPS = 37.0


def action_bytes(C, k_node, gdim, Nv, coeff_dofs, N):
    """Algorithmic bytes of one matrix-free y = A x: cell->node map, vertex
    coordinates, coefficient dofs, x read and y written once."""
    return 4 * k_node * C + 8 * gdim * Nv + 8 * coeff_dofs + 16 * N


def action_flops(C, k):
    """Algorithmic FLOPs of one action: the dense element matrix-vector
    product, 2 k^2 per cell (k dofs per cell)."""
    return 2 * k * k * C


def dofs_per_cell(w):
    k_node = 10 if w["deg"] == 2 else 4
    return k_node * (3 if w["kind"] == "elasticity" else 1)


def measure_action(w, args, flush, peak, repeats=0, precision="fp64"):
    """Matrix-free action on the workload's form: per-action device time
    (L2 flushed between actions), the roofline numbers, and optionally the
    time of `repeats` back-to-back actions (one event window)."""
    import torch
    import dolfin_b200 as d2
    V, mesh = w["V"], w["mesh"]
    x = torch.randn(V.dim(), dtype=torch.float64, device="cuda",
                    generator=torch.Generator("cuda").manual_seed(7))
    xv, y = d2.Vector(x), d2.Vector(n=V.dim())
    act = lambda: d2.assemble_action(w["a"], xv, y, precision=precision)
    for _ in range(args.warmup):
        act()
    ms = float(np.mean(time_steps(act, args.steps, flush)))
    C, Nv = mesh.num_cells(), mesh.num_vertices()
    k_node = 10 if w["deg"] == 2 else 4
    by = action_bytes(C, k_node, 3, Nv, Nv if w["kind"] == "poisson" else 0, V.dim())
    fl = action_flops(C, dofs_per_cell(w))
    gbs = by / (ms * 1e-3) / 1e9
    gfs = fl / (ms * 1e-3) / 1e9
    out = {"ms_per_action": round(ms, 4), "mcells_s": round(C / (ms * 1e-3) / 1e6, 3),
           "roofline": {"bound": "hbm", "algorithmic_bytes": by, "achieved": round(gbs, 1), "peak": peak,
                        "unit": "GB/s", "frac": round(gbs / peak, 4),
                        "algorithmic_flops": fl, "gflops": round(gfs, 1),
                        "fp64_frac_of_nominal": round(gfs / (NOMINAL_FP64_TFLOPS * 1e3), 4),
                        "flops_note": "2 k^2 per cell (dense element mat-vec); FP64 peak nominal "
                                      f"{NOMINAL_FP64_TFLOPS} TFLOP/s, not measured"}}
    if repeats:
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        flush.zero_()
        s.record()
        for _ in range(repeats):
            act()
        e.record()
        torch.cuda.synchronize()
        tot = s.elapsed_time(e)
        out["repeated"] = {"actions": repeats, "ms_total": round(tot, 3),
                           "ms_per_action": round(tot / repeats, 4),
                           "frac": round(by / (tot / repeats * 1e-3) / 1e9 / peak, 4)}
    return out


def measure_assembly(w, args, flush, precision="fp64"):
    """Device time per SystemAssembler step (A and b) at a precision, and
    the matrix it leaves."""
    import dolfin_b200 as d2
    S = w["S"] if precision == "fp64" else d2.SystemAssembler(w["a"], w["L"], precision=precision)
    A = w["A"] if precision == "fp64" else d2.Matrix(w["V"].pattern())
    b = w["b"] if precision == "fp64" else d2.Vector(n=w["V"].dim())
    for _ in range(args.warmup):
        S.assemble(A, b)
    ms = float(np.mean(time_steps(lambda: S.assemble(A, b), args.steps, flush)))
    return ms, A


def extra_config5(args, flush, peak, rank):
    """Scalar P2 Poisson on UnitCubeMesh(96) (5,308,416 cells): FP64 and
    FP32-contraction A+b steps, their roofline, and 100 repeated matrix-free
    actions."""
    import torch
    w = setup_workload("poisson_p2_96", seed=1000 + rank, device=None)
    C = w["mesh"].num_cells()
    ms64, A64 = measure_assembly(w, args, flush, "fp64")
    v64 = A64.values_tensor().clone()
    ms32, A32 = measure_assembly(w, args, flush, "fp32")
    err = float((A32.values_tensor() - v64).abs().max() / v64.abs().max())
    del A32, v64
    by = algorithmic_bytes(w)
    out = {"workload": "poisson_p2_96", "cells": C, "nnz": w["A"].nnz(),
           "fp64": {"ms_per_step": round(ms64, 4), "mcells_s": round(C / (ms64 * 1e-3) / 1e6, 3),
                    "roofline_frac": round(by / (ms64 * 1e-3) / 1e9 / peak, 4)},
           "fp32_contract": {"ms_per_step": round(ms32, 4), "mcells_s": round(C / (ms32 * 1e-3) / 1e6, 3),
                             "roofline_frac": round(by / (ms32 * 1e-3) / 1e9 / peak, 4),
                             "speedup_vs_fp64": round(ms64 / ms32, 3), "max_rel_err_vs_fp64": err},
           "algorithmic_bytes": by, "setup_s": round(w["setup_s"], 2)}
    out["traffic"], out["traffic_source"] = profiled_traffic("poisson_p2_96")
    out["matrix_free"] = measure_action(w, args, flush, peak, repeats=100)
    import dolfin_b200 as d2
    x = torch.randn(w["V"].dim(), dtype=torch.float64, device="cuda",
                    generator=torch.Generator("cuda").manual_seed(7))
    y64 = d2.assemble_action(w["a"], d2.Vector(x)).tensor().clone()
    # the FP32-contraction actions against the FP64 one: element actions by
    # FP32 quadrature ("fp32", the default FP32 path), and the reference
    # tensor x geometry tensor on the tensor cores (tcgen05, "fp32_tc")
    for key, prec, how in (
            ("matrix_free_fp32", "fp32", "FP32 quadrature from the FP64 geometry, FP32 element actions"),
            ("matrix_free_fp32_tensor_core", "fp32_tc",
             "tcgen05 kind::f16, two half limbs of the FP64 geometry tensor, FP32 accumulation")):
        r = measure_action(w, args, flush, peak, repeats=100, precision=prec)
        y32 = d2.assemble_action(w["a"], d2.Vector(x), precision=prec).tensor()
        r["max_rel_err_vs_fp64"] = float((y32 - y64).abs().max() / y64.abs().max())
        r["speedup_vs_fp64"] = round(out["matrix_free"]["ms_per_action"] / r["ms_per_action"], 3)
        r["contraction"] = how
        out[key] = r
    del w
    torch.cuda.empty_cache()
    return out


def extra_adjoint(args, flush, rank):
    """P1 Poisson kappa = exp(g) at n = 64 and 96: the forward A+b step
    against the adjoint dL/dkappa of L = <gA, A(kappa)> + <gb, b(kappa)>
    (b = kappa f v dx, whose derivative term the adjoint includes), FP64 and
    FP32 contraction."""
    import torch
    from dolfin_b200.autodiff import vjp_kappa
    out = {}
    for name in ("poisson_p1_64", "poisson_p1_96"):
        w = setup_workload(name, seed=1000 + rank, device=None)
        ms_fwd, _ = measure_assembly(w, args, flush, "fp64")
        kt = torch.as_tensor(w["fields"]["kappa"], device="cuda")
        ft = torch.as_tensor(w["fields"]["f"], device="cuda")
        g = torch.Generator("cuda").manual_seed(11)
        gA = torch.randn(w["A"].nnz(), dtype=torch.float64, device="cuda", generator=g)
        gb = torch.randn(w["V"].dim(), dtype=torch.float64, device="cuda", generator=g)
        res = {"cells": w["mesh"].num_cells(), "forward_ms": round(ms_fwd, 4)}
        for prec in ("fp64", "fp32"):
            fn = lambda: vjp_kappa(w["V"], kt, gA, f=ft, gb=gb, precision=prec)
            for _ in range(args.warmup):
                fn()
            ms = float(np.mean(time_steps(fn, args.steps, flush)))
            res[f"vjp_{prec}_ms"] = round(ms, 4)
            res[f"ratio_{prec}_to_forward"] = round(ms / ms_fwd, 3)
        out[name] = res
        del w, gA, gb
        torch.cuda.empty_cache()
    return out


def run_split_rows(args, rank, world, local, dist):
    """One mesh over all ranks: rank r assembles and holds only the CSR rows
    (and b entries) of its node range -- shard.row_partition cuts the rows
    at equal incidence counts, shard.RowBlock allocates the block alone.  No
    data-path collective (row owners compute their rows from the cells
    around them); the time is the max over ranks (strong scaling)."""
    import torch
    from dolfin_b200 import _capi, shard
    if WORKLOADS[args.workload][0] == "batched":
        raise SystemExit("--split rows is for single-mesh workloads (the batched one is split by mesh)")
    w = setup_workload(args.workload, seed=1000, device=local)  # the same mesh on every rank
    P = w["V"].pattern()
    cuts = shard.row_partition(P.inc_ptr(), world)
    blk = shard.RowBlock(w["V"], int(cuts[rank]), int(cuts[rank + 1]))
    S = w["S"]
    cells = w["mesh"].num_cells()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    def step():
        S.assemble_into(P, blk.vals, blk.b)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    with ClockSampler(local) as clk:
        sustain(step, 0.6)
        l0 = _capi.kernel_launches()
        ms = float(np.mean(time_steps(step, args.steps, flush)))
        launches = _capi.kernel_launches() - l0
        sustain(step, 0.4)
    ms_max = shard.max_over_ranks(ms) if dist else ms
    peak, peak_kind = load_peaks()
    B = algorithmic_bytes(w)
    h_vals = torch.empty(blk.nnz, dtype=torch.float64, pin_memory=True)
    h_b = torch.empty(blk.nrows, dtype=torch.float64, pin_memory=True)
    h_in = [torch.from_numpy(np.ascontiguousarray(w["x"])).pin_memory()] if w["kind"] == "elasticity" else \
        [torch.from_numpy(w["fields"]["kappa"]).pin_memory(), torch.from_numpy(w["fields"]["f"]).pin_memory()]

    def e2e_step():
        if w["kind"] == "elasticity":
            w["mesh"].set_coordinates(h_in[0].numpy())
        else:
            for fobj, hsrc in zip(w["funcs"], h_in):
                fobj.tensor().copy_(hsrc, non_blocking=True)
        step()
        h_vals.copy_(blk.vals, non_blocking=True)
        h_b.copy_(blk.b, non_blocking=True)
        torch.cuda.current_stream().synchronize()

    e2e_step()
    t0 = time.perf_counter()
    for _ in range(3):
        e2e_step()
    e2e_ms = (time.perf_counter() - t0) / 3 * 1e3
    e2e_ms = shard.max_over_ranks(e2e_ms) if dist else e2e_ms
    if rank == 0:
        _, n, deg, desc = WORKLOADS[args.workload]
        achieved = B / (ms_max * 1e-3) / 1e9
        line = {
            "metric": METRIC, "value": round(cells / (ms_max * 1e-3) / 1e6, 3), "unit": "Mcells/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_max, 4),
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded jittered unit-cube mesh; no external dataset)",
            "config": {"workload": args.workload, "description": desc, "cells": cells,
                       "parallelism": f"row blocks x{world} (one mesh, rows split by incidence count)",
                       "rank0_rows": blk.nrows, "rank0_nnz": blk.nnz,
                       "l2": "flushed between steps (256 MiB write)", "parity": PARITY_NOTE},
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak * world, "unit": "GB/s",
                         "frac": round(achieved / (peak * world), 4), "traffic": None,
                         "peak_source": f"{peak_kind} x{world} GPUs", "algorithmic_bytes": B},
            "e2e": {"value": round(cells / (e2e_ms * 1e-3) / 1e6, 3), "unit": "Mcells/s",
                    "ms_per_step": round(e2e_ms, 3), "h2d_bytes_per_step": sum(t.numel() * 8 for t in h_in),
                    "d2h_bytes_per_step": 8 * (blk.nnz + blk.nrows)},
            "gpu_launches": int(launches), "clocks": clk.summary(),
        }
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def run_profile(args):
    """Only the hot loop of one workload (for ncu captures): warm-up plus
    --steps assembly steps (or matrix-free actions with --profile action),
    no timing, no JSON line."""
    import torch
    import dolfin_b200 as d2
    w = setup_workload(args.workload, seed=1, device=None, n_override=args.mesh_n)
    if args.profile in ("action", "action32", "action32q"):
        x = torch.randn(w["V"].dim(), dtype=torch.float64, device="cuda",
                        generator=torch.Generator("cuda").manual_seed(3))
        xv, y = d2.Vector(x), d2.Vector(n=w["V"].dim())
        prec = {"action": "fp64", "action32": "fp32_tc", "action32q": "fp32"}[args.profile]
        fn = lambda: d2.assemble_action(w["a"], xv, y, precision=prec)
    else:
        fn = lambda: w["S"].assemble(w["A"], w["b"])
    for _ in range(args.warmup + args.steps):
        fn()
    torch.cuda.synchronize()
    print(f"profile {args.workload} n={w['n']} {args.profile}: cells {w['mesh'].num_cells()}, "
          f"launches {d2.kernel_launches()}", flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--workload", default=DEFAULT_WORKLOAD, choices=sorted(WORKLOADS))
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the P2 n=96 and adjoint measurements of the default line")
    ap.add_argument("--profile", choices=["step", "action", "action32", "action32q"], default=None,
                    help="run only the hot loop (for ncu), print no JSON")
    ap.add_argument("--mesh-n", type=int, default=None, help="mesh size override (with --profile)")
    ap.add_argument("--split", choices=["replicas", "rows"], default="replicas",
                    help="N>1: independent replicas per rank (weak scaling) or one mesh whose node "
                         "rows are split into per-rank row blocks (strong scaling)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        run_reference(args, rank, world)
        return

    import torch
    torch.cuda.set_device(local)
    if args.profile:
        run_profile(args)
        return
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    import dolfin_b200 as d2
    from dolfin_b200 import _capi

    if args.workload == "batched_512":
        run_batched(args, rank, world)
        if dist:
            dist.barrier()
            dist.destroy_process_group()
        return

    if args.split == "rows":
        run_split_rows(args, rank, world, local, dist)
        return

    w = setup_workload(args.workload, seed=1000 + rank, device=local)
    S, A, b = w["S"], w["A"], w["b"]
    cells = w["mesh"].num_cells()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    def step():
        S.assemble(A, b)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    with ClockSampler(local) as clk:
        # the sampler polls every 200 ms: keep the same load running around
        # the timed steps so that samples fall inside the loaded window
        sustain(step, 0.6)
        l0 = _capi.kernel_launches()
        t_wall0 = time.perf_counter()
        ms = time_steps(step, args.steps, flush)
        t_wall = time.perf_counter() - t_wall0
        launches = _capi.kernel_launches() - l0
        sustain(step, 0.4)
    if dist:
        dist.barrier()
    ms_step = float(np.mean(ms))
    if dist:
        t = torch.tensor([ms_step], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_step = float(t.item())
    value = cells * world / (ms_step * 1e-3) / 1e6

    # roofline of the step (the pack kernel and the tile-class launches)
    peak, peak_kind = load_peaks()
    B = algorithmic_bytes(w)
    achieved = B / (ms_step * 1e-3) / 1e9

    # FP32 contraction path on the same data
    vals64 = A.values_tensor().clone()
    ms32, A32 = measure_assembly(w, args, flush, "fp32")
    err32 = float((A32.values_tensor() - vals64).abs().max().item() / vals64.abs().max().item())
    del A32, vals64

    # matrix-free action on the same form, FP64 and with the FP32 element
    # actions (FP32 quadrature from the FP64 geometry)
    mf = measure_action(w, args, flush, peak)
    mf32 = measure_action(w, args, flush, peak, precision="fp32")
    xa = torch.randn(w["V"].dim(), dtype=torch.float64, device="cuda",
                     generator=torch.Generator("cuda").manual_seed(7))
    ya64 = d2.assemble_action(w["a"], d2.Vector(xa)).tensor().clone()
    ya32 = d2.assemble_action(w["a"], d2.Vector(xa), precision="fp32").tensor()
    mf["fp32"] = {"ms_per_action": mf32["ms_per_action"], "mcells_s": mf32["mcells_s"],
                  "speedup_vs_fp64": round(mf["ms_per_action"] / mf32["ms_per_action"], 3),
                  "max_rel_err_vs_fp64": float((ya32 - ya64).abs().max() / ya64.abs().max())}
    del xa, ya64, ya32

    # end to end through the public API with host buffers: per step, H2D of the
    # step's input (vertex coordinates for elasticity, kappa and f otherwise)
    # and D2H of the result (CSR values and b)
    nnz = A.nnz()
    h_vals = torch.empty(nnz, dtype=torch.float64, pin_memory=True)
    h_b = torch.empty(w["V"].dim(), dtype=torch.float64, pin_memory=True)
    if w["kind"] == "elasticity":
        h_in = [torch.from_numpy(np.ascontiguousarray(w["x"])).pin_memory()]
    else:
        h_in = [torch.from_numpy(w["fields"]["kappa"]).pin_memory(),
                torch.from_numpy(w["fields"]["f"]).pin_memory()]
    mesh = w["mesh"]

    def e2e_step():
        if w["kind"] == "elasticity":
            mesh.set_coordinates(h_in[0].numpy())  # host -> device coordinate upload
        else:
            for fobj, hsrc in zip(w["funcs"], h_in):
                fobj.tensor().copy_(hsrc, non_blocking=True)
        S.assemble(A, b)
        h_vals.copy_(A.values_tensor(), non_blocking=True)
        h_b.copy_(b.tensor(), non_blocking=True)
        torch.cuda.current_stream().synchronize()

    e2e_step()
    t0 = time.perf_counter()
    n_e2e = max(3, min(args.steps, 10))
    for _ in range(n_e2e):
        e2e_step()
    e2e_ms = (time.perf_counter() - t0) / n_e2e * 1e3
    h2d = sum(t.numel() * 8 for t in h_in)
    ndofs = w["V"].dim()
    d2h = (nnz + ndofs) * 8
    del h_vals, h_b

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline_sample(w)

    extras = {}
    if args.workload == DEFAULT_WORKLOAD and not args.no_extras:
        del w, S, A, b
        torch.cuda.empty_cache()
        extras["config5"] = extra_config5(args, flush, peak, rank)
        extras["adjoint"] = extra_adjoint(args, flush, rank)

    if rank == 0:
        _, n, deg, desc = WORKLOADS[args.workload]
        traffic, traffic_src = profiled_traffic(args.workload)
        line = {
            "metric": METRIC, "value": round(value, 3), "unit": "Mcells/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_step, 4),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded jittered unit-cube mesh; no external dataset)",
            "config": {"workload": args.workload, "description": desc, "cells": cells,
                       "dofs": ndofs, "nnz": nnz, "precision": "fp64",
                       "l2": "flushed between steps (256 MiB write)",
                       "parallelism": f"replicas x{world}",
                       "parity": PARITY_NOTE},
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak,
                         "unit": "GB/s", "frac": round(achieved / peak, 4),
                         "traffic": traffic, "traffic_source": traffic_src,
                         "peak_source": peak_kind, "algorithmic_bytes": B},
            "fp32_contract": {"value": round(cells / (ms32 * 1e-3) / 1e6, 3), "unit": "Mcells/s",
                              "ms_per_step": round(ms32, 4), "speedup_vs_fp64": round(ms_step / ms32, 3),
                              "max_rel_err_vs_fp64": err32},
            "matrix_free": mf,
            "e2e": {"value": round(cells / (e2e_ms * 1e-3) / 1e6, 3), "unit": "Mcells/s",
                    "ms_per_step": round(e2e_ms, 3), "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h},
            "gpu_launches": int(launches),
            "clocks": clk.summary(),
            "wall_s_timed_region": round(t_wall, 3),
        }
        line.update(extras)
        if cpu is not None:
            line["cpu_baseline"] = cpu
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
