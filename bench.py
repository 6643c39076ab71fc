#!/usr/bin/env python
"""Benchmark of the B200 assembly path: assembled elements per second (K + R).

Workload (the 2D cohesive RVE configuration): unit square, 512 x 512 quads split into 524,288
tri3, 200 seeded circular fibers (radius ~ U[0.008, 0.015], minimum gap 0.002), matrix
E = 3.5 GPa / nu = 0.35, fiber E = 72 GPa / nu = 0.22, plane strain, bilinear cohesive law on
every interface (sigma_c = 50 MPa, delta_c2 = 5e-3, delta_c1 = delta_c2 / 1e4).  The state is a
seeded displacement field with tensile interface openings spanning the law's loading, softening
and failed branches.  Synthetic data: the reference publishes no data set (fiber layouts come
from user CSV files in the reference's drivers).

A step is one Assembler::assemble (stiffness blocks K_ff/K_fp/K_pf/K_pp and internal force
P_f/P_p, trial internal variables and damage zones) of that RVE.  `value` is elements/s with the
displacement already resident in HBM (L2 flushed before every timed step); `e2e` is the same
call through the C ABI with host buffers (H2D of U, D2H of all K values and P inside the timed
region).  Multi-GPU runs are independent replicas (one RVE per rank, no collective on the data
path): `scaling` = weak.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
from __future__ import annotations

import argparse
import csv
import io
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from pigfem_b200 import replicas  # noqa: E402  (no torch / CUDA import at module load)

METRIC = "assembled elems/s (K+R) FP64 vs FP32-mixed; served RVE req/s with p50/p99"
UNIT = "elements/s"
L2_FLUSH_BYTES = 256 << 20


def parse():
    return parse_from(None)


def parse_from(argv):
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=300)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", choices=("ours", "reference"), default="ours")
    p.add_argument("--grid", type=int, default=512)
    p.add_argument("--fibers", type=int, default=200)
    p.add_argument("--workload", choices=("cohesive_2d_512", "linear_3d_64", "batched_2d_256", "serving"),
                   default="cohesive_2d_512")
    p.add_argument("--requests", type=int, default=48, help="serving: requests per swept rate")
    p.add_argument("--rates", type=str, default="2,4,8", help="serving: Poisson arrival rates (requests/s)")
    p.add_argument("--session-steps", type=int, default=3,
                   help="serving: load steps per cohesive session (1: every cohesive request stands alone)")
    p.add_argument("--batch", type=int, default=256)
    p.add_argument("--grid3d", type=int, default=64)
    p.add_argument("--spheres", type=int, default=50)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-batched", action="store_true", help="leave the batched sub-object out of the default line")
    p.add_argument("--e2e-steps", type=int, default=0, help="end-to-end steps (default: --steps)")
    p.add_argument("--ref-procs", type=int, default=0, help="reference arm: replica processes (default: one per core)")
    return p.parse_args(argv)


def dist_env():
    return replicas.dist_env()


def algorithmic_bytes(P, fp32: bool) -> dict:
    """Compulsory global traffic of one full assembly, counted from the actual sizes: element
    connectivity (4 B per node slot), a 4 B material tag per element, coordinates and U of every
    node once (8 B per component, 4 B in the FP32-mixed path), a 4 B sub-element table index per
    cut element, cohesive internal variables read + written (16 B each), every CSR value written
    once (8 B) and every residual entry written once (8 B).  Index arrays (row pointers, columns,
    adjacency) are an implementation choice and are not counted."""
    s = P.sizes
    dim = s["dim"]
    npe = dim + 1
    comp = 4 if fp32 else 8
    nnz = sum(s["nnz"])
    b = dict(
        connectivity=4 * npe * s["n_elem"],
        material=4 * s["n_elem"],
        nodes=2 * comp * dim * s["n_nodes"],
        cut_index=4 * s["n_cut_elem"],
        isv=16 * s["n_isv"],
        csr_values=8 * nnz,
        residual=8 * (s["n_free"] + s["n_const"]),
    )
    b["total"] = sum(b.values())
    return b


def fast_kernel_bytes(P, fp32: bool) -> float:
    """Algorithmic bytes of the dominant kernel (rows whose elements are all uncut): the CSR values
    and residual entries of its rows, plus connectivity/material of the uncut elements and the
    coordinates and U of the standard nodes."""
    s = P.sizes
    dim = s["dim"]
    comp = 4 if fp32 else 8
    fast = P.debug("fast_dn")
    dn_node = P.debug("dn_node")
    _, dofs, _ = P.nodes()
    nf = P.n_free
    rows = dofs[dn_node[fast]].reshape(-1)
    total = 0
    for blocks, sel, off in (((0, 1), rows < nf, 0), ((2, 3), rows >= nf, nf)):
        r = rows[sel] - off
        for b in blocks:
            rp, _, _ = P.pattern(b)
            total += 8 * int(np.sum(rp[r + 1] - rp[r]))
    total += 8 * len(rows)
    n_uncut = s["n_elem"] - s["n_cut_elem"]
    total += (4 * (dim + 1) + 4) * n_uncut + 2 * comp * dim * s["n_std_nodes"]
    return float(total)


def general_kernel_bytes(P, fp32: bool) -> float:
    """Algorithmic bytes of the general-row kernel (boundary rows, nodes of cut elements and
    enrichment nodes): the CSR values and residual entries of its rows, connectivity/material of
    the elements adjacent to them, a 4 B sub-element table index per cut element, and the
    coordinates and U of the nodes their rows couple to."""
    s = P.sizes
    dim = s["dim"]
    comp = 4 if fp32 else 8
    slow = P.debug("slow_dn")
    dn_node = P.debug("dn_node")
    _, dofs, _ = P.nodes()
    nf = P.n_free
    rows = dofs[dn_node[slow]].reshape(-1)
    total = 0
    for blocks, sel, off in (((0, 1), rows < nf, 0), ((2, 3), rows >= nf, nf)):
        r = rows[sel] - off
        for b in blocks:
            rp, _, _ = P.pattern(b)
            total += 8 * int(np.sum(rp[r + 1] - rp[r]))
    total += 8 * len(rows)
    ao, adj = P.debug("dn_adj_off"), P.debug("dn_adj")
    no, nbr = P.debug("dn_nbr_off"), P.debug("dn_nbr")
    elems = np.unique(np.concatenate([adj[ao[a]:ao[a + 1]] >> 5 for a in slow])) if len(slow) else np.zeros(0, int)
    nodes = np.unique(np.concatenate([nbr[no[a]:no[a + 1]] for a in slow])) if len(slow) else np.zeros(0, int)
    total += (4 * (dim + 1) + 4) * len(elems) + 4 * s["n_cut_elem"] + 2 * comp * dim * len(nodes)
    return float(total)


def launches_per_step(P, three_d: bool = False) -> int:
    """Kernels one step launches (the L2 flush between steps is a torch fill, not counted).  An
    assembly: k_gen_first (the cohesive elements), the tiles of the structured rows, k_gen_rows
    (the general rows), each only when it has work.  The 3D step adds the multi-strain residual
    pass: its cohesive elements, structured rows and general rows."""
    s = P.sizes
    fast, slow = len(P.debug("fast_dn")) > 0, len(P.debug("slow_dn")) > 0
    n = int(s["n_coh_qp"] > 0) + int(fast) + int(slow)
    if three_d:
        n += int(s["n_coh_qp"] > 0) + int(fast) + int(slow)
    return n


class Clocks:
    """nvidia-smi sampling of SM clock and throttle reasons during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        self.out = ""
        if self.proc is not None:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.out, _ = self.proc.communicate(timeout=5)
            except Exception:
                self.proc.kill()
                self.out = ""

    def summary(self) -> dict:
        rows = [r for r in csv.reader(io.StringIO(getattr(self, "out", ""))) if len(r) >= 9]
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
            except ValueError:
                continue
            for k, name in enumerate(names):
                if r[5 + k].strip().lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def profiled_traffic(kernel: str):
    """DRAM bytes per launch of `kernel` from the committed ncu summary (profiles/*.md lines
    'traffic_bytes_per_launch <kernel> <bytes>'), or None."""
    pdir = os.path.join(ROOT, "profiles")
    try:
        for fn in sorted(os.listdir(pdir)):
            with open(os.path.join(pdir, fn)) as f:
                for line in f:
                    t = line.split()
                    if len(t) == 3 and t[0] == "traffic_bytes_per_launch" and t[1] == kernel:
                        return float(t[2])
    except OSError:
        pass
    return None


def measured_peak_hbm():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


WORKLOADS = {
    "cohesive_2d_512": "cohesive_2d_512: 512x512 tri3 split (524,288 tri3), 200 circular fibers, bilinear cohesive interfaces",
    "linear_3d_64": "linear_3d_64: 64^3 hexes split into 6 tet4 (1,572,864 tet4), 50 spheres, periodic, one K and six unit-strain right-hand sides",
    "serving": "serving: Poisson RVE requests (70% 2D 32^2-512^2 with 5-300 fibers, 30% 3D tet4 16^3-64^3 with 5-60 spheres; 60% homogenization by device PCG to 1e-8, 40% cohesive load-step tangent/residual, each opening a session of --session-steps load steps on a device-resident context)",
    "batched_2d_256": "batched_2d_256: 256 independent 2D cohesive RVEs (grid side log-uniform 32-256, 5-120 fibers, volume fraction 0.2-0.5), one batched assembly of all",
}


def build_problem(args, rank, device=True):
    from pigfem_b200 import capi, rve
    if args.workload == "linear_3d_64":
        R = rve.linear_3d(n=args.grid3d, n_spheres=args.spheres, seed=1, request=rank)
        P = capi.Problem(R.desc, device=device)
        U = np.zeros(P.n_nodes * 3)
        return R, P, U
    R = rve.cohesive_2d(n=args.grid, n_fibers=args.fibers, seed=1, request=rank)
    P = capi.Problem(R.desc, device=device)
    U = rve.interface_state(P, seed=rank)
    return R, P, U


UNIT_STRAINS_3D = [tuple(1.0 if i == k else 0.0 for i in range(6)) for k in range(6)]


def setup_times(R) -> dict:
    """Wall time of the set-up of R's mesh (host-only context, no upload) with every pass on the
    host (pg_create_host), with the per-node / per-element passes on the device, and with the
    pattern on the device too (pg_create_prep_device); each the best of two, outside the timed
    region."""
    from pigfem_b200 import capi
    out = {}
    for key, prep, pat in (("host_s", False, False), ("device_nodes_s", True, False), ("device_prep_s", True, True)):
        best = None
        for _ in range(2):
            t = time.perf_counter()
            Q = capi.Problem(R.desc, device=False, prep_device=prep, prep_pattern=pat)
            dt = time.perf_counter() - t
            if prep and pat:
                out["device_passes_ms"] = Q.prep_device_ms()
            Q.close()
            best = dt if best is None else min(best, dt)
        out[key] = best
    return out


def reference_problem(R, P, U):
    """The reference's own Problem (oracle/_ref) for the same RVE and state as this library's
    problem P; returns it and the DOF vector (free then constrained) of U."""
    from oracle import ref
    RP = ref.RefProblem(ref_spec(R))
    _, dofs, _ = P.nodes()
    Ud = np.zeros(RP.n_free + RP.n_const)
    Ud[dofs.reshape(-1)] = U
    return RP, Ud


def ref_spec(R):
    import dataclasses
    from oracle import ref
    return ref.ProblemSpec(**{f.name: getattr(R.desc, f.name) for f in dataclasses.fields(R.desc)})


def reference_state(args, RP):
    """The workload's displacement state (DOF vector) built from the reference's own mesh tables:
    the same function of the enriched mesh as build_problem's, so both arms time the same state
    (equal to 1e-14; tests/test_config_parity_gpu.py checks it)."""
    from pigfem_b200 import rve
    if args.workload == "linear_3d_64":
        return np.zeros(RP.n_free + RP.n_const)
    U = rve.interface_state_tables(**RP.cut_tables(), seed=0)
    Ud = np.zeros(RP.n_free + RP.n_const)
    Ud[RP.get("node_dofs")] = U
    return Ud


def reference_step_seconds(args, RP, Ud, budget_s: float, max_steps: int):
    """Times the reference's Assembler::assemble for one step of the workload (2D: one K + R;
    3D: one K + R and five residual-only assemblies for the other unit strains), repeated while
    the budget lasts (at most max_steps).  Returns (seconds per step, steps timed)."""
    three_d = args.workload == "linear_3d_64"
    if three_d:
        RP.set_macro(UNIT_STRAINS_3D[0])
    RP.assemble(Ud, None, 1.0)                       # warm-up (and the state for the timed calls)
    times = []
    spent = 0.0
    while len(times) < max_steps and (not times or spent < budget_s):
        if three_d:
            t = 0.0
            for k, e in enumerate(UNIT_STRAINS_3D):
                RP.set_macro(e)
                t += RP.assemble(Ud, None, 1.0, func=True, jac=(k == 0))
        else:
            t = RP.assemble(Ud, None, 1.0)
        times.append(t)
        spent += t
    return float(np.mean(times)), len(times)


def host_info() -> dict:
    """nproc and the CPU model of this host (the cores the CPU figures ran on)."""
    model = None
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    model = line.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    return {"nproc": os.cpu_count(), "cpu_model": model}


def _reference_worker(job):
    """One replica process of the reference arm: builds the reference's Problem for the workload,
    the state from its own tables, and times assemblies for the budget.  Returns (elements,
    seconds per step, steps, config facts)."""
    argv, budget_s, max_steps = job
    args = parse_from(argv)
    from pigfem_b200 import rve
    from oracle import ref
    R = reference_rve(args)
    RP = ref.RefProblem(ref_spec(R))
    Ud = reference_state(args, RP)
    sec, n = reference_step_seconds(args, RP, Ud, budget_s, max_steps)
    facts = {"elements": len(RP.get("elem_cut")), "nnz": int(sum(len(RP.get(f"{b}_cols")) for b in ("K_ff", "K_fp", "K_pf", "K_pp"))),
             "cut_elements": int(np.count_nonzero(RP.get("elem_cut"))), "cohesive_qps": int(RP.get("coh_qp_off")[-1])}
    RP.close()
    return facts["elements"], sec, n, facts


def reference_rve(args):
    """The workload's RVE description, built without this library's set-up (2D: pure numpy)."""
    from pigfem_b200 import rve
    if args.workload == "linear_3d_64":
        return rve.linear_3d(n=args.grid3d, n_spheres=args.spheres, seed=1, request=0)
    return rve.cohesive_2d(n=args.grid, n_fibers=args.fibers, seed=1, request=0)


def reference_workers(max_procs: int, per_proc_bytes: float) -> int:
    """Replica processes the host can hold: one per core, bounded by 80 % of the available memory."""
    avail = None
    try:
        with open("/proc/meminfo") as f:
            for line in f:
                if line.startswith("MemAvailable:"):
                    avail = int(line.split()[1]) * 1024
                    break
    except OSError:
        pass
    n = os.cpu_count() or 1
    if avail:
        n = min(n, max(1, int(0.8 * avail / per_proc_bytes)))
    return max(1, min(n, max_procs))


# resident memory of one reference replica of the 512^2 cohesive workload (measured: set-up plus
# one assembly), used to bound the replica count
REF_PROC_BYTES = {"cohesive_2d_512": 2.5e9, "linear_3d_64": 15e9}


def run_reference(args, ws, rank):
    """The reference's own CPU assembly (oracle/_ref, built from its sources) on rank 0, on all the
    host cores it can use.  The reference assembles serially (one MPI rank, no threads in its
    assembly) and no MPI library is available to partition the mesh, so every core runs an
    independent replica of the workload (its own Problem, same RVE and state); the value is the
    replicas' summed elements/s.  The state comes from the reference's own mesh tables, so this
    arm never loads libpigfem_b200.so."""
    if rank != 0:
        return
    from oracle import ref
    if not ref.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libpigfem_ref.so not built (make -C oracle)"}))
        return
    import multiprocessing as mp
    nproc = reference_workers(args.ref_procs or 256, REF_PROC_BYTES.get(args.workload, 4e9))
    budget = 60.0
    job = (sys.argv[1:], budget, args.steps)
    if nproc == 1:
        results = [_reference_worker(job)]
    else:
        with mp.get_context("spawn").Pool(nproc) as pool:
            results = pool.map(_reference_worker, [job] * nproc)
    ne, _, _, facts = results[0]
    rates = [e / sec for e, sec, _, _ in results]
    value = float(sum(rates))
    n_timed = min(n for _, _, n, _ in results)
    sec_mean = float(np.mean([sec for _, sec, _, _ in results]))
    sample = (f"{nproc} concurrent replica processes (one per core), each a full Assembler::assemble of the {ne}-element RVE" +
              (" with K and 6 right-hand sides" if args.workload == "linear_3d_64" else " (K+R)") +
              f" repeated for up to {budget:.0f} s after 1 warm-up (at least {n_timed} timed steps each); value = sum of the replicas' elements/s")
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps, "steps_timed": n_timed,
            "warmup": args.warmup, "ms_per_step": 1e3 * sec_mean / nproc, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": DATA, "impl": "reference",
            "config": bench_config(args, facts, ws),
            "per_core": {"value": float(np.mean(rates)), "ms_per_step": 1e3 * sec_mean},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": nproc, "kind": "reference", "sample": sample,
                             **host_info()},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


DATA = "synthetic (seeded fiber layout; reference publishes no data set)"


def bench_config(args, facts: dict, ws: int) -> dict:
    """The `config` object of both arms' lines (identical keys and values for one workload)."""
    return {"workload": WORKLOADS[args.workload], "elements": facts["elements"], "nnz": facts["nnz"],
            "cut_elements": facts["cut_elements"], "cohesive_qps": facts["cohesive_qps"],
            "l2": f"GPU arm: flushed before every timed step ({L2_FLUSH_BYTES >> 20} MiB write); CPU arm: host caches",
            "parallelism": f"replicas x{ws} (one RVE per GPU) / one replica per host core"}


def main_batched(args, ws, rank, local):
    """Many RVEs per GPU: one step assembles all of them, batched (persistent kernels, CUDA graph,
    autotuned shape) in FP32-mixed (the value) and FP64, beside the plain path (one
    pg_assemble_device call per RVE, FP64)."""
    import torch
    from concurrent.futures import ThreadPoolExecutor
    from pigfem_b200 import capi, rve
    t_setup = time.time()
    rves = rve.cohesive_batch(count=args.batch, seed=1 + 1000 * rank)
    with ThreadPoolExecutor(max(1, min(16, os.cpu_count() or 1))) as ex:
        probs = list(ex.map(lambda r: capi.Problem(r.desc, device=False), rves))
    for P in probs:
        P.upload()
    Us = [rve.interface_state(P, seed=i) for i, P in enumerate(probs)]
    dUs = [torch.from_numpy(U).cuda() for U in Us]
    ptrs = [u.data_ptr() for u in dUs]
    B = capi.Batch(probs)
    setup_s = time.time() - t_setup
    ne = sum(P.sizes["n_elem"] for P in probs)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")
    stream = torch.cuda.current_stream()
    f64, f32 = capi.FUNC | capi.JAC, capi.FUNC | capi.JAC | capi.FP32
    shape = B.tune(ptrs, f32, reps=3)
    info = B.info()

    def timed_batch(flags, steps, warmup):
        for _ in range(warmup):
            B.assemble(ptrs, flags)
            B.wait()
        replicas.barrier()
        total = 0.0
        for _ in range(steps):
            flush.zero_()
            torch.cuda.synchronize()
            B.assemble(ptrs, flags)
            total += B.wait()      # CUDA events around the graph replay on the batch stream
        return total

    def timed_plain(flags, steps, warmup):
        for P in probs:
            P.set_stream(stream.cuda_stream)
        for _ in range(warmup):
            for P, pu in zip(probs, ptrs):
                P.assemble_device(pu, 1.0, flags)
        torch.cuda.synchronize()
        total = 0.0
        for _ in range(steps):
            flush.zero_()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            for P, pu in zip(probs, ptrs):
                P.assemble_device(pu, 1.0, flags)
            b.record(stream)
            b.synchronize()
            total += a.elapsed_time(b)
        return total

    clk = Clocks(local).__enter__()
    ms32 = timed_batch(f32, args.steps, args.warmup)
    ms64 = timed_batch(f64, args.steps, args.warmup)
    plain_steps = max(3, min(args.steps, 30))
    ms_plain = timed_plain(f64, plain_steps, args.warmup)
    # end to end: every RVE's U from pinned host memory, the batched assembly, every K and P back
    hU = [torch.from_numpy(U).pin_memory() for U in Us]
    outK = [torch.empty(max(sum(P.nnz), 1), dtype=torch.float64).pin_memory() for P in probs]
    outP = [torch.empty(max(P.n_free + P.n_const, 1), dtype=torch.float64).pin_memory() for P in probs]
    bstream = torch.cuda.Stream()
    e2e_steps = args.e2e_steps or min(args.steps, 5)
    e2e_ms = 0.0
    for it in range(e2e_steps + 1):
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for d, h in zip(dUs, hU):
            d.copy_(h, non_blocking=True)
        stream.synchronize()
        B.assemble(ptrs, f32)
        B.wait()
        for P, k, pp in zip(probs, outK, outP):
            K4, pf, ppp = P.device_outputs()
            o = 0
            for blk in range(4):
                if P.nnz[blk]:
                    k[o:o + P.nnz[blk]].copy_(capi.device_view(K4[blk], P.nnz[blk]), non_blocking=True)
                o += P.nnz[blk]
            pp[:P.n_free].copy_(capi.device_view(pf, P.n_free), non_blocking=True)
            if P.n_const:
                pp[P.n_free:P.n_free + P.n_const].copy_(capi.device_view(ppp, P.n_const), non_blocking=True)
        b.record(stream)
        b.synchronize()
        if it > 0:
            e2e_ms += a.elapsed_time(b)
    clk.__exit__(None, None, None)
    ms32, ms64, ms_plain, e2e_ms = replicas.max_over_ranks([ms32, ms64, ms_plain, e2e_ms], "cuda")
    value32 = replicas.aggregate_rate(ne * args.steps, ws, ms32)
    value64 = replicas.aggregate_rate(ne * args.steps, ws, ms64)
    value_plain = replicas.aggregate_rate(ne * plain_steps, ws, ms_plain)
    e2e_value = replicas.aggregate_rate(ne * e2e_steps, ws, e2e_ms)
    alg = sum(algorithmic_bytes(P, True)["total"] for P in probs)
    peak, peak_kind = measured_peak_hbm()
    achieved = alg / (ms32 / args.steps * 1e-3) / 1e9
    replicas.finish()
    if rank != 0:
        return
    line = {
        "metric": METRIC, "value": value32, "unit": UNIT, "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms32 / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32-mixed (FP32 element stiffness, FP64 residual, FP64 scatter)",
        "data": "synthetic (seeded fiber layouts; reference publishes no data set)",
        "config": {"workload": WORKLOADS["batched_2d_256"], "rves": len(probs), "elements": ne,
                   "nnz": int(sum(sum(P.nnz) for P in probs)), "autotuned_shape": info,
                   "mean_volume_fraction": float(np.mean([r.volume_fraction for r in rves])),
                   "l2": f"flushed before every timed step ({L2_FLUSH_BYTES >> 20} MiB write); inputs {alg / 1e9:.2f} GB > L2",
                   "parallelism": f"replicas x{ws} (one batch per GPU)", "setup_s": setup_s},
        "fp64_batched": {"value": value64, "ms_per_step": ms64 / args.steps},
        "plain_fp64_per_rve_calls": {"value": value_plain, "ms_per_step": ms_plain / plain_steps, "steps": plain_steps},
        "speedup_fp32_batched_vs_plain_fp64": value32 / value_plain,
        "roofline": {"bound": "hbm", "kernel": "whole batched assembly (k_batch_coh, k_batch_stencil, k_batch_general)",
                     "achieved": achieved, "peak": peak, "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": None, "bytes_per_launch": alg},
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(sum(U.nbytes for U in Us)),
                "d2h_bytes_per_step": int(sum(8 * (sum(P.nnz) + P.n_free + P.n_const) for P in probs)),
                "ms_per_step": e2e_ms / e2e_steps, "steps": e2e_steps},
        "gpu_launches": 4 * args.steps,
        "clocks": clk.summary(),
        "cpu_baseline": None,
    }
    print(json.dumps(line))


def batched_summary(args, ws, rank, steps: int = 10, warmup: int = 3) -> dict:
    """The batched workload (256 independent 2D cohesive RVEs, grid side log-uniform 32-256, 5-120
    fibers, volume fraction 0.2-0.5) as a compact sub-object of the default line: one batched
    FP32-mixed and one batched FP64 assembly of every RVE per step (persistent kernels replayed
    from a CUDA graph, autotuned shape), beside the plain path (one pg_assemble_device call per
    RVE, FP64), device-resident inputs, L2 flushed before every step.  Every rank runs its own batch
    (the same collective calls in the same order on every rank)."""
    import torch
    from concurrent.futures import ThreadPoolExecutor
    from pigfem_b200 import capi, rve
    t0 = time.time()
    rves = rve.cohesive_batch(count=args.batch, seed=1 + 1000 * rank)
    with ThreadPoolExecutor(max(1, min(16, os.cpu_count() or 1))) as ex:
        probs = list(ex.map(lambda r: capi.Problem(r.desc, device=False), rves))
    for P in probs:
        P.upload()
    dUs = [torch.from_numpy(rve.interface_state(P, seed=i)).cuda() for i, P in enumerate(probs)]
    ptrs = [u.data_ptr() for u in dUs]
    B = capi.Batch(probs)
    setup_s = time.time() - t0
    ne = sum(P.sizes["n_elem"] for P in probs)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")
    stream = torch.cuda.current_stream()
    f64, f32 = capi.FUNC | capi.JAC, capi.FUNC | capi.JAC | capi.FP32
    B.tune(ptrs, f32, reps=3)
    info = B.info()

    def batch_ms(flags):
        for _ in range(warmup):
            B.assemble(ptrs, flags)
            B.wait()
        total = 0.0
        for _ in range(steps):
            flush.zero_()
            torch.cuda.synchronize()
            B.assemble(ptrs, flags)
            total += B.wait()
        return total

    def plain_ms(flags):
        for P in probs:
            P.set_stream(stream.cuda_stream)
        for _ in range(warmup):
            for P, pu in zip(probs, ptrs):
                P.assemble_device(pu, 1.0, flags)
        torch.cuda.synchronize()
        total = 0.0
        for _ in range(steps):
            flush.zero_()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            for P, pu in zip(probs, ptrs):
                P.assemble_device(pu, 1.0, flags)
            b.record(stream)
            b.synchronize()
            total += a.elapsed_time(b)
        return total

    ms32, ms64, ms_plain = replicas.max_over_ranks([batch_ms(f32), batch_ms(f64), plain_ms(f64)], "cuda")
    alg32 = sum(algorithmic_bytes(P, True)["total"] for P in probs)
    alg64 = sum(algorithmic_bytes(P, False)["total"] for P in probs)
    peak, peak_kind = measured_peak_hbm()
    v32 = ws * ne * steps / (ms32 * 1e-3)
    v64 = ws * ne * steps / (ms64 * 1e-3)
    vplain = ws * ne * steps / (ms_plain * 1e-3)
    B.close()
    for P in probs:
        P.close()
    return {"workload": WORKLOADS["batched_2d_256"], "rves": len(probs), "elements": ne, "steps": steps,
            "fp32_mixed": {"value": v32, "unit": UNIT, "ms_per_step": ms32 / steps,
                           "hbm_frac": alg32 / (ms32 / steps * 1e-3) / 1e9 / peak},
            "fp64": {"value": v64, "unit": UNIT, "ms_per_step": ms64 / steps,
                     "hbm_frac": alg64 / (ms64 / steps * 1e-3) / 1e9 / peak},
            "plain_fp64_per_rve_calls": {"value": vplain, "unit": UNIT, "ms_per_step": ms_plain / steps},
            "fp32_batched_over_plain_fp64": v32 / vplain, "fp32_over_fp64_batched": v32 / v64,
            "peak": peak, "peak_kind": peak_kind, "autotuned_shape": info, "setup_s": setup_s,
            "l2": f"flushed before every timed step ({L2_FLUSH_BYTES >> 20} MiB write)"}


def main_serving(args, ws, rank, local):
    """The request loop at swept arrival rates, beside the same requests run one at a time."""
    import torch
    from pigfem_b200 import serving
    torch.cuda.set_device(local)
    free, total = torch.cuda.mem_get_info()
    budget = int(0.5 * free)
    rates = [float(x) for x in args.rates.split(",")]
    # one-at-a-time plain FP64 calls (closed loop): the baseline; a session's steps run on one
    # context, one after the other
    base_reqs = serving.poisson_stream(args.requests, rates[0], seed=11 + rank, session_steps=args.session_steps)
    serving.run_alone(next(q for q in base_reqs if q.session < 0))      # warm-up (module loading, pools)
    t0 = time.perf_counter()
    alone = []
    for q in base_reqs:
        if q.session < 0:
            alone.append(serving.run_alone(q))
        elif q.step == 0:
            alone += serving.run_session_alone([r for r in base_reqs if r.session == q.session])
    wall_alone = time.perf_counter() - t0
    lat_alone = np.array([a.done for a in alone])
    sweep = []
    clk = Clocks(local).__enter__()
    for rate in rates:
        reqs = serving.poisson_stream(args.requests, rate, seed=11 + rank, session_steps=args.session_steps)
        eng = serving.ServingEngine(memory_budget=budget, max_inflight=8, setup_workers=min(16, os.cpu_count() or 1))
        t0 = time.perf_counter()
        res = eng.run(reqs, realtime=True)
        wall = time.perf_counter() - t0
        summ = serving.summarize(res, wall)
        summ["rate"] = rate
        summ["p99_over_p50"] = summ["p99_s"] / summ["p50_s"] if summ["p50_s"] else None
        summ["mean_setup_s"] = float(np.mean([r.setup_done - r.arrival for r in res]))
        summ["mean_queue_s"] = float(np.mean([r.admitted - r.setup_done for r in res]))
        summ["mean_gpu_s"] = float(np.mean([r.done - r.admitted for r in res]))
        summ["session_steps"] = sum(1 for q in reqs if q.session >= 0)
        summ["bytes_calibration"] = eng.calibration
        summ["peak_ledger_bytes"] = eng.peak_charged
        sweep.append(summ)
    clk.__exit__(None, None, None)
    # whole-job request rates: each rank serves its own stream
    for summ in sweep:
        summ["req_per_s"] = replicas.sum_over_ranks([summ["req_per_s"] or 0.0], "cuda")[0]
    best = max(sweep, key=lambda x: x["req_per_s"] or 0)
    if rank != 0:
        return
    line = {
        "metric": METRIC, "value": best["req_per_s"], "unit": "requests/s", "n_gpus": ws, "steps": args.requests,
        "warmup": 1, "ms_per_step": 1e3 / best["req_per_s"] if best["req_per_s"] else None, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded request geometries)",
        "config": {"workload": WORKLOADS["serving"], "requests_per_rate": args.requests, "rates": rates,
                   "memory_budget_bytes": budget, "max_inflight": 8, "session_steps": args.session_steps,
                   "l2": "n/a (request stream)",
                   "parallelism": f"replicas x{ws}"},
        "p50_s": best["p50_s"], "p99_s": best["p99_s"], "sweep": sweep,
        "one_at_a_time_fp64": {"req_per_s": len(alone) / wall_alone, "p50_s": float(np.percentile(lat_alone, 50)),
                               "p99_s": float(np.percentile(lat_alone, 99))},
        "e2e": {"value": best["req_per_s"], "unit": "requests/s", "h2d_bytes_per_step": None, "d2h_bytes_per_step": None,
                "note": "every request is end to end: host set-up, upload, device work, result back"},
        "roofline": None, "gpu_launches": None, "clocks": clk.summary(), "cpu_baseline": None,
    }
    print(json.dumps(line))


def main():
    args = parse()
    ws, rank, local = dist_env()
    if args.impl == "reference":
        run_reference(args, ws, rank)
        return
    if args.workload == "serving":
        import torch
        torch.cuda.set_device(local)
        replicas.init("nccl", local, timeout_s=600)
        main_serving(args, ws, rank, local)
        replicas.finish()
        return
    if args.workload == "batched_2d_256":
        import torch
        torch.cuda.set_device(local)
        replicas.init("nccl", local, timeout_s=300)
        main_batched(args, ws, rank, local)
        return
    import torch
    torch.cuda.set_device(local)
    replicas.init("nccl", local)
    from pigfem_b200 import capi
    R, P, U = build_problem(args, rank)
    ne = P.sizes["n_elem"]
    stream = torch.cuda.current_stream()
    P.set_stream(stream.cuda_stream)
    dU = torch.from_numpy(U).cuda()
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")

    three_d = args.workload == "linear_3d_64"

    if three_d:
        n_more = len(UNIT_STRAINS_3D) - 1
        dRf = torch.empty(n_more * P.n_free, dtype=torch.float64, device="cuda")
        dRp = torch.empty(max(1, n_more * P.n_const), dtype=torch.float64, device="cuda")

    def step_device(flags):
        """One step on device-resident inputs: 2D one assembly; 3D one K and R with the first unit
        strain, then the residuals of the five other unit strains in one multi-strain pass."""
        if not three_d:
            P.assemble_device(dU.data_ptr(), 1.0, flags)
            return
        P.set_macro_strain(UNIT_STRAINS_3D[0])
        P.assemble_device(dU.data_ptr(), 1.0, flags)
        P.residual_strains(dU.data_ptr(), UNIT_STRAINS_3D[1:], dRf.data_ptr(), dRp.data_ptr() if P.n_const else 0)

    def timed(flags, steps, warmup):
        for _ in range(warmup):
            step_device(flags)
        torch.cuda.synchronize()
        replicas.barrier()
        torch.cuda.synchronize()
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        for i in range(steps):
            flush.zero_()
            ev[i][0].record(stream)
            step_device(flags)
            ev[i][1].record(stream)
        torch.cuda.synchronize()
        ms = float(sum(a.elapsed_time(b) for a, b in ev))
        ms = replicas.max_over_ranks([ms], "cuda")[0]
        replicas.barrier()
        torch.cuda.synchronize()
        return ms

    def kernel_times(flags, reps=20):
        """Per-kernel CUDA-event times of the K+R assembly call, outside the timed region."""
        kt = np.zeros(4)
        if three_d:
            P.set_macro_strain(UNIT_STRAINS_3D[0])
        P.set_timing(True)
        for _ in range(reps):
            flush.zero_()
            P.assemble_device(dU.data_ptr(), 1.0, flags)
            kt += P.kernel_times()
        P.set_timing(False)
        return kt / reps

    clk = Clocks(local).__enter__()
    ms64 = timed(capi.FUNC | capi.JAC, args.steps, args.warmup)
    ms32 = timed(capi.FUNC | capi.JAC | capi.FP32, args.steps, args.warmup)
    kt64 = kernel_times(capi.FUNC | capi.JAC)
    kt32 = kernel_times(capi.FUNC | capi.JAC | capi.FP32)
    value = ws * ne * args.steps / (ms64 * 1e-3)
    value32 = ws * ne * args.steps / (ms32 * 1e-3)

    # end to end through the C ABI with host buffers (pinned), H2D of U and D2H of K, P inside
    hU = torch.from_numpy(U).pin_memory()
    outs = {f"K_{b}": torch.empty(max(P.nnz[i], 1), dtype=torch.float64).pin_memory()
            for i, b in enumerate(("ff", "fp", "pf", "pp"))}
    outs["P_f"] = torch.empty(max(P.n_free, 1), dtype=torch.float64).pin_memory()
    outs["P_p"] = torch.empty(max(P.n_const, 1), dtype=torch.float64).pin_memory()
    out_np = {k: v.numpy() for k, v in outs.items()}
    hU_np = hU.numpy()
    if three_d:
        hRf = torch.empty(max(1, dRf.numel()), dtype=torch.float64).pin_memory()
        hRp = torch.empty(max(1, dRp.numel()), dtype=torch.float64).pin_memory()

    # keep: the caller's K arrays keep the values of the previous call (PG_KEEP_STATIC), so only
    # the values that can change come back; the first call of each mode copies everything
    first = P.changing_values()

    def step_host(keep: bool, full_copy: bool):
        if not three_d:
            P.assemble(hU_np, 1.0, capi.FUNC | capi.JAC | (capi.KEEP_STATIC if keep else 0), out=out_np)
            return
        # U in once; K and R of the first strain, the five other residuals in one pass; K (or
        # its changing values) and the six residuals out
        dU.copy_(hU, non_blocking=True)
        P.set_macro_strain(UNIT_STRAINS_3D[0])
        P.assemble_device(dU.data_ptr(), 1.0, capi.FUNC | capi.JAC)
        P.residual_strains(dU.data_ptr(), UNIT_STRAINS_3D[1:], dRf.data_ptr(), dRp.data_ptr() if P.n_const else 0)
        K4, pf, pp = P.device_outputs()
        for i, b in enumerate(("ff", "fp", "pf", "pp")):
            lo = 0 if full_copy else first[i]
            if P.nnz[i] > lo:
                outs[f"K_{b}"][lo:P.nnz[i]].copy_(capi.device_view(K4[i], P.nnz[i])[lo:], non_blocking=True)
        outs["P_f"][:P.n_free].copy_(capi.device_view(pf, P.n_free), non_blocking=True)
        if P.n_const:
            outs["P_p"][:P.n_const].copy_(capi.device_view(pp, P.n_const), non_blocking=True)
            hRp[:dRp.numel()].copy_(dRp, non_blocking=True)
        hRf[:dRf.numel()].copy_(dRf, non_blocking=True)

    def e2e_run(keep: bool):
        # warm-up: the first call copies every value (and fills the kept arrays)
        for w in range(args.warmup):
            step_host(keep, full_copy=(not keep) or w == 0)
        torch.cuda.synchronize()
        replicas.barrier()
        ms = 0.0
        for _ in range(args.e2e_steps or args.steps):
            flush.zero_()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            step_host(keep, full_copy=not keep)
            b.record(stream)
            b.synchronize()
            ms += a.elapsed_time(b)
        return replicas.max_over_ranks([ms], "cuda")[0]

    e2e_full_ms = e2e_run(False)
    e2e_ms = e2e_run(True)
    clk.__exit__(None, None, None)
    e2e_steps = args.e2e_steps or args.steps
    e2e_value = ws * ne * e2e_steps / (e2e_ms * 1e-3)
    e2e_full_value = ws * ne * e2e_steps / (e2e_full_ms * 1e-3)
    n_rhs = 6 if three_d else 1
    h2d = U.nbytes
    d2h_full = 8 * (sum(P.nnz) + n_rhs * (P.n_free + P.n_const))
    d2h = 8 * (sum(max(0, P.nnz[i] - first[i]) for i in range(4)) + n_rhs * (P.n_free + P.n_const))

    batched = None
    if args.workload == "cohesive_2d_512" and not args.no_batched:
        batched = batched_summary(args, ws, rank)
    # roofline of the dominant kernel (the fast row kernel), from the live per-kernel events
    peak, peak_kind = measured_peak_hbm()
    fk_bytes = fast_kernel_bytes(P, False)
    fk_ms = float(kt64[1])
    achieved = fk_bytes / (fk_ms * 1e-3) / 1e9 if fk_ms > 0 else None
    alg = algorithmic_bytes(P, False)
    alg32 = algorithmic_bytes(P, True)
    if three_d:
        # the five extra right-hand sides write their residuals (one pass reads the nodes once)
        extra = 5 * 8 * (P.n_free + P.n_const)
        alg["total"] += extra
    stencil_name = f"k_rows_tile{P.dim}<double,1>"
    general_name = f"k_gen_rows<{P.dim}>"
    gk_bytes = general_kernel_bytes(P, False)
    gk_ms = float(kt64[2])
    g_achieved = gk_bytes / (gk_ms * 1e-3) / 1e9 if gk_ms > 0 else None

    line = None
    if rank == 0:
        cpu = None
        if ws == 1 and not args.no_cpu_baseline:
            cpu = cpu_baseline(args, R, P, U, out_np)
        setup = setup_times(R)
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms64 / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": DATA,
            "config": bench_config(args, {"elements": ne, "nnz": int(sum(P.nnz)), "cut_elements": P.sizes["n_cut_elem"],
                                          "cohesive_qps": P.sizes["n_coh_qp"]}, ws),
            "fp32_mixed": {"value": value32, "unit": UNIT, "ms_per_step": ms32 / args.steps, "speedup_vs_fp64": value32 / value,
                           "kernel_ms": [float(x) for x in kt32]},
            "kernel_ms": {"cohesive_elements_and_records": float(kt64[0]), "rows_stencil": float(kt64[1]),
                          "rows_general": float(kt64[2]), "assembly": float(kt64[3])},
            "algorithmic_bytes_per_step": alg["total"], "algorithmic_bytes_per_element": alg["total"] / ne,
            "algorithmic_gbs": alg["total"] / (ms64 / args.steps * 1e-3) / 1e9,
            "roofline": {"bound": "hbm", "kernel": f"{stencil_name} " + ("(low-priority stream, concurrent with the cohesive and general-row kernels)" if P.dim == 2 else "(main stream, alone)"),
                         "achieved": achieved, "peak": peak,
                         "peak_kind": peak_kind, "unit": "GB/s", "frac": (achieved / peak) if achieved else None,
                         "traffic": profiled_traffic(stencil_name), "bytes_per_launch": fk_bytes,
                         "traffic_note": "ncu dram read+write per launch, cold cache; row writes still in L2 at kernel end are not counted"},
            # the longest-running kernel (the stencil kernel above moves most of the bytes)
            "roofline_general": {"bound": "hbm", "kernel": f"{general_name} " + ("(high-priority stream, after the cohesive elements and records, sharing the SMs with the stencil rows)" if P.dim == 2 else "(main stream, after the stencil rows, alone)"),
                                 "achieved": g_achieved, "peak": peak, "peak_kind": peak_kind, "unit": "GB/s",
                                 "frac": (g_achieved / peak) if g_achieved else None,
                                 "traffic": profiled_traffic(general_name), "bytes_per_launch": gk_bytes},
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "ms_per_step": e2e_ms / e2e_steps, "steps": e2e_steps,
                    "mode": "PG_KEEP_STATIC: the caller's host K arrays keep the previous call's values; every step "
                            "copies U in and, out, the K values that can change (rows of DOFs on cohesive elements) "
                            "and all residuals",
                    "full_copy": {"value": e2e_full_value, "ms_per_step": e2e_full_ms / e2e_steps,
                                  "d2h_bytes_per_step": d2h_full}},
            # 3D: the K-and-R assembly and the multi-strain pass launch the same set of kernels
            "gpu_launches": launches_per_step(P, three_d) * args.steps,
            "clocks": clk.summary(),
            "cpu_baseline": cpu,
            "batched": batched,
            "setup": setup,
        }
    replicas.finish()
    if line is not None:
        print(json.dumps(line))


def cpu_baseline(args, R, P, U, gpu_out):
    """The reference's assembly (oracle/_ref) on this host, one core, same RVE and state; and,
    outside every timed region, the relative Frobenius error of this library's K and R (gpu_out,
    the last end-to-end step's host outputs) against the reference's on that state."""
    try:
        from oracle import ref
        if not ref.available():
            return None
        RP, Ud = reference_problem(R, P, U)
        sec, n_timed = reference_step_seconds(args, RP, Ud, budget_s=20.0, max_steps=5)
        if args.workload == "linear_3d_64":
            RP.set_macro(UNIT_STRAINS_3D[0])
            RP.assemble(Ud, None, 1.0)

        def rel(a, b):
            nb = float(np.linalg.norm(b))
            return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))
        errs = {f"K_{b}": rel(gpu_out[f"K_{b}"][:P.nnz[i]], RP.csr(f"K_{b}")[2]) for i, b in enumerate(("ff", "fp", "pf", "pp"))}
        errs["P_f"] = rel(gpu_out["P_f"][:P.n_free], RP.get("P_f"))
        errs["P_p"] = rel(gpu_out["P_p"][:P.n_const], RP.get("P_p")) if P.n_const else 0.0
        RP.close()
        ne = P.sizes["n_elem"]
        return {"value": ne / sec, "unit": UNIT, "cores": 1, "kind": "reference",
                "sample": f"mean of {n_timed} steps (bounded at ~20 s) of Assembler::assemble on the same {ne}-element RVE and state, after 1 warm-up",
                **host_info(), "fp64_rel_error_vs_reference": errs}
    except Exception as e:  # the baseline is reported, never required
        return {"error": str(e)}


if __name__ == "__main__":
    main()
