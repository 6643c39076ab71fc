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

METRIC = "assembled elems/s (K+R) FP64 vs FP32-mixed; served RVE req/s with p50/p99"
UNIT = "elements/s"
WORKLOAD = "cohesive_2d_512: 512x512 tri3 split (524,288 tri3), 200 circular fibers, bilinear cohesive interfaces"
L2_FLUSH_BYTES = 256 << 20


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=300)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", choices=("ours", "reference"), default="ours")
    p.add_argument("--grid", type=int, default=512)
    p.add_argument("--fibers", type=int, default=200)
    p.add_argument("--no-cpu-baseline", action="store_true")
    return p.parse_args()


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


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


def launches_per_step(P) -> int:
    """Kernels one assembly launches: cohesive points, stencil rows and general rows, each only
    when it has work (the L2 flush between steps is a torch fill, not counted)."""
    s = P.sizes
    return int(s["n_coh_qp"] > 0) + int(len(P.debug("fast_dn")) > 0) + int(len(P.debug("slow_dn")) > 0)


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


def build_problem(args, rank):
    from pigfem_b200 import capi, rve
    R = rve.cohesive_2d(n=args.grid, n_fibers=args.fibers, seed=1, request=rank)
    P = capi.Problem(R.desc)
    U = rve.interface_state(P, seed=rank)
    return R, P, U


def run_reference(args, ws, rank):
    """The reference's own CPU assembly (oracle/_ref, built from its sources) on rank 0."""
    if rank != 0:
        return
    from oracle import ref
    if not ref.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libpigfem_ref.so not built (make -C oracle)"}))
        return
    from pigfem_b200 import rve
    R = rve.cohesive_2d(n=args.grid, n_fibers=args.fibers, seed=1, request=0)
    RP = ref.RefProblem(ref.ProblemSpec(elem_type=0, n=(args.grid, args.grid), inclusions=R.fibers,
                                        coh_law=R.desc.coh_law, coh=R.desc.coh, app_strain=R.desc.app_strain))
    from pigfem_b200 import capi
    P = capi.Problem(R.desc, device=False)
    U = rve.interface_state(P, seed=0)
    _, dofs, _ = P.nodes()
    Ud = np.zeros(RP.n_free + RP.n_const)
    Ud[dofs.reshape(-1)] = U
    RP.assemble(Ud, None, 1.0)
    for _ in range(args.warmup):
        RP.time_assemble(1)
    t = [RP.time_assemble(1) for _ in range(args.steps)]
    ne = P.sizes["n_elem"]
    ms = 1e3 * float(np.mean(t))
    value = ne / (ms * 1e-3)
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded fiber layout)", "impl": "reference",
            "config": {"workload": WORKLOAD, "elements": ne, "l2": "cpu run", "parallelism": "single core"},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": 1, "kind": "reference",
                             "sample": f"{args.steps} full assemblies of the {ne}-element RVE (Assembler::assemble, K+R)"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def main():
    args = parse()
    ws, rank, local = dist_env()
    if args.impl == "reference":
        run_reference(args, ws, rank)
        return
    import torch
    import torch.distributed as dist
    torch.cuda.set_device(local)
    if ws > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    from pigfem_b200 import capi
    R, P, U = build_problem(args, rank)
    ne = P.sizes["n_elem"]
    stream = torch.cuda.current_stream()
    P.set_stream(stream.cuda_stream)
    dU = torch.from_numpy(U).cuda()
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")

    def timed(flags, steps, warmup, kernel_times=False):
        for _ in range(warmup):
            P.assemble_device(dU.data_ptr(), 1.0, flags)
        torch.cuda.synchronize()
        if ws > 1:
            dist.barrier()
        torch.cuda.synchronize()
        P.set_timing(kernel_times)
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        kt = np.zeros(4)
        for i in range(steps):
            flush.zero_()
            ev[i][0].record(stream)
            P.assemble_device(dU.data_ptr(), 1.0, flags)
            ev[i][1].record(stream)
            if kernel_times:
                kt += P.kernel_times()
        torch.cuda.synchronize()
        P.set_timing(False)
        ms = float(sum(a.elapsed_time(b) for a, b in ev))
        if ws > 1:
            t = torch.tensor([ms], device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = float(t.item())
            dist.barrier()
        torch.cuda.synchronize()
        return ms, kt / steps

    clk = Clocks(local).__enter__()
    ms64, kt64 = timed(capi.FUNC | capi.JAC, args.steps, args.warmup, kernel_times=True)
    ms32, kt32 = timed(capi.FUNC | capi.JAC | capi.FP32, args.steps, args.warmup, kernel_times=True)
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
    for _ in range(args.warmup):
        P.assemble(hU_np, 1.0, capi.FUNC | capi.JAC, out=out_np)
    torch.cuda.synchronize()
    if ws > 1:
        dist.barrier()
    e2e_ms = 0.0
    for _ in range(args.steps):
        flush.zero_()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        P.assemble(hU_np, 1.0, capi.FUNC | capi.JAC, out=out_np)
        b.record(stream)
        b.synchronize()
        e2e_ms += a.elapsed_time(b)
    if ws > 1:
        t = torch.tensor([e2e_ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = float(t.item())
    clk.__exit__(None, None, None)
    e2e_value = ws * ne * args.steps / (e2e_ms * 1e-3)
    h2d = U.nbytes
    d2h = 8 * (sum(P.nnz) + P.n_free + P.n_const)

    # roofline of the dominant kernel (the fast row kernel), from the live per-kernel events
    peak, peak_kind = measured_peak_hbm()
    fk_bytes = fast_kernel_bytes(P, False)
    fk_ms = float(kt64[1])
    achieved = fk_bytes / (fk_ms * 1e-3) / 1e9 if fk_ms > 0 else None
    alg = algorithmic_bytes(P, False)
    alg32 = algorithmic_bytes(P, True)

    line = None
    if rank == 0:
        cpu = None
        if ws == 1 and not args.no_cpu_baseline:
            cpu = cpu_baseline(args, R, P, U)
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms64 / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic (seeded fiber layout; reference publishes no data set)",
            "config": {"workload": WORKLOAD, "elements": ne, "nnz": int(sum(P.nnz)), "cut_elements": P.sizes["n_cut_elem"],
                       "cohesive_qps": P.sizes["n_coh_qp"], "l2": f"flushed before every timed step ({L2_FLUSH_BYTES >> 20} MiB write)",
                       "parallelism": f"replicas x{ws} (one RVE per GPU)"},
            "fp32_mixed": {"value": value32, "unit": UNIT, "ms_per_step": ms32 / args.steps, "speedup_vs_fp64": value32 / value,
                           "kernel_ms": [float(x) for x in kt32]},
            "kernel_ms": {"cut_elements": float(kt64[0]), "rows_fast_concurrent": float(kt64[1]),
                          "rows_general": float(kt64[2]), "assembly": float(kt64[3])},
            "algorithmic_bytes_per_step": alg["total"], "algorithmic_bytes_per_element": alg["total"] / ne,
            "algorithmic_gbs": alg["total"] / (ms64 / args.steps * 1e-3) / 1e9,
            "roofline": {"bound": "hbm", "kernel": "k_rows_stencil<2,double> (side stream, concurrent with k_coh_points and k_rows_general)", "achieved": achieved, "peak": peak,
                         "peak_kind": peak_kind, "unit": "GB/s", "frac": (achieved / peak) if achieved else None,
                         "traffic": profiled_traffic("k_rows_stencil<2,double>"), "bytes_per_launch": fk_bytes,
                         "traffic_note": "ncu dram read+write per launch, cold cache; row writes still in L2 at kernel end are not counted"},
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "ms_per_step": e2e_ms / args.steps},
            "gpu_launches": launches_per_step(P) * args.steps,
            "clocks": clk.summary(),
            "cpu_baseline": cpu,
        }
    if ws > 1:
        dist.barrier()
        dist.destroy_process_group()
    if line is not None:
        print(json.dumps(line))


def cpu_baseline(args, R, P, U):
    """The reference's assembly (oracle/_ref) on this host, one core, same RVE and state."""
    try:
        from oracle import ref
        if not ref.available():
            return None
        RP = ref.RefProblem(ref.ProblemSpec(elem_type=0, n=(args.grid, args.grid), inclusions=R.fibers,
                                            coh_law=R.desc.coh_law, coh=R.desc.coh, app_strain=R.desc.app_strain))
        _, dofs, _ = P.nodes()
        Ud = np.zeros(RP.n_free + RP.n_const)
        Ud[dofs.reshape(-1)] = U
        RP.assemble(Ud, None, 1.0)
        med = RP.time_assemble(3)
        RP.close()
        ne = P.sizes["n_elem"]
        return {"value": ne / med, "unit": UNIT, "cores": 1, "kind": "reference",
                "sample": f"median of 3 full Assembler::assemble calls (K+R) on the same {ne}-element RVE and state"}
    except Exception as e:  # the baseline is reported, never required
        return {"error": str(e)}


if __name__ == "__main__":
    main()
