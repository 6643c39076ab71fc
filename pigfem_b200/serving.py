"""Serving loop: RVE requests admitted by device memory and processed concurrently on one GPU.

Requests arrive (Poisson, or as a list), each with a seeded geometry.  Two kinds:

* ``homogenize`` -- linear elastic, periodic (subscale) RVE: one K, one right-hand side per unit
  macroscale strain, all solved together by the device Jacobi-PCG to 1e-8, then the homogenized
  stress of every load case: the effective modulus C (3 x 3 in 2D, 6 x 6 in 3D).
* ``cohesive_step`` -- cohesive RVE under prescribed displacement: the tangent K and residual R
  of one load step at a seeded interface state, with the damage state (internal variables) on the
  device; the result is the residual norm and the damage-zone census of the cohesive points.

Pipeline (all stages run at once on different requests):

1. set-up workers (host threads) run the C++ IGFEM set-up of each arrived request
   (pg_create_host; ctypes releases the GIL, so they run in parallel on the host cores);
2. the admission controller admits set-up requests in arrival order while the sum of the device
   bytes of the admitted requests stays within the budget and a GPU slot is free -- a request
   that arrives while others are on the GPU is admitted as soon as slots and memory free up;
3. GPU workers upload the admitted request (stream-ordered allocations, no device-wide
   synchronisation), run its work on its own CUDA stream, so the work of all admitted requests
   overlaps on the device, read back the small result and free the context.

Every kernel is deterministic (no atomics in the assembly, fixed-order reductions in the norms
and the PCG), and each request runs on its own context, so a request's result is bitwise the same
alone and in the mix; tests/test_serving_gpu.py checks exactly that.
"""
from __future__ import annotations

import math
import queue
import threading
import time
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass, field
from typing import Dict, List, Optional

import numpy as np

from . import capi, rve


@dataclass
class Request:
    rid: int
    kind: str            # "homogenize" | "cohesive_step"
    desc: capi.ProblemDesc
    arrival: float = 0.0  # seconds after the stream start
    seed: int = 0


@dataclass
class Result:
    rid: int
    kind: str
    elements: int
    values: Dict[str, np.ndarray]
    arrival: float = 0.0
    setup_done: float = 0.0
    admitted: float = 0.0
    done: float = 0.0
    device_bytes: int = 0
    error: str = ""

    @property
    def latency(self) -> float:
        return self.done - self.arrival


# ------------------------------------------------------------------ request generation
def make_request(rid: int, seed: int = 1, workload: int = 5, scale: float = 1.0) -> Request:
    """A seeded request: 70 % 2D (grid 32^2-512^2 log-uniform, 5-300 fibers), 30 % 3D tet4 (grid
    16^3-64^3 log-uniform, 5-60 spheres); 60 % homogenization, 40 % cohesive load step.  `scale`
    shrinks the grid ranges and counts (tests)."""
    rng = rve.philox(workload, seed, rid)
    two_d = rng.uniform() < 0.7
    kind = "homogenize" if rng.uniform() < 0.6 else "cohesive_step"
    subscale = kind == "homogenize"
    if two_d:
        n = max(8, int(round(scale * math.exp(rng.uniform(math.log(32), math.log(512))))))
        nf = max(1, int(round(scale * rng.integers(5, 301))))
        fib = np.zeros((0, 3))
        for _ in range(20):
            fib = rve.place_fibers(rng, nf, 0.008, 0.015, 0.002, 2, max_attempts=20000)
            if rve.surface_clearance_ok(fib, n, 2):
                break
        desc = capi.ProblemDesc(elem_type=capi.TRI3, n=(n, n), lo=(0.0, 0.0), hi=(1.0, 1.0), inclusions=fib,
                                E_matrix=rve.E_MATRIX, nu_matrix=rve.NU_MATRIX, E_fiber=rve.E_FIBER,
                                nu_fiber=rve.NU_FIBER, coh_law=capi.COH_NONE if subscale else capi.COH_BL,
                                coh=(0.0,) * 4 if subscale else rve.BL_PARAMS, plane_strain=True, subscale=subscale,
                                eps_macro=(1.0, 0.0, 0.0), app_strain=0.02)
    else:
        n = max(6, int(round(scale * math.exp(rng.uniform(math.log(16), math.log(64))))))
        ns = max(1, int(round(scale * rng.integers(5, 61))))
        h = 1.0 / n
        gap = max(0.01, 1.8 * h)   # keeps tets from seeing two spheres on coarse grids
        fib = np.zeros((0, 4))
        for _ in range(20):
            fib = rve.place_fibers(rng, ns, 0.04, 0.08, gap, 3, max_attempts=20000,
                                   accept=lambda c, r: rve.sphere_box_ok(c, r, n))
            if rve.surface_clearance_ok(fib, n, 3):
                break
        desc = capi.ProblemDesc(elem_type=capi.TET4, n=(n, n, n), lo=(0.0,) * 3, hi=(1.0,) * 3, inclusions=fib,
                                E_matrix=rve.E_MATRIX, nu_matrix=rve.NU_MATRIX, E_fiber=rve.E_FIBER,
                                nu_fiber=rve.NU_FIBER, coh_law=capi.COH_NONE if subscale else capi.COH_BL,
                                coh=(0.0,) * 4 if subscale else rve.BL_PARAMS, plane_strain=False, subscale=subscale,
                                eps_macro=(1.0, 0.0, 0.0, 0.0, 0.0, 0.0), app_strain=0.02)
    return Request(rid, kind, desc, seed=seed)


def poisson_stream(n: int, rate: float, seed: int = 1, scale: float = 1.0) -> List[Request]:
    """n seeded requests with exponential inter-arrival times of mean 1/rate seconds."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for rid in range(n):
        t += rng.exponential(1.0 / rate)
        r = make_request(rid, seed, scale=scale)
        r.arrival = t
        out.append(r)
    return out


# ------------------------------------------------------------------ the work of one request
def device_bytes(P: capi.Problem) -> int:
    """Device memory of a context and its request's work (mesh tables, CSR values, solver
    workspace), estimated from its sizes."""
    s = P.sizes
    nnz = sum(s["nnz"])
    nodes = s["n_nodes"] * s["dim"]
    nv = 3 if s["dim"] == 2 else 6
    return int(12 * nnz + 8 * 12 * nodes + 8 * (4 * nv + 6) * (s["n_free"] + 1) + 200 * s["n_elem"] + (1 << 20))


def run_request(P: capi.Problem, req: Request, stream) -> Dict[str, np.ndarray]:
    """The request's GPU work on `stream` (a torch.cuda.Stream); returns its small result."""
    import torch
    P.set_stream(stream.cuda_stream)
    dim = P.dim
    nn = P.n_nodes * dim
    with torch.cuda.stream(stream):
        if req.kind == "homogenize":
            nv = 3 if dim == 2 else 6
            n = P.n_free
            zero = torch.zeros(nn, dtype=torch.float64, device="cuda")
            rhs = torch.empty(nv * n, dtype=torch.float64, device="cuda")
            rhs_p = torch.empty(max(1, nv * P.n_const), dtype=torch.float64, device="cuda")
            # K once, then the residual of every unit macroscale strain in one pass
            P.assemble_device(zero.data_ptr(), 1.0, capi.JAC)
            P.residual_strains(zero.data_ptr(), [list(np.eye(nv)[k]) for k in range(nv)], rhs.data_ptr(),
                               rhs_p.data_ptr() if P.n_const else 0)
            x = torch.zeros_like(rhs)
            it, rr = P.pcg_solve(rhs.data_ptr(), x.data_ptr(), nv, 1e-8, 200000)
            _, dofs, _ = P.nodes()
            idx = torch.from_numpy(dofs.reshape(-1).astype(np.int64)).to("cuda")
            C = np.zeros((nv, nv))
            U = torch.zeros(n + P.n_const, dtype=torch.float64, device="cuda")
            for k in range(nv):
                e = [0.0] * nv
                e[k] = 1.0
                P.set_macro_strain(e)
                U[:n] = -x[k * n:(k + 1) * n]
                Un = U[idx].contiguous()
                C[:, k] = P.homogenize(Un.data_ptr(), 1.0)[:nv]
            return {"C": C, "pcg_iterations": it.astype(np.int64)}
        # cohesive load step: seeded interface openings, damage state on the device
        U = rve.interface_state(P, seed=req.rid)
        dU = torch.from_numpy(U).to("cuda", non_blocking=False)
        if P.n_isv:
            P.set_isv(np.zeros(P.n_isv))
        P.assemble_device(dU.data_ptr(), 1.0, capi.FUNC | capi.JAC)
        res = P.residual_norm()
        zones = P.damage_zones() if P.n_isv or P.sizes["n_coh_qp"] else np.zeros(0, np.uint8)
        return {"residual_norm": np.array([res]), "zones": np.bincount(zones, minlength=4).astype(np.int64)}


def homogenization_csv(result: Result) -> str:
    """A homogenization request's result as the reference's homogenization CSV
    (WriterHomogenization): one row per unit macroscale strain e_k at t = 1, ``1, e_k..., C[:, k]...``."""
    from . import writers
    C = result.values["C"]
    nv = C.shape[0]
    return writers.homogenization_table(1.0, np.eye(nv), C.T)


def run_alone(req: Request) -> Result:
    """One request by itself: set-up, upload, work, free (the one-at-a-time plain FP64 call)."""
    import torch
    t0 = time.perf_counter()
    P = capi.Problem(req.desc)
    stream = torch.cuda.Stream()
    vals = run_request(P, req, stream)
    stream.synchronize()
    out = Result(req.rid, req.kind, P.sizes["n_elem"], vals, 0.0, 0.0, 0.0, time.perf_counter() - t0, device_bytes(P))
    P.close()
    return out


# ------------------------------------------------------------------ the engine
class ServingEngine:
    """Continuous-batching request loop on one GPU (see the module docstring)."""

    def __init__(self, memory_budget: int, max_inflight: int = 8, setup_workers: int = 8):
        self.budget = int(memory_budget)
        self.max_inflight = max_inflight
        self.setup_workers = setup_workers

    def run(self, requests: List[Request], realtime: bool = True) -> List[Result]:
        import torch
        torch.cuda.init()
        dev = torch.cuda.current_device()
        results: Dict[int, Result] = {}
        ready: "queue.Queue" = queue.Queue()
        lock = threading.Condition()
        state = {"used": 0, "inflight": 0}
        t_start = time.perf_counter()
        now = lambda: time.perf_counter() - t_start

        def setup(req: Request):
            if realtime:
                wait = req.arrival - now()
                if wait > 0:
                    time.sleep(wait)
            r = Result(req.rid, req.kind, 0, {}, arrival=req.arrival if realtime else now())
            try:
                P = capi.Problem(req.desc, device=False)
            except capi.PigfemError as e:
                r.error = str(e)
                r.done = now()
                ready.put((req, None, r))
                return
            r.elements = P.sizes["n_elem"]
            r.device_bytes = device_bytes(P)
            r.setup_done = now()
            ready.put((req, P, r))

        def gpu_work(req: Request, P: capi.Problem, r: Result):
            torch.cuda.set_device(dev)
            stream = torch.cuda.Stream()
            try:
                P.upload()
                r.values = run_request(P, req, stream)
                stream.synchronize()
            except capi.PigfemError as e:
                r.error = str(e)
            finally:
                P.close()
                r.done = now()
                with lock:
                    state["used"] -= r.device_bytes
                    state["inflight"] -= 1
                    results[req.rid] = r
                    lock.notify_all()

        setup_pool = ThreadPoolExecutor(self.setup_workers)
        gpu_pool = ThreadPoolExecutor(self.max_inflight)
        for req in sorted(requests, key=lambda q: q.arrival):
            setup_pool.submit(setup, req)
        # admission in set-up completion order, which follows arrival order up to set-up time
        pending: List = []
        n_left = len(requests)
        while n_left:
            try:
                item = ready.get(timeout=0.05)
                pending.append(item)
            except queue.Empty:
                pass
            pending.sort(key=lambda it: it[0].arrival)
            while pending:
                req, P, r = pending[0]
                if P is None:
                    with lock:
                        results[req.rid] = r
                    pending.pop(0)
                    n_left -= 1
                    continue
                with lock:
                    fits = state["used"] + r.device_bytes <= self.budget or state["inflight"] == 0
                    if not (fits and state["inflight"] < self.max_inflight):
                        break
                    state["used"] += r.device_bytes
                    state["inflight"] += 1
                r.admitted = now()
                pending.pop(0)
                n_left -= 1
                gpu_pool.submit(gpu_work, req, P, r)
        gpu_pool.shutdown(wait=True)
        setup_pool.shutdown(wait=True)
        return [results[q.rid] for q in requests]


def summarize(results: List[Result], wall: float) -> dict:
    lat = np.array([r.latency for r in results if not r.error])
    return {"requests": len(results), "errors": sum(1 for r in results if r.error),
            "req_per_s": len(lat) / wall if wall > 0 else None,
            "p50_s": float(np.percentile(lat, 50)) if len(lat) else None,
            "p99_s": float(np.percentile(lat, 99)) if len(lat) else None,
            "elements": int(sum(r.elements for r in results))}
