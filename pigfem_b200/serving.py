"""Serving loop: RVE requests admitted by device memory and processed concurrently on one GPU.

Requests arrive (Poisson, or as a list), each with a seeded geometry.  Two kinds:

* ``homogenize`` -- linear elastic, periodic (subscale) RVE: one K, one right-hand side per unit
  macroscale strain, all solved together by the device Jacobi-PCG to 1e-8, then the homogenized
  stress of every load case: the effective modulus C (3 x 3 in 2D, 6 x 6 in 3D).
* ``cohesive_step`` -- cohesive RVE under prescribed displacement: the tangent K and residual R
  of one load step at a seeded interface state, with the damage state (internal variables) on the
  device; the result is the residual norm and the damage-zone census of the cohesive points.
  A request may belong to a *session*: the load steps k = 0 .. steps-1 of one RVE, each at the
  fraction (k+1)/steps of the session's interface state, the converged internal variables
  committed after each step (the reference's ``InternalVars::copy_data_in`` after a converged
  load step, src/SolverNonlinear.cpp:96-97, 301).  The session's context -- mesh tables, CSR
  structure, displacements and committed internal variables -- stays on the device from its
  first step to its last; its steps run in order.

Pipeline (all stages run at once on different requests):

1. set-up workers (host threads) run the IGFEM set-up of each arrived request: its per-node and
   per-element passes (detection, enrichment nodes, standard DOF numbering) on the device, on a
   stream of their own, and the cut elements' tables and the CSR pattern in C++
   (pg_create_prep_device with PG_PREP_NODES: the device pattern's sorts would compete with the
   admitted requests' work; ctypes releases the GIL, so the workers run in parallel on the host
   cores);
2. the admission controller admits set-up requests in arrival order while the sum of the device
   bytes of the admitted requests stays within the budget and a GPU slot is free -- a request
   that arrives while others are on the GPU is admitted as soon as slots and memory free up.  A
   request's bytes are its size estimate scaled by the largest ratio of measured to estimated
   bytes seen so far (pg_device_bytes, the peak a finished request held), and once its context is
   on the device the ledger holds the measured bytes; a resident session keeps its bytes until
   its last step;
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

# Ortiz-Pandolfi interfaces of the load-step sessions (sigma_c, delta_c, beta, unused;
# src/Material_OPCohesive.cpp): a law with a committed maximum opening, so the steps carry damage
OP_PARAMS = (50.0, 2e-4, 1.0, 0.0)


@dataclass
class Request:
    rid: int
    kind: str            # "homogenize" | "cohesive_step"
    desc: capi.ProblemDesc
    arrival: float = 0.0  # seconds after the stream start
    seed: int = 0
    session: int = -1     # cohesive load-step session (-1: a one-off request)
    step: int = 0         # load step within the session
    steps: int = 1        # load steps of the session; the last one frees the resident context


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
    device_bytes: int = 0        # bytes the admission ledger charged (estimate x calibration)
    measured_bytes: int = 0      # the most device memory the request's context held
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


def poisson_stream(n: int, rate: float, seed: int = 1, scale: float = 1.0, session_steps: int = 1) -> List[Request]:
    """n seeded requests with exponential inter-arrival times of mean 1/rate seconds.  With
    session_steps > 1 every cohesive request opens a session of that many load steps (the
    Ortiz-Pandolfi law, whose committed maximum opening the steps carry), the later steps
    arriving as further requests of the stream; the stream then holds n first requests."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for base in range(n):
        t += rng.exponential(1.0 / rate)
        r = make_request(base, seed, scale=scale)
        r.arrival = t
        if session_steps > 1 and r.kind == "cohesive_step":
            r.desc.coh_law, r.desc.coh = capi.COH_OP, OP_PARAMS
            r.session, r.steps = base, session_steps
            ts = t
            for k in range(1, session_steps):
                ts += rng.exponential(1.0 / rate)
                out.append(Request(0, r.kind, r.desc, ts, seed, session=base, step=k, steps=session_steps))
        out.append(r)
    out.sort(key=lambda q: (q.arrival, q.session, q.step))
    for rid, q in enumerate(out):
        q.rid = rid
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
        # cohesive load step: seeded interface openings (step k of a session at (k+1)/steps of
        # the session's state), damage state on the device; a session commits the step's
        # internal variables for the next one
        frac = (req.step + 1) / req.steps
        U = rve.interface_state(P, seed=req.session if req.session >= 0 else req.rid) * frac
        dU = torch.from_numpy(U).to("cuda", non_blocking=False)
        if req.step == 0 and P.n_isv:
            P.set_isv(np.zeros(P.n_isv))
        P.assemble_device(dU.data_ptr(), frac, capi.FUNC | capi.JAC)
        res = P.residual_norm()
        zones = P.damage_zones() if P.n_isv or P.sizes["n_coh_qp"] else np.zeros(0, np.uint8)
        out = {"residual_norm": np.array([res]), "zones": np.bincount(zones, minlength=4).astype(np.int64)}
        if req.session >= 0 and P.n_isv:
            P.commit_isv()
            # the carried state: the committed internal variables (maximum openings), summed
            out["committed_isv_sum"] = np.array([float(np.sum(P.get_isv(trial=False)))])
        return out


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
    out.measured_bytes = P.device_bytes()[1]
    P.close()
    return out


def run_session_alone(reqs: List[Request]) -> List[Result]:
    """The steps of one session by themselves, in order, on one context."""
    import torch
    reqs = sorted(reqs, key=lambda q: q.step)
    P = capi.Problem(reqs[0].desc)
    stream = torch.cuda.Stream()
    out = []
    for req in reqs:
        t0 = time.perf_counter()
        vals = run_request(P, req, stream)
        stream.synchronize()
        out.append(Result(req.rid, req.kind, P.sizes["n_elem"], vals, 0.0, 0.0, 0.0, time.perf_counter() - t0,
                          device_bytes(P)))
    P.close()
    return out


# ------------------------------------------------------------------ the engine
class ServingEngine:
    """Continuous-batching request loop on one GPU (see the module docstring)."""

    def __init__(self, memory_budget: int, max_inflight: int = 8, setup_workers: int = 8, prep_device: bool = True):
        self.budget = int(memory_budget)
        self.max_inflight = max_inflight
        self.setup_workers = setup_workers
        self.prep_device = prep_device   # set-up passes on the device (pg_create_prep_device)
        self.calibration = 1.0        # largest measured / estimated device bytes seen so far
        self.peak_charged = 0         # most bytes the ledger held at once

    def run(self, requests: List[Request], realtime: bool = True) -> List[Result]:
        import torch
        torch.cuda.init()
        dev = torch.cuda.current_device()
        results: Dict[int, Result] = {}
        ready: "queue.Queue" = queue.Queue()
        lock = threading.Condition()
        state = {"used": 0, "inflight": 0}
        # resident sessions: id -> {"P", "stream", "bytes", "next" (step), "busy"}; sessions whose
        # set-up or a step failed (their later steps fail too)
        sessions: Dict[int, dict] = {}
        failed: set = set()
        t_start = time.perf_counter()
        now = lambda: time.perf_counter() - t_start

        def setup(req: Request):
            if realtime:
                wait = req.arrival - now()
                if wait > 0:
                    time.sleep(wait)
            r = Result(req.rid, req.kind, 0, {}, arrival=req.arrival if realtime else now())
            if req.session >= 0 and req.step > 0:
                # the session's context is (or will be) resident: no set-up of its own
                r.setup_done = now()
                ready.put((req, None, r))
                return
            try:
                P = capi.Problem(req.desc, device=False, prep_device=self.prep_device, prep_pattern=False)
            except capi.PigfemError as e:
                r.error = str(e)
                r.done = now()
                if req.session >= 0:
                    with lock:
                        failed.add(req.session)
                ready.put((req, None, r))
                return
            r.elements = P.sizes["n_elem"]
            r.device_bytes = device_bytes(P)
            r.setup_done = now()
            ready.put((req, P, r))

        def charge(delta: int):
            state["used"] += delta
            self.peak_charged = max(self.peak_charged, state["used"])

        def gpu_work(req: Request, P: Optional[capi.Problem], r: Result):
            torch.cuda.set_device(dev)
            sess = sessions.get(req.session) if req.session >= 0 else None
            keep = False
            try:
                if sess is not None and req.step > 0:
                    P, stream = sess["P"], sess["stream"]
                    r.elements = P.sizes["n_elem"]
                else:
                    stream = torch.cuda.Stream()
                    P.upload()
                    # from here on the ledger holds the measured bytes, or the calibrated estimate
                    # while that is larger (it covers the solver workspace still to come)
                    with lock:
                        held = max(r.device_bytes, P.device_bytes()[0])
                        charge(held - r.device_bytes)
                        r.device_bytes = held
                    if req.session >= 0:
                        with lock:
                            sessions[req.session] = {"P": P, "stream": stream, "bytes": r.device_bytes,
                                                     "next": 0, "busy": True}
                        sess = sessions[req.session]
                r.values = run_request(P, req, stream)
                stream.synchronize()
                keep = sess is not None and req.step < req.steps - 1
            except capi.PigfemError as e:
                r.error = str(e)
                if req.session >= 0:
                    with lock:
                        failed.add(req.session)
            finally:
                measured = P.device_bytes()[1] if P is not None else 0
                r.measured_bytes = measured
                est = device_bytes(P) if P is not None else 0
                if not keep and P is not None:
                    P.close()
                r.done = now()
                with lock:
                    if est > 0:
                        self.calibration = max(self.calibration, measured / est)
                    if sess is not None:
                        if keep:
                            # the ledger keeps the session's bytes (now the peak it reached)
                            charge(measured - sess["bytes"])
                            sess["bytes"] = measured
                            sess["next"] = req.step + 1
                            sess["busy"] = False
                        else:
                            charge(-sess["bytes"])
                            sessions.pop(req.session, None)
                    else:
                        charge(-r.device_bytes)
                    state["inflight"] -= 1
                    results[req.rid] = r
                    lock.notify_all()

        setup_pool = ThreadPoolExecutor(self.setup_workers)
        gpu_pool = ThreadPoolExecutor(self.max_inflight)
        for req in sorted(requests, key=lambda q: q.arrival):
            setup_pool.submit(setup, req)
        # admission in arrival order: a one-off request or a session's first step that does not
        # fit the budget stops the requests behind it; a later session step needs no new memory
        # and waits only for its session's previous step
        pending: List = []
        n_left = len(requests)
        while n_left:
            try:
                item = ready.get(timeout=0.02)
                pending.append(item)
            except queue.Empty:
                pass
            pending.sort(key=lambda it: it[0].arrival)
            i = 0
            while i < len(pending):
                req, P, r = pending[i]
                continuing = req.session >= 0 and req.step > 0
                if P is None and not continuing:
                    with lock:
                        results[req.rid] = r
                    pending.pop(i)
                    n_left -= 1
                    continue
                with lock:
                    if state["inflight"] >= self.max_inflight:
                        break
                    if continuing and req.session in failed:
                        r.error = "an earlier step of the session failed"
                        r.done = now()
                        results[req.rid] = r
                        pending.pop(i)
                        n_left -= 1
                        continue
                    if continuing:
                        sess = sessions.get(req.session)
                        if sess is None or sess["busy"] or sess["next"] != req.step:
                            i += 1
                            continue
                        sess["busy"] = True
                        r.device_bytes = 0
                    else:
                        want = int(r.device_bytes * self.calibration)
                        if not (state["used"] + want <= self.budget or state["inflight"] == 0):
                            break
                        r.device_bytes = want
                        charge(want)
                    state["inflight"] += 1
                r.admitted = now()
                pending.pop(i)
                n_left -= 1
                gpu_pool.submit(gpu_work, req, P, r)
            with lock:
                # a session step waits for its predecessor: sleep until something finishes
                if pending and state["inflight"] > 0 and ready.empty():
                    lock.wait(timeout=0.02)
        gpu_pool.shutdown(wait=True)
        setup_pool.shutdown(wait=True)
        # a session cut short (an error in one of its steps) frees its context here
        for sess in sessions.values():
            sess["P"].close()
        return [results[q.rid] for q in requests]


def summarize(results: List[Result], wall: float) -> dict:
    lat = np.array([r.latency for r in results if not r.error])
    return {"requests": len(results), "errors": sum(1 for r in results if r.error),
            "req_per_s": len(lat) / wall if wall > 0 else None,
            "p50_s": float(np.percentile(lat, 50)) if len(lat) else None,
            "p99_s": float(np.percentile(lat, 99)) if len(lat) else None,
            "elements": int(sum(r.elements for r in results))}
