"""ctypes binding of the C ABI in include/pigfem_b200.h (libpigfem_b200.so).

:class:`Problem` is the host-side mirror of the reference's ``Problem`` + ``Assembler`` pair for
the assembly path: it builds the enriched mesh (``Problem::init`` / ``Problem::setup``), then
``assemble`` is ``Assembler::assemble`` (src/Assembler.cpp:65-146) with the same argument meaning:
the nodal displacement field in, the four stiffness blocks K_ff / K_fp / K_pf / K_pp and the two
internal-force parts P_f / P_p out, with the trial internal variables updated from the committed
ones.  Errors raise :class:`PigfemError` carrying the library's status code and message (the
reference prints and exits instead; src/common.h:292-297).

The library is required: there is no CPU fallback.  Loading fails loudly when the CUDA library
has not been built (``python -c "import __graft_entry__ as g; g.build()"``).
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libpigfem_b200.so")

TRI3, QUAD4, TET4 = 0, 1, 2
SENS_E, SENS_LAMBDA, SENS_MU, SENS_K, SENS_NU = range(5)
COH_NONE, COH_BL, COH_BLNU, COH_XN, COH_XNNU, COH_OP, COH_OPNU, COH_OPAUG, COH_OPNUAUG = range(9)
COH_TL, COH_TLNU, COH_STL, COH_STLNU = range(9, 13)   # trilinear and smoothed trilinear
FUNC, JAC, FP32, KEEP_STATIC = 1, 2, 4, 8
PREP_NODES, PREP_PATTERN = 1, 2
ERRORS = {2: "PG_ERR_INPUT", 3: "PG_ERR_GEOMETRY", 4: "PG_ERR_UNSUPPORTED", 7: "PG_ERR_JACOBIAN",
          10: "PG_ERR_DEVICE", 11: "PG_ERR_NONFINITE", 12: "PG_ERR_STATE"}

# Every symbol include/pigfem_b200.h declares.
EXPORTED = [
    "pg_create", "pg_create_host", "pg_create_prep_device", "pg_prep_device_ms", "pg_upload", "pg_debug_array", "pg_destroy", "pg_last_error",
    "pg_get_sizes", "pg_device_bytes", "pg_get_pattern", "pg_get_nodes", "pg_assemble", "pg_assemble_device", "pg_residual_strains",
    "pg_device_outputs", "pg_changing_values", "pg_set_stream", "pg_set_isv", "pg_get_isv", "pg_commit_isv",
    "pg_get_damage_zones", "pg_residual_norm", "pg_set_timing", "pg_kernel_times", "pg_set_macro_strain",
    "pg_pcg_solve", "pg_homogenize", "pg_material_sensitivity", "pg_norm2_noalloc",
    "pg_batch_create", "pg_batch_assemble", "pg_batch_wait", "pg_batch_tune", "pg_batch_info",
    "pg_batch_last_error", "pg_batch_destroy",
]


class PigfemError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


class _Desc(ctypes.Structure):
    _fields_ = [
        ("elem_type", ctypes.c_int32), ("n", ctypes.c_int32 * 3), ("lo", ctypes.c_double * 3),
        ("hi", ctypes.c_double * 3), ("n_incl", ctypes.c_int32), ("incl", ctypes.POINTER(ctypes.c_double)),
        ("E_matrix", ctypes.c_double), ("nu_matrix", ctypes.c_double), ("E_fiber", ctypes.c_double),
        ("nu_fiber", ctypes.c_double), ("coh_law", ctypes.c_int32), ("coh", ctypes.c_double * 4),
        ("plane_strain", ctypes.c_int32), ("subscale", ctypes.c_int32), ("eps_macro", ctypes.c_double * 6),
        ("app_strain", ctypes.c_double), ("ply_frac", ctypes.c_double), ("ply", ctypes.c_double * 5),
    ]


class _Sizes(ctypes.Structure):
    _fields_ = [(k, ctypes.c_int32) for k in ("dim", "n_nodes", "n_std_nodes", "n_enrich_nodes", "n_elem",
                                              "n_cut_elem", "n_coh_elem", "n_coh_qp", "n_free", "n_const", "n_isv")] + \
               [("nnz", ctypes.c_int64 * 4), ("cut_scratch_doubles", ctypes.c_int64)]


_lib = None


def load_library(path: Optional[str] = None):
    """Load libpigfem_b200.so (or the build named by PIGFEM_B200_LIB) and declare its signatures;
    raises if it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    path = path or os.environ.get("PIGFEM_B200_LIB") or LIB_PATH
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} is missing: build it first (make -C pigfem_b200/csrc)")
    L = ctypes.CDLL(path)
    vp, i32, dbl, p = ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_void_p
    sig = {
        "pg_create": (i32, [ctypes.POINTER(_Desc), ctypes.POINTER(vp)]),
        "pg_create_host": (i32, [ctypes.POINTER(_Desc), ctypes.POINTER(vp)]),
        "pg_create_prep_device": (i32, [ctypes.POINTER(_Desc), i32, ctypes.POINTER(vp)]),
        "pg_prep_device_ms": (i32, [vp, ctypes.POINTER(ctypes.c_double)]),
        "pg_upload": (i32, [vp]),
        "pg_debug_array": (i32, [vp, ctypes.c_char_p, ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(vp)]),
        "pg_destroy": (None, [vp]),
        "pg_last_error": (ctypes.c_char_p, [vp]),
        "pg_get_sizes": (i32, [vp, ctypes.POINTER(_Sizes)]),
        "pg_device_bytes": (i32, [vp, ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int64)]),
        "pg_get_pattern": (i32, [vp, i32, p, p]),
        "pg_get_nodes": (i32, [vp, p, p, p]),
        "pg_assemble": (i32, [vp, p, dbl, i32, p, p, p, p, p, p]),
        "pg_assemble_device": (i32, [vp, p, dbl, i32]),
        "pg_residual_strains": (i32, [vp, vp, dbl, i32, p, vp, vp]),
        "pg_device_outputs": (i32, [vp, p, p, p]),
        "pg_changing_values": (i32, [vp, p]),
        "pg_set_stream": (i32, [vp, vp]),
        "pg_set_isv": (i32, [vp, p]),
        "pg_get_isv": (i32, [vp, i32, p]),
        "pg_commit_isv": (i32, [vp]),
        "pg_get_damage_zones": (i32, [vp, p]),
        "pg_residual_norm": (i32, [vp, ctypes.POINTER(dbl)]),
        "pg_set_timing": (i32, [vp, i32]),
        "pg_kernel_times": (i32, [vp, p]),
        "pg_set_macro_strain": (i32, [vp, p]),
        "pg_pcg_solve": (i32, [vp, vp, vp, i32, dbl, i32, p, p]),
        "pg_homogenize": (i32, [vp, vp, dbl, p]),
        "pg_material_sensitivity": (i32, [vp, vp, i32, i32, vp, vp]),
        "pg_norm2_noalloc": (i32, [vp, ctypes.c_int64, vp, vp]),
        "pg_batch_create": (i32, [p, i32, ctypes.POINTER(vp)]),
        "pg_batch_assemble": (i32, [vp, p, p, i32]),
        "pg_batch_wait": (i32, [vp, ctypes.POINTER(ctypes.c_float)]),
        "pg_batch_tune": (i32, [vp, p, i32, i32, p]),
        "pg_batch_info": (i32, [vp, p]),
        "pg_batch_last_error": (ctypes.c_char_p, [vp]),
        "pg_batch_destroy": (None, [vp]),
    }
    for name, (rt, args) in sig.items():
        f = getattr(L, name)
        f.restype = rt
        f.argtypes = args
    _lib = L
    return L


def device_view(ptr: int, n: int, typestr: str = "<f8"):
    """A torch tensor viewing n elements of device memory the library owns (e.g. the K values or
    P_f of a context, from Problem.device_outputs); valid while the context lives."""
    import torch

    class _View:
        __cuda_array_interface__ = {"shape": (n,), "typestr": typestr, "data": (int(ptr), False), "version": 3,
                                    "strides": None}
    return torch.as_tensor(_View(), device="cuda")


def _ptr(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data


@dataclass
class ProblemDesc:
    """Problem inputs, as the reference's Tests/Main.cpp assembles them."""
    elem_type: int = TRI3
    n: Sequence[int] = (8, 8)
    lo: Sequence[float] = (0.0, 0.0)
    hi: Sequence[float] = (1.0, 1.0)
    inclusions: np.ndarray = field(default_factory=lambda: np.zeros((0, 3)))
    E_matrix: float = 3.5e3
    nu_matrix: float = 0.35
    E_fiber: float = 72e3
    nu_fiber: float = 0.22
    coh_law: int = COH_NONE
    coh: Sequence[float] = (0.0, 0.0, 0.0, 0.0)
    plane_strain: bool = True
    subscale: bool = False
    eps_macro: Sequence[float] = (0.0,) * 6
    app_strain: float = 0.01
    ply_frac: float = 0.0                       # bounding plies (0: none)
    ply: Sequence[float] = (0.0,) * 5           # E1, E2, G12, G23, nu12

    @property
    def dim(self) -> int:
        return 3 if self.elem_type == TET4 else 2


class Problem:
    """One enriched mesh resident on the GPU (a ``pg_ctx``)."""

    def __init__(self, desc: ProblemDesc, device: bool = True, prep_device: bool = False, prep_pattern: bool = True):
        """``prep_device``: run the set-up's node detection, element pass, enrichment nodes and
        standard DOF numbering on the GPU (pg_create_prep_device), and with ``prep_pattern`` the
        adjacency and CSR pattern too; the tables are the same."""
        L = load_library()
        self.desc = desc
        dim = desc.dim
        self._incl = np.ascontiguousarray(np.asarray(desc.inclusions, dtype=np.float64).reshape(-1, dim + 1))
        d = _Desc()
        d.elem_type = desc.elem_type
        n = list(desc.n) + [0] * 3
        lo = list(desc.lo) + [0.0] * 3
        hi = list(desc.hi) + [0.0] * 3
        for i in range(3):
            d.n[i], d.lo[i], d.hi[i] = n[i], lo[i], hi[i]
        d.n_incl = self._incl.shape[0]
        d.incl = self._incl.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        d.E_matrix, d.nu_matrix, d.E_fiber, d.nu_fiber = desc.E_matrix, desc.nu_matrix, desc.E_fiber, desc.nu_fiber
        d.coh_law = desc.coh_law
        for i, v in enumerate(desc.coh):
            d.coh[i] = v
        d.plane_strain, d.subscale = int(desc.plane_strain), int(desc.subscale)
        for i, v in enumerate(desc.eps_macro):
            d.eps_macro[i] = v
        d.app_strain = desc.app_strain
        d.ply_frac = desc.ply_frac
        for i, v in enumerate(desc.ply):
            d.ply[i] = v
        self._d = d
        h = ctypes.c_void_p(0)
        if prep_device:
            rc = L.pg_create_prep_device(ctypes.byref(d), PREP_NODES | (PREP_PATTERN if prep_pattern else 0), ctypes.byref(h))
        else:
            rc = L.pg_create_host(ctypes.byref(d), ctypes.byref(h))
        self.h = h
        if rc:
            msg = L.pg_last_error(h).decode() if h.value else "invalid description"
            self.close()
            raise PigfemError(rc, msg)
        self.device = False
        self._sizes()
        if device:
            self.upload()

    # ------------------------------------------------------------------ set-up
    def upload(self):
        self._check(load_library().pg_upload(self.h))
        self.device = True
        self._sizes()

    def _check(self, rc: int):
        if rc:
            raise PigfemError(rc, load_library().pg_last_error(self.h).decode())

    def _sizes(self):
        s = _Sizes()
        self._check(load_library().pg_get_sizes(self.h, ctypes.byref(s)))
        self.sizes = {k: getattr(s, k) for k, _ in _Sizes._fields_ if k != "nnz"}
        self.sizes["nnz"] = [int(v) for v in s.nnz]
        self.dim = s.dim
        self.n_nodes, self.n_free, self.n_const, self.n_isv = s.n_nodes, s.n_free, s.n_const, s.n_isv
        self.nnz = self.sizes["nnz"]

    def changing_values(self):
        """First CSR value of each K block from which a later assembly can change values."""
        v = np.zeros(4, np.int64)
        self._check(load_library().pg_changing_values(self.h, _ptr(v)))
        return [int(x) for x in v]

    def device_bytes(self):
        """(bytes held now, most bytes held at once) of this context's device allocations."""
        now, peak = ctypes.c_int64(0), ctypes.c_int64(0)
        self._check(load_library().pg_device_bytes(self.h, ctypes.byref(now), ctypes.byref(peak)))
        return int(now.value), int(peak.value)

    def pattern(self, block: int):
        nrows = [self.n_free, self.n_free, self.n_const, self.n_const][block]
        ncols = [self.n_free, self.n_const, self.n_free, self.n_const][block]
        rp = np.zeros(nrows + 1, np.int32)
        ci = np.zeros(max(self.nnz[block], 1), np.int32)
        self._check(load_library().pg_get_pattern(self.h, block, _ptr(rp), _ptr(ci)))
        return rp, ci[: self.nnz[block]], (nrows, ncols)

    def nodes(self):
        X = np.zeros(self.n_nodes * self.dim)
        dofs = np.zeros(self.n_nodes * self.dim, np.int32)
        dir_ = np.zeros(max(self.n_const, 1))
        self._check(load_library().pg_get_nodes(self.h, _ptr(X), _ptr(dofs), _ptr(dir_)))
        return X.reshape(-1, self.dim), dofs.reshape(-1, self.dim), dir_[: self.n_const]

    def prep_device_ms(self) -> float:
        """Device time of the preprocessing passes (-1 when the set-up ran on the host alone)."""
        ms = ctypes.c_double(0.0)
        self._check(load_library().pg_prep_device_ms(self.h, ctypes.byref(ms)))
        return float(ms.value)

    def debug(self, name: str) -> np.ndarray:
        n = ctypes.c_int64(0)
        p = ctypes.c_void_p(0)
        kind = load_library().pg_debug_array(self.h, name.encode(), ctypes.byref(n), ctypes.byref(p))
        if kind == 0:
            raise KeyError(name)
        if n.value == 0:
            return np.zeros(0, np.int32 if kind == 1 else np.float64)
        ct = ctypes.c_int32 if kind == 1 else ctypes.c_double
        return np.ctypeslib.as_array(ctypes.cast(p, ctypes.POINTER(ct)), shape=(n.value,)).copy()

    # ------------------------------------------------------------------ assembly
    def node_major(self, U_dof: np.ndarray) -> np.ndarray:
        """Scatter a DOF vector (free then constrained) to the node-major NodalData layout."""
        _, dofs, _ = self.nodes()
        return np.ascontiguousarray(np.asarray(U_dof, np.float64)[dofs.reshape(-1)])

    def assemble(self, U_node: np.ndarray, t_frac: float = 1.0, flags: int = FUNC | JAC,
                 out: Optional[dict] = None) -> dict:
        """Assembler::assemble on host buffers; returns {'K_ff','K_fp','K_pf','K_pp','P_f','P_p'}."""
        if not self.device:
            raise PigfemError(12, "context has no device residency (constructed with device=False)")
        U_node = np.ascontiguousarray(U_node, dtype=np.float64)
        if U_node.size != self.n_nodes * self.dim:
            raise PigfemError(2, f"U has {U_node.size} entries, expected {self.n_nodes * self.dim}")
        if out is None:
            out = {f"K_{b}": np.zeros(max(self.nnz[i], 1)) for i, b in enumerate(("ff", "fp", "pf", "pp"))}
            out["P_f"] = np.zeros(max(self.n_free, 1))
            out["P_p"] = np.zeros(max(self.n_const, 1))
        self._check(load_library().pg_assemble(self.h, _ptr(U_node), float(t_frac), int(flags),
                                               _ptr(out["K_ff"]), _ptr(out["K_fp"]), _ptr(out["K_pf"]),
                                               _ptr(out["K_pp"]), _ptr(out["P_f"]), _ptr(out["P_p"])))
        res = {f"K_{b}": out[f"K_{b}"][: self.nnz[i]] for i, b in enumerate(("ff", "fp", "pf", "pp"))}
        res["P_f"] = out["P_f"][: self.n_free]
        res["P_p"] = out["P_p"][: self.n_const]
        return res

    def assemble_device(self, d_U: int, t_frac: float = 1.0, flags: int = FUNC | JAC):
        self._check(load_library().pg_assemble_device(self.h, ctypes.c_void_p(d_U), float(t_frac), int(flags)))

    def device_outputs(self):
        K = (ctypes.c_void_p * 4)()
        pf, pp = ctypes.c_void_p(0), ctypes.c_void_p(0)
        self._check(load_library().pg_device_outputs(self.h, K, ctypes.byref(pf), ctypes.byref(pp)))
        return [K[i] for i in range(4)], pf.value, pp.value

    def set_stream(self, stream_handle: int):
        self._check(load_library().pg_set_stream(self.h, ctypes.c_void_p(stream_handle)))

    def set_isv(self, committed: np.ndarray):
        committed = np.ascontiguousarray(committed, np.float64)
        if committed.size != self.n_isv:
            raise PigfemError(2, f"{committed.size} internal variables given, {self.n_isv} expected")
        self._check(load_library().pg_set_isv(self.h, _ptr(committed)))

    def get_isv(self, trial: bool = True) -> np.ndarray:
        v = np.zeros(max(self.n_isv, 1))
        self._check(load_library().pg_get_isv(self.h, int(trial), _ptr(v)))
        return v[: self.n_isv]

    def commit_isv(self):
        self._check(load_library().pg_commit_isv(self.h))

    def damage_zones(self) -> np.ndarray:
        z = np.zeros(max(self.sizes["n_coh_qp"], 1), np.uint8)
        self._check(load_library().pg_get_damage_zones(self.h, _ptr(z)))
        return z[: self.sizes["n_coh_qp"]]

    def set_macro_strain(self, eps):
        e = np.zeros(6)
        e[:len(eps)] = eps
        self._check(load_library().pg_set_macro_strain(self.h, _ptr(e)))

    def pcg_solve(self, d_b: int, d_x: int, nrhs: int = 1, rtol: float = 1e-10, max_it: int = 100000):
        """Jacobi-PCG on K_ff of the last assembly; d_b / d_x are device pointers to nrhs blocks of
        n_free doubles (x: initial guess in, solution out).  Returns (iterations, relative residuals)."""
        it = np.zeros(nrhs, np.int32)
        rr = np.zeros(nrhs)
        self._check(load_library().pg_pcg_solve(self.h, ctypes.c_void_p(d_b), ctypes.c_void_p(d_x), int(nrhs),
                                                float(rtol), int(max_it), _ptr(it), _ptr(rr)))
        return it, rr

    def residual_strains(self, d_U: int, eps_cases, d_Rf: int, d_Rp: int = 0, t_frac: float = 1.0):
        """Residuals of several macroscale strains in one pass (subscale problems): eps_cases is
        n_cases x (3 or 6) Voigt strains; case k's residual parts land in the device arrays at
        d_Rf + k * n_free and d_Rp + k * n_const (doubles)."""
        e = np.zeros((len(eps_cases), 6))
        for k, ek in enumerate(eps_cases):
            e[k, :len(ek)] = ek
        e = np.ascontiguousarray(e)
        self._check(load_library().pg_residual_strains(self.h, ctypes.c_void_p(d_U), float(t_frac), len(eps_cases),
                                                       _ptr(e), ctypes.c_void_p(d_Rf), ctypes.c_void_p(d_Rp or None)))

    def homogenize(self, d_U: int, t_frac: float = 1.0) -> np.ndarray:
        """Volume-averaged stress (Voigt) and the integrated volume as the last entry."""
        out = np.zeros(7)
        self._check(load_library().pg_homogenize(self.h, ctypes.c_void_p(d_U), float(t_frac), _ptr(out)))
        return out[: (3 if self.dim == 2 else 6) + 1]

    def material_sensitivity(self, d_U: int, material: int, param: int, d_dPf: int, d_dPp: int):
        """dP_int/dp of parameter `param` (SENS_E .. SENS_NU) of `material` (0 matrix, 1 fiber)
        at device displacements d_U, into the device vectors d_dPf (n_free) and d_dPp (n_const)."""
        self._check(load_library().pg_material_sensitivity(self.h, ctypes.c_void_p(d_U), int(material), int(param),
                                                           ctypes.c_void_p(d_dPf), ctypes.c_void_p(d_dPp)))

    def residual_norm(self) -> float:
        v = ctypes.c_double(0.0)
        self._check(load_library().pg_residual_norm(self.h, ctypes.byref(v)))
        return v.value

    def set_timing(self, on: bool = True):
        self._check(load_library().pg_set_timing(self.h, int(on)))

    def kernel_times(self) -> np.ndarray:
        """Device milliseconds of the last assembly: [cohesive points + cut blocks, fast rows
        (concurrent), general rows, whole assembly]."""
        ms = np.zeros(4, np.float32)
        self._check(load_library().pg_kernel_times(self.h, _ptr(ms)))
        return ms

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            load_library().pg_destroy(self.h)
            self.h = ctypes.c_void_p(0)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Several uploaded contexts assembled together by persistent launches replayed from a CUDA
    graph (pg_batch_*).  The Problems must outlive the Batch."""

    def __init__(self, problems):
        L = load_library()
        self.problems = list(problems)
        hs = (ctypes.c_void_p * len(self.problems))(*[p.h.value for p in self.problems])
        self._hs = hs
        h = ctypes.c_void_p(0)
        rc = L.pg_batch_create(ctypes.cast(hs, ctypes.c_void_p), len(self.problems), ctypes.byref(h))
        self.h = h
        if rc:
            msg = L.pg_batch_last_error(h).decode() if h.value else "invalid batch"
            self.close()
            raise PigfemError(rc, msg)
        self._u = None

    def _check(self, rc):
        if rc:
            raise PigfemError(rc, load_library().pg_batch_last_error(self.h).decode())

    def _uptrs(self, d_U):
        arr = (ctypes.c_void_p * len(self.problems))(*[int(u) for u in d_U])
        self._u = arr      # kept alive until the next call
        return ctypes.cast(arr, ctypes.c_void_p)

    def assemble(self, d_U, flags: int = FUNC | JAC, t_frac=None):
        tf = None
        if t_frac is not None:
            tf = np.ascontiguousarray(t_frac, dtype=np.float64)
            self._tf = tf
        self._check(load_library().pg_batch_assemble(self.h, self._uptrs(d_U), _ptr(tf), int(flags)))

    def wait(self) -> float:
        ms = ctypes.c_float(0.0)
        self._check(load_library().pg_batch_wait(self.h, ctypes.byref(ms)))
        return ms.value

    def tune(self, d_U, flags: int = FUNC | JAC, reps: int = 3):
        best = np.zeros(3, np.int32)
        self._check(load_library().pg_batch_tune(self.h, self._uptrs(d_U), int(flags), int(reps), _ptr(best)))
        return tuple(int(x) for x in best)

    def info(self) -> dict:
        v = np.zeros(8, np.int64)
        self._check(load_library().pg_batch_info(self.h, _ptr(v)))
        keys = ("contexts", "elements", "stencil_tile_threads", "general_threads_per_block", "blocks_per_sm",
                "coh_chunks", "stencil_chunks", "general_chunks")
        return {k: int(x) for k, x in zip(keys, v)}

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            load_library().pg_batch_destroy(self.h)
            self.h = ctypes.c_void_p(0)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
