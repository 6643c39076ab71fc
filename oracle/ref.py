"""ctypes binding to oracle/_ref/libpigfem_ref.so: the reference PIGFEM's own C++ assembly,
compiled from its sources against project-written serial shims (oracle/Makefile).

TEST INFRASTRUCTURE ONLY.  Imported by tests/, by __graft_entry__.smoke() and by bench.py's
CPU-baseline leg, never by the product package.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass, field
from typing import Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "libpigfem_ref.so")
# The same reference build with its Assembler::assemble replaced by the drop-in translation unit
# (pigfem_b200/drop_in/Assembler_b200.cpp) and linked against libpigfem_b200.so.
LIB_B200_PATH = os.path.join(HERE, "_ref", "libpigfem_ref_b200.so")

COH_NONE, COH_BL, COH_BLNU, COH_XN, COH_XNNU, COH_OP, COH_OPNU, COH_OPAUG, COH_OPNUAUG = range(9)
TRI3, QUAD4, TET4 = 0, 1, 2


class _Config(ctypes.Structure):
    _fields_ = [
        ("elem_type", ctypes.c_int), ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
        ("xmin", ctypes.c_double), ("xmax", ctypes.c_double), ("ymin", ctypes.c_double),
        ("ymax", ctypes.c_double), ("zmin", ctypes.c_double), ("zmax", ctypes.c_double),
        ("n_incl", ctypes.c_int), ("incl", ctypes.POINTER(ctypes.c_double)),
        ("E_matrix", ctypes.c_double), ("nu_matrix", ctypes.c_double),
        ("E_fiber", ctypes.c_double), ("nu_fiber", ctypes.c_double),
        ("coh_law", ctypes.c_int), ("coh", ctypes.c_double * 4),
        ("plane_strain", ctypes.c_int), ("subscale", ctypes.c_int),
        ("eps_macro", ctypes.c_double * 6), ("app_strain", ctypes.c_double),
        ("ply_frac", ctypes.c_double), ("ply", ctypes.c_double * 5),
        ("sens_mat", ctypes.c_int), ("sens_param", ctypes.c_int),
    ]


_libs = {}


def available(variant: str = "cpu") -> bool:
    return os.path.exists(LIB_B200_PATH if variant == "b200" else LIB_PATH)


def lib(variant: str = "cpu"):
    """The reference library: "cpu" (its own Assembler::assemble) or "b200" (the drop-in)."""
    if variant not in _libs:
        path = LIB_B200_PATH if variant == "b200" else LIB_PATH
        if not os.path.exists(path):
            raise FileNotFoundError(f"oracle library not built: {path} (run `make -C oracle`)")
        L = ctypes.CDLL(path)
        L.pgref_create.restype = ctypes.c_void_p
        L.pgref_create.argtypes = [ctypes.POINTER(_Config)]
        L.pgref_assemble.restype = ctypes.c_double
        L.pgref_assemble.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_double,
                                     ctypes.c_int, ctypes.c_int]
        L.pgref_time_assemble.restype = ctypes.c_double
        L.pgref_time_assemble.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.pgref_solve.restype = ctypes.c_int
        L.pgref_solve.argtypes = [ctypes.c_void_p]
        L.pgref_set_solver.restype = None
        L.pgref_set_solver.argtypes = [ctypes.c_void_p] + [ctypes.c_double] * 5 + [ctypes.c_int]
        L.pgref_get.restype = ctypes.c_int
        L.pgref_get.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.POINTER(ctypes.c_long),
                                ctypes.POINTER(ctypes.c_void_p)]
        L.pgref_homogenize.restype = None
        L.pgref_homogenize.argtypes = [ctypes.c_void_p]
        L.pgref_write_homogenization.restype = None
        L.pgref_write_homogenization.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_double, ctypes.c_int]
        L.pgref_set_macro.restype = None
        L.pgref_set_macro.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        L.pgref_destroy.restype = None
        L.pgref_destroy.argtypes = [ctypes.c_void_p]
        L.pgref_sensitivity.restype = ctypes.c_int
        L.pgref_sensitivity.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        L.pgref_bind_gpu.restype = ctypes.c_int
        L.pgref_bind_gpu.argtypes = [ctypes.c_void_p]
        L.pgref_gpu_error.restype = ctypes.c_char_p
        L.pgref_gpu_error.argtypes = []
        _libs[variant] = L
    return _libs[variant]


@dataclass
class ProblemSpec:
    """A problem as the reference's Tests/Main.cpp builds it (structured mesh + inclusions)."""
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
    ply_frac: float = 0.0
    ply: Sequence[float] = (0.0,) * 5
    sens_mat: int = 0          # material sensitivity parameter: 0 none, 1 matrix, 2 fiber
    sens_param: int = 0        # 0 E, 1 LAMBDA, 2 MU, 3 K, 4 NU


class RefProblem:
    def __init__(self, spec: ProblemSpec, variant: str = "cpu"):
        self.variant = variant
        L = lib(variant)
        self.spec = spec
        dim = 3 if spec.elem_type == TET4 else 2
        self.dim = dim
        self._incl = np.ascontiguousarray(np.asarray(spec.inclusions, dtype=np.float64).reshape(-1, dim + 1))
        c = _Config()
        c.elem_type = spec.elem_type
        n = list(spec.n) + [0] * (3 - len(spec.n))
        lo = list(spec.lo) + [0.0] * (3 - len(spec.lo))
        hi = list(spec.hi) + [0.0] * (3 - len(spec.hi))
        c.nx, c.ny, c.nz = n[:3]
        c.xmin, c.ymin, c.zmin = lo[:3]
        c.xmax, c.ymax, c.zmax = hi[:3]
        c.n_incl = self._incl.shape[0]
        c.incl = self._incl.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        c.E_matrix, c.nu_matrix, c.E_fiber, c.nu_fiber = spec.E_matrix, spec.nu_matrix, spec.E_fiber, spec.nu_fiber
        c.coh_law = spec.coh_law
        for i, v in enumerate(spec.coh):
            c.coh[i] = v
        c.plane_strain = int(spec.plane_strain)
        c.subscale = int(spec.subscale)
        for i, v in enumerate(spec.eps_macro):
            c.eps_macro[i] = v
        c.app_strain = spec.app_strain
        c.ply_frac = spec.ply_frac
        for i, v in enumerate(spec.ply):
            c.ply[i] = v
        c.sens_mat, c.sens_param = spec.sens_mat, spec.sens_param
        self._cfg = c
        self.h = L.pgref_create(ctypes.byref(c))
        nfc = self.get("n_free_const")
        self.n_free, self.n_const = int(nfc[0]), int(nfc[1])

    def get(self, name: str) -> np.ndarray:
        n = ctypes.c_long(0)
        p = ctypes.c_void_p(0)
        kind = lib(self.variant).pgref_get(self.h, name.encode(), ctypes.byref(n), ctypes.byref(p))
        if kind == 0:
            raise KeyError(name)
        if n.value == 0:
            return np.zeros(0, dtype=np.int32 if kind == 1 else np.float64)
        ct = ctypes.c_int32 if kind == 1 else ctypes.c_double
        arr = np.ctypeslib.as_array(ctypes.cast(p, ctypes.POINTER(ct)), shape=(n.value,))
        return arr.copy()

    def cut_tables(self) -> dict:
        """The enriched mesh's cut elements in the terms of pigfem_b200.rve.interface_state_tables,
        read from the reference's own mesh (export_mesh in ref_driver.cpp): node lists of the cut
        elements (parent nodes then enrichment nodes), their cohesive-element ranges, the cohesive
        local node lists and the cohesive quadrature rotations."""
        dim = self.dim
        eoff, enodes, ecut = self.get("elem_node_off"), self.get("elem_nodes"), self.get("elem_cut")
        ecoh = self.get("elem_coh_off")
        cut = np.nonzero(ecut)[0]
        lens = eoff[cut + 1] - eoff[cut]
        cut_node_off = np.concatenate([[0], np.cumsum(lens)]).astype(np.int64)
        cut_nodes = np.concatenate([enodes[eoff[e]:eoff[e + 1]] for e in cut]) if len(cut) else np.zeros(0, np.int64)
        cut_coh_off = np.concatenate([ecoh[cut], [ecoh[-1]]]) if len(cut) else np.zeros(1, np.int64)
        return dict(dim=dim, n_nodes=len(self.get("node_dofs")) // dim, cut_node_off=cut_node_off, cut_nodes=cut_nodes,
                    cut_coh_off=cut_coh_off, coh_local_off=self.get("coh_struct_off"), coh_local=self.get("coh_struct"),
                    coh_qp_off=self.get("coh_qp_off"), cqp_R=self.get("coh_qp_R"))

    def csr(self, block: str):
        rp, ci, v = self.get(f"{block}_rowptr"), self.get(f"{block}_cols"), self.get(f"{block}_vals")
        shape = tuple(int(s) for s in self.get(f"{block}_shape"))
        return rp, ci, v, shape

    def assemble(self, U: np.ndarray, isv_committed: np.ndarray | None = None, t_frac: float = 1.0,
                 func: bool = True, jac: bool = True) -> float:
        U = np.ascontiguousarray(U, dtype=np.float64)
        assert U.shape == (self.n_free + self.n_const,)
        iv = None
        if isv_committed is not None:
            isv_committed = np.ascontiguousarray(isv_committed, dtype=np.float64)
            iv = isv_committed.ctypes.data
        return lib(self.variant).pgref_assemble(self.h, U.ctypes.data, iv, t_frac, int(func), int(jac))

    def sensitivity(self, U: np.ndarray):
        """The reference's dP_int/dp (free, constrained) of the spec's material parameter at the
        full DOF vector U."""
        U = np.ascontiguousarray(U, dtype=np.float64)
        rc = lib(self.variant).pgref_sensitivity(self.h, U.ctypes.data)
        if rc != 0:
            raise RuntimeError("no material sensitivity parameter in this problem's spec")
        return self.get("dP_f"), self.get("dP_p")

    def homogenize(self) -> np.ndarray:
        lib(self.variant).pgref_homogenize(self.h)
        return self.get("homogenized")

    def write_homogenization(self, filename: str, t: float, step: int):
        """The reference's WriterHomogenization::writeConsecutive on the current state."""
        lib(self.variant).pgref_write_homogenization(self.h, filename.encode(), float(t), int(step))

    def set_macro(self, eps):
        e = np.zeros(6)
        e[:len(eps)] = eps
        lib(self.variant).pgref_set_macro(self.h, e.ctypes.data)

    def time_assemble(self, n_rep: int) -> float:
        return lib(self.variant).pgref_time_assemble(self.h, n_rep)

    def set_solver(self, rel_tol=1e-8, abs_tol=1e-8, max_dt=1e-2, min_dt=1e-5, T_final=1.0, max_iter=25):
        lib(self.variant).pgref_set_solver(self.h, rel_tol, abs_tol, max_dt, min_dt, T_final, max_iter)

    def solve(self) -> str:
        lib(self.variant).pgref_solve(self.h)
        return bytes(self.get("log").astype(np.uint8)).decode(errors="replace")

    def bind_gpu(self) -> int:
        """Attach a B200 context through the drop-in (the "b200" variant only): from then on the
        reference's own Assembler::assemble calls, its solvers' included, run on the device."""
        rc = lib(self.variant).pgref_bind_gpu(self.h)
        if rc != 0:
            raise RuntimeError(f"pgref_bind_gpu: {rc} {lib(self.variant).pgref_gpu_error().decode()}")
        return rc

    def close(self):
        if self.h:
            lib(self.variant).pgref_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
