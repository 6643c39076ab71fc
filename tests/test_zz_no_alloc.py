"""pg_norm2_noalloc: the residual norm whose scratch is a fixed __device__ array.

Called through the C ABI on the internal-force vector P_f of an assembled cohesive problem and
compared with pg_residual_norm (the context-scratch norm) on two calls in a row; the second
call reads the partials the first one left behind and must overwrite them all.  Also: a multi-block vector
against torch's FP64 norm, the empty vector, and the size limit.
"""
import ctypes
import os

import numpy as np
import pytest

from tests.golden.cases import CASES, spec_kwargs

pytestmark = pytest.mark.gpu

MAX_N = 33554432          # PG_NORM_NOALLOC_MAX_N
PG_ERR_CAPACITY = 13
TOL = 1e-13               # relative; the two norms sum in different fixed orders


def _fn():
    from pigfem_b200 import capi
    f = capi.load_library().pg_norm2_noalloc
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p]
    return f


def test_matches_context_norm_twice():
    import torch
    from pigfem_b200 import capi
    f = _fn()
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "coh_bl.npz"))
    P = capi.Problem(capi.ProblemDesc(**spec_kwargs(CASES["coh_bl"])))
    P.set_isv(g["isv_committed"])
    P.assemble(g["U_dof"][g["node_dofs"]], 1.0)
    ref = P.residual_norm()
    assert ref > 0
    _, pf, _ = P.device_outputs()
    out = torch.full((2,), -1.0, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    for k in range(2):
        rc = f(ctypes.c_void_p(pf), P.n_free, ctypes.c_void_p(out.data_ptr() + 8 * k), ctypes.c_void_p(stream))
        assert rc == 0
    torch.cuda.synchronize()
    v = out.cpu().numpy()
    assert abs(v[0] - ref) <= TOL * ref and abs(v[1] - ref) <= TOL * ref, (v, ref)
    assert v[0] == v[1]
    P.close()


def test_multi_block_empty_and_limit():
    import torch
    f = _fn()
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    gen = torch.Generator(device="cuda").manual_seed(7)
    x = torch.randn(5_000_003, dtype=torch.float64, device="cuda", generator=gen)
    out = torch.full((3,), -1.0, dtype=torch.float64, device="cuda")
    for k in range(2):
        assert f(ctypes.c_void_p(x.data_ptr()), x.numel(), ctypes.c_void_p(out.data_ptr() + 8 * k), stream) == 0
    assert f(ctypes.c_void_p(x.data_ptr()), 0, ctypes.c_void_p(out.data_ptr() + 16), stream) == 0
    torch.cuda.synchronize()
    ref = torch.linalg.vector_norm(x).item()
    v = out.cpu().numpy()
    assert abs(v[0] - ref) <= TOL * ref and v[0] == v[1], (v, ref)
    assert v[2] == 0.0
    # beyond the fixed scratch: rejected before any launch (the pointer is never read)
    assert f(ctypes.c_void_p(x.data_ptr()), MAX_N + 1, ctypes.c_void_p(out.data_ptr()), stream) == PG_ERR_CAPACITY
    assert f(ctypes.c_void_p(x.data_ptr()), -1, ctypes.c_void_p(out.data_ptr()), stream) != 0
