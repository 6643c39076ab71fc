"""Serving loop: requests admitted against a device-memory budget and processed concurrently give,
for every request, bitwise the result of the same request run alone; the budget and the slot
limit hold while they run."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _requests(n=14):
    from pigfem_b200 import serving
    return [serving.make_request(i, seed=3, scale=0.2) for i in range(n)]


def test_results_alone_equal_results_in_the_mix():
    from pigfem_b200 import serving
    reqs = _requests()
    kinds = {r.kind for r in reqs}
    assert kinds == {"homogenize", "cohesive_step"}
    alone = {r.rid: serving.run_alone(r) for r in reqs}
    # a budget of about three average requests: admission has to wait for memory to free up
    budget = int(3 * np.mean([a.device_bytes for a in alone.values()]))
    eng = serving.ServingEngine(memory_budget=budget, max_inflight=4, setup_workers=4)
    mixed = eng.run(reqs, realtime=False)
    for m in mixed:
        assert not m.error, m.error
        a = alone[m.rid]
        assert sorted(m.values) == sorted(a.values)
        for k in a.values:
            assert np.array_equal(m.values[k], a.values[k]), (m.rid, k)
    # homogenized moduli are symmetric positive definite (a physics check of the solve)
    for m in mixed:
        if m.kind == "homogenize":
            C = m.values["C"]
            assert np.allclose(C, C.T, rtol=1e-6, atol=1e-6 * np.abs(C).max())
            assert np.all(np.linalg.eigvalsh(0.5 * (C + C.T)) > 0)


def test_admission_respects_budget_and_slots():
    from pigfem_b200 import serving
    reqs = _requests(10)
    eng = serving.ServingEngine(memory_budget=1, max_inflight=2, setup_workers=4)
    res = eng.run(reqs, realtime=False)
    # with a budget below every request, requests run one at a time (the engine admits a request
    # that does not fit only when nothing else is in flight)
    spans = sorted((r.admitted, r.done) for r in res)
    for (a0, d0), (a1, d1) in zip(spans, spans[1:]):
        assert a1 >= d0 - 1e-3
