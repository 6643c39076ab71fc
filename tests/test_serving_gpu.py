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


def test_sessions_stay_resident_and_equal_their_steps_alone():
    """Cohesive load-step sessions (3 steps each, Ortiz-Pandolfi interfaces) mixed with one-off
    requests: every step's result is bitwise the same as the session's steps run alone on one
    context, the carried committed internal variables never decrease from step to step (damage
    is irreversible), and later steps need no set-up of their own."""
    from pigfem_b200 import serving
    reqs = serving.poisson_stream(8, rate=50.0, seed=5, scale=0.2, session_steps=3)
    sess = {}
    for q in reqs:
        if q.session >= 0:
            sess.setdefault(q.session, []).append(q)
    assert sess and all(len(v) == 3 for v in sess.values())
    alone = {}
    for v in sess.values():
        for q, a in zip(sorted(v, key=lambda q: q.step), serving.run_session_alone(v)):
            alone[q.rid] = a
    for q in reqs:
        if q.session < 0:
            alone[q.rid] = serving.run_alone(q)
    budget = int(2 * max(a.device_bytes for a in alone.values()))
    eng = serving.ServingEngine(memory_budget=budget, max_inflight=4, setup_workers=4)
    mixed = {r.rid: r for r in eng.run(reqs, realtime=False)}
    for q in reqs:
        m, a = mixed[q.rid], alone[q.rid]
        assert not m.error, m.error
        assert sorted(m.values) == sorted(a.values)
        for k in a.values:
            assert np.array_equal(m.values[k], a.values[k]), (q.rid, q.session, q.step, k)
    for v in sess.values():
        steps = sorted(v, key=lambda q: q.step)
        sums = [mixed[q.rid].values["committed_isv_sum"][0] for q in steps]
        assert all(b >= a for a, b in zip(sums, sums[1:])), sums
        assert sums[-1] > 0
        for q in steps[1:]:
            assert mixed[q.rid].admitted >= mixed[steps[steps.index(q) - 1].rid].done - 1e-3
    # the engine's calibration covers every measured footprint
    for m in mixed.values():
        assert m.measured_bytes > 0
