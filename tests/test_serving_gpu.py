"""Continuous batching: results are the same alone and in the mix, admission
respects the HBM budget, and ensembles step together."""
import numpy as np
import pytest

from weaklycompressiblesph_b200 import _native as N
from weaklycompressiblesph_b200 import cases, ensemble
from weaklycompressiblesph_b200.serving import Server, particle_bytes, run_alone

pytestmark = pytest.mark.gpu


def small_requests(count=4, t_end=4e-3, spacing=0.02):
    reqs = cases.serving_requests(count=count, seed=11, n_min=2e3, n_max=1.2e4, t_end=t_end)
    return [(k * spacing, c) for k, (_, c) in enumerate(reqs)]


def test_same_result_alone_and_in_mix(native):
    """Each request's final state in the served mix equals its state run alone
    (bit-identical: instances share kernels but no arithmetic)."""
    reqs = small_requests()
    total = sum(c.n for _, c in reqs)
    with Server(budget_bytes=1e12, max_particles=total + 1024, chunk_steps=7) as srv:
        out = srv.run(reqs)
    assert len(out["records"]) == len(reqs)
    for rec in out["records"]:
        case = reqs[rec["request"]][1]
        _, steps, alone = run_alone(case, chunk_steps=7)
        assert rec["steps"] == steps
        for key in ("pos", "vel", "dens", "acc"):
            np.testing.assert_array_equal(rec["result"][key], alone[key])
    assert out["p99_s"] >= out["p50_s"] > 0


def test_admission_respects_budget(native):
    """With room for about two requests, the rest queue until memory frees up."""
    reqs = small_requests(count=5, spacing=0.0)
    sizes = sorted(c.n for _, c in reqs)
    budget = (sizes[-1] + sizes[-2] + 512) * (particle_bytes() + 8.0)
    with Server(budget_bytes=budget, chunk_steps=10) as srv:
        cap = srv.capacity
        out = srv.run(reqs)
    recs = out["records"]
    assert len(recs) == 5
    # at any admission instant the admitted-but-unfinished particles fit the budget
    for r in recs:
        live = sum(q["n"] for q in recs if q["admitted"] <= r["admitted"] < q["finished"])
        assert live <= cap
    assert max(r["admitted"] for r in recs) > min(r["finished"] for r in recs)  # some waited for memory


def rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def test_ensemble_batched_matches_serial(native):
    """Instances stepped together in one solver end in the same states as the
    same instances stepped one at a time: bit-identical when every step
    searches (the sums run in the same order), and within the FP32
    summation-order tolerance with neighbour lists (the solver's build
    schedule, and with it each list's order, depends on the whole mix)."""
    ens = cases.ensemble_cases(count=5, seed=3, n_min=2e3, n_max=1.5e4)
    b = ensemble.run_batched(ens, steps=6, warmup=1, read=True)
    s = ensemble.run_serial(ens, steps=6, warmup=1, precision="tiled", read=True)
    assert all(st["steps"] == 7 for st in b["status"])
    assert b["particles"] == s["particles"]
    for got, ref in zip(b["states"], s["states"]):
        for key in ("pos", "vel", "dens", "acc"):
            np.testing.assert_array_equal(got[key], ref[key])
    bl = ensemble.run_batched(ens, steps=30, warmup=1, read=True, list_interval=10)
    sl = ensemble.run_serial(ens, steps=30, warmup=1, precision="tiled", read=True, list_interval=10)
    assert bl["lists"]["list_steps"] > 0
    for got, ref in zip(bl["states"], sl["states"]):
        assert rel(got["pos"], ref["pos"]) < 1e-6
        assert rel(got["dens"], ref["dens"]) < 1e-6
        assert rel(got["vel"], ref["vel"]) < 1e-4


def test_same_result_alone_and_in_mix_lists(native):
    """Continuous batching with neighbour lists: each request's final state in
    the served mix matches the request run alone (also with lists) within the
    FP32 tolerance of a different summation order."""
    reqs = small_requests(count=4, t_end=6e-3)
    total = sum(c.n for _, c in reqs)
    with Server(budget_bytes=1e12, max_particles=total + 1024, chunk_steps=7, list_interval=10) as srv:
        out = srv.run(reqs)
        assert srv.solver.list_stats()["list_steps"] > 0
    assert len(out["records"]) == len(reqs)
    for rec in out["records"]:
        case = reqs[rec["request"]][1]
        _, steps, alone = run_alone(case, chunk_steps=7, list_interval=10)
        assert rec["steps"] == steps
        assert rel(rec["result"]["pos"], alone["pos"]) < 1e-6
        assert rel(rec["result"]["dens"], alone["dens"]) < 1e-6
        assert rel(rec["result"]["vel"], alone["vel"]) < 1e-4
