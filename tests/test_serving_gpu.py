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


def test_ensemble_batched_matches_serial_steps(native):
    ens = cases.ensemble_cases(count=5, seed=3, n_min=2e3, n_max=1.5e4)
    b = ensemble.run_batched(ens, steps=6, warmup=1)
    s = ensemble.run_serial(ens, steps=6, warmup=1, precision="tiled")
    assert all(st["steps"] == 7 for st in b["status"])
    assert b["particles"] == s["particles"]
    assert b["particle_steps_per_s"] > 0 and s["particle_steps_per_s"] > 0
