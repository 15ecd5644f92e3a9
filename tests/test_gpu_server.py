"""The job server (zqd_server_*): a stream of independent requests with HBM admission, grouped
launches of compatible 1-D jobs and the persistent line-service kernel returns, per request, exactly
what the same job run alone with the same launch shape returns (bit for bit)."""
import os

import numpy as np
import pytest

from zinq_b200 import _abi
from zinq_b200 import quantum_dynamics as qd

pytestmark = pytest.mark.gpu


def served_by_service(opt, precision):
    """The server sends 1-D single-solve requests whose line fits one CTA to the persistent kernel."""
    return (len(opt["grid"]["bounds"]) == 1 and (opt.get("imaginary") or {}).get("nstate", 1) <= 1
            and opt["grid"]["npoint"] <= (1024 if precision == "fp64" else 2048))


def alone_as_served(opt, precision, want_wavefunction=False):
    """The job run alone (zqd_run) with the launch shape the server gives it: one CTA per line on the
    persistent kernel, the built-in rules otherwise."""
    if not served_by_service(opt, precision):
        return qd.run(opt, precision=precision, want_wavefunction=want_wavefunction)
    old = os.environ.get("ZQD_LINE_CLUSTER")
    os.environ["ZQD_LINE_CLUSTER"] = "1"
    try:
        return qd.run(opt, precision=precision, want_wavefunction=want_wavefunction)
    finally:
        if old is None:
            del os.environ["ZQD_LINE_CLUSTER"]
        else:
            os.environ["ZQD_LINE_CLUSTER"] = old


def _same(a, b):
    ga, gb = a.observables[0], b.observables[0]
    for name in ga.history:
        np.testing.assert_array_equal(ga.history[name], gb.history[name])
    np.testing.assert_array_equal(ga.pop, gb.pop)
    assert ga.norm == gb.norm and ga.epot == gb.epot and ga.ekin == gb.ekin


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_scaled_stream_equals_jobs_run_alone(precision):
    # the serving workload's generator, 48 requests of at most 200 steps, arrivals compressed
    opts, arrivals = qd.serving_stream(48, seed=7, rate_per_s=2000.0, max_steps=200)
    res, lat, wall, st = qd.serve_stream(opts, arrivals, precision, workers=4, max_batch=8)
    assert st["completed"] == len(opts) and st["failed"] == 0
    assert all(x > 0 for x in lat)
    assert st["service_jobs"] >= 1
    for o, r in zip(opts, res):
        _same(r, alone_as_served(o, precision))


def test_compatible_1d_requests_share_launches():
    base = {"grid": {"bounds": [[-24, 24]], "npoint": 2048},
            "initial_conditions": {"position": [-10.0], "momentum": [0.0], "gamma": [1.0], "state": 0, "adiabatic": True},
            "potential": {"custom": {"ndim": 1, "matrix": [["0.01*tanh(1.6*r1)", "0.005*exp(-r1^2)"],
                                                           ["0.005*exp(-r1^2)", "-0.01*tanh(1.6*r1)"]]}},
            "mass": [2000.0], "iterations": 400, "time_step": 1.0, "adiabatic": True, "write": {"population": "P"}}
    opts = []
    for p0 in np.linspace(10, 30, 12):
        o = {**base, "initial_conditions": {**base["initial_conditions"], "momentum": [float(p0)],
                                            "gamma": [float(p0 * p0 / 400.0)]}}
        opts.append(o)
    srv = qd.Server(workers=1, max_batch=16, persistent_lines=False)
    # one worker: while it runs the first request the others queue up and are taken together
    tickets = [srv.submit(o, "fp32") for o in opts]
    out = [srv.wait(t)[0] for t in tickets]
    st = srv.stats()
    srv.close()
    assert st["grouped_jobs"] >= 2, st
    for o, r in zip(opts, out):
        _same(r, qd.run(o, precision="fp32", want_wavefunction=False))


def test_admission_keeps_device_memory_within_budget():
    opt = {"grid": {"bounds": [[-12, 12], [-12, 12]], "npoint": 256},
           "initial_conditions": {"position": [-2, 0], "momentum": [1, 0], "gamma": [1, 1], "state": 0, "adiabatic": False},
           "potential": {"harmonic": {"k": [1, 1]}}, "mass": [1, 1], "iterations": 50, "time_step": 0.05,
           "adiabatic": False, "write": {"norm": "N"}}
    budget = 40 * 2 ** 20  # about two of these requests at a time
    srv = qd.Server(workers=4, device_budget_bytes=budget)
    tickets = [srv.submit(opt, "fp64") for _ in range(10)]
    for t in tickets:
        r, lat = srv.wait(t)
        assert abs(r.observables[0].norm - 1.0) < 1e-12
    st = srv.stats()
    srv.close()
    assert st["completed"] == 10 and 0 < st["peak_device_bytes"] <= budget


def test_submit_rejects_invalid_and_oversized_requests():
    srv = qd.Server(workers=1, device_budget_bytes=8 * 2 ** 20)
    bad = {"grid": {"bounds": [[-1, 1]], "npoint": 64},
           "initial_conditions": {"position": [0], "momentum": [0], "gamma": [1], "state": 0},
           "potential": {"harmonic": {}}, "mass": [1], "iterations": 10, "time_step": -1.0}
    with pytest.raises(_abi.ZqdError, match="TIME STEP MUST BE GREATER THAN 0"):
        srv.submit(bad, "fp64")
    big = {**bad, "time_step": 0.1, "grid": {"bounds": [[-1, 1], [-1, 1]], "npoint": 1024}, "mass": [1, 1],
           "initial_conditions": {"position": [0, 0], "momentum": [0, 0], "gamma": [1, 1], "state": 0},
           "potential": {"harmonic": {"k": [1, 1]}}}
    with pytest.raises(_abi.ZqdError, match="BUDGET"):
        srv.submit(big, "fp64")
    srv.close()


def test_stream_jobs_with_vanishing_three_state_couplings_stay_finite():
    # three seeded serving jobs whose equal couplings C exp(-r^2) fall to 1e-196 at the grid edge over
    # degenerate diagonals; a reflector norm that underflowed once made their propagators non-unitary
    opts, _ = qd.serving_stream(600, seed=7, rate_per_s=200.0, max_steps=1000)
    for i in (54, 124, 499):
        o = dict(opts[i], iterations=600 if i != 124 else opts[i]["iterations"])
        a = qd.run(o, precision="fp32", want_wavefunction=False).observables[0].history["population"]
        b = qd.run(o, precision="fp64", want_wavefunction=False).observables[0].history["population"]
        assert np.all(np.isfinite(a)) and np.all(np.isfinite(b))
        assert np.max(np.abs(a - b)) <= 1e-5
