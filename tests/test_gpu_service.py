"""The persistent line-service kernel (line_service_kernel): resident CTAs claim single-CTA 1-D jobs
from a table in pinned host memory as the server posts them, run each whole solve with the
wavefunction in shared memory, and publish every row.

* Jobs of uneven sizes (256..2048 points, one to three states, FP32 and FP64) submitted together and
  while earlier ones run give, per job, the bits of the same job run alone with the same one-CTA
  shape, and the FP64 ones match the oracle at the plain form's bars.
* Rows stream as events while the kernel runs.
* A service kernel given no work ends by itself: every CTA's wait for a job has a clock64 budget.
"""
import time

import numpy as np
import pytest

from oracle import qd_ref
from zinq_b200 import _abi
from zinq_b200 import quantum_dynamics as qd

from test_gpu_server import alone_as_served, served_by_service

pytestmark = pytest.mark.gpu


def small_line(n, S, p0, iters=300):
    diag = ["0.01*tanh(1.6*r1)", "-0.01*tanh(1.6*r1)", "0.002+0.01*tanh(1.6*r1)"]
    mat = [[diag[i] if i == j else "0.005*exp(-r1^2)" for j in range(S)] for i in range(S)]
    return {"grid": {"bounds": [[-16, 16]], "npoint": n},
            "initial_conditions": {"position": [-6.0], "momentum": [float(p0)], "gamma": [1.0], "state": 0,
                                   "adiabatic": False},
            "potential": {"custom": {"ndim": 1, "matrix": mat}}, "mass": [2000.0], "iterations": iters,
            "time_step": 1.0, "adiabatic": False, "write": {"population": "P", "norm": "N"}}


def mixed_jobs():
    rng = np.random.default_rng(11)
    out = []
    for k in range(24):
        n = int(2 ** rng.integers(8, 12))
        S = int(rng.integers(1, 4))
        out.append((small_line(n, S, float(rng.uniform(5, 20)), iters=int(rng.integers(50, 400))),
                    "fp32" if k % 2 else "fp64"))
    return out


def test_mixed_small_lines_equal_runs_alone_and_the_oracle():
    jobs = mixed_jobs()
    srv = qd.Server(workers=2, persistent_lines=True)
    first = [srv.submit(o, p) for o, p in jobs[:12]]
    time.sleep(0.02)  # the second half is posted while the first runs
    second = [srv.submit(o, p) for o, p in jobs[12:]]
    res = [srv.wait(t, want_wavefunction=True)[0] for t in first + second]
    st = srv.stats()
    srv.close()
    assert st["service_jobs"] == sum(served_by_service(o, p) for o, p in jobs) and st["failed"] == 0, st
    for (o, p), r in zip(jobs, res):
        a = alone_as_served(o, p, want_wavefunction=True)
        np.testing.assert_array_equal(r.observables[0].history["population"], a.observables[0].history["population"])
        np.testing.assert_array_equal(r.observables[0].wavefunction, a.observables[0].wavefunction)
        if p == "fp64":
            ref = qd_ref.run(o)[0]
            assert np.max(np.abs(r.observables[0].history["population"] - ref.history["pop"])) <= 1e-12
            rel = np.linalg.norm(r.observables[0].wavefunction - ref.wavefunction) / np.linalg.norm(ref.wavefunction)
            assert rel <= 1e-10


def test_service_rows_stream_while_the_kernel_runs():
    srv = qd.Server(workers=1, persistent_lines=True, stream_steps=256)
    opt = small_line(1024, 2, 15.0, iters=4000)
    t = srv.submit(opt, "fp32")
    seen, rows, t0 = [], [], time.time()
    while True:
        evs = srv.poll()
        for e in evs:
            seen.append(e["kind"])
            if e["kind"] == "rows":
                rows.append(e["rows"])
        if "done" in seen:
            break
        assert time.time() - t0 < 60
        time.sleep(0.001)
    r, _ = srv.wait(t)
    srv.close()
    assert seen.count("rows") >= 3  # rows arrived in several pieces before completion
    got = np.concatenate(rows)
    np.testing.assert_array_equal(got[:, 3:5], r.observables[0].history["population"])


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_service_kernel_without_work_ends_on_its_own(precision):
    L = _abi.load()
    import ctypes as C

    exits, wall = C.c_uint32(), C.c_double()
    _abi.check(L.zqd_testing_service_idle(_abi.PRECISION[precision], 2, 8, 500.0, C.byref(exits), C.byref(wall)))
    assert exits.value == 8  # every CTA's wait for work ran out of its budget
    assert wall.value < 2000.0
