"""The oracle against the reference's own known-answer tests.

tests/golden/known_answers.json is extracted from test/quantum_dynamics.zig:8-282
(ten end-to-end propagations, final observables checked at 1e-8 absolute, :6)
by tests/golden/make_known_answers.py.  Passing here pins the CPU restatement
before any GPU result is compared with it.
"""
import numpy as np
import pytest

from oracle import qd_ref


def _field(obs, name, index):
    v = getattr(obs, name)
    return float(v[index]) if index is not None else float(v)


@pytest.mark.parametrize("case", range(10))
def test_oracle_matches_reference_goldens(known_answers, case):
    t = known_answers["tests"][case]
    res = qd_ref.run(t["options"], nthreads=1, want_wavefunction=False)
    tol = known_answers["tolerance"]
    for e in t["expect"]:
        got = _field(res[e["solve"]], e["field"], e["index"])
        assert abs(got - e["value"]) <= tol, (t["name"], e, got)


def test_oracle_relaxed_state_is_stationary():
    # chaining extension: real time from the imaginary-time ground state keeps |acf| = 1
    import numpy as np
    from oracle import qd_ref

    itp = {"grid": {"bounds": [[-8, 8]], "npoint": 128},
           "initial_conditions": {"position": [1], "momentum": [0], "gamma": [1], "state": 0, "adiabatic": False},
           "potential": {"harmonic": {"k": [1]}}, "mass": [1], "iterations": 400, "time_step": 0.05,
           "imaginary": {"nstate": 1}, "write": {}}
    relaxed = qd_ref.run(itp)[0].wavefunction
    rt = dict(itp)
    rt.pop("imaginary")
    rt["iterations"] = 100
    rt["write"] = {"acf": "A"}
    acf = qd_ref.run(rt, initial_wavefunction=relaxed)[0].history["acf"]
    assert np.max(np.abs(np.abs(acf) - 1.0)) < 1e-6
    # the phase advances at the ground-state energy 0.5 (up to the splitting error of dt = 0.05)
    assert abs(np.angle(acf[1]) + 0.5 * 0.05) < 1e-5
