"""Precision "auto" (ZQD_PRECISION_AUTO): a job takes the FP32 form unless the smallest gap
between its adiabatic surfaces on the grid is below ZQD_AUTO_GAP_THRESHOLD (1e-3 Hartree), and
then runs exactly as the explicitly chosen form would (bit for bit), alone, in a batch and
through the job server."""
import numpy as np
import pytest

from zinq_b200 import quantum_dynamics as qd

pytestmark = pytest.mark.gpu


def crossing(coupling, npoint=1024, iters=300):
    # two-state tanh crossing: the surfaces meet at r = 0, where the gap is 2 |coupling|
    c = f"{coupling:.17g}*exp(-r1^2)"
    return {"grid": {"bounds": [[-24, 24]], "npoint": npoint},
            "initial_conditions": {"position": [-10.0], "momentum": [20.0], "gamma": [1.0], "state": 0,
                                   "adiabatic": True},
            "potential": {"custom": {"ndim": 1, "matrix": [["0.01*tanh(1.6*r1)", c], [c, "-0.01*tanh(1.6*r1)"]]}},
            "mass": [2000.0], "iterations": iters, "time_step": 1.0, "adiabatic": True,
            "write": {"population": "P", "norm": "N"}}


def harmonic_1state():
    return {"grid": {"bounds": [[-16, 16]], "npoint": 1024},
            "initial_conditions": {"position": [1.0], "momentum": [0.0], "gamma": [1.0], "state": 0,
                                   "adiabatic": False},
            "potential": {"harmonic": {"k": [1.0]}}, "mass": [1.0], "iterations": 100, "time_step": 0.1,
            "adiabatic": False, "write": {"norm": "N", "position": "X"}}


def _same(a, b):
    ga, gb = a.observables[0], b.observables[0]
    for name in ga.history:
        np.testing.assert_array_equal(ga.history[name], gb.history[name])
    np.testing.assert_array_equal(ga.pop, gb.pop)


@pytest.mark.parametrize("coupling, expected", [(0.005, "fp32"), (2e-4, "fp64"), (-4.9e-4, "fp64"), (6e-4, "fp32")])
def test_auto_picks_the_form_by_the_smallest_gap(coupling, expected):
    opt = crossing(coupling)
    r = qd.run(opt, precision="auto", want_wavefunction=False)
    assert r.precision == expected
    _same(r, qd.run(opt, precision=expected, want_wavefunction=False))


def test_one_state_takes_fp32():
    r = qd.run(harmonic_1state(), precision="auto", want_wavefunction=False)
    assert r.precision == "fp32"


def test_auto_in_a_batch_and_through_the_server():
    opts = [crossing(c, iters=200) for c in (0.005, 2e-4, 0.003, 1e-4)]
    expected = ["fp32", "fp64", "fp32", "fp64"]
    alone = [qd.run(o, precision=e, want_wavefunction=False) for o, e in zip(opts, expected)]
    for r, a, e in zip(qd.run_batch(opts, "auto"), alone, expected):
        assert r.precision == e
        _same(r, a)
    from test_gpu_server import alone_as_served

    for persistent in (False, True):  # grouped launches, then the persistent line-service kernel
        srv = qd.Server(workers=1, max_batch=8, persistent_lines=persistent)
        tickets = [srv.submit(o, "auto") for o in opts]
        out = [srv.wait(t)[0] for t in tickets]
        srv.close()
        for r, o, e in zip(out, opts, expected):
            assert r.precision == e
            _same(r, alone_as_served(o, e) if persistent else qd.run(o, precision=e, want_wavefunction=False))


def test_auto_on_a_2d_grid():
    opt = {"grid": {"bounds": [[-8, 8], [-8, 8]], "npoint": 64},
           "initial_conditions": {"position": [-2, 0], "momentum": [1, 0], "gamma": [1, 1], "state": 0,
                                  "adiabatic": False},
           "potential": {"custom": {"ndim": 2, "matrix": [["0.5*(r1^2+r2^2)", "0.0001*exp(-(r1^2+r2^2))"],
                                                          ["0.0001*exp(-(r1^2+r2^2))", "0.5*(r1^2+r2^2)+0.2*r1"]]}},
           "mass": [1, 1], "iterations": 40, "time_step": 0.05, "adiabatic": False, "write": {"population": "P"}}
    r = qd.run(opt, precision="auto", want_wavefunction=False)
    assert r.precision == "fp64"  # the diagonals cross on r1 = 0 with a 2e-4 gap
    _same(r, qd.run(opt, precision="fp64", want_wavefunction=False))
