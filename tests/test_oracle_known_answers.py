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
