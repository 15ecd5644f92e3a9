"""Oracle-only checks of the `file` potential table generator (no GPU).

The table is built the way tool/genpot.py:16-78 does it (see tests/test_gpu_potentials.py);
on its own grid the interpolated potential (lerp, src/potential.zig:578-615) must reproduce the
tabulated function, so a propagation on it matches the closed-form potential.
"""
from oracle import qd_ref
from test_gpu_potentials import genpot_table


def test_file_table_reproduces_the_expression_potential_in_the_oracle(tmp_path):
    # sanity of the table generator: on its own grid the interpolated potential is the tabulated one
    f = [lambda x: 0.5 * x ** 2]
    path = genpot_table(tmp_path / "H.mat", f, [(-8.0, 8.0)], 256)
    base = {"grid": {"bounds": [[-8, 8]], "npoint": 256},
            "initial_conditions": {"position": [1], "momentum": [0], "gamma": [1], "state": 0},
            "mass": [1], "iterations": 200, "time_step": 0.05, "write": {"total_energy": "E"}}
    a = qd_ref.run(dict(base, potential={"file": {"ndim": 1, "path": path}}), want_wavefunction=False)[0]
    b = qd_ref.run(dict(base, potential={"harmonic": {"k": [1]}}), want_wavefunction=False)[0]
    assert abs(a.history["etot"][-1] - b.history["etot"][-1]) < 1e-10
