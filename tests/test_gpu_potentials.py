"""GPU parity of the `file` and `lvc` potentials against the oracle (FP64 bars).

`file` (src/potential.zig:454-490, multilinear lerp :578-615): the table is generated the way
tool/genpot.py:16-78 does it -- an endpoint-excluded grid per axis (numpy.linspace,
meshgrid "ij"), the upper-triangle functions expanded into the full S x S matrix, written with
"%20.14f" under a "rows cols" header -- and read back from the file, on a table grid coarser
than and offset from the propagation grid so that the interpolation is exercised.
`lvc` (src/potential.zig:493-575): linear vibronic coupling in eV and cm^-1 on
dimensionless normal coordinates.
"""
import math

import numpy as np
import pytest

from test_gpu_parity import compare

pytestmark = pytest.mark.gpu


def genpot_table(path, funcs, bounds, npoint):
    """tool/genpot.py: grid columns, then the S x S matrix built from the upper-triangle functions."""
    d = len(bounds)
    axes = [np.linspace(lo, hi, npoint, endpoint=False) for lo, hi in bounds]
    grid = np.column_stack([m.ravel() for m in np.meshgrid(*axes, indexing="ij")])
    cols = [grid[:, i] for i in range(d)]
    vals = [np.broadcast_to(f(*cols), cols[0].shape).astype(float) for f in funcs]
    N = (math.isqrt(1 + 8 * len(funcs)) - 1) // 2
    r, c = np.minimum(*np.ogrid[:N, :N]), np.maximum(*np.ogrid[:N, :N])
    idx = r * N - r * (r + 1) // 2 + c
    data = np.array(vals)[idx].transpose(2, 0, 1).reshape(grid.shape[0], -1)
    np.savetxt(path, np.column_stack((grid, data)), fmt="%20.14f", header=f"{grid.shape[0]} {d + data.shape[1]}",
               comments="")
    return str(path)


def test_file_potential_1d_two_states(tmp_path):
    # Tully-1-like crossing tabulated on 700 points of [-26, 34): coarser than, and offset from, the 1024-point grid
    funcs = [lambda x: np.sign(x) * 0.01 * (1 - np.exp(-1.6 * np.abs(x))), lambda x: 0.005 * np.exp(-x ** 2),
             lambda x: -np.sign(x) * 0.01 * (1 - np.exp(-1.6 * np.abs(x)))]
    path = genpot_table(tmp_path / "POT.mat", funcs, [(-26.0, 34.0)], 700)
    opt = {"grid": {"bounds": [[-24, 32]], "npoint": 1024},
           "initial_conditions": {"position": [-10], "momentum": [15], "gamma": [2], "state": 0, "adiabatic": True},
           "potential": {"file": {"ndim": 1, "path": path}}, "mass": [2000], "iterations": 1500, "time_step": 1,
           "adiabatic": True, "write": {"population": "P", "position": "X", "total_energy": "E", "norm": "N"}}
    gpu, _, _ = compare(opt)
    # the packet crossed the coupling region: population moved to the upper surface
    assert gpu.observables[0].history["population"][-1, 1] > 1e-3


def test_file_potential_2d_two_states(tmp_path):
    funcs = [lambda x, y: 0.5 * (x ** 2 + y ** 2), lambda x, y: 0.02 * np.exp(-(x ** 2 + y ** 2)),
             lambda x, y: 0.5 * (x ** 2 + y ** 2) + 0.05 + 0.1 * x]
    path = genpot_table(tmp_path / "POT2.mat", funcs, [(-9.0, 9.0), (-9.0, 9.0)], 48)
    opt = {"grid": {"bounds": [[-8, 8], [-8, 8]], "npoint": 64},
           "initial_conditions": {"position": [1, -0.5], "momentum": [0, 1], "gamma": [1, 1], "state": 0,
                                  "adiabatic": False},
           "potential": {"file": {"ndim": 2, "path": path}}, "mass": [1, 1], "iterations": 200, "time_step": 0.05,
           "adiabatic": False, "write": {"population": "P", "potential_energy": "V", "momentum": "K", "norm": "N"}}
    compare(opt)


def lvc_1d():
    return {"frequencies": [1000.0], "excitation_energies": [0.0, 0.3], "kappa": [[-0.1], [0.15]],
            "lambda": [[[0.0], [0.08]], [[0.08], [0.0]]]}


def test_lvc_1d_two_states_adiabatic():
    # dimensionless normal coordinate: V = 0.5 w q^2 with w = 1000 cm^-1 (4.556e-3 Hartree); mass 1/w
    opt = {"grid": {"bounds": [[-10, 10]], "npoint": 512},
           "initial_conditions": {"position": [1.5], "momentum": [0], "gamma": [1], "state": 1, "adiabatic": True},
           "potential": {"lvc": lvc_1d()}, "mass": [219.47463], "iterations": 800, "time_step": 5.0,
           "adiabatic": True, "write": {"population": "P", "position": "X", "total_energy": "E"}}
    compare(opt)


def test_lvc_2d_three_states():
    lvc = {"frequencies": [900.0, 1500.0], "excitation_energies": [0.0, 0.2, 0.45],
           "kappa": [[-0.05, 0.02], [0.1, -0.04], [0.0, 0.08]],
           "lambda": [[[0.0, 0.0], [0.04, 0.0], [0.0, 0.03]],
                      [[0.04, 0.0], [0.0, 0.0], [0.05, 0.02]],
                      [[0.0, 0.03], [0.05, 0.02], [0.0, 0.0]]]}
    opt = {"grid": {"bounds": [[-8, 8], [-8, 8]], "npoint": 64},
           "initial_conditions": {"position": [0.5, -0.5], "momentum": [0, 0], "gamma": [1, 1], "state": 2,
                                  "adiabatic": False},
           "potential": {"lvc": lvc}, "mass": [243.86, 146.32], "iterations": 300, "time_step": 4.0,
           "adiabatic": False, "write": {"population": "P", "total_energy": "E", "norm": "N"}}
    compare(opt)
