"""GPU parity at the benchmark workloads' own sizes (not scaled down).

* 1-D two-state tanh crossing, 8192 points on [-24, 24], mass 2000, dt 1, all five momenta
  p0 in {10, 15, 20, 25, 30}, the full 4000 steps: FP64 against the oracle at the plain
  form's bars (relative L2 of the final wavefunction <= 1e-10, every population sample
  within 1e-12), and the FP32 form's every population sample within 1e-5 of the FP64 oracle.
* 2-D three-state coupled harmonic surfaces on 512^2 for 200 of its 2000 steps.
* 3-D anharmonic well on 128^3: imaginary-time relaxation and real time with the
  autocorrelation, 20 steps each.
* 2-D two-state grid of 2048^2 (larger than L2) for 5 steps.

The oracle runs with every host thread where the grid is large; jobs run in parallel threads
(the oracle releases the GIL inside its C library).
"""
import concurrent.futures as cf
import os

import numpy as np
import pytest

from oracle import qd_ref
from test_gpu_nd import anharmonic_3d, coupled_harmonic_2d
from test_gpu_parity import FP32_POP_TOL, compare, config2

pytestmark = pytest.mark.gpu

MOMENTA = (10.0, 15.0, 20.0, 25.0, 30.0)
NPROC = os.cpu_count() or 1


@pytest.fixture(scope="module")
def config2_oracle():
    """Oracle results of the five 4000-step jobs, computed once in parallel."""
    with cf.ThreadPoolExecutor(max_workers=min(len(MOMENTA), NPROC)) as ex:
        res = list(ex.map(lambda p: qd_ref.run(config2(p)), MOMENTA))
    return dict(zip(MOMENTA, res))


@pytest.mark.parametrize("p0", MOMENTA)
def test_config2_full_4000_steps_fp64(config2_oracle, p0):
    _, _, worst = compare(config2(p0), ref=config2_oracle[p0])
    assert worst["population"] <= 1e-12 and worst["psi_rel_l2"] <= 1e-10


@pytest.mark.parametrize("p0", MOMENTA)
def test_config2_full_4000_steps_fp32_populations(config2_oracle, p0):
    _, _, worst = compare(config2(p0), precision="fp32", pop_tol=FP32_POP_TOL, obs_tol=1e-4, ref=config2_oracle[p0])
    assert worst["population"] <= FP32_POP_TOL


def test_config3_512sq_three_states_200_steps():
    compare(coupled_harmonic_2d(npoint=512, iters=200), nthreads=NPROC)


def test_config4_128cube_imaginary_time():
    opt = anharmonic_3d(npoint=128, iters=20, write={"total_energy": "E", "norm": "N"}, imaginary=1)
    compare(opt, nthreads=NPROC)


def test_config4_128cube_real_time_autocorrelation():
    opt = anharmonic_3d(npoint=128, iters=20, write={"acf": "A", "position": "X", "total_energy": "E"})
    compare(opt, nthreads=NPROC)


def test_2048sq_two_states_larger_than_l2():
    mat = [["0.5*(r1^2+r2^2)", "0.01*exp(-r1^2)"], ["0.01*exp(-r1^2)", "0.5*(r1^2+r2^2)+0.1"]]
    opt = {"grid": {"bounds": [[-20, 20], [-20, 20]], "npoint": 2048},
           "initial_conditions": {"position": [-2, 0], "momentum": [1, 0], "gamma": [1, 1], "state": 0,
                                  "adiabatic": False},
           "potential": {"custom": {"ndim": 2, "matrix": mat}}, "mass": [1, 1], "iterations": 5,
           "time_step": 0.05, "adiabatic": False, "write": {"population": "P", "norm": "N"}}
    _, _, worst = compare(opt, nthreads=NPROC)
    assert np.isfinite(worst["psi_rel_l2"])
