"""The TMA-staged persistent axis passes (nd_row_tma_kernel, nd_tile_tma_kernel).

They run the same radix schedule, twiddles and butterflies as the per-block kernels they replace;
results differ by rounding only: the compiler may fuse a product into a multiply-add differently in
each kernel, and the observables' partial sums are grouped per CTA over its blocks.  Bars against
the per-block kernels: FP64 wavefunction relative L2 <= 1e-12 and observables within 1e-12; FP32
wavefunction relative L2 <= 1e-5 and observables within 1e-6.  A run repeated with the same kernels
is the same bit for bit.  ZQD_ND_TMA=0 at job creation selects the per-block kernels.  Shapes cover
a partial warp's worth of lines, the momentum copy (total energy recorded every step), several
states, the ACF, CAP tracking with stop_norm and imaginary time; three also against the oracle.
"""
import copy
import os

import numpy as np
import pytest

from oracle import qd_ref
from zinq_b200 import quantum_dynamics as qd

from test_gpu_nd import anharmonic_3d, coupled_harmonic_2d
from test_gpu_parity import FP32_POP_TOL, compare

pytestmark = pytest.mark.gpu


def run_without_tma(opt, precision):
    old = os.environ.get("ZQD_ND_TMA")
    os.environ["ZQD_ND_TMA"] = "0"
    try:
        return qd.run(opt, precision=precision)
    finally:
        if old is None:
            del os.environ["ZQD_ND_TMA"]
        else:
            os.environ["ZQD_ND_TMA"] = old


def cases():
    pop_only = coupled_harmonic_2d(npoint=64, iters=120)
    pop_only["write"] = {"population": "P"}
    energy = coupled_harmonic_2d(npoint=64, iters=60)  # total energy every step: the momentum copy
    two_state = {"grid": {"bounds": [[-10, 10], [-10, 10]], "npoint": 128},
                 "initial_conditions": {"position": [-1, 0], "momentum": [2, 0], "gamma": [1, 1], "state": 0,
                                        "adiabatic": True},
                 "potential": {"custom": {"ndim": 2, "matrix": [["0.5*(r1^2+r2^2)", "0.05*exp(-r1^2)"],
                                                                ["0.05*exp(-r1^2)", "0.5*(r1^2+r2^2)+0.2"]]}},
                 "mass": [1, 1], "iterations": 80, "time_step": 0.05, "adiabatic": True,
                 "absorbing_potential": {"bounds": [[-6, 6], [-6, 6]], "exponent": 2.0, "track_population": True,
                                         "stop_norm": 0.2},
                 "write": {"population": "P", "norm": "N", "position": "X"}}
    acf3 = anharmonic_3d(npoint=32, iters=40, write={"acf": "A", "position": "X", "momentum": "K"})
    itp3 = anharmonic_3d(npoint=32, iters=30, write={}, imaginary=2)
    return {"2d_64sq_3states_pop": pop_only, "2d_64sq_3states_energy": energy, "2d_128sq_2states_cap": two_state,
            "3d_32cube_acf": acf3, "3d_32cube_itp2": itp3}


CASES = cases()


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("name", sorted(CASES))
def test_tma_passes_match_the_per_block_kernels(name, precision):
    opt = CASES[name]
    a = qd.run(opt, precision=precision)
    b = run_without_tma(opt, precision)
    assert len(a.observables) == len(b.observables)
    psi_tol, obs_tol = (1e-12, 1e-12) if precision == "fp64" else (1e-5, 1e-6)
    for ga, gb in zip(a.observables, b.observables):
        rel = float(np.linalg.norm(ga.wavefunction - gb.wavefunction) / np.linalg.norm(gb.wavefunction))
        assert rel <= psi_tol, rel
        for k in ga.history:
            assert ga.history[k].shape == gb.history[k].shape, k
            err = float(np.max(np.abs(ga.history[k] - gb.history[k])))
            assert err <= obs_tol, (k, err)


@pytest.mark.parametrize("name", ["2d_64sq_3states_pop", "2d_64sq_3states_energy", "3d_32cube_acf"])
def test_tma_passes_against_the_oracle(name):
    compare(CASES[name])


def test_tma_fp32_populations_within_1e5_of_the_oracle():
    opt = CASES["2d_64sq_3states_energy"]
    gpu = qd.run(opt, precision="fp32")
    ref = qd_ref.run(opt)
    assert float(np.max(np.abs(gpu.observables[0].history["population"] - ref[0].history["pop"]))) <= FP32_POP_TOL


def test_tma_runs_are_bitwise_reproducible():
    opt = copy.deepcopy(CASES["2d_64sq_3states_pop"])
    first = qd.run(opt)
    for _ in range(4):
        again = qd.run(opt)
        np.testing.assert_array_equal(first.observables[0].wavefunction, again.observables[0].wavefunction)
        np.testing.assert_array_equal(first.observables[0].history["population"], again.observables[0].history["population"])


def test_a_tma_wait_that_runs_out_fails_the_run_and_leaves_the_device_usable():
    # every CTA of the next TMA-staged launch withholds its first tile load, so its mbarrier wait
    # runs out of a 100 us budget (nothing completes that phase; no load is left in flight)
    from zinq_b200 import _abi

    opt = copy.deepcopy(CASES["2d_64sq_3states_pop"])
    opt["iterations"] = 5
    _abi.check(_abi.load().zqd_testing_tma_withhold_load(1, 100.0))
    with pytest.raises(_abi.ZqdError) as err:
        qd.run(opt)
    assert err.value.status == -8 and "TMA" in str(err.value)
    # the armed launch is used up: the next run is whole and matches the oracle
    compare(CASES["2d_64sq_3states_pop"])


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_the_workloads_take_the_tma_staged_passes(precision):
    # the 2-D 512^2 three-state grid (total energy; populations only), the 3-D 128^3 well and the 2-D
    # 2048^2 two-state grid: both passes run in their TMA-staged persistent forms, in whole warps
    pop_only = coupled_harmonic_2d(npoint=512, iters=10)
    pop_only["write"] = {"population": "P"}
    wide = {"grid": {"bounds": [[-20, 20], [-20, 20]], "npoint": 2048},
            "initial_conditions": {"position": [-2, 0], "momentum": [1, 0], "gamma": [1, 1], "state": 0,
                                   "adiabatic": False},
            "potential": {"custom": {"ndim": 2, "matrix": [["0.5*(r1^2+r2^2)", "0.01*exp(-r1^2)"],
                                                           ["0.01*exp(-r1^2)", "0.5*(r1^2+r2^2)+0.1"]]}},
            "mass": [1, 1], "iterations": 10, "time_step": 0.05, "write": {"population": "P"}}
    for opt in (coupled_harmonic_2d(npoint=512, iters=10), pop_only, anharmonic_3d(npoint=128, iters=10), wide):
        job = qd.Job(opt, precision)
        try:
            sh = job.nd_shape()
        finally:
            job.close()
        assert sh["tma_row_block"] > 0 and sh["tma_tile_lines"] > 0, sh
        assert sh["tma_row_threads"] % 32 == 0 and sh["tma_tile_threads"] % 32 == 0, sh
        assert sh["tma_row_ctas"] > 0 and sh["tma_tile_ctas"] > 0, sh
