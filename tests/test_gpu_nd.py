"""GPU parity of the 2-D and 3-D propagator (axis-pass kernels) against the oracle.

Same bars as the 1-D parity tests: FP64 relative L2 of the final wavefunction
<= 1e-10, populations within 1e-12, other observables within 1e-10; the FP32
form's populations within 1e-5 of the FP64 oracle.  Grids are scaled-down
versions of the 2-D three-state coupled-harmonic workload (512^2) and the 3-D
anharmonic-well workload (128^3) so that the oracle finishes in seconds.
"""
import copy

import numpy as np
import pytest

from oracle import qd_ref
from zinq_b200 import quantum_dynamics as qd

from test_gpu_parity import FP32_POP_TOL, compare

pytestmark = pytest.mark.gpu


def coupled_harmonic_2d(npoint=64, iters=200, bound=12.0):
    """Three coupled 2-D harmonic surfaces, constants drawn from a fixed seed."""
    rng = np.random.default_rng(20261203)
    a = rng.uniform(-1, 1, 3)
    b = rng.uniform(-1, 1, 3)
    c = rng.uniform(0, 0.2, 3)
    coup = "0.05*exp(-(r1^2+r2^2)/2)"
    mat = [[(f"0.5*(r1^2+r2^2)+{a[i]:.17g}*r1+{b[i]:.17g}*r2+{c[i]:.17g}" if i == j else coup) for j in range(3)]
           for i in range(3)]
    return {"grid": {"bounds": [[-bound, bound], [-bound, bound]], "npoint": npoint},
            "initial_conditions": {"position": [-2, 0], "momentum": [1, 0], "gamma": [1, 1], "state": 0,
                                   "adiabatic": False},
            "potential": {"custom": {"ndim": 2, "matrix": mat}},
            "mass": [1, 1], "iterations": iters, "time_step": 0.05, "adiabatic": False,
            "write": {"population": "P", "total_energy": "E", "norm": "N"}}


def anharmonic_3d(npoint=32, iters=100, write=None, imaginary=None):
    opt = {"grid": {"bounds": [[-8, 8]] * 3, "npoint": npoint},
           "initial_conditions": {"position": [1, 1, 1], "momentum": [0, 0, 0], "gamma": [1, 1, 1], "state": 0,
                                  "adiabatic": False},
           "potential": {"custom": {"ndim": 3, "matrix": [["0.5*(r1^2+r2^2+r3^2)+0.1*(r1^2*r2-r2^3/3)+0.05*r3^4"]]}},
           "mass": [1, 1, 1], "iterations": iters, "time_step": 0.02, "adiabatic": False,
           "write": write if write is not None else {"acf": "A", "position": "X", "momentum": "K", "total_energy": "E"}}
    if imaginary:
        opt["imaginary"] = {"nstate": imaginary}
    return opt


def test_2d_three_state_coupled_harmonic_fp64():
    compare(coupled_harmonic_2d(npoint=128, iters=300))


@pytest.mark.parametrize("npoint", [256, 512])
def test_2d_single_radix4_and_radix8_middle_pass(npoint):
    # 256 and 512 points per axis: one radix-4 / radix-8 Stockham pass between the
    # register-resident first and last passes (its twiddles from the staged per-pass table);
    # 512^2 x 3 states is the benchmark's 2-D grid
    compare(coupled_harmonic_2d(npoint=npoint, iters=12))


def test_2d_three_state_coupled_harmonic_fp32_populations():
    compare(coupled_harmonic_2d(iters=400), precision="fp32", pop_tol=FP32_POP_TOL, obs_tol=1e-4)


def test_2d_all_observables_every_step():
    opt = coupled_harmonic_2d(npoint=32, iters=120)
    opt["write"] = {"population": "P", "position": "X", "momentum": "K", "potential_energy": "V",
                    "kinetic_energy": "T", "total_energy": "E", "norm": "N", "acf": "A"}
    compare(opt)


def test_2d_logged_steps_only():
    # nothing written: only the logged steps compute observables; the final ones must not change
    opt = coupled_harmonic_2d(npoint=32, iters=90)
    opt["write"] = {}
    opt["log_interval"] = 7
    gpu = qd.run(opt, log=True).observables[0]
    ref = qd_ref.run(opt)[0]
    for name in ("pos", "mom", "pop"):
        assert np.max(np.abs(getattr(gpu, name) - getattr(ref, name))) <= 1e-10, name
    for name in ("epot", "ekin", "norm"):
        assert abs(getattr(gpu, name) - getattr(ref, name)) <= 1e-10, name
    assert np.linalg.norm(gpu.wavefunction - ref.wavefunction) / np.linalg.norm(ref.wavefunction) <= 1e-10


def test_3d_real_time_autocorrelation():
    compare(anharmonic_3d(npoint=64))


def test_3d_small_grid_all_observables():
    compare(anharmonic_3d(npoint=8, iters=60, write={"acf": "A", "position": "X", "momentum": "K", "population": "P",
                                                       "kinetic_energy": "T", "potential_energy": "V", "norm": "N"}))


def test_2d_long_lines_one_row_per_block():
    opt = {"grid": {"bounds": [[-30, 30], [-20, 20]], "npoint": 1024},
           "initial_conditions": {"position": [-3, 1], "momentum": [2, -1], "gamma": [0.5, 1], "state": 0,
                                  "adiabatic": False},
           "potential": {"harmonic": {"k": [0.3, 0.7]}}, "mass": [1, 2], "iterations": 20, "time_step": 0.1,
           "adiabatic": False, "write": {"position": "X", "momentum": "K", "total_energy": "E", "norm": "N"}}
    compare(opt)


ALL_OBS = {"population": "P", "position": "X", "momentum": "K", "potential_energy": "V", "kinetic_energy": "T",
           "total_energy": "E", "norm": "N", "acf": "A"}


def itp_2d(write, nstate=1, npoint=64, iters=80, adiabatic=False):
    opt = coupled_harmonic_2d(npoint=npoint, iters=iters)
    opt["imaginary"] = {"nstate": nstate}
    opt["write"] = write
    opt["adiabatic"] = adiabatic
    return opt


@pytest.mark.parametrize("what", ["every_observable", "populations", "nothing", "adiabatic_populations"])
def test_2d_imaginary_time_deferred_renormalisation(what):
    # one relaxed state: the step's renormalisation is deferred into the next step's first pass and
    # the observables row is scaled by its factor (squared for the quadratic sums); every recorded
    # series and the final state against the oracle, which normalises before it observes
    write = {"every_observable": ALL_OBS, "populations": {"population": "P"}, "nothing": {},
             "adiabatic_populations": {"population": "P", "norm": "N"}}[what]
    compare(itp_2d(write, adiabatic=what == "adiabatic_populations"))


def test_2d_imaginary_time_deferred_renormalisation_fp32():
    opt = itp_2d({"population": "P", "total_energy": "E", "norm": "N"})
    gpu = qd.run(opt, precision="fp32").observables[0]
    ref = qd_ref.run(opt)[0]
    assert float(np.max(np.abs(gpu.history["population"] - ref.history["pop"]))) <= FP32_POP_TOL
    assert float(np.max(np.abs(gpu.history["norm"] - ref.history["norm"]))) <= 1e-6


def test_2d_imaginary_time_with_wavefunction_history(tmp_path):
    # a recorded wavefunction history keeps the renormalisation in the step (the history holds
    # normalised states): the other fused form of the step
    opt = itp_2d({"wavefunction": str(tmp_path / "w.mat"), "population": "P", "norm": "N"}, npoint=32, iters=40)
    gpu, ref, _ = compare(opt)
    w = gpu.observables[0].history["wavefunction"]
    r = ref[0].history["wfn"]
    assert w.shape[0] == 41
    assert float(np.max(np.abs(w.reshape(r.shape) - r))) <= 1e-10


def test_3d_imaginary_time_two_states():
    compare(anharmonic_3d(npoint=16, iters=150, write={"total_energy": "E", "norm": "N"}, imaginary=2))


def test_2d_adiabatic_two_states():
    # eigenvector signs follow LAPACK dsyevd for 2 x 2 at every point (no continuity rule off 1-D)
    opt = {"grid": {"bounds": [[-10, 10], [-6, 6]], "npoint": 64},
           "initial_conditions": {"position": [-3, 0], "momentum": [4, 0.5], "gamma": [1, 2], "state": 1,
                                  "adiabatic": True},
           "potential": {"custom": {"ndim": 2, "matrix": [["0.02*tanh(1.2*r1)+0.01*r2^2", "0.01*exp(-r1^2-r2^2)"],
                                                          ["0.01*exp(-r1^2-r2^2)", "-0.02*tanh(1.2*r1)+0.01*r2^2"]]}},
           "mass": [100, 50], "iterations": 300, "time_step": 0.5, "adiabatic": True,
           "write": {"population": "P", "position": "X", "momentum": "K", "total_energy": "E"}}
    compare(opt)


def test_2d_absorbing_potential_tracking_and_stop_norm():
    opt = {"grid": {"bounds": [[-20, 12], [-8, 8]], "npoint": 64},
           "initial_conditions": {"position": [-4, 0], "momentum": [6, 0], "gamma": [1, 1], "state": 0,
                                  "adiabatic": False},
           "potential": {"custom": {"ndim": 2, "matrix": [["0.1*r2^2+0.01*tanh(r1)", "0.005*exp(-r1^2)"],
                                                          ["0.005*exp(-r1^2)", "0.1*r2^2-0.01*tanh(r1)"]]}},
           "mass": [1, 1], "iterations": 1500, "time_step": 0.05, "adiabatic": False,
           "absorbing_potential": {"bounds": [[-15, 4], [-6, 6]], "exponent": 0.5, "track_population": True,
                                   "stop_norm": 0.4},
           "write": {"population": "P", "norm": "N", "position": "X"}}
    gpu, ref, _ = compare(opt)
    rows = gpu.observables[0].history["population"].shape[0]
    assert rows < 1501  # stopped on the norm


def test_2d_time_dependent_potential():
    opt = {"grid": {"bounds": [[-8, 8], [-8, 8]], "npoint": 32},
           "initial_conditions": {"position": [1, 0], "momentum": [0, 0], "gamma": [1, 1], "state": 0,
                                  "adiabatic": False},
           "potential": {"custom": {"ndim": 2, "time_dependent": True,
                                    "matrix": [["0.5*(r1^2+r2^2)+0.1*r1*sin(0.3*t)", "0.02*cos(0.1*t)"],
                                               ["0.02*cos(0.1*t)", "0.5*(r1^2+r2^2)+0.2"]]}},
           "mass": [1, 1], "iterations": 200, "time_step": 0.05, "adiabatic": False,
           "write": {"population": "P", "total_energy": "E", "position": "X"}}
    compare(opt)


def test_nd_runs_are_bitwise_deterministic():
    opt = coupled_harmonic_2d(npoint=32, iters=50)
    a = qd.run(opt)
    b = qd.run(opt)
    np.testing.assert_array_equal(a.observables[0].wavefunction, b.observables[0].wavefunction)
    np.testing.assert_array_equal(a.observables[0].history["population"], b.observables[0].history["population"])


def test_batch_mixing_line_and_nd_jobs():
    one_d = {"grid": {"bounds": [[-24, 32]], "npoint": 512},
             "initial_conditions": {"momentum": [15], "position": [-10], "state": 0, "gamma": [2], "adiabatic": False},
             "potential": {"tully_1": {}}, "mass": [2000], "iterations": 100, "time_step": 1, "adiabatic": False,
             "write": {"population": "P"}}
    two_d = coupled_harmonic_2d(npoint=32, iters=60)
    batch = qd.run_batch([one_d, two_d, copy.deepcopy(one_d)])
    for o, b in zip([one_d, two_d, one_d], batch):
        s = qd.run(o, want_wavefunction=False)
        np.testing.assert_array_equal(b.observables[0].history["population"], s.observables[0].history["population"])


# ---------------------------------------------------------------- relaxation chained into real time
def _chain(opt_itp, opt_rt, run_gpu):
    """Imaginary-time relaxation, then real time from the relaxed state (GPU chain or oracle chain)."""
    if run_gpu:
        relaxed = qd.run(opt_itp).observables[0].wavefunction
        return relaxed, qd.run(opt_rt, initial_wavefunction=relaxed)
    relaxed = qd_ref.run(opt_itp)[0].wavefunction
    return relaxed, qd_ref.run(opt_rt, initial_wavefunction=relaxed)


@pytest.mark.parametrize("npoint", [16, 32])
def test_3d_relaxation_chained_into_real_time(npoint):
    # the anharmonic-well workload at a reduced grid: ITP, then real time with the autocorrelation
    itp = anharmonic_3d(npoint=npoint, iters=150, write={"total_energy": "E"}, imaginary=1)
    rt = anharmonic_3d(npoint=npoint, iters=120, write={"acf": "A", "total_energy": "E", "norm": "N"})
    g_relaxed, g = _chain(itp, rt, True)
    r_relaxed, r = _chain(itp, rt, False)
    assert np.linalg.norm(g_relaxed - r_relaxed) / np.linalg.norm(r_relaxed) <= 1e-10
    ga, ra = g.observables[0].history["acf"], r[0].history["acf"]
    assert float(np.max(np.abs(ga - ra))) <= 1e-10
    for name, key in (("total_energy", "etot"), ("norm", "norm")):
        assert float(np.max(np.abs(g.observables[0].history[name] - r[0].history[key]))) <= 1e-10


def test_1d_relaxation_chained_into_real_time_fp32():
    # FP32 real-time leg from the FP64-relaxed state: autocorrelation within 1e-5 of the oracle chain
    itp = {"grid": {"bounds": [[-10, 10]], "npoint": 256},
           "initial_conditions": {"position": [1], "momentum": [0], "gamma": [1], "state": 0, "adiabatic": False},
           "potential": {"custom": {"ndim": 1, "matrix": [["0.5*r1^2+0.05*r1^4"]]}}, "mass": [1], "iterations": 300,
           "time_step": 0.02, "adiabatic": False, "imaginary": {"nstate": 1}, "write": {}}
    rt = dict(itp)
    rt.pop("imaginary")
    rt["write"] = {"acf": "A"}
    rt["iterations"] = 500
    relaxed = qd_ref.run(itp)[0].wavefunction
    g = qd.run(rt, precision="fp32", initial_wavefunction=relaxed).observables[0].history["acf"]
    r = qd_ref.run(rt, initial_wavefunction=relaxed)[0].history["acf"]
    assert float(np.max(np.abs(g - r))) <= 1e-5


def test_3d_spectrum_of_real_time_leg():
    opt = anharmonic_3d(npoint=16, iters=300, write={})
    opt["spectrum"] = {"padding": 100, "threshold": 1e-5}
    g = qd.run(opt, want_wavefunction=False).observables[0].spectrum
    r = qd_ref.run(opt, want_wavefunction=False)[0].spectrum
    np.testing.assert_allclose(g[0], r[0], rtol=0, atol=1e-10)
    assert float(np.max(np.abs(g[1] - r[1]))) <= 1e-9 * max(1.0, float(np.max(np.abs(r[1]))))


def test_2d_wavefunction_history_adiabatic():
    opt = {"grid": {"bounds": [[-10, 10], [-6, 6]], "npoint": 32},
           "initial_conditions": {"position": [-3, 0], "momentum": [4, 0.5], "gamma": [1, 2], "state": 1,
                                  "adiabatic": True},
           "potential": {"custom": {"ndim": 2, "matrix": [["0.02*tanh(1.2*r1)+0.01*r2^2", "0.01*exp(-r1^2-r2^2)"],
                                                          ["0.01*exp(-r1^2-r2^2)", "-0.02*tanh(1.2*r1)+0.01*r2^2"]]}},
           "mass": [100, 50], "iterations": 40, "time_step": 0.5, "adiabatic": True,
           "write": {"population": "P", "wavefunction": "W", "kinetic_energy": "T"}}
    compare(opt)


def test_2d_time_dependent_adiabatic_wavefunction_history_signs():
    # eigenvector signs flip at t = 2.5 (the diagonal difference changes sign); the global alignment
    # with the previous update (wavepacket.zig:157-167) keeps the adiabatic history continuous
    opt = {"grid": {"bounds": [[-6, 6], [-6, 6]], "npoint": 32},
           "initial_conditions": {"position": [-1, 0.5], "momentum": [0.5, 0], "gamma": [1, 1], "state": 0,
                                  "adiabatic": True},
           "potential": {"custom": {"ndim": 2, "time_dependent": True,
                                    "matrix": [["0.5*(r1^2+r2^2) + (t - 2.5)*0.4", "0.3"],
                                               ["0.3", "0.5*(r1^2+r2^2) - (t - 2.5)*0.4"]]}},
           "mass": [1, 1], "iterations": 500, "time_step": 0.01, "adiabatic": True,
           "write": {"population": "P", "wavefunction": "W"}}
    compare(opt)
    job = qd.Job(opt)  # graph replay: the second run starts again from the t = 0 tables
    job.run()
    job.run()
    g = job.result().observables[0]
    job.close()
    r = qd_ref.run(opt)[0]
    assert float(np.max(np.abs(g.history["wavefunction"] - r.history["wfn"]))) <= 1e-10


def test_2d_three_states_adiabatic_initial_state():
    # toDia with the three-state eigenvectors at every point (LAPACK dsyevd restated on both sides),
    # compared without sign freedom; constant couplings keep the adiabatic gaps open, so that one-ulp
    # differences between CUDA's and the host's exp do not move the adiabatic populations
    opt = coupled_harmonic_2d(npoint=64, iters=100)
    mat = opt["potential"]["custom"]["matrix"]
    opt["potential"]["custom"]["matrix"] = [[mat[i][j] if i == j else "0.05" for j in range(3)] for i in range(3)]
    opt["initial_conditions"] = dict(opt["initial_conditions"], adiabatic=True, state=1)
    opt["adiabatic"] = True
    opt["write"] = {"population": "P", "wavefunction": "W"}
    compare(opt)
