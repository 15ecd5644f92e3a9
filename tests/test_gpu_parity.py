"""GPU parity of the propagator against the oracle and the reference's goldens.

Bars (FP64 plain form): relative L2 of the final wavefunction <= 1e-10 and
every population sample within 1e-12 absolute of the oracle; the reference's
own known answers (test/quantum_dynamics.zig:8-282) within their 1e-8.
FP32 form: every population sample within 1e-5 of the FP64 oracle.
All calls go through the C-ABI (libzinq_qd.so).
"""
import copy
import os

import numpy as np
import pytest

from oracle import qd_ref
from zinq_b200 import quantum_dynamics as qd

pytestmark = pytest.mark.gpu

PSI_TOL = 1e-10
POP_TOL = 1e-12
FP32_POP_TOL = 1e-5

ORACLE_NAMES = {"position": "pos", "momentum": "mom", "population": "pop", "potential_energy": "epot",
                "kinetic_energy": "ekin", "total_energy": "etot", "norm": "norm", "acf": "acf", "wavefunction": "wfn"}


def psi_rel(g, r):
    return float(np.linalg.norm(g - r) / np.linalg.norm(r))


def compare(opt, precision="fp64", pop_tol=POP_TOL, psi_tol=PSI_TOL, obs_tol=1e-10, sign_free=False, nthreads=1,
            ref=None):
    """GPU run of opt against the oracle (or against `ref`, an oracle result already computed)."""
    gpu = qd.run(opt, precision=precision)
    if ref is None:
        ref = qd_ref.run(opt, nthreads=nthreads)
    assert len(gpu.observables) == len(ref)
    worst = {}
    for g, r in zip(gpu.observables, ref):
        for name, series in g.history.items():
            rs = r.history[ORACLE_NAMES[name]]
            assert series.shape[0] == rs.shape[0], name
            tol = pop_tol if name == "population" else obs_tol
            err = float(np.max(np.abs(series - rs)))
            worst[name] = max(worst.get(name, 0.0), err)
            assert err <= tol, (name, err)
        for name in ("pos", "mom", "pop"):
            err = float(np.max(np.abs(getattr(g, name) - getattr(r, name))))
            assert err <= (pop_tol if name == "pop" else obs_tol), (name, err)
        for name in ("epot", "ekin", "norm"):
            assert abs(getattr(g, name) - getattr(r, name)) <= obs_tol, name
        if precision == "fp64":
            gw, rw = g.wavefunction, r.wavefunction
            if sign_free:  # eigenvector sign conventions may differ by a global per-state sign
                for s in range(gw.shape[0]):
                    if np.vdot(gw[s], rw[s]).real < 0:
                        gw[s] = -gw[s]
            rel = psi_rel(gw, rw)
            assert rel <= psi_tol, rel
            worst["psi_rel_l2"] = max(worst.get("psi_rel_l2", 0.0), rel)
    return gpu, ref, worst


def tully(pot, adia, npoint=512, iters=3000):
    return {"grid": {"bounds": [[-24, 32]], "npoint": npoint},
            "initial_conditions": {"momentum": [15], "position": [-10], "state": 0, "gamma": [2], "adiabatic": adia},
            "potential": {pot: {}}, "mass": [2000], "iterations": iters, "time_step": 1, "adiabatic": adia,
            "write": {"population": "P", "position": "X", "momentum": "K", "total_energy": "E", "norm": "N"}}


# ---------------------------------------------------------------- goldens
@pytest.mark.parametrize("case", range(10))
def test_gpu_reproduces_reference_known_answers(known_answers, case):
    t = known_answers["tests"][case]
    res = qd.run(t["options"], want_wavefunction=False)
    for e in t["expect"]:
        v = getattr(res.observables[e["solve"]], e["field"])
        got = float(v[e["index"]]) if e["index"] is not None else float(v)
        assert abs(got - e["value"]) <= known_answers["tolerance"], (t["name"], e, got)


@pytest.mark.parametrize("case", range(10))
def test_gpu_matches_oracle_on_golden_inputs(known_answers, case):
    opt = copy.deepcopy(known_answers["tests"][case]["options"])
    opt["write"] = {"population": "P", "position": "X", "total_energy": "E", "norm": "N"}
    compare(opt)


# ---------------------------------------------------------------- 1-D paths
@pytest.mark.parametrize("pot", ["tully_1", "tully_2", "tully_3"])
def test_adiabatic_initial_state_signs_match_lapack(pot):
    # wavefunction compared without any sign freedom: eigenvector signs follow dsyevd
    compare(tully(pot, True, iters=300))


@pytest.mark.parametrize("cluster", ["1", "2", "4", "8", "16"])
def test_cluster_sizes_agree_with_oracle(cluster, monkeypatch):
    monkeypatch.setenv("ZQD_LINE_CLUSTER", cluster)
    opt = tully("tully_1", True, npoint=1024, iters=400)
    compare(opt)


@pytest.mark.parametrize("cluster", ["1", "2", "4", "8", "16"])
def test_cluster_sizes_agree_with_oracle_fp32(cluster, monkeypatch):
    # FP32 CTAs of at most 256 threads run the kernel form compiled for 256 threads (clusters of 2 to
    # 16 here); one-CTA lines of 1024 points keep the 512-thread form
    monkeypatch.setenv("ZQD_LINE_CLUSTER", cluster)
    opt = tully("tully_1", True, npoint=1024, iters=400)
    compare(opt, precision="fp32", pop_tol=FP32_POP_TOL, obs_tol=1e-4)


def test_custom_expression_potential_matches_builtin():
    # example/input/quantum_dynamics_custom_real.json writes Tully 1 as expressions
    expr = {"custom": {"ndim": 1, "matrix": [
        ["+sgn(r1) * 0.01 * (1.0 - exp(-1.6 * abs(r1)))", "0.005 * exp(-r1^2)"],
        ["0.005 * exp(-r1^2)", "-sgn(r1) * 0.01 * (1.0 - exp(-1.6 * abs(r1)))"]]}}
    opt = tully("tully_1", True, npoint=1024, iters=500)
    opt["potential"] = expr
    g, _, _ = compare(opt)
    b = qd.run(tully("tully_1", True, npoint=1024, iters=500))
    assert np.max(np.abs(g.observables[0].history["population"] - b.observables[0].history["population"])) < 1e-12


def test_time_dependent_custom_potential():
    opt = {"grid": {"bounds": [[-16, 16]], "npoint": 256},
           "initial_conditions": {"momentum": [0], "position": [0], "state": 1, "gamma": [2], "adiabatic": True},
           "potential": {"custom": {"ndim": 1, "time_dependent": True,
                                    "matrix": [["(t - 10) * 10", "2"], ["2", "-(t - 10) * 10"]]}},
           "mass": [1], "iterations": 500, "time_step": 0.01, "adiabatic": True,
           "write": {"population": "P", "potential_energy": "V"}}
    compare(opt)


def test_absorbing_potential_tracking_and_stop_norm():
    opt = tully("tully_1", False, npoint=512, iters=3000)
    # the packet (x0 = -10, v = 15/2000) crosses x = 5 near step 2000 and is absorbed beyond it
    opt["absorbing_potential"] = {"bounds": [[-20, 5]], "exponent": 0.05, "track_population": True,
                                  "stop_norm": 0.5}
    g, r, _ = compare(opt)
    rows = g.observables[0].history["population"].shape[0]
    assert rows < 3001  # stopped early, like the oracle


def test_autocorrelation_and_three_states():
    opt = {"grid": {"bounds": [[-12, 12]], "npoint": 2048},
           "initial_conditions": {"momentum": [1], "position": [-2], "state": 0, "gamma": [1]},
           "potential": {"custom": {"ndim": 1, "matrix": [
               ["0.5*r1^2 + 0.3*r1", "0.05*exp(-r1^2/2)", "0.02"],
               ["0.05*exp(-r1^2/2)", "0.5*r1^2 - 0.2*r1 + 0.1", "0.05*exp(-r1^2/2)"],
               ["0.02", "0.05*exp(-r1^2/2)", "0.5*r1^2 + 0.15"]]}},
           "mass": [1], "iterations": 400, "time_step": 0.05,
           "write": {"population": "P", "acf": "A", "total_energy": "E"}}
    compare(opt)


def test_imaginary_time_three_states_orthogonalised():
    opt = {"grid": {"bounds": [[-8, 8]], "npoint": 256},
           "initial_conditions": {"momentum": [0.3], "position": [1], "gamma": [2]},
           "potential": {"harmonic": {}}, "imaginary": {"nstate": 3}, "mass": [1], "iterations": 600,
           "time_step": 0.01, "write": {"total_energy": "E", "norm": "N"}}
    compare(opt)


# ---------------------------------------------------------------- workloads
def config1():
    return {"grid": {"bounds": [[-16, 16]], "npoint": 1024},
            "initial_conditions": {"position": [1], "momentum": [0], "gamma": [1], "state": 0},
            "potential": {"harmonic": {"k": [1]}}, "mass": [1], "iterations": 1000, "time_step": 0.1,
            "write": {"norm": "N", "total_energy": "E", "position": "X"}}


def config2(p0, iters=4000):
    return {"grid": {"bounds": [[-24, 24]], "npoint": 8192},
            "initial_conditions": {"position": [-10], "momentum": [p0], "gamma": [p0 * p0 / 400.0], "state": 0,
                                   "adiabatic": True},
            "potential": {"custom": {"ndim": 1, "matrix": [["0.01*tanh(1.6*r1)", "0.005*exp(-r1^2)"],
                                                           ["0.005*exp(-r1^2)", "-0.01*tanh(1.6*r1)"]]}},
            "mass": [2000], "iterations": iters, "time_step": 1, "adiabatic": True,
            "write": {"population": "P"}}


def test_config1_harmonic_1024():
    compare(config1())


def test_config2_tanh_crossing_fp64():
    compare(config2(20.0, iters=1500))


@pytest.mark.parametrize("p0", [10.0, 30.0])
def test_config2_fp32_populations_within_1e5(p0):
    compare(config2(p0, iters=1500), precision="fp32", pop_tol=FP32_POP_TOL, obs_tol=1e-4)


def test_batched_jobs_equal_single_jobs():
    opts = [config2(p, iters=300) for p in (10.0, 15.0, 20.0, 25.0, 30.0)]
    batch = qd.run_batch(opts)
    for o, b in zip(opts, batch):
        s = qd.run(o, want_wavefunction=False)
        np.testing.assert_array_equal(b.observables[0].history["population"], s.observables[0].history["population"])


def test_runs_are_bitwise_deterministic():
    a = qd.run(config1())
    b = qd.run(config1())
    np.testing.assert_array_equal(a.observables[0].wavefunction, b.observables[0].wavefunction)
    np.testing.assert_array_equal(a.observables[0].history["total_energy"], b.observables[0].history["total_energy"])


# ---------------------------------------------------------------- spectrum (calcSpectrum on the device)
@pytest.mark.parametrize("padding,threshold,iters", [(0, 1e-6, 400), (700, 1e-4, 513), (1, 0.5, 1)])
def test_spectrum_matches_oracle(padding, threshold, iters):
    opt = {"grid": {"bounds": [[-10, 10]], "npoint": 256},
           "initial_conditions": {"position": [1.5], "momentum": [0.3], "gamma": [1.2], "state": 0, "adiabatic": False},
           "potential": {"custom": {"ndim": 1, "matrix": [["0.5*r1^2+0.05*r1^4"]]}}, "mass": [1],
           "iterations": iters, "time_step": 0.05, "adiabatic": False,
           "spectrum": {"padding": padding, "threshold": threshold}, "write": {}}
    g = qd.run(opt, want_wavefunction=False).observables[0].spectrum
    r = qd_ref.run(opt, want_wavefunction=False)[0].spectrum
    assert g is not None and r is not None
    assert g[0].shape == r[0].shape and g[1].shape == r[1].shape
    np.testing.assert_allclose(g[0], r[0], rtol=0, atol=1e-10)
    scale = max(1.0, float(np.max(np.abs(r[1]))))
    assert float(np.max(np.abs(g[1] - r[1]))) <= 1e-9 * scale


@pytest.mark.parametrize("nstate,precision", [(3, "fp64"), (4, "fp64"), (4, "fp32")])
def test_longest_lines_read_the_propagator_table_from_global_memory(nstate, precision):
    # 16384 points x 3-4 states: the R slice no longer fits in shared memory beside the wavefunction
    mat = [[("0.01*tanh(1.6*r1)" if i % 2 == 0 else "-0.01*tanh(1.6*r1)") if i == j else "0.005*exp(-r1^2)"
            for j in range(nstate)] for i in range(nstate)]
    opt = {"grid": {"bounds": [[-30, 30]], "npoint": 16384},
           "initial_conditions": {"position": [-8], "momentum": [15], "gamma": [0.5], "state": 0, "adiabatic": False},
           "potential": {"custom": {"ndim": 1, "matrix": mat}}, "mass": [2000], "iterations": 200, "time_step": 1,
           "adiabatic": False, "write": {"population": "P", "total_energy": "E"}}
    if precision == "fp64":
        compare(opt)
    else:
        compare(opt, precision="fp32", pop_tol=FP32_POP_TOL, obs_tol=1e-4)


# ---------------------------------------------------------------- .mat writers (History.exportWrite)
def _read_mat(path):
    with open(path) as f:
        lines = f.read().splitlines()
    rows, cols = map(int, lines[0].split())
    body = lines[1:]
    assert len(body) == rows
    for line in body:  # every value "%20.14f": width 20, 14 decimals, one space apart
        fields = [line[i:i + 20] for i in range(0, len(line), 21)]
        assert len(fields) == cols and all(len(x) == 20 and x[-15] == "." for x in fields), line
    return np.array([[float(x) for x in line.split()] for line in body])


def test_history_files_match_the_result(tmp_path):
    names = ["acf", "position", "momentum", "population", "potential_energy", "kinetic_energy", "norm", "total_energy"]
    opt = tully("tully_1", False, npoint=256, iters=120)
    opt["write"] = {n: str(tmp_path / f"{n}.mat") for n in names}
    opt["spectrum"] = {"padding": 30, "threshold": 1e-4,
                       "write": {"acf": str(tmp_path / "spec_acf.mat"), "spectrum": str(tmp_path / "spec.mat")}}
    res = qd.run(opt, export=True).observables[0]
    dt, rows = opt["time_step"], 121
    for n in names:
        m = _read_mat(tmp_path / f"{n}.mat")
        np.testing.assert_allclose(m[:, 0], np.arange(rows) * dt, rtol=0, atol=1e-13)
        h = res.history[n]
        h = np.stack([h.real, h.imag], 1) if n == "acf" else h.reshape(rows, -1)
        np.testing.assert_allclose(m[:, 1:], h, rtol=0, atol=6e-15)
    acfp, sigma = res.spectrum
    m = _read_mat(tmp_path / "spec_acf.mat")
    assert m.shape == (len(acfp), 3)
    np.testing.assert_allclose(m[-1, 0], (rows - 1 + 30) * dt, rtol=1e-14)
    np.testing.assert_allclose(m[:, 1:], np.stack([acfp.real, acfp.imag], 1), rtol=0, atol=6e-15)
    m = _read_mat(tmp_path / "spec.mat")
    nt = len(sigma)
    np.testing.assert_allclose(m[[0, -1], 0], [-np.pi / dt, np.pi / dt * (nt - 2) / nt], rtol=1e-14)
    np.testing.assert_allclose(m[:, 1], sigma, rtol=0, atol=6e-15 * max(1.0, np.max(np.abs(sigma))))


# ---------------------------------------------------------------- wavefunction history (write.wavefunction)
@pytest.mark.parametrize("adia", [False, True])
def test_wavefunction_history_matches_oracle(adia, tmp_path):
    opt = tully("tully_2", adia, npoint=256, iters=60)
    opt["write"] = {"wavefunction": str(tmp_path / "wfn.mat"), "population": "P"}
    gpu, ref, _ = compare(opt)
    w = gpu.observables[0].history["wavefunction"]
    assert w.shape == (61, 2, 256)
    qd.run(opt, export=True)
    lines = open(tmp_path / "wfn.mat").read().splitlines()
    assert lines[0] == f"256 {1 + 2 * 2 * 61}"
    row = np.array([float(x) for x in lines[5].split()])
    np.testing.assert_allclose(row[0], -24 + 4 * 56 / 256, atol=1e-13)
    np.testing.assert_allclose(row[1::2] + 1j * row[2::2], w[:, :, 4].ravel(), atol=6e-15 * 1.5)


def test_radix8_kernel_for_lines_above_the_radix4_thread_limit():
    # 32768 points: CTAs of 2048 points, whose radix-4 passes would need more threads than allowed
    opt = {"grid": {"bounds": [[-40, 40]], "npoint": 32768},
           "initial_conditions": {"position": [-8], "momentum": [10], "gamma": [0.5], "state": 0, "adiabatic": False},
           "potential": {"harmonic": {"k": [0.01]}}, "mass": [2000], "iterations": 100, "time_step": 1,
           "adiabatic": False, "write": {"position": "X", "momentum": "K", "total_energy": "E"}}
    compare(opt)


# ---------------------------------------------------------------- eigenvector signs of time-dependent potentials
def td_crossing_1d(iters=500):
    # the diagonal difference changes sign at t = 2.5: LAPACK's eigenvector signs flip there, the
    # global alignment with the previous update (wavepacket.zig:157-167) flips them back
    return {"grid": {"bounds": [[-8, 8]], "npoint": 256},
            "initial_conditions": {"momentum": [0.5], "position": [-1], "state": 0, "gamma": [1], "adiabatic": True},
            # the diagonal difference 0.8 (t - 2.5) + 0.1 r1 also changes sign along the grid (continuity rule);
            # the constant coupling keeps the adiabatic gap >= 0.6
            "potential": {"custom": {"ndim": 1, "time_dependent": True,
                                     "matrix": [["0.5*r1^2 + (t - 2.5)*0.4 + 0.05*r1", "0.3"],
                                                ["0.3", "0.5*r1^2 - (t - 2.5)*0.4 - 0.05*r1"]]}},
            "mass": [1], "iterations": iters, "time_step": 0.01, "adiabatic": True,
            "write": {"population": "P", "wavefunction": "W"}}


@pytest.mark.parametrize("cluster", ["1", "4"])
def test_time_dependent_adiabatic_wavefunction_history_signs(cluster, monkeypatch):
    # compared without sign freedom: continuity along the grid and alignment across updates
    monkeypatch.setenv("ZQD_LINE_CLUSTER", cluster)
    gpu, _, worst = compare(td_crossing_1d())
    assert gpu.observables[0].history["wavefunction"].shape == (501, 2, 256)


def test_time_dependent_imaginary_time_later_solve_uses_aligned_eigenvectors():
    # the second solve's toDia uses the eigenvectors left by the first solve's last update
    opt = td_crossing_1d(iters=300)
    opt["imaginary"] = {"nstate": 2}
    opt["write"] = {"total_energy": "E", "norm": "N"}
    compare(opt)


def test_time_dependent_job_run_twice_starts_from_t0_tables():
    opt = td_crossing_1d(iters=200)
    job = qd.Job(opt)
    job.run()
    job.run()
    g = job.result().observables[0]
    job.close()
    r = qd_ref.run(opt)[0]
    assert float(np.max(np.abs(g.history["wavefunction"] - r.history["wfn"]))) <= 1e-10
