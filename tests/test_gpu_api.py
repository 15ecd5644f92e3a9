"""The step-wise method API and the server's streaming, cancellation and failure paths, through the C-ABI.

* zqd_job_step in pieces of any size reproduces zqd_job_run bit for bit (1-D resident kernel resumed
  from its saved wavefunction and carried absorbed populations; N-D launch sequence cut between steps),
  including stop_norm, imaginary-time Gram-Schmidt over several solves and time-dependent potentials;
* zqd_job_observables returns every history row exactly once, in order;
* the server streams rows as events whose concatenation is the final history; requests that arrive
  while a group of the same shape is on the GPU join it (continuous batching) with results equal to
  runs alone; cancellation (queued and running), timed waits, a device allocation refused at
  admission, a consumer that stops polling and a job whose norm turns NaN each affect only their
  own request.  Every failure is made on the host; no GPU fault is involved.
"""
import time

import numpy as np
import pytest

from zinq_b200 import _abi
from zinq_b200 import quantum_dynamics as qd

from test_gpu_server import alone_as_served

pytestmark = pytest.mark.gpu


def _same(a, b):
    for ga, gb in zip(a.observables, b.observables):
        for name in ga.history:
            np.testing.assert_array_equal(ga.history[name], gb.history[name])
        np.testing.assert_array_equal(ga.pop, gb.pop)
        assert ga.norm == gb.norm and ga.epot == gb.epot and ga.ekin == gb.ekin
        if ga.wavefunction is not None and gb.wavefunction is not None:
            np.testing.assert_array_equal(ga.wavefunction, gb.wavefunction)


def tully_cap(iters=3000):
    return {"grid": {"bounds": [[-24, 32]], "npoint": 512},
            "initial_conditions": {"momentum": [15], "position": [-10], "state": 0, "gamma": [2], "adiabatic": False},
            "potential": {"tully_1": {}}, "mass": [2000], "iterations": iters, "time_step": 1, "adiabatic": True,
            "absorbing_potential": {"bounds": [[-20, 5]], "exponent": 0.05, "track_population": True, "stop_norm": 0.5},
            "write": {"population": "P", "position": "X", "total_energy": "E", "norm": "N"}}


def harmonic_itp():
    return {"grid": {"bounds": [[-8, 8]], "npoint": 256},
            "initial_conditions": {"momentum": [0.3], "position": [1], "gamma": [2]},
            "potential": {"harmonic": {}}, "imaginary": {"nstate": 3}, "mass": [1], "iterations": 300,
            "time_step": 0.01, "write": {"total_energy": "E", "norm": "N"}}


def td_1d():
    return {"grid": {"bounds": [[-8, 8]], "npoint": 256},
            "initial_conditions": {"momentum": [0.5], "position": [-1], "state": 0, "gamma": [1], "adiabatic": True},
            "potential": {"custom": {"ndim": 1, "time_dependent": True,
                                     "matrix": [["0.5*r1^2 + (t - 2.5)*0.4", "0.3*exp(-r1^2)"],
                                                ["0.3*exp(-r1^2)", "0.5*r1^2 - (t - 2.5)*0.4"]]}},
            "mass": [1], "iterations": 400, "time_step": 0.01, "adiabatic": True,
            "write": {"population": "P", "wavefunction": "W"}}


def coupled_2d(iters=120):
    mat = [["0.5*(r1^2+r2^2)", "0.02*exp(-r1^2)"], ["0.02*exp(-r1^2)", "0.5*(r1^2+r2^2)+0.1"]]
    return {"grid": {"bounds": [[-8, 8], [-8, 8]], "npoint": 64},
            "initial_conditions": {"position": [1, 0], "momentum": [0, 1], "gamma": [1, 1], "state": 0},
            "potential": {"custom": {"ndim": 2, "matrix": mat}}, "mass": [1, 1], "iterations": iters,
            "time_step": 0.05, "write": {"population": "P", "total_energy": "E", "acf": "A"}}


def cap_2d():
    opt = coupled_2d(400)
    opt["initial_conditions"] = {"position": [0, 0], "momentum": [4, 0], "gamma": [1, 1], "state": 0}
    opt["potential"] = {"custom": {"ndim": 2, "matrix": [["0.01*(r1^2+r2^2)", "0.01"], ["0.01", "0.01*(r1^2+r2^2)"]]}}
    opt["absorbing_potential"] = {"bounds": [[-5, 5], [-5, 5]], "exponent": 0.5, "track_population": True,
                                  "stop_norm": 0.6}
    opt["write"] = {"population": "P", "norm": "N"}
    return opt


def stepped(opt, chunk, precision="fp64"):
    job = qd.Job(opt, precision)
    rows = []
    while True:
        job.step(chunk)
        rows += job.observables()
        if job.progress()[2]:
            break
    rows += job.observables()
    res = job.result()
    job.close()
    return res, rows


def itp_2d():
    # the first solve defers each step's renormalisation into the next step's passes; the second
    # (orthogonalised against the first) renormalises in the step
    opt = coupled_2d(60)
    opt["imaginary"] = {"nstate": 2}
    opt["write"] = {"population": "P", "total_energy": "E", "acf": "A", "norm": "N"}
    return opt


CASES = {"tully_cap_stop": tully_cap, "itp_three_solves": harmonic_itp, "time_dependent": td_1d,
         "2d_acf": coupled_2d, "2d_cap_stop": cap_2d, "2d_itp_two_solves": itp_2d}


@pytest.mark.parametrize("case", sorted(CASES))
@pytest.mark.parametrize("chunk", [1, 37, 100000])
def test_step_pieces_equal_whole_run(case, chunk):
    if chunk == 1 and case in ("tully_cap_stop", "2d_cap_stop"):
        chunk = 3  # keep the launch count moderate
    opt = CASES[case]()
    whole = qd.Job(opt)
    whole.run()
    a = whole.result()
    whole.close()
    b, rows = stepped(opt, chunk)
    _same(a, b)
    # every history row exactly once, in order, per solve
    width = rows[0][2].shape[1]
    for s, ob in enumerate(b.observables):
        got = np.concatenate([r for (sv, first, r) in rows if sv == s])
        firsts = [first for (sv, first, r) in rows if sv == s]
        assert firsts[0] == 0 and got.shape[1] == width
        nrows = next(iter(ob.history.values())).shape[0]
        assert got.shape[0] == nrows


def test_step_rows_match_the_history_columns():
    opt = coupled_2d()
    res, rows = stepped(opt, 25)
    got = np.concatenate([r for (_, _, r) in rows])
    h = res.observables[0].history
    S, d = 2, 2
    np.testing.assert_array_equal(got[:, 1 + 2 * d:1 + 2 * d + S], h["population"])
    np.testing.assert_array_equal(got[:, 1 + 2 * d + S] + got[:, 2 + 2 * d + S], h["total_energy"][:, 0]
                                  if h["total_energy"].ndim == 2 else h["total_energy"])
    np.testing.assert_array_equal(got[:, 3 + 2 * d + S] + 1j * got[:, 4 + 2 * d + S], h["acf"])
    assert np.all(np.isnan(got[:, 1:1 + d]))  # position not recorded


def test_step_fp32_equals_fp32_run():
    opt = {"grid": {"bounds": [[-24, 24]], "npoint": 8192},
           "initial_conditions": {"position": [-10], "momentum": [20], "gamma": [1.0], "state": 0, "adiabatic": True},
           "potential": {"custom": {"ndim": 1, "matrix": [["0.01*tanh(1.6*r1)", "0.005*exp(-r1^2)"],
                                                          ["0.005*exp(-r1^2)", "-0.01*tanh(1.6*r1)"]]}},
           "mass": [2000], "iterations": 300, "time_step": 1, "adiabatic": True, "write": {"population": "P"}}
    a = qd.run(opt, precision="fp32")
    b, _ = stepped(opt, 64, "fp32")
    _same(a, b)


def test_result_before_the_end_is_refused():
    job = qd.Job(coupled_2d())
    job.step(10)
    with pytest.raises(_abi.ZqdError, match="NOT FINISHED"):
        job.result()
    job.close()


# ---------------------------------------------------------------- server
def line_job(p0, iters=600, npoint=1024):
    return {"grid": {"bounds": [[-24, 24]], "npoint": npoint},
            "initial_conditions": {"position": [-10.0], "momentum": [float(p0)], "gamma": [float(p0 * p0 / 400.0)],
                                   "state": 0, "adiabatic": True},
            "potential": {"custom": {"ndim": 1, "matrix": [["0.01*tanh(1.6*r1)", "0.005*exp(-r1^2)"],
                                                           ["0.005*exp(-r1^2)", "-0.01*tanh(1.6*r1)"]]}},
            "mass": [2000.0], "iterations": iters, "time_step": 1.0, "adiabatic": True, "write": {"population": "P"}}


def drain(srv, tickets, timeout_s=120):
    """Polls until every ticket has its completion event; returns {ticket: [events]}."""
    ev = {t: [] for t in tickets}
    done = set()
    t0 = time.time()
    while len(done) < len(tickets):
        for e in srv.poll():
            ev.setdefault(e["ticket"], []).append(e)
            if e["kind"] != "rows":
                done.add(e["ticket"])
        assert time.time() - t0 < timeout_s
        time.sleep(0.002)
    return ev


def test_streamed_rows_concatenate_to_the_history():
    # launches of 50 steps (the persistent kernel's streaming is tested with it)
    srv = qd.Server(workers=2, stream_steps=50, persistent_lines=False)
    opts = [line_job(p) for p in (10, 20, 30)] + [coupled_2d(130)]
    tickets = [srv.submit(o, "fp64") for o in opts]
    ev = drain(srv, tickets)
    for t, o in zip(tickets, opts):
        r, _ = srv.wait(t)
        kinds = [e["kind"] for e in ev[t]]
        assert kinds[-1] == "done" and kinds.count("rows") >= 2
        rows = np.concatenate([e["rows"] for e in ev[t] if e["kind"] == "rows"])
        d, S = len(o["grid"]["bounds"]), 2
        np.testing.assert_array_equal(rows[:, 1 + 2 * d:1 + 2 * d + S], r.observables[0].history["population"])
    srv.close()


def test_requests_join_a_group_already_on_the_gpu():
    srv = qd.Server(workers=1, max_batch=8, stream_steps=64, persistent_lines=False)
    first = srv.submit(line_job(15, iters=3000), "fp32")
    time.sleep(0.05)  # the first request is on the GPU now
    later = [srv.submit(line_job(p, iters=400), "fp32") for p in (10, 20, 25, 30)]
    out = {t: srv.wait(t)[0] for t in [first] + later}
    st = srv.stats()
    srv.close()
    assert st["joined_jobs"] >= 1, st
    for t, o in zip([first] + later, [line_job(15, iters=3000)] + [line_job(p, iters=400) for p in (10, 20, 25, 30)]):
        alone = qd.run(o, precision="fp32", want_wavefunction=False)
        np.testing.assert_array_equal(out[t].observables[0].history["population"],
                                      alone.observables[0].history["population"])


def test_cancel_queued_and_running_requests():
    srv = qd.Server(workers=1, stream_steps=32)
    long2d = coupled_2d(20000)
    running = srv.submit(long2d, "fp64")
    queued = srv.submit(line_job(10), "fp64")
    time.sleep(0.2)
    srv.cancel(queued)
    srv.cancel(running)
    for t in (running, queued):
        with pytest.raises(_abi.ZqdError) as ex:
            srv.wait(t)
        assert ex.value.status == -10  # ZQD_ERR_CANCELLED
    after = srv.submit(line_job(20, iters=100), "fp64")  # the server goes on
    r, _ = srv.wait(after)
    st = srv.stats()
    srv.close()
    assert st["cancelled"] == 2
    np.testing.assert_array_equal(r.observables[0].history["population"],
                                  alone_as_served(line_job(20, iters=100), "fp64").observables[0].history["population"])


def test_wait_timeout_then_result():
    srv = qd.Server(workers=1, stream_steps=64)
    t = srv.submit(coupled_2d(3000), "fp64")
    with pytest.raises(_abi.ZqdError) as ex:
        srv.wait(t, timeout_ms=1)
    assert ex.value.status == -9  # ZQD_ERR_TIMEOUT
    r, _ = srv.wait(t)
    assert abs(r.observables[0].norm - 1) < 1e-10
    srv.close()


def test_device_allocation_refused_at_admission_fails_only_that_request():
    lib = _abi.load()
    srv = qd.Server(workers=1)
    try:
        lib.zqd_testing_fail_device_allocations(0, 1)  # the next device allocation fails
        bad = srv.submit(line_job(10, iters=50), "fp64")
        with pytest.raises(_abi.ZqdError) as ex:
            srv.wait(bad)
        assert ex.value.status == -3  # ZQD_ERR_DEVICE_OOM
    finally:
        lib.zqd_testing_fail_device_allocations(0, 0)
    good = srv.submit(line_job(10, iters=50), "fp64")
    r, _ = srv.wait(good)
    st = srv.stats()
    srv.close()
    assert st["failed"] == 1 and st["device_bytes_in_use"] == 0
    assert abs(r.observables[0].norm - 1) < 1e-10


def test_consumer_that_stops_polling_loses_only_row_events():
    srv = qd.Server(workers=2, stream_steps=8, max_events=6)
    opts = [line_job(p, iters=200) for p in (10, 20, 30)]
    tickets = [srv.submit(o, "fp64") for o in opts]
    res = [srv.wait(t)[0] for t in tickets]  # never polled while running
    st = srv.stats()
    events = srv.poll(1000)
    srv.close()
    assert st["dropped_events"] > 0 and st["pending_events"] <= 6
    assert sorted(e["ticket"] for e in events if e["kind"] == "done") == sorted(tickets)
    for o, r in zip(opts, res):
        np.testing.assert_array_equal(r.observables[0].history["population"],
                                      alone_as_served(o, "fp64").observables[0].history["population"])


def test_job_whose_norm_turns_nan_fails_alone():
    nan_job = {"grid": {"bounds": [[-8, 8]], "npoint": 256},
               "initial_conditions": {"position": [0], "momentum": [0], "gamma": [1], "state": 0},
               "potential": {"custom": {"ndim": 1, "matrix": [["sqrt(r1 - 100)"]]}},  # NaN on the whole grid
               "mass": [1], "iterations": 50, "time_step": 0.05, "write": {"norm": "N"}}
    srv = qd.Server(workers=2, stream_steps=16)
    bad = srv.submit(nan_job, "fp64")
    good = srv.submit(line_job(10, iters=100), "fp64")
    with pytest.raises(_abi.ZqdError) as ex:
        srv.wait(bad)
    assert ex.value.status == -13  # ZQD_ERR_NUMERIC
    r, _ = srv.wait(good)
    srv.close()
    assert abs(r.observables[0].norm - 1) < 1e-10
