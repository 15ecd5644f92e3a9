"""CPU-only checks of the C-ABI boundary (no compute without a GPU).

* libzinq_qd.so loads and exports every entry point include/zinq_qd.h declares;
* the ctypes mirror of zqd_options has the C layout (zqd_options_init writes sizeof);
* option validation reproduces checkInvalidInput (src/quantum_dynamics.zig:606-710)
  message by message, before any device is touched;
* expression compilation errors surface as ZQD_ERR_EXPRESSION (exprtk_init's null,
  src/exprtk.cpp:21-23).
"""
import copy
import ctypes as C
import re

import pytest

from zinq_b200 import _abi
from zinq_b200 import quantum_dynamics as qd


def header_functions():
    text = open(_abi.HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(zqd_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = _abi.load()
    names = header_functions()
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    declared = {s[0] for s in _abi.SIGNATURES}
    assert set(names) == declared, set(names) ^ declared


def test_options_struct_layout_matches_header():
    lib = _abi.load()
    o = _abi.ZqdOptions()
    lib.zqd_options_init(C.byref(o))
    assert o.struct_size == C.sizeof(_abi.ZqdOptions)
    assert o.log_interval == 1 and abs(o.cap_exponent - 0.001) < 1e-18 and abs(o.spectrum_threshold - 1e-6) < 1e-20
    p = _abi.ZqdPotential()
    lib.zqd_potential_init(C.byref(p), _abi.POT["tully_2"])
    assert list(p.p) == [0.10, 0.28, 0.015, 0.06, 0.05]


def test_status_strings():
    lib = _abi.load()
    for code in _abi.STATUS:
        assert lib.zqd_status_string(code)


BASE = {
    "grid": {"bounds": [[-16, 16]], "npoint": 256},
    "initial_conditions": {"position": [0], "momentum": [0], "gamma": [2], "state": 0},
    "potential": {"harmonic": {}},
    "mass": [1],
    "iterations": 10,
    "time_step": 0.1,
}

CASES = [
    (lambda o: o.update(time_step=0), "TIME STEP MUST BE GREATER THAN 0"),
    (lambda o: o.update(mass=[-1]), "MASS MUST BE GREATER THAN 0"),
    (lambda o: o.update(log_interval=0), "LOG INTERVAL MUST BE GREATER THAN 0"),
    (lambda o: o["grid"].update(npoint=0), "GRID POINT COUNT MUST BE GREATER THAN 0"),
    (lambda o: o["grid"].update(bounds=[[1, -1]]), "GRID BOUNDS MIN MUST BE LESS THAN MAX"),
    (lambda o: o.update(absorbing_potential={"bounds": [[-20, 10]]}),
     "ABSORBING POTENTIAL BOUNDS MUST LIE WITHIN GRID BOUNDS AND CB[0] < CB[1]"),
    (lambda o: o.update(absorbing_potential={"bounds": [[-10, 10]], "exponent": 0}),
     "ABSORBING POTENTIAL EXPONENT MUST BE GREATER THAN 0"),
    (lambda o: o.update(absorbing_potential={"bounds": [[-10, 10]], "stop_norm": 1.5}),
     "ABSORBING POTENTIAL STOP_NORM MUST BE BETWEEN 0 AND 1"),
    (lambda o: o.update(spectrum={"threshold": 2}), "SPECTRUM THRESHOLD MUST BE BETWEEN 0 AND 1"),
    (lambda o: o["initial_conditions"].update(state=3), "INITIAL STATE INDEX OUT OF RANGE"),
    (lambda o: o.update(potential={"tully_1": {}}, mass=[1, 1], grid={"bounds": [[-1, 1], [-1, 1]], "npoint": 8},
                        initial_conditions={"position": [0, 0], "momentum": [0, 0], "gamma": [1, 1]}),
     "POTENTIAL DIMENSION DOES NOT MATCH GRID DIMENSION"),
]


@pytest.mark.parametrize("mutate,message", CASES)
def test_invalid_input_matches_reference_messages(mutate, message):
    opt = copy.deepcopy(BASE)
    mutate(opt)
    with pytest.raises(qd.ZqdError) as e:
        qd.Job(opt)
    assert e.value.status == -1
    assert message in str(e.value)


def test_imaginary_zero_states_rejected():
    opt = copy.deepcopy(BASE)
    opt["imaginary"] = {"nstate": 0}
    with pytest.raises(qd.ZqdError, match="ITP TARGET STATE COUNT MUST BE GREATER THAN 0"):
        qd.Job(opt)


def test_non_power_of_two_grid_is_unsupported_not_invalid():
    opt = copy.deepcopy(BASE)
    opt["grid"]["npoint"] = 300
    with pytest.raises(qd.ZqdError) as e:
        qd.Job(opt)
    assert e.value.status == -7


@pytest.mark.parametrize("bad", ["exp(", "r2 + 1", "foo(r1)", "1 +* 2", "r1 $ 2"])
def test_expression_errors(bad):
    lib = _abi.load()
    h = C.c_void_p()
    rc = lib.zqd_expr_compile(bad.encode(), len(bad), 1, C.byref(h))
    assert rc == -6, lib.zqd_last_error()
    opt = copy.deepcopy(BASE)
    opt["potential"] = {"custom": {"ndim": 1, "matrix": [[bad]]}}
    with pytest.raises(qd.ZqdError) as e:
        qd.Job(opt)
    assert e.value.status == -6


@pytest.mark.parametrize("good", ["0.5*r1^2", "+sgn(r1) * 0.01 * (1.0 - exp(-1.6 * abs(r1)))",
                                  "0.005 * exp(-r1^2)", "-r1^3/3 + pi*t", "min(r1, 2, t) + max(1, r1)",
                                  "if(r1 < 0, tanh(r1), sqrt(abs(r1)))", "2r1 + 3(r1-1)", "pow(r1, 2.5) + r1^-2"])
def test_expression_compiles(good):
    lib = _abi.load()
    h = C.c_void_p()
    assert lib.zqd_expr_compile(good.encode(), len(good), 1, C.byref(h)) == 0, lib.zqd_last_error()
    lib.zqd_expr_destroy(h)


def test_server_config_defaults_and_no_device_status():
    lib = _abi.load()
    cfg = _abi.ZqdServerConfig()
    lib.zqd_server_config_init(C.byref(cfg))
    assert cfg.struct_size == C.sizeof(_abi.ZqdServerConfig) and cfg.workers == 8 and cfg.max_batch == 16
    import torch

    if not torch.cuda.is_available():
        h = C.c_void_p()
        assert lib.zqd_server_create(C.byref(cfg), C.byref(h)) == -12  # ZQD_ERR_NO_DEVICE


def test_auto_precision_is_a_valid_job_option_but_not_an_fft_precision():
    lib = _abi.load()
    assert _abi.PRECISION["auto"] == 2
    opt = copy.deepcopy(BASE)
    opt["grid"]["npoint"] = 300  # fails after validation: the precision itself was accepted
    with pytest.raises(qd.ZqdError) as e:
        qd.Job(opt, "auto")
    assert e.value.status == -7
    o, keep = qd.to_struct(BASE, "fp64")
    o.precision = 7
    h = C.c_void_p()
    assert lib.zqd_job_create(C.byref(o), C.byref(h)) == -1
    assert "UNKNOWN PRECISION" in lib.zqd_last_error().decode()
    shape = (C.c_int * 1)(64)
    plan = C.c_void_p()
    assert lib.zqd_fft_plan_create(1, shape, -1, 2, C.byref(plan)) == -1
    assert "FFT PRECISION" in lib.zqd_last_error().decode()
    assert lib.zqd_result_precision(None) == -1
