"""TEST INFRASTRUCTURE ONLY: ctypes front end of the oracle (oracle/libqd_ref.so).

The oracle is a CPU restatement of Zinq's grid split-operator path
(src/quantum_dynamics.zig:567-950, src/wavepacket.zig:16-421,
src/potential.zig:19-615 of tjira/zinq).  This module maps a
``quantum_dynamics`` options dict written in the reference's JSON schema
(src/quantum_dynamics.zig:25-67, src/wavepacket.zig:16-23,
src/potential.zig:19-60) onto the oracle's C struct and returns the same
observables ``quantum_dynamics.run`` returns (one entry per imaginary-time
state, quantum_dynamics.zig:70-83).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline legs may
import it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass, field

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libqd_ref.so")

POT_KIND = {"harmonic": 0, "time_linear": 1, "tully_1": 2, "tully_2": 3, "tully_3": 4, "custom": 5, "lvc": 6, "file": 7}
POT_DEFAULTS = {  # src/potential.zig:19-60
    "harmonic": {"k": [1.0]},
    "time_linear": {"a": 10.0, "g": 2.0},
    "tully_1": {"A": 0.010, "B": 1.600, "C": 0.005, "D": 1.000},
    "tully_2": {"A": 0.10, "B": 0.28, "C": 0.015, "D": 0.06, "E0": 0.05},
    "tully_3": {"A": 6.0e-4, "B": 0.10, "C": 0.90},
}
PARAM_ORDER = {
    "time_linear": ["a", "g"],
    "tully_1": ["A", "B", "C", "D"],
    "tully_2": ["A", "B", "C", "D", "E0"],
    "tully_3": ["A", "B", "C"],
}
W_BITS = {"acf": 1, "kinetic_energy": 2, "momentum": 4, "norm": 8, "population": 16, "position": 32,
          "potential_energy": 64, "total_energy": 128, "wavefunction": 256}


class _Pot(C.Structure):
    _fields_ = [
        ("kind", C.c_int), ("params", C.POINTER(C.c_double)), ("nparams", C.c_int),
        ("custom_ndim", C.c_int), ("custom_nstate", C.c_int), ("exprs", C.POINTER(C.c_char_p)),
        ("time_dependent", C.c_int),
        ("lvc_nmode", C.c_int), ("lvc_nstate", C.c_int), ("lvc_freq", C.POINTER(C.c_double)),
        ("lvc_exc", C.POINTER(C.c_double)), ("lvc_kappa", C.POINTER(C.c_double)),
        ("lvc_lambda", C.POINTER(C.c_double)),
        ("file_ndim", C.c_int), ("file_nrow", C.c_int), ("file_ncol", C.c_int),
        ("file_data", C.POINTER(C.c_double)),
    ]


class _Opt(C.Structure):
    _fields_ = [
        ("ndim", C.c_int), ("npoint", C.c_uint32), ("bounds", C.POINTER(C.c_double)),
        ("mass", C.POINTER(C.c_double)), ("time_step", C.c_double), ("iterations", C.c_uint32),
        ("log_interval", C.c_uint32), ("ic_position", C.POINTER(C.c_double)),
        ("ic_momentum", C.POINTER(C.c_double)), ("ic_gamma", C.POINTER(C.c_double)),
        ("ic_state", C.c_uint32), ("ic_adiabatic", C.c_int), ("adiabatic", C.c_int),
        ("has_cap", C.c_int), ("cap_track_population", C.c_int), ("cap_bounds", C.POINTER(C.c_double)),
        ("cap_exponent", C.c_double), ("cap_has_stop_norm", C.c_int), ("cap_stop_norm", C.c_double),
        ("imag_nstate", C.c_uint32), ("has_spectrum", C.c_int), ("spectrum_padding", C.c_uint32),
        ("spectrum_threshold", C.c_double), ("write_mask", C.c_uint32), ("nthreads", C.c_int),
        ("pot", _Pot), ("ic_wavefunction", C.POINTER(C.c_double)),
    ]


_lib = None


def build():
    """Compile the oracle library with its Makefile (g++ only, no GPU needed)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        L.qr_run.argtypes = [C.POINTER(_Opt), C.POINTER(C.c_void_p)]
        L.qr_run.restype = C.c_int
        L.qr_last_error.restype = C.c_char_p
        L.qr_free.argtypes = [C.c_void_p]
        for f in ("qr_nsolve", "qr_nstate", "qr_ndim"):
            getattr(L, f).argtypes = [C.c_void_p]
            getattr(L, f).restype = C.c_int
        L.qr_npoint_total.argtypes = [C.c_void_p]
        L.qr_npoint_total.restype = C.c_size_t
        dp = C.POINTER(C.c_double)
        L.qr_final.argtypes = [C.c_void_p, C.c_int, dp, dp, dp, dp, dp, dp, dp]
        L.qr_hist_rows.argtypes = [C.c_void_p, C.c_int]
        L.qr_hist_rows.restype = C.c_size_t
        L.qr_hist.argtypes = [C.c_void_p, C.c_int, C.c_char_p, dp]
        L.qr_hist.restype = C.c_int
        L.qr_wavefunction.argtypes = [C.c_void_p, C.c_int, dp]
        L.qr_spectrum_len.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_size_t)]
        L.qr_spectrum_len.restype = C.c_size_t
        L.qr_spectrum.argtypes = [C.c_void_p, C.c_int, dp, dp]
        L.qr_eigh.argtypes = [C.c_int, dp, dp, dp]
        L.qr_fft.argtypes = [C.c_int, C.POINTER(C.c_int), C.c_int, dp]
        L.qr_expr_eval.argtypes = [C.c_char_p, C.c_int, dp, C.c_double, dp]
        L.qr_expr_eval.restype = C.c_int
        _lib = L
    return _lib


class OracleError(ValueError):
    pass


def _dptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


@dataclass
class Observables:
    pos: np.ndarray
    mom: np.ndarray
    pop: np.ndarray
    epot: float
    ekin: float
    norm: float
    acf: complex | None
    history: dict = field(default_factory=dict)
    wavefunction: np.ndarray | None = None
    spectrum: tuple | None = None


def _read_matrix(path):
    """readMatrix, src/read_write.zig:24-56: header "rows cols" then whitespace-separated values."""
    with open(path) as f:
        hdr = f.readline().split()
        nrow, ncol = int(hdr[0]), int(hdr[1])
        data = np.array(f.read().split(), dtype=np.float64)
    return data[: nrow * ncol].reshape(nrow, ncol)


def run(opt: dict, nthreads: int = 1, want_wavefunction: bool = True, initial_wavefunction=None):
    """Run one ``quantum_dynamics`` job on the oracle; returns a list of Observables.

    initial_wavefunction: optional complex array (nstate x npoint^ndim) replacing the Gaussian,
    for chaining an imaginary-time relaxation into real time (no reference counterpart)."""
    keep = []

    def arr(x):
        a = np.ascontiguousarray(np.asarray(x, dtype=np.float64).ravel())
        keep.append(a)
        return _dptr(a)

    o = _Opt()
    g = opt["grid"]
    ndim = len(g["bounds"])
    o.ndim = ndim
    o.npoint = int(g["npoint"])
    o.bounds = arr(g["bounds"])
    o.mass = arr(opt["mass"])
    o.time_step = float(opt["time_step"])
    o.iterations = int(opt["iterations"])
    o.log_interval = int(opt.get("log_interval", 1))
    ic = opt["initial_conditions"]
    o.ic_position = arr(ic["position"])
    o.ic_momentum = arr(ic["momentum"])
    o.ic_gamma = arr(ic["gamma"])
    if not (len(opt["mass"]) == len(ic["position"]) == len(ic["momentum"]) == len(ic["gamma"]) == ndim):
        raise OracleError("INITIAL CONDITIONS / MASS DIMENSION MISMATCH")
    o.ic_state = int(ic.get("state", 0))
    o.ic_adiabatic = int(bool(ic.get("adiabatic", False)))
    o.adiabatic = int(bool(opt.get("adiabatic", False)))
    cap = opt.get("absorbing_potential")
    if cap is not None:
        o.has_cap = 1
        o.cap_track_population = int(bool(cap.get("track_population", False)))
        if len(cap["bounds"]) != ndim:
            raise OracleError("ABSORBING POTENTIAL BOUNDS DIMENSION DOES NOT MATCH GRID DIMENSION")
        o.cap_bounds = arr(cap["bounds"])
        o.cap_exponent = float(cap.get("exponent", 0.001))
        if cap.get("stop_norm") is not None:
            o.cap_has_stop_norm = 1
            o.cap_stop_norm = float(cap["stop_norm"])
    imag = opt.get("imaginary")
    if imag is not None:
        o.imag_nstate = int(imag.get("nstate", 1))
        if o.imag_nstate == 0:
            raise OracleError("ITP TARGET STATE COUNT MUST BE GREATER THAN 0")
    spec = opt.get("spectrum")
    if spec is not None:
        o.has_spectrum = 1
        o.spectrum_padding = int(spec.get("padding", 0))
        o.spectrum_threshold = float(spec.get("threshold", 1e-6))
    wm = 0
    for k, v in (opt.get("write") or {}).items():
        if v is not None:
            wm |= W_BITS[k]
    o.write_mask = wm
    o.nthreads = int(nthreads)
    if initial_wavefunction is not None:
        w = np.ascontiguousarray(np.asarray(initial_wavefunction, dtype=np.complex128)).view(np.float64).ravel()
        keep.append(w)
        o.ic_wavefunction = _dptr(w)

    (pname, pval), = opt["potential"].items()
    pval = dict(POT_DEFAULTS.get(pname, {}), **(pval or {}))
    p = o.pot
    p.kind = POT_KIND[pname]
    if pname == "harmonic":
        p.params = arr(pval["k"])
        p.nparams = len(pval["k"])
    elif pname in PARAM_ORDER:
        vals = [pval[k] for k in PARAM_ORDER[pname]]
        p.params = arr(vals)
        p.nparams = len(vals)
    elif pname == "custom":
        mat = pval["matrix"]
        ns = len(mat)
        if any(len(row) != ns for row in mat):
            raise OracleError("NonSquareMatrix")
        strs = [s.encode() for row in mat for s in row]
        cs = (C.c_char_p * len(strs))(*strs)
        keep.append(cs)
        p.exprs = C.cast(cs, C.POINTER(C.c_char_p))
        p.custom_ndim = int(pval["ndim"])
        p.custom_nstate = ns
        p.time_dependent = int(bool(pval.get("time_dependent", False)))
    elif pname == "lvc":
        freq = np.asarray(pval["frequencies"], float)
        exc = np.asarray(pval["excitation_energies"], float)
        p.lvc_nmode, p.lvc_nstate = len(freq), len(exc)
        p.lvc_freq, p.lvc_exc = arr(freq), arr(exc)
        p.lvc_kappa = arr(np.asarray(pval["kappa"], float))
        p.lvc_lambda = arr(np.asarray(pval["lambda"], float))
    elif pname == "file":
        table = pval["data"] if "data" in pval else _read_matrix(pval["path"])
        table = np.ascontiguousarray(table, dtype=np.float64)
        p.file_ndim = int(pval["ndim"])
        p.file_nrow, p.file_ncol = table.shape
        p.file_data = arr(table)

    L = lib()
    h = C.c_void_p()
    rc = L.qr_run(C.byref(o), C.byref(h))
    if rc != 0:
        raise OracleError(L.qr_last_error().decode())
    try:
        out = []
        d, S, N = L.qr_ndim(h), L.qr_nstate(h), L.qr_npoint_total(h)
        for s in range(L.qr_nsolve(h)):
            pos, mom, pop = np.zeros(d), np.zeros(d), np.zeros(S)
            epot, ekin, norm, acf = np.zeros(1), np.zeros(1), np.zeros(1), np.zeros(2)
            L.qr_final(h, s, _dptr(pos), _dptr(mom), _dptr(pop), _dptr(epot), _dptr(ekin), _dptr(norm), _dptr(acf))
            rows = L.qr_hist_rows(h, s)
            hist = {}
            for name in ("pos", "mom", "pop", "epot", "ekin", "etot", "norm", "acf"):
                cols = L.qr_hist(h, s, name.encode(), None)
                if cols > 0:
                    buf = np.zeros(rows * cols)
                    L.qr_hist(h, s, name.encode(), _dptr(buf))
                    hist[name] = buf.reshape(rows, cols)
            if "acf" in hist:
                hist["acf"] = hist["acf"][:, 0] + 1j * hist["acf"][:, 1]
            cols = L.qr_hist(h, s, b"wfn", None)
            if cols > 0:  # History.wfn: rows x S x N complex
                buf = np.zeros(rows * cols)
                L.qr_hist(h, s, b"wfn", _dptr(buf))
                hist["wfn"] = (buf[0::2] + 1j * buf[1::2]).reshape(rows, S, N)
            wf = None
            if want_wavefunction:
                buf = np.zeros(2 * S * N)
                L.qr_wavefunction(h, s, _dptr(buf))
                wf = (buf[0::2] + 1j * buf[1::2]).reshape(S, N)
            spec = None
            if o.has_spectrum:
                plen = C.c_size_t()
                ns = L.qr_spectrum_len(h, s, C.byref(plen))
                ap, sg = np.zeros(2 * plen.value), np.zeros(ns)
                L.qr_spectrum(h, s, _dptr(ap), _dptr(sg))
                spec = (ap[0::2] + 1j * ap[1::2], sg)
            out.append(Observables(pos=pos, mom=mom, pop=pop, epot=float(epot[0]), ekin=float(ekin[0]),
                                   norm=float(norm[0]), acf=None if np.isnan(acf[0]) else complex(acf[0], acf[1]),
                                   history=hist, wavefunction=wf, spectrum=spec))
        return out
    finally:
        L.qr_free(h)


def eigh(V):
    V = np.ascontiguousarray(V, dtype=np.float64)
    n = V.shape[0]
    W, U = np.zeros(n), np.zeros((n, n))
    lib().qr_eigh(n, _dptr(V), _dptr(W), _dptr(U))
    return W, U


def fft(x, sign):
    x = np.ascontiguousarray(x, dtype=np.complex128).copy()
    shape = (C.c_int * x.ndim)(*x.shape)
    buf = x.view(np.float64)
    lib().qr_fft(x.ndim, shape, int(sign), _dptr(buf))
    return x


def expr_eval(expr: str, r, t: float = 0.0):
    r = np.ascontiguousarray(np.asarray(r, dtype=np.float64))
    out = np.zeros(1)
    rc = lib().qr_expr_eval(expr.encode(), len(r), _dptr(r), float(t), _dptr(out))
    if rc != 0:
        raise OracleError(lib().qr_last_error().decode())
    return float(out[0])
