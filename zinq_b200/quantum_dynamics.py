"""Host-side mirror of Zinq's `quantum_dynamics` method over the C-ABI.

`run(options)` takes a ``quantum_dynamics`` options object in the reference's
JSON schema (src/quantum_dynamics.zig:25-67, src/wavepacket.zig:16-23,
src/potential.zig:19-60) and returns a `Result` whose ``observables`` list
holds one `Observables` per imaginary-time state, like
``quantum_dynamics.run(f64, io, opt, log, gpa)`` (:567-603).  Invalid input
raises `ZqdError` with the reference's message (checkInvalidInput, :606-710).
All arithmetic runs on the GPU through libzinq_qd.so.
"""
from __future__ import annotations

import ctypes as C
import json
from dataclasses import dataclass, field

import numpy as np

from . import _abi
from ._abi import ZqdError, check

POT_DEFAULTS = {  # src/potential.zig:24-48
    "harmonic": {"k": [1.0]},
    "time_linear": {"a": 10.0, "g": 2.0},
    "tully_1": {"A": 0.010, "B": 1.600, "C": 0.005, "D": 1.000},
    "tully_2": {"A": 0.10, "B": 0.28, "C": 0.015, "D": 0.06, "E0": 0.05},
    "tully_3": {"A": 6.0e-4, "B": 0.10, "C": 0.90},
}
PARAM_ORDER = {"time_linear": ["a", "g"], "tully_1": ["A", "B", "C", "D"], "tully_2": ["A", "B", "C", "D", "E0"],
               "tully_3": ["A", "B", "C"]}


@dataclass
class Observables:
    """Final expectation values of one solve (Observables, quantum_dynamics.zig:282-375)."""
    pos: np.ndarray
    mom: np.ndarray
    pop: np.ndarray
    epot: float
    ekin: float
    norm: float
    acf: complex | None
    history: dict = field(default_factory=dict)
    wavefunction: np.ndarray | None = None
    spectrum: tuple | None = None  # (windowed, padded acf; sigma) of calcSpectrum when `spectrum` is set


@dataclass
class Result:
    """Result(T) (quantum_dynamics.zig:70-83) plus the device time of the propagation and the
    precision the job ran in ("fp64" or "fp32"; a job submitted as "auto" reports its choice)."""
    observables: list
    device_ms: float = 0.0
    precision: str = ""


_PRECISION_NAME = {0: "fp64", 1: "fp32"}


def _result(L, res, obs) -> "Result":
    return Result(observables=obs, device_ms=L.zqd_result_device_ms(res),
                  precision=_PRECISION_NAME.get(L.zqd_result_precision(res), ""))


def read_matrix(path):
    """readMatrix (src/read_write.zig:24-56): a "rows cols" header, then whitespace-separated values."""
    with open(path) as f:
        hdr = f.readline().split()
        nrow, ncol = int(hdr[0]), int(hdr[1])
        data = np.array(f.read().split(), dtype=np.float64)
    return data[: nrow * ncol].reshape(nrow, ncol)


class _Keep:
    """Owns the ctypes buffers an options struct points at."""

    def __init__(self):
        self.refs = []

    def arr(self, x):
        a = np.ascontiguousarray(np.asarray(x, dtype=np.float64).ravel())
        self.refs.append(a)
        return a.ctypes.data_as(_abi.DP)


def to_struct(opt: dict, precision: str = "fp64", log: bool = False, initial_wavefunction=None):
    """Translate a reference-schema options dict into zqd_options; returns (struct, keepalive).

    initial_wavefunction: optional complex array (nstate x npoint^ndim, state-major, last axis
    fastest) replacing the Gaussian of initial_conditions (zqd_options.ic_wavefunction)."""
    L = _abi.load()
    keep = _Keep()
    o = _abi.ZqdOptions()
    L.zqd_options_init(C.byref(o))
    g = opt["grid"]
    bounds = [list(b) for b in g["bounds"]]
    o.ndim = len(bounds)
    o.npoint = int(g["npoint"])
    o.grid_bounds = keep.arr(bounds)
    ic = opt["initial_conditions"]
    o.ic_position, o.ic_momentum, o.ic_gamma = keep.arr(ic["position"]), keep.arr(ic["momentum"]), keep.arr(ic["gamma"])
    # the C struct carries one length (ndim) for these arrays; mismatches are reported with the reference's messages
    if len(opt["mass"]) != len(ic["position"]):
        raise ZqdError(-1, "MASS VECTOR MUST HAVE THE SAME LENGTH AS POSITION VECTOR")
    if len(ic["momentum"]) != len(ic["position"]):
        raise ZqdError(-1, "INITIAL MOMENTUM AND POSITION VECTORS MUST HAVE THE SAME LENGTH")
    if len(ic["gamma"]) != len(ic["position"]):
        raise ZqdError(-1, "INITIAL GAMMA VECTOR MUST HAVE THE SAME LENGTH AS POSITION VECTOR")
    if len(ic["position"]) == 0:
        raise ZqdError(-1, "INITIAL POSITION VECTOR MUST NOT BE EMPTY")
    if len(ic["position"]) != len(bounds):
        raise ZqdError(-1, "INITIAL CONDITIONS DIMENSION DOES NOT MATCH GRID DIMENSION")
    o.ic_state = int(ic.get("state", 0))
    o.ic_adiabatic = int(bool(ic.get("adiabatic", False)))
    o.time_step = float(opt["time_step"])
    o.iterations = int(opt["iterations"])
    o.mass = keep.arr(opt["mass"])
    wm = 0
    for k, v in (opt.get("write") or {}).items():
        if v is not None:
            wm |= _abi.WRITE[k]
    o.write_mask = wm
    o.adiabatic = int(bool(opt.get("adiabatic", False)))
    o.log_interval = int(opt.get("log_interval", 1))
    cap = opt.get("absorbing_potential")
    if cap is not None:
        if len(cap["bounds"]) != len(bounds):
            raise ZqdError(-1, "ABSORBING POTENTIAL BOUNDS DIMENSION DOES NOT MATCH GRID DIMENSION")
        o.has_absorbing_potential = 1
        o.cap_track_population = int(bool(cap.get("track_population", False)))
        o.cap_bounds = keep.arr(cap["bounds"])
        o.cap_exponent = float(cap.get("exponent", 0.001))
        if cap.get("stop_norm") is not None:
            o.cap_has_stop_norm = 1
            o.cap_stop_norm = float(cap["stop_norm"])
    o.fft_plan = _abi.FFT_PLAN[(opt.get("fft") or {}).get("plan", "measure")]
    imag = opt.get("imaginary")
    if imag is not None:
        o.imaginary_nstate = int(imag.get("nstate", 1))
        if o.imaginary_nstate == 0:
            raise ZqdError(-1, "ITP TARGET STATE COUNT MUST BE GREATER THAN 0")
    spec = opt.get("spectrum")
    if spec is not None:
        o.has_spectrum = 1
        o.spectrum_padding = int(spec.get("padding", 0))
        o.spectrum_threshold = float(spec.get("threshold", 1e-6))
    o.precision = _abi.PRECISION[precision]
    o.log = int(bool(log))
    if initial_wavefunction is not None:
        w = np.ascontiguousarray(np.asarray(initial_wavefunction, dtype=np.complex128)).view(np.float64).ravel()
        o.ic_wavefunction = keep.arr(w)

    (pname, pval), = opt["potential"].items()
    pval = dict(POT_DEFAULTS.get(pname, {}), **(pval or {}))
    p = o.potential
    L.zqd_potential_init(C.byref(p), _abi.POT[pname])
    if pname == "harmonic":
        p.harmonic_k = keep.arr(pval["k"])
        p.harmonic_ndim = len(pval["k"])
    elif pname in PARAM_ORDER:
        for i, k in enumerate(PARAM_ORDER[pname]):
            p.p[i] = float(pval[k])
    elif pname == "custom":
        mat = pval["matrix"]
        ns = len(mat)
        if any(len(row) != ns for row in mat):
            raise ZqdError(-1, "NonSquareMatrix")
        strs = [s.encode() for row in mat for s in row]
        arr = (C.c_char_p * len(strs))(*strs)
        keep.refs.append(arr)
        p.custom_matrix = C.cast(arr, C.POINTER(C.c_char_p))
        p.custom_nstate = ns
        p.custom_ndim = int(pval["ndim"])
        p.custom_time_dependent = int(bool(pval.get("time_dependent", False)))
    elif pname == "lvc":
        freq = np.asarray(pval["frequencies"], float)
        exc = np.asarray(pval["excitation_energies"], float)
        p.lvc_frequencies, p.lvc_nmode = keep.arr(freq), len(freq)
        p.lvc_excitation_energies, p.lvc_nstate = keep.arr(exc), len(exc)
        p.lvc_kappa = keep.arr(np.asarray(pval["kappa"], float))
        p.lvc_lambda = keep.arr(np.asarray(pval["lambda"], float))
    elif pname == "file":
        table = pval["data"] if "data" in pval else read_matrix(pval["path"])
        table = np.ascontiguousarray(table, dtype=np.float64)
        p.file_table = keep.arr(table)
        p.file_nrow, p.file_ncol = table.shape
        p.file_ndim = int(pval["ndim"])
    else:
        raise ZqdError(-1, f"UNKNOWN POTENTIAL {pname}")
    return o, keep


def _collect(res_ptr):
    L = _abi.load()
    out = []
    for s in range(L.zqd_result_nsolve(res_ptr)):
        ob = _abi.ZqdObservables()
        check(L.zqd_result_final(res_ptr, s, C.byref(ob)))
        d, S = ob.ndim, ob.nstate
        hist = {}
        for name, code in _abi.SERIES.items():
            ptr, rows, cols = _abi.DP(), C.c_size_t(), C.c_size_t()
            if L.zqd_result_series(res_ptr, s, code, C.byref(ptr), C.byref(rows), C.byref(cols)) == 0:
                a = np.ctypeslib.as_array(ptr, shape=(rows.value * cols.value,)).copy().reshape(rows.value, cols.value)
                hist[name] = a[:, 0] + 1j * a[:, 1] if name == "acf" else a
        acf = None if np.isnan(ob.acf_re) else complex(ob.acf_re, ob.acf_im)
        nr, nt = C.c_size_t(), C.c_size_t()
        if L.zqd_result_wavefunction_series(res_ptr, s, None, 0, C.byref(nr), C.byref(nt)) == 0:
            buf = np.zeros(2 * nr.value * S * nt.value)
            check(L.zqd_result_wavefunction_series(res_ptr, s, buf.ctypes.data_as(_abi.DP), buf.size, C.byref(nr),
                                                   C.byref(nt)))
            hist["wavefunction"] = (buf[0::2] + 1j * buf[1::2]).reshape(nr.value, S, nt.value)
        spec = None
        ap, na, sg, ns = _abi.DP(), C.c_size_t(), _abi.DP(), C.c_size_t()
        if L.zqd_result_spectrum(res_ptr, s, C.byref(ap), C.byref(na), C.byref(sg), C.byref(ns)) == 0:
            a = np.ctypeslib.as_array(ap, shape=(2 * na.value,)).copy() if na.value else np.zeros(0)
            sig = np.ctypeslib.as_array(sg, shape=(ns.value,)).copy() if ns.value else np.zeros(0)
            spec = (a[0::2] + 1j * a[1::2], sig)
        out.append(Observables(pos=np.array(ob.pos[:d]), mom=np.array(ob.mom[:d]), pop=np.array(ob.pop[:S]),
                               epot=ob.epot, ekin=ob.ekin, norm=ob.norm, acf=acf, history=hist, spectrum=spec))
    return out


def _attach_wavefunctions(res_ptr, obs, npoint_total, nstate):
    L = _abi.load()
    for s, ob in enumerate(obs):
        buf = np.zeros(2 * nstate * npoint_total)
        check(L.zqd_result_wavefunction(res_ptr, s, buf.ctypes.data_as(_abi.DP), buf.size))
        ob.wavefunction = (buf[0::2] + 1j * buf[1::2]).reshape(nstate, npoint_total)


def _shape(opt):
    g = opt["grid"]
    return int(g["npoint"]) ** len(g["bounds"])


def _export(L, res_ptr, opt):
    """History.exportWrite: writes the files named by opt["write"] and opt["spectrum"]["write"]; solve by
    solve to the same paths, so the last solve's history remains, as in the reference."""
    w = opt.get("write") or {}
    sw = (opt.get("spectrum") or {}).get("write") or {}
    vals = {n: w.get(n) for n in _abi.WRITE_PATH_FIELDS[:8]}
    vals["wavefunction"] = w.get("wavefunction")
    vals["spectrum_acf"], vals["spectrum"] = sw.get("acf"), sw.get("spectrum")
    if not any(vals.values()):
        return
    paths = _abi.ZqdWritePaths(**{k: str(v).encode() for k, v in vals.items() if v})
    for s in range(L.zqd_result_nsolve(res_ptr)):
        check(L.zqd_result_export(res_ptr, s, C.byref(paths)))


def run(opt: dict, precision: str = "fp64", log: bool = False, want_wavefunction: bool = True,
        initial_wavefunction=None, export: bool = False) -> Result:
    """quantum_dynamics.run on the GPU (src/quantum_dynamics.zig:567-603).

    initial_wavefunction replaces the initial Gaussian (e.g. the relaxed state of an
    imaginary-time run, to continue in real time); None keeps the reference's behaviour."""
    L = _abi.load()
    o, keep = to_struct(opt, precision, log, initial_wavefunction)
    res = C.c_void_p()
    check(L.zqd_run(C.byref(o), C.byref(res)))
    try:
        if export:
            _export(L, res, opt)
        obs = _collect(res)
        if want_wavefunction and obs:
            S = len(obs[0].pop)
            _attach_wavefunctions(res, obs, _shape(opt), S)
        return _result(L, res, obs)
    finally:
        L.zqd_result_destroy(res)


def run_batch(opts: list, precision: str = "fp64", want_wavefunction: bool = False) -> list:
    """Several independent jobs advanced together (zqd_run_batch); one Result per options dict."""
    L = _abi.load()
    structs = [to_struct(o, precision) for o in opts]
    arr = (C.POINTER(_abi.ZqdOptions) * len(opts))(*[C.pointer(s) for s, _ in structs])
    res = (C.c_void_p * len(opts))()
    check(L.zqd_run_batch(arr, len(opts), res))
    out = []
    try:
        for i, r in enumerate(res):
            obs = _collect(r)
            if want_wavefunction and obs:
                _attach_wavefunctions(r, obs, _shape(opts[i]), len(obs[0].pop))
            out.append(_result(L, r, obs))
    finally:
        for r in res:
            if r:
                L.zqd_result_destroy(r)
    return out


class Job:
    """Staged form: device tables built at construction, `run()` propagates with no host copies."""

    def __init__(self, opt: dict, precision: str = "fp64", initial_wavefunction=None):
        self._L = _abi.load()
        self.opt = opt
        self._o, self._keep = to_struct(opt, precision, False, initial_wavefunction)
        self._h = C.c_void_p()
        check(self._L.zqd_job_create(C.byref(self._o), C.byref(self._h)))

    def info(self):
        d, s, c = C.c_uint32(), C.c_uint32(), C.c_uint32()
        n, b = C.c_uint64(), C.c_size_t()
        check(self._L.zqd_job_info(self._h, C.byref(d), C.byref(s), C.byref(n), C.byref(c), C.byref(b)))
        return {"ndim": d.value, "nstate": s.value, "npoint_total": n.value, "cluster_ctas": c.value,
                "device_bytes": b.value}

    def nd_shape(self):
        """zqd_job_nd_shape: the 2-D / 3-D axis passes' launch shapes (TMA-staged forms, 0 where the
        per-block kernels run, and the per-block shapes)."""
        sh = _abi.ZqdNdShape()
        check(self._L.zqd_job_nd_shape(self._h, C.byref(sh)))
        return {name: getattr(sh, name) for name, _ in sh._fields_}

    def run(self) -> float:
        check(self._L.zqd_job_run(self._h))
        return self._L.zqd_job_device_ms(self._h)

    def step(self, nsteps: int) -> None:
        """zqd_job_step: propagate up to nsteps more steps (the first call also records row 0)."""
        check(self._L.zqd_job_step(self._h, int(nsteps)))

    def progress(self):
        """(solve in progress, rows recorded in it, every solve finished)"""
        s, r, f = C.c_uint32(), C.c_uint32(), C.c_int()
        check(self._L.zqd_job_progress(self._h, C.byref(s), C.byref(r), C.byref(f)))
        return s.value, r.value, bool(f.value)

    def observables(self):
        """Rows recorded since the last call: a list of (solve, first_row, rows[nrows, width]), one
        entry per solve with new rows (zqd_job_observables until it returns none)."""
        out = []
        while True:
            r = _abi.ZqdObsRows()
            check(self._L.zqd_job_observables(self._h, C.byref(r)))
            if r.nrows == 0:
                return out
            a = np.ctypeslib.as_array(r.rows, shape=(r.nrows * r.width,)).copy().reshape(r.nrows, r.width)
            out.append((r.solve, r.first_row, a))

    def result(self, want_wavefunction=True) -> Result:
        res = C.c_void_p()
        check(self._L.zqd_job_result(self._h, C.byref(res)))
        try:
            obs = _collect(res)
            if want_wavefunction and obs:
                _attach_wavefunctions(res, obs, _shape(self.opt), len(obs[0].pop))
            return _result(self._L, res, obs)
        finally:
            self._L.zqd_result_destroy(res)

    def close(self):
        if self._h:
            self._L.zqd_job_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Staged batch: every job's tables resident on the device; run() re-propagates all jobs."""

    def __init__(self, opts: list, precision: str = "fp64"):
        self._L = _abi.load()
        self.opts = opts
        self._structs = [to_struct(o, precision) for o in opts]
        arr = (C.POINTER(_abi.ZqdOptions) * len(opts))(*[C.pointer(s) for s, _ in self._structs])
        self._h = C.c_void_p()
        check(self._L.zqd_batch_create(arr, len(opts), C.byref(self._h)))

    def run(self) -> float:
        """Propagates every job once; returns the device time in ms (CUDA events)."""
        check(self._L.zqd_batch_run(self._h))
        return self._L.zqd_batch_device_ms(self._h)

    @property
    def launches(self) -> int:
        return self._L.zqd_batch_launches(self._h)

    def result(self, i: int, want_wavefunction=False) -> Result:
        res = C.c_void_p()
        check(self._L.zqd_batch_result(self._h, i, C.byref(res)))
        try:
            obs = _collect(res)
            if want_wavefunction and obs:
                _attach_wavefunctions(res, obs, _shape(self.opts[i]), len(obs[0].pop))
            return _result(self._L, res, obs)
        finally:
            self._L.zqd_result_destroy(res)

    def close(self):
        if self._h:
            self._L.zqd_batch_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def transfer_bytes(res_handle) -> tuple:
    L = _abi.load()
    h, d = C.c_uint64(), C.c_uint64()
    check(L.zqd_result_transfer_bytes(res_handle, C.byref(h), C.byref(d)))
    return h.value, d.value


def run_batch_e2e(opts: list, precision: str = "fp64"):
    """zqd_run_batch through the public API; returns (results, h2d bytes, d2h bytes)."""
    L = _abi.load()
    structs = [to_struct(o, precision) for o in opts]
    arr = (C.POINTER(_abi.ZqdOptions) * len(opts))(*[C.pointer(s) for s, _ in structs])
    res = (C.c_void_p * len(opts))()
    check(L.zqd_run_batch(arr, len(opts), res))
    h2d = d2h = 0
    out = []
    try:
        for r in res:
            h, d = transfer_bytes(r)
            h2d += h
            d2h += d
            out.append(_result(L, r, _collect(r)))
    finally:
        for r in res:
            if r:
                L.zqd_result_destroy(r)
    return out, h2d, d2h


def run_file(path: str, precision: str = "fp64", export: bool = True):
    """Runs every quantum_dynamics job of a Zinq input file ({"zinq": [...]}, src/main.zig:63-73,122-135),
    writing the files its `write` options name, like the reference."""
    with open(path) as f:
        doc = json.load(f)
    out = []
    for entry in doc["zinq"]:
        for tag, opt in entry.items():
            if tag != "quantum_dynamics":
                raise ZqdError(-7, f"method {tag!r} is outside this library")
            out.append(run(opt, precision, log=True, export=export))
    return out


class Server:
    """Request loop for streams of independent jobs (zqd_server_*): submit() returns a ticket at once,
    wait() returns (Result, latency in ms from submission to completion)."""

    def __init__(self, workers: int = 8, max_batch: int = 16, device_budget_bytes: int = 0, stream_steps: int = 256,
                 stream_rows: bool = True, max_events: int = 65536, persistent_lines: bool = True,
                 service_ctas: int = 64, service_idle_us: float = 200.0, fetch_wavefunction: bool = True):
        self._L = _abi.load()
        cfg = _abi.ZqdServerConfig()
        self._L.zqd_server_config_init(C.byref(cfg))
        cfg.workers, cfg.max_batch, cfg.device_budget_bytes = workers, max_batch, device_budget_bytes
        cfg.stream_steps, cfg.stream_rows, cfg.max_events = stream_steps, int(bool(stream_rows)), max_events
        cfg.persistent_lines, cfg.service_ctas = int(bool(persistent_lines)), service_ctas
        cfg.service_idle_us = service_idle_us
        cfg.fetch_wavefunction = int(bool(fetch_wavefunction))
        self._h = C.c_void_p()
        check(self._L.zqd_server_create(C.byref(cfg), C.byref(self._h)))
        self._shapes = {}

    def submit(self, opt: dict, precision: str = "fp32", initial_wavefunction=None) -> int:
        o, keep = to_struct(opt, precision, False, initial_wavefunction)
        t = C.c_uint64()
        check(self._L.zqd_server_submit(self._h, C.byref(o), C.byref(t)))
        self._shapes[t.value] = _shape(opt)
        return t.value

    def wait(self, ticket: int, want_wavefunction: bool = False, timeout_ms: int | None = None):
        """(Result, latency ms); with timeout_ms, ZqdError(ZQD_ERR_TIMEOUT) when not done in time."""
        res, lat = C.c_void_p(), C.c_double()
        if timeout_ms is None:
            check(self._L.zqd_server_wait(self._h, ticket, C.byref(res), C.byref(lat)))
        else:
            check(self._L.zqd_server_wait_timeout(self._h, ticket, int(timeout_ms), C.byref(res), C.byref(lat)))
        npt = self._shapes.pop(ticket, None)
        try:
            obs = _collect(res)
            if want_wavefunction and obs:
                _attach_wavefunctions(res, obs, npt, len(obs[0].pop))
            return _result(self._L, res, obs), lat.value
        finally:
            self._L.zqd_result_destroy(res)

    def cancel(self, ticket: int) -> None:
        check(self._L.zqd_server_cancel(self._h, ticket))

    def poll(self, max_events: int = 1024) -> list:
        """Pending events, oldest first: dicts with ticket, kind ("rows", "done", "failed",
        "cancelled"), status, solve, first_row and, for row events, rows (nrows x width)."""
        buf = (_abi.ZqdEvent * max_events)()
        n = C.c_uint32()
        check(self._L.zqd_server_poll(self._h, buf, max_events, C.byref(n)))
        out = []
        for e in buf[:n.value]:
            d = {"ticket": e.ticket, "kind": _abi.EVENT[e.kind], "status": e.status, "solve": e.solve,
                 "first_row": e.first_row, "solve_finished": bool(e.solve_finished)}
            if e.kind == 0:
                d["rows"] = (np.ctypeslib.as_array(e.rows, shape=(e.nrows * e.width,)).copy().reshape(e.nrows, e.width)
                             if e.rows else np.zeros((e.nrows, e.width)))
            out.append(d)
        return out

    def stats(self) -> dict:
        s = _abi.ZqdServerStats()
        check(self._L.zqd_server_stats_get(self._h, C.byref(s)))
        return {name: getattr(s, name) for name, _ in s._fields_}

    def close(self):
        if self._h:
            self._L.zqd_server_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def serve_stream(opts: list, arrivals_s: list, precision: str = "fp32", workers: int = 8, max_batch: int = 16,
                 **server_kw):
    """Submits opts[i] at arrivals_s[i] seconds after the start (a feeder thread sleeps until each
    arrival), waits for all; returns (results, latencies_ms, wall_s from the first arrival to the
    last completion, server stats).  A job that fails leaves None in results and (index, message)
    in stats["failures"]."""
    import threading
    import time

    srv = Server(workers=workers, max_batch=max_batch, **server_kw)
    tickets = [None] * len(opts)
    errors = []
    t0 = time.perf_counter()

    def feed():
        try:
            for i, (o, a) in enumerate(zip(opts, arrivals_s)):
                dt = a - (time.perf_counter() - t0)
                if dt > 0:
                    time.sleep(dt)
                tickets[i] = srv.submit(o, precision)
        except Exception as e:  # surfaced after the join
            errors.append(e)

    th = threading.Thread(target=feed)
    th.start()
    results, lats = [None] * len(opts), [0.0] * len(opts)
    failures = []
    for i in range(len(opts)):
        while tickets[i] is None and th.is_alive():
            time.sleep(0.0005)
        if tickets[i] is None:
            break
        try:
            results[i], lats[i] = srv.wait(tickets[i])
        except ZqdError as e:  # the job failed alone (e.g. ZQD_ERR_NUMERIC); the others stand
            failures.append((i, str(e)))
    th.join()
    wall = time.perf_counter() - t0 - (arrivals_s[0] if arrivals_s else 0.0)
    st = srv.stats()
    st["failures"] = failures
    srv.close()
    if errors:
        raise errors[0]
    return results, lats, wall, st


def serving_stream(njobs: int, seed: int = 7, rate_per_s: float = 200.0, max_steps: int = 5000):
    """The serving workload: njobs jobs with Poisson arrivals, parameters drawn from `seed`.
    dims in {1, 2}; 1-D grids of 2^8..2^14 points on [-L, L], L ~ U(8, 32); 2-D grids of
    2^6..2^9 points per axis on [-L, L]^2, L ~ U(8, 16); states in {1, 2, 3}; harmonic
    (V_ii = 0.5 w^2 r^2 + c_i) or tanh-crossing (V_ii = +-A tanh(B r)) diabatic surfaces with
    couplings C exp(-r^2); A, C, c_i ~ U(-0.02, 0.02); mass ~ U(1, 2000); steps ~ U{100..max_steps};
    dt = 0.05 sqrt(mass); Gaussian at x0 = -L/3, p0 ~ U(0, 10), gamma 1.  Returns (opts, arrivals)."""
    rng = np.random.default_rng(seed)
    opts, arrivals, t = [], [], 0.0
    for _ in range(njobs):
        t += rng.exponential(1.0 / rate_per_s)
        d = int(rng.integers(1, 3))
        if d == 1:
            n, L = 2 ** int(rng.integers(8, 15)), float(rng.uniform(8, 32))
        else:
            n, L = 2 ** int(rng.integers(6, 10)), float(rng.uniform(8, 16))
        S = int(rng.integers(1, 4))
        family = "harmonic" if rng.uniform() < 0.5 else "tanh"
        A, Cc = rng.uniform(-0.02, 0.02), rng.uniform(-0.02, 0.02)
        c = rng.uniform(-0.02, 0.02, S)
        mass = float(rng.uniform(1, 2000))
        steps = int(rng.integers(100, max_steps + 1))
        p0 = float(rng.uniform(0, 10))
        r2 = "r1^2" if d == 1 else "(r1^2+r2^2)"
        w2 = 1.0 / mass  # omega^2: a well of the packet's own time scale
        mat = []
        for i in range(S):
            row = []
            for j in range(S):
                if i == j:
                    if family == "harmonic":
                        row.append(f"0.5*{w2:.17g}*{r2}+{c[i]:.17g}")
                    else:
                        row.append(f"{(A if i % 2 == 0 else -A):.17g}*tanh(1.6*r1)")
                else:
                    row.append(f"{Cc:.17g}*exp(-{r2})")
            mat.append(row)
        opts.append({"grid": {"bounds": [[-L, L]] * d, "npoint": n},
                     "initial_conditions": {"position": [-L / 3] + [0.0] * (d - 1), "momentum": [p0] + [0.0] * (d - 1),
                                            "gamma": [1.0] * d, "state": 0, "adiabatic": False},
                     "potential": {"custom": {"ndim": d, "matrix": mat}}, "mass": [mass] * d,
                     "iterations": steps, "time_step": 0.05 * float(np.sqrt(mass)), "adiabatic": False,
                     "write": {"population": "P"}})
        arrivals.append(t)
    return opts, arrivals


def autotune(ndim: int, npoint: int, nstate: int, precision: str = "fp64") -> dict:
    """zqd_autotune: measure the launch shapes for a (dims, points, states, precision) key on this
    device and record the fastest; returns the entry (0 fields: the built-in rules' shape won)."""
    L = _abi.load()
    e = _abi.ZqdTuneEntry(ndim=ndim, npoint=npoint, nstate=nstate, precision=_abi.PRECISION[precision])
    check(L.zqd_autotune(C.byref(e)))
    return {name: getattr(e, name) for name, _ in e._fields_}


def tune_save(path: str) -> None:
    check(_abi.load().zqd_tune_save(str(path).encode()))


def tune_load(path: str) -> None:
    check(_abi.load().zqd_tune_load(str(path).encode()))


def tune_clear() -> None:
    _abi.load().zqd_tune_clear()


def potential_plot(opt: dict, write: bool = False) -> np.ndarray:
    """potential_plot.run (src/potential_plot.zig:48-106) on the device: the reference's options
    {potential, grid, adiabatic, time, write: {potential: path}}; returns V (or the adiabatic
    diagonal) as an array of npoint^ndim x nstate x nstate and, with write, writes the .mat file."""
    L = _abi.load()
    d = len(opt["grid"]["bounds"])
    full = {"grid": opt["grid"], "potential": opt["potential"], "adiabatic": bool(opt.get("adiabatic", False)),
            "initial_conditions": {"position": [0.0] * d, "momentum": [0.0] * d, "gamma": [1.0] * d, "state": 0},
            "mass": [1.0] * d, "time_step": 1.0, "iterations": 0}
    o, keep = to_struct(full)
    (pname, pval), = opt["potential"].items()
    if pname == "custom":
        S = len(pval["matrix"])
    elif pname == "lvc":
        S = len(pval["excitation_energies"])
    elif pname == "file":
        table = pval["data"] if "data" in pval else read_matrix(pval["path"])
        S = int(round(np.sqrt(np.asarray(table).shape[1] - int(pval["ndim"]))))
    else:
        S = 1 if pname in ("harmonic",) else 2
    N = int(opt["grid"]["npoint"]) ** d
    U = np.zeros(N * S * S)
    path = ((opt.get("write") or {}).get("potential") if write else None)
    check(L.zqd_potential_plot(C.byref(o), float(opt.get("time", 0.0)), U.ctypes.data_as(_abi.DP), U.size,
                               path.encode() if path else None))
    return U.reshape(N, S, S)
