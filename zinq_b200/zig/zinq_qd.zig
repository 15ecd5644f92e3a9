//! Zig host wrapper over the C-ABI of the B200 split-operator propagator (include/zinq_qd.h).
//!
//! Drops into Zinq's source tree as src/zinq_qd.zig and is imported like the other C libraries
//! (src/cimport.zig:3-8 imports FFTW and ExprTk with @cImport).  It maps Zinq's own
//! quantum_dynamics.Options (src/quantum_dynamics.zig:25-67), InitialConditions
//! (src/wavepacket.zig:16-23) and the potential Options union (src/potential.zig:19-60) onto
//! zqd_options, and the library's status codes onto a Zig error set in the spirit of the
//! reference's InvalidInput / PlanCreationFailed / LapackError / OutOfMemory.
//!
//! Written for Zig 0.16 (makefile:6 of the reference); this build image has no Zig toolchain, so the
//! file has not been compiled here.  Link with -lzinq_qd (linkSystemLibrary in build.zig's
//! linkDependencies, build.zig:93-133) and add include/ to the include path.

const std = @import("std");

const Allocator = std.mem.Allocator;

const QdOptions = @import("quantum_dynamics.zig").Options;
const PotentialOptions = @import("potential.zig").Options;
const readMatrix = @import("read_write.zig").readMatrix;

pub const c = @cImport(@cInclude("zinq_qd.h"));

pub const Error = error{
    InvalidInput,
    OutOfMemory,
    DeviceOutOfMemory,
    PlanCreationFailed,
    LapackError,
    ExpressionError,
    Unsupported,
    DeviceError,
    Timeout,
    Cancelled,
    NotFound,
    NoDevice,
    NonFiniteObservable,
};

/// Maps a zqd_status onto the error set; the library's detail text is in lastError().
pub fn check(rc: c_int) Error!void {
    return switch (rc) {
        c.ZQD_OK => {},
        c.ZQD_ERR_INVALID_INPUT => error.InvalidInput,
        c.ZQD_ERR_OUT_OF_MEMORY => error.OutOfMemory,
        c.ZQD_ERR_DEVICE_OOM => error.DeviceOutOfMemory,
        c.ZQD_ERR_PLAN_FAILED => error.PlanCreationFailed,
        c.ZQD_ERR_EIGEN_FAILED => error.LapackError,
        c.ZQD_ERR_EXPRESSION => error.ExpressionError,
        c.ZQD_ERR_UNSUPPORTED => error.Unsupported,
        c.ZQD_ERR_TIMEOUT => error.Timeout,
        c.ZQD_ERR_CANCELLED => error.Cancelled,
        c.ZQD_ERR_NOT_FOUND => error.NotFound,
        c.ZQD_ERR_NO_DEVICE => error.NoDevice,
        c.ZQD_ERR_NUMERIC => error.NonFiniteObservable,
        else => error.DeviceError,
    };
}

/// Detail of the last failing call on this thread (e.g. "MASS MUST BE GREATER THAN 0").
pub fn lastError() []const u8 {
    return std.mem.span(c.zqd_last_error());
}

pub const Precision = enum(c_uint) { fp64 = c.ZQD_FP64, fp32_mixed = c.ZQD_FP32_MIXED, auto = c.ZQD_PRECISION_AUTO };

/// zqd_options built from Zinq's Options.  Every array the struct points at lives in `arena`,
/// which must outlive the library call that takes the options (the library copies what it keeps).
pub fn fillOptions(io: std.Io, opt: QdOptions, precision: Precision, log: bool, arena: Allocator) !c.zqd_options {
    var o: c.zqd_options = undefined;
    c.zqd_options_init(&o);

    const ndim = opt.grid.bounds.len;
    o.ndim = @intCast(ndim);
    o.npoint = opt.grid.npoint;
    o.grid_bounds = try flatPairs(arena, opt.grid.bounds);

    const ic = opt.initial_conditions;
    o.ic_position = ic.position.ptr;
    o.ic_momentum = ic.momentum.ptr;
    o.ic_gamma = ic.gamma.ptr;
    o.ic_state = ic.state;
    o.ic_adiabatic = @intFromBool(ic.adiabatic);

    o.time_step = opt.time_step;
    o.iterations = opt.iterations;
    o.mass = opt.mass.ptr;
    o.adiabatic = @intFromBool(opt.adiabatic);
    o.log_interval = opt.log_interval;
    o.log = @intFromBool(log);
    o.precision = @intFromEnum(precision);

    var mask: u32 = 0;
    inline for (.{
        .{ "acf", c.ZQD_WRITE_ACF },                       .{ "kinetic_energy", c.ZQD_WRITE_KINETIC_ENERGY },
        .{ "momentum", c.ZQD_WRITE_MOMENTUM },             .{ "norm", c.ZQD_WRITE_NORM },
        .{ "population", c.ZQD_WRITE_POPULATION },         .{ "position", c.ZQD_WRITE_POSITION },
        .{ "potential_energy", c.ZQD_WRITE_POTENTIAL_ENERGY }, .{ "total_energy", c.ZQD_WRITE_TOTAL_ENERGY },
        .{ "wavefunction", c.ZQD_WRITE_WAVEFUNCTION },
    }) |w| {
        if (@field(opt.write, w[0]) != null) mask |= w[1];
    }
    o.write_mask = mask;

    if (opt.absorbing_potential) |ap| {
        o.has_absorbing_potential = 1;
        o.cap_track_population = @intFromBool(ap.track_population);
        o.cap_bounds = try flatPairs(arena, ap.bounds);
        o.cap_exponent = ap.exponent;
        if (ap.stop_norm) |s| {
            o.cap_has_stop_norm = 1;
            o.cap_stop_norm = s;
        }
    }
    o.fft_plan = @intFromEnum(opt.fft.plan);
    if (opt.imaginary) |imag| o.imaginary_nstate = imag.nstate;
    if (opt.spectrum) |sp| {
        o.has_spectrum = 1;
        o.spectrum_padding = sp.padding;
        o.spectrum_threshold = sp.threshold;
    }
    try fillPotential(io, &o.potential, opt.potential, arena);
    return o;
}

fn flatPairs(arena: Allocator, pairs: []const [2]f64) ![*c]const f64 {
    const flat = try arena.alloc(f64, 2 * pairs.len);
    for (pairs, 0..) |p, i| {
        flat[2 * i] = p[0];
        flat[2 * i + 1] = p[1];
    }
    return flat.ptr;
}

fn fillPotential(io: std.Io, p: *c.zqd_potential, pot: PotentialOptions, arena: Allocator) !void {
    switch (pot) {
        .harmonic => |h| {
            c.zqd_potential_init(p, c.ZQD_POT_HARMONIC);
            p.harmonic_k = h.k.ptr;
            p.harmonic_ndim = @intCast(h.k.len);
        },
        .time_linear => |t| {
            c.zqd_potential_init(p, c.ZQD_POT_TIME_LINEAR);
            p.p[0] = t.a;
            p.p[1] = t.g;
        },
        .tully_1 => |t| {
            c.zqd_potential_init(p, c.ZQD_POT_TULLY_1);
            p.p[0..4].* = .{ t.A, t.B, t.C, t.D };
        },
        .tully_2 => |t| {
            c.zqd_potential_init(p, c.ZQD_POT_TULLY_2);
            p.p = .{ t.A, t.B, t.C, t.D, t.E0 };
        },
        .tully_3 => |t| {
            c.zqd_potential_init(p, c.ZQD_POT_TULLY_3);
            p.p[0..3].* = .{ t.A, t.B, t.C };
        },
        .custom => |cu| {
            c.zqd_potential_init(p, c.ZQD_POT_CUSTOM);
            const ns = cu.matrix.len;
            const strs = try arena.alloc([*c]const u8, ns * ns);
            for (cu.matrix, 0..) |row, i| {
                if (row.len != ns) return error.InvalidInput;
                for (row, 0..) |expr, j| strs[i * ns + j] = (try arena.dupeZ(u8, expr)).ptr;
            }
            p.custom_matrix = strs.ptr;
            p.custom_nstate = @intCast(ns);
            p.custom_ndim = cu.ndim;
            p.custom_time_dependent = @intFromBool(cu.time_dependent);
        },
        .lvc => |l| {
            c.zqd_potential_init(p, c.ZQD_POT_LVC);
            const nm = l.frequencies.len;
            const ns = l.excitation_energies.len;
            const kappa = try arena.alloc(f64, ns * nm);
            for (l.kappa, 0..) |row, n| @memcpy(kappa[n * nm ..][0..nm], row);
            const lambda = try arena.alloc(f64, ns * ns * nm);
            for (l.lambda, 0..) |rows, m| for (rows, 0..) |row, n| @memcpy(lambda[(m * ns + n) * nm ..][0..nm], row);
            p.lvc_frequencies = l.frequencies.ptr;
            p.lvc_nmode = @intCast(nm);
            p.lvc_excitation_energies = l.excitation_energies.ptr;
            p.lvc_nstate = @intCast(ns);
            p.lvc_kappa = kappa.ptr;
            p.lvc_lambda = lambda.ptr;
        },
        .file => |f| {
            c.zqd_potential_init(p, c.ZQD_POT_FILE);
            // the same table File.init reads (src/potential.zig:460-462)
            const table = try readMatrix(f64, io, f.path, arena);
            p.file_table = table.data.ptr;
            p.file_nrow = @intCast(table.nrow());
            p.file_ncol = @intCast(table.ncol());
            p.file_ndim = f.ndim;
        },
    }
}

/// Result of a run: one final Observables per solve plus the recorded history, owned by the
/// library until deinit (the reference's Result.deinit).
pub const Run = struct {
    res: *c.zqd_result,

    pub fn deinit(self: *Run) void {
        c.zqd_result_destroy(self.res);
    }

    pub fn nsolve(self: Run) u32 {
        return c.zqd_result_nsolve(self.res);
    }

    /// Observables.init(..., log = true) after solve `s` (src/quantum_dynamics.zig:949).
    pub fn final(self: Run, s: u32) Error!c.zqd_observables {
        var ob: c.zqd_observables = undefined;
        try check(c.zqd_result_final(self.res, s, &ob));
        return ob;
    }

    /// One recorded time series (History, src/quantum_dynamics.zig:99-279): rows x cols, row-major.
    pub fn series(self: Run, s: u32, which: c.zqd_series) Error!struct { data: []const f64, cols: usize } {
        var ptr: [*c]const f64 = null;
        var rows: usize = 0;
        var cols: usize = 0;
        try check(c.zqd_result_series(self.res, s, which, &ptr, &rows, &cols));
        return .{ .data = ptr[0 .. rows * cols], .cols = cols };
    }

    /// History.exportWrite: the .mat text files the options' write paths name.
    pub fn exportWrite(self: Run, s: u32, paths: c.zqd_write_paths) Error!void {
        try check(c.zqd_result_export(self.res, s, &paths));
    }
};

/// quantum_dynamics.run on the GPU (src/quantum_dynamics.zig:567-603): same options, same validation
/// messages, one solve per imaginary-time state.  FP64 reproduces the reference's arithmetic.
pub fn run(io: std.Io, opt: QdOptions, precision: Precision, log: bool, gpa: Allocator) !Run {
    var arena_state = std.heap.ArenaAllocator.init(gpa);
    defer arena_state.deinit();
    const o = try fillOptions(io, opt, precision, log, arena_state.allocator());
    var res: ?*c.zqd_result = null;
    try check(c.zqd_run(&o, &res));
    return .{ .res = res.? };
}

/// Step-wise form: the device keeps the wavefunction between step() calls; observables() returns
/// the rows recorded since the previous call (layout documented with zqd_obs_rows).
pub const Job = struct {
    h: *c.zqd_job,

    pub fn init(io: std.Io, opt: QdOptions, precision: Precision, gpa: Allocator) !Job {
        var arena_state = std.heap.ArenaAllocator.init(gpa);
        defer arena_state.deinit();
        const o = try fillOptions(io, opt, precision, false, arena_state.allocator());
        var h: ?*c.zqd_job = null;
        try check(c.zqd_job_create(&o, &h));
        return .{ .h = h.? };
    }

    pub fn deinit(self: *Job) void {
        c.zqd_job_destroy(self.h);
    }

    pub fn step(self: Job, nsteps: u32) Error!void {
        try check(c.zqd_job_step(self.h, nsteps));
    }

    pub fn finished(self: Job) Error!bool {
        var done: c_int = 0;
        try check(c.zqd_job_progress(self.h, null, null, &done));
        return done != 0;
    }

    pub fn observables(self: Job) Error!c.zqd_obs_rows {
        var rows: c.zqd_obs_rows = undefined;
        try check(c.zqd_job_observables(self.h, &rows));
        return rows;
    }

    pub fn result(self: Job) Error!Run {
        var res: ?*c.zqd_result = null;
        try check(c.zqd_job_result(self.h, &res));
        return .{ .res = res.? };
    }
};

/// Request stream: submit from any thread, pull events (rows as they are computed, completion),
/// wait for a result, cancel.
pub const Server = struct {
    h: *c.zqd_server,

    pub fn init(workers: u32, stream_steps: u32) Error!Server {
        var cfg: c.zqd_server_config = undefined;
        c.zqd_server_config_init(&cfg);
        cfg.workers = workers;
        cfg.stream_steps = stream_steps;
        var h: ?*c.zqd_server = null;
        try check(c.zqd_server_create(&cfg, &h));
        return .{ .h = h.? };
    }

    pub fn deinit(self: *Server) void {
        c.zqd_server_destroy(self.h);
    }

    pub fn submit(self: Server, io: std.Io, opt: QdOptions, precision: Precision, gpa: Allocator) !u64 {
        var arena_state = std.heap.ArenaAllocator.init(gpa);
        defer arena_state.deinit();
        const o = try fillOptions(io, opt, precision, false, arena_state.allocator());
        var ticket: u64 = 0;
        try check(c.zqd_server_submit(self.h, &o, &ticket));
        return ticket;
    }

    /// Up to events.len pending events; their rows stay valid until the next poll.
    pub fn poll(self: Server, events: []c.zqd_event) Error![]c.zqd_event {
        var n: u32 = 0;
        try check(c.zqd_server_poll(self.h, events.ptr, @intCast(events.len), &n));
        return events[0..n];
    }

    pub fn wait(self: Server, ticket: u64, timeout_ms: ?u32) Error!Run {
        var res: ?*c.zqd_result = null;
        var latency: f64 = 0;
        if (timeout_ms) |ms| {
            try check(c.zqd_server_wait_timeout(self.h, ticket, ms, &res, &latency));
        } else {
            try check(c.zqd_server_wait(self.h, ticket, &res, &latency));
        }
        return .{ .res = res.? };
    }

    pub fn cancel(self: Server, ticket: u64) Error!void {
        try check(c.zqd_server_cancel(self.h, ticket));
    }
};
