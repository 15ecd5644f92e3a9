// tune.cu -- the launch-shape autotuner, keyed on (dims, points, states, precision).
//
// The kernels take their shape from fixed rules unless this table holds a measured choice:
//   1-D  resident line kernel: CTAs per cluster C (1..16) and the largest local radix (4 or 8);
//   N-D  axis passes: rows per block and lines per tile of the TMA-staged persistent passes (or
//        the per-block kernels instead), and rows of the last axis per per-block row CTA (the
//        launches that take the per-block kernel).
// zqd_autotune times every candidate the kernels accept on the current device (a synthetic job of
// the key's size: harmonic diagonal, constant couplings, populations recorded every step; the
// propagation's device time from CUDA events, best of three runs) and records the fastest.  The
// table is per process; zqd_tune_save / zqd_tune_load keep it in a text file, and the file named by
// ZQD_TUNE_FILE is loaded before the first job is created.  A tuned shape changes the order of
// floating-point operations only inside the transforms (a different factorisation of the same
// DFT), never the algorithm: results stay within the FP64 and FP32 parity bars.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "internal.h"
#include "job.h"

namespace zqd {
namespace {

using Key = std::tuple<int, int, int, int>; // dims, points per axis, states, fp32

struct Table {
    std::mutex mu;
    std::map<Key, ShapeOverride> shapes;
    std::once_flag env_once;
};
Table& table() {
    static Table t;
    return t;
}
thread_local bool t_forcing = false;
thread_local ShapeOverride t_forced;

int load_file(const char* path, bool replace) {
    FILE* f = std::fopen(path, "r");
    if (!f) return fail(ZQD_ERR_NOT_FOUND, std::string("cannot open tuning table ") + path);
    std::map<Key, ShapeOverride> got;
    char line[256];
    int lineno = 0;
    while (std::fgets(line, sizeof line, f)) {
        ++lineno;
        if (line[0] == '#' || line[0] == '\n') continue;
        int d, n, S, fp32;
        ShapeOverride s;
        const int got_fields = std::sscanf(line, "%d %d %d %d %d %d %d %d %d %d", &d, &n, &S, &fp32, &s.C, &s.lrmax, &s.rows,
                                           &s.tile, &s.tma_rows, &s.tma_w);
        if (got_fields != 8 && got_fields != 10) { // 8: a table written before the TMA-staged passes
            std::fclose(f);
            return fail(ZQD_ERR_INVALID_INPUT, std::string("tuning table ") + path + ": bad line " + std::to_string(lineno));
        }
        got[Key{d, n, S, fp32}] = s;
    }
    std::fclose(f);
    Table& t = table();
    std::lock_guard<std::mutex> lk(t.mu);
    if (replace) t.shapes.clear();
    for (auto& kv : got) t.shapes[kv.first] = kv.second;
    return ZQD_OK;
}

// A synthetic job of the key's size: S harmonic surfaces with constant couplings on [-10, 10]^d.
Opts synthetic(int d, int n, int S, bool fp32, int iters) {
    Opts o;
    o.ndim = (uint32_t)d;
    o.npoint = (uint32_t)n;
    for (int j = 0; j < d; ++j) {
        o.bounds.push_back(-10.0);
        o.bounds.push_back(10.0);
        o.pos.push_back(j == 0 ? -1.0 : 0.0);
        o.mom.push_back(j == 0 ? 1.0 : 0.0);
        o.gamma.push_back(1.0);
        o.mass.push_back(1.0);
    }
    o.time_step = 0.01;
    o.iterations = (uint32_t)iters;
    o.write_mask = ZQD_WRITE_POPULATION;
    o.precision = fp32 ? ZQD_FP32_MIXED : ZQD_FP64;
    o.pkind = ZQD_POT_CUSTOM;
    o.custom_ns = (uint32_t)S;
    o.custom_nd = (uint32_t)d;
    std::string r2 = "r1^2";
    for (int j = 1; j < d; ++j) r2 += "+r" + std::to_string(j + 1) + "^2";
    for (int a = 0; a < S; ++a)
        for (int b = 0; b < S; ++b) o.custom.push_back(a == b ? "0.5*(" + r2 + ")+" + std::to_string(0.1 * a) : "0.01");
    o.pot_nd = d;
    o.pot_ns = S;
    return o;
}

// device time per step of one candidate shape, or a negative value when the kernels refuse it
double time_shape(int d, int n, int S, bool fp32, const ShapeOverride& cand) {
    const int iters = d == 1 ? 200 : (n >= 1024 ? 6 : 20);
    t_forcing = true;
    t_forced = cand;
    zqd_job* J = nullptr;
    const int rc = job_create_opts(synthetic(d, n, S, fp32, iters), &J);
    t_forcing = false;
    if (rc) return -1.0;
    if (J->d == 1 && ((cand.C && J->C != cand.C) || (cand.lrmax && J->lrmax != cand.lrmax))) {
        zqd_job_destroy(J); // the rules fell back to another shape: not this candidate
        return -1.0;
    }
    double best = INFINITY;
    for (int rep = 0; rep < 4; ++rep) { // the first run captures the graph (N-D) and warms up
        if (zqd_job_run(J)) {
            zqd_job_destroy(J);
            return -1.0;
        }
        if (rep) best = std::fmin(best, (double)zqd_job_device_ms(J));
    }
    zqd_job_destroy(J);
    return 1e3 * best / iters;
}

} // namespace

int job_create_shaped(Opts&& o, const ShapeOverride& shape, zqd_job** out, cudaStream_t stream) {
    t_forcing = true;
    t_forced = shape;
    const int rc = job_create_opts(std::move(o), out, stream);
    t_forcing = false;
    return rc;
}

bool lookup_shape(int d, int n, int S, bool fp32, ShapeOverride& out) {
    if (t_forcing) {
        out = t_forced;
        return true;
    }
    Table& t = table();
    std::call_once(t.env_once, [] {
        if (const char* path = std::getenv("ZQD_TUNE_FILE")) load_file(path, false); // missing: the rules decide
    });
    std::lock_guard<std::mutex> lk(t.mu);
    auto it = t.shapes.find(Key{d, n, S, fp32 ? 1 : 0});
    if (it == t.shapes.end()) return false;
    out = it->second;
    return true;
}

} // namespace zqd

using namespace zqd;

extern "C" int zqd_autotune(zqd_tune_entry* e) {
    if (!e) return fail(ZQD_ERR_INVALID_INPUT, "NULL ARGUMENT");
    const int d = (int)e->ndim, n = (int)e->npoint, S = (int)e->nstate;
    if (d < 1 || d > ZQD_MAX_NDIM || S < 1 || S > ZQD_MAX_NSTATE || n < 4 || (n & (n - 1)))
        return fail(ZQD_ERR_INVALID_INPUT, "AUTOTUNE KEY OUT OF RANGE (ndim 1..3, states 1..4, npoint a power of two)");
    if (e->precision != ZQD_FP64 && e->precision != ZQD_FP32_MIXED)
        return fail(ZQD_ERR_INVALID_INPUT, "AUTOTUNE PRECISION MUST BE ZQD_FP64 OR ZQD_FP32_MIXED");
    const bool fp32 = e->precision == ZQD_FP32_MIXED;
    std::vector<ShapeOverride> cands;
    if (d == 1) {
        for (int C : {1, 2, 4, 8, 16}) {
            ShapeOverride s;
            s.C = C;
            s.lrmax = 2;
            cands.push_back(s);
        }
        ShapeOverride r8;
        r8.C = 16;
        r8.lrmax = 3;
        cands.push_back(r8);
    }
    const double def = time_shape(d, n, S, fp32, ShapeOverride{}); // the rules' own choice
    if (def < 0) return fail(ZQD_ERR_UNSUPPORTED, "THE KERNELS DO NOT SUPPORT THIS KEY");
    ShapeOverride best{};
    double best_us = def;
    uint32_t tried = 0;
    auto consider = [&](const ShapeOverride& c) {
        const double us = time_shape(d, n, S, fp32, c);
        if (us < 0) return;
        ++tried;
        if (us < best_us) {
            best_us = us;
            best = c;
        }
    };
    if (d == 1) {
        for (const ShapeOverride& c : cands) consider(c);
    } else {
        // one field at a time, each from the best shape so far: the row pass's blocks (or the
        // per-block row kernel with its rows per CTA), then the tile pass's lines (or the
        // per-block tile kernel with its lines per CTA)
        const ShapeOverride base0 = best;
        for (int L : {-1, 1, 2, 4, 8, 16, 32, 64}) {
            ShapeOverride c = base0;
            c.tma_rows = L;
            consider(c);
        }
        if (best.tma_rows < 0) {
            const ShapeOverride base1 = best;
            for (int L = 1; L <= 64; L <<= 1) {
                ShapeOverride c = base1;
                c.rows = L;
                consider(c);
            }
        }
        const ShapeOverride base2 = best;
        for (int W : {-1, 1, 2, 4, 8, 16}) {
            ShapeOverride c = base2;
            c.tma_w = W;
            consider(c);
        }
        if (best.tma_w < 0) {
            const ShapeOverride base3 = best;
            for (int Tn = 1; Tn <= 16; Tn <<= 1) {
                ShapeOverride c = base3;
                c.tile = Tn;
                consider(c);
            }
        }
    }
    e->default_us_per_step = def;
    e->us_per_step = best_us;
    e->candidates = tried;
    e->cluster_ctas = (uint32_t)best.C;
    e->radix_log2 = (uint32_t)best.lrmax;
    e->rows_per_cta = (uint32_t)best.rows;
    e->tile_lines = (uint32_t)best.tile;
    e->tma_row_block = best.tma_rows;
    e->tma_tile_lines = best.tma_w;
    Table& t = table();
    std::lock_guard<std::mutex> lk(t.mu);
    if (best.C || best.rows || best.tile || best.tma_rows || best.tma_w) t.shapes[std::make_tuple(d, n, S, fp32 ? 1 : 0)] = best;
    else t.shapes.erase(std::make_tuple(d, n, S, fp32 ? 1 : 0)); // the rules' shape won
    return ZQD_OK;
}

extern "C" int zqd_tune_save(const char* path) {
    if (!path) return fail(ZQD_ERR_INVALID_INPUT, "NULL PATH");
    Table& t = table();
    std::lock_guard<std::mutex> lk(t.mu);
    FILE* f = std::fopen(path, "w");
    if (!f) return fail(ZQD_ERR_INVALID_INPUT, std::string("cannot write ") + path);
    std::fprintf(f, "# ndim npoint nstate fp32 cluster_ctas radix_log2 rows_per_cta tile_lines tma_row_block tma_tile_lines"
                    " (0: the rules' choice; -1: the per-block kernel)\n");
    for (auto& kv : t.shapes) {
        const Key& k = kv.first;
        const ShapeOverride& s = kv.second;
        std::fprintf(f, "%d %d %d %d %d %d %d %d %d %d\n", std::get<0>(k), std::get<1>(k), std::get<2>(k), std::get<3>(k),
                     s.C, s.lrmax, s.rows, s.tile, s.tma_rows, s.tma_w);
    }
    std::fclose(f);
    return ZQD_OK;
}

extern "C" int zqd_tune_load(const char* path) {
    if (!path) return fail(ZQD_ERR_INVALID_INPUT, "NULL PATH");
    return load_file(path, false);
}

extern "C" void zqd_tune_clear(void) {
    Table& t = table();
    std::lock_guard<std::mutex> lk(t.mu);
    t.shapes.clear();
}

extern "C" uint32_t zqd_tune_size(void) {
    Table& t = table();
    std::lock_guard<std::mutex> lk(t.mu);
    return (uint32_t)t.shapes.size();
}
