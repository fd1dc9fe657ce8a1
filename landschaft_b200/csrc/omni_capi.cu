// omni_capi.cu -- the C ABI (include/lsb_omniscape.h): validation, workspace
// carving, kernel choice and placement, the launch sequence of one call, and
// a cache of CUDA graphs of that sequence.
//
// The call mirrors circuit::omniscape (src/cpp/circuit/omniscape.cpp:394-608):
// targets -> correction -> windows (in batches) -> scatter; the scatter is a
// gather that adds every batch into the maps in target order.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <vector>

#include "../../include/lsb_omniscape.h"
#include "omni_kernels.cuh"
#include "omni_adv.cuh"
#include "omni_windows.cuh"

namespace lsb {
namespace {

thread_local int64_t g_launches = 0;
thread_local bool g_time_windows = false;

void set_err(char *err, size_t len, const char *fmt, ...) {
    if (!err || len == 0) return;
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(err, len, fmt, ap);
    va_end(ap);
}

#define LSB_CK(call)                                                                   \
    do {                                                                               \
        cudaError_t e_ = (call);                                                       \
        if (e_ != cudaSuccess) {                                                       \
            set_err(err, errlen, "CUDA error %s at %s:%d", cudaGetErrorString(e_), __FILE__, __LINE__); \
            return LSB_ERR_CUDA;                                                       \
        }                                                                              \
    } while (0)

constexpr size_t kAlign = 256;
size_t align_up(size_t v, size_t a = kAlign) { return (v + a - 1) / a * a; }

// ---------------------------------------------------------------------------
// Geometry of a call.
// ---------------------------------------------------------------------------
struct Geom {
    int64_t nx, ny;
    int R, B, D, W, bs, br, nbx, nby;
    int64_t NL;
    bool correct, fp, conditions;
};

int make_geom(int64_t nx, int64_t ny, const lsb_omni_params *p, Geom *g, char *err, size_t errlen) {
    if (!p) {
        set_err(err, errlen, "params is NULL");
        return LSB_ERR_ARGUMENT;
    }
    if (p->radius < 0 || p->buffer < 0 || p->block_size < 1 || p->block_size % 2 == 0) {
        set_err(err, errlen, "radius and buffer must be >= 0 and block_size odd");
        return LSB_ERR_ARGUMENT;
    }
    if (nx < 1 || ny < 1) {
        set_err(err, errlen, "the raster must have at least one cell");
        return LSB_ERR_ARGUMENT;
    }
    g->nx = nx;
    g->ny = ny;
    g->R = p->radius;
    g->B = p->buffer;
    g->D = p->radius + p->buffer;
    g->W = 2 * g->D + 1;
    g->bs = p->block_size;
    g->br = (p->block_size - 1) / 2;
    g->nbx = nx - 2 * g->br > 0 ? static_cast<int>((nx - 2 * g->br - 1) / g->bs + 1) : 0;
    g->nby = ny - 2 * g->br > 0 ? static_cast<int>((ny - 2 * g->br - 1) / g->bs + 1) : 0;
    g->NL = static_cast<int64_t>(g->nbx) * g->nby;
    g->correct = p->correct_artifacts && g->bs > 1;
    g->fp = p->flow_potential != 0;
    g->conditions = p->condition1.present != nullptr;
    if (p->condition2.present && !p->condition1.present) {
        set_err(err, errlen, "condition2 needs condition1");
        return LSB_ERR_ARGUMENT;
    }
    if (g->conditions && g->bs * g->bs > kMaxCondCells) {
        set_err(err, errlen, "conditions support block_size <= 31");
        return LSB_ERR_ARGUMENT;
    }
    const int64_t np = static_cast<int64_t>(g->W + 2) * (g->W + 2);
    if (np > 65535) {
        set_err(err, errlen, "radius + buffer must be <= 125 (window of at most 251 x 251 cells)");
        return LSB_ERR_ARGUMENT;
    }
    if (g->NL > (int64_t(1) << 30)) {
        set_err(err, errlen, "too many target blocks");
        return LSB_ERR_ARGUMENT;
    }
    if (p->precision != LSB_PREC_FP64 && p->precision != LSB_PREC_FP32_REFINE) {
        set_err(err, errlen, "precision must be LSB_PREC_FP64 or LSB_PREC_FP32_REFINE");
        return LSB_ERR_ARGUMENT;
    }
    if (p->edge_weights != LSB_EDGE_AVERAGE && p->edge_weights != LSB_EDGE_SERIES) {
        set_err(err, errlen, "edge_weights must be LSB_EDGE_AVERAGE or LSB_EDGE_SERIES");
        return LSB_ERR_ARGUMENT;
    }
    return LSB_OK;
}

// ---------------------------------------------------------------------------
// Kernel variants and the arena layout.
// ---------------------------------------------------------------------------
struct Variant {
    int nt;       // threads per CTA
    int pc;       // preconditioner (resolved)
    bool dbl;     // inner solve in double
    bool mg;      // multigrid compiled in
    bool refine;  // FP64 refinement around the inner solve
    bool four;
};

// ---------------------------------------------------------------------------
// Tuning table: choices for parameters left on auto, per window shape and
// arithmetic (filled by lsb_tune_set, e.g. from an autotuning run).
// ---------------------------------------------------------------------------
struct TuneKey {
    int W, four, edge, prec;
    bool operator<(const TuneKey &o) const {
        if (W != o.W) return W < o.W;
        if (four != o.four) return four < o.four;
        if (edge != o.edge) return edge < o.edge;
        return prec < o.prec;
    }
};
struct TuneVal {
    int pc, nt;
};
std::mutex g_tune_mutex;
std::map<TuneKey, TuneVal> g_tune;
std::atomic<uint64_t> g_tune_generation{0};  // part of the graph key: a new choice is a new launch sequence

bool tune_lookup(const lsb_omni_params *p, int W, TuneVal *out) {
    std::lock_guard<std::mutex> lock(g_tune_mutex);
    auto it = g_tune.find(TuneKey{W, p->four_neighbors != 0, p->edge_weights, p->precision});
    if (it == g_tune.end()) return false;
    *out = it->second;
    return true;
}

Variant choose_variant(const lsb_omni_params *p, const Geom &g) {
    Variant v;
    v.four = p->four_neighbors != 0;
    v.dbl = p->precision == LSB_PREC_FP64;
    v.refine = !v.dbl;
    int pc = p->preconditioner;
    int nt = p->threads_per_window;
    TuneVal tv;
    const auto valid_nt = [](int t) { return t == 128 || t == 256 || t == 512; };
    if ((pc == LSB_PC_AUTO || !valid_nt(nt)) && tune_lookup(p, g.W, &tv)) {
        if (pc == LSB_PC_AUTO) pc = tv.pc;
        if (!valid_nt(nt)) nt = tv.nt;
    }
    if (pc == LSB_PC_AUTO) pc = v.dbl ? LSB_PC_JACOBI : LSB_PC_MG;
    v.pc = pc;
    v.mg = pc == LSB_PC_MG;
    if (!valid_nt(nt)) {
        const int np = (g.W + 2) * (g.W + 2);
        nt = np <= 1200 ? 256 : 512;
    }
    v.nt = nt;
    return v;
}

#ifdef LSB_PHASE_TIMERS
constexpr size_t kStaticSmem = 3072;  // the window kernel's static shared memory with the phase counters
#else
constexpr size_t kStaticSmem = 2048;  // the window kernel's static shared memory, with room to spare
#endif

// H x Wd: the largest box the launch solves (a window, or the largest raster of a batch: every level of a
// smaller box fits the arrays of the larger); raster: the finite-ground arrays of the advanced mode.
ArenaLayout make_layout(const Variant &v, int H, int Wd, size_t smem_budget, bool grad, bool raster = false) {
    ArenaLayout L;
    std::memset(&L, 0, sizeof L);
    const size_t np = static_cast<size_t>(H + 2) * (Wd + 2);
    const size_t ts = v.dbl ? 8 : 4;
    struct Item {
        int arr;
        size_t bytes;
    };
    std::vector<Item> items;  // in smem priority order
    items.push_back({AR_ULIST, np * (raster ? 4 : 2)});  // u16 indices for windows, u32 for whole rasters
    items.push_back({AR_GT, np * ts});
    items.push_back({AR_R, np * ts});
    items.push_back({AR_INVD, np * ts});
    // P, Z, Q, D adjacent: between inner solves they are dead and hold the FP64 residual's staged copies
    items.push_back({AR_P, np * ts});
    if (v.mg) items.push_back({AR_Z, np * ts});
    items.push_back({AR_Q, np * ts});
    const bool has_d = !(v.dbl && !v.refine);
    if (has_d) items.push_back({AR_D, np * ts});
    if (v.mg) {
        const int nlev = mg_levels(H, Wd);
        int h = H, w = Wd;
        for (int l = 1; l < nlev; ++l) {
            h = coarse_dim(h);
            w = coarse_dim(w);
            const size_t npl = static_cast<size_t>(h + 2) * (w + 2);
            for (int k = 0; k < LV_COUNT; ++k) items.push_back({AR_LEVEL + (l - 1) * LV_COUNT + k, npl * ts});
        }
        items.push_back({AR_DENSE, static_cast<size_t>(kNcMax) * (kNcMax + 2) * 8});  // + pivot column, diagonal
    }
    if (raster) items.push_back({AR_FGT, np * ts});
    items.push_back({AR_MASK, np});
    if (!has_d) items.push_back({AR_X64, np * 8});  // the solution is the iterate: keep it close
    if (has_d) items.push_back({AR_X64, np * 8});
    items.push_back({AR_G64, np * 8});
    items.push_back({AR_B64, np * 8});
    if (raster) items.push_back({AR_FG64, np * 8});
    if (grad) {
        items.push_back({AR_V64, np * 8});
        items.push_back({AR_CW, np * 8});
        items.push_back({AR_DG64, np * 8});
    }
    size_t so = 0, go = 0;
    for (const Item &it : items) {
        const size_t b = align_up(it.bytes, 16);
        if (so + b <= smem_budget) {
            L.off[it.arr] = static_cast<uint32_t>(so);
            so += b;
        } else {
            L.off[it.arr] = static_cast<uint32_t>(go) | 0x80000000u;
            go += b;
        }
    }
    L.smem_bytes = static_cast<uint32_t>(so);
    L.gmem_bytes = static_cast<uint32_t>(align_up(go));
    L.hot = 1;
    for (const Item &it : items)
        if (hot_array(it.arr) && (L.off[it.arr] & 0x80000000u)) L.hot = 0;
    // the node currents read the FP64 conductance and potentials at every neighbour: when those sit in global
    // scratch, the span from the stencil conductances to the mask (solver vectors, levels, coarsest inverse: dead
    // by then) holds copies of both if it is large enough
    L.stage = kNoStage;
    L.rstage = kNoStage;
    const bool g_global = (L.off[AR_G64] & 0x80000000u) || (L.off[AR_X64] & 0x80000000u);
    if (L.hot && g_global) {
        // the span of P, Z, Q, D (consecutive items, all in shared memory when hot)
        size_t span = 0;
        for (const Item &it : items)
            if (it.arr == AR_P || it.arr == AR_Z || it.arr == AR_Q || it.arr == AR_D) span += align_up(it.bytes, 16);
        if (span >= 2 * np * 8) L.rstage = L.off[AR_P];
    }
    if (L.hot && g_global && !(L.off[AR_MASK] & 0x80000000u) && L.off[AR_MASK] > L.off[AR_GT] &&
        L.off[AR_MASK] - L.off[AR_GT] >= 2 * np * 8)
        L.stage = L.off[AR_GT];
    return L;
}

// ---------------------------------------------------------------------------
// Kernel dispatch.
// ---------------------------------------------------------------------------
KernelFn pick(const Variant &v, bool hot) {
    if (v.nt == 128) return pick_windows_128_hot(v.four, v.dbl, v.mg);  // (only with a shared-memory layout)
    if (v.nt == 256)
        return hot ? pick_windows_256_hot(v.four, v.dbl, v.mg) : pick_windows_256_gen(v.four, v.dbl, v.mg);
    return hot ? pick_windows_512_hot(v.four, v.dbl, v.mg) : pick_windows_512_gen(v.four, v.dbl, v.mg);
}

struct DeviceInfo {
    int dev = -1, sms = 0;
    size_t smem_optin = 0, smem_sm = 0;
};

cudaError_t device_info(DeviceInfo *d) {
    cudaError_t e = cudaGetDevice(&d->dev);
    if (e != cudaSuccess) return e;
    int v = 0;
    e = cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, d->dev);
    if (e != cudaSuccess) return e;
    d->sms = v;
    e = cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, d->dev);
    if (e != cudaSuccess) return e;
    d->smem_optin = static_cast<size_t>(v);
    e = cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerMultiprocessor, d->dev);
    if (e != cudaSuccess) return e;
    d->smem_sm = static_cast<size_t>(v);
    return cudaSuccess;
}

// ---------------------------------------------------------------------------
// Workspace plan.
// ---------------------------------------------------------------------------
struct Plan {
    Geom g;
    Variant v;
    ArenaLayout lay;
    KernelFn kern;
    int grid;           // persistent CTAs
    int64_t batch;      // windows per batch
    int nbatches;
    int nparts;         // scan blocks
    // workspace offsets
    size_t o_amps, o_tindex, o_targets, o_part, o_count, o_queue, o_err, o_stat, o_condv, o_corr, o_corrwin,
        o_corrstat, o_cur, o_fp, o_gs, o_devstats, o_timers, o_jw, total;
    bool grad;
};

int make_plan(int64_t nx, int64_t ny, const lsb_omni_params *p, Plan *pl, char *err, size_t errlen,
              bool grad = false) {
    int rc = make_geom(nx, ny, p, &pl->g, err, errlen);
    if (rc) return rc;
    pl->grad = grad;
    if (grad) {
        // the gradient windows of a batch (resistance, source) use the two window slots
        pl->g.fp = true;
    }
    const Geom &g = pl->g;
    pl->v = choose_variant(p, g);
    DeviceInfo di;
    LSB_CK(device_info(&di));
    const size_t budget = di.smem_optin > kStaticSmem ? di.smem_optin - kStaticSmem : 0;
    if (pl->v.nt == 128) {
        // four windows per SM: each CTA gets a quarter of the SM's shared memory (less the per-CTA reserve); a
        // window whose solver arrays do not fit runs on 256 threads instead
        const size_t quarter = di.smem_sm / 4, reserve = 1024 + kStaticSmem;
        pl->lay = make_layout(pl->v, g.W, g.W, quarter > reserve ? quarter - reserve : 0, grad);
        if (!pl->lay.hot) pl->v.nt = 256;
    }
    if (pl->v.nt != 128) pl->lay = make_layout(pl->v, g.W, g.W, budget, grad);
    pl->kern = pick(pl->v, pl->lay.hot != 0);
    LSB_CK(cudaFuncSetAttribute(reinterpret_cast<const void *>(pl->kern),
                                cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(pl->lay.smem_bytes)));
    int per_sm = 0;
    LSB_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pl->kern, pl->v.nt, pl->lay.smem_bytes));
    if (per_sm < 1) {
        set_err(err, errlen, "the window kernel does not fit on an SM (%u bytes of shared memory)", pl->lay.smem_bytes);
        return LSB_ERR_ARGUMENT;
    }
    const int64_t NL = std::max<int64_t>(g.NL, 1);
    const size_t per_window = static_cast<size_t>(g.W) * g.W * 8 * (g.fp ? 2 : 1);
    const double lim = p->memory_limit > 0 ? p->memory_limit : 4.0 * (1 << 30);
    int64_t batch = static_cast<int64_t>(lim / static_cast<double>(per_window));
    batch = std::max<int64_t>(1, std::min<int64_t>(batch, NL));
    pl->batch = batch;
    pl->nbatches = static_cast<int>((NL + batch - 1) / batch);
    pl->grid = static_cast<int>(std::min<int64_t>(static_cast<int64_t>(di.sms) * per_sm, std::max<int64_t>(batch, 2)));
    pl->nparts = static_cast<int>((NL + kScanBlock - 1) / kScanBlock);
    size_t o = 0;
    auto take = [&](size_t bytes) {
        const size_t r = o;
        o += align_up(std::max<size_t>(bytes, 1));
        return r;
    };
    pl->o_amps = take(NL * 8);
    pl->o_tindex = take(NL * 4);
    pl->o_targets = take(NL * 4);
    pl->o_part = take((pl->nparts + 1) * 4);
    pl->o_count = take(4);
    pl->o_queue = take((pl->nbatches + 1) * 4);
    pl->o_err = take(4);
    pl->o_stat = take(NL * 2 * sizeof(WinStat));
    pl->o_condv = take(g.conditions ? NL * 16 : 0);
    pl->o_corr = take(g.correct ? static_cast<size_t>(g.W) * g.W * 8 : 0);
    pl->o_corrwin = take(g.correct ? static_cast<size_t>(g.W) * g.W * 16 : 0);
    pl->o_corrstat = take(2 * sizeof(WinStat));
    pl->o_cur = take(static_cast<size_t>(batch) * g.W * g.W * 8);
    pl->o_fp = take(g.fp ? static_cast<size_t>(batch) * g.W * g.W * 8 : 0);
    pl->o_gs = take(static_cast<size_t>(pl->grid) * pl->lay.gmem_bytes);
    pl->o_devstats = take(sizeof(DevStats));
    pl->o_timers = take(sizeof(unsigned long long) * 32);  // >= PH_COUNT
    pl->o_jw = take(grad ? NL * 8 : 0);
    pl->total = o;
    return LSB_OK;
}

SolveParams solve_params(const lsb_omni_params *p, int pc) {
    SolveParams sp;
    sp.tol = p->tol > 0 ? p->tol : 1e-12;
    sp.inner_tol = p->precision == LSB_PREC_FP64 ? sp.tol : 1e-4;
    sp.max_iter = p->max_iter > 0 ? p->max_iter : 20000;
    sp.max_outer = 12;
    sp.pc = pc;
    sp.omega = 0.9f;
    sp.omega_c = 0.7f;
    return sp;
}

// ---------------------------------------------------------------------------
// Graph cache: the launch sequence of a call, keyed by everything it reads.
// ---------------------------------------------------------------------------
struct GraphKey {
    const void *ptrs[8];
    int64_t nx, ny;
    lsb_omni_params p;
    size_t ws_bytes;
    void *stream;
    int dev;
    uint64_t tune_generation;
    bool operator==(const GraphKey &o) const { return std::memcmp(this, &o, sizeof *this) == 0; }
};
struct GraphEntry {
    GraphKey key;
    cudaGraphExec_t exec;
    int64_t launches;
};
std::mutex g_graph_mutex;
std::vector<GraphEntry> g_graphs;
constexpr size_t kMaxGraphs = 16;

// ---------------------------------------------------------------------------
// The launch sequence.
// ---------------------------------------------------------------------------
int enqueue(const Plan &pl, const double *res, const double *src, const lsb_omni_params *p, double *cur, double *fpm,
            double *norm, char *ws, cudaStream_t s, char *err, size_t errlen, cudaEvent_t *ev = nullptr) {
    const Geom &g = pl.g;
    const int64_t n = g.nx * g.ny;
    int64_t launches = 0;
    if (!p->accumulate) {
        LSB_CK(cudaMemsetAsync(cur, 0, n * 8, s));
        if (g.fp) LSB_CK(cudaMemsetAsync(fpm, 0, n * 8, s));
    }
    LSB_CK(cudaMemsetAsync(ws + pl.o_count, 0, 4, s));
    LSB_CK(cudaMemsetAsync(ws + pl.o_queue, 0, (pl.nbatches + 1) * 4, s));
    LSB_CK(cudaMemsetAsync(ws + pl.o_err, 0, 4, s));
    double *amps = reinterpret_cast<double *>(ws + pl.o_amps);
    int *tindex = reinterpret_cast<int *>(ws + pl.o_tindex), *targets = reinterpret_cast<int *>(ws + pl.o_targets);
    int *part = reinterpret_cast<int *>(ws + pl.o_part), *count = reinterpret_cast<int *>(ws + pl.o_count);
    int *queue = reinterpret_cast<int *>(ws + pl.o_queue), *errf = reinterpret_cast<int *>(ws + pl.o_err);
    WinStat *stat = reinterpret_cast<WinStat *>(ws + pl.o_stat);
    LSB_CK(cudaMemsetAsync(stat, 0, std::max<int64_t>(g.NL, 1) * 2 * sizeof(WinStat), s));
    if (g.NL > 0) {
        const int nb = static_cast<int>((g.NL + 255) / 256);
        k_lattice_amps<<<nb, 256, 0, s>>>(src, g.nx, g.ny, g.bs, g.br, g.nbx, g.nby, amps);
        k_scan_count<<<pl.nparts, kScanBlock, 0, s>>>(amps, g.NL, part);
        k_scan_offsets<<<1, 1024, 0, s>>>(part, pl.nparts, count);
        k_scan_write<<<pl.nparts, kScanBlock, 0, s>>>(amps, g.NL, part, tindex, targets);
        launches += 4;
        LSB_CK(cudaGetLastError());
    }
    KArgs a;
    std::memset(&a, 0, sizeof a);
    a.res = res;
    a.src = src;
    a.nx = g.nx;
    a.ny = g.ny;
    a.R = g.R;
    a.D = g.D;
    a.W = g.W;
    a.bs = g.bs;
    a.br = g.br;
    a.nbx = g.nbx;
    a.nby = g.nby;
    a.ric = p->resistance_is_conductance != 0;
    a.series = p->edge_weights == LSB_EDGE_SERIES;
    a.four = p->four_neighbors != 0;
    a.fp = g.fp;
    a.correct = g.correct;
    const lsb_omni_condition *cs[2] = {&p->condition1, &p->condition2};
    for (int k = 0; k < 2; ++k) {
        a.cond_present[k] = cs[k]->present;
        a.cond_future[k] = cs[k]->future;
        a.cond_equal[k] = cs[k]->equal != 0;
        a.cond_lo[k] = cs[k]->lower;
        a.cond_hi[k] = cs[k]->upper;
    }
    a.cond_val = g.conditions ? reinterpret_cast<const double *>(ws + pl.o_condv) : nullptr;
    a.count_ptr = count;
    a.targets = targets;
    a.lat_amps = amps;
    a.corr = g.correct ? reinterpret_cast<const double *>(ws + pl.o_corr) : nullptr;
    a.gscratch = ws + pl.o_gs;
    a.lay = pl.lay;
#ifdef LSB_PHASE_TIMERS
    a.timers = reinterpret_cast<unsigned long long *>(ws + pl.o_timers);
    LSB_CK(cudaMemsetAsync(a.timers, 0, sizeof(unsigned long long) * 30, s));
#endif
    a.sp = solve_params(p, pl.v.pc);
    if (g.conditions && g.NL > 0) {
        k_block_cond<<<static_cast<int>((g.NL + 127) / 128), 128, 0, s>>>(
            a, reinterpret_cast<double *>(ws + pl.o_condv), errf);
        ++launches;
        LSB_CK(cudaGetLastError());
    }
    if (g.correct) {
        KArgs c = a;
        c.mode = 1;
        int nsrc = 0;
        for (int y = 0; y < g.W; ++y)
            for (int x = 0; x < g.W; ++x)
                if ((y - g.D) * (y - g.D) + (x - g.D) * (x - g.D) <= g.R * g.R) ++nsrc;
        c.n_corr_sources = nsrc;
        c.cur_win = reinterpret_cast<double *>(ws + pl.o_corrwin);
        c.stat = reinterpret_cast<WinStat *>(ws + pl.o_corrstat);
        c.queue = queue + pl.nbatches;
        c.correct = 0;
        pl.kern<<<2, pl.v.nt, pl.lay.smem_bytes, s>>>(c);
        k_corr_ratio<<<1, 1024, 0, s>>>(c.cur_win, c.stat, g.W, g.bs, reinterpret_cast<double *>(ws + pl.o_corr));
        launches += 2;
        LSB_CK(cudaGetLastError());
    }
    a.cur_win = reinterpret_cast<double *>(ws + pl.o_cur);
    a.fp_win = g.fp ? reinterpret_cast<double *>(ws + pl.o_fp) : nullptr;
    a.stat = stat;
    a.batch_size = static_cast<int>(pl.batch);
    const int64_t t0 = std::max<int64_t>(p->target_begin, 0);
    const int64_t t1 = p->target_end > 0 ? std::min<int64_t>(p->target_end, g.NL) : g.NL;
    a.target_end = p->target_end > 0 ? static_cast<int>(t1) : 0;
    const int nb = t1 > t0 ? static_cast<int>((t1 - t0 + pl.batch - 1) / pl.batch) : 0;
    const dim3 gg(static_cast<unsigned>((g.nx + kGatherTX - 1) / kGatherTX),
                  static_cast<unsigned>((g.ny + kGatherTY - 1) / kGatherTY));
    for (int b = 0; b < nb && g.NL > 0; ++b) {
        a.batch_start = static_cast<int>(t0 + b * pl.batch);
        a.queue = queue + b;
        if (ev) LSB_CK(cudaEventRecord(ev[2 * b], s));
        pl.kern<<<pl.grid, pl.v.nt, pl.lay.smem_bytes, s>>>(a);
        if (ev) LSB_CK(cudaEventRecord(ev[2 * b + 1], s));
        k_gather<<<gg, kGatherTX * kGatherTY, 0, s>>>(a, tindex, cur, g.fp ? fpm : nullptr);
        launches += 2;
        LSB_CK(cudaGetLastError());
    }
    if ((norm || p->mask_nodata) && p->target_end <= 0) {
        k_finish<<<static_cast<int>((n + 255) / 256), 256, 0, s>>>(res, n, cur, g.fp ? fpm : nullptr, norm,
                                                                  p->mask_nodata);
        ++launches;
        LSB_CK(cudaGetLastError());
    }
    k_stats<<<1, 1024, 0, s>>>(stat, count, 2, reinterpret_cast<DevStats *>(ws + pl.o_devstats));
    ++launches;
    LSB_CK(cudaGetLastError());
    g_launches = launches;
    return LSB_OK;
}

}  // namespace
}  // namespace lsb

using namespace lsb;

// ---------------------------------------------------------------------------
// Raster batches (advanced mode).
// ---------------------------------------------------------------------------
constexpr int kMaxRasterSide = 1024;  // nine multigrid levels; padded indices below 2^22

struct RasterPlan {
    Variant v;
    ArenaLayout lay;
    KernelFn kern;
    int grid;
    int64_t n, cells;
    std::vector<int64_t> off;
    std::vector<int> order;
    size_t o_off, o_nx, o_ny, o_order, o_queue, o_count, o_stat, o_devstats, o_gs, total;
};

int raster_plan(int64_t n, const int32_t *nx, const int32_t *ny, const lsb_raster_params *p, RasterPlan *pl,
                char *err, size_t errlen) {
    if (!p || !nx || !ny || n < 1 || n > (1 << 30)) {
        set_err(err, errlen, "expected at least one raster, its sizes and parameters");
        return LSB_ERR_ARGUMENT;
    }
    if (p->precision != LSB_PREC_FP64 && p->precision != LSB_PREC_FP32_REFINE) {
        set_err(err, errlen, "precision must be LSB_PREC_FP64 or LSB_PREC_FP32_REFINE");
        return LSB_ERR_ARGUMENT;
    }
    int H = 1, Wd = 1;
    pl->n = n;
    pl->off.resize(static_cast<size_t>(n));
    pl->cells = 0;
    for (int64_t k = 0; k < n; ++k) {
        if (nx[k] < 1 || ny[k] < 1 || nx[k] > kMaxRasterSide || ny[k] > kMaxRasterSide) {
            set_err(err, errlen, "raster %lld is %d x %d: sides must be 1..%d", static_cast<long long>(k), ny[k],
                    nx[k], kMaxRasterSide);
            return LSB_ERR_ARGUMENT;
        }
        pl->off[k] = pl->cells;
        pl->cells += static_cast<int64_t>(nx[k]) * ny[k];
        H = std::max<int>(H, ny[k]);
        Wd = std::max<int>(Wd, nx[k]);
    }
    // the largest rasters first, so that the persistent CTAs finish together
    pl->order.resize(static_cast<size_t>(n));
    for (int64_t k = 0; k < n; ++k) pl->order[k] = static_cast<int>(k);
    std::stable_sort(pl->order.begin(), pl->order.end(), [&](int a, int b) {
        return static_cast<int64_t>(nx[a]) * ny[a] > static_cast<int64_t>(nx[b]) * ny[b];
    });
    Variant &v = pl->v;
    v.four = p->four_neighbors != 0;
    v.dbl = p->precision == LSB_PREC_FP64;
    v.refine = !v.dbl;
    v.mg = !v.dbl;
    v.pc = v.dbl ? LSB_PC_JACOBI : LSB_PC_MG;
    v.nt = 512;
    DeviceInfo di;
    LSB_CK(device_info(&di));
    size_t budget = di.smem_optin > kStaticSmem ? di.smem_optin - kStaticSmem : 0;
    if (p->smem_limit_kb > 0) budget = std::min<size_t>(budget, static_cast<size_t>(p->smem_limit_kb) << 10);
    pl->lay = make_layout(v, H, Wd, budget, false, true);
    pl->kern = pick_rasters(pl->lay.hot != 0, v.four, v.dbl);
    LSB_CK(cudaFuncSetAttribute(reinterpret_cast<const void *>(pl->kern),
                                cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(pl->lay.smem_bytes)));
    int per_sm = 0;
    LSB_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pl->kern, v.nt, pl->lay.smem_bytes));
    if (per_sm < 1) {
        set_err(err, errlen, "the raster kernel does not fit on an SM (%u bytes of shared memory)", pl->lay.smem_bytes);
        return LSB_ERR_ARGUMENT;
    }
    const double lim = p->memory_limit > 0 ? p->memory_limit : 8.0 * (1 << 30);
    const int64_t by_mem = std::max<int64_t>(1, static_cast<int64_t>(lim / std::max<double>(pl->lay.gmem_bytes, 1)));
    pl->grid = static_cast<int>(std::min<int64_t>(std::min<int64_t>(static_cast<int64_t>(di.sms) * per_sm, n), by_mem));
    size_t o = 0;
    auto take = [&](size_t bytes) {
        const size_t r = o;
        o += align_up(std::max<size_t>(bytes, 1));
        return r;
    };
    pl->o_off = take(n * 8);
    pl->o_nx = take(n * 4);
    pl->o_ny = take(n * 4);
    pl->o_order = take(n * 4);
    pl->o_queue = take(4);
    pl->o_count = take(4);
    pl->o_stat = take(n * sizeof(WinStat));
    pl->o_devstats = take(sizeof(DevStats));
    pl->o_gs = take(static_cast<size_t>(pl->grid) * pl->lay.gmem_bytes);
    pl->total = o;
    return LSB_OK;
}

extern "C" {

void lsb_params_default(lsb_omni_params *p) {
    std::memset(p, 0, sizeof *p);
    p->radius = 0;
    p->buffer = 0;
    p->block_size = 1;
    p->correct_artifacts = 1;
    p->edge_weights = LSB_EDGE_AVERAGE;
    p->precision = LSB_PREC_FP32_REFINE;
    p->preconditioner = LSB_PC_AUTO;
    p->tol = 1e-12;
    p->max_iter = 20000;
    p->use_graph = 1;
    p->mask_nodata = 0;
}

int lsb_omniscape_workspace_size(int64_t nx, int64_t ny, const lsb_omni_params *p, size_t *bytes) {
    Plan pl;
    char *err = nullptr;
    size_t errlen = 0;
    const int rc = make_plan(nx, ny, p, &pl, err, errlen);
    if (rc) return rc;
    *bytes = pl.total;
    return LSB_OK;
}

int lsb_omniscape(const double *resistance, const double *source, int64_t nx, int64_t ny, const lsb_omni_params *p,
                  double *current, double *flow_potential, double *normalized, void *workspace,
                  size_t workspace_bytes, lsb_omni_stats *stats, char *err, size_t errlen, void *stream) {
    Plan pl;
    int rc = make_plan(nx, ny, p, &pl, err, errlen);
    if (rc) return rc;
    if (!resistance || !source || !current) {
        set_err(err, errlen, "resistance, source and current are required");
        return LSB_ERR_ARGUMENT;
    }
    if (p->flow_potential && !flow_potential) {
        set_err(err, errlen, "flow_potential is requested but its output is NULL");
        return LSB_ERR_ARGUMENT;
    }
    if (normalized && !p->flow_potential) {
        set_err(err, errlen, "the normalised current needs the flow potential");
        return LSB_ERR_ARGUMENT;
    }
    if (!workspace || workspace_bytes < pl.total) {
        set_err(err, errlen, "workspace too small: %zu bytes needed", pl.total);
        return LSB_ERR_WORKSPACE;
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    char *ws = static_cast<char *>(workspace);
    bool graphed = false;
    if (p->use_graph && s != nullptr) {
        GraphKey key;
        std::memset(&key, 0, sizeof key);
        key.ptrs[0] = resistance;
        key.ptrs[1] = source;
        key.ptrs[2] = current;
        key.ptrs[3] = flow_potential;
        key.ptrs[4] = normalized;
        key.ptrs[5] = workspace;
        key.nx = nx;
        key.ny = ny;
        key.p = *p;
        key.ws_bytes = workspace_bytes;
        key.stream = stream;
        key.dev = 0;
        cudaGetDevice(&key.dev);
        key.tune_generation = g_tune_generation.load();
        std::lock_guard<std::mutex> lock(g_graph_mutex);
        cudaGraphExec_t exec = nullptr;
        int64_t launches = 0;
        for (auto &e : g_graphs)
            if (e.key == key) {
                exec = e.exec;
                launches = e.launches;
            }
        if (!exec) {
            LSB_CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
            rc = enqueue(pl, resistance, source, p, current, flow_potential, normalized, ws, s, err, errlen);
            cudaGraph_t graph = nullptr;
            const cudaError_t ce = cudaStreamEndCapture(s, &graph);
            if (rc) {
                if (graph) cudaGraphDestroy(graph);
                return rc;
            }
            LSB_CK(ce);
            const cudaError_t ie = cudaGraphInstantiate(&exec, graph, 0);
            cudaGraphDestroy(graph);
            LSB_CK(ie);
            launches = g_launches;
            if (g_graphs.size() >= kMaxGraphs) {
                cudaGraphExecDestroy(g_graphs.front().exec);
                g_graphs.erase(g_graphs.begin());
            }
            g_graphs.push_back({key, exec, launches});
        }
        LSB_CK(cudaGraphLaunch(exec, s));
        g_launches = launches;
        graphed = true;
    }
    std::vector<cudaEvent_t> ev;
    if (!graphed) {
        if (stats && g_time_windows) {
            ev.resize(2 * static_cast<size_t>(pl.nbatches));
            for (auto &e : ev) LSB_CK(cudaEventCreate(&e));
        }
        rc = enqueue(pl, resistance, source, p, current, flow_potential, normalized, ws, s, err, errlen,
                     ev.empty() ? nullptr : ev.data());
        if (rc) return rc;
    }
    if (stats) {
        DevStats ds;
        int hdr[2] = {0, 0};
        LSB_CK(cudaMemcpyAsync(&ds, ws + pl.o_devstats, sizeof ds, cudaMemcpyDeviceToHost, s));
        LSB_CK(cudaMemcpyAsync(&hdr[0], ws + pl.o_count, 4, cudaMemcpyDeviceToHost, s));
        LSB_CK(cudaMemcpyAsync(&hdr[1], ws + pl.o_err, 4, cudaMemcpyDeviceToHost, s));
        LSB_CK(cudaStreamSynchronize(s));
        stats->window_ms = 0.0;
        for (size_t b = 0; b + 1 < ev.size(); b += 2) {
            float ms = 0.f;
            if (hdr[0] > static_cast<int>(b / 2 * pl.batch) && cudaEventElapsedTime(&ms, ev[b], ev[b + 1]) == cudaSuccess)
                stats->window_ms += ms;
        }
        for (auto &e : ev) cudaEventDestroy(e);
        ev.clear();
#ifdef LSB_PHASE_TIMERS
        {
            unsigned long long tm[PH_COUNT];
            LSB_CK(cudaMemcpy(tm, ws + pl.o_timers, sizeof tm, cudaMemcpyDeviceToHost));
            static const char *names[PH_COUNT] = {"load", "flood", "mark", "assemble", "mg_setup", "resid64", "cg",
                                                  "vcycle", "currents", "other", "v_pre0", "v_restrict1",
                                                  "v_coarsest", "v_prolong0", "v_post0", "s_weights", "s_level1",
                                                  "s_coarser", "s_dense", "c_stage", "c_max", "ds1", "ds2+",
                                                  "dr1", "dr2+", "up1",
                                                  "up2+", "us1", "us2+"};
            double tot = 0;
            for (int k = 0; k < PH_COUNT; ++k) tot += static_cast<double>(tm[k]);
            fprintf(stderr, "[phases] windows=%d cycles/window:", hdr[0]);
            for (int k = 0; k < PH_COUNT; ++k)
                fprintf(stderr, " %s=%.0f(%.0f%%)", names[k], tm[k] / std::max(1.0, static_cast<double>(hdr[0])),
                        100.0 * tm[k] / std::max(tot, 1.0));
            unsigned long long cal[2];
            LSB_CK(cudaMemcpy(cal, ws + pl.o_timers + 30 * sizeof(unsigned long long), sizeof cal,
                              cudaMemcpyDeviceToHost));
            fprintf(stderr, " | barrier=%llu cycles, barrier+smem round trip=%llu cycles\n", cal[0], cal[1]);
        }
#endif
        stats->n_targets = hdr[0];
        stats->n_solved = ds.n_solved;
        stats->n_failed = ds.n_failed;
        stats->iters_total = ds.iters_total;
        stats->iters_max = ds.iters_max;
        stats->refine_max = ds.refine_max;
        stats->batches = pl.nbatches;
        stats->threads_per_window = pl.v.nt;
        stats->preconditioner = pl.v.pc;
        stats->worst_residual = ds.worst_residual;
        stats->unknown_iters = ds.unknown_iters;
        if (hdr[1]) {
            set_err(err, errlen, "a target block has no value of a condition (all NoData)");
            return LSB_ERR_CONDITION;
        }
        if (ds.n_failed > 0) {
            set_err(err, errlen, "%lld Omniscape window solves did not converge (worst relative residual %.3g)",
                    static_cast<long long>(ds.n_failed), ds.worst_residual);
            return LSB_ERR_NOT_CONVERGED;
        }
    }
    return LSB_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// The entry point that allocates nothing.  Its scratch is this file-scope
// device array: every GPU on which the library is loaded holds it until the
// process exits.  In host code the name below is only a stand-in for the
// array; the device address comes from cudaGetSymbolAddress, once per device.
// ---------------------------------------------------------------------------
namespace {
static __device__ __align__(256) unsigned char g_noalloc_scratch[LSB_NOALLOC_SCRATCH_BYTES];

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mutex;
void *g_noalloc_ptr[kMaxDevices] = {};

// The device address of the static scratch on the current device (set up on the first call there).
int noalloc_scratch(void **out, char *err, size_t errlen) {
    int dev = 0;
    LSB_CK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) {
        set_err(err, errlen, "device index %d out of range", dev);
        return LSB_ERR_ARGUMENT;
    }
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_ptr[dev]) {
        void *ptr = nullptr;
        LSB_CK(cudaGetSymbolAddress(&ptr, g_noalloc_scratch));
        g_noalloc_ptr[dev] = ptr;
    }
    *out = g_noalloc_ptr[dev];
    return LSB_OK;
}
}  // namespace

extern "C" {

int lsb_omniscape_noalloc(const double *resistance, const double *source, int64_t nx, int64_t ny,
                          const lsb_omni_params *p, double *current, double *flow_potential, double *normalized,
                          lsb_omni_stats *stats, char *err, size_t errlen, void *stream) {
    if (!p) {
        set_err(err, errlen, "params is NULL");
        return LSB_ERR_ARGUMENT;
    }
    // the same call as lsb_omniscape, launched directly (no graph), with the window buffers of a batch sized
    // so that the whole workspace fits the static array
    lsb_omni_params q = *p;
    q.use_graph = 0;
    const size_t cap = LSB_NOALLOC_SCRATCH_BYTES;
    Plan pl;
    int rc = make_plan(nx, ny, &q, &pl, err, errlen);
    if (rc) return rc;
    if (pl.total > cap) {
        const size_t per_window = static_cast<size_t>(pl.g.W) * pl.g.W * 8 * (pl.g.fp ? 2 : 1);
        const size_t windows = static_cast<size_t>(pl.batch) * per_window;
        const size_t fixed = pl.total - std::min(pl.total, windows);
        int64_t batch = fixed + 4 * kAlign < cap ? static_cast<int64_t>((cap - fixed - 4 * kAlign) / per_window) : 0;
        while (batch >= 1) {
            q.memory_limit = static_cast<double>(batch) * static_cast<double>(per_window);
            rc = make_plan(nx, ny, &q, &pl, err, errlen);
            if (rc) return rc;
            if (pl.total <= cap) break;
            batch = batch * 9 / 10;
        }
        if (batch < 1 || pl.total > cap) {
            set_err(err, errlen,
                    "lsb_omniscape_noalloc: this raster and window size need more than the %zu bytes of static "
                    "scratch (at least %zu); call lsb_omniscape with a workspace instead",
                    cap, fixed + per_window);
            return LSB_ERR_WORKSPACE;
        }
    }
    void *ws = nullptr;
    rc = noalloc_scratch(&ws, err, errlen);
    if (rc) return rc;
    return lsb_omniscape(resistance, source, nx, ny, &q, current, flow_potential, normalized, ws, cap, stats, err,
                         errlen, stream);
}

int lsb_omniscape_correction(int32_t radius, int32_t buffer, int32_t block_size, int32_t four_neighbors,
                             int32_t edge_weights, int64_t nx, int64_t ny, double *corr, void *workspace,
                             size_t workspace_bytes, char *err, size_t errlen, void *stream) {
    lsb_omni_params p;
    lsb_params_default(&p);
    p.radius = radius;
    p.buffer = buffer;
    p.block_size = block_size;
    p.four_neighbors = four_neighbors;
    p.edge_weights = edge_weights;
    p.precision = LSB_PREC_FP64;
    p.preconditioner = LSB_PC_JACOBI;
    // a 1 x 1 raster: no targets, only the correction windows
    Plan pl;
    int rc = make_plan(1, 1, &p, &pl, err, errlen);
    if (rc) return rc;
    const Geom &g0 = pl.g;
    (void)g0;
    // the correction's plan: W from radius/buffer; the raster size only enters through the quirk's min()
    Geom g;
    rc = make_geom(nx, ny, &p, &g, err, errlen);
    if (rc) return rc;
    const size_t need = align_up(static_cast<size_t>(g.W) * g.W * 16) + align_up(2 * sizeof(WinStat)) +
                        align_up(8) + 2 * static_cast<size_t>(pl.lay.gmem_bytes);
    if (!workspace || workspace_bytes < need) {
        set_err(err, errlen, "workspace too small: %zu bytes needed", need);
        return LSB_ERR_WORKSPACE;
    }
    char *ws = static_cast<char *>(workspace);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    KArgs c;
    std::memset(&c, 0, sizeof c);
    c.nx = nx;
    c.ny = ny;
    c.R = g.R;
    c.D = g.D;
    c.W = g.W;
    c.bs = g.bs;
    c.br = g.br;
    c.four = four_neighbors != 0;
    c.series = edge_weights == LSB_EDGE_SERIES;
    c.mode = 1;
    int nsrc = 0;
    for (int y = 0; y < g.W; ++y)
        for (int x = 0; x < g.W; ++x)
            if ((y - g.D) * (y - g.D) + (x - g.D) * (x - g.D) <= g.R * g.R) ++nsrc;
    c.n_corr_sources = nsrc;
    c.cur_win = reinterpret_cast<double *>(ws);
    c.stat = reinterpret_cast<WinStat *>(ws + align_up(static_cast<size_t>(g.W) * g.W * 16));
    int *queue = reinterpret_cast<int *>(ws + align_up(static_cast<size_t>(g.W) * g.W * 16) + align_up(2 * sizeof(WinStat)));
    c.queue = queue;
    c.gscratch = reinterpret_cast<char *>(queue) + align_up(8);
    c.lay = pl.lay;
    c.sp = solve_params(&p, pl.v.pc);
    LSB_CK(cudaMemsetAsync(queue, 0, 4, s));
    pl.kern<<<2, pl.v.nt, pl.lay.smem_bytes, s>>>(c);
    k_corr_ratio<<<1, 1024, 0, s>>>(c.cur_win, c.stat, g.W, g.bs, corr);
    LSB_CK(cudaGetLastError());
    g_launches = 2;
    return LSB_OK;
}

int lsb_omniscape_grad_workspace_size(int64_t nx, int64_t ny, const lsb_omni_params *p, size_t *bytes) {
    Plan pl;
    const int rc = make_plan(nx, ny, p, &pl, nullptr, 0, true);
    if (rc) return rc;
    *bytes = pl.total;
    return LSB_OK;
}

int lsb_omniscape_grad(const double *resistance, const double *source, const double *weight, int64_t nx, int64_t ny,
                       const lsb_omni_params *p, double *grad_resistance, double *grad_source, double *J_out,
                       void *workspace, size_t workspace_bytes, lsb_omni_stats *stats, char *err, size_t errlen,
                       void *stream) {
    if (!p) {
        set_err(err, errlen, "params is NULL");
        return LSB_ERR_ARGUMENT;
    }
    if (p->correct_artifacts && p->block_size > 1) {
        set_err(err, errlen, "the adjoint needs no block-artifact correction (block_size 1 or correct_artifacts 0)");
        return LSB_ERR_ARGUMENT;
    }
    if (p->condition1.present || p->condition2.present) {
        set_err(err, errlen, "the adjoint does not support conditions");
        return LSB_ERR_ARGUMENT;
    }
    Plan pl;
    int rc = make_plan(nx, ny, p, &pl, err, errlen, true);
    if (rc) return rc;
    if (!resistance || !source || !weight || !grad_resistance) {
        set_err(err, errlen, "resistance, source, weight and grad_resistance are required");
        return LSB_ERR_ARGUMENT;
    }
    if (!workspace || workspace_bytes < pl.total) {
        set_err(err, errlen, "workspace too small: %zu bytes needed", pl.total);
        return LSB_ERR_WORKSPACE;
    }
    const Geom &g = pl.g;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    char *ws = static_cast<char *>(workspace);
    const int64_t n = g.nx * g.ny;
    int64_t launches = 0;
    LSB_CK(cudaMemsetAsync(grad_resistance, 0, n * 8, s));
    if (grad_source) LSB_CK(cudaMemsetAsync(grad_source, 0, n * 8, s));
    LSB_CK(cudaMemsetAsync(ws + pl.o_count, 0, 4, s));
    LSB_CK(cudaMemsetAsync(ws + pl.o_queue, 0, (pl.nbatches + 1) * 4, s));
    LSB_CK(cudaMemsetAsync(ws + pl.o_err, 0, 4, s));
    double *amps = reinterpret_cast<double *>(ws + pl.o_amps);
    int *tindex = reinterpret_cast<int *>(ws + pl.o_tindex), *targets = reinterpret_cast<int *>(ws + pl.o_targets);
    int *part = reinterpret_cast<int *>(ws + pl.o_part), *count = reinterpret_cast<int *>(ws + pl.o_count);
    int *queue = reinterpret_cast<int *>(ws + pl.o_queue);
    WinStat *stat = reinterpret_cast<WinStat *>(ws + pl.o_stat);
    double *Jw = reinterpret_cast<double *>(ws + pl.o_jw);
    LSB_CK(cudaMemsetAsync(stat, 0, std::max<int64_t>(g.NL, 1) * 2 * sizeof(WinStat), s));
    if (g.NL > 0) {
        const int nb = static_cast<int>((g.NL + 255) / 256);
        k_lattice_amps<<<nb, 256, 0, s>>>(source, g.nx, g.ny, g.bs, g.br, g.nbx, g.nby, amps);
        k_scan_count<<<pl.nparts, kScanBlock, 0, s>>>(amps, g.NL, part);
        k_scan_offsets<<<1, 1024, 0, s>>>(part, pl.nparts, count);
        k_scan_write<<<pl.nparts, kScanBlock, 0, s>>>(amps, g.NL, part, tindex, targets);
        launches += 4;
        LSB_CK(cudaGetLastError());
    }
    KArgs a;
    std::memset(&a, 0, sizeof a);
    a.res = resistance;
    a.src = source;
    a.nx = g.nx;
    a.ny = g.ny;
    a.R = g.R;
    a.D = g.D;
    a.W = g.W;
    a.bs = g.bs;
    a.br = g.br;
    a.nbx = g.nbx;
    a.nby = g.nby;
    a.ric = p->resistance_is_conductance != 0;
    a.series = p->edge_weights == LSB_EDGE_SERIES;
    a.four = p->four_neighbors != 0;
    a.fp = 0;
    a.correct = 0;
    a.count_ptr = count;
    a.targets = targets;
    a.lat_amps = amps;
    a.gscratch = ws + pl.o_gs;
    a.lay = pl.lay;
    a.sp = solve_params(p, pl.v.pc);
    a.mode = 2;
    a.weight = weight;
    a.Jw = Jw;
    a.cur_win = reinterpret_cast<double *>(ws + pl.o_cur);
    a.fp_win = reinterpret_cast<double *>(ws + pl.o_fp);
    a.stat = stat;
    a.batch_size = static_cast<int>(pl.batch);
    const dim3 gg(static_cast<unsigned>((g.nx + kGatherTX - 1) / kGatherTX),
                  static_cast<unsigned>((g.ny + kGatherTY - 1) / kGatherTY));
    for (int b = 0; b < pl.nbatches && g.NL > 0; ++b) {
        a.batch_start = static_cast<int>(b * pl.batch);
        a.queue = queue + b;
        pl.kern<<<pl.grid, pl.v.nt, pl.lay.smem_bytes, s>>>(a);
        k_gather<<<gg, kGatherTX * kGatherTY, 0, s>>>(a, tindex, grad_resistance, grad_source);
        launches += 2;
        LSB_CK(cudaGetLastError());
    }
    if (J_out) {
        if (g.NL > 0) {
            k_sum_targets<<<1, 1024, 0, s>>>(Jw, count, J_out);
            ++launches;
        } else {
            LSB_CK(cudaMemsetAsync(J_out, 0, 8, s));
        }
        LSB_CK(cudaGetLastError());
    }
    k_stats<<<1, 1024, 0, s>>>(stat, count, 2, reinterpret_cast<DevStats *>(ws + pl.o_devstats));
    ++launches;
    LSB_CK(cudaGetLastError());
    g_launches = launches;
    if (stats) {
        DevStats ds;
        int cnt = 0;
        LSB_CK(cudaMemcpyAsync(&ds, ws + pl.o_devstats, sizeof ds, cudaMemcpyDeviceToHost, s));
        LSB_CK(cudaMemcpyAsync(&cnt, ws + pl.o_count, 4, cudaMemcpyDeviceToHost, s));
        LSB_CK(cudaStreamSynchronize(s));
        std::memset(stats, 0, sizeof *stats);
        stats->n_targets = cnt;
        stats->n_solved = ds.n_solved;
        stats->n_failed = ds.n_failed;
        stats->iters_total = ds.iters_total;
        stats->iters_max = ds.iters_max;
        stats->refine_max = ds.refine_max;
        stats->batches = pl.nbatches;
        stats->threads_per_window = pl.v.nt;
        stats->preconditioner = pl.v.pc;
        stats->worst_residual = ds.worst_residual;
        stats->unknown_iters = ds.unknown_iters;
        if (ds.n_failed > 0) {
            set_err(err, errlen, "%lld window solves of the adjoint did not converge (worst relative residual %.3g)",
                    static_cast<long long>(ds.n_failed), ds.worst_residual);
            return LSB_ERR_NOT_CONVERGED;
        }
    }
    return LSB_OK;
}

int64_t lsb_last_launch_count(void) { return g_launches; }

void lsb_time_window_kernels(int32_t on) { g_time_windows = on != 0; }

void lsb_raster_params_default(lsb_raster_params *p) {
    std::memset(p, 0, sizeof *p);
    p->precision = LSB_PREC_FP32_REFINE;
    p->tol = 1e-12;
    p->max_iter = 20000;
}

int lsb_rasters_workspace_size(int64_t n, const int32_t *nx, const int32_t *ny, const lsb_raster_params *p,
                               size_t *bytes) {
    RasterPlan pl;
    const int rc = raster_plan(n, nx, ny, p, &pl, nullptr, 0);
    if (rc) return rc;
    *bytes = pl.total;
    return LSB_OK;
}

int lsb_rasters(int64_t n, const int32_t *nx, const int32_t *ny, const double *conductance, const double *source,
                const double *ground, const lsb_raster_params *p, double *current, double *voltage, void *workspace,
                size_t workspace_bytes, lsb_omni_stats *stats, char *err, size_t errlen, void *stream) {
    RasterPlan pl;
    int rc = raster_plan(n, nx, ny, p, &pl, err, errlen);
    if (rc) return rc;
    if (!conductance || !source || !ground || !current || !voltage) {
        set_err(err, errlen, "conductance, source, ground, current and voltage are required");
        return LSB_ERR_ARGUMENT;
    }
    if (!workspace || workspace_bytes < pl.total) {
        set_err(err, errlen, "workspace too small: %zu bytes needed", pl.total);
        return LSB_ERR_WORKSPACE;
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    char *ws = static_cast<char *>(workspace);
    const int count = static_cast<int>(n);
    // descriptors (pageable host memory: each copy is staged before the call returns)
    LSB_CK(cudaMemcpyAsync(ws + pl.o_off, pl.off.data(), n * 8, cudaMemcpyHostToDevice, s));
    LSB_CK(cudaMemcpyAsync(ws + pl.o_nx, nx, n * 4, cudaMemcpyHostToDevice, s));
    LSB_CK(cudaMemcpyAsync(ws + pl.o_ny, ny, n * 4, cudaMemcpyHostToDevice, s));
    LSB_CK(cudaMemcpyAsync(ws + pl.o_order, pl.order.data(), n * 4, cudaMemcpyHostToDevice, s));
    LSB_CK(cudaMemcpyAsync(ws + pl.o_count, &count, 4, cudaMemcpyHostToDevice, s));
    LSB_CK(cudaMemsetAsync(ws + pl.o_queue, 0, 4, s));
    KArgs a;
    std::memset(&a, 0, sizeof a);
    a.res = conductance;
    a.src = source;
    a.gnd = ground;
    a.four = pl.v.four;
    a.cur_win = current;
    a.fp_win = voltage;
    a.stat = reinterpret_cast<WinStat *>(ws + pl.o_stat);
    a.queue = reinterpret_cast<int *>(ws + pl.o_queue);
    a.gscratch = ws + pl.o_gs;
    a.lay = pl.lay;
    lsb_omni_params q;
    lsb_params_default(&q);
    q.precision = p->precision;
    q.tol = p->tol;
    q.max_iter = p->max_iter;
    a.sp = solve_params(&q, pl.v.pc);
    a.mode = 3;
    a.ras_off = reinterpret_cast<const int64_t *>(ws + pl.o_off);
    a.ras_nx = reinterpret_cast<const int *>(ws + pl.o_nx);
    a.ras_ny = reinterpret_cast<const int *>(ws + pl.o_ny);
    a.ras_order = reinterpret_cast<const int *>(ws + pl.o_order);
    a.n_rasters = count;
    pl.kern<<<pl.grid, pl.v.nt, pl.lay.smem_bytes, s>>>(a);
    LSB_CK(cudaGetLastError());
    k_stats<<<1, 1024, 0, s>>>(a.stat, reinterpret_cast<const int *>(ws + pl.o_count), 1,
                               reinterpret_cast<DevStats *>(ws + pl.o_devstats));
    LSB_CK(cudaGetLastError());
    g_launches = 2;
    if (stats) {
        DevStats ds;
        LSB_CK(cudaMemcpyAsync(&ds, ws + pl.o_devstats, sizeof ds, cudaMemcpyDeviceToHost, s));
        LSB_CK(cudaStreamSynchronize(s));
        std::memset(stats, 0, sizeof *stats);
        stats->n_targets = n;
        stats->n_solved = ds.n_solved;
        stats->n_failed = ds.n_failed;
        stats->iters_total = ds.iters_total;
        stats->iters_max = ds.iters_max;
        stats->refine_max = ds.refine_max;
        stats->batches = 1;
        stats->threads_per_window = pl.v.nt;
        stats->preconditioner = pl.v.pc;
        stats->worst_residual = ds.worst_residual;
        stats->unknown_iters = ds.unknown_iters;
        if (ds.n_failed > 0) {
            set_err(err, errlen, "%lld raster solves did not converge (worst relative residual %.3g)",
                    static_cast<long long>(ds.n_failed), ds.worst_residual);
            return LSB_ERR_NOT_CONVERGED;
        }
    }
    return LSB_OK;
}

int lsb_tune_set(int32_t window_width, int32_t four_neighbors, int32_t edge_weights, int32_t precision,
                 int32_t preconditioner, int32_t threads_per_window) {
    if (window_width < 1 || (preconditioner != LSB_PC_JACOBI && preconditioner != LSB_PC_MG) ||
        (threads_per_window != 128 && threads_per_window != 256 && threads_per_window != 512))
        return LSB_ERR_ARGUMENT;
    {
        std::lock_guard<std::mutex> lock(g_tune_mutex);
        g_tune[TuneKey{window_width, four_neighbors != 0, edge_weights, precision}] =
            TuneVal{preconditioner, threads_per_window};
    }
    ++g_tune_generation;
    return LSB_OK;
}

int lsb_tune_get(int32_t window_width, int32_t four_neighbors, int32_t edge_weights, int32_t precision,
                 int32_t *preconditioner, int32_t *threads_per_window) {
    std::lock_guard<std::mutex> lock(g_tune_mutex);
    auto it = g_tune.find(TuneKey{window_width, four_neighbors != 0, edge_weights, precision});
    if (it == g_tune.end()) return 0;
    if (preconditioner) *preconditioner = it->second.pc;
    if (threads_per_window) *threads_per_window = it->second.nt;
    return 1;
}

void lsb_tune_clear(void) {
    {
        std::lock_guard<std::mutex> lock(g_tune_mutex);
        g_tune.clear();
    }
    ++g_tune_generation;
}

const char *lsb_version(void) { return "landschaft_b200 0.1 (sm_100a)"; }

}  // extern "C"
