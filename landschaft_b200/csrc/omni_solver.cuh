// omni_solver.cuh -- one window on one CTA: load, flood fill, assembly,
// preconditioned CG (Jacobi or geometric multigrid; FP64, or FP32 inside FP64
// iterative refinement), node currents.  See omni_device.cuh for the layout.
#pragma once

#include <math_constants.h>

#include <type_traits>

#include "omni_device.cuh"

namespace lsb {

// Everything a window kernel reads; passed by value (param space).
struct KArgs {
    const double *res;  // resistance (or conductance), ny x nx
    const double *src;  // sources, ny x nx
    int64_t nx, ny;
    int R, D, W, bs, br, nbx, nby;
    int ric, series, four, fp, correct;
    // conditions
    const double *cond_present[2];
    const double *cond_future[2];
    int cond_equal[2];
    double cond_lo[2], cond_hi[2];
    const double *cond_val;  // per target: 2 block values
    // targets
    const int *count_ptr;   // number of targets (device)
    const int *targets;     // lattice ids of the targets, in lattice order
    const double *lat_amps; // per lattice point: the block's source sum
    const double *corr;     // W x W correction factors, or null
    // outputs of a batch
    double *cur_win;  // batch slots of W*W doubles (pitch w of each window); raster solves: the current maps
    double *fp_win;   // raster solves: the voltage maps
    WinStat *stat;    // per target: [land, flow]
    int *queue;       // work counter of this launch
    int batch_start, batch_size;
    int target_end;   // > 0: targets from target_end on are left out (a streamed range)
    // working memory
    char *gscratch;   // gridDim.x slices of lay.gmem_bytes
    ArenaLayout lay;
    SolveParams sp;
    int mode;         // 0 windows of targets, 1 the two correction windows
    double n_corr_sources;  // cells within radius of the correction disk (mode 1)
    // adjoint (mode 2): weights of J on the map; per-window gradient slots
    const double *weight;
    // per-phase cycle counters (builds with LSB_PHASE_TIMERS only)
    unsigned long long *timers;
    double *Jw;  // mode 2: J's share of every target
    // raster solves (advanced mode): ground rasters, and per raster its offset in the packed maps, its width and
    // height; the queue visits rasters in `order`
    const double *gnd;
    const int64_t *ras_off;
    const int *ras_nx, *ras_ny, *ras_order;
    int n_rasters;
};

using KernelFn = void (*)(const KArgs);

// Phases of a window solve, for the cycle counters of profiling builds.
enum Phase : int { PH_LOAD = 0, PH_FLOOD, PH_MARK, PH_ASSEMBLE, PH_MG_SETUP, PH_RESID, PH_CG, PH_VCYCLE, PH_CURRENTS,
                   PH_OTHER, PH_V_PRE0, PH_V_RESTRICT1, PH_V_COARSEST, PH_V_PROLONG0, PH_V_POST0,
                   // multigrid set-up: level-0 weights, level-1 Galerkin product, coarser products, coarsest inverse
                   PH_S_W, PH_S_L1, PH_S_LC, PH_S_DENSE,
                   // node currents: staging the FP64 arrays, the branch maxima (the rest is PH_CURRENTS)
                   PH_C_STAGE, PH_C_MAX,
                   // levels 1 and 2 (deeper levels count as 2): down smoothing, restriction; up prolongation, smoothing
                   PH_L_DS, PH_L_DR = PH_L_DS + 2, PH_L_UP = PH_L_DR + 2, PH_L_US = PH_L_UP + 2,
                   PH_COUNT = PH_L_US + 2 };
static_assert(PH_COUNT <= 30, "two timer slots are calibration");

template <typename X>
__device__ __forceinline__ X *arena_ptr(const ArenaLayout &L, int a, char *sm, char *gm) {
    const uint32_t o = L.off[a];
    return reinterpret_cast<X *>((o & 0x80000000u) ? gm + (o & 0x7fffffffu) : sm + o);
}

// Scalar type traits for the inner solve.
template <typename T>
struct Sentinel;
template <>
struct Sentinel<float> {
    __device__ static float neg() { return -CUDART_INF_F; }
    __device__ static float pos() { return CUDART_INF_F; }
};
template <>
struct Sentinel<double> {
    __device__ static double neg() { return -CUDART_INF; }
    __device__ static double pos() { return CUDART_INF; }
};

__device__ __forceinline__ float tmax(float a, float b) { return fmaxf(a, b); }
__device__ __forceinline__ double tmax(double a, double b) { return fmax(a, b); }

// Block-wide ordered compaction of flags over [0, n): out[k] = i of the k-th
// flagged i (increasing).  Returns the count.  scan: shared, >= 33 ints.
template <int NT, typename I, typename F>
__device__ __forceinline__ int block_compact(int n, F flag, I *out, int *scan) {
    constexpr int NW = NT / 32;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int base = 0;
    for (int c0 = 0; c0 < n; c0 += NT) {
        const int i = c0 + threadIdx.x;
        const bool f = i < n && flag(i);
        const unsigned m = __ballot_sync(0xffffffffu, f);
        if (lane == 0) scan[warp] = __popc(m);
        __syncthreads();
        int before = 0, total = 0;
#pragma unroll
        for (int k = 0; k < NW; ++k) {
            const int c = scan[k];
            before += k < warp ? c : 0;
            total += c;
        }
        if (f) out[base + before + __popc(m & ((1u << lane) - 1u))] = static_cast<I>(i);
        base += total;
        __syncthreads();
    }
    return base;
}

// ---------------------------------------------------------------------------
// The solver of one window.
// ---------------------------------------------------------------------------
// Arrays a window keeps in shared memory whenever the layout's HOT flag is set: all but the FP64 window arrays.
__host__ __device__ constexpr bool hot_array(int k) {
    return !(k == AR_X64 || k == AR_G64 || k == AR_B64 || k == AR_V64 || k == AR_CW || k == AR_DG64 || k == AR_FG64);
}

// HOT: every hot array of the layout is in shared memory, so their pointers derive from the shared-memory base and
// compile to 32-bit shared addressing (else each pointer is chosen at run time and addressed generically).
// ADV: a whole-raster solve of the advanced mode (grid.cpp:73-210) instead of a moving window: finite grounds add
// their conductance to the diagonal, direct grounds are not unknowns, and the components are solved one by one.
template <int NT, typename T, bool FOUR, bool MG, bool REFINE, bool HOT, bool ADV = false>
struct Win {
    static_assert(REFINE || sizeof(T) == 8, "an FP32 inner solve needs the FP64 refinement");
    // Padded indices of the unknowns: 16 bits for windows (below 65,536 padded cells), 32 for whole rasters.
    using Idx = typename std::conditional<ADV, uint32_t, uint16_t>::type;
    using NB = Nb<FOUR>;
    static constexpr int ND = NB::ND, LOWER = NB::LOWER;

    const KArgs &a;
    char *sm, *gm;
    Reducer<NT> &red;
    int *scan;       // shared scratch (>= 64 ints)
    int *lvh, *lvw;  // shared: level dimensions
    float *lvinv;    // shared: 1 / level width
    uint32_t *lvoff; // shared: arena offsets of the coarse levels' arrays, LV_COUNT per level (from level 1)
    short *cidx;     // shared: padded indices of the coarsest level's cells (kNcMax)
    float invP = 1.f;  // 1 / G.P
    WinGeom G;
    int nu = 0;      // number of unknowns
    int nlev = 1;
    double src_sum = 0.0;  // the landscape window's sum of positive raw sources (the scaling denominator)
#ifdef LSB_PHASE_TIMERS
    unsigned long long *tacc = nullptr;  // shared, PH_COUNT + 1 (the last: time of the previous mark)
#endif

    // Profiling builds: charge the time since the previous mark to phase k (a barrier first).
    __device__ __forceinline__ void mark(int k) {
#ifdef LSB_PHASE_TIMERS
        __syncthreads();
        if (threadIdx.x == 0) {
            const unsigned long long t = clock64();
            tacc[k] += t - tacc[PH_COUNT];
            tacc[PH_COUNT] = t;
        }
#else
        (void)k;
#endif
    }

    __device__ Win(const KArgs &a_, char *sm_, char *gm_, Reducer<NT> &red_, int *scan_, int *lvh_, int *lvw_,
                   float *lvinv_, uint32_t *lvoff_, short *cidx_)
        : a(a_), sm(sm_), gm(gm_), red(red_), scan(scan_), lvh(lvh_), lvw(lvw_), lvinv(lvinv_), lvoff(lvoff_),
          cidx(cidx_) {}

    template <typename X>
    __device__ __forceinline__ X *A(int k) const {
        if (HOT && hot_array(k)) return reinterpret_cast<X *>(sm + a.lay.off[k]);
        return arena_ptr<X>(a.lay, k, sm, gm);
    }
    // (the offsets come from the shared table: a level index known only at run time would otherwise index the
    // kernel's parameters)
    template <typename X>
    __device__ __forceinline__ X *LV(int l, int k) const {
        const uint32_t o = lvoff[(l - 1) * LV_COUNT + k];
        if (HOT) return reinterpret_cast<X *>(sm + o);
        return reinterpret_cast<X *>((o & 0x80000000u) ? gm + (o & 0x7fffffffu) : sm + o);
    }
    __device__ __forceinline__ int noff(int d) const { return NB::dy(d) * G.P + NB::dx(d); }

    // ---- 1. window data ----------------------------------------------------
    // Conductance, candidates and raw sources (omniscape.cpp:495-519).  FLOW
    // keeps the sources the LAND pass scaled.  Returns the sum of positive raw
    // sources (the scaling denominator; 0 for FLOW).
    __device__ __forceinline__ double load(int kind, double amps) {
        uint8_t *mask = A<uint8_t>(AR_MASK);
        double *g64 = A<double>(AR_G64), *x64 = A<double>(AR_X64), *b64 = A<double>(AR_B64);
        const int h = G.h, w = G.w, P = G.P, NP = G.NP;
        const int R = a.R, D = a.D, br = a.br;
        invP = 1.0f / static_cast<float>(P);
        const int64_t ylim = (D + br < a.ny - 1 ? D + br : a.ny - 1), xlim = (D + br < a.nx - 1 ? D + br : a.nx - 1);
        double pos = 0.0;
        for (int i = threadIdx.x; i < NP; i += NT) {
            const int py = i / P, y = py - 1, x = i - py * P - 1;
            double g = 0.0, raw = 0.0;
            uint8_t m = 0;
            if (y >= 0 && y < h && x >= 0 && x < w) {
                const int dy = y - G.gy, dx = x - G.gx, d2 = dy * dy + dx * dx;
                if (kind == KIND_LAND) {
                    const double r = a.res[(G.y0 + y) * a.nx + (G.x0 + x)];
                    g = -9999.0;
                    if (d2 <= D * D && !isnan(r)) g = a.ric ? r : 1.0 / r;
                    if (d2 <= R * R) {
                        raw = a.src[(G.y0 + y) * a.nx + (G.x0 + x)];
                        if (isnan(raw)) raw = 0.0;
                    }
                } else if (kind == KIND_FLOW) {
                    g = 1.0;
                } else {
                    g = d2 <= D * D ? 1.0 : -9999.0;
                    raw = d2 <= R * R ? 1.0 : 0.0;
                    if (kind == KIND_CORR_NULL && dy == 0 && dx == 0) raw = 0.0;
                }
                if (kind == KIND_LAND || kind == KIND_CORR_BLOCK) {
                    // the target block zeroed at radius + buffer from the corner (omniscape.cpp:517-519)
                    if (y >= D - br && y <= ylim && x >= D - br && x <= xlim) raw = 0.0;
                }
                if (g > 0) m = M_CAND;
                if (kind != KIND_FLOW) {
                    b64[i] = raw;
                    if (raw > 0) pos += raw;
                }
            } else if (kind != KIND_FLOW) {
                b64[i] = 0.0;
            }
            g64[i] = g;
            mask[i] = m;
            x64[i] = 0.0;
        }
        if (kind == KIND_FLOW) {
            __syncthreads();
            return 0.0;
        }
        const double sum = red.sum(pos);  // ends with a barrier
        src_sum = sum;
        // rescale the positive sources to the block's amps (omniscape.cpp:520-525)
        if (kind == KIND_CORR_NULL) {
            const double v = 1.0 / (a.n_corr_sources - 1.0);
            for (int i = threadIdx.x; i < NP; i += NT)
                if (b64[i] != 0.0) b64[i] = v;
        } else {
            if (kind == KIND_CORR_BLOCK) amps = static_cast<double>(a.bs) * a.bs;
            for (int i = threadIdx.x; i < NP; i += NT) {
                const double v = b64[i];
                if (v > 0) b64[i] = (v * amps) / sum;
            }
        }
        __syncthreads();
        return sum;
    }

    // Conditions (omniscape.cpp:526-530, match_condition :218-230).
    __device__ __forceinline__ void apply_conditions(double v1, double v2) {
        double *b64 = A<double>(AR_B64);
        for (int k = 0; k < 2; ++k) {
            const double *c = a.cond_present[k];
            if (!c) continue;
            const double val = k == 0 ? v1 : v2;
            for (int i = threadIdx.x; i < G.NP; i += NT) {
                const int py = i / G.P, y = py - 1, x = i - py * G.P - 1;
                if (y < 0 || y >= G.h || x < 0 || x >= G.w) continue;
                const double v = c[(G.y0 + y) * a.nx + (G.x0 + x)];
                if (isnan(v)) continue;
                if (a.cond_equal[k]) {
                    if (v != val) b64[i] = 0.0;
                } else {
                    const double dd = v - val;
                    if (dd > a.cond_hi[k] || dd < a.cond_lo[k]) b64[i] = 0.0;
                }
            }
            __syncthreads();
        }
    }

    // ---- 2. the ground's component -----------------------------------------
    // Monotone label propagation until no cell changes; bounded by the number
    // of cells (every productive sweep adds one).  Returns false when the
    // ground has no node.
    __device__ __forceinline__ bool flood(int kind) {
        uint8_t *mask = A<uint8_t>(AR_MASK);
        const int ground = (G.gy + 1) * G.P + G.gx + 1;
        if (kind == KIND_FLOW) {
            for (int i = threadIdx.x; i < G.NP; i += NT)
                if (mask[i] & M_CAND) mask[i] = M_CAND | M_PRESENT;
            __syncthreads();
            return true;
        }
        const bool has = mask[ground] & M_CAND;
        __syncthreads();
        if (!has) return false;
        // Bit rows over the padded box (bit px of word px / 32 of row py), held in the CG vector P until the
        // assembly clears it: candidates cb and reached cells pb, pb starting at the ground.  A sweep sets in
        // every word the candidates next to a reached cell (word-wise dilation, carries from the neighbouring
        // words); it is monotone, so words written during a sweep may be read old or new, and the sweeps end
        // when one changes nothing: pb is then the ground's component.
        const int P = G.P, words = (P + 31) >> 5, nrow = G.h + 2, ntask = nrow * words;
        const float invwd = 1.0f / static_cast<float>(words);  // (k + 0.5) / words in float: exact row, k < 2^22
        uint32_t *cb = reinterpret_cast<uint32_t *>(A<T>(AR_P)), *pb = cb + ntask;
        const int gpy = G.gy + 1, gpx = G.gx + 1;
        const int lane = threadIdx.x & 31;
        for (int k = threadIdx.x >> 5; k < ntask; k += NT / 32) {
            const int py = static_cast<int>((static_cast<float>(k) + 0.5f) * invwd), w = k - py * words;
            const int px = 32 * w + lane;
            const bool c = px < P && (mask[py * P + px] & M_CAND) != 0;
            const uint32_t bits = __ballot_sync(0xffffffffu, c);
            if (lane == 0) {
                cb[k] = bits;
                pb[k] = (py == gpy && w == (gpx >> 5)) ? (1u << (gpx & 31)) : 0u;
            }
        }
        __syncthreads();
        volatile uint32_t *vp = pb;
        while (true) {
            int changed = 0;
            for (int k = threadIdx.x; k < ntask; k += NT) {
                const uint32_t c = cb[k];
                if (!c) continue;  // padding rows hold no candidate: rows py - 1 and py + 1 exist below
                const int py = static_cast<int>((static_cast<float>(k) + 0.5f) * invwd), w = k - py * words;
                const uint32_t mid = vp[k];
                const bool hl = w > 0, hr = w + 1 < words;
                uint32_t nb;
                if (FOUR) {
                    const uint32_t l = hl ? vp[k - 1] : 0u, r = hr ? vp[k + 1] : 0u;
                    nb = vp[k - words] | vp[k + words] | (mid << 1) | (l >> 31) | (mid >> 1) | (r << 31);
                } else {
                    const uint32_t v = vp[k - words] | mid | vp[k + words];
                    const uint32_t vl = hl ? (vp[k - words - 1] | vp[k - 1] | vp[k + words - 1]) : 0u;
                    const uint32_t vr = hr ? (vp[k - words + 1] | vp[k + 1] | vp[k + words + 1]) : 0u;
                    nb = v | (v << 1) | (vl >> 31) | (v >> 1) | (vr << 31);
                }
                const uint32_t nw = c & (mid | nb);
                if (nw != mid) {
                    vp[k] = nw;
                    changed = 1;
                }
            }
            if (!__syncthreads_or(changed)) break;
        }
        for (int i = threadIdx.x; i < G.NP; i += NT) {
            const int py = row0(i), px = i - py * P;
            if ((pb[py * words + (px >> 5)] >> (px & 31)) & 1u) mask[i] |= M_PRESENT;
        }
        __syncthreads();
        return true;
    }

    // Sum of the sources over the unknowns-to-be (omniscape.cpp:101, 149-150);
    // marks the unknowns and lists them.
    __device__ __forceinline__ double mark_unknowns() {
        uint8_t *mask = A<uint8_t>(AR_MASK);
        const double *b64 = A<double>(AR_B64);
        const int ground = (G.gy + 1) * G.P + G.gx + 1;
        double t = 0.0;
        for (int i = threadIdx.x; i < G.NP; i += NT) {
            uint8_t m = mask[i];
            if ((m & M_PRESENT) && (ADV ? !(m & M_DIRECT) : i != ground)) {
                m |= M_UNKNOWN;
                t += b64[i];
            }
            mask[i] = m;
        }
        const double total = red.sum(t);
        nu = block_compact<NT, Idx>(G.NP, [&](int i) { return (mask[i] & M_UNKNOWN) != 0; }, A<Idx>(AR_ULIST), scan);
        return total;
    }

    // ---- 3. assembly -------------------------------------------------------
    // Diagonal summed in column-major neighbour order with the 10 eps shift
    // (system.cpp:458-487); stencil conductances with sentinels off the nodes.
    __device__ __forceinline__ void assemble() {
        const uint8_t *mask = A<uint8_t>(AR_MASK);
        const double *g64 = A<double>(AR_G64);
        T *gT = A<T>(AR_GT), *invd = A<T>(AR_INVD), *z = A<T>(AR_Z);
        T *d = A<T>(AR_D), *r = A<T>(AR_R), *p = A<T>(AR_P), *q = A<T>(AR_Q);
        const bool series = a.series;
        for (int i = threadIdx.x; i < G.NP; i += NT) {
            const uint8_t m = mask[i];
            const double g = g64[i];
            gT[i] = (m & M_PRESENT) ? static_cast<T>(series ? 1.0 / g : g)
                                    : (series ? Sentinel<T>::pos() : Sentinel<T>::neg());
            invd[i] = T(0);
            p[i] = T(0);
            q[i] = T(0);
            r[i] = T(0);
            if (!(REFINE == false && sizeof(T) == 8)) d[i] = T(0);
            if (MG) z[i] = T(0);
            if (ADV) A<T>(AR_FGT)[i] = static_cast<T>(A<double>(AR_FG64)[i]);
        }
        __syncthreads();
        const Idx *ul = A<Idx>(AR_ULIST);
        for (int k = threadIdx.x; k < nu; k += NT) {
            const int i = ul[k];
            const double gi = g64[i];
            double diag = 0.0;
#pragma unroll
            for (int dd = 0; dd < ND; ++dd) {
                const int n = i + noff(dd);
                if (mask[n] & M_PRESENT) diag += edge_w64(gi, g64[n], NB::diag(dd), series);
            }
            if (ADV) diag += A<double>(AR_FG64)[i];  // a finite ground (system.cpp: the extra diagonal)
            // multigrid kernels keep omega / diag: the damped-Jacobi smoother's factor (a scalar multiple of
            // the Jacobi preconditioner, to which CG is invariant)
            invd[i] = static_cast<T>((MG ? static_cast<double>(a.sp.omega) : 1.0) / (diag + kShift));
            if (MG) z[i] = static_cast<T>(diag);
        }
        __syncthreads();
    }

    // Two values of a cell, computed before either is stored.
    struct TPair {
        T a, b;
    };
    struct DPair {
        double a, b;
    };

    // Visits the unknowns k = threadIdx.x + j NT (increasing j, so per-thread sums keep their order) two at a
    // time: both cells' loads and arithmetic (`calc`, which only reads) come before both stores (`put`), so
    // the two cells' memory latencies overlap.
    template <class C, class Put>
    __device__ __forceinline__ void unknowns2(C calc, Put put) const {
        const Idx *ul = A<Idx>(AR_ULIST);
        for (int k = threadIdx.x; k < nu; k += 2 * NT) {
            const bool two = k + NT < nu;
            const int i1 = ul[k], i2 = two ? ul[k + NT] : i1;
            const auto v1 = calc(i1);
            const auto v2 = calc(i2);
            put(i1, v1);
            if (two) put(i2, v2);
        }
    }

    // ---- level-0 operator in T ---------------------------------------------
    // (A x)_i = sum_d w_id (x_i - x_n); w from the stencil conductances
    // (sentinels give w = 0 off the nodes; x = 0 off the unknowns).
    __device__ __forceinline__ T apply0(const T *gT, const T *x, int i) const {
        const T gi = gT[i], xi = x[i];
        T ao = T(0), ad = T(0);
        if (a.series) {
#pragma unroll
            for (int dd = 0; dd < ND; ++dd) {
                const int n = i + noff(dd);
                const T wv = T(2) / (gi + gT[n]);
                if (NB::diag(dd))
                    ad += wv * (xi - x[n]);
                else
                    ao += wv * (xi - x[n]);
            }
            return ao + ad * T(0.70710678118654752440) + (ADV ? A<T>(AR_FGT)[i] * xi : T(0));
        }
#pragma unroll
        for (int dd = 0; dd < ND; ++dd) {
            const int n = i + noff(dd);
            const T wv = tmax(gi + gT[n], T(0));
            if (NB::diag(dd))
                ad += wv * (xi - x[n]);
            else
                ao += wv * (xi - x[n]);
        }
        return ao * T(0.5) + ad * T(kInvTwoSqrt2) + (ADV ? A<T>(AR_FGT)[i] * xi : T(0));
    }

    // A level-0 entry A(i, i+s) for RAP (s = (sy, sx) in {-1,0,1}^2).
    __device__ __forceinline__ T entry0(int i, int sy, int sx) const {
        const uint8_t *mask = A<uint8_t>(AR_MASK);
        if (sy == 0 && sx == 0) return A<T>(AR_Z)[i];
        if (FOUR && sy != 0 && sx != 0) return T(0);
        const int n = i + sy * G.P + sx;
        if (!(mask[n] & M_UNKNOWN)) return T(0);
        const T *gT = A<T>(AR_GT);
        const bool dg = sy != 0 && sx != 0;
        if (a.series) {
            const T wv = T(2) / (gT[i] + gT[n]);
            return -(dg ? wv * T(0.70710678118654752440) : wv);
        }
        const T wv = tmax(gT[i] + gT[n], T(0));
        return -(dg ? wv * T(kInvTwoSqrt2) : wv * T(0.5));
    }

    // The level-0 entries during the multigrid set-up: with precomputed weights (kWeights), the off-diagonal
    // entries towards E, S, SE and SW of every unknown are held in the (then unused) CG vectors P, Q, R and D,
    // zero where either end is no unknown; the rest by symmetry.  Same values as entry0.
    static constexpr bool kWeights = sizeof(T) == 4 || REFINE;  // D exists
    __device__ __forceinline__ T entry0w(int i, int sy, int sx) const {
        if (!kWeights) return entry0(i, sy, sx);
        if (sy == 0 && sx == 0) return A<T>(AR_Z)[i];
        if (FOUR && sy != 0 && sx != 0) return T(0);
        const T *WE = A<T>(AR_P), *WS = A<T>(AR_Q), *WSE = A<T>(AR_R), *WSW = A<T>(AR_D);
        const int P = G.P;
        if (sy == 0) return sx > 0 ? WE[i] : WE[i - 1];
        if (sx == 0) return sy > 0 ? WS[i] : WS[i - P];
        if (sy > 0) return sx > 0 ? WSE[i] : WSW[i];
        return sx > 0 ? WSW[i - P + 1] : WSE[i - P - 1];
    }
    // Fills (fill == true) or clears the weights of entry0w (the vectors are zero before and after).
    __device__ __forceinline__ void weights0(bool fill) {
        if (!kWeights) return;
        T *WE = A<T>(AR_P), *WS = A<T>(AR_Q), *WSE = A<T>(AR_R), *WSW = A<T>(AR_D);
        unknowns2(
            [&](int i) { return fill ? TPair{entry0(i, 0, 1), entry0(i, 1, 0)} : TPair{T(0), T(0)}; },
            [&](int i, const TPair &v) {
                WE[i] = v.a;
                WS[i] = v.b;
            });
        if (!FOUR) {
            unknowns2(
                [&](int i) {
                    return fill ? TPair{entry0(i, 1, 1), entry0(i, 1, -1)} : TPair{T(0), T(0)};
                },
                [&](int i, const TPair &v) {
                    WSE[i] = v.a;
                    WSW[i] = v.b;
                });
        }
        __syncthreads();
    }

    // The arrays of coarse level l (pointers resolved once, not per cell).
    struct Lvl {
        T *c0, *cE, *cSW, *cS, *cSE, *iv, *x, *b, *t;
        int h, w, P;
    };
    __device__ __forceinline__ Lvl lvl(int l) const {
        Lvl L;
        L.c0 = LV<T>(l, LV_C0);
        L.cE = LV<T>(l, LV_CE);
        L.cSW = LV<T>(l, LV_CSW);
        L.cS = LV<T>(l, LV_CS);
        L.cSE = LV<T>(l, LV_CSE);
        L.iv = LV<T>(l, LV_INVD);
        L.x = LV<T>(l, LV_X);
        L.b = LV<T>(l, LV_B);
        L.t = LV<T>(l, LV_T);
        L.h = lvh[l];
        L.w = lvw[l];
        L.P = L.w + 2;
        return L;
    }

    // A coarse entry A_l(i, i+s) from the symmetric storage.
    __device__ __forceinline__ static T entryc(const Lvl &L, int i, int sy, int sx) {
        const int P = L.P;
        if (sy == 0 && sx == 0) return L.c0[i];
        if (sy == 0 && sx == 1) return L.cE[i];
        if (sy == 1 && sx == -1) return L.cSW[i];
        if (sy == 1 && sx == 0) return L.cS[i];
        if (sy == 1 && sx == 1) return L.cSE[i];
        if (sy == 0 && sx == -1) return L.cE[i - 1];
        if (sy == -1 && sx == 1) return L.cSW[i - P + 1];
        if (sy == -1 && sx == 0) return L.cS[i - P];
        return L.cSE[i - P - 1];  // (-1, -1)
    }
    __device__ __forceinline__ static T applyc(const Lvl &L, const T *x, int i) {
        const int P = L.P;
        T s = L.c0[i] * x[i];
        s += L.cE[i] * x[i + 1] + L.cSW[i] * x[i + P - 1] + L.cS[i] * x[i + P] + L.cSE[i] * x[i + P + 1];
        s += L.cE[i - 1] * x[i - 1] + L.cSW[i - P + 1] * x[i - P + 1] + L.cS[i - P] * x[i - P] +
             L.cSE[i - P - 1] * x[i - P - 1];
        return s;
    }

    // ---- multigrid set-up (Galerkin R A P, masked bilinear P) -------------
    // Coarse point J of a coarsened dimension sits on fine point 2J; a fine
    // point's weight in P is 1 on its coarse point and 1/2 next to one.  P's
    // rows of fine cells that are not unknowns (level 0) or not active are
    // zero, so coarse cells whose support holds no such cell are inactive
    // (identity rows).  Coarse operators are 9-point; each cell stores its
    // diagonal and the 4 entries towards E, SW, S, SE (the rest by symmetry).

    // Cells of level l, warps along rows and lanes along columns (no division).
    // (k + 0.5) / w in float gives the exact row of cell k whenever k + 0.5 < 2^22: the rounding error, at most
    // 2^-23 of the quotient, stays below the quotient's distance 0.5 / w from an integer.
    template <class F>
    __device__ __forceinline__ void for_cells(int l, F f) const {
        const int h = lvh[l], w = lvw[l], P = w + 2, n = h * w;
        const float invw = lvinv[l];
        for (int k = threadIdx.x; k < n; k += NT) {
            const int y = static_cast<int>((static_cast<float>(k) + 0.5f) * invw), x = k - y * w;
            f(y, x, (y + 1) * P + x + 1);
        }
    }

    // Level l -> l + 1 at coarse cell (jy, jx) when both dimensions coarsen:
    // all but the entries resolved at compile time.
    template <int L0>
    __device__ __forceinline__ void rap_cell(const Lvl &F, int jy, int jx, T (&acc)[5], bool &act) const {
        const int hf = F.h, wf = F.w, Pf = F.P;
#pragma unroll
        for (int ay = -1; ay <= 1; ++ay) {
#pragma unroll
            for (int ax = -1; ax <= 1; ++ax) {
                const int fy = 2 * jy + ay, fx = 2 * jx + ax;
                if (fy < 0 || fy >= hf || fx < 0 || fx >= wf) continue;
                const int i = (fy + 1) * Pf + fx + 1;
                if (!(L0 ? (A<uint8_t>(AR_MASK)[i] & M_UNKNOWN) != 0 : F.iv[i] != T(0))) continue;
                act = true;
                const T wi = (ay == 0 ? T(1) : T(0.5)) * (ax == 0 ? T(1) : T(0.5));
#pragma unroll
                for (int sy = -1; sy <= 1; ++sy) {
#pragma unroll
                    for (int sx = -1; sx <= 1; ++sx) {
                        if (FOUR && L0 && sy != 0 && sx != 0) continue;
                        const T v = wi * (L0 ? entry0w(i, sy, sx) : entryc(F, i, sy, sx));
                        const int dy = ay + sy, dx = ax + sx;  // fine j relative to 2J, in [-2, 2]
#pragma unroll
                        for (int py = 0; py < 2; ++py) {
#pragma unroll
                            for (int px = 0; px < 2; ++px) {
                                const bool oy = (dy & 1) != 0, ox = (dx & 1) != 0;
                                if ((!oy && py) || (!ox && px)) continue;
                                const int ky = oy ? (dy - 1) / 2 + py : dy / 2;
                                const int kx = ox ? (dx - 1) / 2 + px : dx / 2;
                                const int slot = (ky == 0 && kx == 0)    ? 0
                                                 : (ky == 0 && kx == 1)  ? 1
                                                 : (ky == 1 && kx == -1) ? 2
                                                 : (ky == 1 && kx == 0)  ? 3
                                                 : (ky == 1 && kx == 1)  ? 4
                                                                         : -1;
                                if (slot < 0) continue;
                                acc[slot] += v * (oy ? T(0.5) : T(1)) * (ox ? T(0.5) : T(1));
                            }
                        }
                    }
                }
            }
        }
    }

    // The general case (a dimension of at most 3 cells does not coarsen).
    __device__ __forceinline__ void rap_cell_general(int l, const Lvl &F, int jy, int jx, bool cy, bool cx,
                                                     T (&acc)[5], bool &act) const {
        const int hf = F.h, wf = F.w, Pf = F.P;
        const int hc = lvh[l + 1], wc = lvw[l + 1];
        for (int ay = (cy ? -1 : 0); ay <= (cy ? 1 : 0); ++ay) {
            const int fy = cy ? 2 * jy + ay : jy;
            if (fy < 0 || fy >= hf) continue;
            for (int ax = (cx ? -1 : 0); ax <= (cx ? 1 : 0); ++ax) {
                const int fx = cx ? 2 * jx + ax : jx;
                if (fx < 0 || fx >= wf) continue;
                const int i = (fy + 1) * Pf + fx + 1;
                if (!(l == 0 ? (A<uint8_t>(AR_MASK)[i] & M_UNKNOWN) != 0 : F.iv[i] != T(0))) continue;
                act = true;
                const T wi = (ay == 0 ? T(1) : T(0.5)) * (ax == 0 ? T(1) : T(0.5));
                for (int sy = -1; sy <= 1; ++sy)
                    for (int sx = -1; sx <= 1; ++sx) {
                        const T aij = l == 0 ? entry0(i, sy, sx) : entryc(F, i, sy, sx);
                        if (aij == T(0)) continue;
                        const int gy = fy + sy, gx = fx + sx;
                        for (int e = 0; e < 5; ++e) {
                            const int ky = jy + (e < 2 ? 0 : 1);
                            const int kx = jx + (e == 0 ? 0 : e == 1 ? 1 : e == 2 ? -1 : e == 3 ? 0 : 1);
                            if (ky >= hc || kx < 0 || kx >= wc) continue;
                            T py, px;
                            if (cy) {
                                const int dd = gy - 2 * ky;
                                py = dd == 0 ? T(1) : (dd == 1 || dd == -1) ? T(0.5) : T(0);
                            } else {
                                py = gy == ky ? T(1) : T(0);
                            }
                            if (cx) {
                                const int dd = gx - 2 * kx;
                                px = dd == 0 ? T(1) : (dd == 1 || dd == -1) ? T(0.5) : T(0);
                            } else {
                                px = gx == kx ? T(1) : T(0);
                            }
                            acc[e] += wi * aij * py * px;
                        }
                    }
            }
        }
    }

    __device__ __forceinline__ void mg_setup() {
        nlev = mg_levels(G.h, G.w);
        Lvl fine0;  // level 0 as a level: only its dimensions are read
        fine0.h = G.h;
        fine0.w = G.w;
        fine0.P = G.P;
        if (threadIdx.x == 0) {
            int h = G.h, w = G.w;
            for (int l = 0; l < nlev; ++l) {
                lvh[l] = h;
                lvw[l] = w;
                lvinv[l] = 1.0f / static_cast<float>(w);
                h = coarse_dim(h);
                w = coarse_dim(w);
            }
        }
        if (nlev > 1) weights0(true);  // ends with a barrier
        __syncthreads();
        mark(PH_S_W);
        for (int l = 1; l < nlev; ++l) {
            const int hf = lvh[l - 1], wf = lvw[l - 1];
            const int hc = lvh[l], wc = lvw[l], NPc = (hc + 2) * (wc + 2);
            const bool cy = hc != hf, cx = wc != wf;
            const Lvl C = lvl(l), F = lvl(l > 1 ? l - 1 : 1);  // (level 0 is read through entry0)
            const Lvl &Fp = l > 1 ? F : C;
            T *c0 = C.c0, *cE = C.cE, *cSW = C.cSW, *cS = C.cS, *cSE = C.cSE, *iv = C.iv, *x = C.x, *b = C.b,
              *t = C.t;
            for (int J = threadIdx.x; J < NPc; J += NT) {
                c0[J] = T(0);
                cE[J] = T(0);
                cSW[J] = T(0);
                cS[J] = T(0);
                cSE[J] = T(0);
                iv[J] = T(0);
                x[J] = T(0);
                b[J] = T(0);
                t[J] = T(0);
            }
            __syncthreads();
            const T om = static_cast<T>(a.sp.omega_c);
            for_cells(l, [&](int jy, int jx, int J) {
                T acc[5] = {T(0), T(0), T(0), T(0), T(0)};
                bool act = false;
                if (cy && cx) {
                    if (l == 1)
                        rap_cell<1>(fine0, jy, jx, acc, act);
                    else
                        rap_cell<0>(Fp, jy, jx, acc, act);
                } else {
                    rap_cell_general(l - 1, l == 1 ? fine0 : Fp, jy, jx, cy, cx, acc, act);
                }
                if (!act) return;
                // entries towards cells outside the coarse box stay zero
                c0[J] = acc[0];
                cE[J] = jx + 1 < wc ? acc[1] : T(0);
                cSW[J] = (jy + 1 < hc && jx > 0) ? acc[2] : T(0);
                cS[J] = jy + 1 < hc ? acc[3] : T(0);
                cSE[J] = (jy + 1 < hc && jx + 1 < wc) ? acc[4] : T(0);
                iv[J] = om / acc[0];
            });
            __syncthreads();
            if (l == 1) weights0(false);
            mark(l == 1 ? PH_S_L1 : PH_S_LC);
        }
        dense_setup();
        mark(PH_S_DENSE);
    }

    // Pseudo-inverse of the coarsest operator (at most kNcMax cells), full and
    // symmetric in M (row stride kNcMax).  Also lists the coarsest cells' padded
    // indices (cidx).
    __device__ __forceinline__ void dense_setup() {
        double *M = A<double>(AR_DENSE);
        const int l = nlev - 1;
        const int hc = lvh[l], wc = lvw[l], Pc = wc + 2, n = hc * wc;
        const Lvl C = lvl(l > 0 ? l : 1);  // (level 0 is read through entry0)
        auto act = [&](int i) {
            return l == 0 ? (A<uint8_t>(AR_MASK)[i] & M_UNKNOWN) != 0 : C.iv[i] != T(0);
        };
        if (threadIdx.x < n) cidx[threadIdx.x] = static_cast<short>((threadIdx.x / wc + 1) * Pc + threadIdx.x % wc + 1);
        for (int e = threadIdx.x; e < kNcMax * kNcMax; e += NT) {
            const int u = e / kNcMax, v = e - u * kNcMax;
            double val = 0.0;
            if (u < n && v < n) {
                const int uy = u / wc, ux = u - uy * wc, vy = v / wc, vx = v - vy * wc;
                const int sy = vy - uy, sx = vx - ux;
                const int iu = (uy + 1) * Pc + ux + 1;
                if (sy >= -1 && sy <= 1 && sx >= -1 && sx <= 1) {
                    if (!act(iu) || !act((vy + 1) * Pc + vx + 1))
                        val = (u == v) ? 1.0 : 0.0;
                    else
                        val = static_cast<double>(l == 0 ? entry0(iu, sy, sx) : entryc(C, iu, sy, sx));
                }
            }
            M[e] = val;
        }
        __syncthreads();
        // Symmetric sweep (Gauss-Jordan on a symmetric matrix), one pivot after another with every thread on the
        // update: at step k the pivot is the Schur complement of the pivots swept before it, the value the
        // Cholesky factorisation meets.  A pivot that vanished against the original diagonal (a dependent
        // direction of the masked prolongation) is skipped.  After the last step the swept block holds minus the
        // inverse of the non-skipped principal submatrix; skipped rows and columns become zero.
        double *colk = M + kNcMax * kNcMax, *od = colk + kNcMax;
        unsigned *skip = reinterpret_cast<unsigned *>(scan);
        if (threadIdx.x < n) od[threadIdx.x] = M[threadIdx.x * kNcMax + threadIdx.x];
        if (threadIdx.x == 0) *skip = 0u;
        const int jl = threadIdx.x & 31;  // column of this thread; rows by warp (n <= kNcMax <= 32)
        for (int k = 0; k < n; ++k) {
            __syncthreads();  // the previous step's writes (and od, skip) visible
            if (threadIdx.x < n) colk[threadIdx.x] = M[threadIdx.x * kNcMax + k];
            if (threadIdx.x == 0) {
                const double piv = M[k * kNcMax + k];
                if (!(piv > 1e-10 * od[k]))
                    *skip |= 1u << k;
                else
                    od[k] = 1.0 / piv;  // the original diagonal of k is not read again
            }
            __syncthreads();
            if ((*skip >> k) & 1u) continue;
            const double inv = od[k];
            if (jl < n) {
                for (int i = threadIdx.x >> 5; i < n; i += NT / 32) {
                    double v;
                    if (i == k && jl == k)
                        v = -inv;
                    else if (i == k)
                        v = colk[jl] * inv;
                    else if (jl == k)
                        v = colk[i] * inv;
                    else
                        v = M[i * kNcMax + jl] - colk[i] * (colk[jl] * inv);
                    M[i * kNcMax + jl] = v;
                }
            }
        }
        __syncthreads();
        const unsigned sk = *skip;
        if (jl < n)
            for (int i = threadIdx.x >> 5; i < n; i += NT / 32)
                M[i * kNcMax + jl] = (((sk >> i) | (sk >> jl)) & 1u) ? 0.0 : -M[i * kNcMax + jl];
        __syncthreads();
    }

    // Row of a padded index of level 0 (i < 2^22, as for_cells): exact in float.
    __device__ __forceinline__ int row0(int i) const {
        return static_cast<int>((static_cast<float>(i) + 0.5f) * invP);
    }

    // z = B r: one V(1,1) cycle, damped-Jacobi smoothing, exact coarsest.
    // r is level-0 (unknowns only); the result goes to AR_Q; AR_Z is scratch.
    // Also adds this thread's terms of r.z and r.r to rz and rr (its unknowns in increasing order), and copies z
    // to pcopy when given.
    __device__ __forceinline__ void vcycle(const T *r, double &rz, double &rr, T *pcopy = nullptr) {
        const Idx *ul = A<Idx>(AR_ULIST);
        const T *gT = A<T>(AR_GT), *invd = A<T>(AR_INVD);
        T *z = A<T>(AR_Z), *q = A<T>(AR_Q);
        if (nlev == 1) {
            // the window is its own coarsest level
            coarse_solve(0, r, q);
            __syncthreads();
            for (int k = threadIdx.x; k < nu; k += NT) {
                const int i = ul[k];
                const T zi = q[i];
                if (pcopy) pcopy[i] = zi;
                rz += static_cast<double>(r[i]) * static_cast<double>(zi);
                rr += static_cast<double>(r[i]) * static_cast<double>(r[i]);
            }
            return;
        }
        // pre-smoothing from zero and the residual in one pass: z = w D^-1 r, q = r - A z (invd holds w / diag)
        mark(PH_VCYCLE);
        unknowns2(
            [&](int i) {
                const T zi = invd[i] * r[i];
                return TPair{zi, r[i] - apply0_scaled(gT, r, invd, i, zi)};
            },
            [&](int i, const TPair &v) {
                z[i] = v.a;
                q[i] = v.b;
            });
        __syncthreads();
        mark(PH_V_PRE0);
        restrict_to(1, q);
        mark(PH_V_RESTRICT1);
        for (int l = 1; l < nlev - 1; ++l) {
            smooth_down(l);
            mark(PH_L_DS + (l < 2 ? 0 : 1));
            restrict_to(l + 1, LV<T>(l, LV_T));
            mark(PH_L_DR + (l < 2 ? 0 : 1));
        }
        coarse_solve(nlev - 1, LV<T>(nlev - 1, LV_B), LV<T>(nlev - 1, LV_X));
        __syncthreads();
        mark(PH_V_COARSEST);
        for (int l = nlev - 2; l >= 1; --l) {
            smooth_up(l);
            mark(PH_L_US + (l < 2 ? 0 : 1));
        }
        prolong_add(0, z, LV<T>(1, nlev - 1 == 1 ? LV_X : LV_T));
        __syncthreads();
        mark(PH_V_PROLONG0);
        unknowns2([&](int i) { return TPair{z[i] + invd[i] * (r[i] - apply0(gT, z, i)), r[i]}; },
                  [&](int i, const TPair &v) {
                      q[i] = v.a;
                      if (pcopy) pcopy[i] = v.a;
                      rz += static_cast<double>(v.b) * static_cast<double>(v.a);
                      rr += static_cast<double>(v.b) * static_cast<double>(v.b);
                  });
        __syncthreads();
        mark(PH_V_POST0);
    }

    // (A z)_i with z_n = w invd_n r_n computed from the neighbours' r (the
    // pre-smoothed iterate without storing it first).
    __device__ __forceinline__ T apply0_scaled(const T *gT, const T *r, const T *invd, int i, T zi) const {
        const T gi = gT[i];
        T ao = T(0), ad = T(0);
        if (a.series) {
#pragma unroll
            for (int dd = 0; dd < ND; ++dd) {
                const int n = i + noff(dd);
                const T wv = T(2) / (gi + gT[n]);
                const T zn = invd[n] * r[n];
                if (NB::diag(dd))
                    ad += wv * (zi - zn);
                else
                    ao += wv * (zi - zn);
            }
            return ao + ad * T(0.70710678118654752440) + (ADV ? A<T>(AR_FGT)[i] * zi : T(0));
        }
#pragma unroll
        for (int dd = 0; dd < ND; ++dd) {
            const int n = i + noff(dd);
            const T wv = tmax(gi + gT[n], T(0));
            const T zn = invd[n] * r[n];
            if (NB::diag(dd))
                ad += wv * (zi - zn);
            else
                ao += wv * (zi - zn);
        }
        return ao * T(0.5) + ad * T(kInvTwoSqrt2) + (ADV ? A<T>(AR_FGT)[i] * zi : T(0));
    }

    // b_{l} = P^T t_{l-1} (level l-1 residual, zero off its active cells); ends with a barrier.
    __device__ __forceinline__ void restrict_to(int l, const T *tf) {
        const int hf = lvh[l - 1], wf = lvw[l - 1], Pf = wf + 2;
        const int hc = lvh[l], wc = lvw[l];
        const bool cy = hc != hf, cx = wc != wf;
        T *b = LV<T>(l, LV_B);
        const T *iv = LV<T>(l, LV_INVD);
        if (cy && cx) {
            for_cells(l, [&](int jy, int jx, int J) {
                if (iv[J] == T(0)) return;
                // fine cells 2J-1 .. 2J+1; the +1 row / column exists only inside the fine box (beyond it the
                // padded box ends: P gives it no weight and it is not read)
                const int c = (2 * jy + 1) * Pf + 2 * jx + 1;
                T s = tf[c] + T(0.5) * (tf[c - 1] + tf[c - Pf]) + T(0.25) * tf[c - Pf - 1];
                const bool yin = 2 * jy + 1 < hf, xin = 2 * jx + 1 < wf;
                if (xin) s += T(0.5) * tf[c + 1] + T(0.25) * tf[c - Pf + 1];
                if (yin) s += T(0.5) * tf[c + Pf] + T(0.25) * tf[c + Pf - 1];
                if (xin && yin) s += T(0.25) * tf[c + Pf + 1];
                b[J] = s;
            });
        } else {
            for_cells(l, [&](int jy, int jx, int J) {
                if (iv[J] == T(0)) return;
                T s = T(0);
                for (int ay = (cy ? -1 : 0); ay <= (cy ? 1 : 0); ++ay) {
                    const int fy = cy ? 2 * jy + ay : jy;
                    if (fy < 0 || fy >= hf) continue;
                    const T wa = ay == 0 ? T(1) : T(0.5);
                    for (int ax = (cx ? -1 : 0); ax <= (cx ? 1 : 0); ++ax) {
                        const int fx = cx ? 2 * jx + ax : jx;
                        if (fx < 0 || fx >= wf) continue;
                        s += wa * (ax == 0 ? T(1) : T(0.5)) * tf[(fy + 1) * Pf + fx + 1];
                    }
                }
                b[J] = s;
            });
        }
        __syncthreads();
    }

    // x_l += P x_{l+1} on the active cells of level l.
    __device__ __forceinline__ void prolong_add(int l, T *x, const T *xc) {
        const int hf = lvh[l], wf = lvw[l], Pf = wf + 2;
        const int hc = lvh[l + 1], wc = lvw[l + 1], Pc = wc + 2;
        const bool cy = hc != hf, cx = wc != wf;
        auto interp = [&](int fy, int fx) {
            int y0, y1, x0, x1;
            T wy0, wy1, wx0, wx1;
            if (cy) {
                y0 = fy >> 1;
                y1 = (fy & 1) ? y0 + 1 : y0;
                wy0 = (fy & 1) ? T(0.5) : T(1);
                wy1 = (fy & 1) ? T(0.5) : T(0);
            } else {
                y0 = y1 = fy;
                wy0 = T(1);
                wy1 = T(0);
            }
            if (cx) {
                x0 = fx >> 1;
                x1 = (fx & 1) ? x0 + 1 : x0;
                wx0 = (fx & 1) ? T(0.5) : T(1);
                wx1 = (fx & 1) ? T(0.5) : T(0);
            } else {
                x0 = x1 = fx;
                wx0 = T(1);
                wx1 = T(0);
            }
            return wy0 * (wx0 * xc[(y0 + 1) * Pc + x0 + 1] + wx1 * xc[(y0 + 1) * Pc + x1 + 1]) +
                   wy1 * (wx0 * xc[(y1 + 1) * Pc + x0 + 1] + wx1 * xc[(y1 + 1) * Pc + x1 + 1]);
        };
        if (l == 0) {
            unknowns2(
                [&](int i) {
                    const int py = row0(i);
                    return TPair{x[i] + interp(py - 1, i - py * Pf - 1), T(0)};
                },
                [&](int i, const TPair &v) { x[i] = v.a; });
        } else {
            const T *iv = LV<T>(l, LV_INVD);
            for_cells(l, [&](int fy, int fx, int i) {
                if (iv[i] != T(0)) x[i] += interp(fy, fx);
            });
        }
    }

    // x = M^+ b on the coarsest level l (its cells in row-major order, padded indices in cidx): one warp per
    // row, lanes over the columns, a fixed shuffle tree for the sum.
    __device__ __forceinline__ void coarse_solve(int l, const T *b, T *x) {
        const double *M = A<double>(AR_DENSE);
        const int n = lvh[l] * lvw[l];
        const int lane = threadIdx.x & 31;
        const double bv = lane < n ? static_cast<double>(b[cidx[lane]]) : 0.0;
        for (int u = threadIdx.x >> 5; u < n; u += NT / 32) {
            double s = lane < n ? M[u * kNcMax + lane] * bv : 0.0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
            if (lane == 0) {
                const int iu = cidx[u];
                if (l != 0 || (A<uint8_t>(AR_MASK)[iu] & M_UNKNOWN)) x[iu] = static_cast<T>(s);
            }
        }
    }

    // Down the V-cycle at coarse level l: damped Jacobi from zero (x = iv b) and the residual t = b - A x.
    __device__ __forceinline__ void smooth_down(int l) {
        const Lvl L = lvl(l);
        T *x = L.x, *t = L.t;
        const T *b = L.b, *iv = L.iv;
        const int P = L.P;
        const T *c0 = L.c0, *cE = L.cE, *cSW = L.cSW, *cS = L.cS, *cSE = L.cSE;
        for_cells(l, [&](int, int, int i) {
            const T ivi = iv[i];
            if (ivi == T(0)) return;
            auto xv = [&](int j) { return iv[j] * b[j]; };
            const T xi = ivi * b[i];
            x[i] = xi;
            T s = c0[i] * xi;
            s += cE[i] * xv(i + 1) + cSW[i] * xv(i + P - 1) + cS[i] * xv(i + P) + cSE[i] * xv(i + P + 1);
            s += cE[i - 1] * xv(i - 1) + cSW[i - P + 1] * xv(i - P + 1) + cS[i - P] * xv(i - P) +
                 cSE[i - P - 1] * xv(i - P - 1);
            t[i] = b[i] - s;
        });
        __syncthreads();
    }

    // Up the V-cycle at coarse level l: x += P x_{l+1}, then one damped-Jacobi step into t.
    __device__ __forceinline__ void smooth_up(int l) {
        const Lvl L = lvl(l);
        T *x = L.x, *t = L.t;
        const T *b = L.b, *iv = L.iv;
        prolong_add(l, x, LV<T>(l + 1, l + 1 == nlev - 1 ? LV_X : LV_T));
        __syncthreads();
        mark(PH_L_UP + (l < 2 ? 0 : 1));
        for_cells(l, [&](int, int, int i) {
            const T ivi = iv[i];
            if (ivi != T(0)) t[i] = x[i] + ivi * (b[i] - applyc(L, x, i));
        });
        __syncthreads();
    }

    // ---- preconditioned CG on the T operator -------------------------------
    // Adds to d the CG solution of A e = r0 (r holds r0 = b - A d on entry, the
    // recursively updated residual on exit), to relative residual rtol or for at
    // most maxit iterations.
    // Returns the iterations; *ok = false on breakdown.
    __device__ __forceinline__ int pcg(T *d, T *r, double rtol, int maxit, bool use_mg, bool *ok) {
        const Idx *ul = A<Idx>(AR_ULIST);
        const T *gT = A<T>(AR_GT), *invd = A<T>(AR_INVD);
        T *p = A<T>(AR_P), *q = A<T>(AR_Q);
        *ok = true;
        double rz = 0.0, rr = 0.0;
        mark(PH_RESID);
        if (MG && use_mg) {
            vcycle(r, rz, rr, p);
            mark(PH_VCYCLE);
        } else {
            for (int k = threadIdx.x; k < nu; k += NT) {
                const int i = ul[k];
                const T zi = invd[i] * r[i];
                p[i] = zi;
                rz += static_cast<double>(r[i]) * static_cast<double>(zi);
                rr += static_cast<double>(r[i]) * static_cast<double>(r[i]);
            }
        }
        red.sum2(rz, rr);  // barrier: p visible
        const double stop = rtol * rtol * rr;
        if (rr == 0.0) return 0;
        int it = 0;
        while (it < maxit) {
            double pq = 0.0;
            unknowns2([&](int i) { return TPair{apply0(gT, p, i), p[i]}; },
                      [&](int i, const TPair &v) {
                          q[i] = v.a;
                          pq += static_cast<double>(v.b) * static_cast<double>(v.a);
                      });
            pq = red.sum(pq);
            ++it;
            if (!(pq > 0.0) || !isfinite(pq)) {
                *ok = false;
                break;
            }
            const T alpha = static_cast<T>(rz / pq);
            double rz2 = 0.0, rr2 = 0.0;
            if (MG && use_mg) {
                for (int k = threadIdx.x; k < nu; k += NT) {
                    const int i = ul[k];
                    d[i] += alpha * p[i];
                    r[i] -= alpha * q[i];
                }
                __syncthreads();  // the pre-smoothing reads r at the neighbours
                mark(PH_CG);
                vcycle(r, rz2, rr2);
                mark(PH_VCYCLE);
            } else {
                for (int k = threadIdx.x; k < nu; k += NT) {
                    const int i = ul[k];
                    d[i] += alpha * p[i];
                    const T ri = r[i] - alpha * q[i];
                    r[i] = ri;
                    rz2 += static_cast<double>(ri) * static_cast<double>(invd[i] * ri);
                    rr2 += static_cast<double>(ri) * static_cast<double>(ri);
                }
            }
            red.sum2(rz2, rr2);
            if (!isfinite(rr2)) {
                *ok = false;
                break;
            }
            if (rr2 <= stop) break;
            const T beta = static_cast<T>(rz2 / rz);
            rz = rz2;
            if (MG && use_mg) {
                for (int k = threadIdx.x; k < nu; k += NT) {
                    const int i = ul[k];
                    p[i] = q[i] + beta * p[i];
                }
            } else {
                for (int k = threadIdx.x; k < nu; k += NT) {
                    const int i = ul[k];
                    p[i] = invd[i] * r[i] + beta * p[i];
                }
            }
            __syncthreads();
        }
        mark(PH_CG);
        return it;
    }

    // r = b - A x in FP64 over the unknowns (exact weights up to the
    // reciprocal of 2 sqrt 2), stored as T in AR_R; returns (||r||^2, ||b||^2).
    // Copies the NP doubles of a and b (global scratch) to as and bs (shared memory), then a barrier.  Each thread
    // issues all its loads of a round before its stores, so that the loads' latencies overlap (the compiler cannot
    // reorder them past the stores itself: it cannot tell the pointers apart).
    __device__ __forceinline__ void stage2(const double *a, const double *b, double *as, double *bs) {
        constexpr int K = 4;
        for (int i0 = threadIdx.x; i0 < G.NP; i0 += K * NT) {
            double va[K], vb[K];
#pragma unroll
            for (int k = 0; k < K; ++k) {
                const int i = i0 + k * NT;
                va[k] = i < G.NP ? a[i] : 0.0;
                vb[k] = i < G.NP ? b[i] : 0.0;
            }
#pragma unroll
            for (int k = 0; k < K; ++k) {
                const int i = i0 + k * NT;
                if (i < G.NP) {
                    as[i] = va[k];
                    bs[i] = vb[k];
                }
            }
        }
        __syncthreads();
    }

    __device__ __forceinline__ void residual64(double *rr_out, double *bb_out, bool first) {
        if (HOT && !first && a.lay.rstage != kNoStage) {
            // the FP64 conductance and solution live in global scratch and the CG vectors P, Z, Q, D are dead
            // between inner solves: both are copied into them first, so that the stencil reads are on chip
            double *gs = reinterpret_cast<double *>(sm + a.lay.rstage), *xs = gs + G.NP;
            stage2(A<double>(AR_G64), A<double>(AR_X64), gs, xs);
            residual64_from(gs, xs, rr_out, bb_out, false);  // ends with a barrier
            // the CG and the V-cycle read P, Z and Q at cells next to the unknowns: zero again
            T *p = A<T>(AR_P), *q = A<T>(AR_Q), *z = A<T>(AR_Z);
            for (int i = threadIdx.x; i < G.NP; i += NT) {
                p[i] = T(0);
                q[i] = T(0);
                if (MG) z[i] = T(0);
            }
            __syncthreads();
        } else {
            residual64_from(A<double>(AR_G64), A<double>(AR_X64), rr_out, bb_out, first);
        }
    }

    __device__ __forceinline__ void residual64_from(const double *g64, const double *x64, double *rr_out,
                                                    double *bb_out, bool first) {
        const uint8_t *mask = A<uint8_t>(AR_MASK);
        const Idx *ul = A<Idx>(AR_ULIST);
        const double *b64 = A<double>(AR_B64);
        T *r = A<T>(AR_R);
        const bool series = a.series;
        double rr = 0.0, bb = 0.0;
        (void)ul;
        unknowns2(
            [&](int i) {
                const double bi = b64[i];
                double ri = bi;
                if (!first) {
                    // every neighbour is read (padded box: finite values everywhere) and weighted 0 when it is no
                    // node, so that all loads can be in flight together
                    const double gi = g64[i], xi = x64[i];
                    double ao = 0.0, ad = 0.0;
#pragma unroll
                    for (int dd = 0; dd < ND; ++dd) {
                        const int n = i + noff(dd);
                        const bool on = (mask[n] & M_PRESENT) != 0;
                        const double gn = g64[n], xn = x64[n];
                        const double wv = on ? (series ? 2.0 / (1.0 / gi + 1.0 / gn) : gi + gn) : 0.0;
                        if (NB::diag(dd))
                            ad += wv * (xi - xn);
                        else
                            ao += wv * (xi - xn);
                    }
                    const double ax = series ? ao + ad * (1.0 / kSqrt2) : ao * 0.5 + ad * kInvTwoSqrt2;
                    ri = ADV ? bi - (ax + (A<double>(AR_FG64)[i] + kShift) * xi) : bi - (ax + kShift * xi);
                }
                return DPair{ri, bi};
            },
            [&](int i, const DPair &v) {
                r[i] = static_cast<T>(v.a);
                rr += v.a * v.a;
                bb += v.b * v.b;
            });
        red.sum2(rr, bb);
        *rr_out = rr;
        *bb_out = bb;
    }

    // ---- the solve ----------------------------------------------------------
    // x64 must be zero on entry; with setup == false the multigrid hierarchy of the previous solve of the same
    // matrix is reused.
    __device__ __forceinline__ void solve(WinStat *st, bool setup = true) {
        const Idx *ul = A<Idx>(AR_ULIST);
        double *x64 = A<double>(AR_X64);
        const bool want_mg = MG && a.sp.pc == 2;
        mark(PH_ASSEMBLE);
        if (MG && want_mg && setup) mg_setup();
        mark(PH_MG_SETUP);
        int iters = 0, outer = 0, status = 1;
        double rel = 0.0;
        if (!REFINE) {
            // CG on the double operator, from the current iterate: the stopping test of CG reads the recursively
            // updated residual, which drifts from b - A x on ill-conditioned windows, so every run ends with the
            // true FP64 residual, and CG restarts from it (residual replacement) until that meets the tolerance
            T *d = reinterpret_cast<T *>(x64);
            T *r = A<T>(AR_R);
            double rr, bb;
            residual64(&rr, &bb, true);  // r = b (barrier)
            double prev = CUDART_INF;
            bool ok = true;
            while (true) {
                rel = bb > 0 ? sqrt(rr / bb) : 0.0;
                if (!isfinite(rel)) {
                    status = 3;
                    break;
                }
                if (rel <= a.sp.tol) break;
                if (!ok) {
                    status = 3;
                    break;
                }
                // a restart that gained less than half an order has met the FP64 rounding floor: accepted
                // within kFloor x tol, as in the refinement below
                constexpr double kFloor = 100.0;
                if (outer >= a.sp.max_outer || iters >= a.sp.max_iter || rel > 0.5 * prev) {
                    status = rel <= kFloor * a.sp.tol ? 1 : 2;
                    break;
                }
                prev = rel;
                const int budget = a.sp.max_iter - iters;
                iters += pcg(d, r, fmin(0.5, a.sp.tol / rel), budget < 1 ? 1 : budget, want_mg, &ok);
                ++outer;
                __syncthreads();
                residual64(&rr, &bb, false);  // the true residual, into r
            }
        } else {
            T *d = A<T>(AR_D), *r = A<T>(AR_R);
            bool use_mg = want_mg;
            double prev = CUDART_INF;
            int stalls = 0;
            while (true) {
                double rr, bb;
                residual64(&rr, &bb, outer == 0);
                rel = bb > 0 ? sqrt(rr / bb) : 0.0;
                if (!isfinite(rel)) {
                    status = 3;
                    break;
                }
                if (rel <= a.sp.tol) break;
                // FP64 rounding bounds the attainable residual; a solve that stagnates within
                // kFloor x tol has reached it and is accepted
                constexpr double kFloor = 100.0;
                if (outer >= a.sp.max_outer || iters >= a.sp.max_iter) {
                    status = rel <= kFloor * a.sp.tol ? 1 : 2;
                    break;
                }
                stalls = rel > 0.5 * prev ? stalls + 1 : 0;
                if (stalls >= 2) {
                    if (rel <= kFloor * a.sp.tol) break;
                    if (!use_mg) {
                        status = 2;
                        break;
                    }
                    use_mg = false;  // the multigrid-preconditioned inner solve stopped helping: Jacobi
                    stalls = 0;
                }
                prev = rel;
                // scale the residual to unit norm for the inner solve
                const double s = sqrt(rr);
                const T inv = static_cast<T>(1.0 / s);
                for (int k = threadIdx.x; k < nu; k += NT) {
                    const int i = ul[k];
                    r[i] *= inv;
                    d[i] = T(0);
                }
                __syncthreads();
                bool ok = true;
                const int budget = a.sp.max_iter - iters;
                // a multigrid-preconditioned step that needs more than kMgSteps iterations for its 1e-4 has a
                // preconditioner that fails on this window: the stall test below then switches to Jacobi
                constexpr int kMgSteps = 200;
                const int cap = use_mg && budget > kMgSteps ? kMgSteps : budget;
                const int it = pcg(d, r, a.sp.inner_tol, cap < 1 ? 1 : cap, use_mg, &ok);
                iters += it;
                ++outer;
                for (int k = threadIdx.x; k < nu; k += NT) {
                    const int i = ul[k];
                    x64[i] += s * static_cast<double>(d[i]);
                }
                __syncthreads();
                if (!ok && use_mg) use_mg = false;
            }
        }
        if (threadIdx.x == 0 && st) {
            st->iters = iters;
            st->outer = outer;
            st->status = status;
            st->resid = static_cast<float>(rel);
            st->nu = nu;
        }
    }

    // ---- adjoint of J = sum over the window of weight x node current ---------
    // With b_qm = w_qm (v_m - v_q) the branch current into q from m, the node
    // current is cur_q = max(in_q, out_q) over the counted branches
    // (grid.cpp:39-71), so dcur_q/db_qm = s_q(m) in {-1, 0, 1}: +1 for a
    // counted inflow when the inflow wins, -1 for a counted outflow when the
    // outflow wins.  With K_nm = W_n s_n(m) - W_m s_m(n):
    //   dJ/dv_n           = -sum_m w_nm K_nm
    //   dJ/dg_n (explicit) = sum_m dw_nm/dg_n (v_m - v_n) K_nm
    //   dJ/dg_n (through A) = -sum_m dw_nm/dg_n (l_n - l_m)(v_n - v_m),  A l = dJ/dv.
    __device__ __forceinline__ int branch_sel(bool use_in, double b, double maxin, double maxout) const {
        if (use_in) return (b > 0 && !(fabs(b / maxin) < 1e-8)) ? 1 : 0;
        return (b < 0 && !(fabs(b / maxout) < 1e-8)) ? -1 : 0;
    }

    // After the forward solve (x64 = v): J's share of the window, dJ/dv as the right-hand side of the adjoint
    // solve (B64), the explicit dJ/dg (DG64), v kept in V64, x64 cleared.  *any: the window has a nonzero
    // J weight on a node.
    __device__ __forceinline__ double adjoint_prep(bool *any) {
        uint8_t *mask = A<uint8_t>(AR_MASK);
        const double *g64 = A<double>(AR_G64);
        double *v = A<double>(AR_X64), *b64 = A<double>(AR_B64), *v64 = A<double>(AR_V64),
               *cw = A<double>(AR_CW), *dg = A<double>(AR_DG64);
        const bool series = a.series;
        double maxout = -CUDART_INF, maxin = -CUDART_INF;
        for (int i = threadIdx.x; i < G.NP; i += NT) {
            if (!(mask[i] & M_PRESENT)) continue;
            const double gi = g64[i], vi = v[i];
#pragma unroll
            for (int dd = LOWER; dd < ND; ++dd) {
                const int n = i + noff(dd);
                if (!(mask[n] & M_PRESENT)) continue;
                const double b = edge_w64(gi, g64[n], NB::diag(dd), series) * (v[n] - vi);
                if (b > maxout) maxout = b;
                if (-b > maxin) maxin = -b;
            }
        }
        red.max2(maxout, maxin);
        const Threshold tin(maxin), tout(maxout);
        double J = 0.0, wabs = 0.0;
        for (int i = threadIdx.x; i < G.NP; i += NT) {
            const int py = row0(i), y = py - 1, x = i - py * G.P - 1;
            double W = 0.0;
            uint8_t m = mask[i];
            if (y >= 0 && y < G.h && x >= 0 && x < G.w && (m & M_PRESENT)) {
                W = a.weight[(G.y0 + y) * a.nx + (G.x0 + x)];
                const double gi = g64[i], vi = v[i];
                double inflow = 0.0, outflow = 0.0;
#pragma unroll
                for (int dd = 0; dd < ND; ++dd) {
                    const int n = i + noff(dd);
                    if (!(mask[n] & M_PRESENT)) continue;
                    const double b = edge_w64(gi, g64[n], NB::diag(dd), series) * (v[n] - vi);
                    if (b > 0) {
                        if (!tin.below(b)) inflow += b;
                    } else if (b < 0) {
                        if (!tout.below(b)) outflow -= b;
                    }
                }
                J += W * (inflow > outflow ? inflow : outflow);
                wabs += fabs(W);
                m = inflow > outflow ? (m | M_USEIN) : (m & ~M_USEIN);
                mask[i] = m;
            }
            cw[i] = W;
        }
        red.sum2(J, wabs);  // barrier: cw and the M_USEIN bits visible
        *any = wabs > 0.0;
        for (int i = threadIdx.x; i < G.NP; i += NT) {
            const uint8_t mi = mask[i];
            double dvi = 0.0, dgi = 0.0;
            if (mi & M_PRESENT) {
                const double gi = g64[i], vi = v[i], Wi = cw[i];
                const bool ini = (mi & M_USEIN) != 0;
#pragma unroll
                for (int dd = 0; dd < ND; ++dd) {
                    const int n = i + noff(dd);
                    const uint8_t mn = mask[n];
                    if (!(mn & M_PRESENT)) continue;
                    const double gn = g64[n];
                    const double we = edge_w64(gi, gn, NB::diag(dd), series);
                    const double b = we * (v[n] - vi);  // into i from n; from n's side it is -b exactly
                    const double K = Wi * branch_sel(ini, b, maxin, maxout) -
                                     cw[n] * branch_sel((mn & M_USEIN) != 0, -b, maxin, maxout);
                    dvi -= we * K;
                    dgi += edge_dw64(gi, gn, NB::diag(dd), series) * (v[n] - vi) * K;
                }
            }
            b64[i] = (mi & M_UNKNOWN) ? dvi : 0.0;
            dg[i] = dgi;
            v64[i] = v[i];
        }
        __syncthreads();
        for (int i = threadIdx.x; i < G.NP; i += NT) v[i] = 0.0;
        __syncthreads();
        return J;
    }

    // The window's raw source at (y, x) (within radius, NaN as 0, the target block zeroed as load() does).
    __device__ __forceinline__ double raw_source(int y, int x) const {
        const int dy = y - G.gy, dx = x - G.gx, R = a.R, D = a.D, br = a.br;
        double s = 0.0;
        if (dy * dy + dx * dx <= R * R) {
            s = a.src[(G.y0 + y) * a.nx + (G.x0 + x)];
            if (isnan(s)) s = 0.0;
        }
        const int64_t ylim = (D + br < a.ny - 1 ? D + br : a.ny - 1), xlim = (D + br < a.nx - 1 ? D + br : a.nx - 1);
        if (y >= D - br && y <= ylim && x >= D - br && x <= xlim) s = 0.0;
        return s;
    }

    // After the adjoint solve (x64 = l): dJ/d(resistance) of the window to out_r and dJ/d(source) to out_s
    // (h x w each, pitch w), chained through g = 1/r and the source scaling src = raw amps / sum.
    __device__ __forceinline__ void grad_finish(double *out_r, double *out_s, double amps) {
        const uint8_t *mask = A<uint8_t>(AR_MASK);
        const double *g64 = A<double>(AR_G64), *lam = A<double>(AR_X64), *v64 = A<double>(AR_V64),
                     *dg = A<double>(AR_DG64);
        const bool series = a.series;
        double slam = 0.0;
        for (int i = threadIdx.x; i < G.NP; i += NT) {
            const int py = row0(i), y = py - 1, x = i - py * G.P - 1;
            if (y < 0 || y >= G.h || x < 0 || x >= G.w) continue;
            const uint8_t mi = mask[i];
            double dr = 0.0;
            if (mi & M_PRESENT) {
                const double gi = g64[i], li = lam[i], vi = v64[i];
                double dgi = dg[i];
#pragma unroll
                for (int dd = 0; dd < ND; ++dd) {
                    const int n = i + noff(dd);
                    if (!(mask[n] & M_PRESENT)) continue;
                    dgi -= edge_dw64(gi, g64[n], NB::diag(dd), series) * (li - lam[n]) * (vi - v64[n]);
                }
                const double r = a.res[(G.y0 + y) * a.nx + (G.x0 + x)];
                dr = a.ric ? dgi : -dgi / (r * r);
            }
            out_r[y * G.w + x] = dr;
            const double raw = raw_source(y, x);
            if (raw > 0) slam += raw * lam[i];
        }
        slam = red.sum(slam);
        const double sum = src_sum;
        for (int i = threadIdx.x; i < G.NP; i += NT) {
            const int py = row0(i), y = py - 1, x = i - py * G.P - 1;
            if (y < 0 || y >= G.h || x < 0 || x >= G.w) continue;
            const double raw = raw_source(y, x);
            double ds = raw > 0 ? (amps / sum) * lam[i] - (amps / (sum * sum)) * slam : 0.0;
            // amps: the block's sum of sources (NaN skipped) around the target
            const int64_t my = G.y0 + y, mx = G.x0 + x;
            if (my >= G.ty - a.br && my <= G.ty + a.br && mx >= G.tx - a.br && mx <= G.tx + a.br &&
                !isnan(a.src[my * a.nx + mx]))
                ds += slam / sum;
            out_s[y * G.w + x] = ds;
        }
        __syncthreads();
    }

    // ---- 5. node currents (grid.cpp:19-71), correction, output --------------
    // out: h x w doubles (pitch w); corr: W x W factors or null, (cy0, cx0) its
    // slice origin.
    __device__ __forceinline__ void currents(double *out, const double *corr, int cy0, int cx0) {
        mark(PH_RESID);
        const double *g64 = A<double>(AR_G64), *v = A<double>(AR_X64);
        if (HOT && a.lay.stage != kNoStage) {
            // the FP64 conductance and potentials live in global scratch; the solver's vectors and levels are
            // dead now, so both are copied into that shared memory first (then every stencil read is on chip)
            double *gs = reinterpret_cast<double *>(sm + a.lay.stage), *vs = gs + G.NP;
            stage2(g64, v, gs, vs);
            mark(PH_C_STAGE);
            currents_from(gs, vs, out, corr, cy0, cx0);
        } else {
            currents_from(g64, v, out, corr, cy0, cx0);
        }
        mark(PH_CURRENTS);
    }

    __device__ __forceinline__ void currents_from(const double *g64, const double *v, double *out, const double *corr,
                                                  int cy0, int cx0) {
        const uint8_t *mask = A<uint8_t>(AR_MASK);
        const bool series = a.series;
        double maxout = -CUDART_INF, maxin = -CUDART_INF;
        for (int i = threadIdx.x; i < G.NP; i += NT) {
            if (!(mask[i] & M_PRESENT)) continue;
            const double gi = g64[i], vi = v[i];
#pragma unroll
            for (int dd = LOWER; dd < ND; ++dd) {
                const int n = i + noff(dd);
                if (!(mask[n] & M_PRESENT)) continue;
                const double b = edge_w64(gi, g64[n], NB::diag(dd), series) * (v[n] - vi);
                if (b > maxout) maxout = b;
                if (-b > maxin) maxin = -b;
            }
        }
        red.max2(maxout, maxin);
        mark(PH_C_MAX);
        const Threshold tin(maxin), tout(maxout);
        const int W = a.W;
        for (int i = threadIdx.x; i < G.NP; i += NT) {
            const int py = row0(i), y = py - 1, x = i - py * G.P - 1;
            if (y < 0 || y >= G.h || x < 0 || x >= G.w) continue;
            double c = 0.0;
            if (mask[i] & M_PRESENT) {
                const double gi = g64[i], vi = v[i];
                double inflow = 0.0, outflow = 0.0;
#pragma unroll
                for (int dd = 0; dd < ND; ++dd) {
                    const int n = i + noff(dd);
                    if (!(mask[n] & M_PRESENT)) continue;
                    const double b = edge_w64(gi, g64[n], NB::diag(dd), series) * (v[n] - vi);
                    if (b > 0) {
                        if (!tin.below(b)) inflow += b;
                    } else if (b < 0) {
                        if (!tout.below(b)) outflow -= b;
                    }
                }
                if (ADV) {
                    // current to a finite ground, never thresholded (grid.cpp:19-71)
                    const double f = A<double>(AR_FG64)[i] * vi;
                    if (f < 0)
                        inflow -= f;
                    else if (f > 0)
                        outflow += f;
                }
                c = inflow > outflow ? inflow : outflow;
                if (corr) c *= corr[(cy0 + y) * W + (cx0 + x)];
                if (ADV) volt_out[y * G.w + x] = vi;
            }
            if (!ADV || (mask[i] & M_PRESENT)) out[y * G.w + x] = c;  // a raster solve writes its component only
        }
        __syncthreads();
    }

    // ---- whole-raster solves (advanced mode, grid.cpp:73-210) -------------------------------------------------
    double *volt_out = nullptr;  // the raster's voltage map (pitch w)

    // Conductance (a node where > 0), sources (0 where the cell is also grounded), finite and direct grounds of
    // the raster at g, s, gr (h x w, pitch w); the outputs start as current 0 and voltage 0 on nodes, NaN off
    // them.  (The reference adds the finite grounds to the diagonal when any is nonzero; zero entries change
    // nothing, so they are always added here.)
    __device__ __forceinline__ void load_raster(const double *g, const double *s, const double *gr, double *cur) {
        uint8_t *mask = A<uint8_t>(AR_MASK);
        double *g64 = A<double>(AR_G64), *x64 = A<double>(AR_X64), *b64 = A<double>(AR_B64),
               *fg = A<double>(AR_FG64);
        const int P = G.P;
        invP = 1.0f / static_cast<float>(P);
        for (int i = threadIdx.x; i < G.NP; i += NT) {
            const int py = row0(i), y = py - 1, x = i - py * P - 1;
            double gi = 0.0, si = 0.0, fi = 0.0;
            uint8_t m = 0;
            if (y >= 0 && y < G.h && x >= 0 && x < G.w) {
                const int c = y * G.w + x;
                gi = g[c];
                const bool node = gi > 0;
                cur[c] = 0.0;
                volt_out[c] = node ? 0.0 : CUDART_NAN;
                if (node) {
                    m = M_CAND;
                    const double gc = gr[c];
                    si = s[c];
                    if (gc != 0) si = 0.0;  // a grounded cell loses its source
                    if (gc == CUDART_INF)
                        m |= M_DIRECT;
                    else
                        fi = gc;
                } else {
                    gi = -9999.0;  // no node (never read as a conductance)
                }
            }
            mask[i] = m;
            g64[i] = gi;
            b64[i] = si;
            fg[i] = fi;
            x64[i] = 0.0;
        }
        __syncthreads();
    }

    // Smallest padded index of a node whose component is not handled yet, or -1.
    __device__ __forceinline__ int next_seed() {
        const uint8_t *mask = A<uint8_t>(AR_MASK);
        int best = 0x7fffffff;
        for (int i = threadIdx.x; i < G.NP; i += NT)
            if ((mask[i] & (M_CAND | M_DONE)) == M_CAND) {
                best = i;
                break;
            }
        scan[0] = 0x7fffffff;
        __syncthreads();
        atomicMin(&scan[0], best);
        __syncthreads();
        const int s = scan[0];
        __syncthreads();
        return s == 0x7fffffff ? -1 : s;
    }

    // The component of `seed` among the nodes not handled yet: bit rows as in flood(); its cells get M_PRESENT
    // and M_DONE.
    __device__ __forceinline__ void flood_from(int seed) {
        uint8_t *mask = A<uint8_t>(AR_MASK);
        const int P = G.P, words = (P + 31) >> 5, nrow = G.h + 2, ntask = nrow * words;
        const float invwd = 1.0f / static_cast<float>(words);
        uint32_t *cb = reinterpret_cast<uint32_t *>(A<T>(AR_P)), *pb = cb + ntask;
        const int spy = row0(seed), spx = seed - spy * P;
        const int lane = threadIdx.x & 31;
        for (int k = threadIdx.x >> 5; k < ntask; k += NT / 32) {
            const int py = static_cast<int>((static_cast<float>(k) + 0.5f) * invwd), w = k - py * words;
            const int px = 32 * w + lane;
            const bool c = px < P && (mask[py * P + px] & (M_CAND | M_DONE)) == M_CAND;
            const uint32_t bits = __ballot_sync(0xffffffffu, c);
            if (lane == 0) {
                cb[k] = bits;
                pb[k] = (py == spy && w == (spx >> 5)) ? (1u << (spx & 31)) : 0u;
            }
        }
        __syncthreads();
        volatile uint32_t *vp = pb;
        while (true) {
            int changed = 0;
            for (int k = threadIdx.x; k < ntask; k += NT) {
                const uint32_t c = cb[k];
                if (!c) continue;
                const int py = static_cast<int>((static_cast<float>(k) + 0.5f) * invwd), w = k - py * words;
                const uint32_t mid = vp[k];
                const bool hl = w > 0, hr = w + 1 < words;
                uint32_t nb;
                if (FOUR) {
                    const uint32_t l = hl ? vp[k - 1] : 0u, r = hr ? vp[k + 1] : 0u;
                    nb = vp[k - words] | vp[k + words] | (mid << 1) | (l >> 31) | (mid >> 1) | (r << 31);
                } else {
                    const uint32_t v = vp[k - words] | mid | vp[k + words];
                    const uint32_t vl = hl ? (vp[k - words - 1] | vp[k - 1] | vp[k + words - 1]) : 0u;
                    const uint32_t vr = hr ? (vp[k - words + 1] | vp[k + 1] | vp[k + words + 1]) : 0u;
                    nb = v | (v << 1) | (vl >> 31) | (v >> 1) | (vr << 31);
                }
                (void)py;
                const uint32_t nw = c & (mid | nb);
                if (nw != mid) {
                    vp[k] = nw;
                    changed = 1;
                }
            }
            if (!__syncthreads_or(changed)) break;
        }
        for (int i = threadIdx.x; i < G.NP; i += NT) {
            const int py = row0(i), px = i - py * P;
            const uint8_t m = mask[i] & static_cast<uint8_t>(~(M_PRESENT | M_UNKNOWN));
            mask[i] = ((pb[py * words + (px >> 5)] >> (px & 31)) & 1u) ? (m | M_PRESENT | M_DONE) : m;
        }
        __syncthreads();
    }

    // The component's source sum and whether it has a ground (a direct one, or finite ones summing to nonzero).
    __device__ __forceinline__ bool component_active() {
        const uint8_t *mask = A<uint8_t>(AR_MASK);
        const double *b64 = A<double>(AR_B64), *fg = A<double>(AR_FG64);
        double s = 0.0, gs = 0.0;
        for (int i = threadIdx.x; i < G.NP; i += NT) {
            const uint8_t m = mask[i];
            if (!(m & M_PRESENT)) continue;
            s += b64[i];
            gs += (m & M_DIRECT) ? CUDART_INF : fg[i];
        }
        red.sum2(s, gs);
        return s != 0 && gs != 0;
    }

    // After a component: its potentials back to zero (the next solve starts from x = 0).
    __device__ __forceinline__ void clear_solution() {
        double *x64 = A<double>(AR_X64);
        for (int i = threadIdx.x; i < G.NP; i += NT) x64[i] = 0.0;
        __syncthreads();
    }
};

}  // namespace lsb
