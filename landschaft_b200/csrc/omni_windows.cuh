// omni_windows.cuh -- the persistent window kernel: each CTA pulls targets
// from a queue and solves their windows (omni_solver.cuh), the landscape and,
// when asked, the flow potential; mode 1 solves the two windows of the
// block-artifact correction instead.
#pragma once

#include "omni_solver.cuh"

namespace lsb {


// ---------------------------------------------------------------------------
// The persistent window solver.
// ---------------------------------------------------------------------------
template <int NT, typename T, bool FOUR, bool MG, bool REFINE, bool HOT>
__global__ void __launch_bounds__(NT, NT == 128 ? 4 : 1) k_windows(const KArgs a) {
    extern __shared__ __align__(16) char smem[];
    __shared__ double red_buf[128];
    __shared__ int scan_buf[64];
    __shared__ int lvh[kMaxLevels], lvw[kMaxLevels];
    __shared__ float lvinv[kMaxLevels];
    __shared__ uint32_t lvoff[(kMaxLevels - 1) * LV_COUNT];
    for (int k = threadIdx.x; k < (kMaxLevels - 1) * LV_COUNT; k += NT) lvoff[k] = a.lay.off[AR_LEVEL + k];
    __shared__ short cidx[kNcMax];
    __shared__ int item_s;
    char *gm = a.gscratch + static_cast<size_t>(blockIdx.x) * a.lay.gmem_bytes;
    Reducer<NT> red{red_buf, 0};
    Win<NT, T, FOUR, MG, REFINE, HOT> win(a, smem, gm, red, scan_buf, lvh, lvw, lvinv, lvoff, cidx);
#ifdef LSB_PHASE_TIMERS
    __shared__ unsigned long long tacc[PH_COUNT + 1];
    if (threadIdx.x <= PH_COUNT) tacc[threadIdx.x] = threadIdx.x == PH_COUNT ? clock64() : 0ull;
    __syncthreads();
    win.tacc = tacc;
    if (blockIdx.x == 0 && a.timers) {
        // calibration: 64 bare barriers, then 64 barrier-separated shared-memory round trips
        __shared__ float cal[64];  // small: the timers build must fit the layouts that fill shared memory
        unsigned long long t0 = clock64();
        for (int k = 0; k < 64; ++k) __syncthreads();
        unsigned long long t1 = clock64();
        for (int k = 0; k < 64; ++k) {
            if (threadIdx.x < 64) cal[threadIdx.x] = cal[(threadIdx.x + 1) & 63] + 1.0f;
            __syncthreads();
        }
        unsigned long long t2 = clock64();
        if (threadIdx.x == 0) {
            a.timers[30] = (t1 - t0) / 64;
            a.timers[31] = (t2 - t1) / 64;
        }
        __syncthreads();
    }
#endif
    int count;
    if (a.mode == 1) {
        count = 2;
    } else {
        const int last = (a.target_end > 0 && a.target_end < *a.count_ptr) ? a.target_end : *a.count_ptr;
        count = last - a.batch_start;
        if (count > a.batch_size) count = a.batch_size;
    }
    const int W = a.W, D = a.D;
    // Every item runs one or two jobs (the landscape, then the flow potential; or one correction window)
    // through a single code path, so that the solver is expanded once in the kernel.
    int item = 0, job = 0, njobs = 0;
    int t = 0, L = 0, cy0 = 0, cx0 = 0;
    bool adj_go = false;  // mode 2: the forward window has a J weight on a node
    while (true) {
        if (job == njobs) {
            if (threadIdx.x == 0) item_s = atomicAdd(a.queue, 1);
            __syncthreads();
            item = item_s;
            __syncthreads();
            if (item >= count) break;
            job = 0;
            WinGeom &G = win.G;
            if (a.mode == 1) {
                njobs = 1;
                G.h = G.w = W;
                G.gy = G.gx = D;
                G.y0 = G.x0 = 0;
                G.ty = G.tx = D;
            } else {
                njobs = (a.fp || a.mode == 2) ? 2 : 1;
                t = a.batch_start + item;
                L = a.targets[t];
                const int ix = L / a.nby, iy = L - ix * a.nby;
                const int64_t tx = a.br + static_cast<int64_t>(ix) * a.bs, ty = a.br + static_cast<int64_t>(iy) * a.bs;
                G.ty = ty;
                G.tx = tx;
                G.y0 = ty - D > 0 ? ty - D : 0;
                G.x0 = tx - D > 0 ? tx - D : 0;
                const int64_t y1 = ty + D < a.ny - 1 ? ty + D : a.ny - 1, x1 = tx + D < a.nx - 1 ? tx + D : a.nx - 1;
                G.h = static_cast<int>(y1 - G.y0 + 1);
                G.w = static_cast<int>(x1 - G.x0 + 1);
                G.gy = static_cast<int>(ty - G.y0);
                G.gx = static_cast<int>(tx - G.x0);
                // the part of the correction under the (clipped) window (omniscape.cpp:559-563)
                cx0 = (tx < D && tx + D <= a.nx - 1) ? W - G.w : 0;
                cy0 = (ty < D && ty + D <= a.ny - 1) ? W - G.h : 0;
            }
            G.P = G.w + 2;
            G.NP = (G.h + 2) * G.P;
        }
        int kind;
        WinStat *st;
        double *out;
        const double *corr = nullptr;
        // mode 2: job 0 solves the forward window, job 1 its adjoint on the same window state
        const bool adjoint = a.mode == 2 && job == 1;
        if (a.mode == 1) {
            kind = item == 0 ? KIND_CORR_BLOCK : KIND_CORR_NULL;
            st = a.stat + item;
            out = a.cur_win + static_cast<size_t>(item) * W * W;
        } else {
            // the landscape window, then the flow potential: conductance 1 on the whole rectangle
            // (omniscape.cpp:127-166), with the sources the landscape pass scaled
            kind = (a.mode == 0 && job == 1) ? KIND_FLOW : KIND_LAND;
            st = a.stat + 2 * static_cast<int64_t>(t) + job;
            out = (job == 0 ? a.cur_win : a.fp_win) + static_cast<size_t>(item) * W * W;
            corr = a.correct ? a.corr : nullptr;
        }
        ++job;
        bool solvable;
        if (adjoint) {
            solvable = adj_go;
        } else {
            win.mark(PH_OTHER);
            win.load(kind, kind == KIND_LAND ? a.lat_amps[L] : 0.0);
            if (kind == KIND_LAND && a.cond_present[0]) win.apply_conditions(a.cond_val[2 * t], a.cond_val[2 * t + 1]);
            win.mark(PH_LOAD);
            const bool ok = win.flood(kind);
            win.mark(PH_FLOOD);
            solvable = ok && win.mark_unknowns() != 0.0;
            if (solvable) {
                win.mark(PH_MARK);
                win.assemble();
            }
        }
        if (solvable) {
            win.solve(st, !adjoint);
            if (a.mode != 2) {
                win.currents(out, corr, cy0, cx0);
            } else if (!adjoint) {
                bool any = false;
                const double J = win.adjoint_prep(&any);
                if (threadIdx.x == 0) {
                    a.Jw[t] = J;
                    if (!any) st->status = 0;  // no gradient window: the gather skips it
                }
                adj_go = any;
            } else {
                win.grad_finish(a.cur_win + static_cast<size_t>(item) * W * W,
                                a.fp_win + static_cast<size_t>(item) * W * W, a.lat_amps[L]);
            }
        } else {
            if (threadIdx.x == 0) {
                *st = WinStat{0, 0, 0, 0.f, 0};
                if (a.mode == 2 && !adjoint) a.Jw[t] = 0.0;
            }
            if (a.mode == 2 && !adjoint) adj_go = false;
        }
    }
#ifdef LSB_PHASE_TIMERS
    win.mark(PH_OTHER);
    if (a.timers && threadIdx.x < PH_COUNT) atomicAdd(a.timers + threadIdx.x, tacc[threadIdx.x]);
#endif
}


// One translation unit per block size and layout kind instantiates the variants of that kind.
KernelFn pick_windows_128_hot(bool four, bool dbl, bool mg);
KernelFn pick_windows_256_hot(bool four, bool dbl, bool mg);
KernelFn pick_windows_256_gen(bool four, bool dbl, bool mg);
KernelFn pick_windows_512_hot(bool four, bool dbl, bool mg);
KernelFn pick_windows_512_gen(bool four, bool dbl, bool mg);

template <int NT, bool HOT>
KernelFn pick_windows_nt(bool four, bool dbl, bool mg) {
    if (four) {
        if (dbl)
            return mg ? k_windows<NT, double, true, true, false, HOT> : k_windows<NT, double, true, false, false, HOT>;
        return mg ? k_windows<NT, float, true, true, true, HOT> : k_windows<NT, float, true, false, true, HOT>;
    }
    if (dbl) return mg ? k_windows<NT, double, false, true, false, HOT> : k_windows<NT, double, false, false, false, HOT>;
    return mg ? k_windows<NT, float, false, true, true, HOT> : k_windows<NT, float, false, false, true, HOT>;
}

}  // namespace lsb
