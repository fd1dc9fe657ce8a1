// omni_windows.cuh -- the persistent window kernel: each CTA pulls targets
// from a queue and solves their windows (omni_solver.cuh), the landscape and,
// when asked, the flow potential; mode 1 solves the two windows of the
// block-artifact correction instead.
#pragma once

#include "omni_solver.cuh"

namespace lsb {

using KernelFn = void (*)(const KArgs);

// ---------------------------------------------------------------------------
// The persistent window solver.
// ---------------------------------------------------------------------------
template <int NT, typename T, bool FOUR, bool MG, bool REFINE>
__global__ void __launch_bounds__(NT) k_windows(const KArgs a) {
    extern __shared__ __align__(16) char smem[];
    __shared__ double red_buf[128];
    __shared__ int scan_buf[64];
    __shared__ int lvh[kMaxLevels], lvw[kMaxLevels];
    __shared__ int item_s;
    char *gm = a.gscratch + static_cast<size_t>(blockIdx.x) * a.lay.gmem_bytes;
    Reducer<NT> red{red_buf, 0};
    Win<NT, T, FOUR, MG, REFINE> win(a, smem, gm, red, scan_buf, lvh, lvw);
    int count;
    if (a.mode == 1) {
        count = 2;
    } else {
        count = *a.count_ptr - a.batch_start;
        if (count > a.batch_size) count = a.batch_size;
    }
    const int W = a.W, D = a.D;
    while (true) {
        if (threadIdx.x == 0) item_s = atomicAdd(a.queue, 1);
        __syncthreads();
        const int item = item_s;
        __syncthreads();
        if (item >= count) break;
        WinGeom &G = win.G;
        if (a.mode == 1) {
            G.h = G.w = W;
            G.gy = G.gx = D;
            G.y0 = G.x0 = 0;
            G.ty = G.tx = D;
            G.P = W + 2;
            G.NP = (W + 2) * (W + 2);
            const int kind = item == 0 ? KIND_CORR_BLOCK : KIND_CORR_NULL;
            win.load(kind, 0.0);
            WinStat *st = a.stat + item;
            if (win.flood(kind) && win.mark_unknowns() != 0.0) {
                win.assemble();
                win.solve(st);
                win.currents(a.cur_win + static_cast<size_t>(item) * W * W, nullptr, 0, 0);
            } else if (threadIdx.x == 0) {
                *st = WinStat{0, 0, 0, 0.f};
            }
            continue;
        }
        const int t = a.batch_start + item;
        const int L = a.targets[t];
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
        G.P = G.w + 2;
        G.NP = (G.h + 2) * G.P;
        // the part of the correction under the (clipped) window (omniscape.cpp:559-563)
        const int cx0 = (tx < D && tx + D <= a.nx - 1) ? W - G.w : 0;
        const int cy0 = (ty < D && ty + D <= a.ny - 1) ? W - G.h : 0;
        const double *corr = a.correct ? a.corr : nullptr;
        // the landscape window
        win.load(KIND_LAND, a.lat_amps[L]);
        if (a.cond_present[0]) win.apply_conditions(a.cond_val[2 * t], a.cond_val[2 * t + 1]);
        WinStat *st = a.stat + 2 * static_cast<int64_t>(t);
        if (win.flood(KIND_LAND) && win.mark_unknowns() != 0.0) {
            win.assemble();
            win.solve(st);
            win.currents(a.cur_win + static_cast<size_t>(item) * W * W, corr, cy0, cx0);
        } else if (threadIdx.x == 0) {
            *st = WinStat{0, 0, 0, 0.f};
        }
        if (a.fp) {
            // the flow potential: conductance 1 on the whole rectangle (omniscape.cpp:127-166)
            win.load(KIND_FLOW, 0.0);
            win.flood(KIND_FLOW);
            if (win.mark_unknowns() != 0.0) {
                win.assemble();
                win.solve(st + 1);
                win.currents(a.fp_win + static_cast<size_t>(item) * W * W, corr, cy0, cx0);
            } else if (threadIdx.x == 0) {
                st[1] = WinStat{0, 0, 0, 0.f};
            }
        }
    }
}


// One translation unit per block size instantiates the variants of that size.
KernelFn pick_windows_256(bool four, bool dbl, bool mg);
KernelFn pick_windows_512(bool four, bool dbl, bool mg);
KernelFn pick_windows_1024(bool four, bool dbl, bool mg);

template <int NT>
KernelFn pick_windows_nt(bool four, bool dbl, bool mg) {
    if (four) {
        if (dbl) return mg ? k_windows<NT, double, true, true, false> : k_windows<NT, double, true, false, false>;
        return mg ? k_windows<NT, float, true, true, true> : k_windows<NT, float, true, false, true>;
    }
    if (dbl) return mg ? k_windows<NT, double, false, true, false> : k_windows<NT, double, false, false, false>;
    return mg ? k_windows<NT, float, false, true, true> : k_windows<NT, float, false, false, true>;
}

}  // namespace lsb
