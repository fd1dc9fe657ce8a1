// omni_kernels.cuh -- the kernels of one Omniscape call.
//
//   k_lattice_amps   block sums of the sources on the target lattice
//                    (omniscape.cpp:406-416, column-major sum, NaN skipped)
//   k_scan_count / k_scan_offsets / k_scan_write
//                    ordered compaction of the blocks with a positive sum into
//                    the target list (lattice order = the reference's
//                    enumeration order: x outer, y inner)
//   k_block_cond     per target, the block's condition values (median or mode)
//   k_windows        the persistent window solver (omni_windows.cuh)
//   k_corr_ratio     the block-artifact correction from its two windows
//   k_gather         adds a batch of windows into the maps, every cell summing
//                    its windows in target order (deterministic, no atomics)
//   k_finish         normalised current and the NoData mask
//   k_stats          aggregates the per-window statistics
#pragma once

#include "omni_solver.cuh"

namespace lsb {

// ---------------------------------------------------------------------------
// Targets.
// ---------------------------------------------------------------------------
__global__ void k_lattice_amps(const double *__restrict__ src, int64_t nx, int64_t ny, int bs, int br, int nbx,
                               int nby, double *__restrict__ amps) {
    const int64_t L = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (L >= static_cast<int64_t>(nbx) * nby) return;
    const int ix = static_cast<int>(L / nby), iy = static_cast<int>(L - static_cast<int64_t>(ix) * nby);
    const int64_t x = br + static_cast<int64_t>(ix) * bs, y = br + static_cast<int64_t>(iy) * bs;
    double s = 0.0;
    for (int64_t xx = x - br; xx <= x + br; ++xx)
        for (int64_t yy = y - br; yy <= y + br; ++yy) {
            const double v = src[yy * nx + xx];
            if (!isnan(v)) s += v;
        }
    amps[L] = s;
}

constexpr int kScanBlock = 1024;

__global__ void __launch_bounds__(kScanBlock) k_scan_count(const double *__restrict__ amps, int64_t NL,
                                                           int *__restrict__ part) {
    __shared__ int warp_c[32];
    const int64_t L = blockIdx.x * static_cast<int64_t>(kScanBlock) + threadIdx.x;
    const bool f = L < NL && amps[L] > 0;
    const unsigned m = __ballot_sync(0xffffffffu, f);
    if ((threadIdx.x & 31) == 0) warp_c[threadIdx.x >> 5] = __popc(m);
    __syncthreads();
    if (threadIdx.x == 0) {
        int s = 0;
        for (int k = 0; k < kScanBlock / 32; ++k) s += warp_c[k];
        part[blockIdx.x] = s;
    }
}

// One CTA: exclusive scan of the per-block counts; the total goes to *count.
__global__ void __launch_bounds__(1024) k_scan_offsets(int *__restrict__ part, int nparts, int *__restrict__ count) {
    __shared__ int warp_c[32];
    __shared__ int carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int c0 = 0; c0 < nparts; c0 += 1024) {
        const int i = c0 + threadIdx.x;
        const int v = i < nparts ? part[i] : 0;
        int incl = v;
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int t = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += t;
        }
        if (lane == 31) warp_c[warp] = incl;
        __syncthreads();
        int before = 0, total = 0;
        for (int k = 0; k < 32; ++k) {
            before += k < warp ? warp_c[k] : 0;
            total += warp_c[k];
        }
        const int base = carry;
        if (i < nparts) part[i] = base + before + incl - v;
        __syncthreads();
        if (threadIdx.x == 0) carry = base + total;
        __syncthreads();
    }
    if (threadIdx.x == 0) *count = carry;
}

__global__ void __launch_bounds__(kScanBlock) k_scan_write(const double *__restrict__ amps, int64_t NL,
                                                           const int *__restrict__ part, int *__restrict__ tindex,
                                                           int *__restrict__ targets) {
    __shared__ int warp_c[32];
    const int64_t L = blockIdx.x * static_cast<int64_t>(kScanBlock) + threadIdx.x;
    const bool f = L < NL && amps[L] > 0;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const unsigned m = __ballot_sync(0xffffffffu, f);
    if (lane == 0) warp_c[warp] = __popc(m);
    __syncthreads();
    int before = 0;
    for (int k = 0; k < warp; ++k) before += warp_c[k];
    const int idx = part[blockIdx.x] + before + __popc(m & ((1u << lane) - 1u));
    if (L < NL) tindex[L] = f ? idx : -1;
    if (f) targets[idx] = static_cast<int>(L);
}

// ---------------------------------------------------------------------------
// Conditions: the target block's value (omniscape.cpp:170-215): median
// ("within", a/2 + b/2 for an even count) or StatsBase mode ("equal": the first
// value in column-major order to reach the highest count; bit patterns
// compared).  At most kMaxCondCells values per block.
// ---------------------------------------------------------------------------
constexpr int kMaxCondCells = 961;  // block_size <= 31

// The k-th smallest (0-based) of the non-NaN values of a block, by counting
// (no buffer: every value is compared with every other).
__device__ double block_kth(const double *f, int64_t nx, int64_t x0, int64_t x1, int64_t y0, int64_t y1, int k) {
    for (int64_t xa = x0; xa <= x1; ++xa)
        for (int64_t ya = y0; ya <= y1; ++ya) {
            const double v = f[ya * nx + xa];
            if (isnan(v)) continue;
            int less = 0, equal = 0;
            for (int64_t xb = x0; xb <= x1; ++xb)
                for (int64_t yb = y0; yb <= y1; ++yb) {
                    const double u = f[yb * nx + xb];
                    less += u < v;
                    equal += u == v;
                }
            if (less <= k && k < less + equal) return v;
        }
    return CUDART_NAN;
}

__global__ void k_block_cond(const KArgs a, double *__restrict__ out, int *__restrict__ error) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= *a.count_ptr) return;
    const int L = a.targets[t];
    const int ix = L / a.nby, iy = L - ix * a.nby;
    const int64_t x = a.br + static_cast<int64_t>(ix) * a.bs, y = a.br + static_cast<int64_t>(iy) * a.bs;
    const int64_t x0 = x - a.br, y0 = y - a.br;
    const int64_t x1 = x + a.br < a.nx - 1 ? x + a.br : a.nx - 1, y1 = y + a.br < a.ny - 1 ? y + a.br : a.ny - 1;
    for (int k = 0; k < 2; ++k) {
        out[2 * static_cast<int64_t>(t) + k] = 0.0;
        const double *pres = a.cond_present[k];
        if (!pres) continue;
        const double *f = a.cond_future[k] ? a.cond_future[k] : pres;
        int n = 0;
        for (int64_t xx = x0; xx <= x1; ++xx)
            for (int64_t yy = y0; yy <= y1; ++yy) n += !isnan(f[yy * a.nx + xx]);
        if (n == 0) {
            atomicExch(error, 1);
            continue;
        }
        double value;
        if (!a.cond_equal[k]) {
            // Statistics.median: the middle value, or a/2 + b/2 of the two middle ones
            if (n & 1) {
                value = block_kth(f, a.nx, x0, x1, y0, y1, n / 2);
            } else {
                const double lo = block_kth(f, a.nx, x0, x1, y0, y1, n / 2 - 1);
                const double hi = block_kth(f, a.nx, x0, x1, y0, y1, n / 2);
                value = lo / 2 + hi / 2;
            }
        } else {
            // StatsBase.mode: the first value (column-major) to exceed the running highest
            // count, values compared by bit pattern
            value = CUDART_NAN;
            int top = 0;
            for (int64_t xa = x0; xa <= x1; ++xa)
                for (int64_t ya = y0; ya <= y1; ++ya) {
                    const double v = f[ya * a.nx + xa];
                    if (isnan(v)) continue;
                    const long long bv = __double_as_longlong(v);
                    int cnt = 0;  // occurrences up to and including this one
                    bool done = false;
                    for (int64_t xb = x0; xb <= x1 && !done; ++xb)
                        for (int64_t yb = y0; yb <= y1; ++yb) {
                            const double u = f[yb * a.nx + xb];
                            if (!isnan(u) && __double_as_longlong(u) == bv) ++cnt;
                            if (xb == xa && yb == ya) {
                                done = true;
                                break;
                            }
                        }
                    if (cnt > top) {
                        top = cnt;
                        value = v;
                    }
                }
        }
        out[2 * static_cast<int64_t>(t) + k] = value;
    }
}

// ---------------------------------------------------------------------------
// Correction factors (omniscape.cpp:369-391) from the block window (slot 0)
// and the null window (slot 1).  One CTA.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(1024) k_corr_ratio(const double *__restrict__ win, const WinStat *__restrict__ st,
                                                     int W, int bs, double *__restrict__ corr) {
    __shared__ double red_buf[128];
    Reducer<1024> red{red_buf, 0};
    const int n = W * W, br = (bs - 1) / 2;
    const double *block = win, *null_ = win + n;
    const bool have_block = st[0].status != 0, have_null = st[1].status != 0;
    double top = -CUDART_INF;
    for (int i = threadIdx.x; i < n; i += 1024) top = fmax(top, have_block ? block[i] : 0.0);
    top = red.max(top);
    const double floor_ = 1e-6 * top;
    for (int i = threadIdx.x; i < n; i += 1024) {
        const int y = i / W, x = i - y * W;
        double b = have_block ? block[i] : 0.0;
        // null current total of the block's targets (i, then j), cut to the window
        double t = 0.0;
        const int Y = y + br, X = x + br;
        for (int ii = 0; ii < bs; ++ii)
            for (int jj = 0; jj < bs; ++jj) {
                const int yy = Y - ii, xx = X - jj;
                if (yy >= 0 && yy < W && xx >= 0 && xx < W) t += have_null ? null_[yy * W + xx] : 0.0;
            }
        if (b <= floor_) b = 0.0;
        if (b == 0.0) t = 0.0;
        if (t == 0.0) t = 1.0;
        if (b == 0.0) b = 1.0;
        corr[i] = t / b;
    }
}

// ---------------------------------------------------------------------------
// Scatter as a gather: every cell adds, in target order, the windows of the
// batch that cover it.  Tiles of 32 x 8 cells; 256 threads.
// ---------------------------------------------------------------------------
constexpr int kGatherTX = 32, kGatherTY = 8;

__global__ void __launch_bounds__(kGatherTX *kGatherTY) k_gather(const KArgs a, const int *__restrict__ tindex,
                                                                 double *__restrict__ cum, double *__restrict__ fpmap) {
    const int64_t X0 = static_cast<int64_t>(blockIdx.x) * kGatherTX, Y0 = static_cast<int64_t>(blockIdx.y) * kGatherTY;
    const int64_t X = X0 + (threadIdx.x % kGatherTX), Y = Y0 + (threadIdx.x / kGatherTX);
    const bool in = X < a.nx && Y < a.ny;
    const int last = (a.target_end > 0 && a.target_end < *a.count_ptr) ? a.target_end : *a.count_ptr;
    const int n_batch = min(last - a.batch_start, a.batch_size);
    if (n_batch <= 0) return;
    const int D = a.D, bs = a.bs, br = a.br, W = a.W;
    const int64_t X1 = X0 + kGatherTX - 1, Y1 = Y0 + kGatherTY - 1;
    // lattice points whose windows can reach the tile: |t - cell| <= D
    auto lo = [&](int64_t c) { const int64_t v = c - D - br; return v <= 0 ? int64_t(0) : (v + bs - 1) / bs; };
    auto hi = [&](int64_t c, int nb) { const int64_t v = (c + D - br); if (v < 0) return int64_t(-1); const int64_t k = v / bs; return k < nb - 1 ? k : int64_t(nb - 1); };
    const int64_t ix0 = lo(X0), ix1 = hi(X1, a.nbx), iy0 = lo(Y0), iy1 = hi(Y1, a.nby);
    // each window is added to the running map value in target order, so that batches do not change the bits
    double c = in ? cum[Y * a.nx + X] : 0.0, f = (in && fpmap) ? fpmap[Y * a.nx + X] : 0.0;
    for (int64_t ix = ix0; ix <= ix1; ++ix) {
        const int64_t tx = br + ix * bs;
        const int64_t x0 = tx - D > 0 ? tx - D : 0, x1 = tx + D < a.nx - 1 ? tx + D : a.nx - 1;
        for (int64_t iy = iy0; iy <= iy1; ++iy) {
            const int t = tindex[ix * a.nby + iy];
            if (t < a.batch_start || t >= a.batch_start + n_batch) continue;
            const int64_t ty = br + iy * bs;
            const int64_t y0 = ty - D > 0 ? ty - D : 0, y1 = ty + D < a.ny - 1 ? ty + D : a.ny - 1;
            if (!in || X < x0 || X > x1 || Y < y0 || Y > y1) continue;
            const int w = static_cast<int>(x1 - x0 + 1);
            const size_t off = static_cast<size_t>(t - a.batch_start) * W * W + (Y - y0) * w + (X - x0);
            if (a.stat[2 * static_cast<int64_t>(t)].status != 0) c += a.cur_win[off];
            if (fpmap && a.stat[2 * static_cast<int64_t>(t) + 1].status != 0) f += a.fp_win[off];
        }
    }
    if (in) {
        cum[Y * a.nx + X] = c;
        if (fpmap) fpmap[Y * a.nx + X] = f;
    }
}

// Normalised current (cum / fp, NaN -> 0; omniscape.py:380-384) and the NoData mask (:387-389).
__global__ void k_finish(const double *__restrict__ res, int64_t n, double *__restrict__ cum, double *__restrict__ fpmap,
                         double *__restrict__ norm, int mask_nodata) {
    const int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    const bool nod = mask_nodata && isnan(res[i]);
    const double c = cum[i];
    if (norm) {
        double v = c / fpmap[i];
        if (isnan(v)) v = 0.0;
        norm[i] = nod ? CUDART_NAN : v;
    }
    if (nod) {
        cum[i] = CUDART_NAN;
        if (fpmap) fpmap[i] = CUDART_NAN;
    }
}

// Sum of the targets' shares of J (one CTA, fixed order): *out = sum over t < count of Jw[t].
__global__ void __launch_bounds__(1024) k_sum_targets(const double *__restrict__ Jw, const int *__restrict__ count_ptr,
                                                      double *__restrict__ out) {
    __shared__ double red_buf[128];
    Reducer<1024> red{red_buf, 0};
    const int n = *count_ptr;
    double s = 0.0;
    for (int i = threadIdx.x; i < n; i += 1024) s += Jw[i];
    s = red.sum(s);
    if (threadIdx.x == 0) *out = s;
}

// Aggregate statistics (one CTA, fixed order).
struct DevStats {
    long long n_solved, n_failed, iters_total;
    int iters_max, refine_max;
    double worst_residual;
    double unknown_iters;
};

__global__ void __launch_bounds__(1024) k_stats(const WinStat *__restrict__ st, const int *__restrict__ count_ptr,
                                                int per_target, DevStats *__restrict__ out) {
    __shared__ double red_buf[128];
    Reducer<1024> red{red_buf, 0};
    const int n = *count_ptr * per_target;
    double solved = 0, failed = 0, iters = 0, imax = 0, omax = 0, rmax = 0, ui = 0;
    for (int i = threadIdx.x; i < n; i += 1024) {
        const WinStat s = st[i];
        if (s.status == 0) continue;
        solved += 1;
        failed += s.status >= 2 ? 1 : 0;
        iters += s.iters;
        ui += static_cast<double>(s.iters) * s.nu;
        imax = fmax(imax, static_cast<double>(s.iters));
        omax = fmax(omax, static_cast<double>(s.outer));
        rmax = fmax(rmax, static_cast<double>(s.resid));
    }
    red.sum2(solved, failed);
    red.sum2(iters, ui);
    red.max2(imax, omax);
    rmax = red.max(rmax);
    if (threadIdx.x == 0) {
        out->n_solved = static_cast<long long>(solved);
        out->n_failed = static_cast<long long>(failed);
        out->iters_total = static_cast<long long>(iters);
        out->iters_max = static_cast<int>(imax);
        out->refine_max = static_cast<int>(omax);
        out->worst_residual = rmax;
        out->unknown_iters = ui;
    }
}

}  // namespace lsb
