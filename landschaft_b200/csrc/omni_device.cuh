// omni_device.cuh -- the per-window circuit solve of the Omniscape path, on one
// CTA of an sm_100a GPU.
//
// One CTA owns one window at a time (a persistent CTA pulls windows from a
// queue).  Per window it
//   1. builds the window's conductance and sources from the rasters
//      (omniscape.cpp:495-530: disk of radius + buffer, NoData = -9999,
//      sources within radius, the target block zeroed at radius + buffer from
//      the window corner, sources rescaled to the block's amps, conditions);
//   2. flood-fills the ground's component (omniscape.cpp:86-101);
//   3. assembles the grounded Laplacian implicitly (system.cpp:458-487): the
//      stencil weights are recomputed from the conductance in every matrix-
//      vector product, the diagonal is summed in column-major neighbour order;
//   4. solves it by preconditioned CG: FP64 Jacobi-PCG ("plain"), or CG whose
//      iterations run in T (float) inside FP64 iterative refinement, with a
//      Jacobi or a geometric multigrid V-cycle preconditioner;
//   5. computes node currents exactly as grid.cpp:19-71 does (FP64, branch
//      threshold 1e-8 of the signed maxima, max(inflow, outflow), column-major
//      neighbour order), applies the block-artifact correction slice
//      (omniscape.cpp:553-571) and writes the window to its output slot.
//
// Memory: every per-cell array of a window lives in a padded (h+2) x (w+2)
// row-major box (pitch P = w + 2), so that stencil reads need no bounds
// checks.  Arrays are placed in shared memory while it lasts and otherwise in
// a per-CTA slice of global scratch (L2-resident); the host decides the
// placement (ArenaLayout).  All reductions are block-wide, in a fixed order:
// results do not depend on scheduling.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>
#include <math_constants.h>

namespace lsb {

constexpr double kTwoSqrt2 = 2.8284271247461903;  // 2*sqrt(2) as the reference evaluates it (grid.hpp:17)
constexpr double kSqrt2 = 1.4142135623730951;
constexpr double kInvTwoSqrt2 = 0.35355339059327373;  // 1 / (2 sqrt 2), for iterative products only
constexpr double kShift = 10.0 * 2.220446049250313080847e-16;  // CHOLMOD's 10 eps (omniscape.cpp:28)

// ---------------------------------------------------------------------------
// Stencils: neighbours in increasing column-major index (grid.hpp:27-35).
// ---------------------------------------------------------------------------
template <bool FOUR>
struct Nb;
template <>
struct Nb<false> {
    static constexpr int ND = 8, LOWER = 4;
    __host__ __device__ static constexpr int dy(int d) {
        return d == 0 ? -1 : d == 1 ? 0 : d == 2 ? 1 : d == 3 ? -1 : d == 4 ? 1 : d == 5 ? -1 : d == 6 ? 0 : 1;
    }
    __host__ __device__ static constexpr int dx(int d) { return d < 3 ? -1 : d < 5 ? 0 : 1; }
    __host__ __device__ static constexpr bool diag(int d) { return d == 0 || d == 2 || d == 5 || d == 7; }
};
template <>
struct Nb<true> {
    static constexpr int ND = 4, LOWER = 2;
    __host__ __device__ static constexpr int dy(int d) { return d == 1 ? -1 : d == 2 ? 1 : 0; }
    __host__ __device__ static constexpr int dx(int d) { return d == 0 ? -1 : d == 3 ? 1 : 0; }
    __host__ __device__ static constexpr bool diag(int) { return false; }
};

// FP64 edge weight of two conductances (grid.hpp:37-40; resistor series:
// circuitscape.cpp:30-33).  The diagonal average multiplies by 1 / (2 sqrt 2)
// where the reference divides by 2 sqrt 2: within one ulp of the reference's
// weight, far below the solver's tolerance.
__device__ __forceinline__ double edge_w64(double a, double b, bool diag, bool series) {
    if (series) return diag ? 1.0 / (kSqrt2 * (1.0 / a + 1.0 / b) / 2.0) : 1.0 / ((1.0 / a + 1.0 / b) / 2.0);
    return diag ? (a + b) * kInvTwoSqrt2 : (a + b) * 0.5;
}

// The reference's test for leaving a branch current out of a node current, fabs(b / m) < 1e-8 (grid.cpp:19-71),
// for one maximum m, decided by comparisons where that is unambiguous: the product 1e-8 m and the quotient b / m
// round differently only within a relative 1e-15 or so of the threshold, so outside a band of 1e-6 around it the
// decision is the same; inside it (and for a maximum that is not positive, finite and normal: empty band) the
// quotient decides.
struct Threshold {
    double m, lo, hi;
    __device__ explicit Threshold(double m_) : m(m_) {
        const bool fast = m_ > 1e-290 && m_ < CUDART_INF;
        lo = fast ? 1e-8 * m_ * (1.0 - 1e-6) : -1.0;
        hi = fast ? 1e-8 * m_ * (1.0 + 1e-6) : -1.0;
    }
    __device__ __forceinline__ bool below(double b) const {
        const double ab = fabs(b);
        if (ab < lo) return true;
        if (ab > hi && hi >= 0.0) return false;
        return fabs(b / m) < 1e-8;
    }
};

// d(edge weight)/d(first conductance); the weights are symmetric in their arguments.
__device__ __forceinline__ double edge_dw64(double a, double b, bool diag, bool series) {
    if (series) {
        // w = 2 / (k (1/a + 1/b)), k = sqrt 2 on diagonals: dw/da = 2 / (k (1/a + 1/b)^2 a^2)
        const double k = diag ? kSqrt2 : 1.0, s = 1.0 / a + 1.0 / b;
        return 2.0 / (k * s * s * a * a);
    }
    return diag ? kInvTwoSqrt2 : 0.5;
}

// ---------------------------------------------------------------------------
// Window descriptions.
// ---------------------------------------------------------------------------
enum WinKind : int { KIND_LAND = 0, KIND_FLOW = 1, KIND_CORR_BLOCK = 2, KIND_CORR_NULL = 3 };

// Per-window geometry in window coordinates.
struct WinGeom {
    int h, w, gy, gx;  // box and ground
    int P, NP;         // padded pitch and padded cell count
    int64_t y0, x0;    // corner on the map
    int64_t ty, tx;    // target on the map
};

// Mask bits of a level-0 cell.
enum : uint8_t { M_UNKNOWN = 1, M_PRESENT = 2, M_CAND = 4, M_USEIN = 8, M_DIRECT = 16, M_DONE = 32 };
// (M_DIRECT: a direct ground of a raster solve; M_DONE: the cell's component has been handled)

constexpr int kMaxLevels = 9;  // level 0 + up to 8 coarse levels (windows up to 513 cells wide)
constexpr int kNcMax = 25;     // cells of the coarsest level (solved by its dense inverse)

// Arrays of a window's working set.
enum LevelArray : int { LV_C0 = 0, LV_CE, LV_CSW, LV_CS, LV_CSE, LV_INVD, LV_X, LV_B, LV_T, LV_COUNT };
enum ArenaArray : int {
    AR_MASK = 0,  // u8
    AR_ULIST,     // u16 (windows) or u32 (whole rasters): padded indices of the unknowns, row-major
    AR_G64,       // f64: conductance (-9999 outside / NoData; 0 on padding)
    AR_X64,       // f64: solution (potentials), 0 off the unknowns
    AR_B64,       // f64: scaled sources (the right-hand side)
    AR_V64,       // f64: the forward potentials, kept during the adjoint solve
    AR_CW,        // f64: J's weight of each cell (adjoint)
    AR_DG64,      // f64: the explicit part of dJ/dg (adjoint)
    AR_GT,        // T: stencil conductance (or resistance with series weights); sentinels off the nodes
    AR_INVD,      // T: 1 / diagonal on the unknowns, 0 elsewhere
    AR_D,         // T: inner solution (refinement correction)
    AR_R,         // T: inner residual
    AR_P,         // T: search direction
    AR_Q,         // T: A p; multigrid fine residual and output
    AR_Z,         // T: multigrid pre-smoothed residual; the fine diagonal during set-up
    AR_DENSE,     // f64: inverse of the coarsest operator (kNcMax^2)
    AR_FG64,      // f64: finite ground conductance of a raster solve (0 elsewhere)
    AR_FGT,       // T: the same for the inner operator
    AR_LEVEL,     // first coarse level; each coarse level has LV_COUNT arrays
    AR_COUNT = AR_LEVEL + (kMaxLevels - 1) * LV_COUNT
};

// Byte offsets of the arrays; bit 31 set: in global scratch, else shared.
constexpr uint32_t kNoStage = 0xffffffffu;

struct ArenaLayout {
    uint32_t off[AR_COUNT];
    uint32_t smem_bytes;
    uint32_t gmem_bytes;  // per CTA
    uint32_t hot;         // 1: every array but the FP64 window arrays is in shared memory
    uint32_t stage;       // shared offset of 2 x (h+2)(w+2) doubles free during the node currents, or kNoStage
    uint32_t rstage;      // the same, free between inner solves (the FP64 residual), or kNoStage
};

// Solver configuration for one launch.
struct SolveParams {
    double tol;        // final relative FP64 residual
    double inner_tol;  // relative residual reduction of one refinement step
    int max_iter;      // cap on CG iterations (all refinement steps)
    int max_outer;     // cap on refinement steps
    int pc;            // 1 Jacobi, 2 multigrid
    float omega;       // damped-Jacobi smoothing weight on the fine level (safe below 1: lambda_max(D^-1 A) <= 2)
    float omega_c;     // the same on the Galerkin coarse levels, which have no such bound
};

// Per-solve statistics written by the kernel.
struct WinStat {
    int iters;
    int outer;
    int status;  // 0 no solve needed, 1 converged, 2 not converged, 3 breakdown / non-finite
    float resid;  // final relative FP64 residual
    int nu;       // unknowns of the system
};

// ---------------------------------------------------------------------------
// Block-wide reductions in a fixed order (every thread gets the same value).
// `red` is shared: 2 slots x 64 doubles.
// ---------------------------------------------------------------------------
template <int NT>
struct Reducer {
    static constexpr int NW = NT / 32;
    double *red;
    int slot;
    __device__ __forceinline__ double *next() {
        double *b = red + (slot & 1) * 64;
        ++slot;
        return b;
    }
    // Lane 0 of every warp holds its warp's value; after the barrier each warp
    // sums the partials with the same shuffle tree (the same order in every
    // warp) and broadcasts lane 0's result.
    __device__ __forceinline__ static double tree_sum(double v) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        return __shfl_sync(0xffffffffu, v, 0);
    }
    __device__ __forceinline__ static double tree_max(double v) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
        return __shfl_sync(0xffffffffu, v, 0);
    }
    __device__ __forceinline__ double sum(double v) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        double *b = next();
        const int lane = threadIdx.x & 31;
        if (lane == 0) b[threadIdx.x >> 5] = v;
        __syncthreads();
        return tree_sum(lane < NW ? b[lane] : 0.0);
    }
    __device__ __forceinline__ void sum2(double &a, double &c) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            a += __shfl_down_sync(0xffffffffu, a, o);
            c += __shfl_down_sync(0xffffffffu, c, o);
        }
        double *b = next();
        const int lane = threadIdx.x & 31;
        if (lane == 0) {
            b[threadIdx.x >> 5] = a;
            b[32 + (threadIdx.x >> 5)] = c;
        }
        __syncthreads();
        a = tree_sum(lane < NW ? b[lane] : 0.0);
        c = tree_sum(lane < NW ? b[32 + lane] : 0.0);
    }
    __device__ __forceinline__ double max(double v) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
        double *b = next();
        const int lane = threadIdx.x & 31;
        if (lane == 0) b[threadIdx.x >> 5] = v;
        __syncthreads();
        return tree_max(lane < NW ? b[lane] : -1.0 / 0.0);
    }
    __device__ __forceinline__ void max2(double &a, double &c) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            a = fmax(a, __shfl_down_sync(0xffffffffu, a, o));
            c = fmax(c, __shfl_down_sync(0xffffffffu, c, o));
        }
        double *b = next();
        const int lane = threadIdx.x & 31;
        if (lane == 0) {
            b[threadIdx.x >> 5] = a;
            b[32 + (threadIdx.x >> 5)] = c;
        }
        __syncthreads();
        a = tree_max(lane < NW ? b[lane] : -1.0 / 0.0);
        c = tree_max(lane < NW ? b[32 + lane] : -1.0 / 0.0);
    }
};

// ---------------------------------------------------------------------------
// Level sizes of the multigrid hierarchy: a dimension of n > 3 cells coarsens
// to n/2 + 1 (coarse point J <-> fine point 2J); the hierarchy ends at the
// first level of at most kNcMax cells.
// ---------------------------------------------------------------------------
__host__ __device__ inline int coarse_dim(int n) { return n > 3 ? n / 2 + 1 : n; }
__host__ __device__ inline int mg_levels(int h, int w) {
    int L = 1;
    while (h * w > kNcMax && L < kMaxLevels) {
        const int hc = coarse_dim(h), wc = coarse_dim(w);
        if (hc == h && wc == w) break;
        h = hc;
        w = wc;
        ++L;
    }
    return L;
}

}  // namespace lsb
