// omni_adv.cuh -- the persistent raster kernel of the advanced mode (grid.cpp:73-210): each CTA pulls rasters
// from a queue; for every connected component of a raster's nodes it decides, as the reference does, whether the
// component has a source and a ground, and if so solves it (the window solver of omni_solver.cuh on the whole
// raster box, with finite grounds on the diagonal and direct grounds as fixed 0 V nodes) and writes its node
// currents and voltages.
#pragma once

#include "omni_solver.cuh"

namespace lsb {

template <int NT, typename T, bool FOUR, bool MG, bool REFINE, bool HOT>
__global__ void __launch_bounds__(NT, 1) k_rasters(const KArgs a) {
    extern __shared__ __align__(16) char smem[];
    __shared__ double red_buf[128];
    __shared__ int scan_buf[64];
    __shared__ int lvh[kMaxLevels], lvw[kMaxLevels];
    __shared__ float lvinv[kMaxLevels];
    __shared__ uint32_t lvoff[(kMaxLevels - 1) * LV_COUNT];
    __shared__ short cidx[kNcMax];
    __shared__ int item_s;
    __shared__ WinStat sst;
    for (int k = threadIdx.x; k < (kMaxLevels - 1) * LV_COUNT; k += NT) lvoff[k] = a.lay.off[AR_LEVEL + k];
    char *gm = a.gscratch + static_cast<size_t>(blockIdx.x) * a.lay.gmem_bytes;
    Reducer<NT> red{red_buf, 0};
    Win<NT, T, FOUR, MG, REFINE, HOT, true> win(a, smem, gm, red, scan_buf, lvh, lvw, lvinv, lvoff, cidx);
#ifdef LSB_PHASE_TIMERS
    __shared__ unsigned long long tacc[PH_COUNT + 1];
    if (threadIdx.x <= PH_COUNT) tacc[threadIdx.x] = threadIdx.x == PH_COUNT ? clock64() : 0ull;
    win.tacc = tacc;
#endif
    __syncthreads();
    while (true) {
        if (threadIdx.x == 0) item_s = atomicAdd(a.queue, 1);
        __syncthreads();
        const int item = item_s;
        __syncthreads();
        if (item >= a.n_rasters) break;
        const int k = a.ras_order[item];
        const int64_t off = a.ras_off[k];
        WinGeom &G = win.G;
        G.h = a.ras_ny[k];
        G.w = a.ras_nx[k];
        G.y0 = G.x0 = G.ty = G.tx = 0;
        G.gy = G.gx = 0;
        G.P = G.w + 2;
        G.NP = (G.h + 2) * G.P;
        win.volt_out = a.fp_win + off;
        double *cur = a.cur_win + off;
        win.load_raster(a.res + off, a.src + off, a.gnd + off, cur);
        int iters = 0, outer = 0, status = 0, nu = 0;
        float resid = 0.f;
        while (true) {
            const int seed = win.next_seed();
            if (seed < 0) break;
            win.flood_from(seed);
            if (!win.component_active()) continue;  // no source or no ground: voltage 0, current 0
            win.mark_unknowns();
            if (win.nu > 0) {
                win.assemble();
                win.solve(&sst);
                __syncthreads();
                if (threadIdx.x == 0) {
                    iters += sst.iters;
                    outer = outer > sst.outer ? outer : sst.outer;
                    status = status > sst.status ? status : sst.status;
                    resid = resid > sst.resid ? resid : sst.resid;
                    nu += sst.nu;
                }
            }
            win.currents(cur, nullptr, 0, 0);
            win.clear_solution();
        }
        if (threadIdx.x == 0) a.stat[k] = WinStat{iters, outer, status, resid, nu};
    }
#ifdef LSB_PHASE_TIMERS
    win.mark(PH_OTHER);
    if (a.timers && threadIdx.x < PH_COUNT) atomicAdd(a.timers + threadIdx.x, tacc[threadIdx.x]);
#endif
}

KernelFn pick_rasters(bool hot, bool four, bool dbl);

}  // namespace lsb
