// graph_solve.cu -- advanced-mode problems on one component of a node graph (lsb_graph_solve of the C ABI).
//
// A job is one of Circuitscape's advanced-mode problems restricted to a component: current sources, direct grounds
// held at 0 V (not unknowns) and finite grounds added to the diagonal.  The reference factorises the component per
// problem, or once with a dense Schur complement on the nodes that carry a source or a ground
// (raster_advanced / raster_advanced_many, src/cpp/circuit/circuitscape.cpp:393-470,904-1083); one-to-all and
// all-to-one are such problems, one per focal point.  Here persistent CTAs take jobs from an atomic counter and
// solve each one by FP64 CG with Jacobi preconditioning, as lsb_graph_pairs does; the job's right-hand side,
// diagonal, finite grounds and direct-ground mask live in the CTA's slice of global scratch.  After the solve the
// CTA computes the node currents of graph_node_currents (circuitscape.cpp:38-77), finite grounds' currents
// included.
//
// Every loop is bounded: the job loop by the number of jobs, CG by max_iter and by a cap on restarts.  Block
// reductions use a fixed association order, so a job's result does not depend on which CTA solves it.
#include <vector>

#include "graph_common.cuh"

namespace lsbg {
namespace {

constexpr int kPerNode = 7;  // doubles of scratch per node: r, p, q, b, diagonal, finite grounds, mask (bytes)

struct SArgs {
    int32_t n;
    const int64_t *ptr;
    const int32_t *adj;
    const double *w, *diag;
    int64_t n_jobs;
    const int64_t *s_ptr, *d_ptr, *f_ptr;  // per-job lists, CSR over the jobs
    const int32_t *s_node, *d_node, *f_node;
    const double *s_val, *f_val;
    double tol, accept;
    int32_t max_iter;
    double *volt, *cur;
    double *scratch;
    unsigned long long *counter;
    JobStat *jstat;
};

// y = A v on the unknowns (rows of direct grounds are 0; v is 0 there); returns this thread's part of v.y, summed in
// row order.  Entries whose column is out of range are skipped and counted in `bad`.
template <int NT>
__device__ __forceinline__ double spmv(const SArgs &a, const double *dg, const uint8_t *mask, const double *v,
                                       double *y, int &bad) {
    double dot = 0.0;
    for (int i = threadIdx.x; i < a.n; i += NT) {
        double s = 0.0;
        if (!mask[i]) {
            s = dg[i] * v[i];
            for (int64_t e = a.ptr[i]; e < a.ptr[i + 1]; ++e) {
                const int c = a.adj[e];
                if (c < 0 || c >= a.n) {
                    bad = 1;
                    continue;
                }
                s -= a.w[e] * v[c];
            }
        }
        y[i] = s;
        dot += v[i] * s;
    }
    return dot;
}

template <int NT>
__device__ void solve_problem(const SArgs &a, int64_t j, double *scr, double2 *red) {
    const int n = a.n;
    double *x = a.volt + static_cast<size_t>(j) * n;
    double *r = scr, *p = r + n, *q = p + n, *b = q + n, *dg = b + n, *fin = dg + n;
    uint8_t *mask = reinterpret_cast<uint8_t *>(fin + n);
    int bad = 0;
    for (int i = threadIdx.x; i < n; i += NT) {
        x[i] = 0.0;
        b[i] = 0.0;
        dg[i] = a.diag[i];
        fin[i] = 0.0;
        mask[i] = 0;
    }
    __syncthreads();
    // the job's lists (nodes unique within each list)
    for (int64_t e = a.d_ptr[j] + threadIdx.x; e < a.d_ptr[j + 1]; e += NT) {
        const int v = a.d_node[e];
        if (v < 0 || v >= n)
            bad = 1;
        else
            mask[v] = 1;
    }
    for (int64_t e = a.f_ptr[j] + threadIdx.x; e < a.f_ptr[j + 1]; e += NT) {
        const int v = a.f_node[e];
        if (v < 0 || v >= n) {
            bad = 1;
        } else {
            fin[v] = a.f_val[e];
            dg[v] = a.diag[v] + a.f_val[e];
        }
    }
    for (int64_t e = a.s_ptr[j] + threadIdx.x; e < a.s_ptr[j + 1]; e += NT) {
        const int v = a.s_node[e];
        if (v < 0 || v >= n)
            bad = 1;
        else
            b[v] = a.s_val[e];
    }
    __syncthreads();
    // b on the unknowns only (a direct ground is not an unknown); r = b, p = D^-1 r
    double pr = 0.0, pz = 0.0;
    for (int i = threadIdx.x; i < n; i += NT) {
        if (mask[i]) b[i] = 0.0;
        const double bi = b[i];
        r[i] = bi;
        p[i] = bi / dg[i];
        pr += bi * bi;
        pz += bi * bi / dg[i];
    }
    double2 t = block_sum2<NT>(pr, pz, red);
    const double bb = t.x;
    double rr = t.x, rz = t.y;
    const double goal = a.tol * a.tol * bb;
    double best = INFINITY;
    int it = 0, stall = 0;
    for (int cycle = 0; cycle < kMaxRestarts; ++cycle) {
        while (it < a.max_iter && rr > goal) {
            const double ppq = spmv<NT>(a, dg, mask, p, q, bad);  // this thread's part of p.q, in row order
            __syncthreads();
            const double pq = block_sum2<NT>(ppq, 0.0, red).x;
            if (!(pq > 0.0)) break;  // breakdown: the true residual decides below
            const double alpha = rz / pq;
            double prr = 0.0, prz = 0.0;
            for (int i = threadIdx.x; i < n; i += NT) {
                x[i] += alpha * p[i];
                const double ri = r[i] - alpha * q[i];
                r[i] = ri;
                prr += ri * ri;
                prz += ri * ri / dg[i];
            }
            t = block_sum2<NT>(prr, prz, red);
            rr = t.x;
            const double beta = t.y / rz;
            rz = t.y;
            for (int i = threadIdx.x; i < n; i += NT) p[i] = r[i] / dg[i] + beta * p[i];
            __syncthreads();
            ++it;
        }
        // the true residual, and a restart from it unless the solve is done
        spmv<NT>(a, dg, mask, x, q, bad);
        __syncthreads();
        pr = 0.0;
        pz = 0.0;
        for (int i = threadIdx.x; i < n; i += NT) {
            const double ri = mask[i] ? 0.0 : b[i] - q[i];
            r[i] = ri;
            p[i] = ri / dg[i];
            pr += ri * ri;
            pz += ri * ri / dg[i];
        }
        t = block_sum2<NT>(pr, pz, red);
        rr = t.x;
        rz = t.y;
        if (rr <= goal || it >= a.max_iter) break;
        if (rr > 0.25 * best) {  // the true residual did not halve: at the arithmetic's floor
            if (++stall >= 2) break;
        } else {
            stall = 0;
        }
        best = fmin(best, rr);
    }
    const double resid = bb > 0.0 ? sqrt(rr / bb) : 0.0;
    __syncthreads();
    if (a.cur) {
        // graph_node_currents with finite grounds: the largest branch current into and out of any node, then each
        // node's inflow and outflow in adjacency order (branches under 1e-8 of the largest left out), plus the
        // current through its finite ground
        double mi = -INFINITY, mo = -INFINITY;
        for (int c = threadIdx.x; c < n; c += NT) {
            const double vc = x[c];
            for (int64_t e = a.ptr[c]; e < a.ptr[c + 1]; ++e) {
                const int k = a.adj[e];
                if (k < 0 || k >= n) continue;
                const double br = fabs(a.w[e]) * (x[k] - vc);
                if (k < c) {
                    if (br > mi) mi = br;
                } else if (br > mo) {
                    mo = br;
                }
            }
        }
        const double2 m = block_max2<NT>(mi, mo, red);
        double *cj = a.cur + static_cast<size_t>(j) * n;
        for (int c = threadIdx.x; c < n; c += NT) {
            const double vc = x[c];
            double in = 0.0, out = 0.0;
            for (int64_t e = a.ptr[c]; e < a.ptr[c + 1]; ++e) {
                const int k = a.adj[e];
                if (k < 0 || k >= n) continue;
                const double br = fabs(a.w[e]) * (x[k] - vc);
                if (br > 0) {
                    if (!(fabs(br / m.x) < 1e-8)) in += br;
                } else if (br < 0) {
                    if (!(fabs(br / m.y) < 1e-8)) out -= br;
                }
            }
            const double f = fin[c] * vc;
            if (f < 0)
                in -= f;
            else if (f > 0)
                out += f;
            cj[c] = in > out ? in : out;
        }
    }
    // `bad` is per thread: any thread that met a node out of range fails the job
    const double anybad = block_sum2<NT>(bad ? 1.0 : 0.0, 0.0, red).x;
    if (threadIdx.x == 0)
        a.jstat[j] = JobStat{anybad > 0 ? -1 : it, (anybad == 0 && resid <= a.accept) ? 1 : 0, resid};
}

template <int NT>
__global__ void __launch_bounds__(NT) k_graph_solve(SArgs a) {
    __shared__ double2 red[NT / 32];
    __shared__ long long s_job;
    double *scr = a.scratch + static_cast<size_t>(blockIdx.x) * kPerNode * a.n;
    // each pass takes a new job index; the counter only grows, so the loop ends after n_jobs + gridDim.x passes
    for (;;) {
        __syncthreads();
        if (threadIdx.x == 0) s_job = static_cast<long long>(atomicAdd(a.counter, 1ull));
        __syncthreads();
        const long long j = s_job;
        if (j >= a.n_jobs) return;
        solve_problem<NT>(a, j, scr, red);
    }
}

struct SolvePlan {
    int64_t ctas;
    size_t off_stats, off_scratch, bytes;
};

SolvePlan plan(int64_t n, int64_t n_jobs, const lsb_graph_params *p) {
    SolvePlan g{};
    const int64_t cap = p->max_ctas > 0 ? p->max_ctas : static_cast<int64_t>(ctas_per_sm(threads_for(n))) * device_sms();
    const int64_t memcap =
        std::max<int64_t>(1, static_cast<int64_t>(kScratchCap / (8.0 * kPerNode * static_cast<double>(n))));
    g.ctas = std::max<int64_t>(1, std::min({n_jobs, cap, memcap}));
    g.off_stats = kAlign;  // the job counter sits at offset 0
    g.off_scratch = g.off_stats + align_up(static_cast<size_t>(std::max<int64_t>(n_jobs, 1)) * sizeof(JobStat));
    g.bytes = g.off_scratch + static_cast<size_t>(g.ctas) * kPerNode * static_cast<size_t>(n) * sizeof(double);
    return g;
}

}  // namespace
}  // namespace lsbg

using namespace lsbg;

extern "C" {

int lsb_graph_solve_workspace_size(int64_t n, int64_t n_jobs, const lsb_graph_params *p, size_t *bytes) {
    if (!bytes || !valid(n, n_jobs, p, nullptr, 0)) return LSB_ERR_ARGUMENT;
    *bytes = plan(n, n_jobs, p).bytes;
    return LSB_OK;
}

int lsb_graph_solve(int64_t n, const int64_t *ptr, const int32_t *adj, const double *w, const double *diag,
                    int64_t n_jobs, const int64_t *src_ptr, const int32_t *src_node, const double *src_val,
                    const int64_t *dir_ptr, const int32_t *dir_node, const int64_t *fin_ptr,
                    const int32_t *fin_node, const double *fin_val, const lsb_graph_params *p, double *volt,
                    double *cur, void *workspace, size_t workspace_bytes, lsb_graph_stats *stats, char *err,
                    size_t errlen, void *stream) {
    if (stats) std::memset(stats, 0, sizeof(*stats));
    if (!valid(n, n_jobs, p, err, errlen)) return LSB_ERR_ARGUMENT;
    if (n_jobs == 0) return LSB_OK;
    if (!ptr || !adj || !w || !diag || !src_ptr || !dir_ptr || !fin_ptr || !volt || !workspace) {
        set_err(err, errlen, "a device pointer is NULL");
        return LSB_ERR_ARGUMENT;
    }
    const SolvePlan g = plan(n, n_jobs, p);
    if (workspace_bytes < g.bytes) {
        set_err(err, errlen, "workspace too small: %zu bytes, %zu needed", workspace_bytes, g.bytes);
        return LSB_ERR_WORKSPACE;
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    char *ws = static_cast<char *>(workspace);
    SArgs a{};
    a.n = static_cast<int32_t>(n);
    a.ptr = ptr;
    a.adj = adj;
    a.w = w;
    a.diag = diag;
    a.n_jobs = n_jobs;
    a.s_ptr = src_ptr;
    a.s_node = src_node;
    a.s_val = src_val;
    a.d_ptr = dir_ptr;
    a.d_node = dir_node;
    a.f_ptr = fin_ptr;
    a.f_node = fin_node;
    a.f_val = fin_val;
    a.tol = p->tol;
    a.accept = p->accept;
    const int64_t mi = p->max_iter > 0 ? p->max_iter : std::min<int64_t>(INT32_MAX, 20 * n + 2000);
    a.max_iter = static_cast<int32_t>(mi);
    a.volt = volt;
    a.cur = cur;
    a.counter = reinterpret_cast<unsigned long long *>(ws);
    a.jstat = reinterpret_cast<JobStat *>(ws + g.off_stats);
    a.scratch = reinterpret_cast<double *>(ws + g.off_scratch);
    cudaError_t e = cudaMemsetAsync(a.counter, 0, sizeof(unsigned long long), st);
    if (e == cudaSuccess) {
        if (threads_for(n) == 512)
            k_graph_solve<512><<<static_cast<unsigned>(g.ctas), 512, 0, st>>>(a);
        else
            k_graph_solve<256><<<static_cast<unsigned>(g.ctas), 256, 0, st>>>(a);
        e = cudaGetLastError();
    }
    if (e != cudaSuccess) {
        set_err(err, errlen, "CUDA error %s in lsb_graph_solve", cudaGetErrorString(e));
        return LSB_ERR_CUDA;
    }
    if (!stats) return LSB_OK;
    std::vector<JobStat> js(static_cast<size_t>(n_jobs));
    e = cudaMemcpyAsync(js.data(), a.jstat, js.size() * sizeof(JobStat), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        set_err(err, errlen, "CUDA error %s in lsb_graph_solve", cudaGetErrorString(e));
        return LSB_ERR_CUDA;
    }
    stats->jobs = n_jobs;
    stats->ctas = static_cast<int32_t>(g.ctas);
    double sum = 0.0;
    for (const JobStat &s : js) {
        if (s.iters < 0 || !s.ok) ++stats->failures;
        stats->iters_max = std::max(stats->iters_max, s.iters);
        sum += std::max(s.iters, 0);
        if (!(s.resid <= stats->worst_residual)) stats->worst_residual = s.resid;
    }
    stats->iters_mean = sum / static_cast<double>(n_jobs);
    if (stats->failures) {
        set_err(err, errlen, "%lld of %lld problem solves failed (worst relative residual %.3g)",
                (long long)stats->failures, (long long)n_jobs, stats->worst_residual);
        return LSB_ERR_NOT_CONVERGED;
    }
    return LSB_OK;
}

}  // extern "C"
