// graph_pairs.cu -- Circuitscape's pairwise solves on a node graph (lsb_graph_pairs of the C ABI).
//
// Input: one connected component of a raster's node graph, in CSR form and grounded at one node, plus a list of
// jobs, each a unit current from one node to another.  The reference factorises the component once and
// back-substitutes every job (src/cpp/circuit/circuitscape.cpp:587-660).  Here persistent CTAs take jobs from an
// atomic counter and solve each one by FP64 CG with Jacobi preconditioning.  The graph's arrays are read by every
// CTA, so they stay in L2; each CTA keeps its three work vectors in its own slice of global scratch and its
// solution in the job's output row.  After the solve the same CTA shifts the voltages to the source's and computes
// the node currents of graph_node_currents (circuitscape.cpp:38-77).
//
// Every loop is bounded: the job loop by the number of jobs, CG by max_iter and by a cap on restarts.  Block
// reductions use a fixed association order, so a job's result does not depend on which CTA solves it.
#include <vector>

#include "graph_common.cuh"

namespace lsbg {
namespace {

struct GArgs {
    int32_t n, ground;
    const int64_t *ptr;
    const int32_t *adj;
    const double *w, *diag;
    int64_t n_jobs;
    const int32_t *src, *dst;
    double tol, accept;
    int32_t max_iter;
    double *volt, *cur;
    double *scratch;  // per CTA: r, p, q (n doubles each)
    unsigned long long *counter;
    JobStat *jstat;
};

// y = A v on the unknowns (the ground's row is 0; v at the ground is 0); returns this thread's part of v.y, summed in
// row order.  Entries whose column is out of range are skipped and counted in `bad`.
template <int NT>
__device__ __forceinline__ double spmv(const GArgs &a, const double *v, double *y, int &bad) {
    double dot = 0.0;
    for (int i = threadIdx.x; i < a.n; i += NT) {
        double s = 0.0;
        if (i != a.ground) {
            s = a.diag[i] * v[i];
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

// Right-hand side: +1 at dst, -1 at src, 0 at the ground.
__device__ __forceinline__ double rhs(const GArgs &a, int i, int s, int d) {
    if (i == a.ground) return 0.0;
    return (i == d ? 1.0 : 0.0) - (i == s ? 1.0 : 0.0);
}

template <int NT>
__device__ void solve_job(const GArgs &a, int64_t j, double *r, double *p, double *q, double2 *red) {
    const int n = a.n, s = a.src[j], d = a.dst[j];
    double *x = a.volt + static_cast<size_t>(j) * n;
    if (s < 0 || s >= n || d < 0 || d >= n) {
        for (int i = threadIdx.x; i < n; i += NT) {
            x[i] = 0.0;
            if (a.cur) a.cur[static_cast<size_t>(j) * n + i] = 0.0;
        }
        if (threadIdx.x == 0) a.jstat[j] = JobStat{-1, 0, INFINITY};
        return;
    }
    int bad = 0;
    // x = 0, r = b, p = D^-1 r
    double pr = 0.0, pz = 0.0;
    for (int i = threadIdx.x; i < n; i += NT) {
        const double b = rhs(a, i, s, d);
        x[i] = 0.0;
        r[i] = b;
        p[i] = b / a.diag[i];
        pr += b * b;
        pz += b * b / a.diag[i];
    }
    double2 t = block_sum2<NT>(pr, pz, red);
    const double bb = t.x;
    double rr = t.x, rz = t.y;
    const double goal = a.tol * a.tol * bb;
    double best = INFINITY;
    int it = 0, stall = 0;
    for (int cycle = 0; cycle < kMaxRestarts; ++cycle) {
        while (it < a.max_iter && rr > goal) {
            const double ppq = spmv<NT>(a, p, q, bad);  // this thread's part of p.q, in row order
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
                prz += ri * ri / a.diag[i];
            }
            t = block_sum2<NT>(prr, prz, red);
            rr = t.x;
            const double beta = t.y / rz;
            rz = t.y;
            for (int i = threadIdx.x; i < n; i += NT) p[i] = r[i] / a.diag[i] + beta * p[i];
            __syncthreads();
            ++it;
        }
        // the true residual, and a restart from it unless the solve is done
        spmv<NT>(a, x, q, bad);
        __syncthreads();
        pr = 0.0;
        pz = 0.0;
        for (int i = threadIdx.x; i < n; i += NT) {
            const double ri = rhs(a, i, s, d) - q[i];
            r[i] = ri;
            p[i] = ri / a.diag[i];
            pr += ri * ri;
            pz += ri * ri / a.diag[i];
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
    // voltages relative to the source
    __syncthreads();
    const double xs = x[s];
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += NT) x[i] -= xs;
    __syncthreads();
    if (a.cur) {
        // graph_node_currents: the largest branch current into and out of any node, then each node's inflow and
        // outflow in adjacency order, leaving out branches under 1e-8 of the largest
        double mi = -INFINITY, mo = -INFINITY;
        for (int c = threadIdx.x; c < n; c += NT) {
            const double vc = x[c];
            for (int64_t e = a.ptr[c]; e < a.ptr[c + 1]; ++e) {
                const int k = a.adj[e];
                if (k < 0 || k >= n) continue;
                const double b = fabs(a.w[e]) * (x[k] - vc);
                if (k < c) {
                    if (b > mi) mi = b;
                } else if (b > mo) {
                    mo = b;
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
                const double b = fabs(a.w[e]) * (x[k] - vc);
                if (b > 0) {
                    if (!(fabs(b / m.x) < 1e-8)) in += b;
                } else if (b < 0) {
                    if (!(fabs(b / m.y) < 1e-8)) out -= b;
                }
            }
            cj[c] = in > out ? in : out;
        }
    }
    // `bad` is per thread: any thread that met an out-of-range column fails the job
    const double anybad = block_sum2<NT>(bad ? 1.0 : 0.0, 0.0, red).x;
    if (threadIdx.x == 0)
        a.jstat[j] = JobStat{anybad > 0 ? -1 : it, (anybad == 0 && resid <= a.accept) ? 1 : 0, resid};
}

template <int NT>
__global__ void __launch_bounds__(NT) k_graph_pairs(GArgs a) {
    __shared__ double2 red[NT / 32];
    __shared__ long long s_job;
    double *r = a.scratch + static_cast<size_t>(blockIdx.x) * 3 * a.n;
    double *p = r + a.n, *q = p + a.n;
    // each pass takes a new job index; the counter only grows, so the loop ends after n_jobs + gridDim.x passes
    for (;;) {
        __syncthreads();
        if (threadIdx.x == 0) s_job = static_cast<long long>(atomicAdd(a.counter, 1ull));
        __syncthreads();
        const long long j = s_job;
        if (j >= a.n_jobs) return;
        solve_job<NT>(a, j, r, p, q, red);
    }
}

struct GraphPlan {
    int64_t ctas;
    size_t off_stats, off_scratch, bytes;
};

GraphPlan plan(int64_t n, int64_t n_jobs, const lsb_graph_params *p) {
    GraphPlan g{};
    const int64_t cap = p->max_ctas > 0 ? p->max_ctas : static_cast<int64_t>(ctas_per_sm(threads_for(n))) * device_sms();
    const int64_t memcap = std::max<int64_t>(1, static_cast<int64_t>(kScratchCap / (24.0 * static_cast<double>(n))));
    g.ctas = std::max<int64_t>(1, std::min({n_jobs, cap, memcap}));
    g.off_stats = kAlign;  // the job counter sits at offset 0
    g.off_scratch = g.off_stats + align_up(static_cast<size_t>(std::max<int64_t>(n_jobs, 1)) * sizeof(JobStat));
    g.bytes = g.off_scratch + static_cast<size_t>(g.ctas) * 3 * static_cast<size_t>(n) * sizeof(double);
    return g;
}

}  // namespace
}  // namespace lsbg

using namespace lsbg;

extern "C" {

void lsb_graph_params_default(lsb_graph_params *p) {
    if (!p) return;
    p->tol = 1e-14;
    p->accept = 1e-9;
    p->max_iter = 0;
    p->max_ctas = 0;
}

int lsb_graph_pairs_workspace_size(int64_t n, int64_t n_jobs, const lsb_graph_params *p, size_t *bytes) {
    if (!bytes || !valid(n, n_jobs, p, nullptr, 0)) return LSB_ERR_ARGUMENT;
    *bytes = plan(n, n_jobs, p).bytes;
    return LSB_OK;
}

int lsb_graph_pairs(int64_t n, const int64_t *ptr, const int32_t *adj, const double *w, const double *diag,
                    int32_t ground, int64_t n_jobs, const int32_t *src, const int32_t *dst,
                    const lsb_graph_params *p, double *volt, double *cur, void *workspace, size_t workspace_bytes,
                    lsb_graph_stats *stats, char *err, size_t errlen, void *stream) {
    if (stats) std::memset(stats, 0, sizeof(*stats));
    if (!valid(n, n_jobs, p, err, errlen)) return LSB_ERR_ARGUMENT;
    if (ground < 0 || ground >= n) {
        set_err(err, errlen, "ground %d is not a node of the component (n = %lld)", ground, (long long)n);
        return LSB_ERR_ARGUMENT;
    }
    if (n_jobs == 0) return LSB_OK;
    if (!ptr || !adj || !w || !diag || !src || !dst || !volt || !workspace) {
        set_err(err, errlen, "a device pointer is NULL");
        return LSB_ERR_ARGUMENT;
    }
    const GraphPlan g = plan(n, n_jobs, p);
    if (workspace_bytes < g.bytes) {
        set_err(err, errlen, "workspace too small: %zu bytes, %zu needed", workspace_bytes, g.bytes);
        return LSB_ERR_WORKSPACE;
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    char *ws = static_cast<char *>(workspace);
    GArgs a{};
    a.n = static_cast<int32_t>(n);
    a.ground = ground;
    a.ptr = ptr;
    a.adj = adj;
    a.w = w;
    a.diag = diag;
    a.n_jobs = n_jobs;
    a.src = src;
    a.dst = dst;
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
            k_graph_pairs<512><<<static_cast<unsigned>(g.ctas), 512, 0, st>>>(a);
        else
            k_graph_pairs<256><<<static_cast<unsigned>(g.ctas), 256, 0, st>>>(a);
        e = cudaGetLastError();
    }
    if (e != cudaSuccess) {
        set_err(err, errlen, "CUDA error %s in lsb_graph_pairs", cudaGetErrorString(e));
        return LSB_ERR_CUDA;
    }
    if (!stats) return LSB_OK;
    std::vector<JobStat> js(static_cast<size_t>(n_jobs));
    e = cudaMemcpyAsync(js.data(), a.jstat, js.size() * sizeof(JobStat), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        set_err(err, errlen, "CUDA error %s in lsb_graph_pairs", cudaGetErrorString(e));
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
        set_err(err, errlen, "%lld of %lld pair solves failed (worst relative residual %.3g)",
                (long long)stats->failures, (long long)n_jobs, stats->worst_residual);
        return LSB_ERR_NOT_CONVERGED;
    }
    return LSB_OK;
}

}  // extern "C"
