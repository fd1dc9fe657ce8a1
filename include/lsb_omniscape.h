/*
 * lsb_omniscape.h -- C ABI of landschaft_b200's Omniscape moving-window
 * circuit solver on one B200 (sm_100a).
 *
 * Plain C types only: pointers, sizes, a parameter struct.  No exceptions
 * cross this boundary; every entry point returns LSB_OK (0) or an error code,
 * with a message in `err` when err != NULL.
 *
 * Reference interfaces replaced (paths within the landschaft source tree):
 *   lsb_omniscape               circuit_omniscape  src/cpp/circuit/python.cpp:90-137
 *                               -> circuit::omniscape  src/cpp/circuit/omniscape.hpp:56-60
 *   lsb_omniscape_correction    circuit_omniscape_correction  src/cpp/circuit/python.cpp:139-153
 *                               -> circuit::omniscape_correction  src/cpp/circuit/omniscape.hpp:62-64
 *   lsb_omniscape_grad          (no reference counterpart: adjoint of the cumulative current)
 *   lsb_params_default          OmniscapeParams defaults  src/cpp/circuit/omniscape.hpp:35-47
 *
 * Memory: resistance, source, condition rasters and every output are DEVICE
 * pointers (row-major ny x nx float64).  The caller owns them and a device
 * workspace of lsb_omniscape_workspace_size() bytes; the library allocates
 * nothing on the device during a call.  Work is enqueued on `stream` (a
 * cudaStream_t, NULL = the legacy default stream); the call returns once the
 * work is enqueued unless `stats` is given, in which case it waits for the
 * stream to read the statistics back.
 */
#ifndef LSB_OMNISCAPE_H
#define LSB_OMNISCAPE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum lsb_status {
    LSB_OK = 0,
    LSB_ERR_ARGUMENT = 1,      /* invalid parameter (reference: std::invalid_argument) */
    LSB_ERR_NOT_CONVERGED = 2, /* a window's solve did not converge (reference: "not positive definite") */
    LSB_ERR_CONDITION = 3,     /* a target block has no value of a condition (all NoData) */
    LSB_ERR_WORKSPACE = 4,     /* workspace too small */
    LSB_ERR_CUDA = 5           /* a CUDA runtime error */
};

enum lsb_precision {
    LSB_PREC_FP64 = 0,        /* FP64 CG throughout */
    LSB_PREC_FP32_REFINE = 1  /* FP32 CG inside FP64 iterative refinement */
};

enum lsb_preconditioner {
    LSB_PC_AUTO = 0,   /* autotuned (or the built-in table) */
    LSB_PC_JACOBI = 1, /* diagonal */
    LSB_PC_MG = 2      /* geometric multigrid V-cycle, Galerkin coarse operators */
};

enum lsb_edge_weights {
    LSB_EDGE_AVERAGE = 0, /* (a + b) / 2, diagonals / (2 sqrt 2): Omniscape / Circuitscape */
    LSB_EDGE_SERIES = 1   /* 1 / ((1/a + 1/b) / 2), diagonals / sqrt 2: resistor series */
};

/* Conditional connectivity of one condition (OmniscapeCondition,
 * omniscape.hpp:21-33).  present == NULL: no condition. */
typedef struct lsb_omni_condition {
    const double *present; /* device, ny x nx; NaN = missing (kept) */
    const double *future;  /* device, ny x nx, or NULL: the present values */
    int32_t equal;         /* 0: "within" (lower <= c - median <= upper), 1: "equal" (c == mode) */
    int32_t pad_;
    double lower, upper;
} lsb_omni_condition;

typedef struct lsb_omni_params {
    /* OmniscapeParams (omniscape.hpp:35-47) */
    int32_t radius;
    int32_t buffer;
    int32_t block_size;                /* odd */
    int32_t four_neighbors;            /* 0/1 */
    int32_t resistance_is_conductance; /* 0/1 */
    int32_t correct_artifacts;         /* 0/1 (only with block_size > 1) */
    int32_t flow_potential;            /* 0/1: also compute the flow potential */
    int32_t edge_weights;              /* lsb_edge_weights */
    lsb_omni_condition condition1, condition2;
    double memory_limit; /* bytes of window buffers per batch (0: library default) */
    /* solver */
    int32_t precision;      /* lsb_precision */
    int32_t preconditioner; /* lsb_preconditioner */
    double tol;             /* relative FP64 residual ||b - A x|| / ||b|| at which a window is solved */
    int32_t max_iter;       /* cap on CG iterations per window (all refinement steps together) */
    int32_t threads_per_window; /* 0: chosen from the window size or the tuning table; else 128 (four windows per
                                   SM, when a window's solver arrays fit a quarter of the SM's shared memory;
                                   else 256), 256 or 512 */
    int32_t use_graph;      /* 1: capture the call's launches in a CUDA graph and replay it on repeat calls */
    int32_t mask_nodata;    /* 1: NaN on NoData cells of the outputs (Python's mask_nodata) */
    /* Streaming (no counterpart in the reference, which streams inside one call): solve only the targets
     * target_begin <= t < target_end of the target order (target_end 0: to the last), adding their currents to
     * the outputs' values when accumulate is 1 (else the outputs start at 0).  The maps of consecutive ranges,
     * each call continuing the previous one's outputs, are bitwise those of one call; the normalised current and
     * the NoData mask are applied by the call whose range reaches the last target. */
    int32_t accumulate;
    int64_t target_begin;
    int64_t target_end;
} lsb_omni_params;

typedef struct lsb_omni_stats {
    int64_t n_targets;      /* targets (blocks with a positive source sum) */
    int64_t n_solved;       /* window solves carried out (cumulative current + flow potential) */
    int64_t n_failed;       /* solves that hit max_iter */
    int64_t iters_total;    /* CG iterations over all solves */
    int32_t iters_max;      /* CG iterations of the longest solve */
    int32_t refine_max;     /* refinement steps of the longest solve */
    int32_t batches;        /* window batches the targets were streamed in */
    int32_t threads_per_window;
    int32_t preconditioner;
    int32_t pad_;
    double worst_residual;  /* largest final relative FP64 residual */
    double window_ms;       /* device time of the window-solve kernels (see lsb_time_window_kernels) */
    double unknown_iters;   /* sum over solves of unknowns x CG iterations (the inner solve's work) */
} lsb_omni_stats;

/* Fill the defaults: radius 0, buffer 0, block 1, average weights, correction
 * on, FP32 + refinement, autotuned preconditioner, tol 1e-12, graphs on. */
void lsb_params_default(lsb_omni_params *p);

/* Device bytes a call needs for an nx x ny raster with these parameters. */
int lsb_omniscape_workspace_size(int64_t nx, int64_t ny, const lsb_omni_params *p, size_t *bytes);

/*
 * Omniscape on one GPU.  resistance, source: device ny x nx float64 (NaN
 * resistance = NoData; the source must already hold Omniscape's thresholds and
 * NaN -> 0, as the reference's Python layer prepares it).  Outputs: current
 * (cumulative current, required), flow_potential and normalized (NULL: not
 * computed / not written).  normalized = current / flow_potential with 0
 * where that is NaN (omniscape.py:380-384); requires p->flow_potential.
 */
int lsb_omniscape(const double *resistance, const double *source, int64_t nx, int64_t ny,
                  const lsb_omni_params *p, double *current, double *flow_potential, double *normalized,
                  void *workspace, size_t workspace_bytes, lsb_omni_stats *stats, char *err, size_t errlen,
                  void *stream);

/* Bytes of the static device scratch of lsb_omniscape_noalloc (32 MiB). */
#define LSB_NOALLOC_SCRATCH_BYTES (32u << 20)

/*
 * lsb_omniscape without a workspace (no counterpart in the reference).  For
 * callers that cannot call cudaMalloc -- for instance a host whose device
 * memory is already reserved by another framework's pool, or code that must
 * not pay an allocation's implicit device synchronization.  Inputs and outputs
 * are the caller's device pointers, as for lsb_omniscape; the scratch is one
 * static device array of LSB_NOALLOC_SCRATCH_BYTES that the library holds on
 * every GPU where it is loaded, until the process exits.  Window buffers are
 * streamed in batches sized to fit it; a raster whose targets alone need more
 * is rejected with LSB_ERR_WORKSPACE and a message.  The first call on a
 * device looks up the array's device address (cudaGetSymbolAddress); make it
 * before any stream capture.  Every call shares the array: calls that overlap
 * on the GPU (other streams, other host threads) race and must be serialised
 * by the caller.  Launches directly (no graph); allocates nothing.
 */
int lsb_omniscape_noalloc(const double *resistance, const double *source, int64_t nx, int64_t ny,
                          const lsb_omni_params *p, double *current, double *flow_potential, double *normalized,
                          lsb_omni_stats *stats, char *err, size_t errlen, void *stream);

/* The (2 (radius + buffer) + 1)^2 block-artifact correction factors
 * (omniscape_correction), written to the device array corr. */
int lsb_omniscape_correction(int32_t radius, int32_t buffer, int32_t block_size, int32_t four_neighbors,
                             int32_t edge_weights, int64_t nx, int64_t ny, double *corr, void *workspace,
                             size_t workspace_bytes, char *err, size_t errlen, void *stream);

/*
 * Adjoint of the cumulative current.  J = sum over cells of weight * current;
 * writes dJ/d(resistance) (dJ/d(conductance) with resistance_is_conductance)
 * to grad_resistance (required) and dJ/d(source) to grad_source (NULL: not
 * written), and J to *J_out when J_out != NULL (device pointer to one double).
 * weight is a device ny x nx raster; backward through J = sum(weight * current)
 * is the vector-Jacobian product of the cumulative current.
 * Forward potentials are recomputed, not stored; each window's adjoint
 * system is the same symmetric Laplacian with the node-current derivative as
 * right-hand side.  Needs no correction (block_size 1 or correct_artifacts 0)
 * and no conditions.
 */
int lsb_omniscape_grad(const double *resistance, const double *source, const double *weight, int64_t nx,
                       int64_t ny, const lsb_omni_params *p, double *grad_resistance, double *grad_source,
                       double *J_out, void *workspace, size_t workspace_bytes, lsb_omni_stats *stats, char *err,
                       size_t errlen, void *stream);

/* Device bytes lsb_omniscape_grad needs. */
int lsb_omniscape_grad_workspace_size(int64_t nx, int64_t ny, const lsb_omni_params *p, size_t *bytes);

/* Number of kernels the last call on this thread launched (from a graph replay: the graph's kernel nodes). */
int64_t lsb_last_launch_count(void);

/* On this thread, record CUDA events around the window-solve kernels of calls that run without a graph and
 * return stats: their device time goes to stats->window_ms (profiling aid; 0 = off, the default). */
void lsb_time_window_kernels(int32_t on);

/* ---------------------------------------------------------------------------
 * Advanced mode on a batch of rasters: replaces circuit_advanced (src/cpp/circuit/python.cpp:65-80; engine
 * circuit::advanced, src/cpp/circuit/grid.cpp:73-210) and solves many independent rasters in one launch.
 * Every cell with conductance > 0 is a node joined to its 8 (or 4) neighbours by the average conductance; a
 * source injects current; a ground connects its cell to 0 V through the given conductance (INFINITY: a direct
 * ground, the cell held at 0 V); a grounded cell loses its source.  Each connected component with a nonzero
 * source sum and a ground is solved; its node currents are max(inflow, outflow) with branch currents below 1e-8
 * of the component's largest left out, and currents to finite grounds counted.  Voltage: the solution on solved
 * components, 0 on the other nodes, NaN off the nodes; current 0 where nothing is solved.
 *
 * The n rasters are packed back to back in the device arrays conductance, source, ground (no NaN: the Python
 * layer maps NaN to 0), current and voltage: raster k (ny[k] x nx[k], row-major) starts at the sum of the
 * earlier rasters' cells.  nx and ny are host arrays; sides from 1 to 1024.
 * ------------------------------------------------------------------------- */
typedef struct lsb_raster_params {
    int32_t four_neighbors; /* 0/1 */
    int32_t precision;      /* lsb_precision: FP32 CG + FP64 refinement (multigrid) or FP64 CG (Jacobi) */
    double tol;             /* relative FP64 residual at which a component is solved */
    int32_t max_iter;       /* cap on CG iterations per component */
    int32_t smem_limit_kb;  /* shared memory per CTA for solver arrays, KiB (0: all there is); what is left over is
                               L1 cache for the arrays in global memory */
    double memory_limit;    /* bytes of solver scratch in global memory (0: 8 GiB); fewer CTAs when exceeded */
} lsb_raster_params;

/* Defaults: 8 neighbours, FP32 + refinement, tol 1e-12, max_iter 20000. */
void lsb_raster_params_default(lsb_raster_params *p);

/* Device bytes lsb_rasters needs for these raster sizes. */
int lsb_rasters_workspace_size(int64_t n, const int32_t *nx, const int32_t *ny, const lsb_raster_params *p,
                               size_t *bytes);

/* Solves the batch on `stream`.  With stats != NULL the call waits for the stream and reports solver failures
 * (LSB_ERR_NOT_CONVERGED); stats->n_targets is the number of rasters, n_solved those with a solved component. */
int lsb_rasters(int64_t n, const int32_t *nx, const int32_t *ny, const double *conductance, const double *source,
                const double *ground, const lsb_raster_params *p, double *current, double *voltage, void *workspace,
                size_t workspace_bytes, lsb_omni_stats *stats, char *err, size_t errlen, void *stream);

/* Tuning table (no counterpart in the reference): the preconditioner and threads per window that calls with
 * preconditioner = LSB_PC_AUTO or threads_per_window = 0 use for windows window_width = 2 (radius + buffer) + 1
 * cells wide, with these neighbours, edge weights and precision.  Entries come from an autotuning run
 * (landschaft_b200.autotune) or a saved table; without one the built-in rule applies (FP64: Jacobi, FP32 +
 * refinement: multigrid; 256 threads up to 1200 padded cells, else 512).  Process-wide and thread-safe.
 * lsb_tune_set returns LSB_OK or LSB_ERR_ARGUMENT; lsb_tune_get returns 1 and fills the outputs when an entry
 * exists, else 0. */
int lsb_tune_set(int32_t window_width, int32_t four_neighbors, int32_t edge_weights, int32_t precision,
                 int32_t preconditioner, int32_t threads_per_window);
int lsb_tune_get(int32_t window_width, int32_t four_neighbors, int32_t edge_weights, int32_t precision,
                 int32_t *preconditioner, int32_t *threads_per_window);
void lsb_tune_clear(void);

/* Library version string. */
const char *lsb_version(void);

/* ---- Circuitscape pairwise solves on a node graph ----------------------------------------------------------------
 * Replace, for one connected component, the factorisation and the batched back substitutions of
 * circuit::raster_pairwise (src/cpp/circuit/circuitscape.cpp:587-660, factor_component :93-141) and the node
 * currents of graph_node_currents (circuitscape.cpp:38-77).  The component has n nodes in CSR form: ptr[n + 1]
 * (int64), adj (int32, ascending within a row, local node numbers in the graph's order), w (edge conductances,
 * >= 0) and diag (the Laplacian's diagonal: the row's conductances summed, plus the shift of the reference's
 * factorisation).  Node `ground` is held at 0 V.  Job j draws a unit current from node src[j] and injects it at
 * dst[j] (either may be the ground); volt[j n + i] = v_i - v_src[j] (the voltages relative to the source, the
 * reference's per-pair voltages), and cur[j n + i] (when cur != NULL) = max(inflow, outflow) at node i, branch
 * currents under 1e-8 of the largest in- / outflow left out.  One CTA solves a job at a time (FP64 CG with Jacobi
 * preconditioning and true-residual restarts).  All pointers but stats and err are device pointers. */
typedef struct lsb_graph_params {
    double tol;        /* target relative residual ||b - A x|| / ||b|| (default 1e-14); the solve also stops when
                          the true residual stops decreasing */
    double accept;     /* a job whose final relative residual exceeds this fails (default 1e-9) */
    int32_t max_iter;  /* cap on CG iterations per job (0: 20 n + 2000) */
    int32_t max_ctas;  /* persistent CTAs (0: 4 per SM, fewer when the scratch exceeds 8 GiB) */
} lsb_graph_params;

typedef struct lsb_graph_stats {
    int64_t jobs;
    int64_t failures;       /* jobs above `accept` or out of iterations */
    int32_t iters_max;
    int32_t ctas;           /* CTAs launched */
    double iters_mean;
    double worst_residual;  /* largest final relative residual */
} lsb_graph_stats;

/* Defaults: tol 1e-14, accept 1e-9, max_iter 0, max_ctas 0. */
void lsb_graph_params_default(lsb_graph_params *p);

/* Device bytes lsb_graph_pairs needs. */
int lsb_graph_pairs_workspace_size(int64_t n, int64_t n_jobs, const lsb_graph_params *p, size_t *bytes);

/* Solves the jobs on `stream`.  With stats != NULL the call waits for the stream, fills the statistics and returns
 * LSB_ERR_NOT_CONVERGED when a job failed. */
int lsb_graph_pairs(int64_t n, const int64_t *ptr, const int32_t *adj, const double *w, const double *diag,
                    int32_t ground, int64_t n_jobs, const int32_t *src, const int32_t *dst,
                    const lsb_graph_params *p, double *volt, double *cur, void *workspace, size_t workspace_bytes,
                    lsb_graph_stats *stats, char *err, size_t errlen, void *stream);

/* Advanced-mode problems on one component (Circuitscape's advanced mode on node graphs, and one-to-all /
 * all-to-one, whose problems are one per focal point).  Replaces, per component and problem, the factorisation and
 * solve of circuit::raster_advanced / raster_advanced_many (src/cpp/circuit/circuitscape.cpp:393-470,904-1083) and
 * graph_node_currents with finite grounds (circuitscape.cpp:38-77).  The component is given as for
 * lsb_graph_pairs, with diag WITHOUT finite grounds.  Job j lists, as CSR over the jobs: its current sources
 * (src_node / src_val over src_ptr[j] .. src_ptr[j + 1]), its direct grounds held at 0 V (dir_node over dir_ptr) and
 * its finite grounds, added to the diagonal (fin_node / fin_val over fin_ptr); nodes are unique within each list,
 * and a direct ground's own source is ignored.  volt[j n + i] = the voltage of node i; cur[j n + i] (when
 * cur != NULL) = max(inflow, outflow), the current through a finite ground included.  All pointers but stats and
 * err are device pointers. */
int lsb_graph_solve_workspace_size(int64_t n, int64_t n_jobs, const lsb_graph_params *p, size_t *bytes);
int lsb_graph_solve(int64_t n, const int64_t *ptr, const int32_t *adj, const double *w, const double *diag,
                    int64_t n_jobs, const int64_t *src_ptr, const int32_t *src_node, const double *src_val,
                    const int64_t *dir_ptr, const int32_t *dir_node, const int64_t *fin_ptr,
                    const int32_t *fin_node, const double *fin_val, const lsb_graph_params *p, double *volt,
                    double *cur, void *workspace, size_t workspace_bytes, lsb_graph_stats *stats, char *err,
                    size_t errlen, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* LSB_OMNISCAPE_H */
