/*
 * oracle/omni_oracle.c -- CPU restatement of landschaft's Omniscape moving-window
 * circuit path, in plain C with FP64 arithmetic.
 *
 * TEST INFRASTRUCTURE ONLY.  Only the test suite, the smoke check and the CPU
 * baseline leg of the benchmark load this library, as the checker.  The
 * product path (landschaft_b200) never calls it.
 *
 * Each function cites the reference function it restates (paths relative to
 * the landschaft source tree):
 *   node_currents        src/cpp/circuit/grid.cpp:19-71
 *   solve_window         src/cpp/circuit/omniscape.cpp:72-122
 *   flow window          src/cpp/circuit/omniscape.cpp:127-166 (one RHS at a time)
 *   block_condition      src/cpp/circuit/omniscape.cpp:170-215
 *   match_condition      src/cpp/circuit/omniscape.cpp:218-230
 *   orc_correction       src/cpp/circuit/omniscape.cpp:326-392
 *   orc_omniscape        src/cpp/circuit/omniscape.cpp:394-608
 *   orc_advanced         src/cpp/circuit/grid.cpp:73-210
 *   assembly             src/cpp/circuit/system.cpp:458-487 (+ edge_weight grid.hpp:37-40)
 *   resistor-series edge src/cpp/circuit/circuitscape.cpp:30-33
 *
 * The factorisation is not the reference's multifrontal Cholesky (which needs
 * Eigen 3.4, absent here); it is an envelope (skyline) Cholesky LL^T over the
 * unknowns in column-major order, exact up to rounding.  Everything around the
 * solve (targets, windows, sources and their quirks, correction, branch-current
 * threshold, scatter order) follows the reference step by step.
 *
 * The adjoint (orc_omniscape_grad) differentiates the same computation: for
 * each window the node currents' derivative with respect to the potentials is
 * solved with the same factor (the Laplacian is symmetric) and chained through
 * the edge weights, the conductance map and the source scaling.
 */
#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef int64_t i64;

#define K_TWO_SQRT2 2.8284271247461903 /* 2*sqrt(2) as Julia evaluates it (grid.hpp:17) */
#define K_SQRT2 1.4142135623730951
#define K_SHIFT (10 * DBL_EPSILON) /* CHOLMOD's diagonal shift (omniscape.cpp:28) */

/* Neighbours in increasing column-major index (grid.hpp:27-35): dy, dx, diagonal. */
static const int NB8[8][3] = {{-1, -1, 1}, {0, -1, 0}, {1, -1, 1}, {-1, 0, 0},
                              {1, 0, 0},   {-1, 1, 1}, {0, 1, 0},  {1, 1, 1}};
static const int NB4[4][3] = {{0, -1, 0}, {-1, 0, 0}, {1, 0, 0}, {0, 1, 0}};

/* Edge weight between two conductances: average conductance (grid.hpp:37-40),
 * or resistor-series (circuitscape.cpp:30-33). */
static double edge_w(double a, double b, int diag, int series) {
    if (series) return diag ? 1 / (K_SQRT2 * (1 / a + 1 / b) / 2) : 1 / ((1 / a + 1 / b) / 2);
    return diag ? (a + b) / K_TWO_SQRT2 : (a + b) / 2;
}

/* ---------------------------------------------------------------------------
 * Envelope Cholesky of a grid Laplacian over a list of unknown cells.
 * ------------------------------------------------------------------------- */
typedef struct {
    i64 n;
    i64 *first; /* first column of row i inside the envelope */
    i64 *off;   /* row i's entries L[i][first..i] start at L + off[i] */
    double *L;
    i64 cap_n, cap_l;
} Env;

static void env_free(Env *e) {
    free(e->first);
    free(e->off);
    free(e->L);
    memset(e, 0, sizeof *e);
}

static int env_reserve(Env *e, i64 n, i64 nl) {
    if (n > e->cap_n) {
        free(e->first);
        free(e->off);
        e->first = (i64 *)malloc(sizeof(i64) * (size_t)n);
        e->off = (i64 *)malloc(sizeof(i64) * (size_t)(n + 1));
        if (!e->first || !e->off) return -1;
        e->cap_n = n;
    }
    if (nl > e->cap_l) {
        free(e->L);
        e->L = (double *)malloc(sizeof(double) * (size_t)nl);
        if (!e->L) return -1;
        e->cap_l = nl;
    }
    return 0;
}

/* Working storage of one thread. */
typedef struct {
    i64 cap;
    unsigned char *present;
    i64 *stack, *idx, *cells;
    double *b, *x, *v, *lam, *dv, *edges;
    Env env;
} WS;

static void ws_free(WS *ws) {
    free(ws->present);
    free(ws->stack);
    free(ws->idx);
    free(ws->cells);
    free(ws->b);
    free(ws->x);
    free(ws->v);
    free(ws->lam);
    free(ws->dv);
    free(ws->edges);
    env_free(&ws->env);
    memset(ws, 0, sizeof *ws);
}

static int ws_reserve(WS *ws, i64 n) {
    if (n <= ws->cap) return 0;
    ws_free(ws);
    ws->present = (unsigned char *)malloc((size_t)n);
    ws->stack = (i64 *)malloc(sizeof(i64) * (size_t)n);
    ws->idx = (i64 *)malloc(sizeof(i64) * (size_t)n);
    ws->cells = (i64 *)malloc(sizeof(i64) * (size_t)n);
    ws->b = (double *)malloc(sizeof(double) * (size_t)n);
    ws->x = (double *)malloc(sizeof(double) * (size_t)n);
    ws->v = (double *)malloc(sizeof(double) * (size_t)n);
    ws->lam = (double *)malloc(sizeof(double) * (size_t)n);
    ws->dv = (double *)malloc(sizeof(double) * (size_t)n);
    ws->edges = (double *)malloc(sizeof(double) * (size_t)n * 4);
    if (!ws->present || !ws->stack || !ws->idx || !ws->cells || !ws->b || !ws->x || !ws->v || !ws->lam ||
        !ws->dv || !ws->edges)
        return -1;
    ws->cap = n;
    return 0;
}

/*
 * Assemble and factorise the grounded Laplacian over the unknown cells of a
 * w x h box (row-major): unknown[c] != 0.  Cells with present[c] != 0 are
 * nodes (a present cell that is not an unknown is a direct ground at 0 V).
 * The diagonal of an unknown is the sum, in column-major neighbour order, of
 * its edges to present cells, plus extra_diag[c] when given, plus the 10 eps
 * shift (system.cpp:458-487).  Unknowns are numbered in column-major order
 * (ws->idx: cell -> unknown, ws->cells: unknown -> cell).  Returns -1 when the
 * matrix is not positive definite, -2 when out of memory.
 */
static int factorise(WS *ws, i64 w, i64 h, const double *g, const unsigned char *present, const unsigned char *unknown,
                     const double *extra_diag, int four, int series, i64 *n_out) {
    const int nd = four ? 4 : 8;
    const int(*nb)[3] = four ? NB4 : NB8;
    i64 n = 0;
    for (i64 x = 0; x < w; ++x)
        for (i64 y = 0; y < h; ++y) {
            const i64 c = y * w + x;
            if (unknown[c]) {
                ws->idx[c] = n;
                ws->cells[n++] = c;
            } else {
                ws->idx[c] = -1;
            }
        }
    *n_out = n;
    /* envelope: first[i] = smallest unknown index among i and its unknown neighbours */
    i64 total = 0;
    if (env_reserve(&ws->env, n, 1) < 0) return -2;
    Env *e = &ws->env;
    for (i64 i = 0; i < n; ++i) {
        const i64 c = ws->cells[i], y = c / w, x = c % w;
        i64 f = i;
        for (int d = 0; d < nd; ++d) {
            const i64 yy = y + nb[d][0], xx = x + nb[d][1];
            if (yy < 0 || yy >= h || xx < 0 || xx >= w) continue;
            const i64 j = ws->idx[yy * w + xx];
            if (j >= 0 && j < f) f = j;
        }
        e->first[i] = f;
        e->off[i] = total;
        total += i - f + 1;
    }
    e->off[n] = total;
    if (env_reserve(e, n, total > 0 ? total : 1) < 0) return -2;
    e->n = n;
    double *L = e->L;
    memset(L, 0, sizeof(double) * (size_t)total);
    /* values: row i holds A[i][first..i] */
    for (i64 i = 0; i < n; ++i) {
        const i64 c = ws->cells[i], y = c / w, x = c % w;
        double *row = L + e->off[i] - e->first[i];
        double diag = 0.0;
        if (!present[c]) {
            row[i] = 1.0; /* identity row for an unknown that is not a node */
            continue;
        }
        for (int d = 0; d < nd; ++d) {
            const i64 yy = y + nb[d][0], xx = x + nb[d][1];
            if (yy < 0 || yy >= h || xx < 0 || xx >= w) continue;
            const i64 q = yy * w + xx;
            if (!present[q]) continue;
            const double wt = edge_w(g[c], g[q], nb[d][2], series);
            diag += wt;
            const i64 j = ws->idx[q];
            if (j >= 0 && j < i) row[j] = -wt;
        }
        if (extra_diag) diag += extra_diag[c];
        row[i] = diag + K_SHIFT;
    }
    /* row-oriented envelope LL^T */
    for (i64 i = 0; i < n; ++i) {
        double *Li = L + e->off[i] - e->first[i];
        const i64 fi = e->first[i];
        for (i64 j = fi; j < i; ++j) {
            double *Lj = L + e->off[j] - e->first[j];
            const i64 k0 = fi > e->first[j] ? fi : e->first[j];
            double s = Li[j];
            for (i64 k = k0; k < j; ++k) s -= Li[k] * Lj[k];
            Li[j] = s / Lj[j];
        }
        double s = Li[i];
        for (i64 k = fi; k < i; ++k) s -= Li[k] * Li[k];
        if (!(s > 0)) return -1;
        Li[i] = sqrt(s);
    }
    return 0;
}

/* x = A^-1 b with the envelope factor (x may alias b). */
static void env_solve(const Env *e, const double *b, double *x) {
    const i64 n = e->n;
    const double *L = e->L;
    if (x != b) memcpy(x, b, sizeof(double) * (size_t)n);
    for (i64 i = 0; i < n; ++i) {
        const double *Li = L + e->off[i] - e->first[i];
        double s = x[i];
        for (i64 k = e->first[i]; k < i; ++k) s -= Li[k] * x[k];
        x[i] = s / Li[i];
    }
    for (i64 i = n - 1; i >= 0; --i) {
        const double *Li = L + e->off[i] - e->first[i];
        const double xi = x[i] / Li[i];
        x[i] = xi;
        for (i64 k = e->first[i]; k < i; ++k) x[k] -= Li[k] * xi;
    }
}

/* ---------------------------------------------------------------------------
 * Node currents (grid.cpp:19-71).
 * ------------------------------------------------------------------------- */
static void node_currents(i64 w, i64 h, const double *g, const unsigned char *present, const double *v,
                          const double *finite, int four, int series, double *cur, double *edges) {
    const int nd = four ? 4 : 8, lower = four ? 2 : 4, nf = nd - lower;
    const int(*nb)[3] = four ? NB4 : NB8;
    const i64 n = w * h;
    double maxin = -INFINITY, maxout = -INFINITY;
    for (i64 q = 0; q < n; ++q) {
        if (!present[q]) continue;
        const i64 y = q / w, x = q % w;
        for (int d = lower; d < nd; ++d) {
            const i64 yy = y + nb[d][0], xx = x + nb[d][1];
            if (yy < 0 || yy >= h || xx < 0 || xx >= w) continue;
            const i64 r = yy * w + xx;
            if (!present[r]) continue;
            const double b = edge_w(g[q], g[r], nb[d][2], series) * (v[r] - v[q]);
            edges[q * nf + (d - lower)] = b;
            if (b > maxout) maxout = b;
            if (-b > maxin) maxin = -b;
        }
    }
    for (i64 q = 0; q < n; ++q) {
        if (!present[q]) continue;
        const i64 y = q / w, x = q % w;
        double inflow = 0.0, outflow = 0.0;
        for (int d = 0; d < nd; ++d) {
            const i64 yy = y + nb[d][0], xx = x + nb[d][1];
            if (yy < 0 || yy >= h || xx < 0 || xx >= w) continue;
            const i64 r = yy * w + xx;
            if (!present[r]) continue;
            const double b = d < lower ? -edges[r * nf + (nd - 1 - d - lower)] : edges[q * nf + (d - lower)];
            if (b > 0) {
                if (!(fabs(b / maxin) < 1e-8)) inflow += b;
            } else if (b < 0) {
                if (!(fabs(b / maxout) < 1e-8)) outflow -= b;
            }
        }
        if (finite) {
            const double f = finite[q] * v[q];
            if (f < 0)
                inflow -= f;
            else if (f > 0)
                outflow += f;
        }
        cur[q] = inflow > outflow ? inflow : outflow;
    }
}

/* ---------------------------------------------------------------------------
 * One window (omniscape.cpp:72-122): the ground's component by flood fill,
 * its RHS, the solve and the node currents.  `v_out` (optional) receives the
 * potentials, `present_out` (optional) the component.
 * ------------------------------------------------------------------------- */
static int solve_window(WS *ws, i64 h, i64 w, const double *g, const double *src, i64 gy, i64 gx, int four,
                        int series, double *cur, double *v_out, unsigned char *present_out) {
    const i64 n = h * w;
    const int nd = four ? 4 : 8;
    const int(*nb)[3] = four ? NB4 : NB8;
    for (i64 q = 0; q < n; ++q) cur[q] = 0.0;
    if (v_out)
        for (i64 q = 0; q < n; ++q) v_out[q] = 0.0;
    unsigned char *present = ws->present;
    memset(present, 0, (size_t)n);
    if (present_out) memset(present_out, 0, (size_t)n);
    const i64 ground = gy * w + gx;
    if (!(g[ground] > 0)) return 0; /* the ground has no node */
    present[ground] = 1;
    i64 top = 0;
    ws->stack[top++] = ground;
    double total = 0.0;
    while (top > 0) {
        const i64 p = ws->stack[--top];
        const i64 y = p / w, x = p % w;
        for (int d = 0; d < nd; ++d) {
            const i64 yy = y + nb[d][0], xx = x + nb[d][1];
            if (yy < 0 || yy >= h || xx < 0 || xx >= w) continue;
            const i64 q = yy * w + xx;
            if (!present[q] && g[q] > 0) {
                present[q] = 1;
                total += src[q];
                ws->stack[top++] = q;
            }
        }
    }
    if (present_out) memcpy(present_out, present, (size_t)n);
    if (total == 0) return 0; /* no source in the ground's component */
    /* unknowns: present cells without the ground */
    unsigned char *unknown = (unsigned char *)malloc((size_t)n);
    if (!unknown) return -2;
    for (i64 q = 0; q < n; ++q) unknown[q] = present[q];
    unknown[ground] = 0;
    i64 m = 0;
    const int rc = factorise(ws, w, h, g, present, unknown, NULL, four, series, &m);
    free(unknown);
    if (rc) return rc;
    for (i64 k = 0; k < m; ++k) ws->b[k] = src[ws->cells[k]];
    env_solve(&ws->env, ws->b, ws->x);
    double *v = ws->v;
    for (i64 q = 0; q < n; ++q) v[q] = 0.0;
    for (i64 k = 0; k < m; ++k) v[ws->cells[k]] = ws->x[k];
    node_currents(w, h, g, present, v, NULL, four, series, cur, ws->edges);
    if (v_out) memcpy(v_out, v, sizeof(double) * (size_t)n);
    return 0;
}

/* The flow potential of one window (omniscape.cpp:127-166 for one RHS):
 * conductance 1 on the whole h x w rectangle. */
static int flow_window(WS *ws, i64 h, i64 w, const double *src, i64 gy, i64 gx, int four, int series, double *cur,
                       double *v_out) {
    const i64 n = h * w, ground = gy * w + gx;
    for (i64 q = 0; q < n; ++q) cur[q] = 0.0;
    if (v_out)
        for (i64 q = 0; q < n; ++q) v_out[q] = 0.0;
    double total = 0.0;
    for (i64 q = 0; q < n; ++q)
        if (q != ground) total += src[q];
    if (total == 0) return 0;
    double *ones = (double *)malloc(sizeof(double) * (size_t)n);
    unsigned char *all = (unsigned char *)malloc((size_t)n), *unknown = (unsigned char *)malloc((size_t)n);
    if (!ones || !all || !unknown) {
        free(ones);
        free(all);
        free(unknown);
        return -2;
    }
    for (i64 q = 0; q < n; ++q) {
        ones[q] = 1.0;
        all[q] = 1;
        unknown[q] = q != ground;
    }
    i64 m = 0;
    int rc = factorise(ws, w, h, ones, all, unknown, NULL, four, series, &m);
    if (!rc) {
        for (i64 k = 0; k < m; ++k) ws->b[k] = src[ws->cells[k]];
        env_solve(&ws->env, ws->b, ws->x);
        double *v = ws->v;
        for (i64 q = 0; q < n; ++q) v[q] = 0.0;
        for (i64 k = 0; k < m; ++k) v[ws->cells[k]] = ws->x[k];
        node_currents(w, h, ones, all, v, NULL, four, series, cur, ws->edges);
        if (v_out) memcpy(v_out, v, sizeof(double) * (size_t)n);
    }
    free(ones);
    free(all);
    free(unknown);
    return rc;
}

/* ---------------------------------------------------------------------------
 * Conditions (omniscape.cpp:170-230).
 * ------------------------------------------------------------------------- */
typedef struct {
    const double *present, *future;
    int equal;
    double lower, upper;
} OrcCondition;

static int cmp_double(const void *a, const void *b) {
    const double x = *(const double *)a, y = *(const double *)b;
    return x < y ? -1 : x > y ? 1 : 0;
}

/* The block's value: median ("within") or StatsBase mode ("equal") of the
 * future (else present) values, column-major, NaN left out.  Returns 0 and
 * sets *out, or -3 when the block has no value. */
static int block_condition(const OrcCondition *c, i64 nx, i64 ny, i64 x, i64 y, i64 br, double *buf, double *out) {
    const double *f = c->future ? c->future : c->present;
    i64 n = 0;
    for (i64 xx = x - br; xx <= (x + br < nx - 1 ? x + br : nx - 1); ++xx)
        for (i64 yy = y - br; yy <= (y + br < ny - 1 ? y + br : ny - 1); ++yy) {
            const double v = f[yy * nx + xx];
            if (!isnan(v)) buf[n++] = v;
        }
    if (n == 0) return -3;
    if (!c->equal) {
        double *tmp = buf + n;
        memcpy(tmp, buf, sizeof(double) * (size_t)n);
        qsort(tmp, (size_t)n, sizeof(double), cmp_double);
        if (n % 2 == 1) {
            *out = tmp[n / 2];
        } else {
            const double b = tmp[n / 2], a = tmp[n / 2 - 1];
            *out = a / 2 + b / 2; /* Statistics.median's middle(a, b) */
        }
        return 0;
    }
    /* first value (in order) to exceed the running highest count; 0.0 and -0.0 apart */
    double best = buf[0];
    int top = 0;
    for (i64 i = 0; i < n; ++i) {
        uint64_t bi;
        memcpy(&bi, &buf[i], sizeof bi);
        int cnt = 0;
        for (i64 j = 0; j <= i; ++j) {
            uint64_t bj;
            memcpy(&bj, &buf[j], sizeof bj);
            if (bj == bi) ++cnt;
        }
        if (cnt > top) {
            top = cnt;
            best = buf[i];
        }
    }
    *out = best;
    return 0;
}

static void match_condition(const OrcCondition *c, double value, i64 nx, i64 x0, i64 y0, i64 h, i64 w, double *src) {
    for (i64 y = 0; y < h; ++y)
        for (i64 x = 0; x < w; ++x) {
            const double v = c->present[(y0 + y) * nx + (x0 + x)];
            if (isnan(v)) continue;
            if (c->equal) {
                if (v != value) src[y * w + x] = 0.0;
            } else {
                const double d = v - value;
                if (d > c->upper || d < c->lower) src[y * w + x] = 0.0;
            }
        }
}

/* ---------------------------------------------------------------------------
 * Parameters and targets.
 * ------------------------------------------------------------------------- */
typedef struct {
    int radius, buffer, block_size;
    int four_neighbors, resistance_is_conductance, correct_artifacts, flow_potential, series;
    OrcCondition cond[2];
} OrcParams;

typedef struct {
    i64 x, y;
    double amps;
    i64 h, w, gy, gx;
    i64 y0, x0;
    i64 order; /* enumeration index (stable-sort tie break) */
} Target;

static int target_cmp(const void *pa, const void *pb) {
    const Target *a = (const Target *)pa, *b = (const Target *)pb;
#define CMP(f)                      \
    if (a->f != b->f) return a->f < b->f ? -1 : 1;
    CMP(h) CMP(w) CMP(gy) CMP(gx) CMP(order)
#undef CMP
    return 0;
}

/* Targets (omniscape.cpp:406-424): block centres with a positive
 * column-major sum of sources, stable-sorted by window shape. */
static Target *enumerate_targets(const double *source, i64 nx, i64 ny, i64 D, i64 bs, i64 *count) {
    const i64 br = (bs - 1) / 2;
    i64 cap = 0;
    for (i64 x = br; x + br < nx; x += bs)
        for (i64 y = br; y + br < ny; y += bs) ++cap;
    Target *t = (Target *)malloc(sizeof(Target) * (size_t)(cap > 0 ? cap : 1));
    if (!t) return NULL;
    i64 n = 0;
    for (i64 x = br; x + br < nx; x += bs)
        for (i64 y = br; y + br < ny; y += bs) {
            double amps = 0.0;
            for (i64 xx = x - br; xx <= x + br; ++xx)
                for (i64 yy = y - br; yy <= y + br; ++yy) {
                    const double v = source[yy * nx + xx];
                    if (!isnan(v)) amps += v;
                }
            if (!(amps > 0)) continue;
            Target *T = &t[n];
            T->x = x;
            T->y = y;
            T->amps = amps;
            T->y0 = y - D > 0 ? y - D : 0;
            T->x0 = x - D > 0 ? x - D : 0;
            const i64 y1 = y + D < ny - 1 ? y + D : ny - 1, x1 = x + D < nx - 1 ? x + D : nx - 1;
            T->h = y1 - T->y0 + 1;
            T->w = x1 - T->x0 + 1;
            T->gy = y - T->y0;
            T->gx = x - T->x0;
            T->order = n;
            ++n;
        }
    qsort(t, (size_t)n, sizeof(Target), target_cmp);
    *count = n;
    return t;
}

/* Window conductance and sources of a target (omniscape.cpp:495-530). */
static int build_window(const Target *t, const double *resistance, const double *source, i64 nx, i64 ny,
                        const OrcParams *p, double *g, double *src, double *cbuf) {
    const i64 R = p->radius, D = R + p->buffer, br = (p->block_size - 1) / 2;
    const i64 h = t->h, w = t->w;
    for (i64 y = 0; y < h; ++y)
        for (i64 x = 0; x < w; ++x) {
            const i64 dy = y - t->gy, dx = x - t->gx;
            const double r = resistance[(t->y0 + y) * nx + (t->x0 + x)];
            double c = -9999.0;
            if (dy * dy + dx * dx <= D * D && !isnan(r)) c = p->resistance_is_conductance ? r : 1 / r;
            g[y * w + x] = c;
        }
    for (i64 y = 0; y < h; ++y)
        for (i64 x = 0; x < w; ++x) {
            const i64 dy = y - t->gy, dx = x - t->gx;
            double v = 0.0;
            if (dy * dy + dx * dx <= R * R) {
                v = source[(t->y0 + y) * nx + (t->x0 + x)];
                if (isnan(v)) v = 0.0;
            }
            src[y * w + x] = v;
        }
    /* the target block zeroed at radius + buffer from the corner (the quirk) */
    for (i64 y = D - br; y <= (D + br < ny - 1 ? D + br : ny - 1); ++y)
        for (i64 x = D - br; x <= (D + br < nx - 1 ? D + br : nx - 1); ++x)
            if (y >= 0 && y < h && x >= 0 && x < w) src[y * w + x] = 0.0;
    double sum = 0.0;
    for (i64 x = 0; x < w; ++x)
        for (i64 y = 0; y < h; ++y)
            if (src[y * w + x] > 0) sum += src[y * w + x];
    for (i64 q = 0; q < h * w; ++q)
        if (src[q] > 0) src[q] = (src[q] * t->amps) / sum;
    for (int k = 0; k < 2; ++k) {
        const OrcCondition *c = &p->cond[k];
        if (!c->present) continue;
        double value;
        if (block_condition(c, nx, ny, t->x, t->y, br, cbuf, &value)) return -3;
        match_condition(c, value, nx, t->x0, t->y0, h, w, src);
    }
    return 0;
}

/* ---------------------------------------------------------------------------
 * Correction (omniscape.cpp:326-392).
 * ------------------------------------------------------------------------- */
int orc_correction(int radius, int buffer, int block_size, int four, int series, i64 nx, i64 ny, double *corr) {
    const i64 R = radius, B = buffer, D = R + B, W = 2 * D + 1;
    const i64 bs = block_size, br = (bs - 1) / 2;
    const i64 n = W * W;
    double *g = (double *)malloc(sizeof(double) * (size_t)n * 5);
    if (!g) return -2;
    double *null_src = g + n, *block_src = g + 2 * n, *block_cur = g + 3 * n, *null_cur = g + 4 * n;
    double n_sources = 0;
    for (i64 y = 0; y < W; ++y)
        for (i64 x = 0; x < W; ++x) {
            const i64 d2 = (y - D) * (y - D) + (x - D) * (x - D);
            g[y * W + x] = d2 <= D * D ? 1.0 : -9999.0;
            null_src[y * W + x] = block_src[y * W + x] = 0.0;
            if (d2 <= R * R) {
                null_src[y * W + x] = 1.0;
                block_src[y * W + x] = 1.0;
                n_sources += 1;
            }
        }
    null_src[D * W + D] = 0.0;
    for (i64 q = 0; q < n; ++q)
        if (null_src[q] != 0.0) null_src[q] = 1 / (n_sources - 1);
    for (i64 y = D - br; y <= (D + br < ny - 1 ? D + br : ny - 1); ++y)
        for (i64 x = D - br; x <= (D + br < nx - 1 ? D + br : nx - 1); ++x)
            if (y >= 0 && y < W && x >= 0 && x < W) block_src[y * W + x] = 0.0;
    double sum = 0.0;
    for (i64 x = 0; x < W; ++x)
        for (i64 y = 0; y < W; ++y)
            if (block_src[y * W + x] > 0) sum += block_src[y * W + x];
    const double amps = (double)(bs * bs);
    for (i64 q = 0; q < n; ++q)
        if (block_src[q] > 0) block_src[q] = (block_src[q] * amps) / sum;
    WS ws;
    memset(&ws, 0, sizeof ws);
    int rc = ws_reserve(&ws, n);
    if (!rc) rc = solve_window(&ws, W, W, g, block_src, D, D, four, series, block_cur, NULL, NULL);
    if (!rc) rc = solve_window(&ws, W, W, g, null_src, D, D, four, series, null_cur, NULL, NULL);
    ws_free(&ws);
    if (rc) {
        free(g);
        return rc;
    }
    const i64 T = 2 * D + bs;
    double *total = (double *)calloc((size_t)(T * T), sizeof(double));
    if (!total) {
        free(g);
        return -2;
    }
    for (i64 i = 0; i < bs; ++i)
        for (i64 j = 0; j < bs; ++j)
            for (i64 y = 0; y < W; ++y)
                for (i64 x = 0; x < W; ++x) total[(i + y) * T + (j + x)] += null_cur[y * W + x];
    double top = -INFINITY;
    for (i64 q = 0; q < n; ++q)
        if (block_cur[q] > top) top = block_cur[q];
    const double floor_ = 1e-6 * top;
    for (i64 y = 0; y < W; ++y)
        for (i64 x = 0; x < W; ++x) {
            double b = block_cur[y * W + x];
            double t = total[(y + br) * T + (x + br)];
            if (b <= floor_) b = 0.0;
            if (b == 0.0) t = 0.0;
            if (t == 0.0) t = 1.0;
            if (b == 0.0) b = 1.0;
            corr[y * W + x] = t / b;
        }
    free(total);
    free(g);
    return 0;
}

/* ---------------------------------------------------------------------------
 * The moving-window run (omniscape.cpp:394-608).
 *
 * Returns 0, or -1 (a window not positive definite), -2 (out of memory), -3 (a
 * block with no condition value), -4 (bad parameters).  `max_targets` >= 0
 * solves only the first targets of the shape-sorted order (a timing sample).
 * ------------------------------------------------------------------------- */
static int run_omniscape(const double *resistance, const double *source, i64 nx, i64 ny, const OrcParams *p,
                         int threads, i64 max_targets, double *cur_out, double *fp_out, i64 *n_targets) {
    if (p->radius < 0 || p->buffer < 0 || p->block_size < 1 || p->block_size % 2 == 0) return -4;
    const i64 R = p->radius, D = R + p->buffer, bs = p->block_size, W = 2 * D + 1;
    const int fp = p->flow_potential;
    const int correct = p->correct_artifacts && bs > 1;
    for (i64 q = 0; q < nx * ny; ++q) {
        cur_out[q] = 0.0;
        if (fp) fp_out[q] = 0.0;
    }
    i64 nt = 0;
    Target *targets = enumerate_targets(source, nx, ny, D, bs, &nt);
    if (!targets) return -2;
    *n_targets = nt;
    if (max_targets >= 0 && max_targets < nt) nt = max_targets;
    if (nt == 0) {
        free(targets);
        return 0;
    }
    double *corr = NULL;
    if (correct) {
        corr = (double *)malloc(sizeof(double) * (size_t)(W * W));
        if (!corr) {
            free(targets);
            return -2;
        }
        const int rc = orc_correction((int)R, p->buffer, (int)bs, p->four_neighbors, p->series, nx, ny, corr);
        if (rc) {
            free(corr);
            free(targets);
            return rc;
        }
    }
#ifdef _OPENMP
    if (threads <= 0) threads = omp_get_max_threads();
#else
    threads = 1;
#endif
    const i64 window = W * W;
    i64 batch = (i64)((size_t)512 << 20) / (window * (fp ? 2 : 1) * (i64)sizeof(double));
    if (batch < 1) batch = 1;
    if (batch > nt) batch = nt;
    double *cur = (double *)malloc(sizeof(double) * (size_t)(batch * window));
    double *fpc = fp ? (double *)malloc(sizeof(double) * (size_t)(batch * window)) : NULL;
    if (!cur || (fp && !fpc)) {
        free(cur);
        free(fpc);
        free(corr);
        free(targets);
        return -2;
    }
    int error = 0;
    for (i64 start = 0; start < nt && !error; start += batch) {
        const i64 count = nt - start < batch ? nt - start : batch;
#pragma omp parallel num_threads(threads)
        {
            WS ws;
            memset(&ws, 0, sizeof ws);
            double *g = (double *)malloc(sizeof(double) * (size_t)window * 2);
            double *cbuf = (double *)malloc(sizeof(double) * (size_t)(2 * bs * bs));
            if (!g || !cbuf || ws_reserve(&ws, window) < 0) {
#pragma omp critical(orc_error)
                error = -2;
            }
#pragma omp for schedule(dynamic, 1)
            for (i64 k = 0; k < count; ++k) {
                if (error) continue;
                const Target *t = &targets[start + k];
                double *src = g + window, *c = cur + k * window;
                int rc = build_window(t, resistance, source, nx, ny, p, g, src, cbuf);
                if (!rc) rc = solve_window(&ws, t->h, t->w, g, src, t->gy, t->gx, p->four_neighbors, p->series, c, NULL,
                                           NULL);
                if (!rc && fp)
                    rc = flow_window(&ws, t->h, t->w, src, t->gy, t->gx, p->four_neighbors, p->series,
                                     fpc + k * window, NULL);
                if (rc) {
#pragma omp critical(orc_error)
                    error = rc;
                    continue;
                }
                if (correct) {
                    const i64 cx0 = t->x < D && t->x + D <= nx - 1 ? W - t->w : 0;
                    const i64 cy0 = t->y < D && t->y + D <= ny - 1 ? W - t->h : 0;
                    for (i64 y = 0; y < t->h; ++y)
                        for (i64 x = 0; x < t->w; ++x) {
                            const double k2 = corr[(cy0 + y) * W + (cx0 + x)];
                            c[y * t->w + x] *= k2;
                            if (fp) fpc[k * window + y * t->w + x] *= k2;
                        }
                }
            }
            ws_free(&ws);
            free(g);
            free(cbuf);
        }
        if (error) break;
        /* add the windows row by row, each row in target order */
#pragma omp parallel for schedule(static) num_threads(threads)
        for (i64 row = 0; row < ny; ++row) {
            for (i64 k = 0; k < count; ++k) {
                const Target *t = &targets[start + k];
                const i64 y = row - t->y0;
                if (y < 0 || y >= t->h) continue;
                const double *c = cur + k * window + y * t->w;
                double *dst = cur_out + row * nx + t->x0;
                for (i64 x = 0; x < t->w; ++x) dst[x] += c[x];
                if (fp) {
                    const double *f = fpc + k * window + y * t->w;
                    double *fdst = fp_out + row * nx + t->x0;
                    for (i64 x = 0; x < t->w; ++x) fdst[x] += f[x];
                }
            }
        }
    }
    free(cur);
    free(fpc);
    free(corr);
    free(targets);
    return error;
}

static void fill_params(OrcParams *p, int radius, int buffer, int block_size, int four, int ric, int correct, int fp,
                        int series, const double *c1p, const double *c1f, int c1eq, double c1lo, double c1hi,
                        const double *c2p, const double *c2f, int c2eq, double c2lo, double c2hi) {
    p->radius = radius;
    p->buffer = buffer;
    p->block_size = block_size;
    p->four_neighbors = four;
    p->resistance_is_conductance = ric;
    p->correct_artifacts = correct;
    p->flow_potential = fp;
    p->series = series;
    p->cond[0].present = c1p;
    p->cond[0].future = c1f;
    p->cond[0].equal = c1eq;
    p->cond[0].lower = c1lo;
    p->cond[0].upper = c1hi;
    p->cond[1].present = c2p;
    p->cond[1].future = c2f;
    p->cond[1].equal = c2eq;
    p->cond[1].lower = c2lo;
    p->cond[1].upper = c2hi;
}

int orc_omniscape(const double *resistance, const double *source, i64 nx, i64 ny, int radius, int buffer,
                  int block_size, int four, int ric, int correct, int fp, int series, const double *c1p,
                  const double *c1f, int c1eq, double c1lo, double c1hi, const double *c2p, const double *c2f,
                  int c2eq, double c2lo, double c2hi, int threads, i64 max_targets, double *cur, double *fpout,
                  i64 *n_targets) {
    OrcParams p;
    fill_params(&p, radius, buffer, block_size, four, ric, correct, fp, series, c1p, c1f, c1eq, c1lo, c1hi, c2p, c2f,
                c2eq, c2lo, c2hi);
    return run_omniscape(resistance, source, nx, ny, &p, threads, max_targets, cur, fpout, n_targets);
}

/* Number of targets without solving anything (for sampling decisions). */
i64 orc_count_targets(const double *source, i64 nx, i64 ny, int radius, int buffer, int block_size) {
    i64 n = 0;
    Target *t = enumerate_targets(source, nx, ny, (i64)radius + buffer, block_size, &n);
    free(t);
    return t ? n : -1;
}

/* ---------------------------------------------------------------------------
 * Advanced mode on one raster (grid.cpp:73-210), components solved one by one.
 * ------------------------------------------------------------------------- */
int orc_advanced(const double *conductance, const double *source, const double *ground, i64 nx, i64 ny, int four,
                 int series, double *current, double *voltage) {
    const i64 n = nx * ny;
    const int nd = four ? 4 : 8;
    const int(*nb)[3] = four ? NB4 : NB8;
    int32_t *comp = (int32_t *)malloc(sizeof(int32_t) * (size_t)n);
    i64 *stack = (i64 *)malloc(sizeof(i64) * (size_t)n);
    double *src = (double *)calloc((size_t)n, sizeof(double)), *gnd = (double *)calloc((size_t)n, sizeof(double));
    double *fin = (double *)calloc((size_t)n, sizeof(double));
    if (!comp || !stack || !src || !gnd || !fin) return -2;
    for (i64 c = 0; c < n; ++c) {
        current[c] = 0.0;
        voltage[c] = NAN;
        comp[c] = -1;
    }
    int32_t n_comp = 0;
    for (i64 c = 0; c < n; ++c) {
        if (!(conductance[c] > 0) || comp[c] >= 0) continue;
        comp[c] = n_comp;
        i64 top = 0;
        stack[top++] = c;
        while (top > 0) {
            const i64 p = stack[--top], y = p / nx, x = p % nx;
            for (int d = 0; d < nd; ++d) {
                const i64 yy = y + nb[d][0], xx = x + nb[d][1];
                if (yy < 0 || yy >= ny || xx < 0 || xx >= nx) continue;
                const i64 q = yy * nx + xx;
                if (conductance[q] > 0 && comp[q] < 0) {
                    comp[q] = n_comp;
                    stack[top++] = q;
                }
            }
        }
        ++n_comp;
    }
    int any_finite = 0;
    for (i64 c = 0; c < n; ++c) {
        if (comp[c] < 0) continue;
        voltage[c] = 0.0;
        src[c] = source ? source[c] : 0.0;
        gnd[c] = ground ? ground[c] : 0.0;
        if (gnd[c] < INFINITY) fin[c] = gnd[c];
        if (fin[c] != 0) any_finite = 1;
        if (src[c] != 0 && gnd[c] != 0) src[c] = 0.0;
    }
    /* per component: bounding box, unknowns, solve, currents */
    int rc = 0;
    for (int32_t k = 0; k < n_comp && !rc; ++k) {
        double s = 0.0, gsum = 0.0;
        i64 x0 = nx, x1 = -1, y0 = ny, y1 = -1;
        for (i64 x = 0; x < nx; ++x)
            for (i64 y = 0; y < ny; ++y) {
                const i64 c = y * nx + x;
                if (comp[c] != k) continue;
                s += src[c];
                gsum += gnd[c];
                if (x < x0) x0 = x;
                if (x > x1) x1 = x;
                if (y < y0) y0 = y;
                if (y > y1) y1 = y;
            }
        if (!(s != 0 && gsum != 0)) continue;
        const i64 bx = x1 - x0 + 1, by = y1 - y0 + 1, bn = bx * by;
        unsigned char *present = (unsigned char *)calloc((size_t)bn, 1), *unknown = (unsigned char *)calloc((size_t)bn, 1);
        double *g = (double *)calloc((size_t)bn, sizeof(double)), *fg = (double *)calloc((size_t)bn, sizeof(double));
        double *b = (double *)calloc((size_t)bn, sizeof(double)), *v = (double *)calloc((size_t)bn, sizeof(double));
        double *cur = (double *)calloc((size_t)bn, sizeof(double)), *edges = (double *)malloc(sizeof(double) * (size_t)bn * 4);
        WS ws;
        memset(&ws, 0, sizeof ws);
        if (!present || !unknown || !g || !fg || !b || !v || !cur || !edges || ws_reserve(&ws, bn) < 0) rc = -2;
        int any_unknown = 0;
        for (i64 y = y0; !rc && y <= y1; ++y)
            for (i64 x = x0; x <= x1; ++x) {
                const i64 c = y * nx + x, q = (y - y0) * bx + (x - x0);
                if (comp[c] != k) continue;
                present[q] = 1;
                unknown[q] = gnd[c] != INFINITY;
                any_unknown |= unknown[q];
                g[q] = conductance[c];
                fg[q] = fin[c];
                b[q] = src[c];
            }
        if (!rc && any_unknown) {
            i64 m = 0;
            rc = factorise(&ws, bx, by, g, present, unknown, any_finite ? fg : NULL, four, series, &m);
            if (!rc) {
                for (i64 i = 0; i < m; ++i) ws.b[i] = b[ws.cells[i]];
                env_solve(&ws.env, ws.b, ws.x);
                for (i64 i = 0; i < m; ++i) v[ws.cells[i]] = ws.x[i];
            }
        }
        if (!rc) {
            node_currents(bx, by, g, present, v, any_finite ? fg : NULL, four, series, cur, edges);
            for (i64 y = y0; y <= y1; ++y)
                for (i64 x = x0; x <= x1; ++x) {
                    const i64 c = y * nx + x, q = (y - y0) * bx + (x - x0);
                    if (comp[c] != k) continue;
                    current[c] = cur[q];
                    voltage[c] = v[q];
                }
        }
        ws_free(&ws);
        free(present);
        free(unknown);
        free(g);
        free(fg);
        free(b);
        free(v);
        free(cur);
        free(edges);
    }
    free(comp);
    free(stack);
    free(src);
    free(gnd);
    free(fin);
    return rc;
}

/* ---------------------------------------------------------------------------
 * FP64 adjoint of the cumulative current (test oracle for the GPU adjoint).
 *
 * J = sum_cells weight[cell] * cum_current[cell].  Returns dJ/dresistance (or
 * dJ/dconductance with resistance_is_conductance) and dJ/dsource, both
 * ny x nx.  Per window: dJ/dv from the node-current formula with the
 * threshold set frozen, lambda = A^-1 dJ/dv (A symmetric), then
 *   dJ/dg_c = explicit part (edge weights in the branch currents)
 *           - sum over edges e=(c,n) of dw_e/dg_c (lambda_c - lambda_n)(v_c - v_n)
 *   dJ/dsrc  = lambda on the unknowns, chained through the source scaling.
 * Windows whose flood fill or threshold set would change under a perturbation
 * are not special-cased: the derivative is that of the branch of the
 * piecewise-smooth map the current inputs sit on.  Only the cumulative current
 * (not the flow potential) is differentiated; conditions are not supported.
 * ------------------------------------------------------------------------- */

/* d(edge weight)/d(first conductance) */
static double edge_dw(double a, double b, int diag, int series) {
    if (series) {
        /* w = 2/(k(1/a + 1/b)), dw/da = 2/(k (1/a+1/b)^2) / a^2 */
        const double k = diag ? K_SQRT2 : 1.0, s = 1 / a + 1 / b;
        return 2.0 / (k * s * s) / (a * a);
    }
    (void)a;
    (void)b;
    return diag ? 1.0 / K_TWO_SQRT2 : 0.5;
}

/* Window adjoint: given the solved window (present, v, branch maxima), the
 * weights wq[] of the window cells in J; accumulates dJ/dg into dg[] and
 * dJ/d(window source, before scaling) into dsrc[] (both h*w). */
static int window_adjoint(WS *ws, i64 h, i64 w, const double *g, const unsigned char *present, const double *v,
                          i64 gy, i64 gx, int four, int series, const double *wq, double *dg, double *dsrc) {
    const int nd = four ? 4 : 8, lower = four ? 2 : 4;
    const int(*nb)[3] = four ? NB4 : NB8;
    const i64 n = h * w, ground = gy * w + gx;
    /* branch maxima as in node_currents */
    double maxin = -INFINITY, maxout = -INFINITY;
    for (i64 q = 0; q < n; ++q) {
        if (!present[q]) continue;
        const i64 y = q / w, x = q % w;
        for (int d = lower; d < nd; ++d) {
            const i64 yy = y + nb[d][0], xx = x + nb[d][1];
            if (yy < 0 || yy >= h || xx < 0 || xx >= w) continue;
            const i64 r = yy * w + xx;
            if (!present[r]) continue;
            const double b = edge_w(g[q], g[r], nb[d][2], series) * (v[r] - v[q]);
            if (b > maxout) maxout = b;
            if (-b > maxin) maxin = -b;
        }
    }
    /* dJ/d(branch b_qn) for every directed branch seen from q: cur_q = max(in, out) */
    double *dv = ws->dv;
    for (i64 q = 0; q < n; ++q) dv[q] = 0.0;
    for (i64 q = 0; q < n; ++q) {
        if (!present[q] || wq[q] == 0) continue;
        const i64 y = q / w, x = q % w;
        double inflow = 0.0, outflow = 0.0;
        for (int d = 0; d < nd; ++d) {
            const i64 yy = y + nb[d][0], xx = x + nb[d][1];
            if (yy < 0 || yy >= h || xx < 0 || xx >= w) continue;
            const i64 r = yy * w + xx;
            if (!present[r]) continue;
            const double b = edge_w(g[q], g[r], nb[d][2], series) * (v[r] - v[q]);
            if (b > 0) {
                if (!(fabs(b / maxin) < 1e-8)) inflow += b;
            } else if (b < 0) {
                if (!(fabs(b / maxout) < 1e-8)) outflow -= b;
            }
        }
        const int use_in = inflow > outflow; /* cur = inflow when inflow > outflow, else outflow */
        for (int d = 0; d < nd; ++d) {
            const i64 yy = y + nb[d][0], xx = x + nb[d][1];
            if (yy < 0 || yy >= h || xx < 0 || xx >= w) continue;
            const i64 r = yy * w + xx;
            if (!present[r]) continue;
            const double we = edge_w(g[q], g[r], nb[d][2], series);
            const double b = we * (v[r] - v[q]);
            double s = 0.0; /* d cur_q / d b */
            if (use_in && b > 0 && !(fabs(b / maxin) < 1e-8)) s = 1.0;
            if (!use_in && b < 0 && !(fabs(b / maxout) < 1e-8)) s = -1.0;
            if (s == 0.0) continue;
            const double c = wq[q] * s; /* dJ/db */
            /* b = we (v_r - v_q) */
            dv[r] += c * we;
            dv[q] -= c * we;
            const double dw_q = edge_dw(g[q], g[r], nb[d][2], series), dw_r = edge_dw(g[r], g[q], nb[d][2], series);
            dg[q] += c * dw_q * (v[r] - v[q]);
            dg[r] += c * dw_r * (v[r] - v[q]);
        }
    }
    /* lambda = A^-1 dJ/dv over the unknowns (the factor of this window is in ws) */
    i64 m = ws->env.n;
    for (i64 k = 0; k < m; ++k) ws->b[k] = dv[ws->cells[k]];
    env_solve(&ws->env, ws->b, ws->x);
    double *lam = ws->lam;
    for (i64 q = 0; q < n; ++q) lam[q] = 0.0;
    for (i64 k = 0; k < m; ++k) lam[ws->cells[k]] = ws->x[k];
    /* dJ/dsrc = lambda (unknowns only; the ground and absent cells get 0) */
    for (i64 q = 0; q < n; ++q) dsrc[q] += (present[q] && q != ground) ? lam[q] : 0.0;
    /* dJ/dg through A: - lambda^T dA/dg v; A = sum_e w_e (e_c - e_n)(e_c - e_n)^T over edges to present cells */
    for (i64 q = 0; q < n; ++q) {
        if (!present[q]) continue;
        const i64 y = q / w, x = q % w;
        for (int d = lower; d < nd; ++d) {
            const i64 yy = y + nb[d][0], xx = x + nb[d][1];
            if (yy < 0 || yy >= h || xx < 0 || xx >= w) continue;
            const i64 r = yy * w + xx;
            if (!present[r]) continue;
            const double t = (lam[q] - lam[r]) * (v[q] - v[r]);
            dg[q] -= edge_dw(g[q], g[r], nb[d][2], series) * t;
            dg[r] -= edge_dw(g[r], g[q], nb[d][2], series) * t;
        }
    }
    return 0;
}

/*
 * J = sum weight * cum_current; grad_r (ny x nx, dJ/dresistance or
 * dJ/dconductance) and grad_s (dJ/dsource), accumulated over the windows.
 * Optionally returns J itself.  Block size must give no correction (bs 1 or
 * correct_artifacts off) and no conditions; flow potential is not included.
 */
int orc_omniscape_grad(const double *resistance, const double *source, i64 nx, i64 ny, int radius, int buffer,
                       int block_size, int four, int ric, int series, const double *weight, int threads,
                       double *grad_r, double *grad_s, double *J_out) {
    OrcParams p;
    fill_params(&p, radius, buffer, block_size, four, ric, 0, 0, series, NULL, NULL, 0, 0, 0, NULL, NULL, 0, 0, 0);
    if (radius < 0 || buffer < 0 || block_size < 1 || block_size % 2 == 0) return -4;
    const i64 R = radius, D = R + buffer, bs = block_size, br = (bs - 1) / 2, W = 2 * D + 1, window = W * W;
    if (br > D) return -4;
    i64 nt = 0;
    Target *targets = enumerate_targets(source, nx, ny, D, bs, &nt);
    if (!targets) return -2;
    for (i64 q = 0; q < nx * ny; ++q) grad_r[q] = grad_s[q] = 0.0;
    double J = 0.0;
#ifdef _OPENMP
    if (threads <= 0) threads = omp_get_max_threads();
#else
    threads = 1;
#endif
    i64 batch = (i64)((size_t)256 << 20) / (window * 2 * (i64)sizeof(double));
    if (batch < 1) batch = 1;
    if (batch > nt) batch = nt > 0 ? nt : 1;
    /* per-target gradient windows of a batch, then summed in target order (deterministic) */
    double *dgw = (double *)malloc(sizeof(double) * (size_t)batch * (size_t)window);
    double *dsw = (double *)malloc(sizeof(double) * (size_t)batch * (size_t)window);
    double *Jw = (double *)calloc((size_t)batch, sizeof(double));
    if (!dgw || !dsw || !Jw) {
        free(dgw);
        free(dsw);
        free(Jw);
        free(targets);
        return -2;
    }
    int error = 0;
    for (i64 start = 0; start < nt && !error; start += batch) {
        const i64 count = nt - start < batch ? nt - start : batch;
#pragma omp parallel num_threads(threads)
        {
            WS ws;
            memset(&ws, 0, sizeof ws);
            double *g = (double *)malloc(sizeof(double) * (size_t)window * 6);
            unsigned char *present = (unsigned char *)malloc((size_t)window);
            if (!g || !present || ws_reserve(&ws, window) < 0) {
#pragma omp critical(orc_error)
                error = -2;
            }
#pragma omp for schedule(dynamic, 1)
            for (i64 k = 0; k < count; ++k) {
                if (error) continue;
                const Target *t = &targets[start + k];
                const i64 h = t->h, w = t->w, n = h * w;
                double *src = g + window, *cur = g + 2 * window, *v = g + 3 * window, *wq = g + 4 * window,
                       *raw = g + 5 * window;
                double *dg = dgw + k * window, *ds = dsw + k * window;
                for (i64 q = 0; q < window; ++q) dg[q] = ds[q] = 0.0;
                Jw[k] = 0.0;
                int rc = build_window(t, resistance, source, nx, ny, &p, g, src, NULL);
                if (!rc) rc = solve_window(&ws, h, w, g, src, t->gy, t->gx, four, series, cur, v, present);
                if (rc) {
#pragma omp critical(orc_error)
                    error = rc;
                    continue;
                }
                double Jk = 0.0;
                int any = 0;
                for (i64 y = 0; y < h; ++y)
                    for (i64 x = 0; x < w; ++x) {
                        const double wt = weight[(t->y0 + y) * nx + (t->x0 + x)];
                        wq[y * w + x] = wt;
                        Jk += wt * cur[y * w + x];
                        if (wt != 0 && cur[y * w + x] != 0) any = 1;
                    }
                Jw[k] = Jk;
                /* no current under the weights: nothing to differentiate (solve_window left the
                   factor of this window in ws only when it solved) */
                if (!any) continue;
                double *dsrc = ds; /* dJ/d(scaled source) first */
                window_adjoint(&ws, h, w, g, present, v, t->gy, t->gx, four, series, wq, dg, dsrc);
                /* chain through the source scaling: src_q = s_q amps / sum over positives (s after the
                   disk, NaN and quirk masking); amps = sum of the block's raw sources */
                double sum = 0.0;
                for (i64 y = 0; y < h; ++y)
                    for (i64 x = 0; x < w; ++x) {
                        const i64 dy = y - t->gy, dx = x - t->gx;
                        double s = 0.0;
                        if (dy * dy + dx * dx <= R * R) {
                            s = source[(t->y0 + y) * nx + (t->x0 + x)];
                            if (isnan(s)) s = 0.0;
                        }
                        raw[y * w + x] = s;
                    }
                for (i64 y = D - br; y <= (D + br < ny - 1 ? D + br : ny - 1); ++y)
                    for (i64 x = D - br; x <= (D + br < nx - 1 ? D + br : nx - 1); ++x)
                        if (y >= 0 && y < h && x >= 0 && x < w) raw[y * w + x] = 0.0;
                for (i64 x = 0; x < w; ++x)
                    for (i64 y = 0; y < h; ++y)
                        if (raw[y * w + x] > 0) sum += raw[y * w + x];
                double slam = 0.0;
                for (i64 q = 0; q < n; ++q)
                    if (raw[q] > 0) slam += raw[q] * dsrc[q];
                const double amps = t->amps;
                for (i64 q = 0; q < n; ++q) {
                    const double lamq = dsrc[q];
                    dsrc[q] = raw[q] > 0 ? (amps / sum) * lamq - (amps / (sum * sum)) * slam : 0.0;
                }
                /* amps: the block around the target (map coordinates), inside the window as br <= D */
                const double damps = slam / sum;
                for (i64 yy = t->y - br; yy <= t->y + br; ++yy)
                    for (i64 xx = t->x - br; xx <= t->x + br; ++xx) {
                        if (isnan(source[yy * nx + xx])) continue;
                        dsrc[(yy - t->y0) * w + (xx - t->x0)] += damps;
                    }
                /* conductance -> resistance */
                for (i64 y = 0; y < h; ++y)
                    for (i64 x = 0; x < w; ++x) {
                        const double r = resistance[(t->y0 + y) * nx + (t->x0 + x)];
                        const i64 q = y * w + x;
                        if (!(g[q] > 0)) {
                            dg[q] = 0.0;
                            continue;
                        }
                        if (!ric) dg[q] *= -1.0 / (r * r);
                    }
            }
            ws_free(&ws);
            free(g);
            free(present);
        }
        if (error) break;
        for (i64 k = 0; k < count; ++k) J += Jw[k];
#pragma omp parallel for schedule(static) num_threads(threads)
        for (i64 row = 0; row < ny; ++row)
            for (i64 k = 0; k < count; ++k) {
                const Target *t = &targets[start + k];
                const i64 y = row - t->y0;
                if (y < 0 || y >= t->h) continue;
                for (i64 x = 0; x < t->w; ++x) {
                    grad_r[row * nx + t->x0 + x] += dgw[k * window + y * t->w + x];
                    grad_s[row * nx + t->x0 + x] += dsw[k * window + y * t->w + x];
                }
            }
    }
    if (J_out) *J_out = J;
    free(dgw);
    free(dsw);
    free(Jw);
    free(targets);
    return error;
}
