// oracle/ref_shim.cpp -- a CellSystem for building the reference's own driver.
//
// TEST INFRASTRUCTURE ONLY (the CPU baseline and the checker).
//
// landschaft's src/cpp/circuit/omniscape.cpp and grid.cpp compile without
// third-party code; src/cpp/circuit/system.cpp does not (it needs Eigen 3.4,
// which its build fetches from the network).  This file implements the
// interface that system.hpp declares (frontal_analyze, CellSystem) with an
// envelope Cholesky written here, so that the reference's driver -- targets,
// windows, source quirks, correction, node currents, scatter -- runs
// unchanged.  Only the factorisation differs from the reference, and only in
// rounding: the matrix is assembled exactly as system.cpp:458-487 does
// (neighbour order, 10 eps shift, identity rows for unknowns that are not
// nodes), and solved exactly.
//
// Layout of the shared structure (the header's fields, used as this file
// defines them):
//   cells       unknown -> box cell, column-major order (row-major when the
//               box is taller than wide: the envelope is the shorter side)
//   unknown_of  box cell -> unknown (-1: none)
//   nbr         unknown k's neighbour unknowns at [k nd, (k+1) nd) (-1: none)
//   relmap      first column of each row of the envelope of L
//   adj_ptr     start of each row of L in the factor (n + 1 entries)
//   lsize       doubles of L
#include <algorithm>
#include <cmath>
#include <cstring>
#include <stdexcept>

#include "circuit/system.hpp"

namespace circuit {

std::shared_ptr<const FrontalSymbolic> frontal_analyze(i64 bx, i64 by, const std::uint8_t* unknown,
                                                       bool four_neighbors) {
    auto s = std::make_shared<FrontalSymbolic>();
    s->bx = bx;
    s->by = by;
    s->four = four_neighbors;
    const int nd = four_neighbors ? 4 : 8;
    const Offset* nb = four_neighbors ? kNeighbours4 : kNeighbours8;
    s->unknown_of.assign(static_cast<std::size_t>(bx * by), -1);
    const bool col_major = by <= bx;
    const i64 outer = col_major ? bx : by, inner = col_major ? by : bx;
    for (i64 a = 0; a < outer; ++a)
        for (i64 b = 0; b < inner; ++b) {
            const i64 c = col_major ? b * bx + a : a * bx + b;
            if (!unknown[c]) continue;
            s->unknown_of[static_cast<std::size_t>(c)] = static_cast<std::int32_t>(s->cells.size());
            s->cells.push_back(c);
        }
    const i64 n = static_cast<i64>(s->cells.size());
    s->nbr.assign(static_cast<std::size_t>(n * nd), -1);
    s->relmap.resize(static_cast<std::size_t>(n));
    s->adj_ptr.resize(static_cast<std::size_t>(n + 1));
    std::int64_t total = 0;
    for (i64 k = 0; k < n; ++k) {
        const i64 c = s->cells[static_cast<std::size_t>(k)], y = c / bx, x = c % bx;
        std::int32_t f = static_cast<std::int32_t>(k);
        for (int d = 0; d < nd; ++d) {
            const i64 yy = y + nb[d].dy, xx = x + nb[d].dx;
            if (yy < 0 || yy >= by || xx < 0 || xx >= bx) continue;
            const std::int32_t j = s->unknown_of[static_cast<std::size_t>(yy * bx + xx)];
            s->nbr[static_cast<std::size_t>(k * nd + d)] = j;
            if (j >= 0 && j < f) f = j;
        }
        s->relmap[static_cast<std::size_t>(k)] = f;
        s->adj_ptr[static_cast<std::size_t>(k)] = total;
        total += k - f + 1;
    }
    s->adj_ptr[static_cast<std::size_t>(n)] = total;
    s->lsize = total;
    s->max_front = 0;
    s->stack_size = 0;
    return s;
}

void CellSystem::analyze(i64 bx, i64 by, const std::uint8_t* unknown, bool four_neighbors) {
    share(frontal_analyze(bx, by, unknown, four_neighbors));
}

void CellSystem::share(std::shared_ptr<const FrontalSymbolic> symbolic) {
    sym_ = std::move(symbolic);
    diag_.assign(sym_->cells.size(), 1.0);
    off_.assign(sym_->nbr.size(), 0.0);
}

void CellSystem::set_values(const double* diag, const double* off) {
    std::copy(diag, diag + diag_.size(), diag_.begin());
    std::copy(off, off + off_.size(), off_.begin());
}

void CellSystem::assemble(const double* g, const std::uint8_t* present, const double* extra_diag, double shift) {
    const FrontalSymbolic& s = *sym_;
    const Offset* nb = s.four ? kNeighbours4 : kNeighbours8;
    const int nd = s.four ? 4 : 8;
    const i64 n = size();
    for (i64 j = 0; j < n; ++j) {
        const i64 c = s.cells[static_cast<std::size_t>(j)];
        double* off = off_.data() + j * nd;
        if (!present[c]) {
            std::fill(off, off + nd, 0.0);
            diag_[static_cast<std::size_t>(j)] = 1.0;
            continue;
        }
        const i64 y = c / s.bx, x = c % s.bx;
        double diag = 0.0;
        for (int d = 0; d < nd; ++d) {
            const i64 yy = y + nb[d].dy, xx = x + nb[d].dx;
            if (yy < 0 || yy >= s.by || xx < 0 || xx >= s.bx || !present[yy * s.bx + xx]) {
                off[d] = 0.0;
                continue;
            }
            const double w = edge_weight(g[c], g[yy * s.bx + xx], nb[d].diagonal);
            diag += w;
            off[d] = -w;
        }
        if (extra_diag) diag += extra_diag[c];
        diag_[static_cast<std::size_t>(j)] = diag + shift;
    }
}

bool CellSystem::factorize() { return factorize(nullptr); }

// Envelope LL^T in l_; with y, also the forward substitution L z = y in place.
bool CellSystem::factorize(double* y) {
    const FrontalSymbolic& s = *sym_;
    const int nd = s.four ? 4 : 8;
    const i64 n = size();
    double* L = l_.get(static_cast<std::size_t>(std::max<std::int64_t>(s.lsize, 1)));
    std::memset(L, 0, sizeof(double) * static_cast<std::size_t>(s.lsize));
    auto row = [&](i64 i) { return L + s.adj_ptr[static_cast<std::size_t>(i)] - s.relmap[static_cast<std::size_t>(i)]; };
    for (i64 i = 0; i < n; ++i) {
        double* Li = row(i);
        Li[i] = diag_[static_cast<std::size_t>(i)];
        for (int d = 0; d < nd; ++d) {
            const std::int32_t j = s.nbr[static_cast<std::size_t>(i * nd + d)];
            if (j >= 0 && j < i) Li[j] = off_[static_cast<std::size_t>(i * nd + d)];
        }
    }
    for (i64 i = 0; i < n; ++i) {
        double* Li = row(i);
        const i64 fi = s.relmap[static_cast<std::size_t>(i)];
        for (i64 j = fi; j < i; ++j) {
            const double* Lj = row(j);
            const i64 k0 = std::max<i64>(fi, s.relmap[static_cast<std::size_t>(j)]);
            double t = Li[j];
            for (i64 k = k0; k < j; ++k) t -= Li[k] * Lj[k];
            Li[j] = t / Lj[j];
        }
        double t = Li[i];
        for (i64 k = fi; k < i; ++k) t -= Li[k] * Li[k];
        if (!(t > 0)) return false;
        Li[i] = std::sqrt(t);
        if (y) {
            double z = y[i];
            for (i64 k = fi; k < i; ++k) z -= Li[k] * y[k];
            y[i] = z / Li[i];
        }
    }
    return true;
}

bool CellSystem::factorize_solve(const double* b, double* x) {
    const i64 n = size();
    if (x != b) std::copy(b, b + n, x);
    if (!factorize(x)) return false;
    // backward L^T x = z
    const FrontalSymbolic& s = *sym_;
    const double* L = l_.get(static_cast<std::size_t>(std::max<std::int64_t>(s.lsize, 1)));
    for (i64 i = n - 1; i >= 0; --i) {
        const double* Li = L + s.adj_ptr[static_cast<std::size_t>(i)] - s.relmap[static_cast<std::size_t>(i)];
        const double xi = x[i] / Li[i];
        x[i] = xi;
        for (i64 k = s.relmap[static_cast<std::size_t>(i)]; k < i; ++k) x[k] -= Li[k] * xi;
    }
    return true;
}

void CellSystem::solve_many(double* x, i64 k, SolveScratch&) const {
    const FrontalSymbolic& s = *sym_;
    const i64 n = static_cast<i64>(s.cells.size());
    // l_ is only read here; AlignedBuffer::get does not reallocate when the size fits.
    const double* L = const_cast<AlignedBuffer&>(l_).get(static_cast<std::size_t>(std::max<std::int64_t>(s.lsize, 1)));
    for (i64 c = 0; c < k; ++c) {
        double* v = x + c * n;
        for (i64 i = 0; i < n; ++i) {
            const double* Li = L + s.adj_ptr[static_cast<std::size_t>(i)] - s.relmap[static_cast<std::size_t>(i)];
            double t = v[i];
            for (i64 q = s.relmap[static_cast<std::size_t>(i)]; q < i; ++q) t -= Li[q] * v[q];
            v[i] = t / Li[i];
        }
        for (i64 i = n - 1; i >= 0; --i) {
            const double* Li = L + s.adj_ptr[static_cast<std::size_t>(i)] - s.relmap[static_cast<std::size_t>(i)];
            const double vi = v[i] / Li[i];
            v[i] = vi;
            for (i64 q = s.relmap[static_cast<std::size_t>(i)]; q < i; ++q) v[q] -= Li[q] * vi;
        }
    }
}

void CellSystem::solve_many(double* x, i64 k) { solve_many(x, k, scratch_); }

void CellSystem::solve(const double* b, double* x) {
    const i64 n = size();
    if (x != b) std::copy(b, b + n, x);
    solve_many(x, 1, scratch_);
}

}  // namespace circuit
