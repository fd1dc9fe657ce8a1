// oracle/ref_capi.cpp -- a C entry point into the reference's own Omniscape
// driver (circuit::omniscape, omniscape.hpp:56-60), its correction
// (omniscape.hpp:62-64) and its single-raster solve (circuit::advanced,
// grid.hpp:62-64), for ctypes.
//
// TEST INFRASTRUCTURE ONLY: the checker and the CPU baseline.  Mirrors what
// the reference's pybind11 binding does (src/cpp/circuit/python.cpp:90-153):
// fill OmniscapeParams, call, copy the result vectors out.
#include <cstdint>
#include <cstring>
#include <exception>
#include <stdexcept>

#include "circuit/grid.hpp"
#include "circuit/omniscape.hpp"

namespace {
void set_error(char* err, std::size_t len, const char* msg) {
    if (!err || len == 0) return;
    std::strncpy(err, msg, len - 1);
    err[len - 1] = '\0';
}
}  // namespace

extern "C" {

// Returns 0, 1 (invalid_argument) or 2 (runtime_error / other).
int ref_omniscape(const double* resistance, const double* source, std::int64_t nx, std::int64_t ny, int radius,
                  int buffer, int block_size, int four, int ric, int correct, int fp, const double* c1p,
                  const double* c1f, int c1eq, double c1lo, double c1hi, const double* c2p, const double* c2f,
                  int c2eq, double c2lo, double c2hi, double memory_limit, int threads, double* cur, double* fpout,
                  std::int64_t* n_targets, int* threads_used, char* err, std::size_t errlen) {
    try {
        circuit::OmniscapeParams p;
        p.radius = radius;
        p.buffer = buffer;
        p.block_size = block_size;
        p.four_neighbors = four != 0;
        p.resistance_is_conductance = ric != 0;
        p.correct_artifacts = correct != 0;
        p.flow_potential = fp != 0;
        p.condition1.present = c1p;
        p.condition1.future = c1f;
        p.condition1.equal = c1eq != 0;
        p.condition1.lower = c1lo;
        p.condition1.upper = c1hi;
        p.condition2.present = c2p;
        p.condition2.future = c2f;
        p.condition2.equal = c2eq != 0;
        p.condition2.lower = c2lo;
        p.condition2.upper = c2hi;
        p.memory_limit = memory_limit;
        circuit::OmniscapeResult r = circuit::omniscape(resistance, source, nx, ny, p, threads);
        std::memcpy(cur, r.current.data(), sizeof(double) * static_cast<std::size_t>(nx * ny));
        if (fp && fpout) std::memcpy(fpout, r.flow_potential.data(), sizeof(double) * static_cast<std::size_t>(nx * ny));
        *n_targets = r.n_targets;
        *threads_used = r.threads;
        return 0;
    } catch (const std::invalid_argument& e) {
        set_error(err, errlen, e.what());
        return 1;
    } catch (const std::exception& e) {
        set_error(err, errlen, e.what());
        return 2;
    }
}

int ref_correction(int radius, int buffer, int block_size, int four, std::int64_t nx, std::int64_t ny, double* corr,
                   char* err, std::size_t errlen) {
    try {
        circuit::OmniscapeParams p;
        p.radius = radius;
        p.buffer = buffer;
        p.block_size = block_size;
        p.four_neighbors = four != 0;
        const std::vector<double> c = circuit::omniscape_correction(p, nx, ny);
        std::memcpy(corr, c.data(), sizeof(double) * c.size());
        return 0;
    } catch (const std::exception& e) {
        set_error(err, errlen, e.what());
        return 2;
    }
}

int ref_advanced(const double* conductance, const double* source, const double* ground, std::int64_t nx,
                 std::int64_t ny, int four, int threads, double* current, double* voltage, char* err,
                 std::size_t errlen) {
    try {
        circuit::AdvancedResult r = circuit::advanced(conductance, source, ground, nx, ny, four != 0, threads);
        std::memcpy(current, r.current.data(), sizeof(double) * static_cast<std::size_t>(nx * ny));
        std::memcpy(voltage, r.voltage.data(), sizeof(double) * static_cast<std::size_t>(nx * ny));
        return 0;
    } catch (const std::exception& e) {
        set_error(err, errlen, e.what());
        return 2;
    }
}

}  // extern "C"
