// SolverNumerics.h - the shared 2-D solver numerics of the SeisWave Lab API
// (Main_header/SolverNumerics.h), over the B200 solver's C ABI (include/seis2d_capi.h).
// Same names and signatures; the checks run in the library and rethrow the reference's
// exception types.
#pragma once

#include <array>
#include <cmath>
#include <cstddef>
#include <limits>
#include <stdexcept>
#include <string>

#include "../seis2d_capi.h"

constexpr int kStencilRadius = SEIS2D_STENCIL_RADIUS;
constexpr int kMaximumActiveSources = SEIS2D_MAX_ACTIVE_SOURCES;
constexpr float kSourceInjectionScale2D = SEIS2D_SOURCE_INJECTION_SCALE;

namespace seis2d_compat {

inline void check(int status) {
    if (status == SEIS2D_OK) return;
    const std::string message = seis2d_last_error();
    if (status == SEIS2D_INVALID_ARGUMENT) throw std::invalid_argument(message);
    if (status == SEIS2D_OVERFLOW_ERROR) throw std::overflow_error(message);
    if (status == SEIS2D_LOGIC_ERROR) throw std::logic_error(message);
    throw std::runtime_error(message);
}

inline std::array<double, 4> weights() {
    std::array<double, 4> w{};
    seis2d_stencil_weights(w.data());
    return w;
}

}  // namespace seis2d_compat

// Eighth-order staggered first-derivative weights (taps at 1/2, 3/2, 5/2, 7/2).
inline const std::array<double, 4> kStaggeredDerivativeWeights = seis2d_compat::weights();
inline const double kDerivativeWeightMagnitude = kStaggeredDerivativeWeights[0] - kStaggeredDerivativeWeights[1] +
                                                 kStaggeredDerivativeWeights[2] - kStaggeredDerivativeWeights[3];
inline const float kCourantLimit2d = seis2d_courant_limit();
inline const float kSafeCourant2d = seis2d_safe_courant();

inline size_t checkedGridElementCount(int nx, int nz) {
    int64_t count = 0;
    seis2d_compat::check(seis2d_checked_grid_element_count(nx, nz, &count));
    return size_t(count);
}

inline void validateBoundaryGeometry(int nx, int nz, int pmlWidth, bool freeSurface) {
    seis2d_compat::check(seis2d_validate_boundary_geometry(nx, nz, pmlWidth, freeSurface ? 1 : 0));
}

inline int getReceiverSamplingStride(double timeStep, double samplingRateHz) {
    int stride = 0;
    seis2d_compat::check(seis2d_receiver_sampling_stride(timeStep, samplingRateHz, &stride));
    return stride;
}
