// tlw_limiter.hpp -- TEST INFRASTRUCTURE ONLY (the oracle): the Zhang-Shu positivity-preserving limiter as
// TrixiLW applies it after a step, restated on the CPU.
//
// Follows my_limiter_zhang_shu! (src/callbacks/callbacks_stage/positivity_zhang_shu.jl:10-42: the
// (threshold, variable) pairs in their order) and, per pair, the element pass of
// src/callbacks/callbacks_stage/positivity_zhang_shu_dg2d.jl:8-45 followed by the TreeMesh mortar pass
// limit_mortars! (:47-176). Parity status: unpinned against the reference itself (no Julia here).
//
// Element pass: value_min over the element's nodes; only if value_min < threshold, the GLL mean
// u_mean = sum_ij u_ij w_i w_j / 4 (reference weights, no Jacobian), theta = (value(u_mean) - threshold) /
// (value(u_mean) - value_min) and u <- theta u + (1 - theta) u_mean on every node.
// Mortar pass, per mortar in order: the large element's mean and the value of the large face trace
// interpolated onto both halves (forward_upper / forward_lower); theta = min(|(value_mean - threshold) /
// (value_mean - value_min)|, 1), applied to the large element unconditionally. Only the large element is read
// or written there (the small elements' traces and means that the reference also fills are not used), so the
// pass touches each large element through its own mortars only. The reference prints theta for every mortar
// (@show): a debugging print, not restated.
//
// Julia's min propagates NaN (min(x, NaN) = NaN, and NaN < threshold is false, so an element holding a NaN is
// left alone); julia_min restates that.
#pragma once
#include <cmath>
#include <limits>
#include <vector>

#include "tlw_oracle.hpp"

namespace tlwo {

enum LimiterVariable { LIMIT_DENSITY = 0, LIMIT_PRESSURE = 1, LIMIT_DENSITY_PRESSURE = 2 };

// Trixi density / pressure / density_pressure of CompressibleEulerEquations2D
inline double limiter_value(const Euler& eq, int variable, const double* u) {
    const double rho = u[0], m1 = u[1], m2 = u[2], e = u[3];
    if (variable == LIMIT_DENSITY) return rho;
    if (variable == LIMIT_PRESSURE) return (eq.gamma - 1.0) * (e - 0.5 * (m1 * m1 + m2 * m2) / rho);
    return (eq.gamma - 1.0) * (e * rho - 0.5 * (m1 * m1 + m2 * m2));
}

inline double julia_min(double a, double b) {
    if (std::isnan(a) || std::isnan(b)) return std::numeric_limits<double>::quiet_NaN();
    return b < a ? b : a;
}

struct PositivityLimiter {
    std::vector<double> thresholds;
    std::vector<int> variables;
};

// mean over the element on the GLL quadrature of the reference element (weights sum to 2 per direction)
inline void element_mean(const Basis& b, const double* u, int e, double* mean) {
    const int n = b.n;
    for (int v = 0; v < NV; ++v) mean[v] = 0.0;
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i)
            for (int v = 0; v < NV; ++v) mean[v] += u[idx_u(n, v, i, j, e)] * b.weights[i] * b.weights[j];
    for (int v = 0; v < NV; ++v) mean[v] = mean[v] / 4.0;
}

inline void blend_element(const Basis& b, double* u, int e, double theta, const double* mean) {
    const int n = b.n;
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i)
            for (int v = 0; v < NV; ++v) {
                double& x = u[idx_u(n, v, i, j, e)];
                x = theta * x + (1.0 - theta) * mean[v];
            }
}

// positivity_zhang_shu_dg2d.jl:8-45 (one threshold / variable)
inline void limit_elements(const Basis& b, const Euler& eq, int n_elements, double* u, double threshold,
                           int variable) {
    const int n = b.n;
    for (int e = 0; e < n_elements; ++e) {
        double vmin = std::numeric_limits<double>::infinity();   // typemax(Float64)
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < n; ++i) {
                double x[NV];
                for (int v = 0; v < NV; ++v) x[v] = u[idx_u(n, v, i, j, e)];
                vmin = julia_min(vmin, limiter_value(eq, variable, x));
            }
        if (!(vmin < threshold)) continue;
        double mean[NV];
        element_mean(b, u, e, mean);
        const double vmean = limiter_value(eq, variable, mean);
        const double theta = (vmean - threshold) / (vmean - vmin);
        blend_element(b, u, e, theta, mean);
    }
}

// limit_mortars!(u, threshold, variable, mesh::TreeMesh{2}, ...) (positivity_zhang_shu_dg2d.jl:47-176)
inline void limit_mortars(const Basis& b, const Euler& eq, const TreeMesh& m, double* u, double threshold,
                          int variable) {
    const int n = b.n;
    std::vector<double> face(n * NV);
    for (int k = 0; k < m.n_mortars; ++k) {
        const int le = m.mortar_large[k];
        const int o = m.mortar_orientation[k];
        // large_sides == 1: the large element is on the -side, its +x (o = 1) or +y (o = 2) face
        const int fi = m.mortar_large_side[k] == 1 ? n - 1 : 0;
        double mean[NV];
        element_mean(b, u, le, mean);
        const double vmean = limiter_value(eq, variable, mean);
        for (int l = 0; l < n; ++l)
            for (int v = 0; v < NV; ++v)
                face[l * NV + v] = o == 1 ? u[idx_u(n, v, fi, l, le)] : u[idx_u(n, v, l, fi, le)];
        double vmin = std::numeric_limits<double>::infinity();   // typemax(Float64)
        for (int jm = 0; jm < n; ++jm) {
            double up[NV] = {0, 0, 0, 0}, lo[NV] = {0, 0, 0, 0};
            for (int l = 0; l < n; ++l)
                for (int v = 0; v < NV; ++v) {
                    up[v] += b.fwd_upper[jm * n + l] * face[l * NV + v];
                    lo[v] += b.fwd_lower[jm * n + l] * face[l * NV + v];
                }
            vmin = julia_min(julia_min(vmin, limiter_value(eq, variable, up)), limiter_value(eq, variable, lo));
        }
        const double theta = julia_min(std::fabs((vmean - threshold) / (vmean - vmin)), 1.0);
        blend_element(b, u, le, theta, mean);
    }
}

// one application of the limiter: every (threshold, variable) pair in order, elements then mortars
inline void apply_positivity_limiter(const Basis& b, const Euler& eq, const TreeMesh& m, int n_elements,
                                     const PositivityLimiter& lim, double* u) {
    for (size_t p = 0; p < lim.thresholds.size(); ++p) {
        limit_elements(b, eq, n_elements, u, lim.thresholds[p], lim.variables[p]);
        if (m.n_mortars > 0) limit_mortars(b, eq, m, u, lim.thresholds[p], lim.variables[p]);
    }
}

}  // namespace tlwo
