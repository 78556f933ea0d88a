// tlw_limiter.cuh -- Zhang-Shu positivity-preserving limiter (Trixi's PositivityPreservingLimiterZhangShu as
// TrixiLW applies it: src/callbacks/callbacks_stage/positivity_zhang_shu.jl:10-42 and
// positivity_zhang_shu_dg2d.jl:8-176), fused into one pass over the state after a step.
//
// Per (threshold, variable) pair, in order: the element pass (value_min over the nodes; if below the threshold,
// theta = (value(u_mean) - threshold) / (value(u_mean) - value_min) with the GLL mean u_mean = sum w_i w_j u / 4
// and u <- theta u + (1 - theta) u_mean), then on a TreeMesh with mortars the mortar pass of limit_mortars!,
// which reads and writes only each mortar's large element: the large face trace interpolated onto both halves,
// theta = min(|(value_mean - threshold) / (value_mean - value_min)|, 1), applied unconditionally. Both passes
// of every pair (and repeated applications) are element-local, so one warp takes an element through all of
// them with its nodes in registers: the state is read once and written back only where something was
// limited. Julia's NaN-propagating min is kept (an element with a NaN value is not limited).
//
// On the plain LW step with CFL slots the kernel also rewrites the slots of the elements it changed (their
// maxima of |v1| + c and |v2| + c), so the next step's dt still comes from the limited state without another
// pass over it.
#pragma once
#include "tlw_device.cuh"
#include "tlw_mortar.cuh"

namespace tlw {

constexpr int LIMITER_MAX_PAIRS = 4;
constexpr int LIMITER_WARPS = 4;   // elements per CTA

struct LimiterArgs {
    double* u;                          // [e][j][i][v]
    int E;
    double gamma;
    int npairs;
    int reps;                           // applications of the whole pair sequence
    double threshold[LIMITER_MAX_PAIRS];
    int variable[LIMITER_MAX_PAIRS];    // 0 density, 1 pressure, 2 density_pressure
    const int* mortar_faces;            // [e]: bits 0-2 count, then 2 bits per mortar (the large face, 0..3), or
                                        // with p4est 3 bits (the large face, whether its index runs backwards)
    int p4est;                          // curvilinear mortars: limit_mortars! of the P4estMesh
                                        // in mortar order; null without mortars
    unsigned long long* cfl_slots;      // or null
    unsigned* status;
};

__device__ __forceinline__ double limiter_value(double gamma, int variable, const double* x) {
    if (variable == 0) return x[0];
    if (variable == 1) return (gamma - 1.0) * (x[3] - 0.5 * (x[1] * x[1] + x[2] * x[2]) / x[0]);
    return (gamma - 1.0) * (x[3] * x[0] - 0.5 * (x[1] * x[1] + x[2] * x[2]));
}

template <int N>
static __global__ void __launch_bounds__(32 * LIMITER_WARPS) positivity_limiter_kernel(LimiterArgs a) {
    constexpr int n = N + 1;
    constexpr int nn = n * n;
    constexpr int S = (nn + 31) / 32;   // nodes per lane
    const int lane = threadIdx.x & 31;
    const int e = blockIdx.x * LIMITER_WARPS + (threadIdx.x >> 5);
    if (e >= a.E) return;   // whole warps leave together
    double* ue = a.u + (size_t)e * nn * NV;
    double x[S][NV];
    double wij[S];
    bool has[S];
#pragma unroll
    for (int s = 0; s < S; ++s) {
        const int k = lane + 32 * s;
        has[s] = k < nn;
        if (has[s]) {
            load4(ue + (size_t)k * NV, x[s]);
            wij[s] = c_tlw_w[N][k % n] * c_tlw_w[N][k / n];
        } else {
            wij[s] = 0.0;
#pragma unroll
            for (int v = 0; v < NV; ++v) x[s][v] = 0.0;
        }
    }
    const int desc = a.mortar_faces ? __ldg(a.mortar_faces + e) : 0;
    const int nmort = desc & 7;
    bool dirty = false;

    auto mean_of = [&](double* m) {
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            double p = 0.0;
#pragma unroll
            for (int s = 0; s < S; ++s) p = fma(x[s][v], wij[s], p);
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) p += __shfl_xor_sync(0xffffffffu, p, o);
            m[v] = p * 0.25;
        }
    };
    auto blend = [&](double theta, const double* m) {
        const double r = 1.0 - theta;
#pragma unroll
        for (int s = 0; s < S; ++s)
#pragma unroll
            for (int v = 0; v < NV; ++v) x[s][v] = fma(theta, x[s][v], r * m[v]);
        dirty = true;
    };
    auto warp_min = [&](double m) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) m = julia_min(m, __shfl_xor_sync(0xffffffffu, m, o));
        return m;
    };

    for (int rep = 0; rep < a.reps; ++rep) {
#pragma unroll
        for (int p = 0; p < LIMITER_MAX_PAIRS; ++p) {   // unrolled: the pair parameters stay in registers
            if (p >= a.npairs) break;
            const double thr = a.threshold[p];
            const int var = a.variable[p];
            // element pass (positivity_zhang_shu_dg2d.jl:8-45)
            double vmin = __longlong_as_double(0x7ff0000000000000ll);
#pragma unroll
            for (int s = 0; s < S; ++s)
                if (has[s]) vmin = julia_min(vmin, limiter_value(a.gamma, var, x[s]));
            vmin = warp_min(vmin);
            if (vmin < thr) {
                double m[NV];
                mean_of(m);
                const double vmean = limiter_value(a.gamma, var, m);
                blend((vmean - thr) / (vmean - vmin), m);
            }
            // mortar pass (limit_mortars!, :47-176 and, P4estMesh, :178-260), this element's mortars as the large
            // element, in order; the P4estMesh pass takes the large face in the mortar's order and the first four
            // nodes of each half only (its loop `for i = 1:4`)
            for (int q = 0; q < nmort; ++q) {
                const int face = (desc >> (3 + (a.p4est ? 3 : 2) * q)) & 3;
                const bool rev = a.p4est && ((desc >> (3 + 3 * q + 2)) & 1);
                double m[NV];
                mean_of(m);
                const double vmean = limiter_value(a.gamma, var, m);
                // lanes 0..n-1: upper half node l; lanes n..2n-1: lower half node l - n
                const int half = lane < n ? 0 : 1;
                const int l = lane - half * n;
                const bool take = lane < 2 * n && (!a.p4est || l < 4);
                const double* fwd = c_tlw_mortar[N][half];   // 0 forward_upper, 1 forward_lower
                double y[NV] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
                for (int f = 0; f < n; ++f) {
                    const int fi = rev ? n - 1 - f : f;
                    const int k = face == 0 ? n * fi : face == 1 ? (n - 1) + n * fi : face == 2 ? fi : fi + n * (n - 1);
                    const int src = k & 31, slot = k >> 5;   // warp-uniform
                    const double c = take ? fwd[(l < n ? l : 0) * n + f] : 0.0;
#pragma unroll
                    for (int v = 0; v < NV; ++v) {
                        double t = x[0][v];
#pragma unroll
                        for (int s = 1; s < S; ++s)
                            if (slot == s) t = x[s][v];
                        y[v] = fma(c, __shfl_sync(0xffffffffu, t, src), y[v]);
                    }
                }
                double mv = __longlong_as_double(0x7ff0000000000000ll);
                if (take) mv = limiter_value(a.gamma, var, y);
                mv = warp_min(mv);
                const double theta = julia_min(fabs((vmean - thr) / (vmean - mv)), 1.0);
                blend(theta, m);
            }
        }
    }
    if (!dirty) return;
#pragma unroll
    for (int s = 0; s < S; ++s)
        if (has[s]) store4(ue + (size_t)(lane + 32 * s) * NV, x[s]);
    if (a.cfl_slots) {
        double m1 = 0.0, m2 = 0.0;
#pragma unroll
        for (int s = 0; s < S; ++s)
            if (has[s]) {
                double l1, l2;
                node_speeds(a.gamma, x[s], a.status, l1, l2);
                m1 = fmax(m1, l1);
                m2 = fmax(m2, l2);
            }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            m1 = fmax(m1, __shfl_xor_sync(0xffffffffu, m1, o));
            m2 = fmax(m2, __shfl_xor_sync(0xffffffffu, m2, o));
        }
        if (lane < CFL_SLOTS) {
            const double m = lane == 0 ? m1 : lane == 1 ? m2 : 0.0;
            a.cfl_slots[(size_t)e * CFL_SLOTS + lane] = (unsigned long long)__double_as_longlong(m);
        }
    }
}

}  // namespace tlw
