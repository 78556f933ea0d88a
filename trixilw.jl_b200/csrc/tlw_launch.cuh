// tlw_launch.cuh -- internal: the kernel launches of one polynomial degree, tlw::Launch<N>. The definitions
// live in tlw_launch.cu, which is compiled once per degree; tlw_capi.cu calls them through dispatch over N.
#pragma once
#include <cuda_runtime.h>

#include "tlw_curved.cuh"
#include "tlw_curved_mortar.cuh"
#include "tlw_halo.cuh"
#include "tlw_handle.h"
#include "tlw_limiter.cuh"
#include "tlw_mortar.cuh"
#include "tlw_parabolic.cuh"
#include "tlw_surface.cuh"
#include "tlw_volume.cuh"

namespace tlw {

template <int N>
struct Launch {
    // this degree's copy of the constant-memory matrices (once per device)
    static cudaError_t upload_constants(const Basis* all);
    static void set_attributes();
    static void par_attributes();
    static void volume(cudaStream_t s, int stage, int mode, bool sc, const VolArgs& a);
    static void interfaces(cudaStream_t s, const SurfArgs& a);
    // all faces of a mesh whose every face is a conforming interface or a boundary, one pass over the elements
    static void surfaces(cudaStream_t s, const SurfArgs& a, const BndArgs& b);
    static void boundaries(cudaStream_t s, const BndArgs& a);
    static void parabolic(cudaStream_t s, const tlw_handle* h, int mode, const double* u, double* out,
                          const double* dtp);
    static void par_speed(cudaStream_t s, const tlw_handle* h, const double* u);
    static void mortars(cudaStream_t s, const MortarArgs& a);
    static void curved_mortars(cudaStream_t s, const CurvedMortarArgs& a);
    static void curved_interfaces(cudaStream_t s, const CurvedSurfArgs& a);
    static void curved_boundaries(cudaStream_t s, const CurvedBndArgs& a);
    static void curved_speed(cudaStream_t s, const double* u, const double* Ja, const double* ij, int E, double g,
                             StepState* st);
    static void halo(cudaStream_t s, const HaloArgs& a, bool pack);
    static void limiter(cudaStream_t s, const LimiterArgs& a);
    static void max_speed(cudaStream_t s, const double* u, const double* ij, int E, double gamma, StepState* st,
                          bool speed, bool ind, const IndicatorArgs& ia);
};

}  // namespace tlw
