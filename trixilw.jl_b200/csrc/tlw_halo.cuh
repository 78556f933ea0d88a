// tlw_halo.cuh -- the faces a rank's part of a partitioned TreeMesh{2} shares with another rank's part (the
// reference's MPI interfaces, src/solvers/dgsem_tree/dg_2d_parallel.jl:23-200, whose message per cut face node is
// the u, U and F.n traces: 3 nv values, src/solvers/dgsem_tree/dg_parallel.jl:12-13).
//
// halo_pack_kernel: after the volume kernel, each cut face node's local u face value, U trace and normal flux
// trace go to the send buffer [halo][l][values] in the caller's order; the caller moves it to the neighbour's
// receive buffer (NCCL, or a device copy). With shock capturing a node also carries the element's first-order
// subcell flux next to the face (fn_low, nv values) and its smoothed blending factor: 3 nv + nv + 1 values in a
// 5 nv record (20 doubles, so that records stay 16-byte aligned).
// halo_face_kernel: the LW surface flux of a cut face node in the TreeMesh argument order, with the local side
// left on a +face and right on a -face, exactly as the interface kernel evaluates it for an interior
// interface (blended with compute_alp from both sides' alpha and fn_low under shock capturing); only the local
// node is updated (the neighbour computes the same flux for its own node).
// x-faces and y-faces run as separate launches (corner nodes), after the interfaces of their orientation.
// halo_alpha_pack_kernel / halo_alpha_smooth_kernel: the raw blending factor of each cut face's element goes to
// the neighbour before the smoothing, which then takes max(alpha, alpha_raw_remote / 2) across the cut faces as
// the interfaces do inside a part (Trixi apply_smoothing!), so the decomposed run blends as the whole mesh does.
// (The reference's own MPI interface flux, calc_mpi_interface_flux!, dg_2d_parallel.jl:370-420, is the plain LW
// flux; blending the cut faces keeps the decomposed solution equal to the undecomposed one.)
#pragma once
#include "tlw_device.cuh"
#include "tlw_surface.cuh"

namespace tlw {

constexpr int HALO_VALUES = 3 * NV;            // u, U, F.n
constexpr int HALO_VALUES_SC = 5 * NV;          // and fn_low, alpha (shock capturing; 3 doubles of padding)
// node records are read and written as 16-byte vectors (load4 / store4): every record starts 16-byte aligned
static_assert(HALO_VALUES * sizeof(double) % 16 == 0 && HALO_VALUES_SC * sizeof(double) % 16 == 0,
              "halo node records must keep 16-byte alignment");

struct HaloArgs {
    const double* u;          // state the jump is taken of
    double* out;              // du (rhs) or the updated state (step)
    const double* tU;         // [v, l, face, e]
    const double* tF;
    double* send;             // [halo][l][12]
    const double* recv;
    const int* elem;          // halo faces of this launch (0-based local elements)
    const int* face;          // 0..3
    const int* slot;          // their position in the caller's order (buffer index)
    int count;
    int orientation;
    const double* inv_jac;
    const double* dt;
    int step_mode;
    double gamma;
    int flux_kind, speed_kind;
    double inv_w_first, inv_w_last;
    unsigned* status;
    int values;               // doubles per node in the buffers: HALO_VALUES or HALO_VALUES_SC
    // shock capturing: smoothed alpha [e], fn_low traces [v, l, face, e], the admissibility test's J^{-1}
    // (element 1's: on a conforming TreeMesh every element's) and the GLL end weights
    const double* alpha;      // or null
    const double* tFn;
    double jac_first, w_first, w_last;
};

__device__ __forceinline__ int halo_face_node(int n, int f, int l) {
    return f == 0 ? n * l : f == 1 ? (n - 1) + n * l : f == 2 ? l : l + n * (n - 1);
}

template <int N>
static __global__ void __launch_bounds__(128) halo_pack_kernel(HaloArgs a) {
    constexpr int n = N + 1, nn = n * n;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int k = t / n, l = t - (t / n) * n;
    if (k >= a.count) return;
    const int e = __ldg(a.elem + k), f = __ldg(a.face + k);
    const int node = halo_face_node(n, f, l);
    double x[NV], y[NV], z[NV];
    load4(a.u + ((size_t)e * nn + node) * NV, x);
    const size_t tb = (((size_t)e * 4 + f) * n + l) * NV;
    load4(a.tU + tb, y);
    load4(a.tF + tb, z);
    double* s = a.send + ((size_t)__ldg(a.slot + k) * n + l) * a.values;
    store4(s, x);
    store4(s + NV, y);
    store4(s + 2 * NV, z);
    if (a.alpha) {
        load4(a.tFn + tb, x);
        store4(s + 3 * NV, x);
        s[4 * NV] = __ldg(a.alpha + e);
    }
}

template <int N>
static __global__ void __launch_bounds__(128) halo_face_kernel(HaloArgs a) {
    constexpr int n = N + 1, nn = n * n;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int k = t / n, l = t - (t / n) * n;
    if (k >= a.count) return;
    const int e = __ldg(a.elem + k), f = __ldg(a.face + k);
    const int node = halo_face_node(n, f, l);
    double ul[NV], Ul[NV], Fl[NV], ur[NV], Ur[NV], Fr[NV], Fn[NV];
    load4(a.u + ((size_t)e * nn + node) * NV, ul);
    const size_t tb = (((size_t)e * 4 + f) * n + l) * NV;
    load4(a.tU + tb, Ul);
    load4(a.tF + tb, Fl);
    const double* r = a.recv + ((size_t)__ldg(a.slot + k) * n + l) * a.values;
    load4(r, ur);
    load4(r + NV, Ur);
    load4(r + 2 * NV, Fr);
    const bool local_left = f & 1;   // +x / +y face: the local element is the interface's left side
    if (local_left)
        lw_surface_flux(a.gamma, a.flux_kind, a.speed_kind, Fl, Fr, Ul, Ur, ul, ur, a.orientation, Fn, a.status);
    else
        lw_surface_flux(a.gamma, a.flux_kind, a.speed_kind, Fr, Fl, Ur, Ul, ur, ul, a.orientation, Fn, a.status);
    if (a.alpha) {
        // the interface kernel's blend with the remote side's alpha and fn_low (compute_alp, dg_2d.jl:1879-1901)
        double fl[NV], fr[NV];
        load4(a.tFn + tb, fl);
        load4(r + 3 * NV, fr);
        const double al = __ldg(a.alpha + e), ar = r[4 * NV];
        if (local_left)
            blend_flux_values(a.gamma, a.speed_kind, a.status, a.jac_first, a.w_first, a.w_last, a.orientation, ul,
                              ur, al, ar, fl, fr, *a.dt, Fn);
        else
            blend_flux_values(a.gamma, a.speed_kind, a.status, a.jac_first, a.w_first, a.w_last, a.orientation, ur,
                              ul, ar, al, fr, fl, *a.dt, Fn);
    }
    const double dts = a.step_mode ? *a.dt : 1.0;
    const double ij = __ldg(a.inv_jac + e);
    // the interface kernel's coefficients, in its order of operations
    const double c = local_left ? -ij * a.inv_w_last * dts : ij * a.inv_w_first * dts;
    double* o = a.out + ((size_t)e * nn + node) * NV;
    double x[NV];
    load4_rw(o, x);
#pragma unroll
    for (int v = 0; v < NV; ++v) x[v] = fma(c, Fn[v], x[v]);
    store4(o, x);
}

// the raw blending factor of each cut face's element into the alpha send buffer [halo] (caller's order)
static __global__ void halo_alpha_pack_kernel(const int* __restrict__ elem, const int* __restrict__ slot, int count,
                                              const double* __restrict__ alpha_raw, double* __restrict__ send) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < count) send[__ldg(slot + k)] = __ldg(alpha_raw + __ldg(elem + k));
}

// alpha_e = max(alpha_e, alpha_raw_remote / 2) across the cut faces (the smoothing of alpha_smooth_kernel)
static __global__ void halo_alpha_smooth_kernel(const int* __restrict__ elem, const int* __restrict__ slot, int count,
                                                const double* __restrict__ recv, double* alpha) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= count) return;
    unsigned long long* ab = reinterpret_cast<unsigned long long*>(alpha);
    atomicMax(ab + __ldg(elem + k), (unsigned long long)__double_as_longlong(0.5 * __ldg(recv + __ldg(slot + k))));
}

}  // namespace tlw
