// tlw_noalloc.cu -- tlw_rhs_lw_noalloc: the LW right-hand side on a periodic TreeMesh{2} for callers that
// must not allocate device memory.
//
// Who needs it: callers that run under a device-memory pool that owns all GPU memory (for example a
// Julia process whose CUDA.jl pool accounts for every byte, or a host application with a fixed memory
// budget), where a foreign cudaMalloc would bypass that accounting or fail, and callers that cannot
// accept the device-wide synchronisation cudaMalloc/cudaFree imply. The handle-based entry points
// (tlw_create + tlw_set_tree_mesh) allocate their own buffers, so these callers use this one instead.
//
// What it does differently: the face traces of U and F.n that the volume kernel hands to the interface
// kernels (the only scratch of the LW rhs) live in a file-scope static __device__ array of
// TLW_NOALLOC_SCRATCH_BYTES; the basis, dt and the status word live in static __device__ variables
// too. Nothing is allocated: no cudaMalloc, cudaFree or allocating library call.
//
// Consequences a caller must respect:
//  * size limit: n_elements * 2 * 4 * (N+1) * 4 * 8 bytes must fit the scratch array (32 MiB: 26214
//    elements at N=4); larger meshes are rejected with TLW_E_ARG;
//  * every GPU that loads the library holds the array until the process exits;
//  * all calls on a device share the array and the dt and status words, which keep the last call's
//    contents: calls that overlap on the GPU (different streams or host threads at once) race and must be
//    serialised by the caller;
//  * each call waits for its stream before it returns;
//  * the first call on each device sets up that device (symbol addresses, basis, kernel attributes)
//    with the device current.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <vector>

#include "../../include/tlw.h"
#include "tlw_basis.h"
#include "tlw_surface.cuh"
#include "tlw_volume.cuh"

using namespace tlw;

namespace {

constexpr size_t kScratchBytes = TLW_NOALLOC_SCRATCH_BYTES;
constexpr int kMaxDevices = 64;

// file-scope device storage: the scratch (face traces), per-degree bases, dt and the status word
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];
static __device__ __align__(256) tlw::Basis g_noalloc_basis[8];
static __device__ double g_noalloc_dt;
static __device__ unsigned g_noalloc_status;

struct DeviceSetup {
    bool done = false;
    double* scratch = nullptr;      // device address of g_noalloc_scratch
    tlw::Basis* basis = nullptr;    // device address of g_noalloc_basis
    double* dt = nullptr;
    unsigned* status = nullptr;
};
DeviceSetup g_setup[kMaxDevices];
std::mutex g_setup_mutex;

template <int N>
void set_attributes() {
    using C = VolCfg<N>;
    cudaFuncSetAttribute(lw_volume_kernel<N, MODE_RHS, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::smem_bytes(4));
}

// once per device, with that device current: symbol addresses (checked), bases, kernel attributes
int setup_device(int dev) {
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    DeviceSetup& s = g_setup[dev];
    if (s.done) return TLW_OK;
    if (cudaGetSymbolAddress((void**)&s.scratch, g_noalloc_scratch) != cudaSuccess) return TLW_E_CUDA;
    if (cudaGetSymbolAddress((void**)&s.basis, g_noalloc_basis) != cudaSuccess) return TLW_E_CUDA;
    if (cudaGetSymbolAddress((void**)&s.dt, g_noalloc_dt) != cudaSuccess) return TLW_E_CUDA;
    if (cudaGetSymbolAddress((void**)&s.status, g_noalloc_status) != cudaSuccess) return TLW_E_CUDA;
    tlw::Basis hb[8];
    for (int N = 1; N <= 7; ++N) host_build_basis(N, hb[N]);
    std::memset(&hb[0], 0, sizeof(hb[0]));
    if (cudaMemcpyToSymbol(g_noalloc_basis, hb, sizeof(hb)) != cudaSuccess) return TLW_E_CUDA;
    if (upload_const_basis(hb) != cudaSuccess) return TLW_E_CUDA;   // this file's constant-memory matrices
    set_attributes<1>(); set_attributes<2>(); set_attributes<3>(); set_attributes<4>();
    set_attributes<5>(); set_attributes<6>(); set_attributes<7>();
    if (cudaGetLastError() != cudaSuccess) return TLW_E_CUDA;
    s.done = true;
    return TLW_OK;
}

template <int N>
void launch(cudaStream_t st, const VolArgs& va, SurfArgs sa, int nx, const int* xl, const int* xr, int ny,
            const int* yl, const int* yr) {
    using C = VolCfg<N>;
    const int grid = (int)((va.E + C::EB - 1) / C::EB);
    lw_volume_kernel<N, MODE_RHS, false><<<grid, C::THREADS, C::smem_bytes(4), st>>>(va);
    sa.left = xl; sa.right = xr; sa.count = nx; sa.orientation = 1;
    if (nx > 0) interface_kernel<N><<<(unsigned)(((long long)nx * (N + 1) + 127) / 128), 128, 0, st>>>(sa);
    sa.left = yl; sa.right = yr; sa.count = ny; sa.orientation = 2;
    if (ny > 0) interface_kernel<N><<<(unsigned)(((long long)ny * (N + 1) + 127) / 128), 128, 0, st>>>(sa);
}

}  // namespace

extern "C" int tlw_rhs_lw_noalloc(int32_t polydeg, double gamma, int32_t surface_flux, int32_t max_speed,
                                  int64_t n_elements, const double* inverse_jacobian, int32_t n_x_interfaces,
                                  const int32_t* x_left, const int32_t* x_right, int32_t n_y_interfaces,
                                  const int32_t* y_left, const int32_t* y_right, const double* u, double* du,
                                  double dt, void* stream) {
    if (polydeg < 1 || polydeg > 7 || !(gamma > 1.0)) return TLW_E_ARG;
    if (surface_flux != TLW_FLUX_RUSANOV && surface_flux != TLW_FLUX_HLL) return TLW_E_ARG;
    if (max_speed != TLW_SPEED_NAIVE && max_speed != TLW_SPEED_DAVIS) return TLW_E_ARG;
    if (n_elements <= 0 || !inverse_jacobian || !u || !du) return TLW_E_ARG;
    if (n_x_interfaces < 0 || n_y_interfaces < 0) return TLW_E_ARG;
    if ((n_x_interfaces > 0 && (!x_left || !x_right)) || (n_y_interfaces > 0 && (!y_left || !y_right))) return TLW_E_ARG;
    const int n = polydeg + 1;
    const size_t trace_doubles = (size_t)NV * n * 4 * (size_t)n_elements;
    if (2 * trace_doubles * sizeof(double) > kScratchBytes) return TLW_E_ARG;   // mesh too large for the scratch
    if (((uintptr_t)u | (uintptr_t)du) % 32 != 0) return TLW_E_ARG;             // 32-byte node records
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return TLW_E_CUDA;
    int rc = setup_device(dev);
    if (rc != TLW_OK) return rc;
    const DeviceSetup& s = g_setup[dev];
    cudaStream_t st = (cudaStream_t)stream;
    // the status word keeps the previous call's value: clear it; dt goes to its device variable
    if (cudaMemsetAsync(s.status, 0, sizeof(unsigned), st) != cudaSuccess) return TLW_E_CUDA;
    if (cudaMemcpyAsync(s.dt, &dt, sizeof(double), cudaMemcpyHostToDevice, st) != cudaSuccess) return TLW_E_CUDA;
    VolArgs va{};
    va.u = u;
    va.u_base = u;
    va.out = du;
    va.tU = s.scratch;
    va.tF = s.scratch + trace_doubles;
    va.inv_jac = inverse_jacobian;
    va.dt = s.dt;
    va.basis = s.basis + polydeg;
    va.E = (int)n_elements;
    va.gamma = gamma;
    SurfArgs sa{};
    sa.u = u;
    sa.out = du;
    sa.tU = va.tU;
    sa.tF = va.tF;
    sa.inv_jac = inverse_jacobian;
    sa.dt = s.dt;
    sa.step_mode = 0;
    sa.gamma = gamma;
    sa.flux_kind = surface_flux;
    sa.speed_kind = max_speed;
    tlw::Basis hb;
    host_build_basis(polydeg, hb);
    sa.inv_w_first = hb.inv_w_first;
    sa.inv_w_last = hb.inv_w_last;
    sa.status = s.status;
    switch (polydeg) {
        case 1: launch<1>(st, va, sa, n_x_interfaces, x_left, x_right, n_y_interfaces, y_left, y_right); break;
        case 2: launch<2>(st, va, sa, n_x_interfaces, x_left, x_right, n_y_interfaces, y_left, y_right); break;
        case 3: launch<3>(st, va, sa, n_x_interfaces, x_left, x_right, n_y_interfaces, y_left, y_right); break;
        case 4: launch<4>(st, va, sa, n_x_interfaces, x_left, x_right, n_y_interfaces, y_left, y_right); break;
        case 5: launch<5>(st, va, sa, n_x_interfaces, x_left, x_right, n_y_interfaces, y_left, y_right); break;
        case 6: launch<6>(st, va, sa, n_x_interfaces, x_left, x_right, n_y_interfaces, y_left, y_right); break;
        default: launch<7>(st, va, sa, n_x_interfaces, x_left, x_right, n_y_interfaces, y_left, y_right); break;
    }
    if (cudaGetLastError() != cudaSuccess) return TLW_E_CUDA;
    unsigned status = 0;
    if (cudaMemcpyAsync(&status, s.status, sizeof(unsigned), cudaMemcpyDeviceToHost, st) != cudaSuccess) return TLW_E_CUDA;
    if (cudaStreamSynchronize(st) != cudaSuccess) return TLW_E_CUDA;
    return status ? TLW_E_NONADMISSIBLE : TLW_OK;
}
