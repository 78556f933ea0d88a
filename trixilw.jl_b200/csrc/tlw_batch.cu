// tlw_batch.cu -- the batched form: many independent TreeMesh{2} LW simulations of uneven size and degree
// advanced together on one GPU.
//
// Instances are grouped by polynomial degree. Inside a group the elements of all its instances are
// concatenated (one state array, one trace array, one interface list with element ids shifted by the
// instance's offset), and every element carries its instance id: the volume and interface kernels read
// the dt of that instance, the CFL pass reduces into per-instance maxima, and one small kernel turns those
// into per-instance dt / t (each instance keeps its own CFL number and final time, exactly as if it ran
// alone). A whole step of all groups - CFL pass, dt, volume, x and y interfaces - is captured once as a
// CUDA graph and replayed, so a step of 512 instances costs a handful of launches instead of thousands.
// The autotuner times, on the actual batch, the elements-per-CTA variant of the volume kernel per degree, the
// element-centric surface pass against the x / y interface sweeps at two CTA sizes (all give the same bits),
// and whether the degree groups run one after another or concurrently on separate streams (graph branches),
// and keeps the fastest.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "../../include/tlw.h"
#include "tlw_basis.h"
#include "tlw_surface.cuh"
#include "tlw_volume.cuh"

using namespace tlw;

namespace {

struct HostInstance {
    int N = 0;
    int64_t E = 0;
    std::vector<double> inv_jac;
    std::vector<int> left, right, orient;   // 0-based, within the instance
};

struct Group {
    int N = 0, n = 0, nn = 0;
    int64_t E = 0;
    std::vector<int> instances;             // global instance ids
    double* d_state[2] = {nullptr, nullptr};
    double *d_tU = nullptr, *d_tF = nullptr, *d_inv_jac = nullptr;
    int* d_inst = nullptr;
    int *d_xl = nullptr, *d_xr = nullptr, *d_yl = nullptr, *d_yr = nullptr;
    int nx = 0, ny = 0;
    int eb_variant = 0;                     // 0: default elements per CTA, 1: the alternative
    int ifc_block = 0;                      // 0: the element-centric surface pass, else the sweeps' CTA size
    int* d_nbr = nullptr;                   // the element across each face (every face an interface)
    Basis basis{};
};

template <class T>
void dfree(T*& p) {
    if (p) cudaFree(p);
    p = nullptr;
}

}  // namespace

struct tlw_batch {
    tlw_opts opts{};
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t side[8] = {};
    std::string err;
    std::vector<HostInstance> host;
    std::vector<int64_t> offset;            // element offset of each instance inside its group
    std::vector<int> group_of;
    std::vector<Group> groups;
    bool finalized = false;
    int concurrent = 0;                     // run degree groups on separate streams
    int cur = 0;
    // per-instance device scalars
    unsigned long long* d_max = nullptr;
    double *d_dt = nullptr, *d_t = nullptr, *d_t_end = nullptr, *d_cfl = nullptr;
    long long* d_steps = nullptr;
    int* d_nnodes = nullptr;
    StepState* d_step = nullptr;            // status word
    cudaGraphExec_t graph[2] = {nullptr, nullptr};
};

namespace {

int bfail(tlw_batch* b, int code, const std::string& msg) {
    if (b) b->err = msg;
    return code;
}

#define TLW_BCUDA(b, call)                                                                       \
    do {                                                                                         \
        cudaError_t e_ = (call);                                                                 \
        if (e_ != cudaSuccess)                                                                   \
            return bfail(b, TLW_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));     \
    } while (0)

// alternative elements-per-CTA choices the autotuner compares with the defaults (N = 3: 8, 4: 5, 5: 3)
template <int N> struct AltEB;
template <> struct AltEB<3> { static constexpr int v = 16; };
template <> struct AltEB<4> { static constexpr int v = 10; };
template <> struct AltEB<5> { static constexpr int v = 7; };

template <int N>
struct BLaunch {
    static void set_attributes() {
        cudaFuncSetAttribute(lw_volume_kernel<N, MODE_STEP, false, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)VolCfg<N, 0>::smem_bytes(4));
        cudaFuncSetAttribute(lw_volume_kernel<N, MODE_STEP, false, AltEB<N>::v>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)VolCfg<N, AltEB<N>::v>::smem_bytes(4));
    }
    static void volume(cudaStream_t s, int variant, const VolArgs& a) {
        if (variant == 0) {
            using C = VolCfg<N, 0>;
            lw_volume_kernel<N, MODE_STEP, false, 0>
                <<<(unsigned)((a.E + C::EB - 1) / C::EB), C::THREADS, C::smem_bytes(4), s>>>(a);
        } else {
            using C = VolCfg<N, AltEB<N>::v>;
            lw_volume_kernel<N, MODE_STEP, false, AltEB<N>::v>
                <<<(unsigned)((a.E + C::EB - 1) / C::EB), C::THREADS, C::smem_bytes(4), s>>>(a);
        }
    }
    static void surfaces(cudaStream_t s, const SurfArgs& a) {
        using C = SurfCfg<N>;
        surface_kernel<N, false, false><<<(unsigned)((a.E + C::EB - 1) / C::EB), C::THREADS, 0, s>>>(a, BndArgs{});
    }
    static void interfaces(cudaStream_t s, int block, const SurfArgs& a) {
        const long long threads = (long long)a.count * (N + 1);
        if (threads == 0) return;
        interface_kernel<N><<<(unsigned)((threads + block - 1) / block), block, 0, s>>>(a);
    }
    static void speed(cudaStream_t s, const double* u, const double* ij, int E, double gamma, StepState* st,
                      BatchSpeedArgs bs) {
        if (E == 0) return;
        const int grid = (E + MsCfg<N>::ELEMS - 1) / MsCfg<N>::ELEMS;
        max_speed_kernel<N, true, false><<<grid, MS_THREADS, 0, s>>>(u, ij, E, gamma, st, IndicatorArgs{}, bs);
    }
};

template <class F>
bool with_degree(int N, F&& f) {
    switch (N) {
        case 3: f(std::integral_constant<int, 3>{}); return true;
        case 4: f(std::integral_constant<int, 4>{}); return true;
        case 5: f(std::integral_constant<int, 5>{}); return true;
        default: return false;
    }
}

VolArgs vol_args(tlw_batch* b, Group& g, int from) {
    VolArgs va{};
    va.u = g.d_state[from];
    va.u_base = g.d_state[from];
    va.out = g.d_state[1 - from];
    va.tU = g.d_tU;
    va.tF = g.d_tF;
    va.inv_jac = g.d_inv_jac;
    va.dt = b->d_dt;
    va.E = (int)g.E;
    va.gamma = b->opts.gamma;
    va.status = &b->d_step->status;
    va.speed_kind = b->opts.max_speed;
    va.inst = g.d_inst;
    return va;
}

SurfArgs surf_args(tlw_batch* b, Group& g, int from) {
    SurfArgs sa{};
    sa.u = g.d_state[from];
    sa.out = g.d_state[1 - from];
    sa.tU = g.d_tU;
    sa.tF = g.d_tF;
    sa.inv_jac = g.d_inv_jac;
    sa.dt = b->d_dt;
    sa.step_mode = 1;
    sa.gamma = b->opts.gamma;
    sa.flux_kind = b->opts.surface_flux;
    sa.speed_kind = b->opts.max_speed;
    sa.inv_w_first = g.basis.inv_w_first;
    sa.inv_w_last = g.basis.inv_w_last;
    sa.status = &b->d_step->status;
    sa.inst = g.d_inst;
    return sa;
}

// rhs + update of one group on stream s (dt of every instance already final)
void enqueue_group_update(tlw_batch* b, Group& g, int from, cudaStream_t s) {
    const VolArgs va = vol_args(b, g, from);
    SurfArgs sa = surf_args(b, g, from);
    with_degree(g.N, [&](auto Nc) {
        constexpr int N = decltype(Nc)::value;
        BLaunch<N>::volume(s, g.eb_variant, va);
        if (g.ifc_block == 0 && g.d_nbr) {
            sa.nbr = g.d_nbr;
            sa.E = (int)g.E;
            BLaunch<N>::surfaces(s, sa);
            return;
        }
        sa.left = g.d_xl; sa.right = g.d_xr; sa.count = g.nx; sa.orientation = 1;
        BLaunch<N>::interfaces(s, g.ifc_block, sa);
        sa.left = g.d_yl; sa.right = g.d_yr; sa.count = g.ny; sa.orientation = 2;
        BLaunch<N>::interfaces(s, g.ifc_block, sa);
    });
}

void enqueue_batch_step(tlw_batch* b, int from) {
    BatchSpeedArgs bs{};
    bs.inst_max = b->d_max;
    for (Group& g : b->groups) {
        bs.inst = g.d_inst;
        with_degree(g.N, [&](auto Nc) {
            constexpr int N = decltype(Nc)::value;
            BLaunch<N>::speed(b->stream, g.d_state[from], g.d_inv_jac, (int)g.E, b->opts.gamma, b->d_step, bs);
        });
    }
    BatchTime bt{b->d_max, b->d_dt, b->d_t, b->d_t_end, b->d_cfl, b->d_steps, b->d_nnodes, (int)b->host.size()};
    batch_finalize_dt_kernel<<<(bt.count + 127) / 128, 128, 0, b->stream>>>(bt);
    if (!b->concurrent || b->groups.size() < 2) {
        for (Group& g : b->groups) enqueue_group_update(b, g, from, b->stream);
        return;
    }
    // fork: one branch per degree group, joined back on the main stream
    cudaEvent_t fork, join[8];
    cudaEventCreateWithFlags(&fork, cudaEventDisableTiming);
    cudaEventRecord(fork, b->stream);
    for (size_t k = 0; k < b->groups.size(); ++k) {
        cudaStreamWaitEvent(b->side[k], fork, 0);
        enqueue_group_update(b, b->groups[k], from, b->side[k]);
        cudaEventCreateWithFlags(&join[k], cudaEventDisableTiming);
        cudaEventRecord(join[k], b->side[k]);
        cudaStreamWaitEvent(b->stream, join[k], 0);
    }
    cudaEventDestroy(fork);
    for (size_t k = 0; k < b->groups.size(); ++k) cudaEventDestroy(join[k]);
}

void drop_batch_graphs(tlw_batch* b) {
    for (auto& g : b->graph)
        if (g) { cudaGraphExecDestroy(g); g = nullptr; }
}

int capture_batch(tlw_batch* b, int from, cudaGraphExec_t& exec) {
    if (exec) return TLW_OK;
    cudaGraph_t gr = nullptr;
    TLW_BCUDA(b, cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    enqueue_batch_step(b, from);
    const cudaError_t e1 = cudaStreamEndCapture(b->stream, &gr);
    if (e1 != cudaSuccess) return bfail(b, TLW_E_CUDA, std::string("batch graph capture: ") + cudaGetErrorString(e1));
    const cudaError_t e2 = cudaGraphInstantiate(&exec, gr, 0);
    cudaGraphDestroy(gr);
    if (e2 != cudaSuccess) {
        exec = nullptr;
        return bfail(b, TLW_E_CUDA, std::string("batch graph instantiate: ") + cudaGetErrorString(e2));
    }
    return TLW_OK;
}

int read_batch_status(tlw_batch* b) {
    unsigned st = 0;
    TLW_BCUDA(b, cudaMemcpyAsync(&st, &b->d_step->status, sizeof(st), cudaMemcpyDeviceToHost, b->stream));
    TLW_BCUDA(b, cudaStreamSynchronize(b->stream));
    if (st) {
        const unsigned zero = 0;
        TLW_BCUDA(b, upload_on(b->stream, &b->d_step->status, &zero, sizeof(zero)));
        return bfail(b, TLW_E_NONADMISSIBLE, "non-admissible state: square root of a negative number (DomainError)");
    }
    return TLW_OK;
}

}  // namespace

extern "C" {

int tlw_batch_create(const tlw_opts* opts, tlw_batch** out) {
    if (!opts || !out) return TLW_E_ARG;
    *out = nullptr;
    if (opts->time_discretization != TLW_LW || opts->volume_integral != TLW_VOLUME_FR) return TLW_E_UNSUPPORTED;
    if (opts->surface_flux != TLW_FLUX_RUSANOV && opts->surface_flux != TLW_FLUX_HLL) return TLW_E_ARG;
    if (opts->max_speed != TLW_SPEED_NAIVE && opts->max_speed != TLW_SPEED_DAVIS) return TLW_E_ARG;
    if (!(opts->gamma > 1.0)) return TLW_E_ARG;
    tlw_batch* b = new (std::nothrow) tlw_batch();
    if (!b) return TLW_E_ARG;
    b->opts = *opts;
    b->device = opts->device;
    if (cudaSetDevice(b->device) != cudaSuccess || cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete b;
        return TLW_E_CUDA;
    }
    for (auto& s : b->side) cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
    Basis all[8];
    std::memset(&all[0], 0, sizeof(all[0]));
    for (int N = 1; N <= 7; ++N) host_build_basis(N, all[N]);
    if (upload_const_basis(all) != cudaSuccess || cudaMalloc(&b->d_step, sizeof(StepState)) != cudaSuccess ||
        zero_on(b->stream, b->d_step, sizeof(StepState)) != cudaSuccess) {
        tlw_batch_destroy(b);
        return TLW_E_CUDA;
    }
    BLaunch<3>::set_attributes();
    BLaunch<4>::set_attributes();
    BLaunch<5>::set_attributes();
    *out = b;
    return TLW_OK;
}

int tlw_batch_destroy(tlw_batch* b) {
    if (!b) return TLW_OK;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    drop_batch_graphs(b);
    for (Group& g : b->groups) {
        dfree(g.d_state[0]); dfree(g.d_state[1]); dfree(g.d_tU); dfree(g.d_tF); dfree(g.d_inv_jac);
        dfree(g.d_inst); dfree(g.d_xl); dfree(g.d_xr); dfree(g.d_yl); dfree(g.d_yr); dfree(g.d_nbr);
    }
    dfree(b->d_max); dfree(b->d_dt); dfree(b->d_t); dfree(b->d_t_end); dfree(b->d_cfl); dfree(b->d_steps);
    dfree(b->d_nnodes); dfree(b->d_step);
    for (auto& s : b->side) if (s) cudaStreamDestroy(s);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
    return TLW_OK;
}

int tlw_batch_add_tree_mesh(tlw_batch* b, int32_t polydeg, int64_t n_elements, const double* inverse_jacobian,
                            int64_t n_interfaces, const int64_t* interface_neighbor_ids,
                            const int64_t* interface_orientations, int32_t* index_out) {
    if (!b) return TLW_E_ARG;
    if (b->finalized) return bfail(b, TLW_E_STATE, "batch already finalized");
    if (polydeg < 3 || polydeg > 5) return bfail(b, TLW_E_UNSUPPORTED, "batched form is built for N = 3, 4, 5");
    if (n_elements <= 0 || !inverse_jacobian || n_interfaces < 0 || (n_interfaces && (!interface_neighbor_ids || !interface_orientations)))
        return bfail(b, TLW_E_ARG, "mesh arrays");
    HostInstance hi;
    hi.N = polydeg;
    hi.E = n_elements;
    hi.inv_jac.assign(inverse_jacobian, inverse_jacobian + n_elements);
    for (int64_t k = 0; k < n_interfaces; ++k) {
        const int64_t l = interface_neighbor_ids[2 * k] - 1, r = interface_neighbor_ids[2 * k + 1] - 1;
        const int64_t o = interface_orientations[k];
        if (l < 0 || l >= n_elements || r < 0 || r >= n_elements || (o != 1 && o != 2))
            return bfail(b, TLW_E_ARG, "interface out of range");
        hi.left.push_back((int)l);
        hi.right.push_back((int)r);
        hi.orient.push_back((int)o);
    }
    b->host.push_back(std::move(hi));
    if (index_out) *index_out = (int32_t)(b->host.size() - 1);
    return TLW_OK;
}

int tlw_batch_finalize(tlw_batch* b) {
    if (!b) return TLW_E_ARG;
    if (b->finalized) return TLW_OK;
    if (b->host.empty()) return bfail(b, TLW_E_STATE, "no instances");
    TLW_BCUDA(b, cudaSetDevice(b->device));
    const int ninst = (int)b->host.size();
    b->offset.assign(ninst, 0);
    b->group_of.assign(ninst, -1);
    for (int N = 3; N <= 5; ++N) {
        Group g;
        g.N = N; g.n = N + 1; g.nn = g.n * g.n;
        host_build_basis(N, g.basis);
        std::vector<double> ij;
        std::vector<int> inst, xl, xr, yl, yr;
        for (int i = 0; i < ninst; ++i) {
            const HostInstance& hi = b->host[i];
            if (hi.N != N) continue;
            b->offset[i] = g.E;
            b->group_of[i] = (int)b->groups.size();
            g.instances.push_back(i);
            ij.insert(ij.end(), hi.inv_jac.begin(), hi.inv_jac.end());
            inst.insert(inst.end(), (size_t)hi.E, i);
            for (size_t k = 0; k < hi.left.size(); ++k) {
                (hi.orient[k] == 1 ? xl : yl).push_back((int)(hi.left[k] + g.E));
                (hi.orient[k] == 1 ? xr : yr).push_back((int)(hi.right[k] + g.E));
            }
            g.E += hi.E;
        }
        if (g.E == 0) continue;
        if (g.E > (int64_t)0x7fffffff / 64) return bfail(b, TLW_E_ARG, "batch group too large");
        auto up_d = [&](double*& d, const std::vector<double>& v) -> int {
            TLW_BCUDA(b, cudaMalloc(&d, v.size() * sizeof(double)));
            TLW_BCUDA(b, upload_on(b->stream, d, v.data(), v.size() * sizeof(double)));
            return TLW_OK;
        };
        auto up_i = [&](int*& d, const std::vector<int>& v) -> int {
            if (v.empty()) return TLW_OK;
            TLW_BCUDA(b, cudaMalloc(&d, v.size() * sizeof(int)));
            TLW_BCUDA(b, upload_on(b->stream, d, v.data(), v.size() * sizeof(int)));
            return TLW_OK;
        };
        int rc;
        if ((rc = up_d(g.d_inv_jac, ij)) || (rc = up_i(g.d_inst, inst)) || (rc = up_i(g.d_xl, xl)) ||
            (rc = up_i(g.d_xr, xr)) || (rc = up_i(g.d_yl, yl)) || (rc = up_i(g.d_yr, yr)))
            return rc;
        g.nx = (int)xl.size();
        g.ny = (int)yl.size();
        if ((int64_t)(xl.size() + yl.size()) == 2 * g.E) {
            // every face an interface: the element-centric surface pass (the element across each face)
            std::vector<int> nbr((size_t)4 * g.E, -1);
            bool ok = true;
            auto put = [&](int e, int f, int other) {
                int& slot = nbr[(size_t)4 * e + f];
                if (slot != -1) ok = false;
                slot = other;
            };
            for (size_t k = 0; k < xl.size(); ++k) { put(xl[k], 1, xr[k]); put(xr[k], 0, xl[k]); }
            for (size_t k = 0; k < yl.size(); ++k) { put(yl[k], 3, yr[k]); put(yr[k], 2, yl[k]); }
            if (ok && (rc = up_i(g.d_nbr, nbr))) return rc;
        }
        if (!g.d_nbr) g.ifc_block = 128;
        const size_t sd = (size_t)NV * g.nn * g.E, td = (size_t)NV * g.n * 4 * g.E;
        TLW_BCUDA(b, cudaMalloc(&g.d_state[0], sd * sizeof(double)));
        TLW_BCUDA(b, cudaMalloc(&g.d_state[1], sd * sizeof(double)));
        TLW_BCUDA(b, cudaMalloc(&g.d_tU, td * sizeof(double)));
        TLW_BCUDA(b, cudaMalloc(&g.d_tF, td * sizeof(double)));
        b->groups.push_back(g);
    }
    TLW_BCUDA(b, cudaMalloc(&b->d_max, ninst * sizeof(unsigned long long)));
    TLW_BCUDA(b, zero_on(b->stream, b->d_max, ninst * sizeof(unsigned long long)));
    TLW_BCUDA(b, cudaMalloc(&b->d_dt, ninst * sizeof(double)));
    TLW_BCUDA(b, zero_on(b->stream, b->d_dt, ninst * sizeof(double)));
    TLW_BCUDA(b, cudaMalloc(&b->d_t, ninst * sizeof(double)));
    TLW_BCUDA(b, zero_on(b->stream, b->d_t, ninst * sizeof(double)));
    TLW_BCUDA(b, cudaMalloc(&b->d_t_end, ninst * sizeof(double)));
    TLW_BCUDA(b, cudaMalloc(&b->d_cfl, ninst * sizeof(double)));
    TLW_BCUDA(b, cudaMalloc(&b->d_steps, ninst * sizeof(long long)));
    TLW_BCUDA(b, zero_on(b->stream, b->d_steps, ninst * sizeof(long long)));
    std::vector<int> nn(ninst);
    std::vector<double> inf(ninst, INFINITY), one(ninst, 0.5);
    for (int i = 0; i < ninst; ++i) nn[i] = b->host[i].N + 1;
    TLW_BCUDA(b, cudaMalloc(&b->d_nnodes, ninst * sizeof(int)));
    TLW_BCUDA(b, upload_on(b->stream, b->d_nnodes, nn.data(), ninst * sizeof(int)));
    TLW_BCUDA(b, upload_on(b->stream, b->d_t_end, inf.data(), ninst * sizeof(double)));
    TLW_BCUDA(b, upload_on(b->stream, b->d_cfl, one.data(), ninst * sizeof(double)));
    b->finalized = true;
    b->cur = 0;
    return TLW_OK;
}

int tlw_batch_set_state(tlw_batch* b, int32_t instance, const double* u, int32_t where, double t, double cfl,
                        double t_end) {
    if (!b || !u) return TLW_E_ARG;
    if (!b->finalized) return bfail(b, TLW_E_STATE, "finalize the batch first");
    if (instance < 0 || instance >= (int)b->host.size()) return bfail(b, TLW_E_ARG, "instance");
    TLW_BCUDA(b, cudaSetDevice(b->device));
    Group& g = b->groups[b->group_of[instance]];
    const size_t off = (size_t)NV * g.nn * b->offset[instance], cnt = (size_t)NV * g.nn * b->host[instance].E;
    const cudaMemcpyKind k = where == TLW_WHERE_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    TLW_BCUDA(b, cudaMemcpyAsync(g.d_state[b->cur] + off, u, cnt * sizeof(double), k, b->stream));
    const long long zero = 0;
    TLW_BCUDA(b, cudaMemcpyAsync(b->d_t + instance, &t, sizeof(double), cudaMemcpyHostToDevice, b->stream));
    TLW_BCUDA(b, cudaMemcpyAsync(b->d_cfl + instance, &cfl, sizeof(double), cudaMemcpyHostToDevice, b->stream));
    TLW_BCUDA(b, cudaMemcpyAsync(b->d_t_end + instance, &t_end, sizeof(double), cudaMemcpyHostToDevice, b->stream));
    TLW_BCUDA(b, cudaMemcpyAsync(b->d_steps + instance, &zero, sizeof(zero), cudaMemcpyHostToDevice, b->stream));
    TLW_BCUDA(b, cudaStreamSynchronize(b->stream));
    return TLW_OK;
}

int tlw_batch_get_state(tlw_batch* b, int32_t instance, double* u, int32_t where, double* t_out, int64_t* steps_out) {
    if (!b || !u) return TLW_E_ARG;
    if (!b->finalized) return bfail(b, TLW_E_STATE, "finalize the batch first");
    if (instance < 0 || instance >= (int)b->host.size()) return bfail(b, TLW_E_ARG, "instance");
    TLW_BCUDA(b, cudaSetDevice(b->device));
    Group& g = b->groups[b->group_of[instance]];
    const size_t off = (size_t)NV * g.nn * b->offset[instance], cnt = (size_t)NV * g.nn * b->host[instance].E;
    const cudaMemcpyKind k = where == TLW_WHERE_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    TLW_BCUDA(b, cudaMemcpyAsync(u, g.d_state[b->cur] + off, cnt * sizeof(double), k, b->stream));
    double t = 0;
    long long st = 0;
    TLW_BCUDA(b, cudaMemcpyAsync(&t, b->d_t + instance, sizeof(double), cudaMemcpyDeviceToHost, b->stream));
    TLW_BCUDA(b, cudaMemcpyAsync(&st, b->d_steps + instance, sizeof(st), cudaMemcpyDeviceToHost, b->stream));
    int rc = read_batch_status(b);
    if (t_out) *t_out = t;
    if (steps_out) *steps_out = st;
    return rc;
}

int tlw_batch_step(tlw_batch* b, int32_t nsteps, int32_t use_graph) {
    if (!b) return TLW_E_ARG;
    if (!b->finalized) return bfail(b, TLW_E_STATE, "finalize the batch first");
    if (nsteps < 0) return bfail(b, TLW_E_ARG, "nsteps");
    TLW_BCUDA(b, cudaSetDevice(b->device));
    if (use_graph) {
        int rc;
        if ((rc = capture_batch(b, 0, b->graph[0])) || (rc = capture_batch(b, 1, b->graph[1]))) return rc;
        for (int s = 0; s < nsteps; ++s) {
            TLW_BCUDA(b, cudaGraphLaunch(b->graph[b->cur], b->stream));
            b->cur ^= 1;
        }
    } else {
        for (int s = 0; s < nsteps; ++s) {
            enqueue_batch_step(b, b->cur);
            b->cur ^= 1;
        }
        TLW_BCUDA(b, cudaGetLastError());
    }
    return TLW_OK;
}

int tlw_batch_synchronize(tlw_batch* b) {
    if (!b) return TLW_E_ARG;
    TLW_BCUDA(b, cudaSetDevice(b->device));
    TLW_BCUDA(b, cudaStreamSynchronize(b->stream));
    TLW_BCUDA(b, cudaGetLastError());
    return read_batch_status(b);
}

int tlw_batch_get_stream(tlw_batch* b, void** stream) {
    if (!b || !stream) return TLW_E_ARG;
    *stream = (void*)b->stream;
    return TLW_OK;
}

int tlw_batch_autotune(tlw_batch* b, int32_t trials, int32_t* choices_out) {
    if (!b) return TLW_E_ARG;
    if (!b->finalized) return bfail(b, TLW_E_STATE, "finalize the batch first");
    if (trials < 1) trials = 3;
    TLW_BCUDA(b, cudaSetDevice(b->device));
    drop_batch_graphs(b);
    cudaEvent_t e0, e1;
    TLW_BCUDA(b, cudaEventCreate(&e0));
    TLW_BCUDA(b, cudaEventCreate(&e1));
    // The timed launches write only into the state buffer that the next step overwrites anyway; the
    // current state, t and dt are untouched.
    auto time_group = [&](Group& g) -> float {
        float best = 1e30f;
        for (int r = 0; r <= trials; ++r) {
            cudaEventRecord(e0, b->stream);
            enqueue_group_update(b, g, b->cur, b->stream);
            cudaEventRecord(e1, b->stream);
            cudaEventSynchronize(e1);
            float ms = 0;
            cudaEventElapsedTime(&ms, e0, e1);
            if (r > 0) best = std::min(best, ms);   // the first launch warms up
        }
        return best;
    };
    int gi = 0;
    for (Group& g : b->groups) {
        float best = 1e30f;
        int bv = 0, bb = g.ifc_block;
        for (int v = 0; v < 2; ++v)
            for (int blk : {0, 128, 256}) {
                if (blk == 0 && !g.d_nbr) continue;
                g.eb_variant = v;
                g.ifc_block = blk;
                const float ms = time_group(g);
                if (ms < best) { best = ms; bv = v; bb = blk; }
            }
        g.eb_variant = bv;
        g.ifc_block = bb;
        if (choices_out) { choices_out[2 * gi] = bv; choices_out[2 * gi + 1] = bb; }
        ++gi;
    }
    // groups one after another or concurrently: time the update phase of a whole step both ways
    if (b->groups.size() >= 2) {
        float best = 1e30f;
        int bc = 0;
        for (int c = 0; c < 2; ++c) {
            b->concurrent = c;
            float cbest = 1e30f;
            for (int r = 0; r <= trials; ++r) {
                cudaEventRecord(e0, b->stream);
                if (!c) {
                    for (Group& g : b->groups) enqueue_group_update(b, g, b->cur, b->stream);
                } else {
                    cudaEvent_t fork, join[8];
                    cudaEventCreateWithFlags(&fork, cudaEventDisableTiming);
                    cudaEventRecord(fork, b->stream);
                    for (size_t k = 0; k < b->groups.size(); ++k) {
                        cudaStreamWaitEvent(b->side[k], fork, 0);
                        enqueue_group_update(b, b->groups[k], b->cur, b->side[k]);
                        cudaEventCreateWithFlags(&join[k], cudaEventDisableTiming);
                        cudaEventRecord(join[k], b->side[k]);
                        cudaStreamWaitEvent(b->stream, join[k], 0);
                    }
                    cudaEventDestroy(fork);
                    for (size_t k = 0; k < b->groups.size(); ++k) cudaEventDestroy(join[k]);
                }
                cudaEventRecord(e1, b->stream);
                cudaEventSynchronize(e1);
                float ms = 0;
                cudaEventElapsedTime(&ms, e0, e1);
                if (r > 0) cbest = std::min(cbest, ms);
            }
            if (cbest < best) { best = cbest; bc = c; }
        }
        b->concurrent = bc;
    }
    if (choices_out) choices_out[2 * b->groups.size()] = b->concurrent;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    TLW_BCUDA(b, cudaGetLastError());
    return read_batch_status(b);
}

int32_t tlw_batch_num_groups(tlw_batch* b) { return b ? (int32_t)b->groups.size() : -1; }

const char* tlw_batch_last_error(tlw_batch* b) { return b ? b->err.c_str() : "null batch"; }

}  // extern "C"
