// tlw_fused.cuh -- the volume and surface passes of an LW step or MDRK stage on a conforming periodic TreeMesh
// in one launch.
//
// The volume pass is FP64-bound and leaves HBM mostly idle; the element-centric surface pass is HBM-bound and
// waits on the volume pass of the element and its four neighbours. lw_fused_kernel runs both in the same CTAs,
// so that the surface work of finished regions streams beside the volume work of the others and reads the
// traces the volume pass has just written while they are still in L2:
//  - every CTA takes a ticket from a counter (atomicAdd), the ticket names its tile of EB elements, and the
//    CTA runs that tile's volume phase (lw_volume_tile), then publishes the tile's flag (release at GPU scope);
//  - the surface of element s reads the volume results of its own tile and its neighbours' tiles; it is
//    assigned to the ticket r(s) = the largest of those tiles, so the CTA holding ticket t computes, after its
//    volume phase, the surfaces of the elements whose last dependency is tile t (groups of surface_group);
//  - before a group it waits (acquire at GPU scope) on the flags of the group's tiles. Every tile waited on has
//    a ticket below t, held by a CTA that is already running and publishes before any wait of its own, so the
//    waits end; each is bounded all the same (STATUS_WAIT_LIMIT, results then invalid, no hang).
// Surfaces may also be scheduled a lag of tickets behind their last dependency (so that the tile has finished when
// they start), with a tail of surface-only tickets after the tiles. The counter runs on across launches: launch L's
// CTAs take tickets L grid .. L grid + grid - 1, so the ticket gives both the CTA's place q (ticket mod grid; a
// volume tile when q < tiles) and the launch (ticket / grid + 1, the value a finished tile's flag holds), and no
// reset is needed between launches. The arithmetic of both phases is that of lw_volume_kernel and
// surface_kernel: the results equal the two-launch path's bit for bit.
#pragma once
#include "tlw_surface.cuh"
#include "tlw_volume.cuh"

namespace tlw {

struct FuseArgs {
    unsigned long long* ticket;   // launch-order counter (zeroed with the flags when the mesh is set)
    unsigned* ready;              // [tiles] launch number (1-based) of the last finished volume phase of each tile
    const int* list;              // [E] elements in the order of their surface ticket
    const int* off;               // [grid + 1] list range of each ticket
    const int* nbr;               // [4, E] element across each face (-x, +x, -y, +y)
    int tiles;                    // volume tiles (tickets below tiles run a volume phase)
    int grid;                     // CTAs (tickets) of every launch: the tiles and the tail of surface-only tickets
};

// iterations of a dependency wait before it gives up (about a second with the back-off below)
constexpr int FUSE_WAIT_LIMIT = 1 << 24;

__device__ __forceinline__ unsigned ld_acquire_gpu(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release_gpu(unsigned* p, unsigned v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ void wait_flag(const unsigned* f, unsigned launch, unsigned* status) {
    for (int it = 0; ld_acquire_gpu(f) < launch; ++it) {
        if (it >= FUSE_WAIT_LIMIT) {
            atomicOr(status, STATUS_WAIT_LIMIT);
            return;
        }
        __nanosleep(64);
    }
}

template <int N>
struct FusedCfg {
    using C = VolCfg<N>;
    static constexpr int n = N + 1;
    // surface elements per group: one phase-1 thread per (element, face, node)
    static constexpr int GROUP = C::THREADS / (4 * n);
    static_assert(GROUP >= 1, "a CTA must hold one element's face nodes");
    static constexpr size_t GROUP_BYTES = (size_t)GROUP * 4 * n * NV * sizeof(double);
    // dynamic shared memory of a launch: the stage's planes, or the surface group if that is larger
    static constexpr size_t smem(size_t stage_bytes) { return stage_bytes > GROUP_BYTES ? stage_bytes : GROUP_BYTES; }
};

// STAGE: TLW_STAGE_LW (lw_volume_tile), TLW_STAGE_MDRK1 / _MDRK2 (mdrk1 / mdrk2_volume_tile; COMPACT: the plain
// step's compact stages)
template <int N, int MODE, int STAGE, bool COMPACT>
static __global__ void __launch_bounds__(VolCfg<N>::THREADS,
                                         STAGE == 0 ? VolCfg<N>::MIN_BLOCKS : VolCfg<N>::MDRK_MIN_BLOCKS)
    lw_fused_kernel(VolArgs a, SurfArgs sa, FuseArgs fa) {
    using C = VolCfg<N>;
    constexpr int EB = C::EB, GS = FusedCfg<N>::GROUP;
    extern __shared__ double smem_d[];
    unsigned long long* s_ticket = reinterpret_cast<unsigned long long*>(smem_d);   // (before the planes' use)
    const int tid = threadIdx.x;
    if (tid == 0) *s_ticket = atomicAdd(fa.ticket, 1ull);
    __syncthreads();
    const unsigned long long tk = *s_ticket;
    __syncthreads();
    const int q = (int)(tk % (unsigned long long)fa.grid);
    const unsigned launch = (unsigned)(tk / (unsigned long long)fa.grid) + 1u;
    if (q < fa.tiles) {
        if constexpr (STAGE == 0) lw_volume_tile<N, MODE, false>(a, q);
        else if constexpr (STAGE == 1) mdrk1_volume_tile<N, MODE, false, false, 0, false, COMPACT>(a, q);
        else mdrk2_volume_tile<N, MODE, false, false, 0, false, COMPACT>(a, q);
        __syncthreads();
        if (tid == 0) {
            __threadfence();
            st_release_gpu(fa.ready + q, launch);
        }
    }
    const int beg = __ldg(fa.off + q), end = __ldg(fa.off + q + 1);
    for (int g = beg; g < end; g += GS) {
        const int cnt = min(GS, end - g);
        if (tid < 5 * cnt) {
            const int el = tid / 5, k = tid - 5 * el;
            const int e = __ldg(fa.list + g + el);
            const int x = k == 4 ? e : __ldg(fa.nbr + 4 * e + k);
            if (x >= 0) wait_flag(fa.ready + x / EB, launch, sa.status);
        }
        __syncthreads();
        surface_group<N, false, false, true, GS>(sa, BndArgs{}, smem_d, tid, 0, fa.list + g, cnt);
        __syncthreads();
    }
}

}  // namespace tlw
