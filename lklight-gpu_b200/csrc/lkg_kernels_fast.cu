// f32 fast path: instantiations and launchers of the fused scoring kernels.
#include "lkg_score_warp.cuh"

namespace lkg {

// warp-independent kernel for scores; the per-thread kernel when per-atom
// outputs are requested (cuda_full_score)
template <int G>
static size_t warp_smem(bool stage = false) {
    return (size_t)(WK_THREADS / 32) * (sizeof(WSlots<G>) + sizeof(WQueue) + (stage ? sizeof(WStage) : 0));
}

// IFACE: the variant that also collects the interface bits (launches with
// restraint or membrane complexes); STAGE: candidates staged in shared
// memory by bulk copies (contexts that ask for it)
template <int G, bool IFACE, bool STAGE>
static cudaError_t launch_warp_gi(const LaunchParams& p, int blocks, cudaStream_t s) {
    const size_t sm = warp_smem<G>(STAGE);
    cudaError_t e = cudaFuncSetAttribute(k_score_warp<G, IFACE, STAGE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)sm);
    if (e != cudaSuccess) return e;
    k_score_warp<G, IFACE, STAGE><<<blocks, WK_THREADS, sm, s>>>(p);
    return cudaGetLastError();
}
template <int G>
static cudaError_t launch_warp_g(const LaunchParams& p, int blocks, cudaStream_t s) {
    if (p.iface) return launch_warp_gi<G, true, false>(p, blocks, s);
    return p.stage ? launch_warp_gi<G, false, true>(p, blocks, s) : launch_warp_gi<G, false, false>(p, blocks, s);
}

cudaError_t launch_score_fast(const LaunchParams& p, int threads, int blocks, cudaStream_t s) {
    if (p.atom_elec) {
        k_score_tiles<float><<<blocks, threads, 0, s>>>(p);
        return cudaGetLastError();
    }
    if (p.tile % p.group) return cudaErrorInvalidValue;
    switch (p.group) {
        case 4: return launch_warp_g<4>(p, blocks, s);
        case 8: return launch_warp_g<8>(p, blocks, s);
        case 16: return launch_warp_g<16>(p, blocks, s);
        default: return launch_warp_g<32>(p, blocks, s);
    }
}

template <int G>
static int occ_warp_g() {
    int m = 0;
    const size_t sm = warp_smem<G>();
    cudaFuncSetAttribute(k_score_warp<G, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&m, k_score_warp<G, false>, WK_THREADS, sm);
    return m;
}

size_t desolv_smem_bytes(int hcap, bool /*exact*/) { return (size_t)hcap * 12; }

// cpydock: the warp kernel for group sizes up to 16 (its per-warp slots and
// the block's minimum hash fit in shared memory), the per-atom kernel above
template <int G, bool IFACE>
static cudaError_t launch_warp_desolv_gi(const LaunchParams& p, int blocks, int hcap, cudaStream_t s) {
    const size_t sm = wd_smem<G>(hcap);
    cudaError_t e = cudaFuncSetAttribute(k_score_warp_desolv<G, IFACE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)sm);
    if (e != cudaSuccess) return e;
    k_score_warp_desolv<G, IFACE><<<blocks, WD_THREADS, sm, s>>>(p);
    return cudaGetLastError();
}
template <int G>
static cudaError_t launch_warp_desolv_g(const LaunchParams& p, int blocks, int hcap, cudaStream_t s) {
    return p.iface ? launch_warp_desolv_gi<G, true>(p, blocks, hcap, s)
                   : launch_warp_desolv_gi<G, false>(p, blocks, hcap, s);
}

cudaError_t launch_far_poses(const LaunchParams& p, int blocks, cudaStream_t s) {
    k_far_poses<<<blocks, FAR_THREADS, 0, s>>>(p);
    return cudaGetLastError();
}

cudaError_t launch_desolv_fast(const LaunchParams& p, int threads, int blocks, int hcap, cudaStream_t s) {
    switch (p.group) {
        case 4: return launch_warp_desolv_g<4>(p, blocks, hcap, s);
        case 8: return launch_warp_desolv_g<8>(p, blocks, hcap, s);
        case 16: return launch_warp_desolv_g<16>(p, blocks, hcap, s);
        default: break;
    }
    size_t sm = desolv_smem_bytes(hcap, false);
    cudaError_t e = cudaFuncSetAttribute(k_score_desolv<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    k_score_desolv<float><<<blocks, threads, sm, s>>>(p);
    return cudaGetLastError();
}

template <int G>
static int occ_warp_desolv_g(int hcap) {
    int n = 0;
    const size_t sm = wd_smem<G>(hcap);
    cudaFuncSetAttribute(k_score_warp_desolv<G, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_score_warp_desolv<G, false>, WD_THREADS, sm);
    return n;
}

// persistent grid of the warp kernel (blocks per SM); the per-thread kernel
// for per-atom outputs reuses the same grid size
int max_blocks_score_fast(int /*threads*/, int group) {
    switch (group) {
        case 4: return occ_warp_g<4>();
        case 8: return occ_warp_g<8>();
        case 16: return occ_warp_g<16>();
        default: return occ_warp_g<32>();
    }
}
int max_blocks_desolv_fast(int threads, int hcap, int group) {
    switch (group) {
        case 4: return occ_warp_desolv_g<4>(hcap);
        case 8: return occ_warp_desolv_g<8>(hcap);
        case 16: return occ_warp_desolv_g<16>(hcap);
        default: break;
    }
    int n = 0;
    size_t sm = desolv_smem_bytes(hcap, false);
    cudaFuncSetAttribute(k_score_desolv<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_score_desolv<float>, threads, sm);
    return n;
}

}  // namespace lkg
