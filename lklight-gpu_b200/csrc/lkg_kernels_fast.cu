// f32 fast path: instantiations and launchers of the fused scoring kernels.
#include "lkg_score_v2.cuh"

namespace lkg {

// warp-cooperative kernel for scores; the per-thread kernel when per-atom
// outputs are requested (cuda_full_score)
template <int TILE, int G>
static size_t v2_smem() { return (size_t)(TILE / 32) * sizeof(V2Warp<G>); }

template <int TILE, int G>
static cudaError_t launch_v2g(const LaunchParams& p, int blocks, cudaStream_t s) {
    const size_t sm = v2_smem<TILE, G>();
    cudaError_t e = cudaFuncSetAttribute(k_score_v2<TILE, G>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    k_score_v2<TILE, G><<<blocks, TILE, sm, s>>>(p);
    return cudaGetLastError();
}

template <int TILE>
static cudaError_t launch_v2(const LaunchParams& p, int blocks, cudaStream_t s) {
    switch (p.group) {
        case 8: return launch_v2g<TILE, 8>(p, blocks, s);
        case 16: return launch_v2g<TILE, 16>(p, blocks, s);
        default: return launch_v2g<TILE, 32>(p, blocks, s);
    }
}

cudaError_t launch_score_fast(const LaunchParams& p, int threads, int blocks, cudaStream_t s) {
    if (p.atom_elec) {
        k_score_tiles<float><<<blocks, threads, 0, s>>>(p);
        return cudaGetLastError();
    }
    switch (threads) {
        case 64: return launch_v2<64>(p, blocks, s);
        case 128: return launch_v2<128>(p, blocks, s);
        default: return launch_v2<256>(p, blocks, s);
    }
}

template <int TILE, int G>
static int occ_v2g() {
    int m = 0;
    const size_t sm = v2_smem<TILE, G>();
    cudaFuncSetAttribute(k_score_v2<TILE, G>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&m, k_score_v2<TILE, G>, TILE, sm);
    return m;
}

template <int TILE>
static int occ_v2(int group) {
    switch (group) {
        case 8: return occ_v2g<TILE, 8>();
        case 16: return occ_v2g<TILE, 16>();
        default: return occ_v2g<TILE, 32>();
    }
}

size_t desolv_smem_bytes(int hcap, bool /*exact*/) { return (size_t)hcap * 12; }

cudaError_t launch_desolv_fast(const LaunchParams& p, int threads, int blocks, int hcap, cudaStream_t s) {
    size_t sm = desolv_smem_bytes(hcap, false);
    cudaError_t e = cudaFuncSetAttribute(k_score_desolv<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    k_score_desolv<float><<<blocks, threads, sm, s>>>(p);
    return cudaGetLastError();
}

int max_blocks_score_fast(int threads, int group) {
    int n = 0, m = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_score_tiles<float>, threads, 0);
    switch (threads) {
        case 64: m = occ_v2<64>(group); break;
        case 128: m = occ_v2<128>(group); break;
        default: m = occ_v2<256>(group); break;
    }
    return n < m ? n : m;  // one grid size serves both kernels
}
int max_blocks_desolv_fast(int threads, int hcap) {
    int n = 0;
    size_t sm = desolv_smem_bytes(hcap, false);
    cudaFuncSetAttribute(k_score_desolv<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_score_desolv<float>, threads, sm);
    return n;
}

}  // namespace lkg
