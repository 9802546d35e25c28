// f32 fast path: instantiations and launchers of the fused scoring kernels.
#include "lkg_score.cuh"

namespace lkg {

cudaError_t launch_score_fast(const LaunchParams& p, int threads, int blocks, cudaStream_t s) {
    k_score_tiles<float><<<blocks, threads, 0, s>>>(p);
    return cudaGetLastError();
}

size_t desolv_smem_bytes(int hcap, bool /*exact*/) { return (size_t)hcap * 12; }

cudaError_t launch_desolv_fast(const LaunchParams& p, int threads, int blocks, int hcap, cudaStream_t s) {
    size_t sm = desolv_smem_bytes(hcap, false);
    cudaError_t e = cudaFuncSetAttribute(k_score_desolv<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    k_score_desolv<float><<<blocks, threads, sm, s>>>(p);
    return cudaGetLastError();
}

int max_blocks_score_fast(int threads) {
    int n = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_score_tiles<float>, threads, 0);
    return n;
}
int max_blocks_desolv_fast(int threads, int hcap) {
    int n = 0;
    size_t sm = desolv_smem_bytes(hcap, false);
    cudaFuncSetAttribute(k_score_desolv<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_score_desolv<float>, threads, sm);
    return n;
}

}  // namespace lkg
