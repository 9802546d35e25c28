// f64 exact path: instantiations and launchers.  This file is compiled with
// --fmad=false so that every f64 multiply-add follows the reference's
// operation order (no contraction), as the oracle and the Rust code do.
#include "lkg_score.cuh"

namespace lkg {

cudaError_t launch_score_exact(const LaunchParams& p, int threads, int blocks, cudaStream_t s) {
    k_score_tiles<double><<<blocks, threads, 0, s>>>(p);
    return cudaGetLastError();
}

cudaError_t launch_desolv_exact(const LaunchParams& p, int threads, int blocks, int hcap, cudaStream_t s) {
    size_t sm = desolv_smem_bytes(hcap, true);
    cudaError_t e = cudaFuncSetAttribute(k_score_desolv<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    k_score_desolv<double><<<blocks, threads, sm, s>>>(p);
    return cudaGetLastError();
}

int max_blocks_score_exact(int threads) {
    int n = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_score_tiles<double>, threads, 0);
    return n;
}
int max_blocks_desolv_exact(int threads, int hcap) {
    int n = 0;
    size_t sm = desolv_smem_bytes(hcap, true);
    cudaFuncSetAttribute(k_score_desolv<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_score_desolv<double>, threads, sm);
    return n;
}

}  // namespace lkg
