// lkg_score_device_noalloc: the tile scoring kernel with its scratch memory
// in a fixed, file-scope device array instead of context-owned allocations.
//
// Who needs it: callers that may not allocate device memory at scoring time —
// a host framework that owns the whole device heap through its own pool or
// caching allocator and forbids side allocations, a real-time docking loop
// that cannot absorb cudaMalloc latency or its implicit device
// synchronisation, or code that scores inside a region where allocation
// calls are not allowed.  This entry point calls no cudaMalloc, cudaFree or
// allocating library routine: the per-tile partial sums, the per-pose
// completion counters, the work counter and the status word all live in
// g_noalloc_scratch below.
//
// Limits and rules:
//   * The array holds LKG_NOALLOC_SCRATCH_BYTES (8 MiB) on every GPU that
//     loads liblkg, for the life of the process.  A call needs
//     32 bytes per (pose, ligand tile) + 4 bytes per pose + 64 bytes;
//     larger batches are rejected with LKG_ERR_CAPACITY before any work.
//   * The host cannot use the array's name as a device address; on the
//     first call on each device (with that device current) the entry point
//     looks the address up once with cudaGetSymbolAddress.  Make that first
//     call before any stream capture.
//   * Every call shares the one array and it keeps the last call's
//     contents, so each call clears the counters it needs with
//     cudaMemsetAsync on its stream first.  Calls whose kernels overlap on
//     the GPU (different streams, or several contexts on one device) race
//     on the array: serialise them.
//   * The complex must already be resident (lkg_complex_add) and its device
//     descriptor uploaded by an earlier scoring call of the context; the
//     fast (f32) tile kernel is used; cpydock complexes (shared-memory
//     desolvation kernel) are rejected.
#include <cstring>
#include <mutex>

#include "lkg_runtime.h"
#include "lkg_score.cuh"

#define LKG_NOALLOC_SCRATCH_BYTES (8u << 20)

namespace {

__device__ __align__(256) static unsigned char g_noalloc_scratch[LKG_NOALLOC_SCRATCH_BYTES];

std::mutex g_mu;
void* g_addr[64] = {nullptr};  // per-device address of g_noalloc_scratch

}  // namespace

using namespace lkg;

extern "C" {

int lkg_score_device_noalloc(lkg_ctx* ctx, int complex_id, int n_pose, const double* d_poses, double* d_scores,
                             double* d_parts) {
    if (!ctx) return set_error(LKG_ERR_ARG, "null ctx");
    if (n_pose == 0) return set_ok();
    if (n_pose < 0 || !d_poses || !d_scores) return set_error(LKG_ERR_ARG, "bad pose buffer");
    if (complex_id < 0 || complex_id >= (int)ctx->cx.size())
        return set_error(LKG_ERR_ARG, "bad complex id %d", complex_id);
    if (ctx->cx_dirty || !ctx->d_cx.p)
        return set_error(LKG_ERR_STATE, "complex descriptors not on the device yet: make one regular scoring call "
                                        "after the last lkg_complex_add");
    const ComplexDev& d = ctx->cx[complex_id]->d;
    if (d.flags & F_DESOLV) return set_error(LKG_ERR_ARG, "cpydock complexes are not supported without allocation");
    if (d.iface_words) return set_error(LKG_ERR_ARG, "complexes with restraints or a membrane are not supported without allocation");
    LKG_CK(cudaSetDevice(ctx->device), "cudaSetDevice");

    // sizes: [work counter 16 B | status 16 B | item tables 32 B | pose counters | partials]
    const size_t head = 64;
    const size_t counters = ((size_t)n_pose * sizeof(int) + 255) & ~(size_t)255;
    const size_t partials = (size_t)n_pose * d.ntiles * 4 * sizeof(double);
    if (head + counters + partials > LKG_NOALLOC_SCRATCH_BYTES)
        return set_error(LKG_ERR_CAPACITY,
                         "batch needs %zu bytes of scratch (%d poses x %d ligand tiles); the fixed array holds %u",
                         head + counters + partials, n_pose, d.ntiles, LKG_NOALLOC_SCRATCH_BYTES);

    char* base;
    {
        std::lock_guard<std::mutex> g(g_mu);
        if (ctx->device >= 64) return set_error(LKG_ERR_ARG, "device index too large");
        if (!g_addr[ctx->device]) {
            void* p = nullptr;
            cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
            if (e != cudaSuccess)
                return set_error(cuda_to_status(e), "cudaGetSymbolAddress: %s", cudaGetErrorString(e));
            g_addr[ctx->device] = p;
        }
        base = (char*)g_addr[ctx->device];
    }
    cudaStream_t s = ctx->stream;
    // the array keeps the previous call's contents: zero the counters, the
    // status word and the item table region before this launch
    LKG_CK(cudaMemsetAsync(base, 0, head + counters, s), "scratch clear");
    long long work0[2] = {0, (long long)n_pose * d.ntiles};
    int items[4] = {complex_id, 0, n_pose, 0};
    LKG_CK(cudaMemcpyAsync(base + 32, work0, sizeof(work0), cudaMemcpyHostToDevice, s), "item table");
    LKG_CK(cudaMemcpyAsync(base + 48, items, sizeof(items), cudaMemcpyHostToDevice, s), "item table");

    LaunchParams p{};
    p.cx = ctx->d_cx.as<ComplexDev>();
    p.item_work0 = (const long long*)(base + 32);
    p.item_complex = (const int*)(base + 48);
    p.item_pose0 = p.item_complex + 1;
    p.item_npose = p.item_complex + 2;
    p.n_items = 1;
    p.total_work = work0[1];
    p.tile = ctx->tile;
    p.poses = d_poses;
    p.scores = d_scores;
    p.parts = d_parts;
    p.work_counter = (unsigned long long*)base;
    p.status = (int*)(base + 16);
    p.pose_counter = (int*)(base + head);
    p.partials = (double*)(base + head + counters);
    p.max_tiles = d.ntiles;
    int occ = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_score_tiles<float>, ctx->tile, 0);
    long long blocks = (long long)ctx->sm_count * (occ > 0 ? occ : 1);
    if (blocks > p.total_work) blocks = p.total_work;
    k_score_tiles<float><<<(int)blocks, ctx->tile, 0, s>>>(p);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return set_error(cuda_to_status(e), "score launch: %s", cudaGetErrorString(e));
    ctx->launches++;
    return set_ok();
}

}  // extern "C"
