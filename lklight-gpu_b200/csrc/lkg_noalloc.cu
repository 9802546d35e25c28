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
//     32 bytes per (pose, ligand tile) + 4 bytes per pose (rounded up to a
//     multiple of 8) + 64 bytes; larger batches are rejected with
//     LKG_ERR_CAPACITY before any work.
//   * The host cannot use the array's name as a device address; on the
//     first call on each device (with that device current) the entry point
//     looks the address up once with cudaGetSymbolAddress and keeps it for
//     the process.  Make that first call before any stream capture, and do
//     not use the entry point across a cudaDeviceReset (the reset unloads
//     the module and the kept address would be stale).
//   * Every call shares the one array and it keeps the last call's
//     contents, so each call clears the counters it needs with
//     cudaMemsetAsync on its stream and writes its one-item work table with
//     a one-thread kernel (values passed by value: nothing is read from
//     host memory).  Calls whose kernels overlap on the GPU (different
//     streams, or several contexts on one device) race on the array:
//     serialise them.
//   * The kernel reports errors in a status word inside the array;
//     lkg_ctx_sync (which waits for the context stream) reads and clears it
//     after a no-allocation call, as it does the context's own word.
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

// byte offsets inside the array
constexpr size_t OFF_WORK = 0, OFF_STATUS = 16, OFF_WORK0 = 32, OFF_ITEMS = 48, OFF_HEAD = 64;

// the call's one-item work table, written on the device from values
// passed by value: (work0[0], work0[1]) = (0, total), items = (complex, first
// pose, pose count, 0)
__global__ void k_noalloc_table(unsigned char* base, int complex_id, int n_pose, long long total) {
    long long* w0 = reinterpret_cast<long long*>(base + OFF_WORK0);
    int* it = reinterpret_cast<int*>(base + OFF_ITEMS);
    w0[0] = 0;
    w0[1] = total;
    it[0] = complex_id; it[1] = 0; it[2] = n_pose; it[3] = 0;
}

}  // namespace

namespace lkg {
// status word of the last no-allocation call on the context's device (the
// context's stream has been waited for by the caller)
int noalloc_check_status(lkg_ctx* ctx) {
    void* base = nullptr;
    {
        std::lock_guard<std::mutex> g(g_mu);
        if (ctx->device >= 0 && ctx->device < 64) base = g_addr[ctx->device];
    }
    if (!base) return set_ok();
    return check_status_word(reinterpret_cast<int*>(static_cast<char*>(base) + OFF_STATUS));
}
}  // namespace lkg

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
    const size_t head = OFF_HEAD;
    const size_t counters = ((size_t)n_pose * sizeof(int) + 7) & ~(size_t)7;   // partials stay 8-byte aligned
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
    // the array keeps the previous call's contents: zero the work counter,
    // the status word and the pose counters, then write this call's table
    const long long total = (long long)n_pose * d.ntiles;
    LKG_CK(cudaMemsetAsync(base, 0, head + counters, s), "scratch clear");
    k_noalloc_table<<<1, 1, 0, s>>>((unsigned char*)base, complex_id, n_pose, total);
    LKG_CK(cudaGetLastError(), "work table");
    ctx->launches++;
    ctx->noalloc_used = true;

    LaunchParams p{};
    p.cx = ctx->d_cx.as<ComplexDev>();
    p.item_work0 = (const long long*)(base + OFF_WORK0);
    p.item_complex = (const int*)(base + OFF_ITEMS);
    p.item_pose0 = p.item_complex + 1;
    p.item_npose = p.item_complex + 2;
    p.n_items = 1;
    p.total_work = total;
    p.tile = ctx->tile;
    p.poses = d_poses;
    p.scores = d_scores;
    p.parts = d_parts;
    p.work_counter = (unsigned long long*)(base + OFF_WORK);
    p.status = (int*)(base + OFF_STATUS);
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
