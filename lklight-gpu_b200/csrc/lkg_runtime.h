// Host runtime types of liblkg (context, device-resident complexes).
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <memory>
#include <string>
#include <vector>

#include "../../include/lkg.h"
#include "lkg_internal.h"

namespace lkg {

int set_error(int status, const char* fmt, ...);
int set_ok();
int cuda_to_status(cudaError_t e);

#define LKG_CK(call, what)                                                                    \
    do {                                                                                      \
        cudaError_t e_ = (call);                                                              \
        if (e_ != cudaSuccess) return ::lkg::set_error(::lkg::cuda_to_status(e_), "%s: %s", \
                                                       what, cudaGetErrorString(e_));         \
    } while (0)

// owning device allocation
struct DBuf {
    void* p = nullptr;
    size_t bytes = 0;
    DBuf() = default;
    DBuf(const DBuf&) = delete;
    DBuf& operator=(const DBuf&) = delete;
    ~DBuf() { release(); }
    void release() { if (p) cudaFree(p); p = nullptr; bytes = 0; }
    // grow-only, contents not kept; a buffer that has to grow again grows
    // by at least half its size, so slowly rising demands (the candidate
    // counts of successive GSO steps) do not reallocate every time (each
    // cudaFree synchronises the device)
    cudaError_t reserve(size_t n) {
        if (n <= bytes && p) return cudaSuccess;
        const size_t want = p ? std::max(n, bytes + bytes / 2) : n;
        release();
        cudaError_t e = cudaMalloc(&p, want ? want : 16);
        if (e == cudaSuccess) bytes = want ? want : 16;
        else p = nullptr;
        return e;
    }
    template <class T> T* as() const { return (T*)p; }
};

// pinned host allocation
struct HBuf {
    void* p = nullptr;
    size_t bytes = 0;
    HBuf() = default;
    HBuf(const HBuf&) = delete;
    HBuf& operator=(const HBuf&) = delete;
    ~HBuf() { if (p) cudaFreeHost(p); }
    cudaError_t reserve(size_t n) {   // grow-only, geometric like DBuf
        if (n <= bytes && p) return cudaSuccess;
        const size_t want = p ? std::max(n, bytes + bytes / 2) : n;
        if (p) cudaFreeHost(p);
        p = nullptr; bytes = 0;
        cudaError_t e = cudaMallocHost(&p, want ? want : 16);
        if (e == cudaSuccess) bytes = want ? want : 16;
        return e;
    }
    template <class T> T* as() const { return (T*)p; }
};

// one molecule in the library's unified host form (f64, caller order)
struct MolIn {
    int n = 0;
    std::vector<double> c, q, svdw, eps, rad, des, asa;
    std::vector<uint8_t> heavy, excl;
};

// device arrays of one complex; `d` points into them
struct ComplexRec {
    int family = -1;
    DBuf rpos, rpar, rsolv, rpos64, rpar64, rsolv64, rorig, cell_start;
    DBuf rlb;   // distance lower bound of the receptor (ComplexDev::rlb)
    DBuf lpos, lpar, lsolv, lpos64, lpar64, lsolv64, lorig, lgrp;
    DBuf phi;
    DBuf rtag, ltag;   // interface tags (restraints / membrane), when set
    ComplexDev d{};
    int n_cells = 0;
};

struct Occupancy { int threads = 0, hcap = 0, blocks = 0; };

// per-launch scratch: per-unit partial sums, per-pose counters, the work
// counter and the status word (counters reset themselves after a launch)
struct Scratch {
    DBuf partials, pose_counter, work_counter, status, iface;
    DBuf far;   // [poses] far-field terms of the fast cpydock group
    size_t cap_units = 0, cap_poses = 0, cap_iface = 0;
    // desolvation spill tables (every slot empty between launches)
    DBuf spill;
    // iface_words: interface bit words of the whole batch (poses x stride)
    cudaError_t ensure(size_t units, size_t poses, cudaStream_t s, size_t iface_words = 0);
    // at least `bytes` of spill tables, all slots empty (0xff bytes)
    cudaError_t ensure_spill(size_t bytes, cudaStream_t s);
};

// one launch group's item tables: (complex, first pose, pose count) per item
// and cumulative work units; `kind` 0 = tile kernels, 1 = fused desolvation
struct Group {
    int kind = 0;
    std::vector<int> ic, ip0, inp;
    std::vector<long long> w0{0};
    int hcap = 64;
    int spill_cap = 0;     // desolvation spill slots per block: a power of two above the largest receptor
    int iface_words = 0;   // interface bit words per pose (the batch's largest)
    size_t bytes() const { return (ic.size() + 1) * sizeof(long long) + ic.size() * 3 * sizeof(int); }
    void pack(char* dst) const;
};

}  // namespace lkg

struct lkg_ctx {
    int device = 0;
    int sm_count = 148;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    int precision = LKG_PREC_FAST;
    int tile = 128;                 // ligand atoms per work unit
    int group = 8;                  // ligand atoms per candidate-search group
    int desolv_threads = 512;
    float cell_h = 0.f;             // receptor cell edge in y and z (A); 0: per family
    int xsub = 0;                   // x sub-cells per cell edge; 0: per family
    std::vector<std::unique_ptr<lkg::ComplexRec>> cx;
    lkg::DBuf d_cx;                 // ComplexDev[] on the device
    bool cx_dirty = true;
    uint64_t cx_version = 0;        // bumped by every change of a complex (captured graphs check it)
    lkg::Scratch scratch;
    // item tables
    lkg::DBuf d_items;
    lkg::HBuf h_items;
    std::vector<char> last_items;   // tables currently in d_items
    // host-buffer call staging
    lkg::DBuf d_poses, d_scores, d_parts;
    lkg::HBuf h_poses, h_out;
    int64_t launches = 0;
    lkg::Occupancy occ_tiles[2], occ_desolv[2];
    bool noalloc_used = false;      // lkg_score_device_noalloc ran on this context (its status word is checked)
    bool setup_on_device = true;    // receptor cell sort and packing on the GPU (false: the host build)
    bool stage_tma = false;         // plain warp kernel: candidates staged by bulk copies (measured alternative)
};

namespace lkg {
// build + upload one complex (receptor / ligand already in unified form);
// field: either provided (phi host pointer + geometry) or built on the GPU
int complex_create(lkg_ctx* ctx, int family, unsigned flags, int lj_form, const MolIn& rec,
                   const MolIn& lig, const lkg_field* field, bool build_field, double solv_const,
                   int* out_id);
// lower bound of the distance to the nearest of n receptor atoms on a
// coarse grid (dims, origin out; ComplexDev::rlb)
std::vector<float> receptor_distance_bound(const double* c, int n, int dims[3], float origin[3]);
// the receptor's cell-sorted arrays and cell_start built on the GPU
// (lkg_cells.cu), bit for bit the host build's
int build_receptor_device(lkg_ctx* ctx, const MolIn& R, ComplexRec& cr, const float o[3], const int nc[3],
                          const float inv_e[3]);
// replace the ligand of an existing complex (cuda_full_score)
int complex_set_ligand(lkg_ctx* ctx, int id, const MolIn& lig);
// a complex changed: descriptors to upload, captured graphs out of date
inline void mark_dirty(lkg_ctx* ctx) { ctx->cx_dirty = true; ++ctx->cx_version; }
// interface tags (restraints / membrane) of a complex, caller atom order
int complex_set_restraints(lkg_ctx* ctx, int id, const int32_t* rres, int nres_r, const int32_t* lres, int nres_l,
                           const int32_t* mem, int nmem);
// one persistent launch group over items; device pointers
int launch_items(lkg_ctx* ctx, int n_items, const int* ids, const int* counts, const double* d_poses,
                 double* d_scores, double* d_parts, int raw_pairs, int solv_only, float* atom_e,
                 float* atom_v, double* d_iface = nullptr);
int wait_stream(lkg_ctx* ctx, double timeout_s);
int check_status(lkg_ctx* ctx);
int check_status_word(int* d_status);
// status word of the no-allocation entry point's array on the context's device
int noalloc_check_status(lkg_ctx* ctx);
// item tables of the two launch groups for a batch
int build_groups(lkg_ctx* ctx, int n_items, const int* ids, const int* counts, Group g[2], size_t* n_poses);
int sync_descriptors(lkg_ctx* ctx);
// persistent grid of a launch group at the given precision
long long group_blocks(lkg_ctx* ctx, const Group& g, bool exact);
// spill table bytes of a desolvation group at the given precision
size_t group_spill_bytes(lkg_ctx* ctx, const Group& g, bool exact);
// launch one prepared group (kernel launches only: stream-capturable)
int launch_group(lkg_ctx* ctx, const Group& g, const char* d_tables, Scratch& sc, const double* d_poses,
                 double* d_scores, double* d_parts, int raw_pairs, int solv_only, float* atom_e, float* atom_v,
                 const unsigned char* pose_mask = nullptr, double* d_iface = nullptr);
// a plan's launch group(s) scoring only the poses whose mask byte is set
int plan_launch_masked(lkg_plan* plan, const double* d_poses, double* d_scores, const unsigned char* d_mask);
void field_geometry(const double* coords, int n, double lo[3], int dims[3], double* spacing);
}  // namespace lkg
