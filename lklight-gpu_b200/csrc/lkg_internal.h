// Internal types shared by the lkg kernels and the host runtime.
//
// Device layout of one complex (all arrays in HBM, built once per complex):
//   receptor atoms sorted by a fine cell grid (edge h in y and z, default
//   2.5 A; edge h / xsub in x, cells x-fastest), so that one (z, y) row of
//   consecutive x cells is one contiguous span of atoms
//   [cell_start[row+cx0], cell_start[row+cx1+1]);
//     rpos  float4 (x, y, z, q)              rpos64 double4 (same, f64)
//     rpar  float4 (sqrt eps, r, heavy, excl) rpar64 double4 (sqrt eps, r, eps, heavy)
//     rsolv float2 (des, asa)                rsolv64 double2
//   ligand atoms ordered by recursive coordinate bisection of the reference
//   frame into groups of `group` atoms (groups and tiles of consecutive
//   atoms are spatially compact), same three arrays;
//   receptor far field phi (f32, x fastest, the ReceptorField layout).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace lkg {

enum : unsigned { F_FAR = 1u, F_ELEC = 2u, F_CLASH = 4u, F_DESOLV = 16u };
// LJ formula variants of the exact (f64) path:
//   0: sqrt(eps_i)*sqrt(eps_j) * (p6^2 - 2 p6), f64::min cap   (dna, pydock)
//   1: sqrt(eps_i*eps_j) * (p6^2 - 2 p6), cap by `if k > 1`     (vdw)
//   2: as 1 with p6 = pow(r,6)/pow(d2,3)                          (cpydock)
enum { LJ_SVDW = 0, LJ_SQRT = 1, LJ_POW = 2 };

struct ComplexDev {
    int nr, nl;
    unsigned flags;          // F_* of this complex's family
    int lj_form;             // LJ_* (exact path)
    // receptor (sorted by fine cell)
    const float4* rpos;
    const float4* rpar;
    const float2* rsolv;
    const double4* rpos64;
    const double4* rpar64;
    const double2* rsolv64;
    const int* rorig;        // sorted -> caller index
    const int* cell_start;   // ncx*ncy*ncz + 1
    int ncx, ncy, ncz;       // ncx counts x sub-cells
    float ox, oy, oz, h, inv_h, hx, inv_hx;
    // ligand (bisection-ordered)
    const float4* lpos;
    const float4* lpar;
    const float2* lsolv;
    const double4* lpos64;
    const double4* lpar64;
    const double2* lsolv64;
    const int* lorig;
    // lower bound of the distance to the nearest receptor atom on cells of
    // rlb_s A (x fastest) over the receptor's box grown by rlb_m A; points
    // outside are farther than rlb_m from every atom; null: no bound
    const float* rlb;
    int rlbx, rlby, rlbz;
    float rlbox, rlboy, rlboz, rlb_inv, rlb_m;
    const float4* lgrp;      // per group of `group` atoms: ligand-frame centre, radius
    int group;               // ligand atoms per candidate-search group
    int ntiles;              // ceil(nl / tile)
    // far field: fnx x fny x fnz points in bricks of 4 x 4 x 4 (fbx x fby x
    // fbz bricks, x-fastest; points x-fastest inside a brick)
    const float* phi;
    int fnx, fny, fnz;
    int fbx, fby, fbz;
    float fox, foy, foz, fsp;
    double fox64, foy64, foz64, fsp64;
    double finv64;           // 1 / spacing when the spacing is a power of two (then x * finv64 == x / spacing), else 0
    // desolvation
    int hcap;                // receptor-minimum hash capacity (power of two)
    double solv_const;       // sum over asa<0 atoms of asa*des (CPU-grid semantics)
    // interface flags (active restraints, membrane): per pose, one bit per
    // receptor restraint residue, ligand restraint residue and membrane bead
    // (in that order) set when one of its atoms lies within 3.9 A of an
    // atom of the other molecule; null tags = no restraints or membrane
    const int2* rtag;        // sorted receptor atom -> (restraint bit, membrane bit), -1 = none
    const int* ltag;         // bisection-ordered ligand atom -> restraint bit, -1 = none
    int nres_r, nres_l, nmem;
    int iface_words;         // 32-bit words of one pose's interface bits (0: none)
    int iface_form;          // IF_* score combination of the family
};

// how the restraint fractions and the membrane penalty enter the score
//   IF_DNA: s += pr*s + pl*s - pen              (dna.rs:989-995)
//   IF_SUM: s = s + pr*s + pl*s - pen           (pydock.rs:440-445, cpydock.rs:670-675)
//   IF_VDW: s = s + pr*s + pl*s, no membrane    (vdw.rs:146-149)
enum { IF_NONE = 0, IF_DNA = 1, IF_SUM = 2, IF_VDW = 3 };

// One launch over a batch of (complex, pose range) items.
struct LaunchParams {
    const ComplexDev* cx;        // device array of complex descriptors
    const int* item_complex;     // [n_items]
    const int* item_pose0;       // [n_items] global pose offset
    const int* item_npose;       // [n_items]
    const long long* item_work0; // [n_items+1] cumulative work units
    int n_items;
    long long total_work;
    int tile;                    // ligand atoms per work unit (non-desolv kernel)
    int group;                   // ligand atoms per candidate-search group
    const double* poses;         // global N x 7 (w,x,y,z,tx,ty,tz)
    double* scores;              // [N] final score, or N x 2 raw (elec, vdw) when raw_pairs
    double* parts;               // [N x 4] or null: elec_raw, vdw, solv, near pairs
    int raw_pairs;               // compat: scores holds (elec_raw, vdw) pairs
    int solv_only;               // compat cuda_cpydock_solv: scores[k] = S
    // scratch (self-resetting between launches)
    double* partials;            // [total_work x 4] per-unit partial sums
    int* pose_counter;           // [N]
    unsigned long long* work_counter;  // [2]: next unit, CTAs done
    int* status;                 // [4]: error flags (capacity overflow, bad index)
    int max_tiles;               // unused by the kernels (kept for layout)
    // per-atom outputs (cuda_full_score): pose 0 of item 0, caller atom order
    float* atom_elec;
    float* atom_vdw;
    // optional [N]: poses whose byte is 0 are skipped (their score and parts
    // keep their previous values: the device GSO's unmoved glowworms)
    const unsigned char* pose_mask;
    // interface bits: iface_stride words per pose (global pose index),
    // all zero between launches (the pose's last unit clears them);
    // null when no complex of the launch has restraints or a membrane
    unsigned* iface;
    int iface_stride;
    // optional [N x 3]: restraint fractions (receptor, ligand) and membrane
    // intersection of each scored pose
    double* iface_out;
    // desolvation spill tables: one region of spill_cap slots per block
    // (SPILL_SLOT_BYTES each), all slots empty between poses; null: none
    unsigned char* spill;
    int spill_cap;
    // plain warp kernel: stage candidates in shared memory by bulk copies
    int stage;
    // [N] far-field term of each pose from k_far_poses (fast cpydock
    // launch groups), added to the pose's electrostatics; null: inline
    double* far;
};

// bytes per spill slot: the exact kernel's 8-byte value + 4-byte key (the
// fast kernel's packed 8-byte slots use the first 8 x spill_cap bytes)
constexpr int SPILL_SLOT_BYTES = 12;

constexpr double FACTOR = 332.0;
constexpr double EPSILON = 4.0;
constexpr float ES_CAP_F = (float)(4.0 / 332.0);
constexpr double ES_CAP_D = 1.0 * 4.0 / 332.0;
constexpr float NEAR_R = 10.0f;
constexpr float SCAN_R = 10.001f;   // candidate radius (superset margin over 10 A)
constexpr float SOLV2_F = 40.96f;   // 6.4^2 as the reference GPU writes it
constexpr double SOLV2_D = 6.4 * 6.4;
constexpr double IFACE2_D = 3.9 * 3.9;   // INTERFACE_CUTOFF^2 (constants.rs:14-15)
constexpr float IFACE2_F = 15.2115f;    // f32 prefilter, 1e-4 above IFACE2_D
constexpr double MEMBRANE_PENALTY = 999.0;   // MEMBRANE_PENALTY_SCORE (constants.rs:21)

// launches (defined in lkg_kernels_*.cu)
cudaError_t launch_score_fast(const LaunchParams& p, int threads, int blocks, cudaStream_t s);
cudaError_t launch_desolv_fast(const LaunchParams& p, int threads, int blocks, int hcap, cudaStream_t s);
cudaError_t launch_score_exact(const LaunchParams& p, int threads, int blocks, cudaStream_t s);
cudaError_t launch_desolv_exact(const LaunchParams& p, int threads, int blocks, int hcap, cudaStream_t s);
// the far-field pass of a fast cpydock launch group (fills p.far)
cudaError_t launch_far_poses(const LaunchParams& p, int blocks, cudaStream_t s);
size_t desolv_smem_bytes(int hcap, bool exact);

// GPU far-field builder (lkg_field.cu), bit-identical to the reference's
// host builder: writes phi (n[0]*n[1]*n[2] floats) for receptor atoms
// given in their original order.
cudaError_t build_field_device(const double* d_coords, const double* d_q, int n,
                               const double lo[3], const int dims[3], double spacing,
                               float* d_phi, cudaStream_t s);
// the x-fastest grid src (nx x ny x nz) rearranged into 4 x 4 x 4 bricks
// (dst: nbx * nby * nbz * 64 floats, points past the grid 0)
cudaError_t phi_to_bricks(const float* src, int nx, int ny, int nz, float* dst, cudaStream_t s);
// far-field sum for cuda_far_field
cudaError_t launch_far_field_sum(const float* phi, int nx, int ny, int nz, float ox, float oy,
                                 float oz, float sp, const float* coords, const float* q, int n,
                                 double* d_result, cudaStream_t s);

}  // namespace lkg
