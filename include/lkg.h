/* lkg — B200-native batched pose scoring for LKlight GSO docking.
 *
 * C ABI of liblkg.so.  Two groups of entry points:
 *
 *  1. Drop-in replacements for the reference's CUDA C ABI (same names, same
 *     signatures, same argument meaning, same 0 / -1 return convention and
 *     the same stderr message on failure), so src/gpu_score.rs,
 *     src/gpu_family.rs and src/gpu_field.rs link against liblkg unchanged.
 *     Host buffers are borrowed for the call; device copies of the constant
 *     receptor / ligand / field arrays are cached keyed on the host pointers,
 *     as the reference's cache does (full_score.cu:350-387).
 *
 *  2. A handle API (lkg_*) for callers that batch many complexes: device-
 *     resident complexes, one persistent launch per GSO step over all of them,
 *     CUDA-graph capture, device pointers, an exact (FP64) parity mode and
 *     enumerated status codes.  There is no CPU fallback anywhere: a missing
 *     device or a failed launch is reported as an error.
 *
 * Pose layout everywhere: 7 doubles per pose (w, x, y, z, tx, ty, tz) — the
 * unit quaternion then the translation, as full_score.cu:230 reads them.
 */
#ifndef LKG_H
#define LKG_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------------- */
/* Status codes                                                            */
/* ---------------------------------------------------------------------- */
typedef enum {
    LKG_OK = 0,
    LKG_ERR_ARG = 1,        /* bad argument / size */
    LKG_ERR_OOM = 2,        /* device allocation failed */
    LKG_ERR_LAUNCH = 3,     /* kernel launch / configuration failed */
    LKG_ERR_TIMEOUT = 4,    /* a bounded device wait or host poll ran out */
    LKG_ERR_DEVICE = 5,     /* sticky CUDA error or device fault */
    LKG_ERR_CAPACITY = 6,   /* a fixed-capacity device structure overflowed */
    LKG_ERR_NO_DEVICE = 7,  /* no CUDA device visible */
    LKG_ERR_STATE = 8       /* call not valid in the handle's current state */
} lkg_status;

const char* lkg_status_string(int status);
/* status / message of the last failing call on this thread */
int lkg_last_status(void);
const char* lkg_last_error(void);
/* 1 when a usable CUDA device is present (replaces gpu_score.rs:226-232) */
int lkg_device_available(void);
const char* lkg_version(void);

/* family flags (gpu_score.rs:15-21) and family ids */
#define LKG_F_FAR 1u
#define LKG_F_ELEC 2u
#define LKG_F_CLASH 4u
#define LKG_F_DESOLV 16u
enum { LKG_DNA = 0, LKG_VDW = 1, LKG_PYDOCK = 2, LKG_CPYDOCK = 3 };

/* ---------------------------------------------------------------------- */
/* 1. Reference-compatible entry points                                    */
/* ---------------------------------------------------------------------- */

/* Replaces src/cuda/full_score.cu:359-371 (Rust decls src/gpu_score.rs:252-262,
 * src/gpu_family.rs:209-221).  out[2k] = raw electrostatics of pose k (near
 * clamped sum + far-field q*phi; multiply by 332/4 on the host), out[2k+1] =
 * LJ (+ clash when LKG_F_CLASH).  flags: dna 7, pydock/cpydock 3, vdw 0; with
 * no LKG_F_FAR, phi may be a dummy and its dims 0. */
int cuda_batch_score(const float* phi, int nx, int ny, int nz, float ox, float oy, float oz, float sp,
                     const float* r_coords, const float* r_ele, const float* r_svdw,
                     const float* r_vdwr, const unsigned char* r_heavy, int nr,
                     const int* cell_start, const int* cell_atoms, int ncx, int ncy, int ncz,
                     float c_ox, float c_oy, float c_oz, float c_sp,
                     const float* l_base, const double* poses, const float* l_ele,
                     const float* l_svdw, const float* l_vdwr, const unsigned char* l_heavy,
                     int nl, int N, unsigned flags, double* out);

/* Replaces src/cuda/full_score.cu:571-581 (Rust decl src/gpu_family.rs:361-372).
 * outS[k] = sum over receptor and ligand atoms of g(min d^2)*des, with the
 * minimum taken over non-excluded opposite atoms (r_flag / l_flag == 0) and
 * g(d2) = min(-10*sqrt(d2) + 65, asa) when 0 < d2 <= 6.4^2 and asa > 0.
 * The minima, the reduction and the pose transform run in one fused kernel
 * with no N x nr scratch.  l_ele is unused (as in the reference). */
int cuda_cpydock_solv(const float* r_coords, const unsigned char* r_flag, int nr,
                      const int* cell_start, const int* cell_atoms, int ncx, int ncy, int ncz,
                      float c_ox, float c_oy, float c_oz, float c_sp,
                      const float* l_base, const double* poses, const unsigned char* l_flag,
                      const float* l_ele, int nl, int N,
                      const float* r_des, const float* r_asa, const float* l_des, const float* l_asa,
                      double* outS);

/* Replaces src/cuda/full_score.cu:140-150 (Rust decl src/gpu_score.rs:159-168):
 * one pose given as already-transformed ligand coordinates; per-atom outputs
 * (dna terms: far field, clamped electrostatics, LJ, clash). */
int cuda_full_score(const float* phi, int nx, int ny, int nz, float ox, float oy, float oz, float sp,
                    const float* r_coords, const float* r_ele, const float* r_svdw,
                    const float* r_vdwr, const unsigned char* r_heavy, int nr,
                    const int* cell_start, const int* cell_atoms, int ncx, int ncy, int ncz,
                    float c_ox, float c_oy, float c_oz, float c_sp,
                    const float* l_coords, const float* l_ele, const float* l_svdw,
                    const float* l_vdwr, const unsigned char* l_heavy, int nl,
                    float* out_elec, float* out_vdw);

/* Replaces src/cuda/far_field.cu:59-63 (Rust decl src/gpu_field.rs:20-33):
 * *result = sum_j q_j * phi(x_j) by trilinear interpolation. */
int cuda_far_field(const float* phi, int nx, int ny, int nz, float ox, float oy, float oz, float sp,
                   const float* coords, const float* charges, int n, double* result);

/* Drops every cached device copy made by the entry points above. */
void lkg_compat_cache_clear(void);

/* ---------------------------------------------------------------------- */
/* 2. Handle API                                                           */
/* ---------------------------------------------------------------------- */
typedef struct lkg_ctx lkg_ctx;

enum { LKG_PREC_FAST = 0,   /* f32 pair math, f64 transform and sums */
       LKG_PREC_EXACT = 1   /* f64 pair math in the reference's operation order */ };

/* One molecule, host arrays (borrowed for the call), f64 as the reference's
 * models hold them.  vdw = vdW well depth (vdw_charges); heavy = dna clash
 * flag; hyd = cpydock hydrogens array (1 = heavy; the exclusion mask is
 * derived from it as cpydock.rs:808-819 does); des/asa = cpydock desolvation
 * coefficient / reference ASA.  Unused arrays may be NULL. */
typedef struct {
    int32_t n;
    const double* coords;   /* n x 3 */
    const double* ele;
    const double* vdw;
    const double* radius;
    const uint8_t* heavy;
    const int32_t* hyd;
    const double* des;
    const double* asa;
} lkg_mol;

/* Receptor far field (optional, ReceptorField layout).  When NULL the
 * library builds it (bit-identical to grid_dna.rs:44-149). */
typedef struct {
    const float* phi;       /* nx*ny*nz, x fastest */
    int32_t nx, ny, nz;
    double ox, oy, oz, spacing;
} lkg_field;

int lkg_ctx_create(int device, lkg_ctx** out);
int lkg_ctx_destroy(lkg_ctx* ctx);
int lkg_ctx_set_precision(lkg_ctx* ctx, int precision);
/* Tile shape: ligand atoms per work unit (64, 128 or 256; default 128) and
 * the receptor cell edge in 1/1000 A (default: 4 A; 2.5 A for cpydock
 * complexes with groups of 32); 0 keeps the current value. */
int lkg_ctx_set_tiles(lkg_ctx* ctx, int threads_per_block, int cell_size_milli_angstrom);
/* Ligand atoms per candidate-search group of the warp kernel (4, 8, 16 or
 * 32; default 8); fixed once complexes exist. */
int lkg_ctx_set_group(lkg_ctx* ctx, int group);
/* x sub-cells per receptor cell edge (1..8; default 8, 4 for cpydock
 * complexes with groups of 32): the near scan trims each (z, y) cell row to
 * the 10 A sphere at this finer x resolution; fixed once complexes exist. */
int lkg_ctx_set_xsub(lkg_ctx* ctx, int xsub);
/* No counterpart in the reference (its cell list, gpu_score.rs:75-144, is
 * built on the host).  Where complex set-up sorts the receptor into its cell
 * grid and packs the sorted device arrays: 1 = on the GPU (the default:
 * counting sort, stable inside each cell), 0 = on the host.  Both give the
 * same arrays bit for bit; the host build is kept as the check. */
int lkg_ctx_set_setup(lkg_ctx* ctx, int on_device);
/* No counterpart in the reference (it reads receptor atoms one thread per
 * ligand atom, full_score.cu:279-319).  How the plain warp kernel brings the
 * receptor atoms of its candidate row spans in: 0 (default) = coalesced
 * float4 loads through L1, the next chunk of 32 fetched while the current
 * one is tested; 1 = windows of 64 atoms copied into shared memory by bulk
 * copies (cp.async.bulk, one per row span and window, completing on a
 * per-warp mbarrier).  Same scores bit for bit; kept as the measured
 * alternative. */
int lkg_ctx_set_staging(lkg_ctx* ctx, int tma);
/* Work on this CUDA stream (cudaStream_t) instead of the context's own. */
int lkg_ctx_set_stream(lkg_ctx* ctx, void* stream);
void* lkg_ctx_stream(lkg_ctx* ctx);

/* Upload one complex; returns its id in *complex_id. */
int lkg_complex_add(lkg_ctx* ctx, int family, const lkg_mol* receptor, const lkg_mol* ligand,
                    const lkg_field* field, int* complex_id);
/* Receptor / ligand atom counts and near-cell geometry of a complex. */
int lkg_complex_info(lkg_ctx* ctx, int complex_id, int* nr, int* nl, int* n_cells);

/* Active restraints and membrane of a complex, scored in the batch kernels
 * (the reference sends such runs to its CPU path: dna.rs:885-897,1047-1056,
 * pydock.rs:461-470, vdw.rs:262-272, cpydock.rs:690-700).
 *   rec_residue[i]: for receptor atom i (caller order), the index
 *     0..n_rec_res-1 of its active-restraint residue, or -1.  One index per
 *     key of the reference's `active_restraints` map (every index must have
 *     at least one atom, as the map's keys do); lig_residue likewise.
 *   membrane: receptor atom indices of the membrane beads (MMB.BJ,
 *     pydock.rs:77-80), each at most once.
 * A pair within INTERFACE_CUTOFF (3.9 A) marks both atoms as interface
 * atoms; per pose pr / pl = satisfied restraint residues / all (receptor /
 * ligand) and m = membrane beads at the interface / all (scoring.rs:83-108);
 * the score s becomes s + pr*s + pl*s - (m > 0 ? 999 m : 0) in the family's
 * operation order (dna.rs:989-995; vdw: no membrane term, vdw.rs:146-149).
 * The reference's passive restraints and ligand membrane do not enter the
 * score and are not taken.  All counts 0 clears the complex's restraints.
 * Plans made before the call must be made again. */
int lkg_complex_set_restraints(lkg_ctx* ctx, int complex_id, const int32_t* rec_residue, int n_rec_res,
                               const int32_t* lig_residue, int n_lig_res, const int32_t* membrane,
                               int n_membrane);

/* Score::batch_energy for one complex, host buffers: poses N x 7 -> scores.
 * parts (optional, N x 4): raw near+far electrostatics, LJ (+clash),
 * desolvation sum, near pairs (d <= 10 A) counted by the kernel. */
int lkg_score(lkg_ctx* ctx, int complex_id, int n_pose, const double* poses,
              double* scores, double* parts);

/* lkg_score plus the interface terms of every pose, host buffers:
 * iface N x 3 = (pr, pl, m) as above (zeros for a complex without
 * restraints or membrane). */
int lkg_score_interface(lkg_ctx* ctx, int complex_id, int n_pose, const double* poses, double* scores,
                        double* iface);

/* Device-pointer variant, asynchronous on the context stream. */
int lkg_score_device(lkg_ctx* ctx, int complex_id, int n_pose, const double* d_poses,
                     double* d_scores, double* d_parts);

/* Many complexes in one persistent launch.  For item i: complex ids[i],
 * counts[i] poses starting at pose offset sum(counts[:i]) of d_poses; scores
 * and parts use the same offsets.  Device pointers, asynchronous. */
int lkg_score_multi_device(lkg_ctx* ctx, int n_items, const int* complex_ids, const int* counts,
                           const double* d_poses, double* d_scores, double* d_parts);

/* Same batch with HOST buffers (synchronous): poses are copied to the
 * device (directly by DMA when the caller's buffer is page-locked), one
 * launch group scores every item, scores (and optional N x 4 parts) are
 * copied back. */
int lkg_score_multi(lkg_ctx* ctx, int n_items, const int* complex_ids, const int* counts,
                    const double* poses, double* scores, double* parts);

/* No counterpart in the reference.  lkg_score_device with no device
 * allocation, for callers that may not allocate while scoring (a framework
 * owning the device heap through its own pool, a latency-bound loop, code
 * where allocation calls are not allowed).  The fast tile kernel's scratch
 * lives in a fixed 8 MiB array inside liblkg (held on every GPU that loads
 * the library); a batch needing more (32 B per pose and ligand tile + 4 B
 * per pose rounded up to a multiple of 8 + 64 B) fails with
 * LKG_ERR_CAPACITY.  The first call on a device looks the array's address
 * up (cudaGetSymbolAddress) and keeps it: make that call before any stream
 * capture, and do not use the entry point across a cudaDeviceReset.  Each
 * call clears the counters it uses; calls overlapping on the GPU race on
 * the shared array.  The complex must be resident and already scored once
 * through a regular entry point; cpydock complexes and complexes with
 * restraints are refused.  Asynchronous on the context stream: lkg_ctx_sync
 * waits for it and reports the kernel's status word. */
int lkg_score_device_noalloc(lkg_ctx* ctx, int complex_id, int n_pose, const double* d_poses,
                             double* d_scores, double* d_parts);

/* Kernel launches made by this context so far (for launch accounting). */
int64_t lkg_ctx_launches(lkg_ctx* ctx);
/* Wait (bounded host poll) for the context stream and check the device
 * status words: the context's (LKG_ERR_CAPACITY after a desolvation-hash
 * overflow) and, after lkg_score_device_noalloc, that entry point's. */
int lkg_ctx_sync(lkg_ctx* ctx);

/* Plans: one batch (complexes x pose counts) prepared once — descriptors,
 * item tables and the plan's own scratch on the device — so that a launch
 * is kernel launches only.  lkg_plan_capture records n_launches launches
 * on the context stream into a CUDA graph; lkg_plan_replay launches it.
 * Adding complexes to the context afterwards invalidates the graph
 * (replay returns LKG_ERR_STATE).  Plans of one context must not run
 * concurrently with each other on different streams. */
typedef struct lkg_plan lkg_plan;
int lkg_plan_create(lkg_ctx* ctx, int n_items, const int* complex_ids, const int* counts, lkg_plan** out);
int lkg_plan_launch(lkg_plan* plan, const double* d_poses, double* d_scores, double* d_parts);
int lkg_plan_capture(lkg_plan* plan, const double* d_poses, double* d_scores, double* d_parts, int n_launches);
int lkg_plan_replay(lkg_plan* plan);
int lkg_plan_sync(lkg_plan* plan);
int lkg_plan_destroy(lkg_plan* plan);

/* ---------------------------------------------------------------------- */
/* Learned surrogate of the pose energy (no counterpart in the reference)  */
/* ---------------------------------------------------------------------- */
/* 64 -> 256 -> 256 -> 256 -> 1 ReLU MLP, BF16 weights and activations with
 * FP32 accumulation on the tensor cores, trained online on exact scores.
 * Features: pose quaternion, translation / box scale, and at 16 ligand anchor
 * atoms (farthest-point sampled) the far-field potential and receptor atom
 * counts from the fine cell grid.  Target: asinh(score / s) standardised
 * (lkg_surrogate_set_target_scale fits s, mean and spread). */
typedef struct lkg_surrogate lkg_surrogate;
int lkg_surrogate_create(lkg_ctx* ctx, int complex_id, uint64_t seed, lkg_surrogate** out);
int lkg_surrogate_destroy(lkg_surrogate* s);
int lkg_surrogate_set_target_scale(lkg_surrogate* s, int n, const double* scores);
/* predicted scores (lkg_score units) for n device poses, device output */
int lkg_surrogate_predict(lkg_surrogate* s, int n, const double* d_poses, double* d_pred);
/* Allocate the activation buffers for predictions of up to n_predict poses
 * per call and training batches of train_batch rows now (growing them
 * later reallocates, which synchronises the device). */
int lkg_surrogate_reserve(lkg_surrogate* s, int n_predict, int train_batch);
/* minibatch Adam over n device poses with their exact scores (device) */
int lkg_surrogate_train(lkg_surrogate* s, int n, const double* d_poses, const double* d_scores, int epochs,
                        int batch, float lr, float* loss);
int64_t lkg_surrogate_nparams(void);
int lkg_surrogate_get_params(lkg_surrogate* s, float* out);
int lkg_surrogate_set_params(lkg_surrogate* s, const float* in);
/* one forward + backward on host feature rows (bf16 bits) and standardised
 * targets: outputs, flat FP32 gradient, loss (for gradient checks) */
int lkg_surrogate_grad(lkg_surrogate* s, int n, const uint16_t* feats, const float* targets, float* y,
                       float* grad, float* loss);
int lkg_surrogate_features(lkg_surrogate* s, int n, const double* d_poses, uint16_t* out);
/* forward layers on the tcgen05 tensor cores (TMEM accumulators; 1,
 * default) or on the mma.sync kernel (0) */
int lkg_surrogate_set_backend(lkg_surrogate* s, int tcgen05);
/* kernel status bits since the last call (4: a tcgen05 accumulator wait ran
 * out and that tile was skipped); cleared by the call */
int lkg_surrogate_status(lkg_surrogate* s, int* bits);

/* ---------------------------------------------------------------------- */
/* Setup helpers (host)                                                    */
/* ---------------------------------------------------------------------- */
/* Receptor far field, bit-identical to ReceptorField::build
 * (grid_dna.rs:44-149).  Query dims with phi == NULL. */
int lkg_field_build(const double* coords, const double* charges, int32_t n,
                    double origin[3], int32_t dims[3], double* spacing, float* phi);
/* Lower bound of the distance from each of m points (x, y, z) to the
 * nearest of n receptor atoms, as the warp kernels use it to skip ligand
 * groups that no receptor atom can reach (a 2 A grid over the receptor's
 * box grown by 24 A; 24 outside it).  No counterpart in the reference. */
int lkg_receptor_distance_bound(const double* coords, int32_t n, const double* points, int32_t m, float* out);
/* Lee & Richards SASA, probe 1.4, 20 slices (lr_sasa.rs:277-291). */
int lkg_lr_sasa(const double* coords, const double* radii, int32_t n, double* out);
/* Self-avoiding random chain for synthetic receptors (see lkg_setup.cpp). */
int lkg_synth_chain(uint64_t seed, int32_t n, double r0, double bond, double min_sep, int32_t patience,
                    double* coords, double* r_final);

/* rand 0.7.3 StdRng::seed_from_u64 stream (Rng::gen::<f64>) for callers
 * that reproduce the reference's setup poses and GSO draws. */
void* lkg_rng_new(uint64_t seed);
double lkg_rng_f64(void* rng);
void lkg_rng_free(void* rng);

/* ---------------------------------------------------------------------- */
/* GSO driver (GSO::run, lib.rs:66-78; Swarm / Glowworm, swarm.rs,         */
/* glowworm.rs) over the batched scorer                                    */
/* ---------------------------------------------------------------------- */
typedef struct lkg_gso lkg_gso;
/* n_groups groups of (complex, n_swarms[g] swarms x n_glow[g] glowworms);
 * positions: all glowworms in group, swarm, glowworm order, 7 doubles each
 * as initial_positions_*.dat holds them (tx ty tz qw qx qy qz); every swarm
 * of group g draws from StdRng::seed_from_u64(seeds[g]). */
int lkg_gso_create(lkg_ctx* ctx, int n_groups, const int* complex_ids, const int* n_swarms,
                   const int* n_glow, const double* positions, const uint64_t* seeds, lkg_gso** out);
/* steps x (score moved glowworms of all swarms in one launch group; move) */
int lkg_gso_run(lkg_gso* gso, int steps);
/* The same GSO steps with the whole step on the device (no counterpart in
 * the reference): scoring, luciferin, neighbour selection (the swarm's
 * StdRng stream, drawn on the device) and movement as kernel launches
 * replayed from one CUDA graph.  Its f64 arithmetic is the host GSO's
 * except acos / sin in the slerp (device library), so runs agree closely at
 * first and then drift apart.  On a screened GSO (lkg_gso_set_screen) the
 * training steps are plain device steps whose exact pairs train the
 * surrogates, and the screened steps after them run on the device too
 * (candidates, predictions, the exact choice, the move; a full rescoring
 * fine-tunes from the host); the no-network ablation is refused
 * (LKG_ERR_STATE).  Host and device steps can be mixed. */
int lkg_gso_run_device(lkg_gso* gso, int steps);
int lkg_gso_state(lkg_gso* gso, double* trans, double* rot, double* luc, double* scoring,
                  double* vision, int32_t* nneigh);
int64_t lkg_gso_scored(lkg_gso* gso);
/* Swarm::save (swarm.rs:232-271): write swarm `swarm` (index over all
 * groups, in creation order) as <directory>/gso_<step>.out in the
 * reference's format (what `lklight rank` and `generate` read). */
int lkg_gso_save(lkg_gso* gso, int swarm, int step, const char* directory);
int lkg_gso_destroy(lkg_gso* gso);

/* Surrogate screening of GSO moves (no counterpart in the reference; the
 * plain run above stays the reference GSO).  The first train_steps steps run
 * plainly and their exact energies train one surrogate per group; from then
 * on every glowworm with neighbours draws `candidates` moves from its
 * neighbour distribution, the surrogate ranks them, the glowworm takes the
 * best, and per swarm the exact_fraction of moves with the largest
 * predicted change |gain| is scored exactly (the others keep their last exact score,
 * or with carry_prediction = 1 take it plus the predicted gain); every
 * rescore_every steps all glowworms are rescored exactly and the surrogate
 * is fine-tuned on them.  random_rank = 1 is the same search without the
 * network (seeded random ranks; unscored moves keep their previous score),
 * for ablations. */
typedef struct {
    int32_t candidates;       /* moves screened per glowworm (4) */
    double exact_fraction;    /* fraction of moves per swarm scored exactly (0.25) */
    int32_t rescore_every;    /* full exact rescoring period in steps (10; 0 = never) */
    int32_t train_steps;      /* plain steps whose energies train the surrogate (20) */
    int32_t train_epochs;     /* epochs of the first training */
    int32_t finetune_epochs;  /* epochs at every full rescoring */
    float lr;                 /* Adam learning rate */
    uint64_t seed;            /* surrogate initialisation, shuffles, ablation ranks */
    int32_t random_rank;
    int32_t batch;            /* training minibatch (1024; 0 = 1024) */
    int32_t carry_prediction; /* 1: unscored moves score current + predicted gain (0) */
} lkg_screen;
int lkg_gso_set_screen(lkg_gso* gso, const lkg_screen* cfg);
/* exact rescoring of every glowworm (the final poses of a screened run) */
int lkg_gso_finalize(lkg_gso* gso);
int64_t lkg_gso_predicted(lkg_gso* gso);
/* wall seconds so far in: out[0] exact scoring (launch, copies, wait),
 * out[1] host movement, out[2] surrogate inference, out[3] training */
int lkg_gso_timing(lkg_gso* gso, double* out);

#ifdef __cplusplus
}
#endif
#endif
