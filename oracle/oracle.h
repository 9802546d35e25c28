/* Oracle for the lkg parity tests: a CPU restatement of LKlight's CPU grid
 * scoring path, its GSO driver and its random-number stream.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product library links, loads or
 * calls this code; only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline use it, and only as the checker or as the timed CPU reference.
 *
 * Every routine cites the reference function it restates (paths are relative
 * to the LKlight-GPU source tree).  Pinned against the reference's own
 * known-answer tests (1AZP pydock/dna/vdw/cpydock, the far-field unit charge,
 * the cell-list all-pairs equivalence, the seeded quaternion) in
 * tests/test_oracle.py.
 */
#ifndef LKG_ORACLE_H
#define LKG_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* family ids (same numbering as the product library) */
enum { ORC_DNA = 0, ORC_VDW = 1, ORC_PYDOCK = 2, ORC_CPYDOCK = 3 };

/* rand 0.7.3 StdRng (ChaCha20, seed_from_u64 via PCG32) */
void*  orc_rng_new(uint64_t seed);
void   orc_rng_free(void* rng);
double orc_rng_f64(void* rng);          /* Rng::gen::<f64>() */
uint64_t orc_rng_u64(void* rng);

/* synthetic receptor chain of the benchmark inputs (the generator liblkg's
 * lkg_synth_chain runs, restated so that the CPU reference arm makes its
 * inputs without the product library); 0 = ok, -1 = bad arguments or no fit */
int orc_synth_chain(uint64_t seed, int32_t n, double r0, double bond, double min_sep, int32_t patience,
                    double* coords, double* r_final);

/* Lee & Richards SASA (src/lr_sasa.rs: probe 1.4 A, 20 slices): per-atom
 * areas of n atoms with bare radii `radii` */
void orc_lr_sasa(const double* coords, const double* radii, int32_t n, double* out);

/* quaternions (src/qt.rs) */
void orc_quat_random(void* rng, double out[4]);                       /* qt.rs:106-117 */
void orc_quat_slerp(const double a[4], const double b[4], double t, double out[4]); /* qt.rs:80-104 */
void orc_quat_normalize(double q[4]);                                 /* qt.rs:40-46 */

/* receptor far field (src/grid_dna.rs).  fp64 != 0 accumulates and stores
 * phi in double (the "FP64 evaluation of the same function"). */
void*  orc_field_new(const double* coords, const double* q, int64_t n, int fp64);
/* the same field by the plain single-threaded per-atom scatter (the check
 * of orc_field_new's parallel brick order) */
void*  orc_field_new_scatter(const double* coords, const double* q, int64_t n, int fp64);
void   orc_field_info(const void* f, double origin[3], int64_t dims[3], double* spacing);
const float*  orc_field_phi32(const void* f);
const double* orc_field_phi64(const void* f);
double orc_field_sample(const void* f, double x, double y, double z);
void   orc_field_free(void* f);

/* GPU-bridge receptor cell list (src/gpu_score.rs:75-144): 10 A cells,
 * origin floor(min - 0.01).  Returns the cell_start length
 * ((ncx+1)(ncy+1)(ncz+1) + 1); cell_start/cell_atoms may be NULL to query. */
int64_t orc_crec_build(const double* coords, int64_t n, int32_t nc[3], float origin[3],
                       float* cell_sp, int32_t* cell_start, int32_t* cell_atoms);

/* NearCells (src/nearcell.rs) all-pairs equivalence helper: number of
 * distinct pairs (i<j) within `cell` found through the 27-cell stencil. */
int64_t orc_nearcell_pair_count(const double* coords, int64_t n, double cell);
int64_t orc_allpairs_count(const double* coords, int64_t n, double cut);

/* scoring model: per-atom f64 arrays.  `vdw` is the vdW well depth (the
 * reference's vdw_charges); sqrt is taken inside as the reference does.
 * heavy: dna clash flag; hyd: cpydock hydrogens flag (1 = heavy); des/asa:
 * cpydock desolvation coefficient / reference ASA.  Unused arrays may be NULL. */
void* orc_model_new(int family,
                    int64_t nr, const double* rc, const double* rq, const double* rvdw,
                    const double* rrad, const uint8_t* rheavy, const int32_t* rhyd,
                    const double* rdes, const double* rasa,
                    int64_t nl, const double* lc, const double* lq, const double* lvdw,
                    const double* lrad, const uint8_t* lheavy, const int32_t* lhyd,
                    const double* ldes, const double* lasa);
void  orc_model_free(void* m);
/* build (and cache) the model's far field now; returns its handle */
const void* orc_model_field(void* m, int fp64);

/* Score::energy_grid for one pose (t = translation, q = w,x,y,z).
 * parts (may be NULL) receives {e_near_raw, e_far_raw, vdw, solv, near_pairs}. */
double orc_energy_grid(void* m, const double t[3], const double q[4], int fp64, double parts[5]);
/* Active restraints and membrane (dna.rs:885-897,970-995, pydock.rs:427-445,
 * vdw.rs:139-149, cpydock.rs:639-675, scoring.rs:83-108): restraint residue
 * index per atom (-1 = none; n x 1, NULL when the count is 0) and the
 * receptor atom indices of the membrane beads.  energy_grid then applies the
 * restraint fractions and the membrane penalty. */
void orc_model_set_restraints(void* m, const int32_t* rec_res, int nres_r, const int32_t* lig_res, int nres_l,
                              const int32_t* membrane, int64_t n_membrane);
/* batch with the interface terms per pose (iface N x 3: pr, pl, membrane
 * intersection; may be NULL) */
void orc_batch_energy_grid_iface(void* m, int64_t N, const double* poses, int fp64, int threads,
                                 double* out, double* iface);
/* energy_exact (all-pairs reference path) */
double orc_energy_exact(void* m, const double t[3], const double q[4]);
/* batch of poses, N x 7 in the reference's kernel order (w,x,y,z,tx,ty,tz);
 * OpenMP over poses with `threads` threads (<= 0: all).  parts N x 5 or NULL. */
void orc_batch_energy_grid(void* m, int64_t N, const double* poses, int fp64, int threads,
                           double* out, double* parts);

/* GSO (src/lib.rs, src/swarm.rs, src/glowworm.rs).  positions: n x 7 rows of
 * (tx, ty, tz, qw, qx, qy, qz), as initial_positions_*.dat holds them. */
void* orc_gso_new(void* model, int64_t n, const double* positions, uint64_t seed, int fp64, int threads);
void  orc_gso_run(void* g, int steps);
/* trans n x 3, rot n x 4, luc/scoring/vision n, nneigh n, moved n (any may be NULL) */
void  orc_gso_state(const void* g, double* trans, double* rot, double* luc, double* scoring,
                    double* vision, int32_t* nneigh, uint8_t* moved);
int64_t orc_gso_scored(const void* g);   /* poses scored so far */
void  orc_gso_free(void* g);

#ifdef __cplusplus
}
#endif
#endif
