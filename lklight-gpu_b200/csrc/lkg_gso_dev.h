// Device-resident state of a GSO run (structure of arrays over all
// glowworms of all swarms, swarms in group order) and the kernels of one
// step after scoring.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace lkg {

struct GsoDevState {
    int n, n_swarms, max_swarm;
    int reserved;                  // keeps the struct free of padding (it is compared bytewise)
    double *tx, *ty, *tz, *qw, *qx, *qy, *qz, *luc, *vis, *score;   // current state
    double *ntx, *nty, *ntz, *nqw, *nqx, *nqy, *nqz, *nvis;          // after the move
    double* poses;                 // scorer input, n x 7 (w, x, y, z, tx, ty, tz)
    int *nid, *nnb;                // selected neighbour (index in the swarm), neighbour count
    const int *swarm_first, *swarm_n, *swarm_of;
    const uint32_t* keys;          // 8 ChaCha key words per swarm
    unsigned long long* draws;     // 64-bit draws consumed per swarm
    unsigned char* mask;           // 1: pose to score this step (moved, or never scored)
    unsigned long long* nscored;   // poses scored so far
};

// luciferin update, selection, movement and commit of one step, given the
// step's scores in S.score
cudaError_t gso_dev_after_scoring(const GsoDevState& S, cudaStream_t s);

// Screened steps: K candidate moves per glowworm (row 0 of a glowworm's
// K + 1 candidate rows is its current pose), ranked by surrogate
// predictions, the exact fraction with the largest predicted gain per
// swarm scored exactly in the next step
struct GsoDevScreen {
    int K;                   // candidates per glowworm
    int carry;               // 1: unscored moves take current + gain (also keeps the struct free of padding)
    double frac;             // exact fraction per swarm
    double* cand;            // n x (K + 1) x 7 candidate poses (w, x, y, z, tx, ty, tz)
    double* pred;            // n x (K + 1) predicted scores
    int* knid;               // n x K selected neighbour per candidate (index in the swarm)
    int* best;               // n: chosen candidate row (1..K), 0 without neighbours
    double* gain;            // n: prediction at the chosen move minus at the current pose
    unsigned char* exact;    // n: the move is scored exactly in the next step
    unsigned char* pend;     // n: score += gain before the next luciferin update (carry only)
};

// luciferin update (with the pending predicted scores), K selections per
// glowworm and the candidate rows, given the step's exact scores in S.score
cudaError_t gso_dev_screen_propose(const GsoDevState& S, const GsoDevScreen& X, cudaStream_t s);
// best candidate, per-swarm exact selection and the move, given X.pred
cudaError_t gso_dev_screen_move(const GsoDevState& S, const GsoDevScreen& X, cudaStream_t s);

}  // namespace lkg
