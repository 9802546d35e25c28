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

}  // namespace lkg
