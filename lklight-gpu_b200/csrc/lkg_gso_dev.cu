// Device-resident GSO step (plain GSO only): luciferin update, neighbour
// selection and movement of every glowworm of every swarm on the GPU, so
// that one whole GSO step (score, luciferin, select, move) is a sequence of
// kernel launches that a CUDA graph replays.
//
// The arithmetic follows the host GSO (swarm.rs:96-174, glowworm.rs:84-166)
// operation by operation and this file is compiled without FMA contraction,
// so every f64 result matches the host's except the slerp: its acos / sin
// come from the device math library instead of glibc, which can differ in
// the last place; trajectories therefore agree closely for a few steps and
// then drift apart as chaotic runs do.  The host GSO stays the parity mode.
//
// Random numbers: the swarm's StdRng stream (ChaCha20, 64-bit counter) is
// counter-based, so draw i of swarm s is computed directly from block i / 8
// of the swarm's keystream (words 2i, 2i + 1: every GSO draw is a 64-bit
// draw, so draws never straddle a word pair).
#include <algorithm>
#include <cstdint>

#include "lkg_gso_dev.h"

namespace lkg {
namespace {

constexpr double RHO = 0.5, GAMMA = 0.4, BETA = 0.08, MAX_VISION = 5.0;
constexpr int MAX_NEIGHBORS = 5;

__device__ __forceinline__ uint32_t rotl32(uint32_t v, int c) { return (v << c) | (v >> (32 - c)); }

// draw `i` of the stream with key k (gen::<f64>: top 53 bits of the u64
// whose low word comes first)
__device__ double chacha_f64(const uint32_t* __restrict__ k, unsigned long long i) {
    const unsigned long long blk = i >> 3;
    uint32_t s[16] = {0x61707865u, 0x3320646eu, 0x79622d32u, 0x6b206574u, k[0], k[1], k[2], k[3],
                      k[4], k[5], k[6], k[7], (uint32_t)blk, (uint32_t)(blk >> 32), 0u, 0u};
    uint32_t x[16];
#pragma unroll
    for (int j = 0; j < 16; ++j) x[j] = s[j];
#define QR(a, b, c, d)                              \
    x[a] += x[b]; x[d] = rotl32(x[d] ^ x[a], 16);   \
    x[c] += x[d]; x[b] = rotl32(x[b] ^ x[c], 12);   \
    x[a] += x[b]; x[d] = rotl32(x[d] ^ x[a], 8);    \
    x[c] += x[d]; x[b] = rotl32(x[b] ^ x[c], 7);
    for (int r = 0; r < 10; ++r) {
        QR(0, 4, 8, 12) QR(1, 5, 9, 13) QR(2, 6, 10, 14) QR(3, 7, 11, 15)
        QR(0, 5, 10, 15) QR(1, 6, 11, 12) QR(2, 7, 8, 13) QR(3, 4, 9, 14)
    }
#undef QR
    const int w = (int)(i & 7) * 2;
    uint32_t lo = 0, hi = 0;
#pragma unroll
    for (int j = 0; j < 16; ++j) {
        if (j == w) lo = x[j] + s[j];
        if (j == w + 1) hi = x[j] + s[j];
    }
    const unsigned long long v = ((unsigned long long)hi << 32) | lo;
    return (double)(v >> 11) * (1.0 / 9007199254740992.0);
}

// luciferin update with this step's scores (swarm.rs:96-99); unmoved
// glowworms were not rescored and keep their score (swarm.rs:79-85)
__global__ void k_gso_luciferin(GsoDevState S) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool scored = i < S.n && S.mask[i];
    const unsigned b = __ballot_sync(0xffffffffu, scored);
    if ((threadIdx.x & 31) == 0 && b) atomicAdd(S.nscored, (unsigned long long)__popc(b));
    if (i >= S.n) return;
    S.luc[i] = (1.0 - RHO) * S.luc[i] + GAMMA * S.score[i];
}

// neighbours (brighter, within the vision range, in id order) and K
// roulette selections with the glowworm's draws li*K .. li*K + K - 1 of the
// step (glowworm.rs:114-142); out[i*K + k]: the selected neighbour (index
// in the swarm, the glowworm itself when it has none).
//
// One warp per glowworm.  The lanes test 32 swarm members at a time (the
// exact f64 test of the host); the neighbours of a chunk (a ballot) are then
// walked in id order with every lane doing the same f64 additions, so the
// total and the running sum are the host's, bit for bit.  Lane k keeps draw
// k (and k + 32): the roulette for a draw stops at the first neighbour whose
// running sum before it is not below the draw, as the host's loop does; the
// sums of the draws agree until they stop, so one running sum serves all.
__global__ void k_gso_select(GsoDevState S, int K, int* __restrict__ out) {
    const int lane = threadIdx.x & 31;
    const int i = (int)((blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5);
    if (i >= S.n) return;   // warp-uniform
    const int sw = S.swarm_of[i];
    const int first = S.swarm_first[sw], n = S.swarm_n[sw], li = i - first;
    const double x = S.tx[i], y = S.ty[i], z = S.tz[i], l1 = S.luc[i], v = S.vis[i];
    const double vr2 = v * v;
    // pass 1: count and total of the luciferin differences, id order
    int cnt = 0;
    double total = 0.0;
    for (int j0 = 0; j0 < n; j0 += 32) {
        const int jl = j0 + lane;
        bool nb = false;
        double lj = 0.0;
        if (jl < n) {
            const int j = first + jl;
            const double dx = x - S.tx[j], dy = y - S.ty[j], dz = z - S.tz[j];
            lj = S.luc[j];
            nb = jl != li && l1 < lj && dx * dx + dy * dy + dz * dz < vr2;
        }
        unsigned m = __ballot_sync(0xffffffffu, nb);
        cnt += __popc(m);
        while (m) {
            const int b = __ffs(m) - 1;
            m &= m - 1;
            total += __shfl_sync(0xffffffffu, lj, b) - l1;
        }
    }
    // pass 2: the roulettes over prob = (l_j - l_i) / total in id order
    const unsigned long long d0 = S.draws[sw] + (unsigned long long)li * K;
    const double u0 = lane < K ? chacha_f64(S.keys + 8 * sw, d0 + lane) : 0.0;
    const double u1 = lane + 32 < K ? chacha_f64(S.keys + 8 * sw, d0 + lane + 32) : 0.0;
    int sel0 = -1, sel1 = -1, firstnb = -1;
    bool stop0 = lane >= K, stop1 = lane + 32 >= K;
    double sum = 0.0;
    for (int j0 = 0; j0 < n && cnt > 0 && !__all_sync(0xffffffffu, stop0 && stop1); j0 += 32) {
        const int jl = j0 + lane;
        bool nb = false;
        double lj = 0.0;
        if (jl < n) {
            const int j = first + jl;
            const double dx = x - S.tx[j], dy = y - S.ty[j], dz = z - S.tz[j];
            lj = S.luc[j];
            nb = jl != li && l1 < lj && dx * dx + dy * dy + dz * dz < vr2;
        }
        unsigned m = __ballot_sync(0xffffffffu, nb);
        while (m) {
            const int b = __ffs(m) - 1;
            m &= m - 1;
            const int jn = j0 + b;
            const double p = (__shfl_sync(0xffffffffu, lj, b) - l1) / total;
            if (firstnb < 0) firstnb = jn;
            if (!stop0) { if (sum < u0) sel0 = jn; else stop0 = true; }
            if (!stop1) { if (sum < u1) sel1 = jn; else stop1 = true; }
            sum += p;
        }
    }
    int* o = out + (size_t)i * K;
    if (lane < K) o[lane] = cnt == 0 ? li : (sel0 >= 0 ? sel0 : firstnb);
    if (lane + 32 < K) o[lane + 32] = cnt == 0 ? li : (sel1 >= 0 ? sel1 : firstnb);
    if (lane == 0) S.nnb[i] = cnt;
}

__device__ __forceinline__ void qnorm(double& w, double& x, double& y, double& z) {   // qt.rs:36-46
    const double n = sqrt(w * w + x * x + y * y + z * z);
    w /= n; x /= n; y /= n; z /= n;
}

// pose of glowworm i after a move towards glowworm nid (glowworm.rs:144-166,
// qt.rs:80-104), from the step's starting state; nid == i: unchanged
__device__ void moved_pose(const GsoDevState& S, int i, int nid, double& tx, double& ty, double& tz, double& w,
                           double& x, double& y, double& z) {
    tx = S.tx[i]; ty = S.ty[i]; tz = S.tz[i];
    w = S.qw[i]; x = S.qx[i]; y = S.qy[i]; z = S.qz[i];
    if (nid != i) {
        const double dx = S.tx[nid] - tx, dy = S.ty[nid] - ty, dz = S.tz[nid] - tz;
        const double norm = sqrt(dx * dx + dy * dy + dz * dz);
        const double coef = 0.5 / norm;
        tx += dx * coef; ty += dy * coef; tz += dz * coef;
        double w2 = S.qw[nid], x2 = S.qx[nid], y2 = S.qy[nid], z2 = S.qz[nid];
        qnorm(w, x, y, z);
        qnorm(w2, x2, y2, z2);
        double dot = w * w2 + x * x2 + y * y2 + z * z2;
        if (dot < 0.0) { w = -w; x = -x; y = -y; z = -z; dot *= -1.0; }
        if (dot > 0.9995) {
            w = w + (w2 - w) * 0.5; x = x + (x2 - x) * 0.5; y = y + (y2 - y) * 0.5; z = z + (z2 - z) * 0.5;
            qnorm(w, x, y, z);
        } else {
            dot = fmax(fmin(dot, 1.0), -1.0);
            const double omega = acos(dot), so = sin(omega);
            const double a = sin((1.0 - 0.5) * omega) / so, b = sin(0.5 * omega) / so;
            w = w * a + w2 * b; x = x * a + x2 * b; y = y * a + y2 * b; z = z * a + z2 * b;
        }
        qnorm(w, x, y, z);
    }
}

__device__ __forceinline__ double new_vision(const GsoDevState& S, int i) {
    const double v = S.vis[i] + BETA * (double)(MAX_NEIGHBORS - S.nnb[i]);
    return fmin(MAX_VISION, fmax(0.0, v));
}

// movement towards the selected neighbour and vision update; reads the
// step's starting state, writes the new one into the second buffer
__global__ void k_gso_move(GsoDevState S) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= S.n) return;
    const int sw = S.swarm_of[i];
    const int nid = S.swarm_first[sw] + S.nid[i];
    double tx, ty, tz, w, x, y, z;
    moved_pose(S, i, nid, tx, ty, tz, w, x, y, z);
    S.ntx[i] = tx; S.nty[i] = ty; S.ntz[i] = tz;
    S.nqw[i] = w; S.nqx[i] = x; S.nqy[i] = y; S.nqz[i] = z;
    S.nvis[i] = new_vision(S, i);
    S.mask[i] = nid != i;   // the next step scores the moved glowworms
}

// the new state becomes current; scorer poses (w, x, y, z, tx, ty, tz);
// each swarm's draw counter advances by its size
__global__ void k_gso_commit(GsoDevState S) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < S.n_swarms) S.draws[i] += (unsigned long long)S.swarm_n[i];
    if (i >= S.n) return;
    S.tx[i] = S.ntx[i]; S.ty[i] = S.nty[i]; S.tz[i] = S.ntz[i];
    S.qw[i] = S.nqw[i]; S.qx[i] = S.nqx[i]; S.qy[i] = S.nqy[i]; S.qz[i] = S.nqz[i];
    S.vis[i] = S.nvis[i];
    double* p = S.poses + 7 * (size_t)i;
    p[0] = S.qw[i]; p[1] = S.qx[i]; p[2] = S.qy[i]; p[3] = S.qz[i];
    p[4] = S.tx[i]; p[5] = S.ty[i]; p[6] = S.tz[i];
}

// ---------------------------------------------------------------------------
// screened steps (lkg_gso.cpp screened_movement, the same operations)
// ---------------------------------------------------------------------------

// with X.carry, moves left unscored take their predicted score (current +
// predicted gain) before the luciferin update; without it they keep their
// last exact score.  The exact ones were scored this step
__global__ void k_gso_luciferin_screened(GsoDevState S, GsoDevScreen X) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool scored = i < S.n && S.mask[i];
    const unsigned b = __ballot_sync(0xffffffffu, scored);
    if ((threadIdx.x & 31) == 0 && b) atomicAdd(S.nscored, (unsigned long long)__popc(b));
    if (i >= S.n) return;
    if (X.pend[i]) {   // a full rescoring step scored it exactly instead
        if (!S.mask[i]) S.score[i] = S.score[i] + X.gain[i];
        X.pend[i] = 0;
    }
    S.luc[i] = (1.0 - RHO) * S.luc[i] + GAMMA * S.score[i];
}

// candidate rows of glowworm i: its current pose, then the K moves (all
// rows the current pose when it has no neighbours); the new vision range
__global__ void k_gso_cand(GsoDevState S, GsoDevScreen X) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= S.n) return;
    const int K = X.K, first = S.swarm_first[S.swarm_of[i]];
    double* row = X.cand + (size_t)i * (K + 1) * 7;
    const double cur[7] = {S.qw[i], S.qx[i], S.qy[i], S.qz[i], S.tx[i], S.ty[i], S.tz[i]};
    for (int c = 0; c < 7; ++c) row[c] = cur[c];
    for (int k = 0; k < K; ++k) {
        double* r = row + 7 * (k + 1);
        if (S.nnb[i] > 0) {
            double tx, ty, tz, w, x, y, z;
            moved_pose(S, i, first + X.knid[(size_t)i * K + k], tx, ty, tz, w, x, y, z);
            r[0] = w; r[1] = x; r[2] = y; r[3] = z; r[4] = tx; r[5] = ty; r[6] = tz;
        } else {
            for (int c = 0; c < 7; ++c) r[c] = cur[c];
        }
    }
    S.nvis[i] = new_vision(S, i);
}

// the best predicted move (first maximum over rows 1..K) and its gain over
// the current pose
__global__ void k_gso_best(GsoDevState S, GsoDevScreen X) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= S.n) return;
    const int K = X.K;
    const double* p = X.pred + (size_t)i * (K + 1);
    if (S.nnb[i] == 0) { X.best[i] = 0; X.gain[i] = 0.0; return; }
    int best = 1;
    for (int c = 2; c <= K; ++c)
        if (p[c] > p[best]) best = c;
    X.best[i] = best;
    X.gain[i] = p[best] - p[0];
}

// per swarm, the ceil(frac * movers) movers with the largest |gain| (ties:
// the lower id first) are scored exactly (the host GSO's rule).  One warp per glowworm counts, 32
// swarm members at a time, the movers and the movers ranked ahead of it.
__global__ void k_gso_rank(GsoDevState S, GsoDevScreen X) {
    const int lane = threadIdx.x & 31;
    const int i = (int)((blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5);
    if (i >= S.n) return;   // warp-uniform
    const int sw = S.swarm_of[i];
    const int first = S.swarm_first[sw], n = S.swarm_n[sw], li = i - first;
    const bool mine = S.nnb[i] > 0;
    const double gi = fabs(X.gain[i]);
    int movers = 0, ahead = 0;
    for (int j0 = 0; j0 < n; j0 += 32) {
        const int jl = j0 + lane;
        bool mv = false, up = false;
        if (jl < n) {
            const int j = first + jl;
            mv = S.nnb[j] > 0;
            const double gj = fabs(X.gain[j]);
            up = mv && (gj > gi || (gj == gi && jl < li));
        }
        movers += __popc(__ballot_sync(0xffffffffu, mv));
        ahead += __popc(__ballot_sync(0xffffffffu, up));
    }
    const int nx = (int)ceil(X.frac * (double)movers);
    if (lane == 0) X.exact[i] = mine && ahead < nx;
}

// every glowworm with neighbours takes its best candidate; the exact ones
// are scored next step, the others (with X.carry) take current + gain
// before the next luciferin update; the swarm's draw counter advances by K
// per glowworm
__global__ void k_gso_commit_screened(GsoDevState S, GsoDevScreen X) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < S.n_swarms) S.draws[i] += (unsigned long long)X.K * S.swarm_n[i];
    if (i >= S.n) return;
    const bool moved = S.nnb[i] > 0;
    if (moved) {
        const double* r = X.cand + ((size_t)i * (X.K + 1) + X.best[i]) * 7;
        S.qw[i] = r[0]; S.qx[i] = r[1]; S.qy[i] = r[2]; S.qz[i] = r[3];
        S.tx[i] = r[4]; S.ty[i] = r[5]; S.tz[i] = r[6];
    }
    S.vis[i] = S.nvis[i];
    S.mask[i] = moved && X.exact[i];
    X.pend[i] = X.carry && moved && !X.exact[i];
    double* p = S.poses + 7 * (size_t)i;
    p[0] = S.qw[i]; p[1] = S.qx[i]; p[2] = S.qy[i]; p[3] = S.qz[i];
    p[4] = S.tx[i]; p[5] = S.ty[i]; p[6] = S.tz[i];
}

}  // namespace

cudaError_t gso_dev_screen_propose(const GsoDevState& S, const GsoDevScreen& X, cudaStream_t s) {
    const int t = 256, b = (S.n + t - 1) / t;
    k_gso_luciferin_screened<<<b, t, 0, s>>>(S, X);
    const int wb = (int)(((size_t)S.n * 32 + 255) / 256);   // one warp per glowworm
    k_gso_select<<<wb, 256, 0, s>>>(S, X.K, X.knid);
    k_gso_cand<<<b, t, 0, s>>>(S, X);
    return cudaGetLastError();
}

cudaError_t gso_dev_screen_move(const GsoDevState& S, const GsoDevScreen& X, cudaStream_t s) {
    const int t = 256, b = (S.n + t - 1) / t;
    k_gso_best<<<b, t, 0, s>>>(S, X);
    k_gso_rank<<<(int)(((size_t)S.n * 32 + 255) / 256), 256, 0, s>>>(S, X);
    k_gso_commit_screened<<<(std::max(S.n, S.n_swarms) + t - 1) / t, t, 0, s>>>(S, X);
    return cudaGetLastError();
}

cudaError_t gso_dev_after_scoring(const GsoDevState& S, cudaStream_t s) {
    const int t = 256, b = (S.n + t - 1) / t;   // full warps: the ballot in k_gso_luciferin
    k_gso_luciferin<<<b, t, 0, s>>>(S);
    k_gso_select<<<(int)(((size_t)S.n * 32 + 255) / 256), 256, 0, s>>>(S, 1, S.nid);   // a warp per glowworm
    k_gso_move<<<b, t, 0, s>>>(S);
    k_gso_commit<<<(std::max(S.n, S.n_swarms) + t - 1) / t, t, 0, s>>>(S);
    return cudaGetLastError();
}

}  // namespace lkg
