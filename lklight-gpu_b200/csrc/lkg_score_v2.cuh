// Warp-cooperative fused scorer (f32 fast path, dna / pydock / vdw and the
// reference-compatible flag combinations).
//
// A work unit is a tile of TILE ligand atoms of one pose.  The tile is split
// into groups of G consecutive (Morton-ordered, hence compact) ligand atoms
// whose bounding sphere in the ligand frame (centre, radius rho) is computed
// on the host; the warps of the block take the groups in turn.  Per group:
//   1. lanes 0..G-1 transform their ligand atom in f64 (kept as an f32 value
//      plus its rounding residual), add the far-field term, and park
//      position and parameters in shared memory;
//   2. the receptor cell rows (z, y) that intersect the sphere of radius
//      10 A + rho around the posed group centre are enumerated lane-parallel,
//      trimmed in x, and concatenated into one candidate index space by a
//      warp prefix sum (a table of at most V2_ROWS rows, flushed as needed);
//   3. candidates are read 32 at a time (one per lane, coalesced float4);
//      each lane tests its receptor atom against the G ligand atoms
//      (broadcast shared-memory reads) into a G-bit mask, and one warp
//      prefix sum of the mask popcounts appends every hit to the warp's ring
//      buffer in shared memory;
//   4. while 32 or more hits are pending, each lane takes one and evaluates
//      the pair terms with compensated distances and the exact d^2 <= 100
//      test, accumulating in f64: the expensive math runs on 32 busy lanes.
// The per-pose reduction and the last-tile finalisation are those of
// k_score_tiles (deterministic: the hit order is fixed by the algorithm).
#pragma once
#include "lkg_score.cuh"

namespace lkg {

constexpr int V2_ROWS = 256;

template <int G> struct V2Ring { static constexpr int N = (G <= 8) ? 512 : (G <= 16) ? 1024 : 2048; };

template <int G>
struct V2Warp {
    float4 lpos[G];     // x, y, z (f32 part), q
    float4 lres[G];     // x, y, z residuals, sqrt eps
    float2 lpar[G];     // r, heavy
    int row_start[V2_ROWS];
    int row_pref[V2_ROWS];
    unsigned hit[V2Ring<G>::N];   // (ligand slot << 26) | receptor index
};

__device__ __forceinline__ int v2_find_row(const int* pref, int nrows, int k) {
    int lo = 0, hi = nrows - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (pref[mid] <= k) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// pair terms of one queued hit (exact d^2 <= 100 test on compensated d^2)
template <int G>
__device__ __forceinline__ void v2_pair(const ComplexDev& c, const V2Warp<G>& W, unsigned e, unsigned flags,
                                        double& elec, double& vdw, int& np) {
    const int l = (int)(e >> 26), k = (int)(e & 0x3ffffffu);
    const float4 lp = W.lpos[l], lr = W.lres[l];
    const float2 lq = W.lpar[l];
    const float4 a = __ldg(c.rpos + k);
    float dx = (lp.x - a.x) + lr.x, dy = (lp.y - a.y) + lr.y, dz = (lp.z - a.z) + lr.z;
    float d2 = dx * dx + dy * dy + dz * dz;
    if (!(d2 <= 100.f)) return;
    const float4 pr = __ldg(c.rpar + k);
    ++np;
    pair_fast(flags, lp.w, lr.w, lq.x, lq.y != 0.f, a, pr, d2, elec, vdw);
}

template <int TILE, int G>
__global__ void __launch_bounds__(TILE) k_score_v2(LaunchParams p) {
    static_assert(TILE % 32 == 0 && TILE % G == 0 && G <= 32, "tile shape");
    constexpr int NW = TILE / 32, RING = V2Ring<G>::N;
    __shared__ long long s_work;
    __shared__ double s_red[4][32];
    extern __shared__ __align__(16) unsigned char v2_smem[];   // NW x V2Warp<G>
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    V2Warp<G>& W = reinterpret_cast<V2Warp<G>*>(v2_smem)[wid];
    const unsigned lt_mask = (1u << lane) - 1u;
    for (;;) {
        if (threadIdx.x == 0) s_work = (long long)atomicAdd(p.work_counter, 1ull);
        __syncthreads();
        const long long w = s_work;
        __syncthreads();
        if (w >= p.total_work) break;
        const int b = find_item(p.item_work0, p.n_items, w);
        const ComplexDev& c = p.cx[__ldg(p.item_complex + b)];
        const long long local = w - __ldg(p.item_work0 + b);
        const int pose = (int)(local / c.ntiles), tile = (int)(local % c.ntiles);
        const long long g = (long long)__ldg(p.item_pose0 + b) + pose;
        const unsigned flags = c.flags;
        const int ngrp = (c.nl + G - 1) / G;
        const Rot rot = pose_matrix(p.poses + 7 * g);
        double elec = 0.0, vdw = 0.0;
        int np = 0;
        unsigned head = 0, tail = 0;
        for (int gi = wid; gi < TILE / G; gi += NW) {
            const int grp = tile * (TILE / G) + gi;
            if (grp >= ngrp) break;
            // drain what the previous group left before its slots are reused
            __syncwarp();
            if ((int)(tail - head) > lane) v2_pair<G>(c, W, W.hit[(head + lane) & (RING - 1)], flags, elec, vdw, np);
            head = tail;
            __syncwarp();
            // 1. the group's ligand atoms
            if (lane < G) {
                const int j = grp * G + lane;
                const bool valid = j < c.nl;
                const float4 b4 = valid ? __ldg(c.lpos + j) : make_float4(0.f, 0.f, 0.f, 0.f);
                const float4 lp4 = valid ? __ldg(c.lpar + j) : make_float4(0.f, 0.f, 0.f, 0.f);
                double xd, yd, zd;
                apply(rot, (double)b4.x, (double)b4.y, (double)b4.z, xd, yd, zd);
                float x = (float)xd, y = (float)yd, z = (float)zd;
                const float4 res = make_float4((float)(xd - (double)x), (float)(yd - (double)y),
                                               (float)(zd - (double)z), lp4.x);
                if (valid && (flags & F_FAR) && b4.w != 0.f) elec += (double)(b4.w * sample_phi(c, x, y, z));
                if (!valid) { x = y = z = 1e30f; }   // never within reach of a receptor atom
                W.lpos[lane] = make_float4(x, y, z, b4.w);
                W.lres[lane] = res;
                W.lpar[lane] = make_float2(lp4.y, lp4.z);
            }
            __syncwarp();
            // 2. candidate rows of the group sphere
            const float4 gs = __ldg(c.lgrp + grp);   // ligand-frame centre, radius
            double cxd, cyd, czd;
            apply(rot, (double)gs.x, (double)gs.y, (double)gs.z, cxd, cyd, czd);
            const float gx = (float)cxd, gy = (float)cyd, gz = (float)czd;
            const float R = SCAN_R + gs.w, R2 = R * R;
            const int cz0 = max(0, (int)floorf((gz - R - c.oz) * c.inv_h));
            const int cz1 = min(c.ncz - 1, (int)floorf((gz + R - c.oz) * c.inv_h));
            const int cy0 = max(0, (int)floorf((gy - R - c.oy) * c.inv_h));
            const int cy1 = min(c.ncy - 1, (int)floorf((gy + R - c.oy) * c.inv_h));
            const int nyr = cy1 - cy0 + 1, nzr = cz1 - cz0 + 1;
            const int nbox = (nyr > 0 && nzr > 0) ? nyr * nzr : 0;
            int nrows = 0, total = 0;
            for (int r0 = 0; r0 < nbox; r0 += 32) {
                const int r = r0 + lane;
                int st = 0, len = 0;
                if (r < nbox) {
                    const int cz = cz0 + r / nyr, cy = cy0 + r % nyr;
                    const float zlo = c.oz + cz * c.h, ylo = c.oy + cy * c.h;
                    const float dzm = fmaxf(0.f, fmaxf(zlo - gz, gz - (zlo + c.h)));
                    const float dym = fmaxf(0.f, fmaxf(ylo - gy, gy - (ylo + c.h)));
                    const float rem = R2 - dzm * dzm - dym * dym;
                    if (rem >= 0.f) {
                        const float wx = sqrtf(rem);
                        const int cx0 = max(0, (int)floorf((gx - wx - c.ox) * c.inv_h));
                        const int cx1 = min(c.ncx - 1, (int)floorf((gx + wx - c.ox) * c.inv_h));
                        if (cx0 <= cx1) {
                            const int row = (cz * c.ncy + cy) * c.ncx;
                            st = __ldg(c.cell_start + row + cx0);
                            len = __ldg(c.cell_start + row + cx1 + 1) - st;
                        }
                    }
                }
                const unsigned m = __ballot_sync(0xffffffffu, len > 0);
                int inc = len;   // inclusive prefix of len over lanes
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const int v = __shfl_up_sync(0xffffffffu, inc, o);
                    if (lane >= o) inc += v;
                }
                if (len > 0) {
                    const int slot = nrows + __popc(m & lt_mask);
                    W.row_start[slot] = st;
                    W.row_pref[slot] = total + inc - len;
                }
                nrows += __popc(m);
                total += __shfl_sync(0xffffffffu, inc, 31);
                if (nrows > V2_ROWS - 32 || r0 + 32 >= nbox) {
                    __syncwarp();
                    // 3. candidate chunks: G tests per lane into a mask, one
                    //    prefix sum appends the hits
                    for (int k0 = 0; k0 < total; k0 += 32) {
                        const int kk = k0 + lane;
                        float4 a = make_float4(3e30f, 3e30f, 3e30f, 0.f);
                        int ridx = 0;
                        if (kk < total) {
                            const int rr = v2_find_row(W.row_pref, nrows, kk);
                            ridx = W.row_start[rr] + (kk - W.row_pref[rr]);
                            a = __ldg(c.rpos + ridx);
                        }
                        unsigned mask = 0;
#pragma unroll
                        for (int l = 0; l < G; ++l) {
                            const float4 lp = W.lpos[l];
                            const float dx = lp.x - a.x, dy = lp.y - a.y, dz = lp.z - a.z;
                            mask |= (dx * dx + dy * dy + dz * dz <= 100.01f ? 1u : 0u) << l;
                        }
                        const int nh = __popc(mask);
                        int ex = nh;   // inclusive prefix of hit counts
#pragma unroll
                        for (int o = 1; o < 32; o <<= 1) {
                            const int v = __shfl_up_sync(0xffffffffu, ex, o);
                            if (lane >= o) ex += v;
                        }
                        unsigned pos = tail + (unsigned)(ex - nh);
                        while (mask) {
                            const int l = __ffs(mask) - 1;
                            mask &= mask - 1u;
                            W.hit[pos & (RING - 1)] = ((unsigned)l << 26) | (unsigned)ridx;
                            ++pos;
                        }
                        tail += (unsigned)__shfl_sync(0xffffffffu, ex, 31);
                        __syncwarp();
                        // 4. evaluate full batches of 32 hits
                        while (tail - head >= 32) {
                            v2_pair<G>(c, W, W.hit[(head + lane) & (RING - 1)], flags, elec, vdw, np);
                            head += 32;
                        }
                        __syncwarp();
                    }
                    nrows = 0;
                    total = 0;
                }
            }
        }
        __syncwarp();
        if ((int)(tail - head) > lane) v2_pair<G>(c, W, W.hit[(head + lane) & (RING - 1)], flags, elec, vdw, np);
        __syncwarp();
        double v[3] = {elec, vdw, (double)np};
        block_sum<3>(v, s_red);
        if (threadIdx.x == 0) {
            // partial of work unit w; the pose's units are w - tile .. w - tile + ntiles - 1
            double* part = p.partials + (size_t)w * 4;
            part[0] = v[0]; part[1] = v[1]; part[2] = 0.0; part[3] = v[2];
            __threadfence();
            int done = atomicAdd(p.pose_counter + g, 1);
            if (done == c.ntiles - 1) {
                __threadfence();
                double e = 0.0, vv = 0.0, nps = 0.0;
                const double* pp = p.partials + (size_t)(w - tile) * 4;
                for (int t = 0; t < c.ntiles; ++t) {
                    e += __ldcg(pp + 4 * t); vv += __ldcg(pp + 4 * t + 1); nps += __ldcg(pp + 4 * t + 3);
                }
                write_pose(p, c, g, e, vv, 0.0, nps);
                p.pose_counter[g] = 0;
            }
        }
    }
    finish_launch(p);
}

}  // namespace lkg
