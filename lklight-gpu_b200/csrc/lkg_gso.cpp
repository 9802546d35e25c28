// GSO driver over the batched GPU scorer: the caller side of the hot path
// (GSO::run, src/lib.rs:66-78; Swarm, src/swarm.rs:70-230; Glowworm,
// src/glowworm.rs), for many swarms of many complexes at once.
//
// Each step scores every moved (or first-step) glowworm of every swarm of
// every complex in ONE batched device launch group (lkg_score_multi), then
// applies the luciferin update and the movement phase on the host exactly as
// the reference does (neighbour lists, probabilities, one serial uniform draw
// per glowworm from the swarm's StdRng, 0.5 A translation step, slerp 0.5,
// vision-range update).  Every swarm of a complex is seeded with the same
// seed, as every `LKlight run` of a setup is (simulator.rs:184, lib.rs:58).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <unordered_map>
#include <vector>

#include "lkg_rng.h"
#include "lkg_runtime.h"

using namespace lkg;

namespace {

struct Quat { double w, x, y, z; };

void q_normalize(Quat& q) {  // qt.rs:36-46
    double n = std::sqrt(q.w * q.w + q.x * q.x + q.y * q.y + q.z * q.z);
    q.w /= n; q.x /= n; q.y /= n; q.z /= n;
}

Quat q_slerp(Quat q1, Quat q2, double t) {  // qt.rs:80-104
    q_normalize(q1);
    q_normalize(q2);
    double dot = q1.w * q2.w + q1.x * q2.x + q1.y * q2.y + q1.z * q2.z;
    if (dot < 0.0) { q1 = {-q1.w, -q1.x, -q1.y, -q1.z}; dot *= -1.0; }
    if (dot > 0.9995) {
        Quat r{q1.w + (q2.w - q1.w) * t, q1.x + (q2.x - q1.x) * t, q1.y + (q2.y - q1.y) * t, q1.z + (q2.z - q1.z) * t};
        q_normalize(r);
        return r;
    }
    dot = std::fmax(std::fmin(dot, 1.0), -1.0);
    double omega = std::acos(dot), so = std::sin(omega);
    double a = std::sin((1.0 - t) * omega) / so, b = std::sin(t * omega) / so;
    return {q1.w * a + q2.w * b, q1.x * a + q2.x * b, q1.y * a + q2.y * b, q1.z * a + q2.z * b};
}

struct Glow {
    double t[3];
    Quat r;
    double luciferin = 5.0, vision = 0.2, scoring = 0.0;   // glowworm.rs:45-51
    bool moved = false;
    uint32_t step = 0;
    std::vector<uint32_t> nb;
    std::vector<double> prob;
};

constexpr double RHO = 0.5, GAMMA = 0.4, BETA = 0.08, MAX_VISION = 5.0;
constexpr int MAX_NEIGHBORS = 5;

struct Swarm {
    std::vector<Glow> g;
    StdRng rng;
    std::vector<double> pos;
    std::vector<Quat> rot;
    std::vector<double> luc;

    // neighbour lists: uniform hash with cell = max vision range, candidates
    // re-sorted by id (swarm.rs:181-230), identical to the all-pairs scan
    void neighbours() {
        const size_t n = g.size();
        const double cell = MAX_VISION;
        std::unordered_map<int64_t, std::vector<uint32_t>> cells;
        cells.reserve(n * 2);
        auto key = [](int64_t x, int64_t y, int64_t z) {
            return ((x & 0x1fffff) << 42) | ((y & 0x1fffff) << 21) | (z & 0x1fffff);
        };
        for (size_t i = 0; i < n; ++i)
            cells[key((int64_t)std::floor(g[i].t[0] / cell), (int64_t)std::floor(g[i].t[1] / cell),
                      (int64_t)std::floor(g[i].t[2] / cell))].push_back((uint32_t)i);
        for (size_t i = 0; i < n; ++i) {
            Glow& g1 = g[i];
            double vr2 = g1.vision * g1.vision;
            int64_t cx = (int64_t)std::floor(g1.t[0] / cell), cy = (int64_t)std::floor(g1.t[1] / cell),
                    cz = (int64_t)std::floor(g1.t[2] / cell);
            g1.nb.clear();
            for (int64_t dz = -1; dz <= 1; ++dz)
                for (int64_t dy = -1; dy <= 1; ++dy)
                    for (int64_t dx = -1; dx <= 1; ++dx) {
                        auto it = cells.find(key(cx + dx, cy + dy, cz + dz));
                        if (it == cells.end()) continue;
                        for (uint32_t id : it->second) {
                            const Glow& g2 = g[id];
                            if (id == i || !(g1.luciferin < g2.luciferin)) continue;
                            double ddx = g1.t[0] - g2.t[0], ddy = g1.t[1] - g2.t[1], ddz = g1.t[2] - g2.t[2];
                            if (ddx * ddx + ddy * ddy + ddz * ddz < vr2) g1.nb.push_back(id);
                        }
                    }
            std::sort(g1.nb.begin(), g1.nb.end());
        }
    }

    void movement() {  // swarm.rs:105-174
        const size_t n = g.size();
        if (!n) return;
        pos.resize(3 * n);
        rot.resize(n);
        luc.resize(n);
        for (size_t i = 0; i < n; ++i) {
            for (int a = 0; a < 3; ++a) pos[3 * i + a] = g[i].t[a];
            rot[i] = g[i].r;
            luc[i] = g[i].luciferin;
        }
        neighbours();
        for (size_t i = 0; i < n; ++i) {  // glowworm.rs:114-128
            Glow& gw = g[i];
            gw.prob.clear();
            double total = 0.0;
            for (uint32_t id : gw.nb) {
                double d = luc[id] - gw.luciferin;
                gw.prob.push_back(d);
                total += d;
            }
            for (auto& p : gw.prob) p /= total;
        }
        std::vector<double> rnd(n);
        for (size_t i = 0; i < n; ++i) rnd[i] = rng.gen_f64();
        for (size_t i = 0; i < n; ++i) {
            Glow& gw = g[i];
            uint32_t nid = (uint32_t)i;
            if (!gw.nb.empty()) {  // glowworm.rs:130-142
                double sum = 0.0;
                size_t k = 0;
                while (sum < rnd[i] && k < gw.prob.size()) { sum += gw.prob[k]; ++k; }
                nid = gw.nb[k == 0 ? 0 : k - 1];
            }
            gw.moved = nid != (uint32_t)i;  // glowworm.rs:144-166
            if (gw.moved) {
                double dx = pos[3 * nid] - gw.t[0], dy = pos[3 * nid + 1] - gw.t[1], dz = pos[3 * nid + 2] - gw.t[2];
                double norm = std::sqrt(dx * dx + dy * dy + dz * dz);
                double coef = 0.5 / norm;
                gw.t[0] += dx * coef;
                gw.t[1] += dy * coef;
                gw.t[2] += dz * coef;
                gw.r = q_slerp(gw.r, rot[nid], 0.5);
                q_normalize(gw.r);
            }
            double v = gw.vision + BETA * (double)(MAX_NEIGHBORS - (int)gw.nb.size());
            gw.vision = std::fmin(MAX_VISION, std::fmax(0.0, v));
        }
    }
};

}  // namespace

struct lkg_gso {
    lkg_ctx* ctx;
    std::vector<int> group_complex, group_first_swarm, group_nswarm;
    std::vector<Swarm> swarms;
    std::vector<int> need_idx;  // per scored pose: swarm * 2^20 + glowworm
    int64_t scored = 0;
    lkg::DBuf d_poses, d_scores;
    lkg::HBuf h_poses, h_scores;
};

extern "C" {

int lkg_gso_create(lkg_ctx* ctx, int n_groups, const int* complex_ids, const int* n_swarms,
                   const int* n_glow, const double* positions, const uint64_t* seeds, lkg_gso** out) {
    if (!ctx || !out || n_groups <= 0 || !complex_ids || !n_swarms || !n_glow || !positions || !seeds)
        return set_error(LKG_ERR_ARG, "bad gso arguments");
    auto* G = new lkg_gso();
    G->ctx = ctx;
    size_t row = 0;
    for (int gi = 0; gi < n_groups; ++gi) {
        if (complex_ids[gi] < 0 || complex_ids[gi] >= (int)ctx->cx.size() || n_swarms[gi] < 0 || n_glow[gi] < 0 ||
            n_glow[gi] >= (1 << 20)) {
            delete G;
            return set_error(LKG_ERR_ARG, "bad gso group %d", gi);
        }
        G->group_complex.push_back(complex_ids[gi]);
        G->group_first_swarm.push_back((int)G->swarms.size());
        G->group_nswarm.push_back(n_swarms[gi]);
        for (int s = 0; s < n_swarms[gi]; ++s) {
            Swarm sw;
            sw.rng.seed_from_u64(seeds[gi]);
            sw.g.resize(n_glow[gi]);
            for (int k = 0; k < n_glow[gi]; ++k, ++row) {
                const double* p = positions + 7 * row;  // tx ty tz qw qx qy qz
                Glow& gw = sw.g[k];
                gw.t[0] = p[0]; gw.t[1] = p[1]; gw.t[2] = p[2];
                gw.r = {p[3], p[4], p[5], p[6]};
            }
            G->swarms.push_back(std::move(sw));
        }
    }
    *out = G;
    return set_ok();
}

// one GSO step: batched scoring of moved glowworms + movement
static int gso_step(lkg_gso* G) {
    lkg_ctx* ctx = G->ctx;
    const int ng = (int)G->group_complex.size();
    std::vector<int> counts(ng, 0);
    G->need_idx.clear();
    for (int gi = 0; gi < ng; ++gi)
        for (int s = G->group_first_swarm[gi]; s < G->group_first_swarm[gi] + G->group_nswarm[gi]; ++s) {
            const Swarm& sw = G->swarms[s];
            for (size_t k = 0; k < sw.g.size(); ++k)
                if (sw.g[k].moved || sw.g[k].step == 0) {  // swarm.rs:79-85
                    G->need_idx.push_back((s << 20) | (int)k);
                    counts[gi]++;
                }
        }
    const size_t n = G->need_idx.size();
    if (n) {
        LKG_CK(G->h_poses.reserve(n * 7 * sizeof(double)), "gso staging");
        LKG_CK(G->h_scores.reserve(n * sizeof(double)), "gso staging");
        LKG_CK(G->d_poses.reserve(n * 7 * sizeof(double)), "gso staging");
        LKG_CK(G->d_scores.reserve(n * sizeof(double)), "gso staging");
        double* hp = G->h_poses.as<double>();
        for (size_t i = 0; i < n; ++i) {
            const Glow& gw = G->swarms[G->need_idx[i] >> 20].g[G->need_idx[i] & 0xfffff];
            double* p = hp + 7 * i;  // kernel layout w,x,y,z,tx,ty,tz (gpu_score.rs:292-301)
            p[0] = gw.r.w; p[1] = gw.r.x; p[2] = gw.r.y; p[3] = gw.r.z;
            p[4] = gw.t[0]; p[5] = gw.t[1]; p[6] = gw.t[2];
        }
        LKG_CK(cudaMemcpyAsync(G->d_poses.p, hp, n * 7 * sizeof(double), cudaMemcpyHostToDevice, ctx->stream),
               "gso pose upload");
        int st = launch_items(ctx, ng, G->group_complex.data(), counts.data(), G->d_poses.as<double>(),
                              G->d_scores.as<double>(), nullptr, 0, 0, nullptr, nullptr);
        if (st) return st;
        LKG_CK(cudaMemcpyAsync(G->h_scores.p, G->d_scores.p, n * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream),
               "gso score readback");
        if ((st = wait_stream(ctx, 300.0))) return st;
        if ((st = check_status(ctx))) return st;
        const double* hs = G->h_scores.as<double>();
        for (size_t i = 0; i < n; ++i) G->swarms[G->need_idx[i] >> 20].g[G->need_idx[i] & 0xfffff].scoring = hs[i];
        G->scored += (int64_t)n;
    }
    const int ns = (int)G->swarms.size();
#pragma omp parallel for schedule(dynamic, 1)
    for (int s = 0; s < ns; ++s) {
        Swarm& sw = G->swarms[s];
        for (auto& gw : sw.g) {  // swarm.rs:96-99
            gw.luciferin = (1.0 - RHO) * gw.luciferin + GAMMA * gw.scoring;
            gw.step += 1;
        }
        sw.movement();
    }
    return set_ok();
}

int lkg_gso_run(lkg_gso* G, int steps) {
    if (!G || steps < 0) return set_error(LKG_ERR_ARG, "bad gso run");
    cudaSetDevice(G->ctx->device);
    for (int s = 0; s < steps; ++s) {
        int st = gso_step(G);
        if (st) return st;
    }
    return set_ok();
}

int lkg_gso_state(lkg_gso* G, double* trans, double* rot, double* luc, double* scoring, double* vision,
                  int32_t* nneigh) {
    if (!G) return set_error(LKG_ERR_ARG, "null gso");
    size_t row = 0;
    for (const Swarm& sw : G->swarms)
        for (const Glow& g : sw.g) {
            if (trans) for (int a = 0; a < 3; ++a) trans[3 * row + a] = g.t[a];
            if (rot) { rot[4 * row] = g.r.w; rot[4 * row + 1] = g.r.x; rot[4 * row + 2] = g.r.y; rot[4 * row + 3] = g.r.z; }
            if (luc) luc[row] = g.luciferin;
            if (scoring) scoring[row] = g.scoring;
            if (vision) vision[row] = g.vision;
            if (nneigh) nneigh[row] = (int32_t)g.nb.size();
            ++row;
        }
    return set_ok();
}

int64_t lkg_gso_scored(lkg_gso* G) { return G ? G->scored : 0; }

int lkg_gso_destroy(lkg_gso* G) {
    delete G;
    return set_ok();
}

// rand 0.7.3 StdRng for callers (setup pose generation, tests)
void* lkg_rng_new(uint64_t seed) { return new StdRng(seed); }
double lkg_rng_f64(void* r) { return ((StdRng*)r)->gen_f64(); }
void lkg_rng_free(void* r) { delete (StdRng*)r; }

}  // extern "C"
