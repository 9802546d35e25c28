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
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <unordered_map>
#include <vector>

#include "lkg_gso_dev.h"
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
    bool exact_next = false;      // screened run: score this move exactly
    double pred = 0.0;            // screened run: surrogate score of the move
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

    // neighbour lists (swarm.rs:181-230), identical to the all-pairs scan:
    // the neighbours of glowworm i are the glowworms brighter than i within
    // its vision range, in id order.  Two orders of the swarm are built
    // once per step: by x and by luciferin.  Each glowworm scans the shorter
    // of (a) its x-window [x - v, x + v] and (b) the glowworms brighter than
    // itself, testing every candidate exactly.  (a) is short for the dim,
    // short-sighted majority, (b) for the brightest glowworms, whose vision
    // grows to the 5 A maximum because nobody outshines them.
    std::vector<uint32_t> xorder, lorder, lrank;
    std::vector<double> xs, ys, zs, ls, bx, by, bz, bl;   // sorted copies (contiguous scans)
    std::vector<uint32_t> tmp;
    void neighbours() {
        const size_t n = g.size();
        // NaN coordinates / luciferin sort last and never pass a test
        auto kx = [this](uint32_t i) { const double v = g[i].t[0]; return v == v ? v : INFINITY; };
        auto kl = [this](uint32_t i) { const double v = g[i].luciferin; return v == v ? v : INFINITY; };
        xorder.resize(n);
        lorder.resize(n);
        for (size_t i = 0; i < n; ++i) xorder[i] = lorder[i] = (uint32_t)i;
        std::sort(xorder.begin(), xorder.end(), [&](uint32_t a, uint32_t b) {
            const double xa = kx(a), xb = kx(b);
            return xa < xb || (xa == xb && a < b);
        });
        std::sort(lorder.begin(), lorder.end(), [&](uint32_t a, uint32_t b) {
            const double la = kl(a), lb = kl(b);
            return la < lb || (la == lb && a < b);
        });
        lrank.resize(n);
        xs.resize(n); ys.resize(n); zs.resize(n); ls.resize(n);
        bx.resize(n); by.resize(n); bz.resize(n); bl.resize(n);
        for (size_t k = 0; k < n; ++k) {
            const Glow& q = g[xorder[k]];
            xs[k] = kx(xorder[k]); ys[k] = q.t[1]; zs[k] = q.t[2]; ls[k] = q.luciferin;
            const Glow& b = g[lorder[k]];
            bx[k] = b.t[0]; by[k] = b.t[1]; bz[k] = b.t[2]; bl[k] = b.luciferin;
            lrank[lorder[k]] = (uint32_t)k;
        }
        for (size_t i = 0; i < n; ++i) {
            Glow& g1 = g[i];
            g1.nb.clear();
            const double v = g1.vision, vr2 = v * v;
            if (!(v > 0.0)) continue;   // d^2 < 0 never holds
            const double x = g1.t[0], y = g1.t[1], z = g1.t[2], l1 = g1.luciferin;
            // the window is widened past the rounding of x +- v: extra
            // candidates are harmless, each is tested exactly
            const double w = v * (1.0 + 1e-9) + 1e-12;
            const size_t k0 = (size_t)(std::lower_bound(xs.begin(), xs.end(), x - w) - xs.begin());
            const size_t k1 = (size_t)(std::upper_bound(xs.begin() + k0, xs.end(), x + w) - xs.begin());
            const size_t r = lrank[i];
            // branch-free appends: the brighter / in-range tests are coin
            // flips for the branch predictor
            size_t cnt = 0;
            if (k1 - k0 <= n - 1 - r) {
                if (tmp.size() < k1 - k0) tmp.resize(k1 - k0);
                for (size_t k = k0; k < k1; ++k) {
                    const double ddx = x - xs[k], ddy = y - ys[k], ddz = z - zs[k];
                    tmp[cnt] = xorder[k];
                    // l1 < l1 is false: i itself never passes
                    cnt += (size_t)((l1 < ls[k]) & (ddx * ddx + ddy * ddy + ddz * ddz < vr2));
                }
            } else {
                if (tmp.size() < n - 1 - r) tmp.resize(n - 1 - r);
                for (size_t k = r + 1; k < n; ++k) {
                    const double ddx = x - bx[k], ddy = y - by[k], ddz = z - bz[k];
                    tmp[cnt] = lorder[k];
                    // equal luciferin does not count
                    cnt += (size_t)((l1 < bl[k]) & (ddx * ddx + ddy * ddy + ddz * ddz < vr2));
                }
            }
            g1.nb.assign(tmp.begin(), tmp.begin() + cnt);
            std::sort(g1.nb.begin(), g1.nb.end());
        }
    }

    // neighbour lists and selection probabilities (swarm.rs:105-128,
    // glowworm.rs:114-128) of every glowworm from the current state
    void prepare() {
        const size_t n = g.size();
        pos.resize(3 * n);
        rot.resize(n);
        luc.resize(n);
        for (size_t i = 0; i < n; ++i) {
            for (int a = 0; a < 3; ++a) pos[3 * i + a] = g[i].t[a];
            rot[i] = g[i].r;
            luc[i] = g[i].luciferin;
        }
        neighbours();
        for (size_t i = 0; i < n; ++i) {
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
    }

    // the neighbour a uniform draw selects (glowworm.rs:130-142)
    uint32_t select(const Glow& gw, uint32_t self, double u) const {
        if (gw.nb.empty()) return self;
        double sum = 0.0;
        size_t k = 0;
        while (sum < u && k < gw.prob.size()) { sum += gw.prob[k]; ++k; }
        return gw.nb[k == 0 ? 0 : k - 1];
    }

    // pose after a move towards neighbour nid (glowworm.rs:144-166)
    void moved_pose(const Glow& gw, uint32_t nid, double t[3], Quat& r) const {
        double dx = pos[3 * nid] - gw.t[0], dy = pos[3 * nid + 1] - gw.t[1], dz = pos[3 * nid + 2] - gw.t[2];
        double norm = std::sqrt(dx * dx + dy * dy + dz * dz);
        double coef = 0.5 / norm;
        t[0] = gw.t[0] + dx * coef;
        t[1] = gw.t[1] + dy * coef;
        t[2] = gw.t[2] + dz * coef;
        r = q_slerp(gw.r, rot[nid], 0.5);
        q_normalize(r);
    }

    void update_vision(Glow& gw) {
        double v = gw.vision + BETA * (double)(MAX_NEIGHBORS - (int)gw.nb.size());
        gw.vision = std::fmin(MAX_VISION, std::fmax(0.0, v));
    }

    void movement() {  // swarm.rs:105-174
        const size_t n = g.size();
        if (!n) return;
        prepare();
        std::vector<double> rnd(n);
        for (size_t i = 0; i < n; ++i) rnd[i] = rng.gen_f64();
        for (size_t i = 0; i < n; ++i) {
            Glow& gw = g[i];
            const uint32_t nid = select(gw, (uint32_t)i, rnd[i]);
            gw.moved = nid != (uint32_t)i;
            if (gw.moved) moved_pose(gw, nid, gw.t, gw.r);
            update_vision(gw);
        }
    }

    // screened movement, part 1: K draws per glowworm (serially, glowworm
    // by glowworm); for those with neighbours the current pose and the K
    // candidate poses (kernel layout w, x, y, z, tx, ty, tz); vision update
    void propose(int K, std::vector<double>& cand, std::vector<uint32_t>& owner) {
        const size_t n = g.size();
        cand.clear();
        owner.clear();
        if (!n) return;
        prepare();
        std::vector<double> rnd(n * (size_t)K);
        for (auto& u : rnd) u = rng.gen_f64();
        for (size_t i = 0; i < n; ++i) {
            Glow& gw = g[i];
            gw.moved = false;
            gw.exact_next = false;
            if (!gw.nb.empty()) {
                // candidate 0 is the glowworm's current pose: the surrogate's
                // gain estimate is relative to its own value there
                const double cur[7] = {gw.r.w, gw.r.x, gw.r.y, gw.r.z, gw.t[0], gw.t[1], gw.t[2]};
                cand.insert(cand.end(), cur, cur + 7);
                owner.push_back((uint32_t)i);
                for (int k = 0; k < K; ++k) {
                    const uint32_t nid = select(gw, (uint32_t)i, rnd[i * K + k]);
                    double t[3];
                    Quat r;
                    moved_pose(gw, nid, t, r);
                    const double row[7] = {r.w, r.x, r.y, r.z, t[0], t[1], t[2]};
                    cand.insert(cand.end(), row, row + 7);
                    owner.push_back((uint32_t)i);
                }
            }
            update_vision(gw);
        }
    }
};

}  // namespace

struct lkg_gso {
    lkg_ctx* ctx;
    std::vector<int> group_complex, group_first_swarm, group_nswarm;
    std::vector<Swarm> swarms;
    std::vector<int> need_idx;  // per scored pose: swarm * 2^20 + glowworm
    int64_t scored = 0, predicted = 0;
    int step = 0;
    // wall seconds per phase: exact scoring, host movement, surrogate
    // inference, surrogate training
    double t_exact = 0.0, t_move = 0.0, t_infer = 0.0, t_train = 0.0;
    std::vector<int> last_counts;   // exact scorings per group in the last scoring phase
    lkg::DBuf d_poses, d_scores;
    lkg::HBuf h_poses, h_scores;
    // surrogate screening (off unless lkg_gso_set_screen)
    bool screen = false;
    lkg_screen cfg{};
    std::vector<lkg_surrogate*> sur;             // one per group (complex)
    std::vector<std::vector<double>> tr_pose;    // per group: exact (pose, score) pairs
    std::vector<std::vector<double>> tr_score;
    std::vector<bool> scaled;
    StdRng rank_rng;                             // candidate ranks of the no-network ablation
    lkg::DBuf d_tp, d_ts, d_cand, d_pred;
    lkg::HBuf h_cand, h_pred;
    // device-resident plain GSO (lkg_gso_run_device)
    lkg_plan* dplan = nullptr;
    cudaGraphExec_t dexec = nullptr, sexec = nullptr;   // plain / screened device step graphs
    lkg::GsoDevState ds{}, ds_captured{};
    lkg::GsoDevScreen dx{}, dx_captured{};
    lkg::DBuf dbuf[24], sbuf[6];
    std::vector<int> dcounts;   // glowworms per group (device order)
    ~lkg_gso() {
        for (auto* s : sur) lkg_surrogate_destroy(s);
        if (dexec) cudaGraphExecDestroy(dexec);
        if (sexec) cudaGraphExecDestroy(sexec);
        if (dplan) lkg_plan_destroy(dplan);
    }
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

}  // extern "C"

namespace {

inline Glow& glow_of(lkg_gso* G, int idx) { return G->swarms[idx >> 20].g[idx & 0xfffff]; }

inline double now_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// Train (or fine-tune) the surrogate of group gi on its exact pairs (the
// last `recent` of them when recent > 0; at most 65,536 are kept), in a
// seeded shuffled order.
// most recent exact (pose, score) pairs kept per group for training
constexpr size_t TRAIN_CAP = 65536;

int train_group(lkg_gso* G, int gi, int epochs, size_t recent) {
    auto& P = G->tr_pose[gi];
    auto& S0 = G->tr_score[gi];
    const size_t cap = TRAIN_CAP;
    if (S0.size() > cap) {
        const size_t drop = S0.size() - cap;
        P.erase(P.begin(), P.begin() + 7 * drop);
        S0.erase(S0.begin(), S0.begin() + drop);
    }
    const size_t first = (recent > 0 && recent < S0.size()) ? S0.size() - recent : 0;
    const int n = (int)(S0.size() - first);
    if (n < 64 || epochs <= 0) return set_ok();
    const double t0 = now_s();
    const double* S = S0.data() + first;
    const double* PP = P.data() + 7 * first;
    int st;
    if (!G->scaled[gi]) {
        if ((st = lkg_surrogate_set_target_scale(G->sur[gi], n, S))) return st;
        G->scaled[gi] = true;
    }
    std::vector<int> perm(n);
    for (int i = 0; i < n; ++i) perm[i] = i;
    StdRng r(G->cfg.seed ^ (0x9e3779b97f4a7c15ull * (uint64_t)(G->step + 1)) ^ (uint64_t)gi);
    for (int i = n - 1; i > 0; --i) std::swap(perm[i], perm[(int)(r.gen_f64() * (i + 1)) % (i + 1)]);
    std::vector<double> hp(7 * (size_t)n), hs(n);
    for (int i = 0; i < n; ++i) {
        std::memcpy(&hp[7 * (size_t)i], PP + 7 * (size_t)perm[i], 7 * sizeof(double));
        hs[i] = S[perm[i]];
    }
    LKG_CK(G->d_tp.reserve(hp.size() * sizeof(double)), "surrogate training set");
    LKG_CK(G->d_ts.reserve(hs.size() * sizeof(double)), "surrogate training set");
    cudaStream_t s = G->ctx->stream;
    LKG_CK(cudaMemcpyAsync(G->d_tp.p, hp.data(), hp.size() * sizeof(double), cudaMemcpyHostToDevice, s), "train upload");
    LKG_CK(cudaMemcpyAsync(G->d_ts.p, hs.data(), hs.size() * sizeof(double), cudaMemcpyHostToDevice, s), "train upload");
    float loss = 0.f;
    st = lkg_surrogate_train(G->sur[gi], n, G->d_tp.as<double>(), G->d_ts.as<double>(), epochs,
                             G->cfg.batch > 0 ? G->cfg.batch : 1024, G->cfg.lr, &loss);
    G->t_train += now_s() - t0;
    return st;
}

// Exact scoring of the selected glowworms in one batched launch group;
// `all` selects every glowworm, otherwise first-step ones and moves marked
// for exact scoring.  Moves scored by the surrogate take its prediction
// (the no-network ablation keeps the previous score).  `learn` appends the
// exact pairs to the surrogate training sets.
int score_phase(lkg_gso* G, bool all, bool learn) {
    struct Acc { double& t; double t0; ~Acc() { t += now_s() - t0; } } acc{G->t_exact, now_s()};
    lkg_ctx* ctx = G->ctx;
    const int ng = (int)G->group_complex.size();
    std::vector<int> counts(ng, 0);
    G->need_idx.clear();
    for (int gi = 0; gi < ng; ++gi)
        for (int s = G->group_first_swarm[gi]; s < G->group_first_swarm[gi] + G->group_nswarm[gi]; ++s) {
            Swarm& sw = G->swarms[s];
            for (size_t k = 0; k < sw.g.size(); ++k) {
                Glow& gw = sw.g[k];
                if (all || gw.step == 0 || (gw.moved && gw.exact_next)) {  // swarm.rs:79-85
                    G->need_idx.push_back((s << 20) | (int)k);
                    counts[gi]++;
                } else if (gw.moved && G->screen && !G->cfg.random_rank && G->cfg.carry_prediction) {
                    gw.scoring = gw.pred;
                }
            }
        }
    G->last_counts = counts;
    const size_t n = G->need_idx.size();
    if (!n) return set_ok();
    LKG_CK(G->h_poses.reserve(n * 7 * sizeof(double)), "gso staging");
    LKG_CK(G->h_scores.reserve(n * sizeof(double)), "gso staging");
    LKG_CK(G->d_poses.reserve(n * 7 * sizeof(double)), "gso staging");
    LKG_CK(G->d_scores.reserve(n * sizeof(double)), "gso staging");
    double* hp = G->h_poses.as<double>();
    for (size_t i = 0; i < n; ++i) {
        const Glow& gw = glow_of(G, G->need_idx[i]);
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
    for (size_t i = 0; i < n; ++i) glow_of(G, G->need_idx[i]).scoring = hs[i];
    G->scored += (int64_t)n;
    if (learn) {
        size_t i = 0;
        for (int gi = 0; gi < ng; ++gi)
            for (int k = 0; k < counts[gi]; ++k, ++i) {
                G->tr_pose[gi].insert(G->tr_pose[gi].end(), hp + 7 * i, hp + 7 * i + 7);
                G->tr_score[gi].push_back(hs[i]);
            }
    }
    return set_ok();
}

// Screened movement: K candidate moves per glowworm with neighbours, all
// ranked by the surrogate (or, for the ablation, by seeded random numbers);
// each glowworm takes its best candidate, and per swarm the fraction
// exact_fraction of the moves with the largest predicted gain (surrogate at
// the move minus surrogate at the current pose) is marked for exact
// scoring; the others carry current score + predicted gain.
int screened_movement(lkg_gso* G) {
    double t0 = now_s();
    const int ns = (int)G->swarms.size(), ng = (int)G->group_complex.size(), K = G->cfg.candidates;
    std::vector<std::vector<double>> cand(ns);
    std::vector<std::vector<uint32_t>> owner(ns);
#pragma omp parallel for schedule(dynamic, 1)
    for (int s = 0; s < ns; ++s) G->swarms[s].propose(K, cand[s], owner[s]);
    std::vector<size_t> off(ns + 1, 0);
    for (int s = 0; s < ns; ++s) off[s + 1] = off[s] + owner[s].size();
    const size_t total = off[ns];
    if (total == 0) return set_ok();
    LKG_CK(G->h_cand.reserve(total * 7 * sizeof(double)), "candidate staging");
    LKG_CK(G->h_pred.reserve(total * sizeof(double)), "candidate staging");
    double* hc = G->h_cand.as<double>();
    double* hpred = G->h_pred.as<double>();
    for (int s = 0; s < ns; ++s)
        if (!cand[s].empty()) std::memcpy(hc + 7 * off[s], cand[s].data(), cand[s].size() * sizeof(double));
    G->t_move += now_s() - t0;
    t0 = now_s();
    if (G->cfg.random_rank) {
        for (size_t i = 0; i < total; ++i) hpred[i] = G->rank_rng.gen_f64();
    } else {
        LKG_CK(G->d_cand.reserve(total * 7 * sizeof(double)), "candidate staging");
        LKG_CK(G->d_pred.reserve(total * sizeof(double)), "candidate staging");
        cudaStream_t st = G->ctx->stream;
        LKG_CK(cudaMemcpyAsync(G->d_cand.p, hc, total * 7 * sizeof(double), cudaMemcpyHostToDevice, st), "candidates");
        for (int gi = 0; gi < ng; ++gi) {
            const int s0 = G->group_first_swarm[gi], s1 = s0 + G->group_nswarm[gi];
            const size_t a = off[s0], b = off[s1];
            if (b == a) continue;
            int rc = lkg_surrogate_predict(G->sur[gi], (int)(b - a), G->d_cand.as<double>() + 7 * a,
                                           G->d_pred.as<double>() + a);
            if (rc) return rc;
        }
        LKG_CK(cudaMemcpyAsync(hpred, G->d_pred.p, total * sizeof(double), cudaMemcpyDeviceToHost, st), "predictions");
        int rc = wait_stream(G->ctx, 300.0);
        if (rc) return rc;
        G->predicted += (int64_t)total;
    }
    G->t_infer += now_s() - t0;
    t0 = now_s();
    const double frac = G->cfg.exact_fraction;
#pragma omp parallel for schedule(dynamic, 1)
    for (int s = 0; s < ns; ++s) {
        Swarm& sw = G->swarms[s];
        std::vector<std::pair<double, uint32_t>> gain;
        for (size_t c0 = 0; c0 < owner[s].size(); c0 += K + 1) {
            const uint32_t i = owner[s][c0];
            size_t best = c0 + 1;
            for (size_t c = c0 + 2; c <= c0 + K; ++c)
                if (hpred[off[s] + c] > hpred[off[s] + best]) best = c;
            Glow& gw = sw.g[i];
            const double* row = hc + 7 * (off[s] + best);
            gw.r = {row[0], row[1], row[2], row[3]};
            gw.t[0] = row[4]; gw.t[1] = row[5]; gw.t[2] = row[6];
            // predicted change from the current pose, applied to its score
            const double g = hpred[off[s] + best] - hpred[off[s] + c0];
            gw.pred = gw.scoring + g;
            gw.moved = true;
            // the moves whose predicted score changes most are scored
            // exactly: an unscored move keeps a score that is off by about
            // its change, so the stale scores left are the smallest ones
            gain.push_back({std::fabs(g), i});
        }
        std::sort(gain.begin(), gain.end(), [](const std::pair<double, uint32_t>& a, const std::pair<double, uint32_t>& b) {
            return a.first > b.first || (a.first == b.first && a.second < b.second);
        });
        const size_t nx = (size_t)std::ceil(frac * (double)gain.size());
        for (size_t k = 0; k < nx && k < gain.size(); ++k) sw.g[gain[k].second].exact_next = true;
    }
    G->t_move += now_s() - t0;
    return set_ok();
}

// one GSO step: scoring, luciferin update, movement (swarm.rs:70-103)
int gso_step(lkg_gso* G) {
    const lkg_screen& c = G->cfg;
    const bool training = G->screen && G->step < c.train_steps;
    const bool screened = G->screen && G->step >= c.train_steps;
    const bool rescore = screened && c.rescore_every > 0 && G->step > c.train_steps &&
                         (G->step - c.train_steps) % c.rescore_every == 0;
    int st = score_phase(G, rescore, training || rescore);
    if (st) return st;
    if (G->screen && !c.random_rank) {
        const int ng = (int)G->group_complex.size();
        const bool first = G->step == c.train_steps - 1;
        // first training: every exact pair so far; fine-tuning: the pairs of
        // this full rescoring
        for (int gi = 0; gi < ng && (first || rescore); ++gi)
            if ((st = train_group(G, gi, first ? c.train_epochs : c.finetune_epochs,
                                  first ? 0 : (size_t)G->last_counts[gi])))
                return st;
    }
    const int ns = (int)G->swarms.size();
#pragma omp parallel for schedule(dynamic, 1)
    for (int s = 0; s < ns; ++s) {
        for (auto& gw : G->swarms[s].g) {  // swarm.rs:96-99
            gw.luciferin = (1.0 - RHO) * gw.luciferin + GAMMA * gw.scoring;
            gw.step += 1;
        }
    }
    if (G->screen && G->step + 1 >= c.train_steps) {
        if ((st = screened_movement(G))) return st;
    } else {
        const double t0 = now_s();
#pragma omp parallel for schedule(dynamic, 1)
        for (int s = 0; s < ns; ++s) {
            Swarm& sw = G->swarms[s];
            sw.movement();
            for (auto& gw : sw.g) gw.exact_next = gw.moved;
        }
        G->t_move += now_s() - t0;
    }
    G->step++;
    return set_ok();
}

}  // namespace

extern "C" {

int lkg_gso_set_screen(lkg_gso* G, const lkg_screen* cfg) {
    if (!G || !cfg) return set_error(LKG_ERR_ARG, "bad screen arguments");
    if (G->step != 0) return set_error(LKG_ERR_STATE, "screening must be set before the first step");
    if (cfg->candidates < 1 || cfg->candidates > 64 || !(cfg->exact_fraction > 0.0 && cfg->exact_fraction <= 1.0) ||
        cfg->rescore_every < 0 || cfg->train_steps < 1 || cfg->train_epochs < 0 || cfg->finetune_epochs < 0 ||
        !(cfg->lr > 0.f) || (cfg->carry_prediction != 0 && cfg->carry_prediction != 1))
        return set_error(LKG_ERR_ARG, "bad screen configuration");
    for (auto* s : G->sur) lkg_surrogate_destroy(s);
    G->sur.clear();
    G->cfg = *cfg;
    const int ng = (int)G->group_complex.size();
    G->tr_pose.assign(ng, {});
    G->tr_score.assign(ng, {});
    G->scaled.assign(ng, false);
    G->rank_rng.seed_from_u64(cfg->seed);
    // every buffer the screened steps use is allocated here, at its final
    // size: growing one inside the step loop would reallocate (each free
    // synchronises the device) and a fresh allocation maps new pages
    size_t total = 0;
    for (int gi = 0; gi < ng; ++gi) {
        size_t ng_glow = 0;
        for (int s = G->group_first_swarm[gi]; s < G->group_first_swarm[gi] + G->group_nswarm[gi]; ++s)
            ng_glow += G->swarms[s].g.size();
        total += ng_glow * (size_t)(cfg->candidates + 1);
        if (cfg->random_rank) continue;
        lkg_surrogate* s = nullptr;
        int st = lkg_surrogate_create(G->ctx, G->group_complex[gi], cfg->seed + (uint64_t)gi, &s);
        if (st) return st;
        G->sur.push_back(s);
        const int batch = cfg->batch > 0 ? cfg->batch : 1024;
        if ((st = lkg_surrogate_reserve(s, (int)std::min<size_t>(ng_glow * (cfg->candidates + 1), INT32_MAX), batch)))
            return st;
    }
    LKG_CK(G->h_cand.reserve(total * 7 * sizeof(double)), "candidate staging");
    LKG_CK(G->h_pred.reserve(total * sizeof(double)), "candidate staging");
    if (!cfg->random_rank) {
        LKG_CK(G->d_cand.reserve(total * 7 * sizeof(double)), "candidate staging");
        LKG_CK(G->d_pred.reserve(total * sizeof(double)), "candidate staging");
        LKG_CK(G->d_tp.reserve(TRAIN_CAP * 7 * sizeof(double)), "surrogate training set");
        LKG_CK(G->d_ts.reserve(TRAIN_CAP * sizeof(double)), "surrogate training set");
    }
    G->screen = true;
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

// Swarm::save (swarm.rs:232-271): one swarm's glowworms as gso_<step>.out.
// Rust's {:.N} prints the correctly rounded fixed-point decimal of the f64
// (ties to even), as glibc's %.Nf does; NaN and infinities are spelled the
// Rust way.
static void put_fixed(std::string& out, double v, int prec) {
    if (std::isnan(v)) { out += "NaN"; return; }
    if (std::isinf(v)) { out += v < 0 ? "-inf" : "inf"; return; }
    char b[400];
    std::snprintf(b, sizeof(b), "%.*f", prec, v);
    out += b;
}

int lkg_gso_save(lkg_gso* G, int swarm, int step, const char* directory) {
    if (!G || !directory || swarm < 0 || swarm >= (int)G->swarms.size() || step < 0)
        return set_error(LKG_ERR_ARG, "bad save arguments");
    std::string text = "#Coordinates  RecID  LigID  Luciferin  Neighbor's number  Vision Range  Scoring\n";
    for (const Glow& g : G->swarms[swarm].g) {
        const double v[7] = {g.t[0], g.t[1], g.t[2], g.r.w, g.r.x, g.r.y, g.r.z};
        text += "(";
        for (int k = 0; k < 7; ++k) {
            if (k) text += ", ";
            put_fixed(text, v[k], 7);
        }
        text += ")    0    0   ";
        put_fixed(text, g.luciferin, 8);
        text += "  " + std::to_string(g.nb.size()) + " ";
        put_fixed(text, g.vision, 3);
        text += " ";
        put_fixed(text, g.scoring, 8);
        text += "\n";
    }
    const std::string path = std::string(directory) + "/gso_" + std::to_string(step) + ".out";
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) return set_error(LKG_ERR_ARG, "cannot create %s", path.c_str());
    const size_t w = std::fwrite(text.data(), 1, text.size(), f);
    const int c = std::fclose(f);
    if (w != text.size() || c != 0) return set_error(LKG_ERR_ARG, "cannot write %s", path.c_str());
    return set_ok();
}

int64_t lkg_gso_scored(lkg_gso* G) { return G ? G->scored : 0; }
int64_t lkg_gso_predicted(lkg_gso* G) { return G ? G->predicted : 0; }

// ---------------------------------------------------------------------------
// device-resident GSO (lkg_gso_run_device)
// ---------------------------------------------------------------------------
}  // extern "C"

namespace {

// Host state -> device arrays, the scoring plan, the GsoDevState views.
// `screened`: the mask marks the moves chosen for exact scoring, and the
// others carry their predicted score.
int dev_setup(lkg_gso* G, bool screened) {
    lkg_ctx* ctx = G->ctx;
    const int ns = (int)G->swarms.size(), ng = (int)G->group_complex.size();
    std::vector<int> first(ns), cnt(ns), of, counts(ng, 0);
    int n = 0, maxs = 0;
    for (int s = 0; s < ns; ++s) {
        first[s] = n;
        cnt[s] = (int)G->swarms[s].g.size();
        maxs = std::max(maxs, cnt[s]);
        for (int k = 0; k < cnt[s]; ++k) of.push_back(s);
        n += cnt[s];
    }
    for (int gi = 0; gi < ng; ++gi)
        for (int s = G->group_first_swarm[gi]; s < G->group_first_swarm[gi] + G->group_nswarm[gi]; ++s)
            counts[gi] += cnt[s];
    G->dcounts = counts;
    std::vector<double> a[10];
    for (auto& v : a) v.resize(n);
    std::vector<double> pose(7 * (size_t)n);
    std::vector<uint32_t> keys(8 * (size_t)ns);
    std::vector<unsigned long long> draws(ns);
    std::vector<unsigned char> mask(n + 64, 0);   // the counter after the mask starts at zero
    for (int s = 0, i = 0; s < ns; ++s) {
        const Swarm& sw = G->swarms[s];
        for (int k = 0; k < 8; ++k) keys[8 * s + k] = sw.rng.key()[k];
        draws[s] = sw.rng.words_used() / 2;
        for (const Glow& gw : sw.g) {
            a[0][i] = gw.t[0]; a[1][i] = gw.t[1]; a[2][i] = gw.t[2];
            a[3][i] = gw.r.w; a[4][i] = gw.r.x; a[5][i] = gw.r.y; a[6][i] = gw.r.z;
            a[7][i] = gw.luciferin; a[8][i] = gw.vision; a[9][i] = gw.scoring;
            const double row[7] = {gw.r.w, gw.r.x, gw.r.y, gw.r.z, gw.t[0], gw.t[1], gw.t[2]};
            std::memcpy(&pose[7 * (size_t)i], row, sizeof(row));
            if (screened) {   // score_phase: exact for the chosen moves, the carried prediction for the others
                mask[i] = ((gw.moved && gw.exact_next) || gw.step == 0) ? 1 : 0;
                if (G->cfg.carry_prediction && gw.moved && !gw.exact_next && gw.step != 0) a[9][i] = gw.pred;
            } else {
                mask[i] = (gw.moved || gw.step == 0) ? 1 : 0;   // swarm.rs:79-85
            }
            ++i;
        }
    }
    cudaStream_t st = ctx->stream;
    lkg::DBuf* b = G->dbuf;
    for (int k = 0; k < 18; ++k) LKG_CK(b[k].reserve(n * sizeof(double)), "device gso");
    LKG_CK(b[18].reserve(7 * (size_t)n * sizeof(double)), "device gso");
    LKG_CK(b[19].reserve(2 * (size_t)n * sizeof(int)), "device gso");
    LKG_CK(b[20].reserve((2 * (size_t)ns + n) * sizeof(int)), "device gso");
    LKG_CK(b[21].reserve(keys.size() * sizeof(uint32_t)), "device gso");
    LKG_CK(b[22].reserve(ns * sizeof(unsigned long long)), "device gso");
    LKG_CK(b[23].reserve(n + 64), "device gso");   // mask bytes, then the scored counter (8-aligned)
    for (int k = 0; k < 10; ++k)
        LKG_CK(cudaMemcpyAsync(b[k].p, a[k].data(), n * sizeof(double), cudaMemcpyHostToDevice, st), "device gso");
    LKG_CK(cudaMemcpyAsync(b[18].p, pose.data(), pose.size() * sizeof(double), cudaMemcpyHostToDevice, st), "device gso");
    std::vector<int> meta;
    meta.insert(meta.end(), first.begin(), first.end());
    meta.insert(meta.end(), cnt.begin(), cnt.end());
    meta.insert(meta.end(), of.begin(), of.end());
    LKG_CK(cudaMemcpyAsync(b[20].p, meta.data(), meta.size() * sizeof(int), cudaMemcpyHostToDevice, st), "device gso");
    LKG_CK(cudaMemcpyAsync(b[21].p, keys.data(), keys.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, st),
           "device gso");
    LKG_CK(cudaMemcpyAsync(b[22].p, draws.data(), ns * sizeof(unsigned long long), cudaMemcpyHostToDevice, st),
           "device gso");
    LKG_CK(cudaMemcpyAsync(b[23].p, mask.data(), mask.size(), cudaMemcpyHostToDevice, st), "device gso");
    lkg::GsoDevState& S = G->ds;
    S.n = n; S.n_swarms = ns; S.max_swarm = maxs;
    double* d[18];
    for (int k = 0; k < 18; ++k) d[k] = b[k].as<double>();
    S.tx = d[0]; S.ty = d[1]; S.tz = d[2]; S.qw = d[3]; S.qx = d[4]; S.qy = d[5]; S.qz = d[6];
    S.luc = d[7]; S.vis = d[8]; S.score = d[9];
    S.ntx = d[10]; S.nty = d[11]; S.ntz = d[12]; S.nqw = d[13]; S.nqx = d[14]; S.nqy = d[15]; S.nqz = d[16];
    S.nvis = d[17];
    S.poses = b[18].as<double>();
    S.nid = b[19].as<int>(); S.nnb = S.nid + n;
    S.swarm_first = b[20].as<int>(); S.swarm_n = S.swarm_first + ns; S.swarm_of = S.swarm_n + ns;
    S.keys = b[21].as<uint32_t>();
    S.draws = b[22].as<unsigned long long>();
    S.mask = b[23].as<unsigned char>();
    S.nscored = reinterpret_cast<unsigned long long*>(b[23].as<unsigned char>() + ((n + 7) & ~7));
    if (screened) {
        const int K = G->cfg.candidates;
        lkg::GsoDevScreen& X = G->dx;
        lkg::DBuf* c = G->sbuf;
        LKG_CK(c[0].reserve((size_t)n * (K + 1) * 7 * sizeof(double)), "device gso");
        LKG_CK(c[1].reserve((size_t)n * (K + 1) * sizeof(double)), "device gso");
        LKG_CK(c[2].reserve((size_t)n * K * sizeof(int)), "device gso");
        LKG_CK(c[3].reserve((size_t)n * sizeof(int)), "device gso");
        LKG_CK(c[4].reserve((size_t)n * sizeof(double)), "device gso");
        LKG_CK(c[5].reserve(2 * (size_t)n), "device gso");
        LKG_CK(cudaMemsetAsync(c[5].p, 0, 2 * (size_t)n, st), "device gso");   // no pending predictions
        X.K = K; X.carry = G->cfg.carry_prediction ? 1 : 0; X.frac = G->cfg.exact_fraction;
        X.cand = c[0].as<double>(); X.pred = c[1].as<double>(); X.knid = c[2].as<int>(); X.best = c[3].as<int>();
        X.gain = c[4].as<double>(); X.exact = c[5].as<unsigned char>(); X.pend = X.exact + n;
    }
    int rc;
    if (!G->dplan && (rc = lkg_plan_create(ctx, ng, G->group_complex.data(), counts.data(), &G->dplan))) return rc;
    return set_ok();
}

// device arrays -> host state after `steps` device steps
int dev_download(lkg_gso* G, int steps, bool screened) {
    const lkg::GsoDevState& S = G->ds;
    const int n = S.n, ns = S.n_swarms;
    lkg::DBuf* b = G->dbuf;
    std::vector<double> a[10];
    for (int k = 0; k < 10; ++k) {
        a[k].resize(n);
        LKG_CK(cudaMemcpy(a[k].data(), b[k].p, n * sizeof(double), cudaMemcpyDeviceToHost), "device gso");
    }
    std::vector<int> nid(2 * (size_t)n);
    LKG_CK(cudaMemcpy(nid.data(), b[19].p, nid.size() * sizeof(int), cudaMemcpyDeviceToHost), "device gso");
    std::vector<unsigned long long> draws(ns);
    LKG_CK(cudaMemcpy(draws.data(), S.draws, ns * sizeof(unsigned long long), cudaMemcpyDeviceToHost), "device gso");
    std::vector<double> gain;
    std::vector<unsigned char> ex;
    if (screened) {
        gain.resize(n);
        ex.resize(2 * (size_t)n);
        LKG_CK(cudaMemcpy(gain.data(), G->dx.gain, n * sizeof(double), cudaMemcpyDeviceToHost), "device gso");
        LKG_CK(cudaMemcpy(ex.data(), G->dx.exact, 2 * (size_t)n, cudaMemcpyDeviceToHost), "device gso");
    }
    for (int s = 0, i = 0; s < ns; ++s) {
        Swarm& sw = G->swarms[s];
        for (size_t k = 0; k < sw.g.size(); ++k, ++i) {
            Glow& gw = sw.g[k];
            gw.t[0] = a[0][i]; gw.t[1] = a[1][i]; gw.t[2] = a[2][i];
            gw.r = {a[3][i], a[4][i], a[5][i], a[6][i]};
            gw.luciferin = a[7][i]; gw.vision = a[8][i]; gw.scoring = a[9][i];
            if (screened) {   // as screened_movement leaves them
                gw.moved = nid[n + i] > 0;
                gw.exact_next = ex[i] != 0;
                gw.pred = ex[n + i] ? gw.scoring + gain[i] : gw.scoring;
            } else {
                gw.moved = nid[i] != (int)k;
                gw.exact_next = gw.moved;
            }
            gw.nb.assign((size_t)nid[n + i], 0u);   // the count only (state reports it)
            gw.step += (uint32_t)steps;
        }
        sw.rng.set_words_used(2 * draws[s]);
    }
    unsigned long long nsc = 0;
    LKG_CK(cudaMemcpy(&nsc, S.nscored, sizeof(nsc), cudaMemcpyDeviceToHost), "device gso");
    G->scored += (int64_t)nsc;
    return set_ok();
}

// one graph (or eager) step of the plain device GSO
int dev_plain_steps(lkg_gso* G, int steps) {
    lkg_ctx* ctx = G->ctx;
    cudaStream_t st = ctx->stream;
    lkg::GsoDevState& S = G->ds;
    int rc;
    // first step eagerly (it also makes the plan's host-side queries)
    if ((rc = lkg::plan_launch_masked(G->dplan, S.poses, S.score, S.mask))) return rc;
    LKG_CK(lkg::gso_dev_after_scoring(S, st), "device gso step");
    if (steps > 1) {
        if (G->dexec && std::memcmp(&G->ds_captured, &S, sizeof(S)) != 0) {
            cudaGraphExecDestroy(G->dexec);
            G->dexec = nullptr;
        }
        if (!G->dexec) {
            LKG_CK(cudaStreamSynchronize(st), "device gso");
            LKG_CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal), "device gso capture");
            rc = lkg::plan_launch_masked(G->dplan, S.poses, S.score, S.mask);
            const cudaError_t e1 = rc ? cudaSuccess : lkg::gso_dev_after_scoring(S, st);
            cudaGraph_t graph = nullptr;
            const cudaError_t e2 = cudaStreamEndCapture(st, &graph);
            if (rc) { if (graph) cudaGraphDestroy(graph); return rc; }
            if (e1 != cudaSuccess || e2 != cudaSuccess) {
                if (graph) cudaGraphDestroy(graph);
                return set_error(cuda_to_status(e1 != cudaSuccess ? e1 : e2), "device gso capture failed");
            }
            const cudaError_t e3 = cudaGraphInstantiate(&G->dexec, graph, 0);
            cudaGraphDestroy(graph);
            if (e3 != cudaSuccess) return set_error(cuda_to_status(e3), "device gso graph: %s", cudaGetErrorString(e3));
            G->ds_captured = S;
        }
        for (int k = 1; k < steps; ++k) LKG_CK(cudaGraphLaunch(G->dexec, st), "device gso step");
    }
    return set_ok();
}

// luciferin, candidates, predictions and the move of one screened step
// (kernel launches only: capturable)
int dev_screened_tail(lkg_gso* G) {
    cudaStream_t st = G->ctx->stream;
    const lkg::GsoDevState& S = G->ds;
    const lkg::GsoDevScreen& X = G->dx;
    LKG_CK(lkg::gso_dev_screen_propose(S, X, st), "device gso step");
    const int ng = (int)G->group_complex.size(), R = X.K + 1;
    for (int gi = 0, g0 = 0; gi < ng; g0 += G->dcounts[gi], ++gi) {
        if (!G->dcounts[gi]) continue;
        int rc = lkg_surrogate_predict(G->sur[gi], G->dcounts[gi] * R, X.cand + (size_t)g0 * R * 7,
                                       X.pred + (size_t)g0 * R);
        if (rc) return rc;
    }
    LKG_CK(lkg::gso_dev_screen_move(S, X, st), "device gso step");
    return set_ok();
}

// the exactly scored (pose, score) pairs of the step just scored (mask set)
// appended to the groups' training sets, in the host's order
int dev_learn(lkg_gso* G, bool all) {
    lkg_ctx* ctx = G->ctx;
    const lkg::GsoDevState& S = G->ds;
    cudaStream_t st = ctx->stream;
    std::vector<double> hp(7 * (size_t)S.n), hs(S.n);
    std::vector<unsigned char> hm(S.n, 1);
    LKG_CK(cudaMemcpyAsync(hp.data(), S.poses, hp.size() * sizeof(double), cudaMemcpyDeviceToHost, st), "device gso learn");
    LKG_CK(cudaMemcpyAsync(hs.data(), S.score, hs.size() * sizeof(double), cudaMemcpyDeviceToHost, st), "device gso learn");
    if (!all) LKG_CK(cudaMemcpyAsync(hm.data(), S.mask, hm.size(), cudaMemcpyDeviceToHost, st), "device gso learn");
    int rc;
    if ((rc = wait_stream(ctx, 300.0)) || (rc = check_status(ctx))) return rc;
    const int ng = (int)G->group_complex.size();
    G->last_counts.assign(ng, 0);
    for (int gi = 0, g0 = 0; gi < ng; g0 += G->dcounts[gi], ++gi)
        for (int i = g0; i < g0 + G->dcounts[gi]; ++i) {
            if (!hm[i]) continue;
            G->tr_pose[gi].insert(G->tr_pose[gi].end(), hp.begin() + 7 * (size_t)i, hp.begin() + 7 * (size_t)(i + 1));
            G->tr_score[gi].push_back(hs[i]);
            G->last_counts[gi]++;
        }
    return set_ok();
}

// the training steps of a screened run on the device (eagerly): plain steps
// whose exact pairs join the training sets; the last one also trains the
// surrogates and makes the first screened move (gso_step does the same on
// the host).  Returns the steps done in *done.
int dev_training_steps(lkg_gso* G, int steps, int* done) {
    cudaStream_t st = G->ctx->stream;
    lkg::GsoDevState& S = G->ds;
    const lkg_screen& c = G->cfg;
    const int ng = (int)G->group_complex.size();
    int rc;
    *done = 0;
    while (*done < steps && G->step < c.train_steps) {
        if ((rc = lkg::plan_launch_masked(G->dplan, S.poses, S.score, S.mask)) || (rc = dev_learn(G, false)))
            return rc;
        if (G->step == c.train_steps - 1) {
            for (int gi = 0; gi < ng; ++gi)
                if ((rc = train_group(G, gi, c.train_epochs, 0))) return rc;
            if ((rc = dev_screened_tail(G))) return rc;
            G->predicted += (int64_t)S.n * (c.candidates + 1);
        } else {
            LKG_CK(lkg::gso_dev_after_scoring(S, st), "device gso step");
        }
        G->step++;
        ++*done;
    }
    return set_ok();
}

// screened steps on the device: every `rescore_every` steps a full exact
// rescoring fine-tunes the surrogates (host-driven, as gso_step does); the
// steps between replay one captured graph
int dev_screened_steps(lkg_gso* G, int steps) {
    lkg_ctx* ctx = G->ctx;
    cudaStream_t st = ctx->stream;
    lkg::GsoDevState& S = G->ds;
    const lkg_screen& c = G->cfg;
    const int ng = (int)G->group_complex.size();
    for (int k = 0; k < steps; ++k) {
        const bool rescore = c.rescore_every > 0 && G->step > c.train_steps &&
                             (G->step - c.train_steps) % c.rescore_every == 0;
        int rc;
        if (rescore) {
            LKG_CK(cudaMemsetAsync(S.mask, 1, (size_t)S.n, st), "device gso rescoring");
            if ((rc = lkg::plan_launch_masked(G->dplan, S.poses, S.score, S.mask))) return rc;
            // the exact pairs train the surrogates (score_phase learn + train_group)
            if ((rc = dev_learn(G, true))) return rc;
            for (int gi = 0; gi < ng; ++gi)
                if ((rc = train_group(G, gi, c.finetune_epochs, (size_t)G->dcounts[gi]))) return rc;
            if ((rc = dev_screened_tail(G))) return rc;
        } else {
            const bool same = G->sexec && std::memcmp(&G->ds_captured, &S, sizeof(S)) == 0 &&
                              std::memcmp(&G->dx_captured, &G->dx, sizeof(G->dx)) == 0;
            if (!same) {
                if (G->sexec) { cudaGraphExecDestroy(G->sexec); G->sexec = nullptr; }
                // one eager step first (host-side queries of the plan and the surrogate)
                if ((rc = lkg::plan_launch_masked(G->dplan, S.poses, S.score, S.mask)) || (rc = dev_screened_tail(G)))
                    return rc;
                G->step++;
                G->predicted += (int64_t)S.n * (c.candidates + 1);
                if (++k == steps) break;
                if (G->step > c.train_steps && c.rescore_every > 0 && (G->step - c.train_steps) % c.rescore_every == 0) {
                    --k;   // the next step is a rescoring one: no capture yet
                    continue;
                }
                LKG_CK(cudaStreamSynchronize(st), "device gso");
                LKG_CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal), "device gso capture");
                rc = lkg::plan_launch_masked(G->dplan, S.poses, S.score, S.mask);
                if (!rc) rc = dev_screened_tail(G);
                cudaGraph_t graph = nullptr;
                const cudaError_t e2 = cudaStreamEndCapture(st, &graph);
                if (rc) { if (graph) cudaGraphDestroy(graph); return rc; }
                if (e2 != cudaSuccess) {
                    if (graph) cudaGraphDestroy(graph);
                    return set_error(cuda_to_status(e2), "device gso capture failed");
                }
                const cudaError_t e3 = cudaGraphInstantiate(&G->sexec, graph, 0);
                cudaGraphDestroy(graph);
                if (e3 != cudaSuccess) return set_error(cuda_to_status(e3), "device gso graph: %s", cudaGetErrorString(e3));
                G->ds_captured = S;
                G->dx_captured = G->dx;
            }
            LKG_CK(cudaGraphLaunch(G->sexec, st), "device gso step");
        }
        G->step++;
        G->predicted += (int64_t)S.n * (c.candidates + 1);
    }
    return set_ok();
}

}  // namespace

extern "C" {

// GSO steps on the device: the state goes up once, every step runs as kernel
// launches (steps between full rescorings replayed from one CUDA graph), and
// the state comes back at the end.  Plain runs: score (unmoved glowworms
// are rescored with the same pose, which gives the same score), luciferin,
// select, move.  Screened runs: the first train_steps steps run on the host
// (they train the surrogates), then score the chosen moves, luciferin, K
// selections, candidate predictions, the per-swarm exact choice and the
// move, as screened_movement does.
int lkg_gso_run_device(lkg_gso* G, int steps) {
    if (!G || steps < 0) return set_error(LKG_ERR_ARG, "bad gso run");
    if (G->screen && G->cfg.random_rank)
        return set_error(LKG_ERR_STATE, "the device GSO screens with the surrogate only (not the ablation)");
    cudaSetDevice(G->ctx->device);
    int rc;
    if (steps == 0 || G->swarms.empty()) return set_ok();
    const double t0 = now_s(), tt0 = G->t_train;
    if ((rc = dev_setup(G, G->screen))) return rc;
    if (G->ds.n == 0) return set_ok();
    const int step0 = G->step;
    if (G->screen) {
        int done = 0;
        if (G->step < G->cfg.train_steps && (rc = dev_training_steps(G, steps, &done))) return rc;
        if (done < steps && (rc = dev_screened_steps(G, steps - done))) return rc;
    } else if ((rc = dev_plain_steps(G, steps))) {
        return rc;
    }
    if ((rc = wait_stream(G->ctx, 300.0)) || (rc = check_status(G->ctx))) return rc;
    if (!G->screen) G->step += steps;
    // a screened run that stopped inside its training steps left a plain move
    const bool screened_move = G->screen && G->step >= G->cfg.train_steps;
    if ((rc = dev_download(G, G->step - step0, screened_move))) return rc;
    G->t_exact += now_s() - t0 - (G->t_train - tt0);
    return set_ok();
}

int lkg_gso_timing(lkg_gso* G, double* out) {
    if (!G || !out) return set_error(LKG_ERR_ARG, "bad timing arguments");
    out[0] = G->t_exact; out[1] = G->t_move; out[2] = G->t_infer; out[3] = G->t_train;
    return set_ok();
}

int lkg_gso_finalize(lkg_gso* G) {
    if (!G) return set_error(LKG_ERR_ARG, "null gso");
    cudaSetDevice(G->ctx->device);
    return score_phase(G, true, false);
}

int lkg_gso_destroy(lkg_gso* G) {
    delete G;
    return set_ok();
}

// rand 0.7.3 StdRng for callers (setup pose generation, tests)
void* lkg_rng_new(uint64_t seed) { return new StdRng(seed); }
double lkg_rng_f64(void* r) { return ((StdRng*)r)->gen_f64(); }
void lkg_rng_free(void* r) { delete (StdRng*)r; }

}  // extern "C"
