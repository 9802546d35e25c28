// liblkg host runtime: contexts, device-resident complexes, persistent
// launches over batches of complexes, and the lkg_* handle API.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <numeric>
#include <thread>

#include "lkg_runtime.h"

namespace lkg {

int max_blocks_score_fast(int threads, int group);
int max_blocks_desolv_fast(int threads, int hcap, int group);
int max_blocks_score_exact(int threads);
int max_blocks_desolv_exact(int threads, int hcap);

namespace {
thread_local int t_status = 0;
thread_local char t_msg[512] = "";
}  // namespace

int set_error(int status, const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(t_msg, sizeof(t_msg), fmt, ap);
    va_end(ap);
    t_status = status;
    return status;
}

int set_ok() {
    t_status = 0;
    t_msg[0] = 0;
    return 0;
}

int cuda_to_status(cudaError_t e) {
    switch (e) {
        case cudaSuccess: return LKG_OK;
        case cudaErrorMemoryAllocation: return LKG_ERR_OOM;
        case cudaErrorNoDevice:
        case cudaErrorInsufficientDriver: return LKG_ERR_NO_DEVICE;
        case cudaErrorInvalidConfiguration:
        case cudaErrorInvalidValue:
        case cudaErrorLaunchOutOfResources:
        case cudaErrorInvalidDeviceFunction:
        case cudaErrorNoKernelImageForDevice: return LKG_ERR_LAUNCH;
        default: return LKG_ERR_DEVICE;
    }
}

// ReceptorField box geometry (grid_dna.rs:45-61)
void field_geometry(const double* c, int n, double lo[3], int dims[3], double* spacing) {
    const double RMAX = 30.0, S = 0.5;
    double mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int i = 0; i < n; ++i)
        for (int a = 0; a < 3; ++a) {
            mn[a] = std::fmin(mn[a], c[3 * i + a]);
            mx[a] = std::fmax(mx[a], c[3 * i + a]);
        }
    for (int a = 0; a < 3; ++a) {
        lo[a] = std::floor(mn[a] - RMAX - 2.0 * S);
        double hi = std::ceil(mx[a] + RMAX + 2.0 * S);
        dims[a] = (int)((hi - lo[a]) / S) + 1;
    }
    *spacing = S;
}

namespace {

template <class T>
cudaError_t upload(DBuf& b, const std::vector<T>& v, cudaStream_t s) {
    cudaError_t e = b.reserve(v.size() * sizeof(T));
    if (e != cudaSuccess) return e;
    if (v.empty()) return cudaSuccess;
    return cudaMemcpyAsync(b.p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, s);
}

// Lower bound of the distance from a point to the nearest receptor atom,
// on cells of RLB_S A over the receptor's box grown by RLB_M A (x fastest).
// Cell A holds max(0, |c_A - c_B| - RLB_S sqrt(3) - 0.01), B the nearest
// cell that holds an atom (cell centres c): a point lies within
// RLB_S sqrt(3) / 2 of its cell's centre and so does every atom of its
// cell, so no point of A is closer to an atom.  |c_A - c_B| comes from an
// exact squared Euclidean distance transform over the cell centres (three
// separable passes of the lower envelope of parabolas, Felzenszwalb and
// Huttenlocher, "Distance transforms of sampled functions", 2012).  A point
// outside the grid is farther than RLB_M from every atom.  The warp kernels
// skip a ligand group whose centre's bound exceeds its candidate radius.
constexpr float RLB_S = 2.0f, RLB_M = 24.0f;
constexpr size_t RLB_MAX_CELLS = (size_t)1 << 26;   // 256 MB of bound at most

// one line of the squared transform: d[q] = min_p (q - p)^2 + f[p]
void edt_line(const float* f, float* d, int n, int* v, float* z) {
    int k = 0;
    v[0] = 0;
    z[0] = -INFINITY;
    z[1] = INFINITY;
    for (int q = 1; q < n; ++q) {
        if (f[q] == INFINITY) continue;
        while (true) {
            if (f[v[k]] == INFINITY) { v[k] = q; z[k] = -INFINITY; z[k + 1] = INFINITY; break; }
            const float sq = ((f[q] + (float)q * q) - (f[v[k]] + (float)v[k] * v[k])) / (2.0f * (q - v[k]));
            if (sq <= z[k]) {
                if (k == 0) { v[0] = q; z[0] = -INFINITY; z[1] = INFINITY; break; }
                --k;
                continue;
            }
            ++k;
            v[k] = q;
            z[k] = sq;
            z[k + 1] = INFINITY;
            break;
        }
    }
    k = 0;
    for (int q = 0; q < n; ++q) {
        while (z[k + 1] < (float)q) ++k;
        d[q] = f[v[k]] == INFINITY ? INFINITY : (float)(q - v[k]) * (q - v[k]) + f[v[k]];
    }
}

}  // namespace

// the bound grid of n receptor atoms (host); dims and origin out; empty
// when the grid would exceed RLB_MAX_CELLS
std::vector<float> receptor_distance_bound(const double* c, int n, int dims[3], float origin[3]) {
    float mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int i = 0; i < n; ++i)
        for (int a = 0; a < 3; ++a) {
            mn[a] = std::min(mn[a], (float)c[3 * i + a]);
            mx[a] = std::max(mx[a], (float)c[3 * i + a]);
        }
    if (n == 0) { mn[0] = mn[1] = mn[2] = 0.f; mx[0] = mx[1] = mx[2] = 0.f; }
    double cells = 1.0;
    for (int a = 0; a < 3; ++a) {
        origin[a] = std::floor(mn[a] - RLB_M);
        const double w = std::ceil(((double)mx[a] + RLB_M - origin[a]) / RLB_S);
        cells *= std::max(1.0, w);
        dims[a] = (int)std::min(std::max(1.0, w), 1e9);
    }
    // an implausibly spread receptor (or non-finite coordinates) gets no
    // bound: the kernels then enumerate every group's rows
    if (!(cells <= (double)RLB_MAX_CELLS)) return {};
    const size_t nc = (size_t)dims[0] * dims[1] * dims[2];
    std::vector<float> g(nc, INFINITY);
    for (int i = 0; i < n; ++i) {
        int ci[3];
        for (int a = 0; a < 3; ++a)
            ci[a] = std::min(std::max((int)std::floor(((float)c[3 * i + a] - origin[a]) / RLB_S), 0), dims[a] - 1);
        g[((size_t)ci[2] * dims[1] + ci[1]) * dims[0] + ci[0]] = 0.f;
    }
    const int L = std::max(dims[0], std::max(dims[1], dims[2]));
    std::vector<float> f(L), d(L), z(L + 1);
    std::vector<int> v(L);
    for (int a = 0; a < 3; ++a) {   // the squared transform along x, then y, then z
        const int n0 = dims[a];
        const size_t stride = a == 0 ? 1 : (a == 1 ? (size_t)dims[0] : (size_t)dims[0] * dims[1]);
        const int o1 = a == 0 ? 1 : 0, o2 = a == 2 ? 1 : 2;
        for (int j2 = 0; j2 < dims[o2]; ++j2)
            for (int j1 = 0; j1 < dims[o1]; ++j1) {
                size_t base = 0;
                const size_t st1 = o1 == 0 ? 1 : (size_t)dims[0], st2 = o2 == 1 ? (size_t)dims[0] : (size_t)dims[0] * dims[1];
                base = (size_t)j1 * st1 + (size_t)j2 * st2;
                for (int q = 0; q < n0; ++q) f[q] = g[base + q * stride];
                edt_line(f.data(), d.data(), n0, v.data(), z.data());
                for (int q = 0; q < n0; ++q) g[base + q * stride] = d[q];
            }
    }
    const float slack = RLB_S * std::sqrt(3.0f) + 0.01f;
    for (size_t i = 0; i < nc; ++i)
        g[i] = g[i] == INFINITY ? RLB_M : std::max(0.f, std::min(RLB_M, std::sqrt(g[i]) * RLB_S - slack));
    return g;
}

namespace {

// receptor: sort by fine cell (x fastest), pack device arrays; the sort and
// packing run on the GPU (lkg_cells.cu) unless the context asks for the
// host build
int build_receptor(lkg_ctx* ctx, const MolIn& R, ComplexRec& cr) {
    ComplexDev& d = cr.d;
    const int n = R.n;
    // the warp kernel's hit queue packs a receptor index into 26 bits
    if (n >= (1 << 26)) return set_error(LKG_ERR_ARG, "receptor has %d atoms (limit %d)", n, (1 << 26) - 1);
    // grid shape: the caller's, else per kernel: the warp kernels enumerate
    // rows per ligand group (coarser rows, finer x trim pay off); cpydock
    // with groups of 32 runs the per-atom kernel, which scans rows per atom
    const bool per_atom = cr.family == LKG_CPYDOCK && ctx->group > 16;
    const float h = ctx->cell_h > 0.f ? ctx->cell_h : (per_atom ? 2.5f : 4.0f), inv_h = 1.0f / h;
    const int xsub = ctx->xsub > 0 ? ctx->xsub : (per_atom ? 4 : 8);
    const float hx = h / (float)xsub, inv_hx = 1.0f / hx;
    const float inv_e[3] = {inv_hx, inv_h, inv_h};
    float mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int i = 0; i < n; ++i)
        for (int a = 0; a < 3; ++a) {
            float v = (float)R.c[3 * i + a];
            mn[a] = std::min(mn[a], v);
            mx[a] = std::max(mx[a], v);
        }
    if (n == 0) { mn[0] = mn[1] = mn[2] = 0.f; mx[0] = mx[1] = mx[2] = 0.f; }
    float o[3];
    int nc[3];
    for (int a = 0; a < 3; ++a) {
        o[a] = std::floor(mn[a]) - 1.0f;
        nc[a] = std::max(1, (int)std::floor((mx[a] - o[a]) * inv_e[a]) + 2);
    }
    const size_t ncell = (size_t)nc[0] * nc[1] * nc[2];
    if (ncell > (size_t)1 << 28) return set_error(LKG_ERR_ARG, "receptor cell grid too large (%zu cells)", ncell);
    if (ctx->setup_on_device) {
        const int st = build_receptor_device(ctx, R, cr, o, nc, inv_e);
        if (st) return st;
    } else {
        // the host counting sort (the check of the device build)
        std::vector<int> cell_of(n), cs(ncell + 1, 0);
        for (int i = 0; i < n; ++i) {
            int ci[3];
            for (int a = 0; a < 3; ++a)
                ci[a] = std::min(std::max((int)std::floor(((float)R.c[3 * i + a] - o[a]) * inv_e[a]), 0), nc[a] - 1);
            cell_of[i] = (ci[2] * nc[1] + ci[1]) * nc[0] + ci[0];
            cs[cell_of[i] + 1]++;
        }
        for (size_t k = 0; k < ncell; ++k) cs[k + 1] += cs[k];
        std::vector<int> cur(cs.begin(), cs.end() - 1), order(n);
        for (int i = 0; i < n; ++i) order[cur[cell_of[i]]++] = i;
        std::vector<float4> pos(n), par(n);
        std::vector<float2> sol(n);
        std::vector<double4> pos64(n), par64(n);
        std::vector<double2> sol64(n);
        for (int k = 0; k < n; ++k) {
            int i = order[k];
            pos[k] = make_float4((float)R.c[3 * i], (float)R.c[3 * i + 1], (float)R.c[3 * i + 2], (float)R.q[i]);
            par[k] = make_float4((float)R.svdw[i], (float)R.rad[i], R.heavy[i] ? 1.f : 0.f, R.excl[i] ? 1.f : 0.f);
            sol[k] = make_float2((float)R.des[i], (float)R.asa[i]);
            pos64[k] = make_double4(R.c[3 * i], R.c[3 * i + 1], R.c[3 * i + 2], R.q[i]);
            par64[k] = make_double4(R.svdw[i], R.rad[i], R.eps[i], R.heavy[i] ? 1.0 : 0.0);
            sol64[k] = make_double2(R.des[i], R.asa[i]);
        }
        cudaStream_t s = ctx->stream;
        LKG_CK(upload(cr.rpos, pos, s), "upload receptor");
        LKG_CK(upload(cr.rpar, par, s), "upload receptor");
        LKG_CK(upload(cr.rsolv, sol, s), "upload receptor");
        LKG_CK(upload(cr.rpos64, pos64, s), "upload receptor");
        LKG_CK(upload(cr.rpar64, par64, s), "upload receptor");
        LKG_CK(upload(cr.rsolv64, sol64, s), "upload receptor");
        LKG_CK(upload(cr.rorig, order, s), "upload receptor");
        LKG_CK(upload(cr.cell_start, cs, s), "upload receptor");
        LKG_CK(cudaStreamSynchronize(s), "upload receptor");
    }
    d.nr = n;
    d.rpos = cr.rpos.as<float4>(); d.rpar = cr.rpar.as<float4>(); d.rsolv = cr.rsolv.as<float2>();
    d.rpos64 = cr.rpos64.as<double4>(); d.rpar64 = cr.rpar64.as<double4>(); d.rsolv64 = cr.rsolv64.as<double2>();
    d.rorig = cr.rorig.as<int>(); d.cell_start = cr.cell_start.as<int>();
    d.ncx = nc[0]; d.ncy = nc[1]; d.ncz = nc[2];
    d.ox = o[0]; d.oy = o[1]; d.oz = o[2]; d.h = h; d.inv_h = inv_h; d.hx = hx; d.inv_hx = inv_hx;
    {   // the distance bound the warp kernels skip far ligand groups with
        int ld[3];
        float lo[3];
        const std::vector<float> lb = receptor_distance_bound(R.c.data(), n, ld, lo);
        if (!lb.empty()) {
            LKG_CK(upload(cr.rlb, lb, ctx->stream), "upload receptor bound");
            LKG_CK(cudaStreamSynchronize(ctx->stream), "upload receptor bound");
        }
        d.rlb = lb.empty() ? nullptr : cr.rlb.as<float>();
        d.rlbx = ld[0]; d.rlby = ld[1]; d.rlbz = ld[2];
        d.rlbox = lo[0]; d.rlboy = lo[1]; d.rlboz = lo[2];
        d.rlb_inv = 1.0f / RLB_S;
        d.rlb_m = RLB_M;
    }
    cr.n_cells = (int)ncell;
    // desolvation hash capacity: >= 2 x receptor atoms up to 2048 slots
    // (16 KB of shared memory in the fast kernel, 24 KB in the exact one); a
    // pose touching more receptor atoms within 6.4 A continues in the launch
    // group's global spill tables (more slots than receptor atoms).  The
    // small table leaves room for several blocks per SM with groups of 16
    // and for L1: on a 101k-atom receptor with a 12k-atom ligand 2048 slots
    // score 1.3x faster than 8192 (whose larger tables spilled less) and
    // 1.24x faster than 1024 (which spill more)
    int cap = 64;
    while (cap < 2 * n && cap < 2048) cap <<= 1;
    d.hcap = cap;
    return set_ok();
}

// recursive coordinate bisection: order idx[0..n) so that every run of G
// consecutive atoms (and every run of a power-of-two number of groups) is
// spatially compact; each split cuts the longest extent at a multiple of G
void bisect_groups(const double* c, int* idx, int n, int G) {
    if (n <= G) return;
    double mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int i = 0; i < n; ++i)
        for (int a = 0; a < 3; ++a) {
            mn[a] = std::fmin(mn[a], c[3 * idx[i] + a]);
            mx[a] = std::fmax(mx[a], c[3 * idx[i] + a]);
        }
    int ax = 0;
    for (int a = 1; a < 3; ++a)
        if (mx[a] - mn[a] > mx[ax] - mn[ax]) ax = a;
    auto key = [&](int u) { const double v = c[3 * u + ax]; return std::isnan(v) ? INFINITY : v; };
    std::sort(idx, idx + n, [&](int u, int v) {
        const double cu = key(u), cv = key(v);
        return cu < cv || (cu == cv && u < v);
    });
    const int ng = (n + G - 1) / G, left = (ng / 2) * G;
    bisect_groups(c, idx, left, G);
    bisect_groups(c, idx + left, n - left, G);
}

// ligand: bisection order in groups of ctx->group atoms
int build_ligand(lkg_ctx* ctx, const MolIn& L, ComplexRec& cr) {
    ComplexDev& d = cr.d;
    const int n = L.n;
    std::vector<int> order(n);
    std::iota(order.begin(), order.end(), 0);
    bisect_groups(L.c.data(), order.data(), n, ctx->group);
    std::vector<float4> pos(n), par(n);
    std::vector<float2> sol(n);
    std::vector<double4> pos64(n), par64(n);
    std::vector<double2> sol64(n);
    for (int k = 0; k < n; ++k) {
        int i = order[k];
        pos[k] = make_float4((float)L.c[3 * i], (float)L.c[3 * i + 1], (float)L.c[3 * i + 2], (float)L.q[i]);
        par[k] = make_float4((float)L.svdw[i], (float)L.rad[i], L.heavy[i] ? 1.f : 0.f, L.excl[i] ? 1.f : 0.f);
        sol[k] = make_float2((float)L.des[i], (float)L.asa[i]);
        pos64[k] = make_double4(L.c[3 * i], L.c[3 * i + 1], L.c[3 * i + 2], L.q[i]);
        par64[k] = make_double4(L.svdw[i], L.rad[i], L.eps[i], L.heavy[i] ? 1.0 : 0.0);
        sol64[k] = make_double2(L.des[i], L.asa[i]);
    }
    // bounding sphere of every group of ctx->group consecutive atoms (ligand
    // frame), for the warp-cooperative kernel's candidate search
    const int G = ctx->group;
    const int ngrp = (n + G - 1) / G;
    std::vector<float4> grp(std::max(ngrp, 1));
    for (int gi = 0; gi < ngrp; ++gi) {
        const int a0 = gi * G, a1 = std::min(n, a0 + G);
        double cen[3] = {0, 0, 0};
        for (int k = a0; k < a1; ++k)
            for (int a = 0; a < 3; ++a) cen[a] += L.c[3 * order[k] + a];
        for (int a = 0; a < 3; ++a) cen[a] /= (a1 - a0);
        double r2 = 0;
        for (int k = a0; k < a1; ++k) {
            double dd = 0;
            for (int a = 0; a < 3; ++a) dd += (L.c[3 * order[k] + a] - cen[a]) * (L.c[3 * order[k] + a] - cen[a]);
            r2 = std::max(r2, dd);
        }
        grp[gi] = make_float4((float)cen[0], (float)cen[1], (float)cen[2], (float)(std::sqrt(r2) * (1.0 + 1e-6) + 1e-3));
    }
    cudaStream_t s = ctx->stream;
    LKG_CK(upload(cr.lgrp, grp, s), "upload ligand");
    LKG_CK(upload(cr.lpos, pos, s), "upload ligand");
    LKG_CK(upload(cr.lpar, par, s), "upload ligand");
    LKG_CK(upload(cr.lsolv, sol, s), "upload ligand");
    LKG_CK(upload(cr.lpos64, pos64, s), "upload ligand");
    LKG_CK(upload(cr.lpar64, par64, s), "upload ligand");
    LKG_CK(upload(cr.lsolv64, sol64, s), "upload ligand");
    LKG_CK(upload(cr.lorig, order, s), "upload ligand");
    LKG_CK(cudaStreamSynchronize(s), "upload ligand");
    d.nl = n;
    d.lpos = cr.lpos.as<float4>(); d.lpar = cr.lpar.as<float4>(); d.lsolv = cr.lsolv.as<float2>();
    d.lpos64 = cr.lpos64.as<double4>(); d.lpar64 = cr.lpar64.as<double4>(); d.lsolv64 = cr.lsolv64.as<double2>();
    d.lorig = cr.lorig.as<int>();
    d.lgrp = cr.lgrp.as<float4>();
    d.group = G;
    d.ntiles = std::max(1, (n + ctx->tile - 1) / ctx->tile);
    return set_ok();
}

int build_field(lkg_ctx* ctx, const MolIn& R, const lkg_field* f, bool build, ComplexRec& cr) {
    ComplexDev& d = cr.d;
    cudaStream_t s = ctx->stream;
    if (f && f->phi) {
        size_t n = (size_t)f->nx * f->ny * f->nz;
        LKG_CK(cr.phi.reserve(n * sizeof(float)), "field alloc");
        LKG_CK(cudaMemcpyAsync(cr.phi.p, f->phi, n * sizeof(float), cudaMemcpyHostToDevice, s), "field upload");
        d.fnx = f->nx; d.fny = f->ny; d.fnz = f->nz;
        d.fox64 = f->ox; d.foy64 = f->oy; d.foz64 = f->oz; d.fsp64 = f->spacing;
    } else if (build && R.n > 0) {
        double lo[3], sp;
        int dims[3];
        field_geometry(R.c.data(), R.n, lo, dims, &sp);
        std::vector<double4> atoms;
        for (int i = 0; i < R.n; ++i)
            if (R.q[i] != 0.0) atoms.push_back(make_double4(R.c[3 * i], R.c[3 * i + 1], R.c[3 * i + 2], R.q[i]));
        size_t n = (size_t)dims[0] * dims[1] * dims[2];
        LKG_CK(cr.phi.reserve(n * sizeof(float)), "field alloc");
        DBuf d_atoms;
        LKG_CK(upload(d_atoms, atoms, s), "field atoms");
        LKG_CK(build_field_device(d_atoms.as<double>(), nullptr, (int)atoms.size(), lo, dims, sp,
                                  cr.phi.as<float>(), s), "field build");
        ctx->launches++;
        LKG_CK(cudaStreamSynchronize(s), "field build");
        d.fnx = dims[0]; d.fny = dims[1]; d.fnz = dims[2];
        d.fox64 = lo[0]; d.foy64 = lo[1]; d.foz64 = lo[2]; d.fsp64 = sp;
    } else {
        d.phi = nullptr; d.fnx = d.fny = d.fnz = 0;
        d.fox = d.foy = d.foz = 0.f; d.fsp = 1.f;
        return set_ok();
    }
    LKG_CK(cudaStreamSynchronize(s), "field upload");
    {   // the kernels read the grid in 4 x 4 x 4 bricks
        d.fbx = (d.fnx + 3) / 4; d.fby = (d.fny + 3) / 4; d.fbz = (d.fnz + 3) / 4;
        DBuf bricks;
        LKG_CK(bricks.reserve((size_t)d.fbx * d.fby * d.fbz * 64 * sizeof(float)), "field bricks");
        LKG_CK(phi_to_bricks(cr.phi.as<float>(), d.fnx, d.fny, d.fnz, bricks.as<float>(), s), "field bricks");
        ctx->launches++;
        LKG_CK(cudaStreamSynchronize(s), "field bricks");
        std::swap(cr.phi.p, bricks.p);
        std::swap(cr.phi.bytes, bricks.bytes);   // the x-fastest grid is freed with `bricks`
    }
    d.phi = cr.phi.as<float>();
    d.fox = (float)d.fox64; d.foy = (float)d.foy64; d.foz = (float)d.foz64; d.fsp = (float)d.fsp64;
    {
        int ex = 0;
        const double m = std::frexp(d.fsp64, &ex);
        d.finv64 = (m == 0.5 && d.fsp64 > 0.0) ? 1.0 / d.fsp64 : 0.0;   // exact reciprocal of 2^k
    }
    return set_ok();
}

int occupancy(lkg_ctx* ctx, bool desolv, bool exact, int threads, int hcap) {
    Occupancy& o = desolv ? ctx->occ_desolv[exact] : ctx->occ_tiles[exact];
    if (o.threads == threads && o.hcap == hcap && o.blocks > 0) return o.blocks;
    int b;
    if (desolv) b = exact ? max_blocks_desolv_exact(threads, hcap) : max_blocks_desolv_fast(threads, hcap, ctx->group);
    else b = exact ? max_blocks_score_exact(threads) : max_blocks_score_fast(threads, ctx->group);
    o.threads = threads; o.hcap = hcap; o.blocks = std::max(1, b);
    return o.blocks;
}

}  // namespace

int complex_create(lkg_ctx* ctx, int family, unsigned flags, int lj_form, const MolIn& rec,
                   const MolIn& lig, const lkg_field* field, bool build_field_flag, double solv_const,
                   int* out_id) {
    if (cudaSetDevice(ctx->device) != cudaSuccess) return set_error(LKG_ERR_DEVICE, "cudaSetDevice failed");
    auto cr = std::make_unique<ComplexRec>();
    cr->family = family;
    int st;
    if ((st = build_receptor(ctx, rec, *cr))) return st;
    if ((st = build_ligand(ctx, lig, *cr))) return st;
    if ((st = build_field(ctx, rec, field, build_field_flag && (flags & F_FAR), *cr))) return st;
    cr->d.flags = flags;
    cr->d.lj_form = lj_form;
    cr->d.solv_const = solv_const;
    ctx->cx.push_back(std::move(cr));
    mark_dirty(ctx);
    *out_id = (int)ctx->cx.size() - 1;
    return set_ok();
}

// The fast kernels find tagged receptor atoms by the sign bit of their heavy
// flag (rpar.z is +-0 or +-1; the kernels only test it against 0): set it
// for the atoms with a tag in rt (sorted order), clear it everywhere else.
static int set_rpar_tag_signs(lkg_ctx* ctx, ComplexRec& cr, const std::vector<int2>* rt) {
    const int nr = cr.d.nr;
    if (nr <= 0) return 0;
    std::vector<float4> par(nr);
    LKG_CK(cudaStreamSynchronize(ctx->stream), "receptor tags");
    LKG_CK(cudaMemcpy(par.data(), cr.rpar.p, nr * sizeof(float4), cudaMemcpyDeviceToHost), "receptor tags");
    for (int k = 0; k < nr; ++k) {
        const bool tagged = rt && ((*rt)[k].x >= 0 || (*rt)[k].y >= 0);
        par[k].z = tagged ? -std::fabs(par[k].z) : std::fabs(par[k].z);
    }
    LKG_CK(cudaMemcpy(cr.rpar.p, par.data(), nr * sizeof(float4), cudaMemcpyHostToDevice), "receptor tags");
    return 0;
}

int complex_set_ligand(lkg_ctx* ctx, int id, const MolIn& lig) {
    if (id < 0 || id >= (int)ctx->cx.size()) return set_error(LKG_ERR_ARG, "bad complex id %d", id);
    ComplexRec& cr = *ctx->cx[id];
    int st = build_ligand(ctx, lig, cr);
    // interface tags refer to the old ligand's atoms
    if (!st && cr.d.iface_words && (st = set_rpar_tag_signs(ctx, cr, nullptr))) return st;
    cr.d.rtag = nullptr; cr.d.ltag = nullptr;
    cr.d.nres_r = cr.d.nres_l = cr.d.nmem = cr.d.iface_words = 0;
    cr.d.iface_form = IF_NONE;
    mark_dirty(ctx);
    return st;
}

// Interface tags of one complex in kernel atom order (see
// lkg_complex_set_restraints).
int complex_set_restraints(lkg_ctx* ctx, int id, const int32_t* rres, int nres_r, const int32_t* lres, int nres_l,
                           const int32_t* mem, int nmem) {
    if (id < 0 || id >= (int)ctx->cx.size()) return set_error(LKG_ERR_ARG, "bad complex id %d", id);
    if (nres_r < 0 || nres_l < 0 || nmem < 0 || (nres_r && !rres) || (nres_l && !lres) || (nmem && !mem))
        return set_error(LKG_ERR_ARG, "bad restraint arguments");
    ComplexRec& cr = *ctx->cx[id];
    const int nr = cr.d.nr, nl = cr.d.nl;
    const long long total = (long long)nres_r + nres_l + nmem;
    if (total > (1ll << 24)) return set_error(LKG_ERR_ARG, "too many restraint residues and membrane beads");
    // the reference's restraint maps hold only residues that have atoms
    auto check = [&](const int32_t* res, int n_atoms, int nres, const char* side) -> int {
        if (!nres) return 0;
        std::vector<char> seen(nres, 0);
        for (int i = 0; i < n_atoms; ++i) {
            const int r = res[i];
            if (r < -1 || r >= nres) return set_error(LKG_ERR_ARG, "%s atom %d: residue %d out of range", side, i, r);
            if (r >= 0) seen[r] = 1;
        }
        for (int r = 0; r < nres; ++r)
            if (!seen[r]) return set_error(LKG_ERR_ARG, "%s restraint residue %d has no atom", side, r);
        return 0;
    };
    int st;
    if ((st = check(rres, nr, nres_r, "receptor")) || (st = check(lres, nl, nres_l, "ligand"))) return st;
    std::vector<int> mbit(nr, -1);
    for (int m = 0; m < nmem; ++m) {
        if (mem[m] < 0 || mem[m] >= nr) return set_error(LKG_ERR_ARG, "membrane bead %d: atom %d out of range", m, mem[m]);
        if (mbit[mem[m]] >= 0) return set_error(LKG_ERR_ARG, "membrane atom %d listed twice", mem[m]);
        mbit[mem[m]] = nres_r + nres_l + m;
    }
    if (total == 0) {   // cleared
        if ((st = set_rpar_tag_signs(ctx, cr, nullptr))) return st;
        cr.d.rtag = nullptr; cr.d.ltag = nullptr;
        cr.d.nres_r = cr.d.nres_l = cr.d.nmem = cr.d.iface_words = 0;
        cr.d.iface_form = IF_NONE;
        mark_dirty(ctx);
        return set_ok();
    }
    std::vector<int> rorig(nr), lorig(nl);
    LKG_CK(cudaStreamSynchronize(ctx->stream), "restraints");
    LKG_CK(cudaMemcpy(rorig.data(), cr.d.rorig, nr * sizeof(int), cudaMemcpyDeviceToHost), "restraints");
    LKG_CK(cudaMemcpy(lorig.data(), cr.d.lorig, nl * sizeof(int), cudaMemcpyDeviceToHost), "restraints");
    std::vector<int2> rt(nr);
    std::vector<int> lt(nl);
    for (int k = 0; k < nr; ++k) {
        const int o = rorig[k];
        rt[k] = make_int2(nres_r ? rres[o] : -1, mbit[o]);
    }
    for (int j = 0; j < nl; ++j) {
        const int r = nres_l ? lres[lorig[j]] : -1;
        lt[j] = r >= 0 ? nres_r + r : -1;
    }
    if ((st = set_rpar_tag_signs(ctx, cr, &rt))) return st;
    LKG_CK(upload(cr.rtag, rt, ctx->stream), "restraint tags");
    LKG_CK(upload(cr.ltag, lt, ctx->stream), "restraint tags");
    LKG_CK(cudaStreamSynchronize(ctx->stream), "restraint tags");
    cr.d.rtag = cr.rtag.as<int2>();
    cr.d.ltag = cr.ltag.as<int>();
    cr.d.nres_r = nres_r; cr.d.nres_l = nres_l; cr.d.nmem = nmem;
    cr.d.iface_words = (int)((total + 31) / 32);
    cr.d.iface_form = cr.family == LKG_DNA ? IF_DNA : cr.family == LKG_VDW ? IF_VDW : IF_SUM;
    mark_dirty(ctx);
    return set_ok();
}

int sync_descriptors(lkg_ctx* ctx) {
    if (!ctx->cx_dirty) return 0;
    std::vector<ComplexDev> v;
    for (auto& c : ctx->cx) v.push_back(c->d);
    LKG_CK(upload(ctx->d_cx, v, ctx->stream), "descriptor upload");
    LKG_CK(cudaStreamSynchronize(ctx->stream), "descriptor upload");
    ctx->cx_dirty = false;
    return 0;
}

cudaError_t Scratch::ensure(size_t units, size_t poses, cudaStream_t s, size_t iface_words) {
    cudaError_t e;
    if (!status.p) {
        if ((e = work_counter.reserve(2 * sizeof(unsigned long long))) != cudaSuccess) return e;
        if ((e = cudaMemsetAsync(work_counter.p, 0, 2 * sizeof(unsigned long long), s)) != cudaSuccess) return e;
        if ((e = status.reserve(4 * sizeof(int))) != cudaSuccess) return e;
        if ((e = cudaMemsetAsync(status.p, 0, 4 * sizeof(int), s)) != cudaSuccess) return e;
    }
    if (units > cap_units) {
        if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return e;
        units = std::max<size_t>(units, 4096);
        if ((e = partials.reserve(units * 4 * sizeof(double))) != cudaSuccess) return e;
        cap_units = units;
    }
    if (poses > cap_poses) {
        if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return e;
        poses = std::max<size_t>(poses, 1024);
        if ((e = pose_counter.reserve(poses * sizeof(int))) != cudaSuccess) return e;
        if ((e = far.reserve(poses * sizeof(double))) != cudaSuccess) return e;
        if ((e = cudaMemsetAsync(pose_counter.p, 0, poses * sizeof(int), s)) != cudaSuccess) return e;
        cap_poses = poses;
    }
    if (iface_words > cap_iface) {   // zero between launches (the kernels clear what they set)
        if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return e;
        if ((e = iface.reserve(iface_words * sizeof(unsigned))) != cudaSuccess) return e;
        cap_iface = iface.bytes / sizeof(unsigned);
        if ((e = cudaMemsetAsync(iface.p, 0, iface.bytes, s)) != cudaSuccess) return e;
    }
    return cudaSuccess;
}

cudaError_t Scratch::ensure_spill(size_t bytes, cudaStream_t s) {
    if (bytes == 0 || (spill.p && bytes <= spill.bytes)) return cudaSuccess;
    cudaError_t e;
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return e;   // a launch may still use the old tables
    if ((e = spill.reserve(bytes)) != cudaSuccess) return e;
    return cudaMemsetAsync(spill.p, 0xff, spill.bytes, s);
}

void Group::pack(char* dst) const {
    const size_t ni = ic.size();
    memcpy(dst, w0.data(), (ni + 1) * sizeof(long long));
    int* t = (int*)(dst + (ni + 1) * sizeof(long long));
    memcpy(t, ic.data(), ni * sizeof(int));
    memcpy(t + ni, ip0.data(), ni * sizeof(int));
    memcpy(t + 2 * ni, inp.data(), ni * sizeof(int));
}

int build_groups(lkg_ctx* ctx, int n_items, const int* ids, const int* counts, Group g[2], size_t* n_poses) {
    for (int i = 0; i < n_items; ++i) {
        if (ids[i] < 0 || ids[i] >= (int)ctx->cx.size()) return set_error(LKG_ERR_ARG, "bad complex id %d", ids[i]);
        if (counts[i] < 0) return set_error(LKG_ERR_ARG, "negative pose count");
    }
    g[0] = Group();
    g[1] = Group();
    g[1].kind = 1;
    long long pose0 = 0;
    for (int i = 0; i < n_items; ++i) {
        const ComplexDev& d = ctx->cx[ids[i]]->d;
        const int k = (d.flags & F_DESOLV) ? 1 : 0;
        if (counts[i] > 0) {
            Group& G = g[k];
            G.ic.push_back(ids[i]);
            G.ip0.push_back((int)pose0);
            G.inp.push_back(counts[i]);
            G.w0.push_back(G.w0.back() + (k ? (long long)counts[i] : (long long)counts[i] * d.ntiles));
            G.hcap = std::max(G.hcap, d.hcap);
            if (k) {   // spill slots: more than the receptor has atoms, so a spill insert always succeeds
                int sc = 64;
                while (sc <= d.nr) sc <<= 1;
                G.spill_cap = std::max(G.spill_cap, sc);
            }
            // one stride for both groups: a pose's bits sit at pose * stride
            g[0].iface_words = g[1].iface_words = std::max(g[0].iface_words, d.iface_words);
        }
        pose0 += counts[i];
    }
    *n_poses = (size_t)pose0;
    return set_ok();
}

long long group_blocks(lkg_ctx* ctx, const Group& G, bool exact) {
    const long long work = std::max(1LL, G.w0.back());
    long long blocks;
    if (G.kind == 0) blocks = (long long)ctx->sm_count * occupancy(ctx, false, exact, ctx->tile, 0);
    else blocks = (long long)ctx->sm_count * occupancy(ctx, true, exact, ctx->desolv_threads, G.hcap);
    return std::max(1LL, std::min(blocks, work));
}

size_t group_spill_bytes(lkg_ctx* ctx, const Group& G, bool exact) {
    if (G.kind != 1 || G.ic.empty()) return 0;
    return (size_t)group_blocks(ctx, G, exact) * (size_t)G.spill_cap * SPILL_SLOT_BYTES;
}

int launch_group(lkg_ctx* ctx, const Group& G, const char* db, Scratch& sc, const double* d_poses,
                 double* d_scores, double* d_parts, int raw_pairs, int solv_only, float* atom_e, float* atom_v,
                 const unsigned char* pose_mask, double* d_iface) {
    const bool exact = ctx->precision == LKG_PREC_EXACT;
    const int ni = (int)G.ic.size();
    LaunchParams p{};
    p.cx = ctx->d_cx.as<ComplexDev>();
    p.item_work0 = (const long long*)db;
    p.item_complex = (const int*)(db + (size_t)(ni + 1) * sizeof(long long));
    p.item_pose0 = p.item_complex + ni;
    p.item_npose = p.item_complex + 2 * ni;
    p.n_items = ni;
    p.total_work = G.w0.back();
    p.tile = ctx->tile;
    p.group = ctx->group;
    p.poses = d_poses;
    p.scores = d_scores;
    p.parts = d_parts;
    p.raw_pairs = raw_pairs;
    p.solv_only = solv_only;
    p.partials = sc.partials.as<double>();
    p.pose_counter = sc.pose_counter.as<int>();
    p.work_counter = sc.work_counter.as<unsigned long long>();
    p.status = sc.status.as<int>();
    p.max_tiles = 0;
    p.atom_elec = atom_e;
    p.atom_vdw = atom_v;
    p.pose_mask = pose_mask;
    p.stage = ctx->stage_tma ? 1 : 0;
    for (int c : G.ic)   // restraints set after the groups were built (a plan made before)
        if (ctx->cx[c]->d.iface_words > G.iface_words)
            return set_error(LKG_ERR_STATE, "complex %d has restraints the prepared batch has no room for", c);
    if (G.iface_words > 0) {   // callers size sc.iface for their poses x stride
        if (!sc.iface.p) return set_error(LKG_ERR_STATE, "interface scratch missing");
        p.iface = sc.iface.as<unsigned>();
        p.iface_stride = G.iface_words;
    }
    p.iface_out = d_iface;
    cudaError_t e;
    const long long blocks = group_blocks(ctx, G, exact);
    if (G.kind == 0) {
        e = exact ? launch_score_exact(p, ctx->tile, (int)blocks, ctx->stream)
                  : launch_score_fast(p, ctx->tile, (int)blocks, ctx->stream);
    } else {
        int threads = ctx->desolv_threads;
        size_t smem = desolv_smem_bytes(G.hcap, exact);
        if (smem > 227 * 1024) return set_error(LKG_ERR_CAPACITY, "desolvation hash too large");
        const size_t need = group_spill_bytes(ctx, G, exact);
        if (need > sc.spill.bytes || !sc.spill.p) {
            // tables are sized before capture by the callers; grow here only outside a capture
            cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
            cudaStreamIsCapturing(ctx->stream, &cs);
            if (cs != cudaStreamCaptureStatusNone)
                return set_error(LKG_ERR_STATE, "desolvation spill tables not sized before the capture");
            LKG_CK(sc.ensure_spill(need, ctx->stream), "spill tables");
        }
        p.spill = sc.spill.as<unsigned char>();
        p.spill_cap = G.spill_cap;
        // the fast warp kernel (groups up to 16) takes the far field from a
        // pass of its own (k_far_poses), launched first on the same stream
        if (!exact && ctx->group <= 16 && !solv_only) {
            p.far = sc.far.as<double>();
            e = launch_far_poses(p, (int)std::min<long long>(p.total_work, (long long)ctx->sm_count * 8),
                                 ctx->stream);
            if (e != cudaSuccess) return set_error(cuda_to_status(e), "far-field launch: %s", cudaGetErrorString(e));
            ctx->launches++;
        }
        e = exact ? launch_desolv_exact(p, threads, (int)blocks, G.hcap, ctx->stream)
                  : launch_desolv_fast(p, threads, (int)blocks, G.hcap, ctx->stream);
    }
    if (e != cudaSuccess) return set_error(cuda_to_status(e), "score launch: %s", cudaGetErrorString(e));
    ctx->launches++;
    return set_ok();
}

int launch_items(lkg_ctx* ctx, int n_items, const int* ids, const int* counts, const double* d_poses,
                 double* d_scores, double* d_parts, int raw_pairs, int solv_only, float* atom_e,
                 float* atom_v, double* d_iface) {
    if (n_items <= 0) return set_ok();
    Group g[2];
    size_t n_poses = 0;
    int st;
    if ((st = build_groups(ctx, n_items, ids, counts, g, &n_poses))) return st;
    if (n_poses == 0) return set_ok();
    if ((st = sync_descriptors(ctx))) return st;
    const size_t units = std::max<size_t>(g[0].w0.back(), 1);
    LKG_CK(ctx->scratch.ensure(units, n_poses, ctx->stream, n_poses * (size_t)g[0].iface_words), "scratch");
    const size_t b0 = (g[0].bytes() + 255) & ~(size_t)255, b1 = (g[1].bytes() + 255) & ~(size_t)255;
    std::vector<char> packed(b0 + b1, 0);
    g[0].pack(packed.data());
    g[1].pack(packed.data() + b0);
    if (packed != ctx->last_items || !ctx->d_items.p) {
        // new tables: the previous upload may still be reading the staging buffer
        LKG_CK(cudaStreamSynchronize(ctx->stream), "item staging");
        LKG_CK(ctx->h_items.reserve(b0 + b1), "item staging");
        LKG_CK(ctx->d_items.reserve(b0 + b1), "item staging");
        memcpy(ctx->h_items.p, packed.data(), b0 + b1);
        LKG_CK(cudaMemcpyAsync(ctx->d_items.p, ctx->h_items.p, b0 + b1, cudaMemcpyHostToDevice, ctx->stream),
               "item upload");
        ctx->last_items.swap(packed);
    }
    for (int k = 0; k < 2; ++k) {
        if (g[k].ic.empty()) continue;
        st = launch_group(ctx, g[k], ctx->d_items.as<char>() + (k ? b0 : 0), ctx->scratch, d_poses, d_scores, d_parts,
                          raw_pairs, solv_only, atom_e, atom_v, nullptr, d_iface);
        if (st) return st;
    }
    return set_ok();
}

int wait_stream(lkg_ctx* ctx, double timeout_s) {
    // bounded host poll: the kernels hold no unbounded waits, but a device
    // that stops answering must still surface as an error, not a hang
    auto t0 = std::chrono::steady_clock::now();
    int spins = 0;
    for (;;) {
        cudaError_t e = cudaStreamQuery(ctx->stream);
        if (e == cudaSuccess) return set_ok();
        if (e != cudaErrorNotReady) return set_error(cuda_to_status(e), "stream: %s", cudaGetErrorString(e));
        double el = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        if (el > timeout_s) return set_error(LKG_ERR_TIMEOUT, "stream did not finish within %.0f s", timeout_s);
        if (++spins < 2000) std::this_thread::yield();
        else std::this_thread::sleep_for(std::chrono::microseconds(50));
    }
}

int check_status_word(int* d_status) {
    if (!d_status) return set_ok();
    int h[4] = {0, 0, 0, 0};
    LKG_CK(cudaMemcpy(h, d_status, sizeof(h), cudaMemcpyDeviceToHost), "status read");
    if (h[0] & 1) {
        cudaMemset(d_status, 0, sizeof(h));
        return set_error(LKG_ERR_CAPACITY, "desolvation hash overflow (too many receptor atoms within 6.4 A of one pose)");
    }
    if (h[0] & 2) {
        cudaMemset(d_status, 0, sizeof(h));
        return set_error(LKG_ERR_STATE, "restraints or membrane set after the batch was prepared: prepare it again");
    }
    if (h[0] & 8) {
        cudaMemset(d_status, 0, sizeof(h));
        return set_error(LKG_ERR_TIMEOUT, "a staged candidate copy did not complete in time");
    }
    return set_ok();
}

int check_status(lkg_ctx* ctx) { return check_status_word(ctx->scratch.status.as<int>()); }

}  // namespace lkg

using namespace lkg;

// ---------------------------------------------------------------------------
// C ABI: status, device, context, complexes, scoring
// ---------------------------------------------------------------------------
extern "C" {

const char* lkg_status_string(int s) {
    switch (s) {
        case LKG_OK: return "ok";
        case LKG_ERR_ARG: return "invalid argument";
        case LKG_ERR_OOM: return "device out of memory";
        case LKG_ERR_LAUNCH: return "kernel launch failed";
        case LKG_ERR_TIMEOUT: return "timed out";
        case LKG_ERR_DEVICE: return "device error";
        case LKG_ERR_CAPACITY: return "device capacity exceeded";
        case LKG_ERR_NO_DEVICE: return "no CUDA device";
        case LKG_ERR_STATE: return "invalid state";
        default: return "unknown status";
    }
}

int lkg_last_status(void) { return t_status; }
const char* lkg_last_error(void) { return t_msg; }
const char* lkg_version(void) { return "lkg 0.1 (sm_100a)"; }

int lkg_device_available(void) {
    int n = 0;
    return cudaGetDeviceCount(&n) == cudaSuccess && n > 0 ? 1 : 0;
}

int lkg_ctx_create(int device, lkg_ctx** out) {
    if (!out) return set_error(LKG_ERR_ARG, "null out");
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) return set_error(LKG_ERR_NO_DEVICE, "no CUDA device");
    if (device < 0 || device >= n) return set_error(LKG_ERR_ARG, "device %d out of range", device);
    LKG_CK(cudaSetDevice(device), "cudaSetDevice");
    auto* c = new lkg_ctx();
    c->device = device;
    cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, device);
    cudaError_t e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) { delete c; return set_error(cuda_to_status(e), "stream create: %s", cudaGetErrorString(e)); }
    c->own_stream = true;
    *out = c;
    return set_ok();
}

int lkg_ctx_destroy(lkg_ctx* ctx) {
    if (!ctx) return set_ok();
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    if (ctx->own_stream && ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
    return set_ok();
}

int lkg_ctx_set_precision(lkg_ctx* ctx, int precision) {
    if (!ctx || (precision != LKG_PREC_FAST && precision != LKG_PREC_EXACT))
        return set_error(LKG_ERR_ARG, "bad precision");
    ctx->precision = precision;
    return set_ok();
}

int lkg_ctx_set_tiles(lkg_ctx* ctx, int threads, int cell_milli) {
    if (!ctx) return set_error(LKG_ERR_ARG, "null ctx");
    if (threads) {
        if (threads != 64 && threads != 128 && threads != 256) return set_error(LKG_ERR_ARG, "tile must be 64, 128 or 256");
        if (!ctx->cx.empty() && threads != ctx->tile) return set_error(LKG_ERR_STATE, "tile fixed once complexes exist");
        ctx->tile = threads;
    }
    if (cell_milli) {
        if (cell_milli < 1500 || cell_milli > 10000) return set_error(LKG_ERR_ARG, "cell edge must be 1.5..10 A");
        if (!ctx->cx.empty()) return set_error(LKG_ERR_STATE, "cell edge fixed once complexes exist");
        ctx->cell_h = cell_milli / 1000.0f;
    }
    return set_ok();
}

int lkg_ctx_set_group(lkg_ctx* ctx, int group) {
    if (!ctx) return set_error(LKG_ERR_ARG, "null ctx");
    if (group != 4 && group != 8 && group != 16 && group != 32)
        return set_error(LKG_ERR_ARG, "group must be 4, 8, 16 or 32");
    if (!ctx->cx.empty() && group != ctx->group) return set_error(LKG_ERR_STATE, "group fixed once complexes exist");
    ctx->group = group;
    return set_ok();
}

int lkg_ctx_set_xsub(lkg_ctx* ctx, int xsub) {
    if (!ctx) return set_error(LKG_ERR_ARG, "null ctx");
    if (xsub < 1 || xsub > 8) return set_error(LKG_ERR_ARG, "xsub must be 1..8");
    if (!ctx->cx.empty() && xsub != ctx->xsub) return set_error(LKG_ERR_STATE, "xsub fixed once complexes exist");
    ctx->xsub = xsub;
    return set_ok();
}

int lkg_ctx_set_staging(lkg_ctx* ctx, int tma) {
    if (!ctx) return set_error(LKG_ERR_ARG, "null ctx");
    ctx->stage_tma = tma != 0;
    return set_ok();
}

int lkg_ctx_set_setup(lkg_ctx* ctx, int on_device) {
    if (!ctx) return set_error(LKG_ERR_ARG, "null ctx");
    ctx->setup_on_device = on_device != 0;
    return set_ok();
}

int lkg_ctx_set_stream(lkg_ctx* ctx, void* stream) {
    if (!ctx) return set_error(LKG_ERR_ARG, "null ctx");
    cudaStreamSynchronize(ctx->stream);
    if (ctx->own_stream) cudaStreamDestroy(ctx->stream);
    ctx->stream = (cudaStream_t)stream;
    ctx->own_stream = false;
    return set_ok();
}

void* lkg_ctx_stream(lkg_ctx* ctx) { return ctx ? (void*)ctx->stream : nullptr; }
int64_t lkg_ctx_launches(lkg_ctx* ctx) { return ctx ? ctx->launches : 0; }

}  // extern "C"

namespace {

int mol_from_api(const lkg_mol* m, int family, bool receptor_side, MolIn& out, double* solv_const) {
    (void)receptor_side;
    if (!m || m->n < 0 || (m->n > 0 && (!m->coords || !m->ele || !m->vdw || !m->radius)))
        return set_error(LKG_ERR_ARG, "molecule arrays missing");
    const int n = m->n;
    out.n = n;
    out.c.assign(m->coords, m->coords + 3 * n);
    out.q.assign(m->ele, m->ele + n);
    out.eps.assign(m->vdw, m->vdw + n);
    out.svdw.resize(n);
    for (int i = 0; i < n; ++i) out.svdw[i] = std::sqrt(out.eps[i]);
    out.rad.assign(m->radius, m->radius + n);
    out.heavy.assign(n, 0);
    if (m->heavy) out.heavy.assign(m->heavy, m->heavy + n);
    out.excl.assign(n, 0);
    out.des.assign(n, 0.0);
    out.asa.assign(n, 0.0);
    if (family == LKG_CPYDOCK) {
        if (!m->hyd || !m->des || !m->asa) return set_error(LKG_ERR_ARG, "cpydock needs hyd, des and asa");
        // C-binary exclusion view of the hydrogens array (cpydock.rs:808-819)
        for (int i = 0; i < n; ++i) out.excl[i] = (i % 2 == 0 && m->hyd[i / 2] != 0) ? 1 : 0;
        out.des.assign(m->des, m->des + n);
        out.asa.assign(m->asa, m->asa + n);
        for (int i = 0; i < n; ++i)
            if (out.asa[i] < 0.0) *solv_const += out.asa[i] * out.des[i];
    }
    return 0;
}

}  // namespace

extern "C" {

int lkg_complex_add(lkg_ctx* ctx, int family, const lkg_mol* rec, const lkg_mol* lig,
                    const lkg_field* field, int* complex_id) {
    if (!ctx || !complex_id) return set_error(LKG_ERR_ARG, "null argument");
    unsigned flags;
    int lj;
    switch (family) {
        case LKG_DNA: flags = F_FAR | F_ELEC | F_CLASH; lj = LJ_SVDW; break;
        case LKG_PYDOCK: flags = F_FAR | F_ELEC; lj = LJ_SVDW; break;
        case LKG_VDW: flags = 0; lj = LJ_SQRT; break;
        case LKG_CPYDOCK: flags = F_FAR | F_ELEC | F_DESOLV; lj = LJ_POW; break;
        default: return set_error(LKG_ERR_ARG, "unknown family %d", family);
    }
    MolIn R, L;
    double solv_const = 0.0;
    int st;
    if ((st = mol_from_api(rec, family, true, R, &solv_const))) return st;
    if ((st = mol_from_api(lig, family, false, L, &solv_const))) return st;
    if (L.n == 0) return set_error(LKG_ERR_ARG, "empty ligand");
    return complex_create(ctx, family, flags, lj, R, L, field, true, solv_const, complex_id);
}

int lkg_complex_info(lkg_ctx* ctx, int id, int* nr, int* nl, int* n_cells) {
    if (!ctx || id < 0 || id >= (int)ctx->cx.size()) return set_error(LKG_ERR_ARG, "bad complex id");
    if (nr) *nr = ctx->cx[id]->d.nr;
    if (nl) *nl = ctx->cx[id]->d.nl;
    if (n_cells) *n_cells = ctx->cx[id]->n_cells;
    return set_ok();
}

int lkg_score_device(lkg_ctx* ctx, int id, int n, const double* d_poses, double* d_scores, double* d_parts) {
    if (!ctx) return set_error(LKG_ERR_ARG, "null ctx");
    if (n == 0) return set_ok();
    if (n < 0 || !d_poses || !d_scores) return set_error(LKG_ERR_ARG, "bad pose buffer");
    cudaSetDevice(ctx->device);
    return launch_items(ctx, 1, &id, &n, d_poses, d_scores, d_parts, 0, 0, nullptr, nullptr);
}

int lkg_score_multi_device(lkg_ctx* ctx, int n_items, const int* ids, const int* counts,
                           const double* d_poses, double* d_scores, double* d_parts) {
    if (!ctx || n_items < 0 || (n_items && (!ids || !counts))) return set_error(LKG_ERR_ARG, "bad items");
    cudaSetDevice(ctx->device);
    return launch_items(ctx, n_items, ids, counts, d_poses, d_scores, d_parts, 0, 0, nullptr, nullptr);
}

// host-buffer scoring of one complex; parts (N x 4) and iface (N x 3) optional
static int score_host(lkg_ctx* ctx, int id, int n, const double* poses, double* scores, double* parts,
                      double* iface) {
    if (!ctx) return set_error(LKG_ERR_ARG, "null ctx");
    if (n == 0) return set_ok();
    if (n < 0 || !poses || !scores) return set_error(LKG_ERR_ARG, "bad pose buffer");
    cudaSetDevice(ctx->device);
    const size_t pb = (size_t)n * 7 * sizeof(double), ob = (size_t)n * sizeof(double),
                 qb = (size_t)n * 4 * sizeof(double), ib = (size_t)n * 3 * sizeof(double);
    LKG_CK(ctx->h_poses.reserve(pb), "staging");
    LKG_CK(ctx->h_out.reserve(ob + qb + ib), "staging");
    LKG_CK(ctx->d_poses.reserve(pb), "staging");
    LKG_CK(ctx->d_scores.reserve(ob), "staging");
    LKG_CK(ctx->d_parts.reserve(qb + ib), "staging");
    memcpy(ctx->h_poses.p, poses, pb);
    LKG_CK(cudaMemcpyAsync(ctx->d_poses.p, ctx->h_poses.p, pb, cudaMemcpyHostToDevice, ctx->stream), "pose upload");
    double* d_iface = iface ? (double*)(ctx->d_parts.as<char>() + qb) : nullptr;
    if (iface) LKG_CK(cudaMemsetAsync(d_iface, 0, ib, ctx->stream), "interface output");
    int st = launch_items(ctx, 1, &id, &n, ctx->d_poses.as<double>(), ctx->d_scores.as<double>(),
                          parts ? ctx->d_parts.as<double>() : nullptr, 0, 0, nullptr, nullptr, d_iface);
    if (st) return st;
    LKG_CK(cudaMemcpyAsync(ctx->h_out.p, ctx->d_scores.p, ob, cudaMemcpyDeviceToHost, ctx->stream), "score readback");
    if (parts)
        LKG_CK(cudaMemcpyAsync(ctx->h_out.as<char>() + ob, ctx->d_parts.p, qb, cudaMemcpyDeviceToHost, ctx->stream),
               "parts readback");
    if (iface)
        LKG_CK(cudaMemcpyAsync(ctx->h_out.as<char>() + ob + qb, d_iface, ib, cudaMemcpyDeviceToHost, ctx->stream),
               "interface readback");
    if ((st = wait_stream(ctx, 300.0))) return st;
    if ((st = check_status(ctx))) return st;
    memcpy(scores, ctx->h_out.p, ob);
    if (parts) memcpy(parts, ctx->h_out.as<char>() + ob, qb);
    if (iface) memcpy(iface, ctx->h_out.as<char>() + ob + qb, ib);
    return set_ok();
}

int lkg_score(lkg_ctx* ctx, int id, int n, const double* poses, double* scores, double* parts) {
    return score_host(ctx, id, n, poses, scores, parts, nullptr);
}

int lkg_score_interface(lkg_ctx* ctx, int id, int n, const double* poses, double* scores, double* iface) {
    if (!iface) return set_error(LKG_ERR_ARG, "null interface output");
    return score_host(ctx, id, n, poses, scores, nullptr, iface);
}

int lkg_complex_set_restraints(lkg_ctx* ctx, int id, const int32_t* rec_residue, int n_rec_res,
                               const int32_t* lig_residue, int n_lig_res, const int32_t* membrane, int n_membrane) {
    if (!ctx) return set_error(LKG_ERR_ARG, "null ctx");
    cudaSetDevice(ctx->device);
    return complex_set_restraints(ctx, id, rec_residue, n_rec_res, lig_residue, n_lig_res, membrane, n_membrane);
}

int lkg_score_multi(lkg_ctx* ctx, int n_items, const int* ids, const int* counts, const double* poses,
                    double* scores, double* parts) {
    if (!ctx || n_items < 0 || (n_items && (!ids || !counts || !poses || !scores)))
        return set_error(LKG_ERR_ARG, "bad items");
    size_t n = 0;
    for (int i = 0; i < n_items; ++i) {
        if (counts[i] < 0) return set_error(LKG_ERR_ARG, "negative pose count");
        n += (size_t)counts[i];
    }
    if (n == 0) return set_ok();
    cudaSetDevice(ctx->device);
    const size_t pb = n * 7 * sizeof(double), ob = n * sizeof(double), qb = n * 4 * sizeof(double);
    LKG_CK(ctx->d_poses.reserve(pb), "staging");
    LKG_CK(ctx->d_scores.reserve(ob), "staging");
    LKG_CK(ctx->d_parts.reserve(qb), "staging");
    // page-locked caller buffers are DMA'd directly; pageable ones go
    // through the context's pinned staging buffer
    auto pinned = [](const void* p) {
        cudaPointerAttributes a;
        if (cudaPointerGetAttributes(&a, p) != cudaSuccess) { cudaGetLastError(); return false; }
        return a.type == cudaMemoryTypeHost;
    };
    const bool pin_in = pinned(poses), pin_out = pinned(scores) && (!parts || pinned(parts));
    const double* src = poses;
    if (!pin_in) {
        LKG_CK(ctx->h_poses.reserve(pb), "staging");
        memcpy(ctx->h_poses.p, poses, pb);
        src = ctx->h_poses.as<double>();
    }
    LKG_CK(cudaMemcpyAsync(ctx->d_poses.p, src, pb, cudaMemcpyHostToDevice, ctx->stream), "pose upload");
    int st = launch_items(ctx, n_items, ids, counts, ctx->d_poses.as<double>(), ctx->d_scores.as<double>(),
                          parts ? ctx->d_parts.as<double>() : nullptr, 0, 0, nullptr, nullptr);
    if (st) return st;
    double* dst_s = scores;
    double* dst_p = parts;
    if (!pin_out) {
        LKG_CK(ctx->h_out.reserve(ob + qb), "staging");
        dst_s = ctx->h_out.as<double>();
        dst_p = parts ? (double*)(ctx->h_out.as<char>() + ob) : nullptr;
    }
    LKG_CK(cudaMemcpyAsync(dst_s, ctx->d_scores.p, ob, cudaMemcpyDeviceToHost, ctx->stream), "score readback");
    if (parts) LKG_CK(cudaMemcpyAsync(dst_p, ctx->d_parts.p, qb, cudaMemcpyDeviceToHost, ctx->stream), "parts readback");
    if ((st = wait_stream(ctx, 300.0))) return st;
    if ((st = check_status(ctx))) return st;
    if (!pin_out) {
        memcpy(scores, dst_s, ob);
        if (parts) memcpy(parts, dst_p, qb);
    }
    return set_ok();
}

int lkg_field_build(const double* coords, const double* charges, int32_t n, double origin[3],
                    int32_t dims[3], double* spacing, float* phi) {
    if (!coords || !charges || n <= 0 || !origin || !dims || !spacing) return set_error(LKG_ERR_ARG, "bad field args");
    int d[3];
    field_geometry(coords, n, origin, d, spacing);
    for (int a = 0; a < 3; ++a) dims[a] = d[a];
    if (!phi) return set_ok();
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return set_error(LKG_ERR_NO_DEVICE, "no CUDA device");
    std::vector<double4> atoms;
    for (int i = 0; i < n; ++i)
        if (charges[i] != 0.0) atoms.push_back(make_double4(coords[3 * i], coords[3 * i + 1], coords[3 * i + 2], charges[i]));
    size_t np = (size_t)d[0] * d[1] * d[2];
    DBuf d_atoms, d_phi;
    LKG_CK(upload(d_atoms, atoms, 0), "field atoms");
    LKG_CK(d_phi.reserve(np * sizeof(float)), "field alloc");
    LKG_CK(build_field_device(d_atoms.as<double>(), nullptr, (int)atoms.size(), origin, d, *spacing,
                              d_phi.as<float>(), 0), "field build");
    LKG_CK(cudaMemcpy(phi, d_phi.p, np * sizeof(float), cudaMemcpyDeviceToHost), "field readback");
    return set_ok();
}

}  // extern "C"

// ---------------------------------------------------------------------------
// plans: a batch prepared once (descriptors, item tables, own scratch); its
// launch is kernel launches only, so it can be captured in a CUDA graph
// ---------------------------------------------------------------------------
struct lkg_plan {
    lkg_ctx* ctx = nullptr;
    lkg::Group g[2];
    size_t b0 = 0, n_poses = 0;
    lkg::DBuf d_tables;
    lkg::Scratch scratch;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    const void* captured_cx = nullptr;
    uint64_t captured_version = 0;
    int captured_launches = 0;
};

extern "C" {

int lkg_plan_create(lkg_ctx* ctx, int n_items, const int* ids, const int* counts, lkg_plan** out) {
    if (!ctx || !out || n_items <= 0 || !ids || !counts) return set_error(LKG_ERR_ARG, "bad plan arguments");
    cudaSetDevice(ctx->device);
    auto* P = new lkg_plan();
    P->ctx = ctx;
    int st = build_groups(ctx, n_items, ids, counts, P->g, &P->n_poses);
    if (!st) st = sync_descriptors(ctx);
    if (st) { delete P; return st; }
    const size_t b0 = (P->g[0].bytes() + 255) & ~(size_t)255, b1 = (P->g[1].bytes() + 255) & ~(size_t)255;
    std::vector<char> packed(b0 + b1, 0);
    P->g[0].pack(packed.data());
    P->g[1].pack(packed.data() + b0);
    P->b0 = b0;
    cudaError_t e;
    if ((e = P->d_tables.reserve(b0 + b1)) != cudaSuccess ||
        (e = cudaMemcpy(P->d_tables.p, packed.data(), b0 + b1, cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = P->scratch.ensure(std::max<size_t>(P->g[0].w0.back(), 1), std::max<size_t>(P->n_poses, 1), ctx->stream,
                               P->n_poses * (size_t)P->g[0].iface_words)) != cudaSuccess ||
        (e = P->scratch.ensure_spill(std::max(group_spill_bytes(ctx, P->g[1], false),
                                              group_spill_bytes(ctx, P->g[1], true)), ctx->stream)) != cudaSuccess ||
        (e = cudaStreamSynchronize(ctx->stream)) != cudaSuccess) {
        delete P;
        return set_error(cuda_to_status(e), "plan setup: %s", cudaGetErrorString(e));
    }
    *out = P;
    return set_ok();
}

int lkg_plan_launch(lkg_plan* P, const double* d_poses, double* d_scores, double* d_parts) {
    if (!P || !d_poses || !d_scores) return set_error(LKG_ERR_ARG, "bad plan launch");
    if (P->ctx->cx_dirty) {   // a complex changed since the plan was made: upload its descriptor first
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        cudaStreamIsCapturing(P->ctx->stream, &cs);
        if (cs != cudaStreamCaptureStatusNone) return set_error(LKG_ERR_STATE, "complexes changed during capture");
        int st = sync_descriptors(P->ctx);
        if (st) return st;
    }
    for (int k = 0; k < 2; ++k) {
        if (P->g[k].ic.empty()) continue;
        int st = launch_group(P->ctx, P->g[k], P->d_tables.as<char>() + (k ? P->b0 : 0), P->scratch, d_poses,
                              d_scores, d_parts, 0, 0, nullptr, nullptr);
        if (st) return st;
    }
    return set_ok();
}

}  // extern "C"

namespace lkg {
int plan_launch_masked(lkg_plan* P, const double* d_poses, double* d_scores, const unsigned char* d_mask) {
    if (!P || !d_poses || !d_scores) return set_error(LKG_ERR_ARG, "bad plan launch");
    for (int k = 0; k < 2; ++k) {
        if (P->g[k].ic.empty()) continue;
        int st = launch_group(P->ctx, P->g[k], P->d_tables.as<char>() + (k ? P->b0 : 0), P->scratch, d_poses,
                              d_scores, nullptr, 0, 0, nullptr, nullptr, d_mask);
        if (st) return st;
    }
    return set_ok();
}
}  // namespace lkg

extern "C" {

int lkg_plan_capture(lkg_plan* P, const double* d_poses, double* d_scores, double* d_parts, int n_launches) {
    if (!P || n_launches <= 0) return set_error(LKG_ERR_ARG, "bad capture");
    lkg_ctx* ctx = P->ctx;
    cudaSetDevice(ctx->device);
    if (P->exec) { cudaGraphExecDestroy(P->exec); P->exec = nullptr; }
    if (P->graph) { cudaGraphDestroy(P->graph); P->graph = nullptr; }
    // occupancy queries are host-side; make them before capture
    lkg_plan_launch(P, d_poses, d_scores, d_parts);
    LKG_CK(cudaStreamSynchronize(ctx->stream), "pre-capture launch");
    LKG_CK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal), "begin capture");
    int st = 0;
    for (int i = 0; i < n_launches && !st; ++i) st = lkg_plan_launch(P, d_poses, d_scores, d_parts);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(ctx->stream, &g);
    if (st) { if (g) cudaGraphDestroy(g); return st; }
    if (e != cudaSuccess) return set_error(cuda_to_status(e), "end capture: %s", cudaGetErrorString(e));
    P->graph = g;
    LKG_CK(cudaGraphInstantiate(&P->exec, g, 0), "graph instantiate");
    P->captured_cx = ctx->d_cx.p;
    P->captured_version = ctx->cx_version;
    P->captured_launches = n_launches * ((P->g[0].ic.empty() ? 0 : 1) + (P->g[1].ic.empty() ? 0 : 1));
    return set_ok();
}

int lkg_plan_replay(lkg_plan* P) {
    if (!P || !P->exec) return set_error(LKG_ERR_STATE, "no captured graph");
    if (P->captured_cx != P->ctx->d_cx.p || P->captured_version != P->ctx->cx_version)
        return set_error(LKG_ERR_STATE, "complexes were added or changed after capture; capture again");
    cudaSetDevice(P->ctx->device);
    LKG_CK(cudaGraphLaunch(P->exec, P->ctx->stream), "graph launch");
    P->ctx->launches += P->captured_launches;
    return set_ok();
}

int lkg_plan_destroy(lkg_plan* P) {
    if (!P) return set_ok();
    cudaSetDevice(P->ctx->device);
    cudaStreamSynchronize(P->ctx->stream);
    if (P->exec) cudaGraphExecDestroy(P->exec);
    if (P->graph) cudaGraphDestroy(P->graph);
    delete P;
    return set_ok();
}

int lkg_ctx_sync(lkg_ctx* ctx) {
    if (!ctx) return set_error(LKG_ERR_ARG, "null ctx");
    cudaSetDevice(ctx->device);
    int st = wait_stream(ctx, 300.0);
    if (st) return st;
    st = check_status(ctx);
    if (st) return st;
    return ctx->noalloc_used ? noalloc_check_status(ctx) : set_ok();
}

int lkg_plan_sync(lkg_plan* P) {
    if (!P) return set_error(LKG_ERR_ARG, "null plan");
    cudaSetDevice(P->ctx->device);
    int st = wait_stream(P->ctx, 300.0);
    if (st) return st;
    return check_status_word(P->scratch.status.as<int>());
}

}  // extern "C"

extern "C" {

// The lower bound of the distance to the nearest of n receptor atoms that
// the warp kernels skip far ligand groups with, at m points (host; for
// checks of the bound).
int lkg_receptor_distance_bound(const double* coords, int32_t n, const double* points, int32_t m, float* out) {
    if (n < 0 || m < 0 || (n > 0 && !coords) || (m > 0 && (!points || !out)))
        return set_error(LKG_ERR_ARG, "bad distance-bound args");
    int dims[3];
    float o[3];
    const std::vector<float> g = receptor_distance_bound(coords, n, dims, o);
    for (int i = 0; i < m && g.empty(); ++i) out[i] = 0.f;   // no bound: 0 bounds every distance
    for (int i = 0; i < m && !g.empty(); ++i) {
        int ix[3];
        bool inside = true;
        for (int a = 0; a < 3; ++a) {
            ix[a] = (int)std::floor(((float)points[3 * i + a] - o[a]) * (1.0f / RLB_S));
            inside = inside && ix[a] >= 0 && ix[a] < dims[a];
        }
        out[i] = inside ? g[((size_t)ix[2] * dims[1] + ix[1]) * dims[0] + ix[0]] : RLB_M;
    }
    return set_ok();
}

}  // extern "C"
