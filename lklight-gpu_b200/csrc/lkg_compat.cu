// Reference-compatible C ABI: cuda_batch_score, cuda_cpydock_solv,
// cuda_full_score, cuda_far_field (src/cuda/full_score.cu, far_field.cu).
//
// Same names, signatures, argument meaning and 0 / -1 return convention,
// with a one-line "<symbol> error ..." message on stderr on failure (the Rust
// bridges map -1 to None).  Host buffers are borrowed for the call.  Device
// copies of the constant arrays are cached keyed on the host pointers and
// sizes, as the reference's cache is (full_score.cu:350-387), but several
// complexes stay resident at once instead of one.  The caller's 10 A cell
// list (cell_start / cell_atoms) is validated for size only: the kernels use
// their own fine cell grid, built once per receptor, which enumerates the
// same pair set (every pair with d^2 <= 100 in f32).  Calls are serialised by
// a mutex (the reference entry points are not re-entrant at all).
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>

#include "lkg_runtime.h"

using namespace lkg;

namespace {

struct Compat {
    std::mutex mu;
    lkg_ctx* ctx = nullptr;
    // key -> complex id
    std::map<std::tuple<const void*, const void*, const void*, const void*, int, int, unsigned, int>, int> batch;
    std::map<std::tuple<const void*, const void*, const void*, const void*, const void*, int, int>, int> solv;
    std::map<std::tuple<const void*, const void*, const void*, int>, int> full;
    std::map<std::tuple<const void*, int, int, int>, std::shared_ptr<DBuf>> fields;
    DBuf d_out, d_coords, d_q;
    HBuf h_out;
};

Compat& compat() {
    static Compat* c = new Compat();  // never destroyed: outlives static destructors
    return *c;
}

int ensure_ctx(Compat& C) {
    if (C.ctx) return 0;
    cudaGetLastError();  // drain a stale sticky error (full_score.cu:375)
    int st = lkg_ctx_create(0, &C.ctx);
    if (st) return st;
    // the reference's GSO calls these entry points once per swarm and step
    // (swarm.rs:70-100: a few hundred poses): work units of 64 ligand atoms
    // spread such a call over twice the warps of 128-atom units (a 300-pose
    // call takes ~320 instead of ~400 us on the batched workload's complexes)
    return lkg_ctx_set_tiles(C.ctx, 64, 0);
}

void clear_locked(Compat& C) {
    if (C.ctx) lkg_ctx_destroy(C.ctx);
    C.ctx = nullptr;
    C.batch.clear();
    C.solv.clear();
    C.full.clear();
    C.fields.clear();
}

MolIn mol_f32(int n, const float* c, const float* q, const float* svdw, const float* rad,
              const unsigned char* heavy, const unsigned char* excl, const float* des, const float* asa) {
    MolIn m;
    m.n = n;
    m.c.resize(3 * (size_t)n);
    for (size_t i = 0; i < 3 * (size_t)n; ++i) m.c[i] = c[i];
    m.q.assign(n, 0.0); m.svdw.assign(n, 0.0); m.eps.assign(n, 0.0); m.rad.assign(n, 0.0);
    m.des.assign(n, 0.0); m.asa.assign(n, 0.0);
    m.heavy.assign(n, 0); m.excl.assign(n, 0);
    for (int i = 0; i < n; ++i) {
        if (q) m.q[i] = q[i];
        if (svdw) { m.svdw[i] = svdw[i]; m.eps[i] = (double)svdw[i] * (double)svdw[i]; }
        if (rad) m.rad[i] = rad[i];
        if (heavy) m.heavy[i] = heavy[i];
        if (excl) m.excl[i] = excl[i];
        if (des) m.des[i] = des[i];
        if (asa) m.asa[i] = asa[i];
    }
    return m;
}

int report(const char* sym, int st, int N, int nl) {
    fprintf(stderr, "%s error status=%d(%s) N=%d nl=%d: %s\n", sym, st, lkg_status_string(st), N, nl,
            lkg_last_error());
    return -1;
}

// stage N x 7 poses, run one launch, read back `out_count` doubles
int run_compat(Compat& C, int id, int N, const double* poses, double* out, size_t out_count, int raw, int solv) {
    lkg_ctx* ctx = C.ctx;
    const size_t pb = (size_t)N * 7 * sizeof(double), ob = out_count * sizeof(double);
    LKG_CK(ctx->h_poses.reserve(pb), "staging");
    LKG_CK(ctx->d_poses.reserve(pb), "staging");
    LKG_CK(C.h_out.reserve(ob), "staging");
    LKG_CK(C.d_out.reserve(ob), "staging");
    memcpy(ctx->h_poses.p, poses, pb);
    LKG_CK(cudaMemcpyAsync(ctx->d_poses.p, ctx->h_poses.p, pb, cudaMemcpyHostToDevice, ctx->stream), "copy-poses");
    int st = launch_items(ctx, 1, &id, &N, ctx->d_poses.as<double>(), C.d_out.as<double>(), nullptr, raw, solv,
                          nullptr, nullptr);
    if (st) return st;
    LKG_CK(cudaMemcpyAsync(C.h_out.p, C.d_out.p, ob, cudaMemcpyDeviceToHost, ctx->stream), "readback");
    if ((st = wait_stream(ctx, 300.0))) return st;
    if ((st = check_status(ctx))) return st;
    memcpy(out, C.h_out.p, ob);
    return 0;
}

}  // namespace

extern "C" {

void lkg_compat_cache_clear(void) {
    Compat& C = compat();
    std::lock_guard<std::mutex> g(C.mu);
    clear_locked(C);
}

int cuda_batch_score(const float* phi, int nx, int ny, int nz, float ox, float oy, float oz, float sp,
                     const float* r_coords, const float* r_ele, const float* r_svdw,
                     const float* r_vdwr, const unsigned char* r_heavy, int nr,
                     const int* cell_start, const int* cell_atoms, int ncx, int ncy, int ncz,
                     float c_ox, float c_oy, float c_oz, float c_sp,
                     const float* l_base, const double* poses, const float* l_ele,
                     const float* l_svdw, const float* l_vdwr, const unsigned char* l_heavy,
                     int nl, int N, unsigned flags, double* out) {
    (void)cell_atoms; (void)c_ox; (void)c_oy; (void)c_oz; (void)c_sp;
    Compat& C = compat();
    std::lock_guard<std::mutex> g(C.mu);
    if (N < 0 || nl <= 0 || nr < 0 || !poses || !out || !l_base || (nr > 0 && !r_coords) ||
        ((flags & F_FAR) && (!phi || nx < 2 || ny < 2 || nz < 2)) || (nr > 0 && !cell_start) ||
        ncx < 1 || ncy < 1 || ncz < 1) {
        set_error(LKG_ERR_ARG, "invalid arguments");
        return report("cuda_batch_score", LKG_ERR_ARG, N, nl);
    }
    if (N == 0) return 0;
    int st = ensure_ctx(C);
    if (st) return report("cuda_batch_score", st, N, nl);
    const unsigned f = flags & (F_FAR | F_ELEC | F_CLASH);
    auto key = std::make_tuple((const void*)(f & F_FAR ? phi : nullptr), (const void*)r_coords,
                               (const void*)cell_start, (const void*)l_base, nl, nr, f, nx);
    auto it = C.batch.find(key);
    int id;
    if (it == C.batch.end()) {
        if (C.batch.size() >= 16) C.batch.clear();  // bound the resident set
        MolIn R = mol_f32(nr, r_coords, r_ele, r_svdw, r_vdwr, r_heavy, nullptr, nullptr, nullptr);
        MolIn L = mol_f32(nl, l_base, l_ele, l_svdw, l_vdwr, l_heavy, nullptr, nullptr, nullptr);
        lkg_field fld{phi, nx, ny, nz, ox, oy, oz, sp};
        st = complex_create(C.ctx, LKG_DNA, f, LJ_SVDW, R, L, (f & F_FAR) ? &fld : nullptr, false, 0.0, &id);
        if (st) return report("cuda_batch_score", st, N, nl);
        C.batch[key] = id;
    } else {
        id = it->second;
    }
    st = run_compat(C, id, N, poses, out, (size_t)2 * N, 1, 0);
    if (st) return report("cuda_batch_score", st, N, nl);
    return 0;
}

int cuda_cpydock_solv(const float* r_coords, const unsigned char* r_flag, int nr,
                      const int* cell_start, const int* cell_atoms, int ncx, int ncy, int ncz,
                      float c_ox, float c_oy, float c_oz, float c_sp,
                      const float* l_base, const double* poses, const unsigned char* l_flag,
                      const float* l_ele, int nl, int N,
                      const float* r_des, const float* r_asa, const float* l_des, const float* l_asa,
                      double* outS) {
    (void)cell_atoms; (void)c_ox; (void)c_oy; (void)c_oz; (void)c_sp; (void)l_ele; (void)ncx; (void)ncy; (void)ncz;
    Compat& C = compat();
    std::lock_guard<std::mutex> g(C.mu);
    if (N < 0 || nl <= 0 || nr <= 0 || !poses || !outS || !l_base || !r_coords || !r_flag || !l_flag ||
        !r_des || !r_asa || !l_des || !l_asa || !cell_start) {
        set_error(LKG_ERR_ARG, "invalid arguments");
        return report("cuda_cpydock_solv", LKG_ERR_ARG, N, nl);
    }
    if (N == 0) return 0;
    int st = ensure_ctx(C);
    if (st) return report("cuda_cpydock_solv", st, N, nl);
    auto key = std::make_tuple((const void*)r_coords, (const void*)r_flag, (const void*)r_des,
                               (const void*)l_base, (const void*)l_flag, nl, nr);
    auto it = C.solv.find(key);
    int id;
    if (it == C.solv.end()) {
        if (C.solv.size() >= 16) C.solv.clear();
        MolIn R = mol_f32(nr, r_coords, nullptr, nullptr, nullptr, nullptr, r_flag, r_des, r_asa);
        MolIn L = mol_f32(nl, l_base, nullptr, nullptr, nullptr, nullptr, l_flag, l_des, l_asa);
        st = complex_create(C.ctx, LKG_CPYDOCK, F_DESOLV, LJ_SVDW, R, L, nullptr, false, 0.0, &id);
        if (st) return report("cuda_cpydock_solv", st, N, nl);
        C.solv[key] = id;
    } else {
        id = it->second;
    }
    st = run_compat(C, id, N, poses, outS, (size_t)N, 0, 1);
    if (st) return report("cuda_cpydock_solv", st, N, nl);
    return 0;
}

int cuda_full_score(const float* phi, int nx, int ny, int nz, float ox, float oy, float oz, float sp,
                    const float* r_coords, const float* r_ele, const float* r_svdw,
                    const float* r_vdwr, const unsigned char* r_heavy, int nr,
                    const int* cell_start, const int* cell_atoms, int ncx, int ncy, int ncz,
                    float c_ox, float c_oy, float c_oz, float c_sp,
                    const float* l_coords, const float* l_ele, const float* l_svdw,
                    const float* l_vdwr, const unsigned char* l_heavy, int nl,
                    float* out_elec, float* out_vdw) {
    (void)cell_atoms; (void)c_ox; (void)c_oy; (void)c_oz; (void)c_sp; (void)ncx; (void)ncy; (void)ncz;
    Compat& C = compat();
    std::lock_guard<std::mutex> g(C.mu);
    if (nl <= 0 || nr < 0 || !l_coords || !out_elec || !out_vdw || !phi || nx < 2 || ny < 2 || nz < 2 ||
        (nr > 0 && (!r_coords || !cell_start))) {
        set_error(LKG_ERR_ARG, "invalid arguments");
        return report("cuda_full_score", LKG_ERR_ARG, 1, nl);
    }
    int st = ensure_ctx(C);
    if (st) return report("cuda_full_score", st, 1, nl);
    auto key = std::make_tuple((const void*)phi, (const void*)r_coords, (const void*)cell_start, nr);
    MolIn L = mol_f32(nl, l_coords, l_ele, l_svdw, l_vdwr, l_heavy, nullptr, nullptr, nullptr);
    auto it = C.full.find(key);
    int id;
    if (it == C.full.end()) {
        if (C.full.size() >= 16) C.full.clear();
        MolIn R = mol_f32(nr, r_coords, r_ele, r_svdw, r_vdwr, r_heavy, nullptr, nullptr, nullptr);
        lkg_field fld{phi, nx, ny, nz, ox, oy, oz, sp};
        st = complex_create(C.ctx, LKG_DNA, F_FAR | F_ELEC | F_CLASH, LJ_SVDW, R, L, &fld, false, 0.0, &id);
        if (st) return report("cuda_full_score", st, 1, nl);
        C.full[key] = id;
    } else {
        id = it->second;
        if ((st = complex_set_ligand(C.ctx, id, L))) return report("cuda_full_score", st, 1, nl);
    }
    lkg_ctx* ctx = C.ctx;
    const double ident[7] = {1, 0, 0, 0, 0, 0, 0};  // coordinates are already transformed
    auto fail = [&](cudaError_t e, const char* what) {
        set_error(cuda_to_status(e), "%s: %s", what, cudaGetErrorString(e));
        return report("cuda_full_score", cuda_to_status(e), 1, nl);
    };
    cudaError_t e;
    if ((e = ctx->d_poses.reserve(7 * sizeof(double))) != cudaSuccess) return fail(e, "alloc");
    if ((e = C.d_out.reserve(2 * sizeof(double) + 2 * (size_t)nl * sizeof(float))) != cudaSuccess) return fail(e, "alloc");
    if ((e = cudaMemcpyAsync(ctx->d_poses.p, ident, sizeof(ident), cudaMemcpyHostToDevice, ctx->stream)) != cudaSuccess)
        return fail(e, "copy");
    float* d_ae = (float*)(C.d_out.as<char>() + 2 * sizeof(double));
    float* d_av = d_ae + nl;
    const int one = 1;
    st = launch_items(ctx, 1, &id, &one, ctx->d_poses.as<double>(), C.d_out.as<double>(), nullptr, 1, 0, d_ae, d_av);
    if (st) return report("cuda_full_score", st, 1, nl);
    if ((e = cudaMemcpyAsync(out_elec, d_ae, nl * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream)) != cudaSuccess)
        return fail(e, "readback");
    if ((e = cudaMemcpyAsync(out_vdw, d_av, nl * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream)) != cudaSuccess)
        return fail(e, "readback");
    if ((st = wait_stream(ctx, 300.0))) return report("cuda_full_score", st, 1, nl);
    return 0;
}

int cuda_far_field(const float* phi, int nx, int ny, int nz, float ox, float oy, float oz, float sp,
                   const float* coords, const float* charges, int n, double* result) {
    Compat& C = compat();
    std::lock_guard<std::mutex> g(C.mu);
    if (!phi || !coords || !charges || !result || n < 0 || nx < 1 || ny < 1 || nz < 1) {
        set_error(LKG_ERR_ARG, "invalid arguments");
        return report("cuda_far_field", LKG_ERR_ARG, 1, n);
    }
    if (n == 0) { *result = 0.0; return 0; }
    int st = ensure_ctx(C);
    if (st) return report("cuda_far_field", st, 1, n);
    lkg_ctx* ctx = C.ctx;
    auto key = std::make_tuple((const void*)phi, nx, ny, nz);
    auto it = C.fields.find(key);
    std::shared_ptr<DBuf> fb;
    cudaError_t e = cudaSuccess;
    size_t np = (size_t)nx * ny * nz;
    if (it == C.fields.end()) {
        if (C.fields.size() >= 8) C.fields.clear();
        fb = std::make_shared<DBuf>();
        if ((e = fb->reserve(np * sizeof(float))) == cudaSuccess)
            e = cudaMemcpy(fb->p, phi, np * sizeof(float), cudaMemcpyHostToDevice);
        if (e != cudaSuccess) {
            set_error(cuda_to_status(e), "field upload: %s", cudaGetErrorString(e));
            return report("cuda_far_field", cuda_to_status(e), 1, n);
        }
        C.fields[key] = fb;
    } else {
        fb = it->second;
    }
    if ((e = C.d_coords.reserve((size_t)n * 3 * sizeof(float))) == cudaSuccess &&
        (e = C.d_q.reserve((size_t)n * sizeof(float))) == cudaSuccess &&
        (e = C.d_out.reserve(sizeof(double))) == cudaSuccess &&
        (e = cudaMemcpyAsync(C.d_coords.p, coords, (size_t)n * 3 * sizeof(float), cudaMemcpyHostToDevice, ctx->stream)) == cudaSuccess &&
        (e = cudaMemcpyAsync(C.d_q.p, charges, (size_t)n * sizeof(float), cudaMemcpyHostToDevice, ctx->stream)) == cudaSuccess &&
        (e = cudaMemsetAsync(C.d_out.p, 0, sizeof(double), ctx->stream)) == cudaSuccess &&
        (e = launch_far_field_sum(fb->as<float>(), nx, ny, nz, ox, oy, oz, sp, C.d_coords.as<float>(),
                                  C.d_q.as<float>(), n, C.d_out.as<double>(), ctx->stream)) == cudaSuccess &&
        (e = cudaMemcpyAsync(result, C.d_out.p, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream)) == cudaSuccess) {
        ctx->launches++;
        if ((st = wait_stream(ctx, 300.0))) return report("cuda_far_field", st, 1, n);
        return 0;
    }
    set_error(cuda_to_status(e), "%s", cudaGetErrorString(e));
    return report("cuda_far_field", cuda_to_status(e), 1, n);
}

}  // extern "C"
