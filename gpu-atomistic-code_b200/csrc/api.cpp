// C ABI implementation (include/asd.h): handle life cycle, uploads into the
// device layouts, step scheduling (direct launches for the FP64 plain form,
// CUDA-graph chunks for the fused forms), read-backs and timing.
#include "internal.h"
#include <algorithm>
#include <array>
#include <map>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

using namespace asd;

namespace {

const double REF_GYRO = 1.76e11, REF_MUB = 9.27e-24, REF_KB = 1.38e-23;  // src/llg.cpp:25

struct Fail {
    int code;
    std::string msg;
};

#define CK(call)                                                                                   \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess)                                                                     \
            throw Fail{e_ == cudaErrorMemoryAllocation ? ASD_ENOMEM : ASD_ECUDA,                   \
                       std::string(#call) + ": " + cudaGetErrorString(e_)};                        \
    } while (0)
#define CKFFT(call)                                                                                \
    do {                                                                                           \
        cufftResult r_ = (call);                                                                   \
        if (r_ != CUFFT_SUCCESS) throw Fail{ASD_ECUFFT, std::string(#call) + " failed (" + std::to_string((int)r_) + ")"}; \
    } while (0)
#define REQUIRE(cond, msg) \
    do { if (!(cond)) throw Fail{ASD_EINVAL, msg}; } while (0)

template <typename T>
T* dalloc(size_t n) {
    T* p = nullptr;
    CK(cudaMalloc(&p, sizeof(T) * (n ? n : 1)));
    CK(cudaMemset(p, 0, sizeof(T) * (n ? n : 1)));
    return p;
}

template <typename T>
T* dupload(const T* src, size_t n) {
    T* p = dalloc<T>(n);
    if (n) CK(cudaMemcpy(p, src, sizeof(T) * n, cudaMemcpyHostToDevice));
    return p;
}

int fail(asd_handle* h, const Fail& f) {
    if (h) h->err = f.msg;
    return f.code;
}

void free_all(asd_handle* h) {
    auto F = [](void* p) { if (p) cudaFree(p); };
    F(h->d_rep_off); F(h->d_rep_stream); F(h->d_atom); F(h->d_rep_sqrtT); F(h->d_dyn); F(h->d_step);
    F(h->d_rep_sqrtT_f); F(h->d_dynf);
    for (int c = 0; c < 3; c++) {
        F(h->sf[c]); F(h->sl[c]); F(h->esf[c]); F(h->fnf[c]); F(h->detf[c]); F(h->stagf[c]);
        F(h->sd[c]); F(h->esd[c]); F(h->fnd[c]); F(h->detd[c]); F(h->stagd[c]);
        F(h->nzf[c]); F(h->nzd[c]);
        for (int q = 0; q < 6; q++) { F(h->kf[q][c]); F(h->kd[q][c]); }
    }
    if (h->h_err) cudaFreeHost(h->h_err);
    F(h->d_err); F(h->d_aos); F(h->d_check); F(h->d_rep_of_tile); F(h->d_ttm); F(h->d_q4ptr); F(h->d_q4jkl);
    F(h->sell.lwords); F(h->sell.span_ptr); F(h->sell.spans);
    F(h->sell.slice_ptr); F(h->sell.a); F(h->sell.b); F(h->sell.c); F(h->sell.col); F(h->sell.val);
    F(h->sell.typed); F(h->sell.tab_f); F(h->sell.tab_d);
    F(h->dia.tile_ptr); F(h->dia.tile_diag);
    F(h->dia.off); F(h->dia.valf); F(h->dia.vald); F(h->dia.dtype); F(h->dia.tab_f); F(h->dia.tab_d);
    F(h->p_s); F(h->p_es); F(h->p_fn); F(h->p_ch); F(h->p_hdemag); F(h->p_rand); F(h->p_det); F(h->p_hstg); F(h->p_hinit);
    for (int q = 0; q < 6; q++) F(h->p_k[q]);
    F(h->p_sigma); F(h->p_llgpf); F(h->p_lambda); F(h->p_k1u); F(h->p_k1udir);
    F(h->pex.xadj); F(h->pex.adjncy); F(h->pex.off);
    for (int q = 0; q < 9; q++) F(h->pex.v[q]);
    LongRange& L = h->lr;
    F(L.mesh_idx); F(L.w); F(L.r); F(L.k); F(L.nkr); F(L.nkc); F(L.zr); F(L.zk); F(L.zh); F(L.znk);
    if (L.r2c) cufftDestroy(L.r2c);
    if (L.c2r) cufftDestroy(L.c2r);
    if (L.z2z) cufftDestroy(L.z2z);
    if (L.c2c) cufftDestroy(L.c2c);
    F(L.k1); F(L.k2); F(L.yk); F(L.nkt); F(L.twt); F(L.xq);
    F(h->sq.idx); F(h->sq.sub); F(h->sq.uo); F(h->sq.kidx); F(h->sq.grid); F(h->sq.series);
    if (h->sq.plan) cufftDestroy(h->sq.plan);
    F(h->d_magpart); F(h->d_mag); F(h->d_magcnt); F(h->d_inv_count); F(h->d_sub_of_atom); F(h->d_stats);
    if (h->graph) cudaGraphExecDestroy(h->graph);
    if (h->graph1) cudaGraphExecDestroy(h->graph1);
    if (h->graph1_src) cudaGraphDestroy(h->graph1_src);
    if (h->kev[0]) cudaEventDestroy(h->kev[0]);
    if (h->kev[1]) cudaEventDestroy(h->kev[1]);
    if (h->stream) cudaStreamDestroy(h->stream);
}

// Distinct tensors of an exchange matrix (id 0 = the zero tensor), at most 256.
struct TensorTable {
    int nc;
    std::map<std::array<double, 9>, uint32_t> ids;
    std::vector<std::array<double, 9>> list;
    std::array<double, 9> last{};
    int64_t last_id = 0;
    explicit TensorTable(int ncomp) : nc(ncomp) {
        std::array<double, 9> z{};
        ids[z] = 0;
        list.push_back(z);
    }
    int64_t id(const std::array<double, 9>& key) {
        if (key == last) return last_id;
        auto it = ids.find(key);
        int64_t t;
        if (it != ids.end()) t = it->second;
        else {
            if (list.size() >= 256) return -1;
            t = (int64_t)list.size();
            ids[key] = (uint32_t)t;
            list.push_back(key);
        }
        last = key;
        last_id = t;
        return t;
    }
    uint32_t size() const { return (uint32_t)list.size(); }
    uint32_t bits() const {
        uint32_t b = 1;
        while ((1u << b) < list.size()) b++;
        return b;
    }
    template <typename T>
    std::vector<T> table() const {   // type-major [ntypes][stride], stride 4 (xx,yy,zz,0) or 12 (9 + 3 zeros)
        const size_t stride = nc == 9 ? 12 : 4;
        std::vector<T> t(stride * list.size(), (T)0);
        for (size_t k = 0; k < list.size(); k++)
            for (int q = 0; q < nc; q++) t[k * stride + q] = (T)list[k][q];
        return t;
    }
};

// CSR (all replicas concatenated) -> SELL-32 device layout.
void build_sell(asd_handle* h, const std::vector<uint32_t>& xadj, const std::vector<uint32_t>& adj,
                const std::vector<double>& val9) {
    const uint32_t n = h->n;
    const bool full = h->full != 0;
    const bool zz_yy = (h->p.flags & ASD_FLAG_GPU_DZZ_FROM_DYY) != 0;
    const uint32_t ns = (n + 31) / 32;
    std::vector<uint32_t> sp(ns + 1, 0);
    for (uint32_t s = 0; s < ns; s++) {
        uint32_t w = 0;
        for (uint32_t r = 32 * s; r < std::min(n, 32 * s + 32); r++) w = std::max(w, xadj[r + 1] - xadj[r]);
        sp[s + 1] = sp[s] + 32 * w;
    }
    const uint32_t E = sp[ns];
    h->sell.nslices = ns;
    h->sell.entries = E;
    h->sell.slice_ptr = dupload(sp.data(), sp.size());
    h->h_slice_ptr = sp;
    auto value = [&](uint32_t k, int q) {
        if (q == 8 && zz_yy) q = 4;
        return val9[9 * (size_t)k + q];
    };
    // typed layout: (column, tensor id) in one word when the matrix has few distinct tensors
    if (!(h->p.flags & ASD_FLAG_STREAMED_EXCHANGE)) {
        const int nc = full ? 9 : 3;
        const int qmap[9] = {0, 4, 8, 0, 0, 0, 0, 0, 0};
        TensorTable tt(nc);
        std::vector<uint32_t> id(adj.size());
        bool ok = true;
        for (size_t k = 0; k < adj.size() && ok; k++) {
            std::array<double, 9> key{};
            for (int q = 0; q < nc; q++) key[q] = value((uint32_t)k, full ? q : qmap[q]);
            const int64_t t = tt.id(key);
            if (t < 0) ok = false; else id[k] = (uint32_t)t;
        }
        const uint32_t tb = tt.bits();
        if (ok && (uint64_t)n <= (1ull << (32 - tb))) {
            std::vector<uint32_t> w(E);
            for (uint32_t s = 0; s < ns; s++) {
                const uint32_t wd = (sp[s + 1] - sp[s]) / 32;
                for (uint32_t k = 0; k < wd; k++)
                    for (uint32_t lane = 0; lane < 32; lane++) {
                        const uint32_t r = 32 * s + lane, e = sp[s] + 32 * k + lane;
                        uint32_t col = r < n ? r : 0, t = 0;
                        if (r < n && k < xadj[r + 1] - xadj[r]) { col = adj[xadj[r] + k]; t = id[xadj[r] + k]; }
                        w[e] = col | (t << (32 - tb));
                    }
            }
            h->sell.typed = dupload(w.data(), w.size());
            h->h_words = std::move(w);
            h->sell.colbits = 32 - tb;
            h->sell.ntypes = tt.size();
            if (h->p.precision == ASD_FP32) {
                std::vector<float> tf = tt.table<float>();
                h->sell.tab_f = dupload(tf.data(), tf.size());
            } else {
                std::vector<double> td = tt.table<double>();
                h->sell.tab_d = dupload(td.data(), td.size());
            }
            return;
        }
    }
    if (h->p.precision == ASD_FP32) {
        std::vector<float4> a(E), b(full ? E : 0);
        std::vector<float2> c(full ? E : 0);
        for (uint32_t s = 0; s < ns; s++) {
            const uint32_t w = (sp[s + 1] - sp[s]) / 32;
            for (uint32_t k = 0; k < w; k++)
                for (uint32_t lane = 0; lane < 32; lane++) {
                    const uint32_t r = 32 * s + lane, e = sp[s] + 32 * k + lane;
                    int col = r < n ? (int)r : 0;
                    float v[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
                    if (r < n && k < xadj[r + 1] - xadj[r]) {
                        const uint32_t kk = xadj[r] + k;
                        col = (int)adj[kk];
                        for (int q = 0; q < 9; q++) v[q] = (float)value(kk, q);
                    }
                    int ci;
                    memcpy(&ci, &col, 4);
                    float cf;
                    memcpy(&cf, &ci, 4);
                    if (!full) a[e] = make_float4(cf, v[0], v[4], v[8]);
                    else {
                        a[e] = make_float4(cf, v[0], v[1], v[2]);
                        b[e] = make_float4(v[3], v[4], v[5], v[6]);
                        c[e] = make_float2(v[7], v[8]);
                    }
                }
        }
        h->sell.a = dupload(a.data(), a.size());
        if (full) { h->sell.b = dupload(b.data(), b.size()); h->sell.c = dupload(c.data(), c.size()); }
    } else {
        const int nc = full ? 9 : 3;
        const int qmap3[3] = {0, 4, 8};
        std::vector<int32_t> col(E);
        std::vector<double> v((size_t)nc * E, 0.0);
        for (uint32_t s = 0; s < ns; s++) {
            const uint32_t w = (sp[s + 1] - sp[s]) / 32;
            for (uint32_t k = 0; k < w; k++)
                for (uint32_t lane = 0; lane < 32; lane++) {
                    const uint32_t r = 32 * s + lane, e = sp[s] + 32 * k + lane;
                    col[e] = r < n ? (int)r : 0;
                    if (r < n && k < xadj[r + 1] - xadj[r]) {
                        const uint32_t kk = xadj[r] + k;
                        col[e] = (int)adj[kk];
                        for (int q = 0; q < nc; q++) v[(size_t)q * E + e] = value(kk, full ? q : qmap3[q]);
                    }
                }
        }
        h->sell.col = dupload(col.data(), col.size());
        h->sell.val = dupload(v.data(), v.size());
    }
}

// A CSR matrix whose entries lie on few diagonals (col - row takes at most 32 values, as on a
// regular lattice) is also held in the typed DIA layout, whose gather forms each column from the
// row and the diagonal (one id byte per entry instead of a 4-byte word, every load of a warp
// contiguous); the autotuner picks the faster layout.  Entries of one row on one diagonal are
// summed.  Builds nothing (returns false) for other matrices, several replicas or the streamed
// layout.
bool build_dia_alt(asd_handle* h, const std::vector<uint32_t>& xadj, const std::vector<uint32_t>& adj,
                   const std::vector<double>& val9) {
    if (h->nrep != 1 || (h->p.flags & ASD_FLAG_STREAMED_EXCHANGE) || h->p.precision == ASD_FP64_PLAIN) return false;
    const uint32_t n = h->n;
    constexpr uint32_t MAXD = 32;
    std::map<int64_t, uint32_t> offs;
    for (uint32_t i = 0; i < n; i++)
        for (uint32_t k = xadj[i]; k < xadj[i + 1]; k++) {
            offs.emplace((int64_t)adj[k] - (int64_t)i, 0u);
            if (offs.size() > MAXD) return false;
        }
    if (offs.empty()) return false;
    std::vector<int32_t> off;
    for (auto& kv : offs) { kv.second = (uint32_t)off.size(); off.push_back((int32_t)kv.first); }
    const uint32_t nd = (uint32_t)off.size();
    const bool full = h->full != 0, zz_yy = (h->p.flags & ASD_FLAG_GPU_DZZ_FROM_DYY) != 0;
    const int nc = full ? 9 : 3;
    const int qmap[3] = {0, 4, zz_yy ? 4 : 8};
    TensorTable tt(nc);
    std::vector<uint8_t> ids((size_t)nd * n, 0);
    std::array<std::array<double, 9>, MAXD> loc;
    std::array<bool, MAXD> used;
    for (uint32_t i = 0; i < n; i++) {
        used.fill(false);
        for (uint32_t k = xadj[i]; k < xadj[i + 1]; k++) {
            const uint32_t d = offs[(int64_t)adj[k] - (int64_t)i];
            if (!used[d]) { loc[d].fill(0.0); used[d] = true; }
            for (int q = 0; q < nc; q++) {
                int src = full ? q : qmap[q];
                if (full && q == 8 && zz_yy) src = 4;
                loc[d][q] += val9[9 * (size_t)k + src];
            }
        }
        for (uint32_t d = 0; d < nd; d++) {
            if (!used[d]) continue;
            const int64_t t = tt.id(loc[d]);
            if (t < 0 || t > 255) return false;
            ids[(size_t)d * n + i] = (uint8_t)t;
        }
    }
    const uint32_t nt = (n + 31) / 32;
    std::vector<uint32_t> tp(nt + 1, 0), td;
    for (uint32_t w = 0; w < nt; w++) {
        const uint32_t r0 = 32 * w, r1 = std::min(n, r0 + 32);
        for (uint32_t d = 0; d < nd; d++) {
            bool any = false;
            for (uint32_t r = r0; r < r1 && !any; r++) any = ids[(size_t)d * n + r] != 0;
            if (any) td.push_back(d);
        }
        tp[w + 1] = (uint32_t)td.size();
    }
    DiaDev& m = h->dia;
    m.ndiag = nd;
    m.off = dupload(off.data(), off.size());
    m.dtype = dupload(ids.data(), ids.size());
    m.ntypes = tt.size();
    if (h->p.precision == ASD_FP32) { std::vector<float> tf = tt.table<float>(); m.tab_f = dupload(tf.data(), tf.size()); }
    else { std::vector<double> tdd = tt.table<double>(); m.tab_d = dupload(tdd.data(), tdd.size()); }
    m.tile_ptr = dupload(tp.data(), tp.size());
    m.tile_diag = dupload(td.data(), std::max<size_t>(td.size(), 1));
    h->dia_alt = true;
    return true;
}

void setup_lr(asd_handle* h, const asd_system& s, bool plain) {
    LongRange& L = h->lr;
    L.mode = (int)s.lr;
    for (int a = 0; a < 3; a++) L.mesh[a] = s.mesh[a];
    REQUIRE(L.mesh[0] && L.mesh[1] && L.mesh[2], "long-range field needs a mesh");
    REQUIRE(L.mesh[2] % 2 == 0, "last mesh dimension must be even");
    L.P = (size_t)L.mesh[0] * L.mesh[1] * L.mesh[2];
    L.Pk = (size_t)L.mesh[0] * L.mesh[1] * (L.mesh[2] / 2 + 1);
    REQUIRE(s.mesh_xyz && s.nr, "long-range field needs mesh_xyz and nr");
    std::vector<uint32_t> idx(h->n);
    std::vector<float> w(h->n);
    for (uint32_t i = 0; i < h->n; i++) {
        const uint32_t x = s.mesh_xyz[3 * i], y = s.mesh_xyz[3 * i + 1], z = s.mesh_xyz[3 * i + 2];
        REQUIRE(x < L.mesh[0] && y < L.mesh[1] && z < L.mesh[2], "mesh_xyz outside the mesh");
        idx[i] = (uint32_t)(((size_t)x * L.mesh[1] + y) * L.mesh[2] + z);
        const uint32_t at = s.atom ? s.atom[i] : i % s.nmat;
        w[i] = s.lr == ASD_LR_DIPOLE ? (float)s.mat[at].mu : 1.0f;
    }
    L.mesh_idx = dupload(idx.data(), idx.size());
    L.w = dupload(w.data(), w.size());
    // symmetry of N_r (up to rounding of (3 e_a) e_b) decides 6 or 9 stored components;
    // a symmetric matrix is stored as the mean of each (a,b),(b,a) pair
    double amax = 0.0;
    for (size_t q = 0; q < 9 * L.P; q++) amax = std::max(amax, std::fabs(s.nr[q]));
    bool sym = true;
    const int pairs[3][2] = {{1, 3}, {2, 6}, {5, 7}};
    for (size_t c = 0; c < L.P && sym; c++)
        for (auto& pr : pairs)
            if (std::fabs(s.nr[pr[0] * L.P + c] - s.nr[pr[1] * L.P + c]) > 1e-13 * amax) sym = false;
    L.ncomp = sym ? 6 : 9;
    std::vector<double> nrs(s.nr, s.nr + 9 * L.P);
    if (sym)
        for (size_t c = 0; c < L.P; c++)
            for (auto& pr : pairs) {
                const double m = 0.5 * (nrs[pr[0] * L.P + c] + nrs[pr[1] * L.P + c]);
                nrs[pr[0] * L.P + c] = m;
                nrs[pr[1] * L.P + c] = m;
            }
    uint32_t lo[3] = {~0u, ~0u, ~0u}, hi[3] = {0, 0, 0};    // bounding box of the spins on the mesh
    for (uint32_t i = 0; i < h->n; i++)
        for (int a = 0; a < 3; a++) {
            lo[a] = std::min(lo[a], s.mesh_xyz[3 * i + a]);
            hi[a] = std::max(hi[a], s.mesh_xyz[3 * i + a]);
        }
    if (!plain) {
        // On an even mesh axis the plane at index m/2 holds the aliased displacement +-m/2; when
        // the spins span fewer than m/2 mesh points along that axis no two spins are that far
        // apart, so the plane never reaches a spin and is cleared.  N_r is then exactly even
        // (N(-r) = N(r)), its transform real, and the convolution takes the 6-component real form.
        for (int a = 0; a < 3; a++) {
            const uint32_t m = L.mesh[a];
            if (m % 2 || h->n == 0 || hi[a] - lo[a] >= m / 2) continue;
            for (uint32_t x = 0; x < L.mesh[0]; x++)
                for (uint32_t y = 0; y < L.mesh[1]; y++)
                    for (uint32_t z = 0; z < L.mesh[2]; z++) {
                        const uint32_t v[3] = {x, y, z};
                        if (v[a] != m / 2) continue;
                        const size_t c = ((size_t)x * L.mesh[1] + y) * L.mesh[2] + z;
                        for (int q = 0; q < 9; q++) nrs[q * L.P + c] = 0.0;
                    }
        }
    }
    double* d_nr = dupload(plain ? s.nr : nrs.data(), 9 * L.P);
    int dims[3] = {(int)L.mesh[0], (int)L.mesh[1], (int)L.mesh[2]};
    cudaError_t e;
    if (plain) {
        L.zr = dalloc<double2>(3 * L.P);
        L.zk = dalloc<double2>(3 * L.P);
        L.zh = dalloc<double2>(3 * L.P);
        L.znk = dalloc<double2>(9 * L.P);
        CKFFT(cufftPlanMany(&L.z2z, 3, dims, nullptr, 1, (int)L.P, nullptr, 1, (int)L.P, CUFFT_Z2Z, 3));
        CKFFT(cufftSetStream(L.z2z, h->stream));
        e = build_nk_plain(h, d_nr);
    } else {
        L.r = dalloc<float>(6 * L.P);   // [0,3P): M_r, [3P,6P): H_r
        const uint32_t mz = L.mesh[2];
        // pruned transform when the last axis is a power of two: z transforms only for the rows
        // of the spins' box, 2D transforms of the (x, y) planes by cuFFT
        L.pruned = (mz >= 4 && mz <= 2048 && (mz & (mz - 1)) == 0 && h->n > 0) ? 1 : 0;   // z-pass smem <= 45 KB
        if (L.pruned) for (int a = 0; a < 3; a++) { L.box0[a] = lo[a]; L.box1[a] = hi[a]; }
        // the library's plane kernels replace cuFFT's (x, y) passes where every axis fits them
        L.planes = (L.pruned && !(h->p.flags & ASD_FLAG_CUFFT_PLANES) && plane_path_fits(L, false) &&
                    plane_path_fits(L, true)) ? 1 : 0;
        if (L.planes) {
            // buffers are allocated with the tiled N_k (build_nk_f32)
        } else if (L.pruned) {
            for (int a = 0; a < 3; a++) { L.box0[a] = lo[a]; L.box1[a] = hi[a]; }
            L.k1 = dalloc<float2>(3 * L.Pk);
            L.k2 = dalloc<float2>(3 * L.Pk);
            int d2[2] = {(int)L.mesh[0], (int)L.mesh[1]};
            const int plane = (int)(L.mesh[0] * L.mesh[1]);
            CKFFT(cufftPlanMany(&L.c2c, 2, d2, nullptr, 1, plane, nullptr, 1, plane, CUFFT_C2C, 3 * (int)(mz / 2 + 1)));
            CKFFT(cufftSetStream(L.c2c, h->stream));
        } else {
            L.k = dalloc<float2>(3 * L.Pk);
            CKFFT(cufftPlanMany(&L.r2c, 3, dims, nullptr, 1, (int)L.P, nullptr, 1, (int)L.Pk, CUFFT_R2C, 3));
            CKFFT(cufftPlanMany(&L.c2r, 3, dims, nullptr, 1, (int)L.Pk, nullptr, 1, (int)L.P, CUFFT_C2R, 3));
            CKFFT(cufftSetStream(L.r2c, h->stream));
            CKFFT(cufftSetStream(L.c2r, h->stream));
        }
        e = build_nk_f32(h, d_nr);
        if (e == cudaSuccess && L.pruned && !L.planes) e = permute_nk_pruned(h);
        if (e == cudaSuccess && L.planes) e = build_plane_twiddles(h);
    }
    cudaFree(d_nr);
    CK(e);
}

void set_dyn(asd_handle* h, int idx, double v) {
    CK(launch_set_scalar(h, h->d_dyn + idx, v));
    if (idx != DYN_DET_STEP) CK(launch_set_scalar_f(h, h->d_dynf + idx, (float)v));
}

// The long-range input from the current spins (after new spins).
void scatter_if_needed(asd_handle* h) {
    if (h->lr.mode == ASD_LR_NONE || h->p.precision == ASD_FP64_PLAIN || h->lr_scattered) return;
    CK(launch_lr_scatter(h));
    h->lr_scattered = true;
}

// Largest count of typed words that a block of B threads stages: its B/32 consecutive slices.
uint32_t stage_capacity(const asd_handle* h, int B) {
    const std::vector<uint32_t>& sp = h->h_slice_ptr;
    if (sp.size() < 2) return 0;
    const uint32_t ns = (uint32_t)sp.size() - 1, spb = (uint32_t)B / 32;
    uint32_t m = 0;
    for (uint32_t s0 = 0; s0 < ns; s0 += spb) m = std::max(m, sp[std::min(s0 + spb, ns)] - sp[s0]);
    return m;
}

// Shared memory a block may spend on the tensor table plus the staged words (keeps at least
// two blocks per SM), and on staged neighbour spins on top of that.
constexpr size_t STAGE_SMEM_MAX = 96 * 1024;

void free_spin_stage(asd_handle* h) {
    SellDev& m = h->sell;
    if (m.lwords) cudaFree(m.lwords);
    if (m.lwords16) cudaFree(m.lwords16);
    if (m.span_ptr) cudaFree(m.span_ptr);
    if (m.spans) cudaFree(m.spans);
    m.lwords = nullptr; m.lwords16 = nullptr; m.lbits = 0; m.span_ptr = nullptr; m.spans = nullptr;
    m.spin_slots = 0; m.spin_block = 0;
}

// Neighbour-spin spans and local words for blocks of B rows (asd_plan_spin_spans); returns
// false when no block can stage.
bool build_spin_stage(asd_handle* h, int B) {
    free_spin_stage(h);
    const std::vector<uint32_t>& sp = h->h_slice_ptr;
    const std::vector<uint32_t>& w = h->h_words;
    if (sp.size() < 2 || w.empty()) return false;
    const uint32_t rb = h->p.precision == ASD_FP32 ? 4 : 8;
    const uint32_t ns = (uint32_t)sp.size() - 1, spb = (uint32_t)B / 32;
    const uint32_t nblk = (ns + spb - 1) / spb;
    std::vector<uint32_t> ptr(nblk + 1);
    uint32_t nspans = 0, slots = 0;
    if (asd_plan_spin_spans(h->n, ns, sp.data(), w.data(), h->sell.colbits, rb, (uint32_t)B, ptr.data(), nullptr, 0,
                            nullptr, &nspans, &slots) != ASD_OK || nspans == 0)
        return false;
    std::vector<uint32_t> spans(4 * (size_t)nspans), lw(w.size());
    if (asd_plan_spin_spans(h->n, ns, sp.data(), w.data(), h->sell.colbits, rb, (uint32_t)B, ptr.data(), spans.data(),
                            nspans, lw.data(), &nspans, &slots) != ASD_OK)
        return false;
    SellDev& m = h->sell;
    m.lwords = dupload(lw.data(), lw.size());
    // 16-bit words: slot in the low lbits bits, tensor id above, for the blocks with spans
    uint32_t lbits = 1;
    while ((1u << lbits) < slots) lbits++;
    if (lbits < 16 && (uint64_t)h->sell.ntypes <= (1ull << (16 - lbits))) {
        const uint32_t cmask = h->sell.colbits >= 32 ? 0xFFFFFFFFu : (1u << h->sell.colbits) - 1u;
        std::vector<uint16_t> w16(lw.size(), 0);
        for (uint32_t b = 0; b < nblk; b++) {
            if (ptr[b + 1] == ptr[b]) continue;                  // no spans: global words, unstaged
            const uint32_t e0 = sp[b * spb], e1 = sp[std::min((b + 1) * spb, ns)];
            for (uint32_t e = e0; e < e1; e++) {
                const uint32_t slot = lw[e] & cmask, t = lw[e] >> h->sell.colbits;
                w16[e] = (uint16_t)(slot | (t << lbits));
            }
        }
        m.lwords16 = dupload(w16.data(), w16.size());
        m.lbits = lbits;
    }
    m.span_ptr = dupload(ptr.data(), ptr.size());
    m.spans = reinterpret_cast<uint4*>(dupload(spans.data(), spans.size()));
    m.spin_slots = slots;
    m.spin_block = (uint32_t)B;
    return true;
}

// Launch shape of the fused stage kernel: block size and the staging mode of typed SELL
// words (0 none, 1 words, 2 words and neighbour spins).
void configure_stage(asd_handle* h, int B, int mode) {
    h->block = B;
    h->sell.stage = 0;
    h->sell.stage_words = 0;
    if (mode == 0 || !h->sell.typed || h->dexch != ASD_EXCH_CSR) return;
    const size_t rb = h->p.precision == ASD_FP32 ? 4 : 8;
    const size_t tab = ((rb * (h->full ? 12 : 4) * h->sell.ntypes) + 15) & ~(size_t)15;
    const uint32_t w = stage_capacity(h, B);
    if (w == 0 || tab + 4 * (size_t)w > STAGE_SMEM_MAX) return;
    h->sell.stage = 1;
    h->sell.stage_words = w;
    if (mode == 2) {
        if (h->sell.spin_block != (uint32_t)B && !build_spin_stage(h, B)) return;
        if (h->sell.spin_block == (uint32_t)B) h->sell.stage = 2;
    }
}

// Project autotuner: time the first stage kind of the step (it writes only scratch buffers)
// for every block size in {64, 128, 256} with and without staging, keep the fastest.
void autotune(asd_handle* h) {
    struct Cand { uint32_t layout; int B; int mode; };
    static const char* names[3] = {"direct", "words", "words+spins"};
    std::vector<Cand> cs;
    // DIA input also exists as SELL-32, and a CSR matrix on few diagonals as DIA: both device
    // layouts are candidates
    std::vector<uint32_t> layouts{h->dexch};
    if ((h->exch == ASD_EXCH_DIA && h->sell.slice_ptr) || (h->exch == ASD_EXCH_CSR && h->dia_alt))
        layouts = {ASD_EXCH_CSR, ASD_EXCH_DIA};
    for (uint32_t lay : layouts)
        for (int B : {64, 128, 256}) {
            cs.push_back({lay, B, 0});
            if (h->sell.typed && lay == ASD_EXCH_CSR) { cs.push_back({lay, B, 1}); cs.push_back({lay, B, 2}); }
        }
    double best = 1e300;
    Cand bc{layouts[0], 256, 1};
    std::string log;
    char buf[96];
    for (const Cand& cd : cs) {
        h->dexch = cd.layout;
        configure_stage(h, cd.B, cd.mode);
        if ((int)h->sell.stage != cd.mode) continue;
        float ms = 0.f;
        CK(time_first_stage(h, 2, 8, &ms));
        std::snprintf(buf, sizeof buf, "%s%sB=%d/%s:%.4f", log.empty() ? "" : " ",
                      layouts.size() > 1 ? (cd.layout == ASD_EXCH_CSR ? "SELL:" : "DIA:") : "", cd.B, names[cd.mode],
                      (double)ms);
        log += buf;
        if (ms < best) { best = ms; bc = cd; }
    }
    h->dexch = bc.layout;
    configure_stage(h, bc.B, bc.mode);
    std::snprintf(buf, sizeof buf, "%sblock=%d staging=%s; ", layouts.size() > 1 ? (bc.layout == ASD_EXCH_CSR ? "layout=SELL " : "layout=DIA ") : "",
                  h->block, names[h->sell.stage]);
    h->tune = std::string(buf) + "ms per stage launch: " + log;
}

void destroy_graph(asd_handle* h) {
    if (h->graph) { cudaGraphExecDestroy(h->graph); h->graph = nullptr; h->graph_steps = 0; }
    if (h->graph1) { cudaGraphExecDestroy(h->graph1); h->graph1 = nullptr; }
    if (h->graph1_src) { cudaGraphDestroy(h->graph1_src); h->graph1_src = nullptr; }
    h->det_node = nullptr;
}

// The applied field on the device, where a single-step graph has not yet written it.
void flush_applied(asd_handle* h) {
    if (!h->applied_pending) return;
    CK(launch_set_vec3(h, h->d_dyn + DYN_APPLIED, h->d_dynf + DYN_APPLIED, h->p.applied));
    h->applied_pending = false;
}

// Capture `steps` fused steps + the counter advance into one graph, and a one-step graph for
// single-step calls: the det-field step taken from the device counter, the step, the advance.
void build_graph(asd_handle* h, uint32_t steps) {
    destroy_graph(h);
    cudaGraph_t g;
    const uint64_t before = h->launches;
    // the captured launch pattern depends only on the step phase modulo the dipole
    // refresh period; chunks are replayed from phase 0 (see run_steps)
    const uint64_t saved = h->step;
    h->step = 0;
    CK(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
    cudaError_t e = cudaSuccess;
    for (uint32_t r = 0; r < steps && e == cudaSuccess; r++) e = launch_fused_step(h, r, true);
    if (e == cudaSuccess) e = launch_step_advance(h, steps);
    cudaError_t e2 = cudaStreamEndCapture(h->stream, &g);
    h->step = saved;
    h->graph_launches = h->launches - before;
    h->launches = before;
    CK(e);
    CK(e2);
    CK(cudaGraphInstantiate(&h->graph, g, 0));
    cudaGraphDestroy(g);
    h->graph_steps = steps;
    // one step: valid whatever the phase when the long-range refresh pattern does not depend on it
    const uint32_t upd = h->p.update ? h->p.update : 1;
    if (h->lr.mode == ASD_LR_DIPOLE && upd != 1) return;
    h->step = 0;
    CK(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
    e = launch_det_here(h);
    if (e == cudaSuccess) e = launch_fused_step(h, 0, true);
    if (e == cudaSuccess) e = launch_step_advance(h, 1);
    e2 = cudaStreamEndCapture(h->stream, &g);
    h->step = saved;
    h->graph1_launches = h->launches - before;
    h->launches = before;
    CK(e);
    CK(e2);
    CK(cudaGraphInstantiate(&h->graph1, g, 0));
    // keep the captured graph and its det_here_k node: asd_set_applied updates the node in place
    h->graph1_src = g;
    size_t nn = 0;
    CK(cudaGraphGetNodes(g, nullptr, &nn));
    std::vector<cudaGraphNode_t> nodes(nn);
    CK(cudaGraphGetNodes(g, nodes.data(), &nn));
    for (cudaGraphNode_t nd : nodes) {
        cudaGraphNodeType ty;
        CK(cudaGraphNodeGetType(nd, &ty));
        if (ty != cudaGraphNodeTypeKernel) continue;
        cudaKernelNodeParams kp{};
        CK(cudaGraphKernelNodeGetParams(nd, &kp));
        if (kp.func == det_here_kernel()) { h->det_node = nd; break; }
    }
}

void run_steps(asd_handle* h, uint64_t nsteps) {
    if (nsteps == 0) return;
    if (h->p.precision == ASD_FP64_PLAIN) {
        for (uint64_t q = 0; q < nsteps; q++) CK(launch_plain_step(h, h->step + q));
        h->step += nsteps;
        return;
    }
    scatter_if_needed(h);
    if (nsteps == 1 && h->graph1 && !h->timing) {
        // one launch: the graph sets the det-field step to the step it runs, and the applied field
        CK(cudaGraphLaunch(h->graph1, h->stream));
        h->launches += h->graph1_launches;
        h->applied_pending = false;
        h->step += 1;
        return;
    }
    flush_applied(h);
    set_dyn(h, DYN_DET_STEP, (double)(h->step + nsteps - 1));
    const uint32_t upd = h->p.update ? h->p.update : 1;
    const uint32_t G = h->graph_steps;
    uint64_t left = nsteps;
    auto direct = [&](uint64_t k) {
        for (uint64_t r = 0; r < k; r++) CK(launch_fused_step(h, (uint32_t)r, false));
        CK(launch_step_advance(h, (uint32_t)k));
        h->step += k;
    };
    // align to the dipole refresh period so that one captured chunk fits every chunk
    if (h->lr.mode == ASD_LR_DIPOLE && h->step % upd) {
        const uint64_t k = std::min<uint64_t>(left, upd - h->step % upd);
        direct(k);
        left -= k;
    }
    while (G && left >= G) {
        CK(cudaGraphLaunch(h->graph, h->stream));
        h->launches += h->graph_launches;
        h->step += G;
        left -= G;
    }
    if (left) direct(left);
}

}  // namespace

extern "C" {

const char* asd_version(void) { return "asd-b200 0.1 (sm_100a)"; }

namespace {
thread_local std::string g_create_err;   // message of the calling thread's last failed asd_create
}

const char* asd_last_error(const asd_handle* h) { return h ? h->err.c_str() : g_create_err.c_str(); }

int asd_create(const asd_params* pp, const asd_system* sys, uint32_t nsys, asd_handle** out) {
    if (!out) return ASD_EINVAL;
    *out = nullptr;
    if (!pp || !sys || nsys == 0) return ASD_EINVAL;
    asd_handle* h = new asd_handle();
    h->p = *pp;
    try {
        asd_params& p = h->p;
        if (p.gyro == 0) p.gyro = REF_GYRO;
        if (p.muB == 0) p.muB = REF_MUB;
        if (p.kB == 0) p.kB = REF_KB;
        if (p.update == 0) p.update = 1;
        REQUIRE(p.integrator <= ASD_RK5, "unknown integrator");
        REQUIRE(p.precision <= ASD_FP64_FUSED, "unknown precision");
        REQUIRE(p.dt > 0 && std::isfinite(p.dt), "dt must be positive");
        CK(cudaGetDevice(&h->device));
        CK(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
        // ---- replicas, materials
        const asd_system& s0 = sys[0];
        h->nrep = nsys;
        h->exch = s0.exch;
        h->full = s0.exch_full ? 1 : 0;
        h->nmat = s0.nmat;
        REQUIRE(h->nmat >= 1 && h->nmat <= ASD_MAX_MAT, "nmat must be 1..16");
        REQUIRE(h->exch <= ASD_EXCH_NONE, "unknown exchange storage");
        h->h_rep_off.assign(1, 0);
        uint64_t ntot = 0;
        for (uint32_t r = 0; r < nsys; r++) {
            const asd_system& s = sys[r];
            REQUIRE(s.nspins > 0, "empty lattice");
            REQUIRE(s.exch == h->exch && (s.exch_full ? 1u : 0u) == h->full, "replicas must share the exchange storage");
            REQUIRE(s.nmat == h->nmat && s.mat, "replicas must share the material table");
            for (uint32_t t = 0; t < s.nmat; t++)
                REQUIRE(memcmp(&s.mat[t], &s0.mat[t], sizeof(asd_material)) == 0, "replicas must share the material table");
            REQUIRE(s.lr == ASD_LR_NONE || nsys == 1, "long-range field supports one replica per handle");
            REQUIRE(s.temperature >= 0 && std::isfinite(s.temperature), "temperature must be >= 0");
            ntot += s.nspins;
            REQUIRE(ntot < (1ull << 31), "too many spins");
            h->h_rep_off.push_back((uint32_t)ntot);
            h->h_rep_T.push_back(s.temperature);
        }
        h->n = (uint32_t)ntot;
        const uint32_t n = h->n;
        if (s0.lr == ASD_LR_FFT) REQUIRE(h->exch == ASD_EXCH_FFT || h->exch == ASD_EXCH_NONE, "FFT field excludes CSR/DIA exchange");
        if (h->exch == ASD_EXCH_FFT) REQUIRE(s0.lr == ASD_LR_FFT, "exchange method fft needs lr = ASD_LR_FFT");
        h->dexch = h->exch;
        // material constants (src/llg.cpp:591-592, src/geom.cpp:244)
        StepConst& sc = h->sc;
        sc.n = n; sc.nmat = h->nmat; sc.nrep = nsys; sc.flags = p.flags;
        const double basemm = s0.mat[0].mu * p.muB;
        std::vector<uint32_t> subs;
        for (uint32_t t = 0; t < h->nmat; t++) {
            const asd_material& m = s0.mat[t];
            REQUIRE(m.mu > 0 && m.lambda >= 0 && m.gamma > 0, "material needs mu>0, lambda>=0, gamma>0");
            REQUIRE(m.sublattice < ASD_MAX_SUB, "sublattice index out of range");
            MatConst& mc = sc.mat[t];
            mc.llgpf = -1. / (1.0 + m.lambda * m.lambda);
            mc.lambda = m.lambda;
            mc.sigma = sqrt(2.0 * p.kB * m.lambda / (m.mu * p.muB * p.dt * m.gamma * p.gyro));
            mc.k1u = 2.0 * m.k1u / (p.muB * m.mu);
            for (int a = 0; a < 3; a++) mc.k1udir[a] = m.k1u_dir[a];
            mc.sub = m.sublattice;
            mc.llgpf_f = (float)mc.llgpf; mc.lambda_f = (float)mc.lambda; mc.sigma_f = (float)mc.sigma;
            mc.k1u_f = (float)mc.k1u;
            for (int a = 0; a < 3; a++) mc.k1udir_f[a] = (float)mc.k1udir[a];
            h->h_sub_of_mat.push_back(m.sublattice);
            h->nsub = std::max(h->nsub, m.sublattice + 1);
        }
        sc.rdt = p.dt * p.gyro;
        sc.dt = p.dt;
        sc.k2perp_f = 2.0 * p.k2perp / basemm;
        sc.k2par_f = 2.0 * p.k2par / basemm;
        sc.k4perp_f = 2.0 * p.k4perp / basemm;
        sc.k4par_f = 2.0 * p.k4par / basemm;
        for (int a = 0; a < 3; a++) { sc.k2perpdir[a] = p.k2perpdir[a]; sc.k2pardir[a] = p.k2pardir[a]; }
        for (int a = 0; a < 9; a++) { sc.k4perpdirs[a] = p.k4perpdirs[a]; sc.k4pardirs[a] = p.k4pardirs[a]; }
        sc.seed = p.seed;
        sc.rdt_f = (float)sc.rdt;
        sc.k2perp_ff = (float)sc.k2perp_f; sc.k2par_ff = (float)sc.k2par_f;
        sc.k4perp_ff = (float)sc.k4perp_f; sc.k4par_ff = (float)sc.k4par_f;
        for (int a = 0; a < 3; a++) { sc.k2perpdir_f[a] = (float)sc.k2perpdir[a]; sc.k2pardir_f[a] = (float)sc.k2pardir[a]; }
        for (int a = 0; a < 9; a++) { sc.k4perpdirs_f[a] = (float)sc.k4perpdirs[a]; sc.k4pardirs_f[a] = (float)sc.k4pardirs[a]; }
        // per-spin atom table (only when not i % nmat)
        bool need_atom = false;
        std::vector<uint32_t> atom(n);
        for (uint32_t r = 0; r < nsys; r++) {
            const asd_system& s = sys[r];
            for (uint32_t i = 0; i < s.nspins; i++) {
                const uint32_t a = s.atom ? s.atom[i] : i % h->nmat;
                REQUIRE(a < h->nmat, "atom index out of range");
                atom[h->h_rep_off[r] + i] = a;
                if (a != (h->h_rep_off[r] + i) % h->nmat) need_atom = true;
            }
        }
        if (need_atom) { h->h_atom = atom; h->d_atom = dupload(atom.data(), n); }
        sc.atom = h->d_atom;
        h->d_rep_off = dupload(h->h_rep_off.data(), h->h_rep_off.size());
        std::vector<double> sq(nsys);
        std::vector<uint32_t> strm(nsys);
        for (uint32_t r = 0; r < nsys; r++) { sq[r] = sqrt(h->h_rep_T[r]); strm[r] = sys[r].stream; }
        h->d_rep_sqrtT = dupload(sq.data(), nsys);
        std::vector<float> sqf(sq.begin(), sq.end());
        h->d_rep_sqrtT_f = dupload(sqf.data(), nsys);
        sc.rep_sqrtT_f = h->d_rep_sqrtT_f;
        h->d_rep_stream = dupload(strm.data(), nsys);
        sc.rep_off = h->d_rep_off; sc.rep_sqrtT = h->d_rep_sqrtT; sc.rep_stream = h->d_rep_stream;
        {
            std::vector<uint32_t> rt((n + 31) / 32);
            uint32_t r = 0;
            for (size_t t = 0; t < rt.size(); t++) {
                while (r + 1 < nsys && h->h_rep_off[r + 1] <= 32 * t) r++;
                rt[t] = r;
            }
            h->d_rep_of_tile = dupload(rt.data(), rt.size());
            sc.rep_of_tile = h->d_rep_of_tile;
        }
        std::vector<double> dyn(DYN_COUNT, 0.0);
        for (int a = 0; a < 3; a++) dyn[DYN_APPLIED + a] = p.applied[a];
        dyn[DYN_STAG_SCALE] = 1.0;
        dyn[DYN_DET_STEP] = -1.0;
        dyn[DYN_PULSE_AMP] = 0.0;
        dyn[DYN_PULSE_T0] = 0.0;
        dyn[DYN_PULSE_ISIG] = 1.0;
        h->d_dyn = dupload(dyn.data(), dyn.size());
        std::vector<float> dynf(dyn.begin(), dyn.end());
        h->d_dynf = dupload(dynf.data(), dynf.size());
        sc.dynf = h->d_dynf;
        h->d_step = dalloc<uint64_t>(1);
        sc.dyn = h->d_dyn; sc.step_base = h->d_step;
        // ---- exchange, concatenated over replicas
        std::vector<uint32_t> xadj(1, 0), adj;
        std::vector<double> val9;
        std::vector<int32_t> doff;
        if (h->exch == ASD_EXCH_CSR) {
            for (uint32_t r = 0; r < nsys; r++) {
                const asd_system& s = sys[r];
                REQUIRE(s.xadj && (s.nnz == 0 || (s.adjncy && s.csr_val)), "CSR arrays missing");
                REQUIRE(s.xadj[0] == 0 && s.xadj[s.nspins] == s.nnz, "xadj must start at 0 and end at nnz");
                const uint32_t off = h->h_rep_off[r], base = (uint32_t)adj.size();
                for (uint32_t i = 0; i < s.nspins; i++) {
                    REQUIRE(s.xadj[i + 1] >= s.xadj[i], "xadj must be non-decreasing");
                    xadj.push_back(base + s.xadj[i + 1]);
                }
                for (uint32_t k = 0; k < s.nnz; k++) {
                    REQUIRE(s.adjncy[k] < s.nspins, "adjncy index out of range");
                    adj.push_back(off + s.adjncy[k]);
                    for (int q = 0; q < 9; q++) {
                        REQUIRE(std::isfinite(s.csr_val[9 * (size_t)k + q]), "non-finite exchange value");
                        val9.push_back(s.csr_val[9 * (size_t)k + q]);
                    }
                }
            }
            h->nnz_per_row = (double)adj.size() / n;
        } else if (h->exch == ASD_EXCH_DIA) {
            REQUIRE(nsys == 1, "DIA exchange supports one replica per handle");
            REQUIRE(s0.ndiag == 0 || (s0.dia_offset && s0.dia_val), "DIA arrays missing");
            doff.assign(s0.dia_offset, s0.dia_offset + s0.ndiag);
            size_t nz = 0;
            const size_t m = (size_t)s0.ndiag * n;
            const int nc = h->full ? 9 : 3;
            for (uint32_t d = 0; d < s0.ndiag; d++)
                for (uint32_t i = 0; i < n; i++) {
                    const int64_t col = (int64_t)i + doff[d];
                    if (col < 0 || col >= (int64_t)n) continue;
                    bool any = false;
                    for (int q = 0; q < nc; q++) any |= s0.dia_val[(size_t)q * m + (size_t)d * n + i] != 0.0;
                    nz += any;
                }
            h->nnz_per_row = (double)nz / n;
        }
        const bool plain = p.precision == ASD_FP64_PLAIN;
        const bool zz_yy = (p.flags & ASD_FLAG_GPU_DZZ_FROM_DYY) != 0;
        // component q (row-major alpha,beta) of the caller's DIA values; the diagonal form
        // carries only xx, yy, zz (q = 0, 4, 8)
        const size_t mdia = (size_t)s0.ndiag * n;
        auto dia_comp = [&](int q) -> const double* {
            if (h->full) return s0.dia_val + (size_t)q * mdia;
            return (q % 4 == 0) ? s0.dia_val + (size_t)(q / 4) * mdia : nullptr;
        };
        if (plain) {
            // reference-structured arrays: per-spin parameters, separate component arrays
            std::vector<double> sig(n), lpf(n), lam(n), k1(n), k1d(3 * (size_t)n);
            for (uint32_t i = 0; i < n; i++) {
                const MatConst& mc = sc.mat[atom[i]];
                sig[i] = mc.sigma; lpf[i] = mc.llgpf; lam[i] = mc.lambda; k1[i] = mc.k1u;
                for (int a = 0; a < 3; a++) k1d[3 * (size_t)i + a] = mc.k1udir[a];
            }
            h->p_sigma = dupload(sig.data(), n); h->p_llgpf = dupload(lpf.data(), n); h->p_lambda = dupload(lam.data(), n);
            h->p_k1u = dupload(k1.data(), n); h->p_k1udir = dupload(k1d.data(), 3 * (size_t)n);
            const size_t n3 = 3 * (size_t)n;
            h->p_s = dalloc<double>(n3); h->p_es = dalloc<double>(n3); h->p_fn = dalloc<double>(n3);
            h->p_ch = dalloc<double>(n3); h->p_hdemag = dalloc<double>(n3); h->p_rand = dalloc<double>(n3);
            h->p_det = dalloc<double>(n3); h->p_hstg = dalloc<double>(n3); h->p_hinit = dalloc<double>(n3);
            if (p.integrator != ASD_HEUN)
                for (int q = 0; q < (p.integrator == ASD_RK4 ? 4 : 6); q++) h->p_k[q] = dalloc<double>(n3);
            if (h->exch == ASD_EXCH_CSR) {
                h->pex.xadj = dupload(xadj.data(), xadj.size());
                h->pex.adjncy = dupload(adj.data(), adj.size());
                std::vector<double> comp(adj.size());
                for (int q = 0; q < 9; q++) {
                    for (size_t k = 0; k < adj.size(); k++) comp[k] = val9[9 * k + q];
                    h->pex.v[q] = dupload(comp.data(), comp.size());
                }
            } else if (h->exch == ASD_EXCH_DIA) {
                h->pex.ndiag = s0.ndiag;
                h->pex.off = dupload(doff.data(), doff.size());
                for (int q = 0; q < 9; q++)
                    if (dia_comp(q)) h->pex.v[q] = dupload(dia_comp(q), mdia);
            }
            (void)zz_yy;  // applied inside the plain kernels
        } else {
            const size_t bytes = p.precision == ASD_FP32 ? 4 : 8;
            for (int c = 0; c < 3; c++) {
                // gather sources carry SPIN_PAD zeroed elements so 16-byte-aligned span copies
                // of neighbour spins stay inside the allocation
                if (bytes == 4) {
                    h->sf[c] = dalloc<float>(n + SPIN_PAD); h->esf[c] = dalloc<float>(n + SPIN_PAD);
                    h->fnf[c] = dalloc<float>(n + SPIN_PAD);
                    h->nzf[c] = dalloc<float>(n);
                    h->detf[c] = dalloc<float>(n);
                    if (p.flags & ASD_FLAG_COMPENSATED) h->sl[c] = dalloc<float>(n);
                    if (p.integrator != ASD_HEUN)
                        for (int q = 0; q < (p.integrator == ASD_RK4 ? 3 : 5); q++) h->kf[q][c] = dalloc<float>(n);
                } else {
                    h->sd[c] = dalloc<double>(n + SPIN_PAD); h->esd[c] = dalloc<double>(n + SPIN_PAD);
                    h->fnd[c] = dalloc<double>(n + SPIN_PAD);
                    h->nzd[c] = dalloc<double>(n);
                    h->detd[c] = dalloc<double>(n);
                    if (p.integrator != ASD_HEUN)
                        for (int q = 0; q < (p.integrator == ASD_RK4 ? 3 : 5); q++) h->kd[q][c] = dalloc<double>(n);
                }
            }
            if (h->exch == ASD_EXCH_CSR) {
                build_sell(h, xadj, adj, val9);
                build_dia_alt(h, xadj, adj, val9);
            } else if (h->exch == ASD_EXCH_DIA) {
                h->dia.ndiag = s0.ndiag;
                h->dia.off = dupload(doff.data(), doff.size());
                const size_t m = (size_t)s0.ndiag * n;
                const int nc = h->full ? 9 : 3;
                const int qmap3[3] = {0, 4, zz_yy ? 4 : 8};
                {
                    // active diagonals of every 32-row tile: a periodic lattice has many distinct
                    // offsets, each row only a few nonzero ones
                    const uint32_t nt = (n + 31) / 32;
                    std::vector<uint32_t> tp(nt + 1, 0), td;
                    const double* comp[9];
                    for (int q = 0; q < nc; q++) comp[q] = dia_comp(h->full ? q : qmap3[q]);
                    for (uint32_t w = 0; w < nt; w++) {
                        const uint32_t r0 = 32 * w, r1 = std::min(n, r0 + 32);
                        for (uint32_t d = 0; d < s0.ndiag; d++) {
                            bool any = false;
                            for (uint32_t r = r0; r < r1 && !any; r++) {
                                const int64_t col = (int64_t)r + doff[d];
                                if (col < 0 || col >= (int64_t)n) continue;
                                for (int q = 0; q < nc && !any; q++) any = comp[q][(size_t)d * n + r] != 0.0;
                            }
                            if (any) td.push_back(d);
                        }
                        tp[w + 1] = (uint32_t)td.size();
                    }
                    h->dia.tile_ptr = dupload(tp.data(), tp.size());
                    h->dia.tile_diag = dupload(td.data(), std::max<size_t>(td.size(), 1));
                }
                bool typed = false;
                if (!(p.flags & ASD_FLAG_STREAMED_EXCHANGE)) {
                    // typed DIA: one id byte per (diagonal, row) into the distinct tensors
                    TensorTable tt(nc);
                    std::vector<uint8_t> ids(m, 0);
                    const double* comp[9];
                    for (int q = 0; q < nc; q++) comp[q] = dia_comp(h->full ? (q == 8 && zz_yy ? 4 : q) : qmap3[q]);
                    bool ok = true;
                    for (size_t k = 0; k < m && ok; k++) {
                        std::array<double, 9> key{};
                        for (int q = 0; q < nc; q++) key[q] = comp[q][k];
                        const int64_t t = tt.id(key);
                        if (t < 0) ok = false; else ids[k] = (uint8_t)t;
                    }
                    if (ok) {
                        h->dia.dtype = dupload(ids.data(), ids.size());
                        h->dia.ntypes = tt.size();
                        if (bytes == 4) { std::vector<float> tf = tt.table<float>(); h->dia.tab_f = dupload(tf.data(), tf.size()); }
                        else { std::vector<double> td = tt.table<double>(); h->dia.tab_d = dupload(td.data(), td.size()); }
                        typed = true;
                    }
                }
                if (typed) {
                } else if (bytes == 4) {
                    std::vector<float> v(nc * m);
                    for (int q = 0; q < nc; q++) {
                        int src = h->full ? (q == 8 && zz_yy ? 4 : q) : qmap3[q];
                        const double* sp = dia_comp(src);
                        for (size_t k = 0; k < m; k++) v[q * m + k] = (float)sp[k];
                    }
                    h->dia.valf = dupload(v.data(), v.size());
                } else {
                    std::vector<double> v(nc * m);
                    for (int q = 0; q < nc; q++) {
                        int src = h->full ? (q == 8 && zz_yy ? 4 : q) : qmap3[q];
                        const double* sp = dia_comp(src);
                        for (size_t k = 0; k < m; k++) v[q * m + k] = sp[k];
                    }
                    h->dia.vald = dupload(v.data(), v.size());
                }
                // the same matrix as SELL-32 for the fused kernels: rows take their entries in
                // ascending diagonal order, the order the DIA gather sums them in
                {
                    std::vector<uint32_t> cx(n + 1, 0), ca;
                    std::vector<double> cv;
                    for (uint32_t i = 0; i < n; i++) {
                        for (uint32_t d = 0; d < s0.ndiag; d++) {
                            const int64_t col = (int64_t)i + doff[d];
                            if (col < 0 || col >= (int64_t)n) continue;
                            double v9[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
                            bool any = false;
                            for (int q = 0; q < 9; q++) {
                                const double* cp = dia_comp(q);
                                if (cp) { v9[q] = cp[(size_t)d * n + i]; any |= v9[q] != 0.0; }
                            }
                            if (!any) continue;
                            ca.push_back((uint32_t)col);
                            cv.insert(cv.end(), v9, v9 + 9);
                        }
                        cx[i + 1] = (uint32_t)ca.size();
                    }
                    build_sell(h, cx, ca, cv);
                    h->dexch = ASD_EXCH_CSR;
                }
            }
        }
        // ---- site fields
        bool any_site = false;
        for (uint32_t r = 0; r < nsys; r++) any_site |= sys[r].site_field != nullptr;
        h->has_site = any_site;
        if (any_site) {
            std::vector<double> prof(3 * (size_t)n, 0.0);
            for (uint32_t r = 0; r < nsys; r++)
                if (sys[r].site_field)
                    std::copy(sys[r].site_field, sys[r].site_field + 3 * (size_t)sys[r].nspins, prof.begin() + 3 * (size_t)h->h_rep_off[r]);
            if (plain) {
                CK(cudaMemcpy(h->p_hinit, prof.data(), prof.size() * 8, cudaMemcpyHostToDevice));
                CK(cudaMemcpy(h->p_hstg, prof.data(), prof.size() * 8, cudaMemcpyHostToDevice));
            } else {
                for (int c = 0; c < 3; c++) {
                    std::vector<double> comp(n);
                    for (uint32_t i = 0; i < n; i++) comp[i] = prof[3 * (size_t)i + c];
                    if (p.precision == ASD_FP32) {
                        std::vector<float> f(comp.begin(), comp.end());
                        h->stagf[c] = dupload(f.data(), n);
                    } else {
                        h->stagd[c] = dupload(comp.data(), n);
                    }
                }
            }
        }
        // ---- long-range field
        if (s0.lr != ASD_LR_NONE) setup_lr(h, s0, plain);
        // ---- magnetisation buffers
        {
            uint32_t maxrep = 0;
            for (uint32_t r = 0; r < nsys; r++) maxrep = std::max(maxrep, h->h_rep_off[r + 1] - h->h_rep_off[r]);
            const uint32_t nchunk = (maxrep + MAG_CHUNK - 1) / MAG_CHUNK;
            h->magpart_len = (size_t)nsys * nchunk * h->nsub * 3;
            h->d_magpart = dalloc<double>(h->magpart_len);
            h->d_mag = dalloc<double>((size_t)nsys * h->nsub * 3);
            h->d_magcnt = dalloc<uint32_t>(1);
            CK(cudaMemset(h->d_magcnt, 0, sizeof(uint32_t)));
            h->d_stats = dalloc<double>((size_t)nsys * h->nsub * 4);
            std::vector<double> inv((size_t)nsys * h->nsub, 0.0);
            for (uint32_t r = 0; r < nsys; r++) {
                std::vector<uint32_t> cnt(h->nsub, 0);
                for (uint32_t i = h->h_rep_off[r]; i < h->h_rep_off[r + 1]; i++) cnt[h->h_sub_of_mat[atom[i]]]++;
                for (uint32_t s = 0; s < h->nsub; s++) inv[r * h->nsub + s] = cnt[s] ? 1. / (double)cnt[s] : 0.0;
            }
            h->d_inv_count = dupload(inv.data(), inv.size());
            h->d_sub_of_atom = dupload(h->h_sub_of_mat.data(), h->h_sub_of_mat.size());
        }
        // ---- default spins +z, then a graph for the fused forms
        {
            std::vector<double> s3(3 * (size_t)n, 0.0);
            for (uint32_t i = 0; i < n; i++) s3[3 * (size_t)i + 2] = 1.0;
            int rc = asd_set_spins(h, s3.data(), n);
            if (rc != ASD_OK) throw Fail{rc, h->err};
        }
        CK(cudaEventCreate(&h->kev[0]));
        CK(cudaEventCreate(&h->kev[1]));
        h->d_err = dalloc<uint32_t>(1);
        h->sell.err = h->d_err;
        CK(cudaHostAlloc(reinterpret_cast<void**>(&h->h_err), sizeof(uint32_t), cudaHostAllocDefault));
        if (!plain) {
            if (p.flags & ASD_FLAG_AUTOTUNE) autotune(h);
            else configure_stage(h, 256, 1);
            if (h->tune.empty()) {
                static const char* names[3] = {"direct", "words", "words+spins"};
                char b[64];
                std::snprintf(b, sizeof b, "block=%d staging=%s (default)", h->block, names[h->sell.stage]);
                h->tune = b;
            }
            const uint32_t upd = p.update;
            uint32_t G = 32;
            if (s0.lr == ASD_LR_DIPOLE) G = upd * std::max<uint32_t>(1, 32 / upd);
            if (G > 4096) G = upd;
            build_graph(h, G);
        }
        CK(cudaStreamSynchronize(h->stream));
    } catch (const Fail& f) {
        g_create_err = f.msg;
        int code = f.code;
        free_all(h);
        delete h;
        return code;
    }
    *out = h;
    return ASD_OK;
}

int asd_destroy(asd_handle* h) {
    if (!h) return ASD_EINVAL;
    cudaSetDevice(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    free_all(h);
    delete h;
    return ASD_OK;
}

// Device staging buffer of 3N doubles for the spin / field transfers, allocated on first use
// and kept (no allocation or device-wide synchronisation per call).
static double* aos_buffer(asd_handle* h) {
    if (!h->d_aos) h->d_aos = dalloc<double>(3 * (size_t)h->n);
    return h->d_aos;
}

// The spins are uploaded to the staging buffer and checked there (every component finite, every
// squared length above 1e-24: the first offender is reported, as a host scan would); only a
// valid array is converted into the state, so a rejected call leaves the state unchanged.
int asd_set_spins(asd_handle* h, const double* s, size_t n_spins) {
    if (!h) return ASD_EINVAL;
    try {
        REQUIRE(s && n_spins == h->n, "spin array must hold 3*nspins doubles");
        CK(cudaSetDevice(h->device));
        double* d = aos_buffer(h);
        if (!h->d_check) h->d_check = dalloc<unsigned long long>(2);
        unsigned long long bad[2] = {0, 0};
        cudaError_t e = cudaMemcpyAsync(d, s, 3 * n_spins * sizeof(double), cudaMemcpyHostToDevice, h->stream);
        if (e == cudaSuccess) e = launch_check_spins(h, d, h->d_check);
        if (e == cudaSuccess) e = cudaMemcpyAsync(bad, h->d_check, sizeof(bad), cudaMemcpyDeviceToHost, h->stream);
        cudaError_t e2 = cudaStreamSynchronize(h->stream);
        CK(e);
        CK(e2);
        if (bad[0] != ~0ull) throw Fail{ASD_ENOTFINITE, "non-finite spin component at index " + std::to_string(bad[0])};
        REQUIRE(bad[1] == ~0ull, "zero-length spin at index " + std::to_string(bad[1]));
        e = launch_convert_spins_in(h, d);
        e2 = cudaStreamSynchronize(h->stream);
        CK(e);
        CK(e2);
        h->lr_scattered = false;
    } catch (const Fail& f) { return fail(h, f); }
    return ASD_OK;
}

static int read_back(asd_handle* h, int what, double* out, size_t n_spins) {
    try {
        REQUIRE(out && n_spins == h->n, "output must hold 3*nspins doubles");
        CK(cudaSetDevice(h->device));
        const size_t bytes = 3 * n_spins * sizeof(double);
        if (h->p.precision == ASD_FP64_PLAIN && what != 2) {
            CK(cudaMemcpyAsync(out, what == 0 ? h->p_s : h->p_det, bytes, cudaMemcpyDeviceToHost, h->stream));
            CK(cudaStreamSynchronize(h->stream));
            return ASD_OK;
        }
        double* d = aos_buffer(h);
        if (what == 2) flush_applied(h);
        cudaError_t e = what == 2 ? launch_field_only(h, d) : launch_convert_out(h, what, d);
        if (e == cudaSuccess) e = cudaMemcpyAsync(out, d, bytes, cudaMemcpyDeviceToHost, h->stream);
        cudaError_t e2 = cudaStreamSynchronize(h->stream);
        CK(e);
        CK(e2);
    } catch (const Fail& f) { return fail(h, f); }
    return ASD_OK;
}

int asd_get_spins(asd_handle* h, double* s, size_t n) { return h ? read_back(h, 0, s, n) : ASD_EINVAL; }
int asd_get_det_field(asd_handle* h, double* o, size_t n) { return h ? read_back(h, 1, o, n) : ASD_EINVAL; }
int asd_get_field(asd_handle* h, double* o, size_t n) {
    if (!h) return ASD_EINVAL;
    try { CK(cudaSetDevice(h->device)); scatter_if_needed(h); } catch (const Fail& f) { return fail(h, f); }
    return read_back(h, 2, o, n);
}

int asd_step(asd_handle* h, uint64_t nsteps) {
    if (!h) return ASD_EINVAL;
    try {
        CK(cudaSetDevice(h->device));
        run_steps(h, nsteps);
        CK(cudaGetLastError());
    } catch (const Fail& f) { return fail(h, f); }
    return ASD_OK;
}

int asd_get_step(const asd_handle* h, uint64_t* t) {
    if (!h || !t) return ASD_EINVAL;
    *t = h->step;
    return ASD_OK;
}

int asd_set_step(asd_handle* h, uint64_t t) {
    if (!h) return ASD_EINVAL;
    try {
        CK(cudaSetDevice(h->device));
        CK(cudaMemcpyAsync(h->d_step, &t, sizeof(t), cudaMemcpyHostToDevice, h->stream));
        CK(cudaStreamSynchronize(h->stream));
        h->step = t;
    } catch (const Fail& f) { return fail(h, f); }
    return ASD_OK;
}

// ---- exact state (checkpoint and restart)
namespace {
struct StateHeader {
    char magic[4];          // "ASDS"
    uint32_t version;       // 1
    uint32_t precision, flags_comp, n, nrep, has_ttm, reserved;
    uint64_t step;
};

size_t state_bytes(const asd_handle* h) {
    size_t b = sizeof(StateHeader);
    const size_t n3 = 3 * (size_t)h->n;
    if (h->p.precision == ASD_FP32) b += n3 * sizeof(float) * ((h->p.flags & ASD_FLAG_COMPENSATED) ? 2 : 1);
    else b += n3 * sizeof(double);
    b += (size_t)h->nrep * (sizeof(double) + sizeof(float));
    if (h->d_ttm) b += sizeof(TtmDev);
    return b;
}
}  // namespace

int asd_get_state(asd_handle* h, void* buf, size_t* len) {
    if (!h || !len) return ASD_EINVAL;
    try {
        const size_t need = state_bytes(h);
        if (!buf) { *len = need; return ASD_OK; }
        REQUIRE(*len >= need, "state buffer too small (asd_get_state with buf = NULL gives the size)");
        CK(cudaSetDevice(h->device));
        StateHeader hd{};
        memcpy(hd.magic, "ASDS", 4);
        hd.version = 1;
        hd.precision = h->p.precision;
        hd.flags_comp = (h->p.flags & ASD_FLAG_COMPENSATED) ? 1 : 0;
        hd.n = h->n; hd.nrep = h->nrep; hd.has_ttm = h->d_ttm ? 1 : 0;
        hd.step = h->step;
        unsigned char* o = static_cast<unsigned char*>(buf);
        memcpy(o, &hd, sizeof hd);
        o += sizeof hd;
        const size_t n = h->n;
        auto get = [&](const void* d, size_t bytes) {
            CK(cudaMemcpyAsync(o, d, bytes, cudaMemcpyDeviceToHost, h->stream));
            o += bytes;
        };
        if (h->p.precision == ASD_FP32) {
            for (int c = 0; c < 3; c++) get(h->sf[c], n * sizeof(float));
            if (hd.flags_comp)
                for (int c = 0; c < 3; c++) get(h->sl[c], n * sizeof(float));
        } else if (h->p.precision == ASD_FP64_FUSED) {
            for (int c = 0; c < 3; c++) get(h->sd[c], n * sizeof(double));
        } else {
            get(h->p_s, 3 * n * sizeof(double));
        }
        get(h->d_rep_sqrtT, h->nrep * sizeof(double));
        get(h->d_rep_sqrtT_f, h->nrep * sizeof(float));
        if (h->d_ttm) get(h->d_ttm, sizeof(TtmDev));
        CK(cudaStreamSynchronize(h->stream));
        *len = need;
    } catch (const Fail& f) { return fail(h, f); }
    return ASD_OK;
}

int asd_set_state(asd_handle* h, const void* buf, size_t len) {
    if (!h || !buf) return ASD_EINVAL;
    try {
        StateHeader hd{};
        REQUIRE(len >= sizeof hd, "state too short");
        memcpy(&hd, buf, sizeof hd);
        REQUIRE(memcmp(hd.magic, "ASDS", 4) == 0 && hd.version == 1, "not a state of this library");
        REQUIRE(hd.precision == h->p.precision && hd.n == h->n && hd.nrep == h->nrep &&
                    hd.flags_comp == ((h->p.flags & ASD_FLAG_COMPENSATED) ? 1u : 0u),
                "state taken from a handle of another form or lattice");
        REQUIRE(len == state_bytes(h) + (hd.has_ttm && !h->d_ttm ? sizeof(TtmDev) : 0) -
                           (!hd.has_ttm && h->d_ttm ? sizeof(TtmDev) : 0),
                "state size does not match the handle");
        REQUIRE(!hd.has_ttm || h->d_ttm, "the state carries a two-temperature model: start it (asd_set_ttm) first");
        CK(cudaSetDevice(h->device));
        const unsigned char* in = static_cast<const unsigned char*>(buf) + sizeof hd;
        const size_t n = h->n;
        auto put = [&](void* d, size_t bytes) {
            CK(cudaMemcpyAsync(d, in, bytes, cudaMemcpyHostToDevice, h->stream));
            in += bytes;
        };
        if (h->p.precision == ASD_FP32) {
            for (int c = 0; c < 3; c++) put(h->sf[c], n * sizeof(float));
            if (hd.flags_comp)
                for (int c = 0; c < 3; c++) put(h->sl[c], n * sizeof(float));
        } else if (h->p.precision == ASD_FP64_FUSED) {
            for (int c = 0; c < 3; c++) put(h->sd[c], n * sizeof(double));
        } else {
            put(h->p_s, 3 * n * sizeof(double));
        }
        put(h->d_rep_sqrtT, h->nrep * sizeof(double));
        put(h->d_rep_sqrtT_f, h->nrep * sizeof(float));
        if (hd.has_ttm) put(h->d_ttm, sizeof(TtmDev));
        CK(cudaMemcpyAsync(h->d_step, &hd.step, sizeof hd.step, cudaMemcpyHostToDevice, h->stream));
        CK(cudaStreamSynchronize(h->stream));
        h->step = hd.step;
        // host copies of the bath temperatures follow the device
        std::vector<double> sq(h->nrep);
        memcpy(sq.data(), static_cast<const unsigned char*>(buf) + len - (hd.has_ttm ? sizeof(TtmDev) : 0) -
                              h->nrep * (sizeof(double) + sizeof(float)),
               h->nrep * sizeof(double));
        for (uint32_t r = 0; r < h->nrep; r++) h->h_rep_T[r] = sq[r] * sq[r];
        h->lr_scattered = false;    // the long-range input is formed again from these spins
    } catch (const Fail& f) { return fail(h, f); }
    return ASD_OK;
}

int asd_sync(asd_handle* h) {
    if (!h) return ASD_EINVAL;
    try {
        CK(cudaSetDevice(h->device));
        // the error bits ride the stream behind its work: one copy, one wait
        uint32_t e = 0;
        if (h->d_err) CK(cudaMemcpyAsync(h->h_err, h->d_err, sizeof e, cudaMemcpyDeviceToHost, h->stream));
        CK(cudaStreamSynchronize(h->stream));
        if (h->d_err) e = *h->h_err;
        if (e & 2u) {
            CK(cudaMemset(h->d_err, 0, sizeof(uint32_t)));
            throw Fail{ASD_ETIMEOUT, "a long-range transform block's bulk-copy wait ran out; the long-range field of "
                                     "that evaluation is invalid"};
        }
        if (e & 1u) {
            CK(cudaMemset(h->d_err, 0, sizeof(uint32_t)));
            throw Fail{ASD_ETIMEOUT, "a stage kernel's shared-memory staging wait ran out; those blocks read the "
                                     "exchange words from global memory instead (results unaffected)"};
        }
    } catch (const Fail& f) { return fail(h, f); }
    return ASD_OK;
}

int asd_set_launch_shape(asd_handle* h, uint32_t block, uint32_t staging) {
    if (!h) return ASD_EINVAL;
    try {
        REQUIRE(block == 64 || block == 128 || block == 256, "block must be 64, 128 or 256");
        REQUIRE(staging <= 2, "staging must be 0, 1 or 2");
        if (h->p.precision == ASD_FP64_PLAIN) return ASD_OK;
        CK(cudaSetDevice(h->device));
        CK(cudaStreamSynchronize(h->stream));
        configure_stage(h, (int)block, (int)staging);
        static const char* names[3] = {"direct", "words", "words+spins"};
        char b[64];
        std::snprintf(b, sizeof b, "block=%d staging=%s (set)", h->block, names[h->sell.stage]);
        h->tune = b;
        if (h->graph_steps) build_graph(h, h->graph_steps);
    } catch (const Fail& f) { return fail(h, f); }
    return ASD_OK;
}

int asd_set_device_layout(asd_handle* h, uint32_t layout) {
    if (!h) return ASD_EINVAL;
    try {
        REQUIRE(layout == ASD_EXCH_CSR || layout == ASD_EXCH_DIA, "layout must be ASD_EXCH_CSR or ASD_EXCH_DIA");
        if (h->p.precision == ASD_FP64_PLAIN) return ASD_OK;
        REQUIRE(layout == h->exch || (h->exch == ASD_EXCH_DIA && h->sell.slice_ptr) ||
                    (h->exch == ASD_EXCH_CSR && h->dia_alt),
                "this CSR matrix has no DIA device layout (more than 32 diagonals, several replicas or streamed)");
        CK(cudaSetDevice(h->device));
        CK(cudaStreamSynchronize(h->stream));
        h->dexch = layout;
        configure_stage(h, h->block, h->sell.stage);
        h->tune = std::string(layout == ASD_EXCH_CSR ? "layout=SELL " : "layout=DIA ") + h->tune;
        if (h->graph_steps) build_graph(h, h->graph_steps);
    } catch (const Fail& f) { return fail(h, f); }
    return ASD_OK;
}

int asd_set_four_spin(asd_handle* h, const uint32_t* xadj_jkl, const uint32_t* adj_j, const uint32_t* adj_k,
                      const uint32_t* adj_l, double JQ, int divide_by_3) {
    if (!h) return ASD_EINVAL;
    try {
        CK(cudaSetDevice(h->device));
        CK(cudaStreamSynchronize(h->stream));
        if (h->d_q4ptr) { CK(cudaFree(h->d_q4ptr)); h->d_q4ptr = nullptr; }
        if (h->d_q4jkl) { CK(cudaFree(h->d_q4jkl)); h->d_q4jkl = nullptr; }
        h->sc.q4_ptr = nullptr;
        h->sc.q4_jkl = nullptr;
        if (xadj_jkl) {
            REQUIRE(adj_j && adj_k && adj_l && std::isfinite(JQ), "quartet lists and a finite JQ are required");
            REQUIRE(xadj_jkl[0] == 0, "xadj_jkl[0] must be 0");
            for (uint32_t i = 0; i < h->n; i++) REQUIRE(xadj_jkl[i + 1] >= xadj_jkl[i], "xadj_jkl must not decrease");
            const uint32_t nq = xadj_jkl[h->n];
            std::vector<uint4> q(std::max<uint32_t>(nq, 1), make_uint4(0, 0, 0, 0));
            for (uint32_t k = 0; k < nq; k++) {
                REQUIRE(adj_j[k] < h->n && adj_k[k] < h->n && adj_l[k] < h->n, "quartet spin index out of range");
                q[k] = make_uint4(adj_j[k], adj_k[k], adj_l[k], 0);
            }
            h->d_q4ptr = dupload(xadj_jkl, (size_t)h->n + 1);
            h->d_q4jkl = dupload(q.data(), q.size());
            h->sc.q4_ptr = h->d_q4ptr;
            h->sc.q4_jkl = h->d_q4jkl;
            h->sc.q4_jq = JQ;
            h->sc.q4_div3 = divide_by_3 ? 1 : 0;
            h->sc.q4_jq_f = (float)(divide_by_3 ? JQ / 3.0 : JQ);
        }
        if (h->graph_steps) build_graph(h, h->graph_steps);   // the step kernels carry the constants
    } catch (const Fail& f) { return fail(h, f); }
    return ASD_OK;
}

int asd_set_ttm(asd_handle* h, const asd_ttm* m) {
    if (!h) return ASD_EINVAL;
    try {
        CK(cudaSetDevice(h->device));
        CK(cudaStreamSynchronize(h->stream));
        if (!m) {
            if (h->d_ttm) { CK(cudaFree(h->d_ttm)); h->d_ttm = nullptr; }
        } else {
            // the model divides by gamma_e Te, Cl and the cooling time (src/laser_heating.cpp:79-83)
            REQUIRE(m->initial_T > 1e-5 && std::isfinite(m->initial_T), "initial temperature must be > 1e-5 K");
            REQUIRE(m->gamma_e > 0 && m->Cl > 0 && m->cooling_time > 0 && m->pump_time > 0,
                    "gamma_e, Cl, cooling_time and pump_time must be positive");
            REQUIRE(std::isfinite(m->G_ep) && std::isfinite(m->pump_fluence), "G_ep, pump_fluence");
            REQUIRE(m->npulses <= ASD_TTM_MAX_PULSES, "too many pulses");
            TtmDev d{};
            d.Te = d.Tl = d.T0 = m->initial_T;
            d.G = m->G_ep; d.Cl = m->Cl; d.ge = m->gamma_e; d.dt = h->p.dt; d.ct = m->cooling_time;
            d.tau = m->pump_time; d.P = m->pump_fluence; d.t0 = h->step; d.np = m->npulses;
            d.bath_e = m->bath_is_electrons ? 1u : 0u;
            for (uint32_t q = 0; q < m->npulses; q++) { d.scale[q] = m->pulse_scale[q]; d.delay[q] = m->pulse_delay[q]; }
            if (!h->d_ttm) CK(cudaMalloc(&h->d_ttm, sizeof(TtmDev)));
            CK(cudaMemcpy(h->d_ttm, &d, sizeof d, cudaMemcpyHostToDevice));
            for (auto& T : h->h_rep_T) T = m->initial_T;   // the bath is hot from now on
        }
        if (h->graph_steps) build_graph(h, h->graph_steps);   // the step kernels change
    } catch (const Fail& f) { return fail(h, f); }
    return ASD_OK;
}

int asd_get_ttm_temperatures(asd_handle* h, double* Te, double* Tl) {
    if (!h || !Te || !Tl) return ASD_EINVAL;
    try {
        if (!h->d_ttm) throw Fail{ASD_ESTATE, "the two-temperature model is not running"};
        CK(cudaSetDevice(h->device));
        TtmDev d{};
        CK(cudaMemcpyAsync(&d, h->d_ttm, sizeof d, cudaMemcpyDeviceToHost, h->stream));
        CK(cudaStreamSynchronize(h->stream));
        *Te = d.Te;
        *Tl = d.Tl;
    } catch (const Fail& f) { return fail(h, f); }
    return ASD_OK;
}

int asd_tuning(const asd_handle* h, char* out, size_t out_len) {
    if (!h || !out || out_len == 0) return ASD_EINVAL;
    const LongRange& L = h->lr;
    const char* lr = L.mode == ASD_LR_NONE ? "" : h->p.precision == ASD_FP64_PLAIN ? "; long-range: cuFFT Z2Z 3D"
                     : L.planes ? "; long-range: plane kernels" : L.pruned ? "; long-range: z-pass + cuFFT 2D planes"
                                                                       : "; long-range: cuFFT R2C/C2R 3D";
    std::snprintf(out, out_len, "%s%s", h->tune.c_str(), lr);
    return ASD_OK;
}

int asd_set_temperature(asd_handle* h, uint32_t replica, double T) {
    if (!h) return ASD_EINVAL;
    try {
        REQUIRE(T >= 0 && std::isfinite(T), "temperature must be >= 0");
        REQUIRE(replica == ASD_ALL_REPLICAS || replica < h->nrep, "replica out of range");
        CK(cudaSetDevice(h->device));
        for (uint32_t r = 0; r < h->nrep; r++) {
            if (replica != ASD_ALL_REPLICAS && r != replica) continue;
            h->h_rep_T[r] = T;
            CK(launch_set_scalar(h, h->d_rep_sqrtT + r, sqrt(T)));
            CK(launch_set_scalar_f(h, h->d_rep_sqrtT_f + r, (float)sqrt(T)));
        }
    } catch (const Fail& f) { return fail(h, f); }
    return ASD_OK;
}

int asd_set_applied(asd_handle* h, const double applied[3]) {
    if (!h || !applied) return ASD_EINVAL;
    try {
        CK(cudaSetDevice(h->device));
        for (int a = 0; a < 3; a++) REQUIRE(std::isfinite(applied[a]), "non-finite applied field");
        for (int a = 0; a < 3; a++) h->p.applied[a] = applied[a];
        if (h->graph1 && h->det_node) {
            // the one-step graph's first node carries it (a parameter update, no launch); any
            // other work that reads it flushes it first
            CK(update_det_applied(h));
            h->applied_pending = true;
        } else {
            CK(launch_set_vec3(h, h->d_dyn + DYN_APPLIED, h->d_dynf + DYN_APPLIED, applied));
            h->applied_pending = false;
        }
    } catch (const Fail& f) { return fail(h, f); }
    return ASD_OK;
}

int asd_set_site_field(asd_handle* h, const double* prof, size_t n_spins) {
    if (!h) return ASD_EINVAL;
    try {
        REQUIRE(prof == nullptr || n_spins == h->n, "site field must hold 3*nspins doubles");
        CK(cudaSetDevice(h->device));
        const uint32_t n = h->n;
        std::vector<double> v(3 * (size_t)n, 0.0);
        if (prof) v.assign(prof, prof + 3 * (size_t)n);
        if (h->p.precision == ASD_FP64_PLAIN) {
            CK(cudaMemcpy(h->p_hinit, v.data(), v.size() * 8, cudaMemcpyHostToDevice));
            CK(cudaMemcpy(h->p_hstg, v.data(), v.size() * 8, cudaMemcpyHostToDevice));
        } else {
            bool had = h->stagf[0] || h->stagd[0];
            for (int c = 0; c < 3; c++) {
                std::vector<double> comp(n);
                for (uint32_t i = 0; i < n; i++) comp[i] = v[3 * (size_t)i + c];
                if (h->p.precision == ASD_FP32) {
                    std::vector<float> f(comp.begin(), comp.end());
                    if (!h->stagf[c]) h->stagf[c] = dalloc<float>(n);
                    CK(cudaMemcpy(h->stagf[c], f.data(), 4 * (size_t)n, cudaMemcpyHostToDevice));
                } else {
                    if (!h->stagd[c]) h->stagd[c] = dalloc<double>(n);
                    CK(cudaMemcpy(h->stagd[c], comp.data(), 8 * (size_t)n, cudaMemcpyHostToDevice));
                }
            }
            if (!had) build_graph(h, h->graph_steps ? h->graph_steps : 32);  // kernels now read the profile
        }
        // CsetStagFields resets the ramp: CHstg = CInitHstg
        set_dyn(h, DYN_STAG_SCALE, 1.0);
        h->stag_rv = 1.0;
        h->has_site = prof != nullptr;
    } catch (const Fail& f) { return fail(h, f); }
    return ASD_OK;
}

int asd_set_site_field_scale(asd_handle* h, double rv) {
    if (!h) return ASD_EINVAL;
    try {
        REQUIRE(std::isfinite(rv), "non-finite scale");
        CK(cudaSetDevice(h->device));
        if (h->p.precision == ASD_FP64_PLAIN) CK(launch_plain_ramp(h, rv));
        else set_dyn(h, DYN_STAG_SCALE, rv);
        h->stag_rv = rv;
    } catch (const Fail& f) { return fail(h, f); }
    return ASD_OK;
}

int asd_set_site_field_pulse(asd_handle* h, double amp, double t0, double sigma) {
    if (!h) return ASD_EINVAL;
    try {
        REQUIRE(std::isfinite(amp) && std::isfinite(t0) && std::isfinite(sigma), "non-finite pulse parameter");
        REQUIRE(amp == 0.0 || sigma > 0.0, "pulse width must be positive");
        CK(cudaSetDevice(h->device));
        h->pulse_amp = amp;
        h->pulse_t0 = t0;
        h->pulse_sigma = amp == 0.0 ? 1.0 : sigma;
        if (h->p.precision == ASD_FP64_PLAIN) {
            if (amp == 0.0) CK(launch_plain_ramp(h, h->stag_rv));   // back to the plain ramp value
        } else {
            set_dyn(h, DYN_PULSE_T0, t0);
            set_dyn(h, DYN_PULSE_ISIG, 1.0 / h->pulse_sigma);
            set_dyn(h, DYN_PULSE_AMP, amp);
        }
    } catch (const Fail& f) { return fail(h, f); }
    return ASD_OK;
}

int asd_sample_magnetisation(asd_handle* h) {
    if (!h) return ASD_EINVAL;
    try {
        CK(cudaSetDevice(h->device));
        CK(launch_magnetisation(h));
        CK(launch_mag_push(h));
    } catch (const Fail& f) { return fail(h, f); }
    return ASD_OK;
}

int asd_magnetisation_stats(asd_handle* h, double* out, size_t out_len) {
    if (!h) return ASD_EINVAL;
    try {
        const size_t m = (size_t)h->nrep * h->nsub * 4;
        REQUIRE(out && out_len >= m, "output must hold nrep*nsub*4 doubles");
        CK(cudaSetDevice(h->device));
        CK(cudaMemcpyAsync(out, h->d_stats, m * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
        CK(cudaStreamSynchronize(h->stream));
        for (size_t q = 0; q < m; q += 4) {           // M2 -> variance (n-1 normalised), inc/util.h:68-71
            const double n = out[q];
            out[q + 2] = n > 1 ? out[q + 2] / (n - 1) : 0.0;
        }
    } catch (const Fail& f) { return fail(h, f); }
    return ASD_OK;
}

int asd_sq_setup(asd_handle* h, uint32_t qaxis, const double* uo, const uint32_t mesh[3], const uint32_t* mesh_xyz,
                 uint32_t nk, const uint32_t* kpoints, uint32_t max_samples) {
    if (!h) return ASD_EINVAL;
    try {
        REQUIRE(h->nrep == 1, "S(q,t) sampling supports one replica per handle");
        REQUIRE(qaxis <= 2, "qaxis must be 0, 1 or 2");
        REQUIRE(mesh && mesh_xyz && kpoints && nk > 0 && max_samples > 0, "mesh, mesh_xyz, kpoints, nk, max_samples");
        REQUIRE(mesh[0] && mesh[1] && mesh[2], "empty mesh");
        const size_t P = (size_t)mesh[0] * mesh[1] * mesh[2];
        REQUIRE(P < (1ull << 31) && (size_t)max_samples * nk < (1ull << 31), "sampler too large");
        CK(cudaSetDevice(h->device));
        SqSampler& S = h->sq;
        auto F = [](void* p) { if (p) cudaFree(p); };
        F(S.idx); F(S.sub); F(S.uo); F(S.kidx); F(S.grid); F(S.series);
        if (S.plan) cufftDestroy(S.plan);
        S = SqSampler{};
        std::vector<uint32_t> idx(h->n), sub(h->n), kidx(nk);
        for (uint32_t i = 0; i < h->n; i++) {
            const uint32_t x = mesh_xyz[3 * i], y = mesh_xyz[3 * i + 1], z = mesh_xyz[3 * i + 2];
            REQUIRE(x < mesh[0] && y < mesh[1] && z < mesh[2], "mesh_xyz outside the mesh");
            idx[i] = (uint32_t)(((size_t)x * mesh[1] + y) * mesh[2] + z);
            sub[i] = h->h_sub_of_mat[h->h_atom.empty() ? i % h->nmat : h->h_atom[i]];
        }
        for (uint32_t q = 0; q < nk; q++) {
            const uint32_t* k = kpoints + 3 * q;
            REQUIRE(k[0] < mesh[0] && k[1] < mesh[1] && k[2] < mesh[2], "k-point outside the mesh");
            kidx[q] = (uint32_t)(((size_t)k[0] * mesh[1] + k[1]) * mesh[2] + k[2]);
        }
        std::vector<double> u(3 * (size_t)h->nsub, 1.0);
        if (uo) u.assign(uo, uo + 3 * (size_t)h->nsub);
        S.idx = dupload(idx.data(), idx.size());
        S.sub = dupload(sub.data(), sub.size());
        S.uo = dupload(u.data(), u.size());
        S.kidx = dupload(kidx.data(), kidx.size());
        S.grid = dalloc<double2>(P);
        S.series = dalloc<double2>((size_t)max_samples * nk);
        int dims[3] = {(int)mesh[0], (int)mesh[1], (int)mesh[2]};
        CKFFT(cufftPlanMany(&S.plan, 3, dims, nullptr, 1, (int)P, nullptr, 1, (int)P, CUFFT_Z2Z, 1));
        CKFFT(cufftSetStream(S.plan, h->stream));
        S.qaxis = qaxis; S.nk = nk; S.max_samples = max_samples; S.P = P; S.on = true;
    } catch (const Fail& f) { return fail(h, f); }
    return ASD_OK;
}

int asd_sq_sample(asd_handle* h) {
    if (!h) return ASD_EINVAL;
    try {
        if (!h->sq.on) throw Fail{ASD_ESTATE, "asd_sq_setup has not been called"};
        if (h->sq.nsamples >= h->sq.max_samples) throw Fail{ASD_ESTATE, "S(q,t) series is full"};
        CK(cudaSetDevice(h->device));
        CK(launch_sq_sample(h));
    } catch (const Fail& f) { return fail(h, f); }
    return ASD_OK;
}

int asd_sq_get(asd_handle* h, double* out, size_t out_len, uint32_t* nsamples) {
    if (!h) return ASD_EINVAL;
    try {
        if (!h->sq.on) throw Fail{ASD_ESTATE, "asd_sq_setup has not been called"};
        const size_t m = (size_t)h->sq.nsamples * h->sq.nk * 2;
        REQUIRE(out && out_len >= m, "output must hold nsamples*nk*2 doubles");
        CK(cudaSetDevice(h->device));
        CK(cudaMemcpyAsync(out, h->sq.series, m * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
        CK(cudaStreamSynchronize(h->stream));
        if (nsamples) *nsamples = h->sq.nsamples;
    } catch (const Fail& f) { return fail(h, f); }
    return ASD_OK;
}

int asd_sq_spectrum(asd_handle* h, uint32_t window, double alpha, double beta, double width_hz, double sample_dt,
                    double fcut_lo, double fcut_hi, double* raw, double* smooth, size_t len, uint32_t* peak_raw,
                    uint32_t* peak_smooth) {
    if (!h) return ASD_EINVAL;
    double* d = nullptr;
    uint32_t* dp = nullptr;
    try {
        if (!h->sq.on) throw Fail{ASD_ESTATE, "asd_sq_setup has not been called"};
        const uint32_t ns = h->sq.nsamples, nk = h->sq.nk, half = ns / 2;
        REQUIRE(ns >= 2, "the spectrum needs at least 2 samples");
        REQUIRE(window <= 1, "window must be 0 (none) or 1 (generalised Hamming)");
        REQUIRE(sample_dt > 0.0 && std::isfinite(sample_dt) && std::isfinite(width_hz), "sample_dt, width_hz");
        const double pw = width_hz * (double)ns * sample_dt + 0.5;
        REQUIRE(pw >= 1.0 && pw < 4294967296.0, "the Gaussian width rounds to less than one bin");
        const size_t m = (size_t)nk * half;
        REQUIRE(!(raw || smooth) || len >= m, "raw/smooth must hold nk*(nsamples/2) doubles");
        CK(cudaSetDevice(h->device));
        d = dalloc<double>(2 * m);
        dp = dalloc<uint32_t>(2 * (size_t)nk);
        CK(launch_sq_spectrum(h, (int)window, alpha, beta, (uint32_t)pw, sample_dt, fcut_lo, fcut_hi, d, d + m, dp));
        if (raw) CK(cudaMemcpy(raw, d, m * sizeof(double), cudaMemcpyDeviceToHost));
        if (smooth) CK(cudaMemcpy(smooth, d + m, m * sizeof(double), cudaMemcpyDeviceToHost));
        if (peak_raw) CK(cudaMemcpy(peak_raw, dp, nk * sizeof(uint32_t), cudaMemcpyDeviceToHost));
        if (peak_smooth) CK(cudaMemcpy(peak_smooth, dp + nk, nk * sizeof(uint32_t), cudaMemcpyDeviceToHost));
    } catch (const Fail& f) {
        if (d) cudaFree(d);
        if (dp) cudaFree(dp);
        return fail(h, f);
    }
    cudaFree(d);
    cudaFree(dp);
    return ASD_OK;
}

int asd_reset_magnetisation_stats(asd_handle* h) {
    if (!h) return ASD_EINVAL;
    try {
        CK(cudaSetDevice(h->device));
        CK(cudaMemsetAsync(h->d_stats, 0, (size_t)h->nrep * h->nsub * 4 * sizeof(double), h->stream));
        CK(cudaStreamSynchronize(h->stream));
    } catch (const Fail& f) { return fail(h, f); }
    return ASD_OK;
}

int asd_magnetisation(asd_handle* h, double* out, size_t out_len) {
    if (!h) return ASD_EINVAL;
    try {
        REQUIRE(out && out_len >= (size_t)h->nrep * h->nsub * 3, "output must hold nrep*nsub*3 doubles");
        CK(cudaSetDevice(h->device));
        // a page-locked caller buffer this device can address takes the means straight from the
        // kernel; any other buffer gets them by a copy
        double* hout = nullptr;
        cudaPointerAttributes pa{};
        if (cudaPointerGetAttributes(&pa, out) == cudaSuccess) {
            if (pa.type == cudaMemoryTypeHost && pa.devicePointer) hout = static_cast<double*>(pa.devicePointer);
        } else {
            (void)cudaGetLastError();
        }
        CK(launch_magnetisation(h, hout));
        if (!hout)
            CK(cudaMemcpyAsync(out, h->d_mag, (size_t)h->nrep * h->nsub * 3 * 8, cudaMemcpyDeviceToHost, h->stream));
        CK(cudaStreamSynchronize(h->stream));
    } catch (const Fail& f) { return fail(h, f); }
    return ASD_OK;
}

int asd_num_sublattices(const asd_handle* h, uint32_t* nsub) {
    if (!h || !nsub) return ASD_EINVAL;
    *nsub = h->nsub;
    return ASD_OK;
}

int asd_time_steps(asd_handle* h, uint64_t nsteps, double* ms, uint64_t* launches) {
    if (!h || !ms) return ASD_EINVAL;
    try {
        CK(cudaSetDevice(h->device));
        CK(cudaStreamSynchronize(h->stream));
        const uint64_t l0 = h->launches;
        CK(cudaEventRecord(h->kev[0], h->stream));
        run_steps(h, nsteps);
        CK(cudaEventRecord(h->kev[1], h->stream));
        CK(cudaEventSynchronize(h->kev[1]));
        float f = 0.f;
        CK(cudaEventElapsedTime(&f, h->kev[0], h->kev[1]));
        *ms = f;
        if (launches) *launches = h->launches - l0;
    } catch (const Fail& f) { return fail(h, f); }
    return ASD_OK;
}

int asd_time_kernels(asd_handle* h, uint64_t nsteps) { return asd_time_kernels_cold(h, nsteps, 0); }

int asd_time_kernels_cold(asd_handle* h, uint64_t nsteps, uint64_t flush_bytes) {
    if (!h) return ASD_EINVAL;
    try {
        CK(cudaSetDevice(h->device));
        CK(cudaStreamSynchronize(h->stream));
        h->ktab.clear();
        if (flush_bytes) {
            CK(cudaMalloc(&h->flush_buf, flush_bytes));
            h->flush_bytes = flush_bytes;
        }
        h->timing = true;
        const uint32_t G = h->graph_steps;
        h->graph_steps = 0;  // direct launches so each stage kernel is bracketed by events
        auto restore = [&]() {
            h->timing = false;
            h->graph_steps = G;
            cudaStreamSynchronize(h->stream);
            if (h->flush_buf) cudaFree(h->flush_buf);
            h->flush_buf = nullptr;
            h->flush_bytes = 0;
        };
        try { run_steps(h, nsteps); } catch (...) { restore(); throw; }
        restore();
        CK(cudaGetLastError());
    } catch (const Fail& f) { return fail(h, f); }
    return ASD_OK;
}

int asd_time_steps_cold(asd_handle* h, uint64_t nsteps, uint64_t flush_bytes, double* ms, uint64_t* launches) {
    if (!h || !ms || flush_bytes == 0) return ASD_EINVAL;
    void* buf = nullptr;
    std::vector<cudaEvent_t> ev;
    try {
        CK(cudaSetDevice(h->device));
        CK(cudaStreamSynchronize(h->stream));
        CK(cudaMalloc(&buf, flush_bytes));
        ev.assign(2 * nsteps, nullptr);
        for (auto& e : ev) CK(cudaEventCreate(&e));
        const uint64_t l0 = h->launches;
        for (uint64_t q = 0; q < nsteps; q++) {
            // the flush is enqueued first and runs longer than the host takes to enqueue the
            // step, so the events bracket device time of the step alone
            CK(cudaMemsetAsync(buf, (int)(q & 0xFF), flush_bytes, h->stream));
            CK(cudaEventRecord(ev[2 * q], h->stream));
            run_steps(h, 1);
            CK(cudaEventRecord(ev[2 * q + 1], h->stream));
        }
        CK(cudaStreamSynchronize(h->stream));
        double tot = 0.0;
        for (uint64_t q = 0; q < nsteps; q++) {
            float f = 0.f;
            CK(cudaEventElapsedTime(&f, ev[2 * q], ev[2 * q + 1]));
            tot += f;
        }
        *ms = tot;
        if (launches) *launches = h->launches - l0;
    } catch (const Fail& f) {
        for (auto e : ev) if (e) cudaEventDestroy(e);
        if (buf) cudaFree(buf);
        return fail(h, f);
    }
    for (auto e : ev) cudaEventDestroy(e);
    cudaFree(buf);
    return ASD_OK;
}

// The dominant kernel of the last asd_time_kernels: the largest device time summed over its
// launches.
int asd_kernel_stats(const asd_handle* h, char* name, size_t name_len, double* avg_ms, uint64_t* count,
                     double* bytes_per_launch) {
    if (!h) return ASD_EINVAL;
    const KernelTimer* kt = nullptr;
    for (const auto& k : h->ktab)
        if (!kt || k.total_ms > kt->total_ms) kt = &k;
    const KernelTimer none{};
    if (!kt) kt = &none;
    if (name && name_len) snprintf(name, name_len, "%s", kt->name.c_str());
    if (avg_ms) *avg_ms = kt->count ? kt->total_ms / kt->count : 0.0;
    if (count) *count = kt->count;
    if (bytes_per_launch) *bytes_per_launch = kt->bytes;
    return ASD_OK;
}

int asd_kernel_table(const asd_handle* h, char* out, size_t out_len) {
    if (!h || !out || out_len == 0) return ASD_EINVAL;
    std::string t;
    char line[512];
    for (const auto& k : h->ktab) {
        snprintf(line, sizeof line, "%s|%.6f|%llu|%.0f\n", k.name.c_str(), k.count ? k.total_ms / k.count : 0.0,
                 (unsigned long long)k.count, k.bytes);
        t += line;
    }
    if (t.size() + 1 > out_len) return ASD_EINVAL;
    snprintf(out, out_len, "%s", t.c_str());
    return ASD_OK;
}

int asd_thermal_normals(uint64_t seed, uint32_t stream, uint64_t step, uint32_t nspins, double* out) {
    if (!out || nspins == 0) return ASD_EINVAL;
    double* d = nullptr;
    if (cudaMalloc(&d, 3 * (size_t)nspins * sizeof(double)) != cudaSuccess) return ASD_ENOMEM;
    cudaError_t e = launch_thermal_normals(seed, stream, step, nspins, d, 0);
    if (e == cudaSuccess) e = cudaMemcpy(out, d, 3 * (size_t)nspins * sizeof(double), cudaMemcpyDeviceToHost);
    cudaFree(d);
    return e == cudaSuccess ? ASD_OK : ASD_ECUDA;
}

int asd_thermal_normals_f32(uint64_t seed, uint32_t stream, uint64_t step, uint32_t nspins, float* out) {
    if (!out || nspins == 0) return ASD_EINVAL;
    float* d = nullptr;
    if (cudaMalloc(&d, 3 * (size_t)nspins * sizeof(float)) != cudaSuccess) return ASD_ENOMEM;
    cudaError_t e = launch_thermal_normals_f(seed, stream, step, nspins, d, 0);
    if (e == cudaSuccess) e = cudaMemcpy(out, d, 3 * (size_t)nspins * sizeof(float), cudaMemcpyDeviceToHost);
    cudaFree(d);
    return e == cudaSuccess ? ASD_OK : ASD_ECUDA;
}

}  // extern "C"
