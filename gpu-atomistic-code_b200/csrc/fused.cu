// Fused stage kernels: one bandwidth-bound pass per integrator stage that
// gathers the exchange field (SELL-32 or DIA layout, streamed or typed), adds
// the long-range, site, thermal (in-kernel Philox), applied and anisotropy
// fields, forms the LLG torque and writes the next stage spin renormalised in
// FP64.  The same templates serve the FP32 form (R=float) and the fused FP64
// form (R=double).
//
// Reference computation per stage: the field kernel CSpMV_* / CCopyFields
// (src/cufields.cu:97-246, 386-407) followed by CHeun1/CHeun2
// (src/cuint.cu:60-242) or CdetRK4k*/CdetRK5k* + CdetSnp1
// (src/cuintRK4.cu:62-457, src/cuintRK5.cu:79-651).
#include "gather.cuh"

namespace asd {
namespace {

struct LrArgs {
    const float* hr;            // padded real field [3][P] to gather (nullptr: none)
    float inv_p;
    float* mr;                  // padded real input [3][P] to scatter the output spins into (nullptr: none)
    const float* w;             // per-spin weight for the scatter
    const uint32_t* idx;        // per-spin mesh index
    size_t P;
};

template <typename R>
struct StageArgs {
    CVec3<R> src;        // spins the field is gathered from (S or a stage spin)
    CVec3<R> base;       // S (hi part)
    CVec3<float> base_lo;// S lo part (compensated storage) or nullptrs
    Vec3<R> out;         // next stage spin or new S (hi)
    Vec3<float> out_lo;  // new S lo part
    Vec3<R> fn;          // Heun f_n (stage 1 writes, stage 2 reads)
    Vec3<R> det;         // det field (stage 2, at the det step)
    CVec3<R> stag;       // site-field profile or nullptrs
    Vec3<R> k[6];        // RK stage increments
    Vec3<R> nz;          // sigma sqrt(T) xi of this step: the first stage writes it, later stages read it
    const void* pf[24];  // per-spin arrays this stage reads at its own rows: prefetched into L2
    uint32_t npf;        // at the start of each block
    int nz_mode;         // 0: draw only, 1: draw and store in nz, 2: load from nz
    int kind;            // 1: Heun predictor, 2: Heun corrector, 10+st: RK stage st
    int nst;             // RK stages
    uint32_t rel;        // step offset inside a graph chunk
    LrArgs lr;
};

// Anisotropy field (src/cuint.cu:76-137): per-atom K1u plus global K2 / K4 terms, with the
// constants taken in the kernel's own precision from the parameter block.
template <typename R>
struct AnisConst {
    R k1u, d[3], k2perp, k2perpdir[3], k2par, k2pardir[3], k4perp, k4perpdirs[9], k4par, k4pardirs[9];
};

template <typename R>
__device__ __forceinline__ void anis_field(const StepConst& c, const MatConst& mc, const R s[3], R h[3]) {
    const R *d, *k2pd, *k2ad, *k4pd, *k4ad;
    R k1u, k2perp, k2par, k4perp, k4par;
    if constexpr (sizeof(R) == 4) {
        d = mc.k1udir_f; k1u = mc.k1u_f;
        k2pd = c.k2perpdir_f; k2ad = c.k2pardir_f; k4pd = c.k4perpdirs_f; k4ad = c.k4pardirs_f;
        k2perp = c.k2perp_ff; k2par = c.k2par_ff; k4perp = c.k4perp_ff; k4par = c.k4par_ff;
    } else {
        d = mc.k1udir; k1u = mc.k1u;
        k2pd = c.k2perpdir; k2ad = c.k2pardir; k4pd = c.k4perpdirs; k4ad = c.k4pardirs;
        k2perp = c.k2perp_f; k2par = c.k2par_f; k4perp = c.k4perp_f; k4par = c.k4par_f;
    }
    const R k1 = k1u * (s[0] * d[0] + s[1] * d[1] + s[2] * d[2]);
    h[0] += k1 * d[0]; h[1] += k1 * d[1]; h[2] += k1 * d[2];
    if (k2perp != R(0)) {
        const R t = k2perp * (s[0] * k2pd[0] + s[1] * k2pd[1] + s[2] * k2pd[2]);
        h[0] += t * k2pd[0]; h[1] += t * k2pd[1]; h[2] += t * k2pd[2];
    }
    if (k2par != R(0)) {
        const R t = k2par * (s[0] * k2ad[0] + s[1] * k2ad[1] + s[2] * k2ad[2]);
        h[0] += t * k2ad[0]; h[1] += t * k2ad[1]; h[2] += t * k2ad[2];
    }
    if (k4perp != R(0) || k4par != R(0)) {
#pragma unroll
        for (int dir = 0; dir < 3; dir++) {
            const R* p = k4pd + 3 * dir;
            const R* q = k4ad + 3 * dir;
            const R tp = k4perp * (s[0] * p[0] + s[1] * p[1] + s[2] * p[2]);
            const R tq = k4par * (s[0] * q[0] + s[1] * q[1] + s[2] * q[2]);
            h[0] += tp * p[0] + tq * q[0]; h[1] += tp * p[1] + tq * q[1]; h[2] += tp * p[2] + tq * q[2];
        }
    }
}

template <typename R>
__device__ __forceinline__ void llg_rhs(R llgpf, R lambda, const R s[3], const R h[3], R f[3]) {
    const R a0 = s[1] * h[2] - s[2] * h[1], a1 = s[2] * h[0] - s[0] * h[2], a2 = s[0] * h[1] - s[1] * h[0];
    const R b0 = s[1] * a2 - s[2] * a1, b1 = s[2] * a0 - s[0] * a2, b2 = s[0] * a1 - s[1] * a0;
    f[0] = llgpf * (a0 + lambda * b0);
    f[1] = llgpf * (a1 + lambda * b1);
    f[2] = llgpf * (a2 + lambda * b2);
}

__device__ __forceinline__ void renorm(double v[3]) {
    const double inv = rsqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    v[0] *= inv; v[1] *= inv; v[2] *= inv;
}

__constant__ double FRK5B[5][5] = {
    {0.2, 0, 0, 0, 0},
    {3.0 / 40.0, 9.0 / 40.0, 0, 0, 0},
    {0.3, -0.9, 1.2, 0, 0},
    {-11.0 / 54, 2.5, -70.0 / 27.0, 35.0 / 27.0, 0},
    {1631.0 / 55296.0, 175.0 / 512.0, 575.0 / 13824.0, 44275.0 / 110592.0, 253.0 / 4096.0}};
__constant__ double FRK5C[6] = {37.0 / 378.0, 0.0, 250.0 / 621.0, 125.0 / 594.0, 0.0, 512.0 / 1771.0};
__constant__ double FRK4C[4] = {1.0 / 6.0, 1.0 / 3.0, 1.0 / 3.0, 1.0 / 6.0};

// Register caps of the FP32 kernels: 6 blocks of 256 per SM (40 registers) for the SELL and
// the field-only kernels, 5 (48) for the DIA kernels; the FP64 kernels keep the default cap.
// At 40 the diagonal-tensor SELL kernels spill 76 bytes a thread (the others none), and still
// run faster than at 48: the extra warps hide more of the gather's latency than the spills add
// (96 replicas 564 → 534 µs per step, the north star unchanged, A/B on one box).
template <typename R, int EX, bool FULL, int K>
struct MinBlocks {
    static constexpr int value =
        sizeof(R) != 4 ? 1 : (EX == ASD_EXCH_CSR || EX == ASD_EXCH_NONE) ? 6 : 5;
};

// K: the stage kind at compile time (1 Heun predictor, 2 Heun corrector, 3 RK stage before the
// last, 4 last RK stage); a.kind still carries the RK stage index.
template <typename R, int EX, bool FULL, bool COMP, int K>
__global__ void __launch_bounds__(256, MinBlocks<R, EX, FULL, K>::value)
    stage_kernel(const StepConst c, const SellDev sell, const DiaDev dia, const StageArgs<R> a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ __align__(8) uint64_t stage_bar;
    R* tab = reinterpret_cast<R*>(smem_raw);
    // Until pdl_enter below the block touches only set-up data (the exchange words, the tensor
    // table, the spans, the mesh index): the copies of the words and the table start while the
    // previous kernel's last blocks run; the neighbour-spin spans are copied after the wait.
    const uint32_t* staged = nullptr;
    const uint16_t* staged16 = nullptr;
    const R* sspin = nullptr;
    R* span_dst = nullptr;           // shared-memory spin buffer the span copies fill after the wait
    uint32_t span0 = 0, nspan = 0;
    uint32_t wbase = 0;
    if constexpr (EX == ASD_EXCH_CSR) {
        if (sell.typed) {
            // the tensor table: with staging, one more bulk copy on the staging barrier; else a
            // block-wide load
            bool tab_staged = false;
            const uint32_t tab_bytes = (uint32_t)sizeof(R) * table_stride<FULL>() * sell.ntypes;
            if (sell.stage) {
                // this block's slices are contiguous in the SELL stream: one bulk copy into
                // shared memory behind the tensor table; with stage 2 also one copy per
                // (neighbour-spin span, component); all overlap the noise draw below
                const uint32_t tb = (tab_bytes + 15u) & ~15u;
                const uint32_t spb = blockDim.x >> 5;
                const uint32_t s0 = blockIdx.x * spb, s1 = min(s0 + spb, sell.nslices);
                wbase = __ldg(sell.slice_ptr + s0);
                const uint32_t bytes = (__ldg(sell.slice_ptr + s1) - wbase) * 4u;
                uint32_t sp0 = 0, nsp = 0;
                if (sell.stage == 2) {
                    sp0 = __ldg(sell.span_ptr + blockIdx.x);
                    nsp = __ldg(sell.span_ptr + blockIdx.x + 1) - sp0;
                }
                const bool w16 = sell.stage == 2 && sell.lwords16;
                if (w16 && bytes && nsp) {
                    // 16-bit local words (half the copy and the buffer) and the spans; a block
                    // without spans stages nothing and reads its global words
                    const uint32_t bytes16 = bytes >> 1;
                    uint16_t* wbuf = reinterpret_cast<uint16_t*>(smem_raw + tb);
                    R* sbuf = reinterpret_cast<R*>(smem_raw + tb + ((2u * sell.stage_words + 15u) & ~15u));
                    if (threadIdx.x == 0) mbar_init(&stage_bar, 1);
                    __syncthreads();
                    if (threadIdx.x < 32) {
                        if (threadIdx.x == 0) {
                            uint32_t tx = bytes16 + tab_bytes;
                            for (uint32_t q = 0; q < nsp; q++) tx += 3u * sell.spans[sp0 + q].y * (uint32_t)sizeof(R);
                            mbar_arrive_expect_tx(&stage_bar, tx);
                        }
                        __syncwarp();
                        if (threadIdx.x == 0) bulk_copy_stream(wbuf, sell.lwords16 + wbase, bytes16, &stage_bar);
                        if (threadIdx.x == 1) bulk_copy(tab, table_of<R>(sell), tab_bytes, &stage_bar);
                    }
                    staged16 = wbuf;
                    sspin = sbuf;
                    span_dst = sbuf; span0 = sp0; nspan = nsp;
                    tab_staged = true;
                } else if (!w16 && bytes) {
                    uint32_t* wbuf = reinterpret_cast<uint32_t*>(smem_raw + tb);
                    R* sbuf = reinterpret_cast<R*>(smem_raw + tb + 4u * sell.stage_words);
                    if (threadIdx.x == 0) mbar_init(&stage_bar, 1);
                    __syncthreads();
                    if (threadIdx.x < 32) {
                        if (threadIdx.x == 0) {
                            uint32_t tx = bytes + tab_bytes;
                            for (uint32_t q = 0; q < nsp; q++) tx += 3u * sell.spans[sp0 + q].y * (uint32_t)sizeof(R);
                            mbar_arrive_expect_tx(&stage_bar, tx);
                        }
                        __syncwarp();
                        if (threadIdx.x == 0)
                            bulk_copy_stream(wbuf, (nsp ? sell.lwords : sell.typed) + wbase, bytes, &stage_bar);
                        if (threadIdx.x == 1) bulk_copy(tab, table_of<R>(sell), tab_bytes, &stage_bar);
                    }
                    staged = wbuf;
                    if (nsp) { sspin = sbuf; span_dst = sbuf; span0 = sp0; nspan = nsp; }
                    tab_staged = true;
                }
            }
            if (!tab_staged) load_table<R>(table_of<R>(sell), table_stride<FULL>() * sell.ntypes, tab);
        }
    }
    if constexpr (EX == ASD_EXCH_DIA) {
        if (dia.dtype) load_table<R>(table_of<R>(dia), table_stride<FULL>() *dia.ntypes, tab);
    }
    pdl_enter();
    if constexpr (EX == ASD_EXCH_CSR) {
        // the neighbour-spin spans: one copy per (span, component), on the staging barrier
        if (threadIdx.x < 32)
            for (uint32_t k = threadIdx.x; k < 3 * nspan; k += 32) {
                const uint4 sp = sell.spans[span0 + k / 3];
                const uint32_t cc = k % 3;
                bulk_copy(span_dst + cc * sell.spin_slots + sp.z, a.src.p[cc] + sp.x, sp.y * (uint32_t)sizeof(R),
                          &stage_bar);
            }
    }
    if (threadIdx.x == 0 && a.npf) {
        // the block's rows of every per-spin input: one bulk L2 prefetch each, so the loads
        // after the exchange gather find them in L2; sizes stop at the last row (whole
        // 16-byte units), so no prefetch reaches past an array
        const uint32_t r0 = blockIdx.x * blockDim.x;
        const uint32_t rows = min(blockDim.x, c.n - r0);
        const uint32_t bytes = (rows * (uint32_t)sizeof(R)) & ~15u;
        if (bytes)
            for (uint32_t q = 0; q < a.npf; q++)
                bulk_prefetch_l2(static_cast<const char*>(a.pf[q]) + (size_t)r0 * sizeof(R), bytes);
    }
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= c.n) return;     // thread 0 of every block has i < n and always waits below
    const uint64_t t = *c.step_base + a.rel;
    const uint32_t at = atom_of(c, i);
    const MatConst& mc = c.mat[at];
    const uint32_t r = replica_of(c, i);
    constexpr bool F32 = sizeof(R) == 4;
    // one thermal draw per spin and step serves every stage (src/cuint.cu:72): the first stage
    // draws it, later stages of the step load what the first stored
    R lrn[3] = {R(0), R(0), R(0)};
    bool hot;
    if constexpr (F32) hot = __ldg(c.rep_sqrtT_f + r) > 0.0f; else hot = __ldg(c.rep_sqrtT + r) > 0.0;
    if (hot && a.nz_mode == 2) {
        lrn[0] = a.nz.p[0][i]; lrn[1] = a.nz.p[1][i]; lrn[2] = a.nz.p[2][i];
    } else if (hot) {
        if constexpr (F32) {
            float xi[3];
            thermal_normals_f(c.seed, __ldg(c.rep_stream + r), i - __ldg(c.rep_off + r), t, xi);
            const float tp = __ldg(c.rep_sqrtT_f + r) * mc.sigma_f;
            lrn[0] = xi[0] * tp; lrn[1] = xi[1] * tp; lrn[2] = xi[2] * tp;
        } else {
            double xi[3];
            thermal_normals(c.seed, __ldg(c.rep_stream + r), i - __ldg(c.rep_off + r), t, xi);
            const double tp = __ldg(c.rep_sqrtT + r) * mc.sigma;
            lrn[0] = xi[0] * tp; lrn[1] = xi[1] * tp; lrn[2] = xi[2] * tp;
        }
        if (a.nz_mode == 1) { a.nz.p[0][i] = lrn[0]; a.nz.p[1][i] = lrn[1]; a.nz.p[2][i] = lrn[2]; }
    }
    // the long-range field at this site: with diagonal tensors it is loaded before the staging
    // wait, so that its two dependent loads (mesh index, field) overlap the copies and the
    // gather; the full-tensor kernels have no registers to spare and load it after the gather
    uint32_t midx = 0;
    float hl[3] = {0.f, 0.f, 0.f};
    auto load_lr = [&]() {
        if (a.lr.hr || a.lr.mr) midx = __ldg(a.lr.idx + i);
        if (a.lr.hr) {
            hl[0] = __ldg(a.lr.hr + midx);
            hl[1] = __ldg(a.lr.hr + a.lr.P + midx);
            hl[2] = __ldg(a.lr.hr + 2 * a.lr.P + midx);
        }
    };
    if constexpr (!FULL) load_lr();
    bool stage_timeout = false;
    const uint32_t polls = (c.flags & ASD_FLAG_WAIT_TIMEOUT) ? 0u : STAGE_WAIT_POLLS;
    if ((staged || staged16) && !mbar_wait_bounded(&stage_bar, polls)) {
        // the copy did not land in time: record it and read the words and the table from
        // global memory
        atomicOr(sell.err, ERR_STAGE_TIMEOUT);
        staged = nullptr;      // the global words carry global columns
        staged16 = nullptr;
        sspin = nullptr;
        tab = const_cast<R*>(table_of<R>(sell));
        stage_timeout = true;
    }
    R h[3] = {R(0), R(0), R(0)};
    if constexpr (EX == ASD_EXCH_CSR) gather_sell<R, FULL>(sell, i, a.src, tab, h, staged, wbase, sspin, staged16);
    if constexpr (EX == ASD_EXCH_DIA) gather_dia<R, FULL>(dia, c.n, i, a.src, tab, h);
    if (c.q4_ptr) {
        R h4[3];
        four_spin<R>(c, i, [&](uint32_t j, R v[3]) { v[0] = a.src.p[0][j]; v[1] = a.src.p[1][j]; v[2] = a.src.p[2][j]; }, h4);
        h[0] += h4[0]; h[1] += h4[1]; h[2] += h4[2];
    }
    if constexpr (FULL) load_lr();
    if (a.lr.hr) {
        h[0] += (R)(hl[0] * a.lr.inv_p);
        h[1] += (R)(hl[1] * a.lr.inv_p);
        h[2] += (R)(hl[2] * a.lr.inv_p);
    }
    const double* dyn = c.dyn;
    const R* dynr;
    if constexpr (F32) dynr = c.dynf; else dynr = c.dyn;
    if (a.stag.p[0]) {
        R sc;
        if constexpr (F32) sc = site_scale_f(c.dynf, dyn, t, c.dt); else sc = site_scale_d(dyn, t, c.dt);
        h[0] += sc * a.stag.p[0][i]; h[1] += sc * a.stag.p[1][i]; h[2] += sc * a.stag.p[2][i];
    }
    h[0] += lrn[0] + dynr[DYN_APPLIED];
    h[1] += lrn[1] + dynr[DYN_APPLIED + 1];
    h[2] += lrn[2] + dynr[DYN_APPLIED + 2];

    // stage spin at this site
    R sv[3] = {a.src.p[0][i], a.src.p[1][i], a.src.p[2][i]};
    const int kind = a.kind;
    if constexpr (K >= 3) {
        if (kind >= 11 && (c.flags & ASD_FLAG_RK_STAGE_SPIN_MIXED)) sv[1] = a.base.p[1][i];
    }
    anis_field<R>(c, mc, sv, h);
    R f[3];
    if constexpr (F32) llg_rhs<R>(mc.llgpf_f, mc.lambda_f, sv, h, f);
    else llg_rhs<R>(mc.llgpf, mc.lambda, sv, h, f);

    constexpr bool final_spin = K == 2 || K == 4;
    R out[3];
    if constexpr (!final_spin && F32) {
        // FP32 form: intermediate stage spins (Heun S', RK stage vectors) only feed field
        // evaluations, so they are formed and renormalised in single precision
        const float rdt = c.rdt_f;
        float o[3];
        const float S[3] = {(float)a.base.p[0][i], (float)a.base.p[1][i], (float)a.base.p[2][i]};
        if constexpr (K == 1) {
            for (int j = 0; j < 3; j++) { a.fn.p[j][i] = f[j]; o[j] = fmaf(rdt, (float)f[j], S[j]); }
        } else {
            const int st = kind - 10, nst = a.nst;
            const bool dbl = (c.flags & ASD_FLAG_RK_DOUBLE_RDT) != 0;
            for (int j = 0; j < 3; j++) {
                const float k = rdt * (float)f[j];
                a.k[st].p[j][i] = (R)k;
                float inc;
                if (nst == 4) {
                    inc = k * (st == 2 ? 1.0f : 0.5f);
                } else {
                    inc = (float)FRK5B[st][st] * k;
                    for (int b = 0; b < st; b++) inc = fmaf((float)FRK5B[st][b], (float)a.k[b].p[j][i], inc);
                }
                o[j] = S[j] + (dbl ? rdt * inc : inc);
            }
        }
        const float inv = rsqrtf(o[0] * o[0] + o[1] * o[1] + o[2] * o[2]);
        for (int j = 0; j < 3; j++) out[j] = (R)(o[j] * inv);
        for (int j = 0; j < 3; j++) a.out.p[j][i] = out[j];
    } else {
        // new S (and every stage of the FP64 fused form): FP64 accumulation from the
        // full-precision base, FP64 renormalisation
        double S[3] = {(double)a.base.p[0][i], (double)a.base.p[1][i], (double)a.base.p[2][i]};
        if constexpr (COMP && final_spin) {
            S[0] += (double)a.base_lo.p[0][i]; S[1] += (double)a.base_lo.p[1][i]; S[2] += (double)a.base_lo.p[2][i];
        }
        const double rdt = c.rdt;
        double o[3];
        if constexpr (K == 1) {
            for (int j = 0; j < 3; j++) { a.fn.p[j][i] = f[j]; o[j] = S[j] + rdt * (double)f[j]; }
        } else if constexpr (K == 2) {
            for (int j = 0; j < 3; j++) o[j] = S[j] + 0.5 * rdt * (double)(a.fn.p[j][i] + f[j]);
            if ((double)t == dyn[DYN_DET_STEP])
                for (int j = 0; j < 3; j++) a.det.p[j][i] = h[j] - lrn[j];
        } else {
            const int st = kind - 10, nst = a.nst;
            const bool dbl = (c.flags & ASD_FLAG_RK_DOUBLE_RDT) != 0;
            double k[3];
            for (int j = 0; j < 3; j++) k[j] = rdt * (double)f[j];
            if constexpr (K == 3) {
                for (int j = 0; j < 3; j++) a.k[st].p[j][i] = (R)k[j];
                for (int j = 0; j < 3; j++) {
                    double inc;
                    if (nst == 4) {
                        inc = k[j] * (st == 2 ? 1.0 : 0.5);
                    } else {
                        inc = FRK5B[st][st] * k[j];
                        for (int b = 0; b < st; b++) inc += FRK5B[st][b] * (double)a.k[b].p[j][i];
                    }
                    o[j] = S[j] + (dbl ? rdt * inc : inc);
                }
            } else {
                const double* C = nst == 4 ? FRK4C : FRK5C;
                for (int j = 0; j < 3; j++) {
                    double acc = C[st] * k[j];
                    for (int b = 0; b < st; b++) acc += C[b] * (double)a.k[b].p[j][i];
                    o[j] = S[j] + acc;
                }
            }
        }
        renorm(o);
        for (int j = 0; j < 3; j++) {
            const R hi = (R)o[j];
            out[j] = hi;
            a.out.p[j][i] = hi;
            if constexpr (COMP && final_spin) a.out_lo.p[j][i] = (float)(o[j] - (double)hi);
        }
    }
    if (a.lr.mr) {
        const float wv = __ldg(a.lr.w + i);
        a.lr.mr[midx] = (float)out[0] * wv;
        a.lr.mr[a.lr.P + midx] = (float)out[1] * wv;
        a.lr.mr[2 * a.lr.P + midx] = (float)out[2] * wv;
    }
    // a block must not retire while its bulk copy may still be writing shared memory
    if (stage_timeout) mbar_wait_bounded(&stage_bar, STAGE_WAIT_POLLS);
}

__global__ void advance_k(uint64_t* step, uint32_t n) {
    pdl_enter();
    *step += n;
}
// The det field is written at the step the device counter holds (the one-step graph's step).
// The applied field rides in the parameters of this first node of the one-step graph: a new
// value updates the node in place, so a single-step call needs no launch of its own for it.
struct AppliedArg { double v[3]; };
__global__ void det_here_k(const uint64_t* step, double* dyn, float* dynf, AppliedArg applied) {
    pdl_enter();
    dyn[DYN_DET_STEP] = (double)*step;
    for (int k = 0; k < 3; k++) {
        dyn[DYN_APPLIED + k] = applied.v[k];
        dynf[DYN_APPLIED + k] = (float)applied.v[k];
    }
}

template <typename R>
Vec3<R> v3(R* const p[3]) { return Vec3<R>{{p[0], p[1], p[2]}}; }
template <typename R>
CVec3<R> c3(R* const p[3]) { return CVec3<R>{{p[0], p[1], p[2]}}; }

// Bytes one stage launch must move (algorithmic: each array element once,
// gathered neighbour spins counted once, the matrix at its nnz in the layout used).
template <typename R>
double stage_bytes(const asd_handle* h, const StageArgs<R>& a, bool comp) {
    const double vb = sizeof(R), n = h->n;
    const double c = h->full ? 9.0 : 3.0;
    double m = 0.0;
    if (h->dexch == ASD_EXCH_CSR) m = 4.0 + h->nnz_per_row * (h->sell.typed ? 4.0 : 4.0 + vb * c);
    else if (h->dexch == ASD_EXCH_DIA) m = h->nnz_per_row * (h->dia.dtype ? 1.0 : vb * c);
    double st = 3 * vb;                                  // src spin (gathered once)
    const int kind = a.kind;
    const bool final_spin = kind == 2 || (kind >= 10 && kind - 10 == a.nst - 1);
    if (kind != 1 && kind != 10) st += 3 * vb;           // base S differs from src
    st += 3 * vb;                                        // output spin
    if (kind == 1) st += 3 * vb;                         // f_n written
    if (kind == 2) st += 3 * vb;                         // f_n read
    if (kind >= 10) {
        const int s = kind - 10;
        if (s < a.nst - 1) st += 3 * vb;                 // k_s written
        const int reads = a.nst == 4 ? (s == a.nst - 1 ? s : 0) : s;
        st += reads * 3 * vb;                            // earlier k read
    }
    if (comp && final_spin) st += 24;                    // lo part read + written
    if (a.stag.p[0]) st += 3 * vb;
    if (a.lr.hr) st += 12;
    if (a.lr.mr) st += 12;
    double hot = 0.0;                                    // spins with T > 0: the step's draw is
    for (uint32_t r = 0; r < h->nrep; r++)               // stored by the first stage, loaded by the rest
        if (h->h_rep_T[r] > 0.0) hot += h->h_rep_off[r + 1] - h->h_rep_off[r];
    return n * (m + st) + (a.nz_mode ? hot * 3 * vb : 0.0);
}

template <typename R, int EX, bool FULL, bool COMP, int K>
cudaError_t launch_stage_k(asd_handle* hd, const StageArgs<R>& a) {
    const int B = hd->block;
    const unsigned grid = (hd->n + B - 1) / B;
    size_t smem = 0;
    if (EX == ASD_EXCH_CSR && hd->sell.typed) {
        smem = sizeof(R) * table_stride<FULL>() * hd->sell.ntypes;
        if (hd->sell.stage == 2 && hd->sell.lwords16)
            smem = ((smem + 15) & ~(size_t)15) + ((2 * (size_t)hd->sell.stage_words + 15) & ~(size_t)15);
        else if (hd->sell.stage)
            smem = ((smem + 15) & ~(size_t)15) + 4 * (size_t)hd->sell.stage_words;
        if (hd->sell.stage == 2) smem += 3 * sizeof(R) * (size_t)hd->sell.spin_slots;
    }
    if (EX == ASD_EXCH_DIA && hd->dia.dtype) smem = sizeof(R) * table_stride<FULL>() *hd->dia.ntypes;
    {
        const cudaError_t e = raise_smem_limit(reinterpret_cast<const void*>(stage_kernel<R, EX, FULL, COMP, K>), smem);
        if (e != cudaSuccess) return e;
    }
    timer_begin(hd);
    {
        const cudaError_t e = launch_step_kernel(stage_kernel<R, EX, FULL, COMP, K>, dim3(grid), dim3(B), smem,
                                                 hd->stream, 1, step_pdl(hd), hd->sc, hd->sell, hd->dia, a);
        if (e != cudaSuccess) return e;
    }
    hd->launches += 1;
    if (hd->timing) {
        const bool typed = (EX == ASD_EXCH_CSR && hd->sell.typed) || (EX == ASD_EXCH_DIA && hd->dia.dtype);
        const std::string name = std::string("stage_kernel<") + (sizeof(R) == 4 ? "float" : "double") + "," +
                                 (EX == ASD_EXCH_CSR ? "SELL32" : EX == ASD_EXCH_DIA ? "DIA" : "NONE") +
                                 (typed ? "-typed" : "") + (FULL ? ",full" : ",diag") + (COMP ? ",comp" : "") +
                                 (K == 1 ? ",predictor>" : K == 2 ? ",corrector>" : K == 3 ? ",rk-stage>" : ",rk-last>");
        timer_end(hd, name, stage_bytes<R>(hd, a, COMP));
    }
    return cudaGetLastError();
}

template <typename R, int EX, bool FULL, bool COMP>
cudaError_t launch_stage_t(asd_handle* hd, const StageArgs<R>& a) {
    if (a.kind == 1) return launch_stage_k<R, EX, FULL, COMP, 1>(hd, a);
    if (a.kind == 2) return launch_stage_k<R, EX, FULL, COMP, 2>(hd, a);
    if (a.kind - 10 == a.nst - 1) return launch_stage_k<R, EX, FULL, COMP, 4>(hd, a);
    return launch_stage_k<R, EX, FULL, COMP, 3>(hd, a);
}

template <typename R, bool COMP>
cudaError_t launch_stage(asd_handle* hd, const StageArgs<R>& a) {
    if (hd->dexch == ASD_EXCH_CSR) {
        return hd->full ? launch_stage_t<R, ASD_EXCH_CSR, true, COMP>(hd, a) : launch_stage_t<R, ASD_EXCH_CSR, false, COMP>(hd, a);
    } else if (hd->dexch == ASD_EXCH_DIA) {
        return hd->full ? launch_stage_t<R, ASD_EXCH_DIA, true, COMP>(hd, a) : launch_stage_t<R, ASD_EXCH_DIA, false, COMP>(hd, a);
    }
    return launch_stage_t<R, ASD_EXCH_NONE, false, COMP>(hd, a);
}

template <typename R>
void state_ptrs(asd_handle* h, R* const** s, R* const** es, R* const** fn, R* const** det, R* const** stag) {
    if constexpr (sizeof(R) == 4) { *s = h->sf; *es = h->esf; *fn = h->fnf; *det = h->detf; *stag = h->stagf; }
    else { *s = h->sd; *es = h->esd; *fn = h->fnd; *det = h->detd; *stag = h->stagd; }
}

// Per-spin arrays a stage reads at its own rows, for the kernel's L2 prefetch: base S, the stage
// spin if it differs, the lo part (last stage, compensated), f_n (Heun corrector), the carried
// thermal field, the site-field profile, earlier RK increments.
template <typename R>
void set_prefetch(StageArgs<R>& a, bool comp) {
    const bool last = a.kind == 2 || (a.kind >= 10 && a.kind - 10 == a.nst - 1);
    uint32_t k = 0;
    auto add3 = [&](const void* p0, const void* p1, const void* p2) {
        if (!p0 || k + 3 > 24) return;
        a.pf[k++] = p0; a.pf[k++] = p1; a.pf[k++] = p2;
    };
    add3(a.base.p[0], a.base.p[1], a.base.p[2]);
    if (a.src.p[0] != a.base.p[0]) add3(a.src.p[0], a.src.p[1], a.src.p[2]);
    if (comp && last) add3(a.base_lo.p[0], a.base_lo.p[1], a.base_lo.p[2]);
    if (a.kind == 2) add3(a.fn.p[0], a.fn.p[1], a.fn.p[2]);
    if (a.nz_mode == 2) add3(a.nz.p[0], a.nz.p[1], a.nz.p[2]);
    add3(a.stag.p[0], a.stag.p[1], a.stag.p[2]);
    if (a.kind >= 10)
        for (int b = 0; b < a.kind - 10; b++) add3(a.k[b].p[0], a.k[b].p[1], a.k[b].p[2]);
    a.npf = k;
}

template <typename R>
cudaError_t fused_step_t(asd_handle* h, uint32_t rel) {
    R* const* s; R* const* es; R* const* fn; R* const* det; R* const* stag;
    state_ptrs<R>(h, &s, &es, &fn, &det, &stag);
    const bool comp = sizeof(R) == 4 && (h->p.flags & ASD_FLAG_COMPENSATED);
    StageArgs<R> a{};
    a.base = c3<R>(s);
    if (comp) a.base_lo = CVec3<float>{{h->sl[0], h->sl[1], h->sl[2]}};
    if (stag[0]) a.stag = c3<R>(stag);
    a.rel = rel;
    if constexpr (sizeof(R) == 4) a.nz = v3<R>(h->nzf); else a.nz = v3<R>(h->nzd);
    const uint64_t t = h->step + rel;
    const uint32_t upd = h->p.update ? h->p.update : 1;
    LongRange& L = h->lr;
    LrArgs none{};
    none.P = L.P; none.idx = L.mesh_idx; none.w = L.w; none.inv_p = L.P ? 1.0f / (float)L.P : 0.f;
    cudaError_t e;
    cudaError_t e0;
    if (h->d_ttm && (e0 = launch_ttm_step(h, h->d_step, rel)) != cudaSuccess) return e0;
    auto run = [&](const StageArgs<R>& a0) {
        StageArgs<R> aa = a0;
        set_prefetch(aa, comp);
        if constexpr (sizeof(R) == 4) return comp ? launch_stage<R, true>(h, aa) : launch_stage<R, false>(h, aa);
        else return launch_stage<R, false>(h, aa);
    };
    if (h->p.integrator == ASD_HEUN) {
        // predictor
        a.src = c3<R>(s); a.out = v3<R>(es); a.fn = v3<R>(fn); a.kind = 1; a.nz_mode = 1;
        a.lr = none;
        if (L.mode == ASD_LR_FFT) {
            if ((e = launch_lr_eval_f32(h)) != cudaSuccess) return e;   // field of S (scattered before)
            a.lr.hr = L.r + 3 * L.P; a.lr.mr = L.r;                    // gather H(S), scatter S'
        } else if (L.mode == ASD_LR_DIPOLE) {
            if (t % upd == 0 && (e = launch_lr_eval_f32(h)) != cudaSuccess) return e;
            a.lr.hr = L.r + 3 * L.P;
        }
        if ((e = run(a)) != cudaSuccess) return e;
        // corrector
        a.src = c3<R>(es); a.out = v3<R>(s); a.kind = 2; a.det = v3<R>(det); a.nz_mode = 2;
        if (comp) a.out_lo = Vec3<float>{{h->sl[0], h->sl[1], h->sl[2]}};
        a.lr = none;
        if (L.mode == ASD_LR_FFT) {
            if ((e = launch_lr_eval_f32(h)) != cudaSuccess) return e;   // field of S'
            a.lr.hr = L.r + 3 * L.P; a.lr.mr = L.r;                    // gather H(S'), scatter S_{n+1}
        } else if (L.mode == ASD_LR_DIPOLE) {
            a.lr.hr = L.r + 3 * L.P;
            if ((t + 1) % upd == 0) a.lr.mr = L.r;                     // next step refreshes from S_{n+1}
        }
        return run(a);
    }
    const int nst = h->p.integrator == ASD_RK4 ? 4 : 6;
    a.nst = nst;
    R* const* pp[2] = {es, fn};  // stage spins ping-pong between the es and fn buffers
    if (L.mode == ASD_LR_DIPOLE && t % upd == 0 && (e = launch_lr_eval_f32(h)) != cudaSuccess) return e;
    for (int st = 0; st < nst; st++) {
        a.kind = 10 + st;
        a.nz_mode = st == 0 ? 1 : 2;
        a.src = st == 0 ? c3<R>(s) : c3<R>(pp[(st - 1) & 1]);
        for (int q = 0; q < 6; q++) {
            if constexpr (sizeof(R) == 4) a.k[q] = v3<R>(h->kf[q]); else a.k[q] = v3<R>(h->kd[q]);
        }
        a.lr = none;
        if (L.mode == ASD_LR_FFT) {
            if ((e = launch_lr_eval_f32(h)) != cudaSuccess) return e;   // field of this stage's spins
            a.lr.hr = L.r + 3 * L.P; a.lr.mr = L.r;
        } else if (L.mode == ASD_LR_DIPOLE) {
            a.lr.hr = L.r + 3 * L.P;
            if (st == nst - 1 && (t + 1) % upd == 0) a.lr.mr = L.r;
        }
        if (st == nst - 1) {
            a.out = v3<R>(s);
            if (comp) a.out_lo = Vec3<float>{{h->sl[0], h->sl[1], h->sl[2]}};
        } else {
            a.out = v3<R>(pp[st & 1]);
        }
        if ((e = run(a)) != cudaSuccess) return e;
    }
    return cudaSuccess;
}

}  // namespace

template <typename R>
cudaError_t time_first_stage_t(asd_handle* h, int warm, int reps, float* ms) {
    R* const* s; R* const* es; R* const* fn; R* const* det; R* const* stag;
    state_ptrs<R>(h, &s, &es, &fn, &det, &stag);
    const bool comp = sizeof(R) == 4 && (h->p.flags & ASD_FLAG_COMPENSATED);
    StageArgs<R> a{};
    a.base = c3<R>(s);
    a.src = c3<R>(s);
    a.out = v3<R>(es);
    a.fn = v3<R>(fn);
    if (stag[0]) a.stag = c3<R>(stag);
    a.lr.P = h->lr.P; a.lr.idx = h->lr.mesh_idx; a.lr.w = h->lr.w;
    if constexpr (sizeof(R) == 4) a.nz = v3<R>(h->nzf); else a.nz = v3<R>(h->nzd);
    a.nz_mode = 1;
    if (h->p.integrator == ASD_HEUN) {
        a.kind = 1;
    } else {
        a.kind = 10;
        a.nst = h->p.integrator == ASD_RK4 ? 4 : 6;
        for (int q = 0; q < 6; q++) {
            if constexpr (sizeof(R) == 4) a.k[q] = v3<R>(h->kf[q]); else a.k[q] = v3<R>(h->kd[q]);
        }
    }
    set_prefetch(a, comp);
    auto run = [&]() {
        if constexpr (sizeof(R) == 4) return comp ? launch_stage<R, true>(h, a) : launch_stage<R, false>(h, a);
        else return launch_stage<R, false>(h, a);
    };
    cudaError_t e = cudaSuccess;
    for (int q = 0; q < warm && e == cudaSuccess; q++) e = run();
    if (e != cudaSuccess) return e;
    cudaEventRecord(h->kev[0], h->stream);
    for (int q = 0; q < reps && e == cudaSuccess; q++) e = run();
    cudaEventRecord(h->kev[1], h->stream);
    if (e != cudaSuccess) return e;
    if ((e = cudaEventSynchronize(h->kev[1])) != cudaSuccess) return e;
    float t = 0.f;
    if ((e = cudaEventElapsedTime(&t, h->kev[0], h->kev[1])) != cudaSuccess) return e;
    *ms = t / (float)reps;
    h->launches -= (uint64_t)(warm + reps);   // tuning launches are not step launches
    return cudaSuccess;
}

cudaError_t time_first_stage(asd_handle* h, int warm, int reps, float* ms) {
    if (h->p.precision == ASD_FP32) return time_first_stage_t<float>(h, warm, reps, ms);
    return time_first_stage_t<double>(h, warm, reps, ms);
}

cudaError_t launch_fused_step(asd_handle* h, uint32_t rel, bool) {
    if (h->p.precision == ASD_FP32) return fused_step_t<float>(h, rel);
    return fused_step_t<double>(h, rel);
}

cudaError_t launch_det_here(asd_handle* h) {
    const AppliedArg ap{{h->p.applied[0], h->p.applied[1], h->p.applied[2]}};
    const cudaError_t e = launch_step_kernel(det_here_k, dim3(1), dim3(1), 0, h->stream, 1, step_pdl(h),
                                             (const uint64_t*)h->d_step, h->d_dyn, h->d_dynf, ap);
    h->launches += 1;
    return e != cudaSuccess ? e : cudaGetLastError();
}

const void* det_here_kernel() { return reinterpret_cast<const void*>(det_here_k); }

cudaError_t update_det_applied(asd_handle* h) {
    if (!h->graph1 || !h->det_node) return cudaErrorInvalidValue;
    const uint64_t* step = h->d_step;
    double* dyn = h->d_dyn;
    float* dynf = h->d_dynf;
    AppliedArg ap{{h->p.applied[0], h->p.applied[1], h->p.applied[2]}};
    void* args[] = {&step, &dyn, &dynf, &ap};
    cudaKernelNodeParams kp{};
    kp.func = reinterpret_cast<void*>(det_here_k);
    kp.gridDim = dim3(1);
    kp.blockDim = dim3(1);
    kp.sharedMemBytes = 0;
    kp.kernelParams = args;
    kp.extra = nullptr;
    return cudaGraphExecKernelNodeSetParams(h->graph1, h->det_node, &kp);
}

cudaError_t launch_step_advance(asd_handle* h, uint32_t nsteps) {
    const cudaError_t e = launch_step_kernel(advance_k, dim3(1), dim3(1), 0, h->stream, 1, step_pdl(h), h->d_step, nsteps);
    h->launches += 1;
    return e != cudaSuccess ? e : cudaGetLastError();
}

}  // namespace asd
