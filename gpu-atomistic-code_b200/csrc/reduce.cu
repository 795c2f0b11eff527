// Magnetisation reduction, layout conversions at the host boundary, and the
// field-only evaluation behind asd_get_field.
#include "gather.cuh"
#include <algorithm>
#include <map>
#include <mutex>

namespace asd {
namespace {

inline unsigned nb(size_t n, int b) { return (unsigned)((n + b - 1) / b); }
constexpr int MAG_BLOCK = 256;

__device__ __forceinline__ double block_sum(double v, double* sm) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) sm[w] = v;
    __syncthreads();
    double r = 0.0;
    if (w == 0) {
        r = l < (int)(blockDim.x >> 5) ? sm[l] : 0.0;
        for (int o = 16; o > 0; o >>= 1) r += __shfl_down_sync(0xffffffffu, r, o);
    }
    return r;
}

struct MagFinish {
    uint32_t* cnt;              // block ticket counter (nullptr: mag_final forms the means)
    uint32_t nrep;
    const double* inv_count;    // 1 / spins per (replica, sublattice)
    double* out;                // means [nrep][nsub][3]
};

// The last block of a partial-sum launch to finish (ticket on *cnt) also forms the means:
// out[q] = inv_count * (the chunk partials of output q summed by the block in a fixed order),
// the same whatever the order the blocks finish in; it then rearms the counter.  Used
// when the outputs are few (cnt == nullptr: a separate mag_final launch does it).
__device__ __forceinline__ void mag_finish_last(uint32_t* cnt, uint32_t nblocks, uint32_t nrep, uint32_t nsub,
                                                uint32_t nchunk, const double* part, const double* inv_count,
                                                double* out, double* sm) {
    if (!cnt) return;
    __shared__ uint32_t last;
    __threadfence();                                   // this block's partials before its ticket
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(cnt, 1u) == nblocks - 1 ? 1u : 0u;
    __syncthreads();
    if (!last) return;
    __threadfence();
    // the whole block per output: thread t sums the chunks t, t + blockDim, ..., then a block sum
    for (uint32_t q = 0; q < nrep * nsub * 3; q++) {
        const uint32_t comp = q % 3, s = (q / 3) % nsub, r = q / (3 * nsub);
        double acc = 0.0;
        for (uint32_t ch = threadIdx.x; ch < nchunk; ch += blockDim.x)
            acc += __ldcg(part + (((size_t)r * nchunk + ch) * nsub + s) * 3 + comp);
        const double t = block_sum(acc, sm);
        if (threadIdx.x == 0) out[q] = t * inv_count[r * nsub + s];
    }
    if (threadIdx.x == 0) *cnt = 0;
}

// Partial sums of S over one chunk of one replica, per sublattice, in FP64 and
// a fixed reduction order (deterministic): part[((r*nchunk + c)*nsub + s)*3 + comp].
template <typename R>
__global__ void mag_partial(StepConst c, uint32_t nsub, const uint32_t* __restrict__ sub_of_atom,
                            const R* __restrict__ sx, const R* __restrict__ sy, const R* __restrict__ sz,
                            const float* __restrict__ lx, const float* __restrict__ ly, const float* __restrict__ lz,
                            uint32_t nchunk, double* __restrict__ part, MagFinish f) {
    __shared__ double sm[32];
    const uint32_t r = blockIdx.y, ch = blockIdx.x;
    const uint32_t beg = c.rep_off[r] + ch * MAG_CHUNK;
    const uint32_t end = min(c.rep_off[r + 1], beg + MAG_CHUNK);
    for (uint32_t s = 0; s < nsub; s++) {
        double a0 = 0.0, a1 = 0.0, a2 = 0.0;
        for (uint32_t i = beg + threadIdx.x; i < end; i += blockDim.x) {
            if (sub_of_atom[atom_of(c, i)] != s) continue;
            a0 += (double)sx[i]; a1 += (double)sy[i]; a2 += (double)sz[i];
            if (lx) { a0 += (double)lx[i]; a1 += (double)ly[i]; a2 += (double)lz[i]; }
        }
        const double t0 = block_sum(a0, sm), t1 = block_sum(a1, sm), t2 = block_sum(a2, sm);
        if (threadIdx.x == 0) {
            double* o = part + (((size_t)r * nchunk + ch) * nsub + s) * 3;
            o[0] = t0; o[1] = t1; o[2] = t2;
        }
    }
    mag_finish_last(f.cnt, gridDim.x * gridDim.y, f.nrep, nsub, nchunk, part, f.inv_count, f.out, sm);
}

// One pass over the chunk for up to NS sublattices, each spin added to its own sublattice's
// register accumulators (the general kernel above re-reads the chunk once per sublattice).
template <typename R, int NS>
__global__ void mag_partial_ns(StepConst c, uint32_t nsub, const uint32_t* __restrict__ sub_of_atom,
                               const R* __restrict__ sx, const R* __restrict__ sy, const R* __restrict__ sz,
                               const float* __restrict__ lx, const float* __restrict__ ly,
                               const float* __restrict__ lz, uint32_t nchunk, double* __restrict__ part,
                               MagFinish f) {
    __shared__ double sm[32];
    const uint32_t r = blockIdx.y, ch = blockIdx.x;
    const uint32_t beg = c.rep_off[r] + ch * MAG_CHUNK;
    const uint32_t end = min(c.rep_off[r + 1], beg + MAG_CHUNK);
    double a[NS][3];
#pragma unroll
    for (int q = 0; q < NS; q++) a[q][0] = a[q][1] = a[q][2] = 0.0;
    for (uint32_t i = beg + threadIdx.x; i < end; i += blockDim.x) {
        const uint32_t s = NS == 1 ? 0u : sub_of_atom[atom_of(c, i)];
        double v0 = (double)sx[i], v1 = (double)sy[i], v2 = (double)sz[i];
        if (lx) { v0 += (double)lx[i]; v1 += (double)ly[i]; v2 += (double)lz[i]; }
#pragma unroll
        for (int q = 0; q < NS; q++)
            if (s == (uint32_t)q) { a[q][0] += v0; a[q][1] += v1; a[q][2] += v2; }
    }
    for (uint32_t q = 0; q < nsub; q++) {
        double t[3];
#pragma unroll
        for (int k = 0; k < 3; k++) {
            double v = 0.0;
#pragma unroll
            for (int qq = 0; qq < NS; qq++) if ((uint32_t)qq == q) v = a[qq][k];
            t[k] = block_sum(v, sm);
        }
        if (threadIdx.x == 0) {
            double* o = part + (((size_t)r * nchunk + ch) * nsub + q) * 3;
            o[0] = t[0]; o[1] = t[1]; o[2] = t[2];
        }
    }
    mag_finish_last(f.cnt, gridDim.x * gridDim.y, f.nrep, nsub, nchunk, part, f.inv_count, f.out, sm);
}

// Plain form: AoS doubles.
__global__ void mag_partial_aos(StepConst c, uint32_t nsub, const uint32_t* __restrict__ sub_of_atom,
                                const double* __restrict__ s3, uint32_t nchunk, double* __restrict__ part,
                                MagFinish f) {
    __shared__ double sm[32];
    const uint32_t r = blockIdx.y, ch = blockIdx.x;
    const uint32_t beg = c.rep_off[r] + ch * MAG_CHUNK;
    const uint32_t end = min(c.rep_off[r + 1], beg + MAG_CHUNK);
    for (uint32_t s = 0; s < nsub; s++) {
        double a0 = 0.0, a1 = 0.0, a2 = 0.0;
        for (uint32_t i = beg + threadIdx.x; i < end; i += blockDim.x) {
            if (sub_of_atom[atom_of(c, i)] != s) continue;
            a0 += s3[3 * (size_t)i]; a1 += s3[3 * (size_t)i + 1]; a2 += s3[3 * (size_t)i + 2];
        }
        const double t0 = block_sum(a0, sm), t1 = block_sum(a1, sm), t2 = block_sum(a2, sm);
        if (threadIdx.x == 0) {
            double* o = part + (((size_t)r * nchunk + ch) * nsub + s) * 3;
            o[0] = t0; o[1] = t1; o[2] = t2;
        }
    }
    mag_finish_last(f.cnt, gridDim.x * gridDim.y, f.nrep, nsub, nchunk, part, f.inv_count, f.out, sm);
}

__global__ void mag_final(uint32_t nrep, uint32_t nsub, uint32_t nchunk, const double* __restrict__ part,
                          const double* __restrict__ inv_count, double* __restrict__ out) {
    // one block per (replica, sublattice, component): its threads stride over the chunks, then a
    // block sum (fixed order, so the result does not depend on timing)
    __shared__ double sm[32];
    const uint32_t q = blockIdx.x;
    if (q >= nrep * nsub * 3) return;
    const uint32_t comp = q % 3, s = (q / 3) % nsub, r = q / (3 * nsub);
    double acc = 0.0;
    for (uint32_t ch = threadIdx.x; ch < nchunk; ch += blockDim.x)
        acc += part[(((size_t)r * nchunk + ch) * nsub + s) * 3 + comp];
    const double t = block_sum(acc, sm);
    if (threadIdx.x == 0) out[q] = t * inv_count[r * nsub + s];
}

template <typename R>
__global__ void spins_in_k(uint32_t n, const double* __restrict__ aos, R* __restrict__ x, R* __restrict__ y,
                           R* __restrict__ z, float* __restrict__ lx, float* __restrict__ ly, float* __restrict__ lz) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double v[3] = {aos[3 * (size_t)i], aos[3 * (size_t)i + 1], aos[3 * (size_t)i + 2]};
    const double m = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    v[0] /= m; v[1] /= m; v[2] /= m;
    const R hx = (R)v[0], hy = (R)v[1], hz = (R)v[2];
    x[i] = hx; y[i] = hy; z[i] = hz;
    if (lx) { lx[i] = (float)(v[0] - (double)hx); ly[i] = (float)(v[1] - (double)hy); lz[i] = (float)(v[2] - (double)hz); }
}

// Input checks of a spin array (AoS doubles), as the host-side checks they replace: bad[0] =
// the first non-finite component, bad[1] = the first spin of squared length <= 1e-24 (both
// ~0 when none; the caller sets them to ~0 first).  The squared length is formed without
// contraction, as the host's scalar code forms it.
__global__ void spins_check_k(uint32_t n, const double* __restrict__ aos, unsigned long long* bad) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double x = aos[3 * (size_t)i], y = aos[3 * (size_t)i + 1], z = aos[3 * (size_t)i + 2];
    const double v[3] = {x, y, z};
    for (int c = 0; c < 3; c++)
        if (!isfinite(v[c])) { atomicMin(bad, 3ull * i + c); break; }
    const double m = __dadd_rn(__dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y)), __dmul_rn(z, z));
    if (!(m > 1e-24)) atomicMin(bad + 1, (unsigned long long)i);
}

// FP64 plain form: S / |S| with the host's operations in the host's order (IEEE square root and
// division, no contraction), into the plain form's AoS state.
__global__ void spins_in_plain_k(uint32_t n, const double* __restrict__ aos, double* __restrict__ s) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double x = aos[3 * (size_t)i], y = aos[3 * (size_t)i + 1], z = aos[3 * (size_t)i + 2];
    const double m = __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y)), __dmul_rn(z, z)));
    s[3 * (size_t)i] = __ddiv_rn(x, m);
    s[3 * (size_t)i + 1] = __ddiv_rn(y, m);
    s[3 * (size_t)i + 2] = __ddiv_rn(z, m);
}

template <typename R>
__global__ void soa_out_k(uint32_t n, const R* __restrict__ x, const R* __restrict__ y, const R* __restrict__ z,
                          const float* __restrict__ lx, const float* __restrict__ ly, const float* __restrict__ lz,
                          double* __restrict__ aos) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double v0 = (double)x[i], v1 = (double)y[i], v2 = (double)z[i];
    if (lx) { v0 += (double)lx[i]; v1 += (double)ly[i]; v2 += (double)lz[i]; }
    aos[3 * (size_t)i] = v0; aos[3 * (size_t)i + 1] = v1; aos[3 * (size_t)i + 2] = v2;
}

// Exchange (+ held long-range) field of the current spins, AoS double out.
template <typename R, int EX, bool FULL>
__global__ void field_k(StepConst c, SellDev sell, DiaDev dia, const R* __restrict__ sx, const R* __restrict__ sy,
                        const R* __restrict__ sz, const float* __restrict__ hr, float inv_p, size_t P,
                        const uint32_t* __restrict__ idx, double* __restrict__ out) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    R* tab = reinterpret_cast<R*>(smem_raw);
    if constexpr (EX == ASD_EXCH_CSR) {
        if (sell.typed) load_table<R>(table_of<R>(sell), table_stride<FULL>() *sell.ntypes, tab);
    }
    if constexpr (EX == ASD_EXCH_DIA) {
        if (dia.dtype) load_table<R>(table_of<R>(dia), table_stride<FULL>() *dia.ntypes, tab);
    }
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= c.n) return;
    R hr3[3] = {R(0), R(0), R(0)};
    const CVec3<R> src{{sx, sy, sz}};
    if constexpr (EX == ASD_EXCH_CSR) gather_sell<R, FULL>(sell, i, src, tab, hr3);
    if constexpr (EX == ASD_EXCH_DIA) gather_dia<R, FULL>(dia, c.n, i, src, tab, hr3);
    if (c.q4_ptr) {
        R h4[3];
        four_spin<R>(c, i, [&](uint32_t j, R v[3]) { v[0] = src.p[0][j]; v[1] = src.p[1][j]; v[2] = src.p[2][j]; }, h4);
        hr3[0] += h4[0]; hr3[1] += h4[1]; hr3[2] += h4[2];
    }
    double h[3] = {(double)hr3[0], (double)hr3[1], (double)hr3[2]};
    if (hr) {
        const uint32_t m = idx[i];
        for (int a = 0; a < 3; a++) h[a] += (double)(hr[a * P + m] * inv_p);
    }
    out[3 * (size_t)i] = h[0]; out[3 * (size_t)i + 1] = h[1]; out[3 * (size_t)i + 2] = h[2];
}

template <typename R>
void state(asd_handle* h, R** s) {
    for (int c = 0; c < 3; c++) {
        if constexpr (sizeof(R) == 4) s[c] = h->sf[c]; else s[c] = h->sd[c];
    }
}

template <typename R>
cudaError_t field_t(asd_handle* h, double* out) {
    R* s[3];
    state<R>(h, s);
    const float* hr = nullptr;
    if (h->lr.mode != ASD_LR_NONE) {
        if (h->lr.mode == ASD_LR_FFT) {
            cudaError_t e = launch_lr_eval_f32(h);
            if (e != cudaSuccess) return e;
        }
        hr = h->lr.r + 3 * h->lr.P;
    }
    const float inv_p = h->lr.P ? 1.0f / (float)h->lr.P : 0.f;
    const unsigned g = nb(h->n, 256);
    const size_t cs = sizeof(R) * (h->full ? table_stride<true>() : table_stride<false>());
    if (h->dexch == ASD_EXCH_CSR) {
        const size_t sm = h->sell.typed ? cs * h->sell.ntypes : 0;
        if (h->full) field_k<R, ASD_EXCH_CSR, true><<<g, 256, sm, h->stream>>>(h->sc, h->sell, h->dia, s[0], s[1], s[2], hr, inv_p, h->lr.P, h->lr.mesh_idx, out);
        else field_k<R, ASD_EXCH_CSR, false><<<g, 256, sm, h->stream>>>(h->sc, h->sell, h->dia, s[0], s[1], s[2], hr, inv_p, h->lr.P, h->lr.mesh_idx, out);
    } else if (h->dexch == ASD_EXCH_DIA) {
        const size_t sm = h->dia.dtype ? cs * h->dia.ntypes : 0;
        if (h->full) field_k<R, ASD_EXCH_DIA, true><<<g, 256, sm, h->stream>>>(h->sc, h->sell, h->dia, s[0], s[1], s[2], hr, inv_p, h->lr.P, h->lr.mesh_idx, out);
        else field_k<R, ASD_EXCH_DIA, false><<<g, 256, sm, h->stream>>>(h->sc, h->sell, h->dia, s[0], s[1], s[2], hr, inv_p, h->lr.P, h->lr.mesh_idx, out);
    } else {
        field_k<R, ASD_EXCH_NONE, false><<<g, 256, 0, h->stream>>>(h->sc, h->sell, h->dia, s[0], s[1], s[2], hr, inv_p, h->lr.P, h->lr.mesh_idx, out);
    }
    h->launches += 1;
    return cudaGetLastError();
}

// Welford update of |m_s| per (replica, sublattice), the RunningStat::Push of inc/util.h:30-50:
// st[4q..4q+3] = n, mean, M2, mean before this sample.
__global__ void mag_push_k(uint32_t m, const double* __restrict__ mag, double* __restrict__ st) {
    const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= m) return;
    const double x = sqrt(mag[3 * q] * mag[3 * q] + mag[3 * q + 1] * mag[3 * q + 1] + mag[3 * q + 2] * mag[3 * q + 2]);
    double* s = st + 4 * (size_t)q;
    const double n = s[0] + 1.0;
    const double old = s[1];
    s[3] = old;
    if (n == 1.0) {
        s[1] = x;
        s[2] = 0.0;
    } else {
        const double mean = old + (x - old) / n;
        s[2] = s[2] + (x - old) * (x - mean);
        s[1] = mean;
    }
    s[0] = n;
}

__global__ void set_scalar_k(double* dst, double v) { *dst = v; }

struct Dyn3 { double v[3]; };
// dst[0..2] = v and, when dstf is set, dstf[0..2] = (float)v: the three components of one
// mutable vector (the applied field) in one launch.
__global__ void set_vec3_k(double* dst, float* dstf, Dyn3 v) {
    const int k = threadIdx.x;
    if (k < 3) {
        dst[k] = v.v[k];
        if (dstf) dstf[k] = (float)v.v[k];
    }
}
__global__ void set_scalar_f_k(float* dst, float v) { *dst = v; }

}  // namespace

cudaError_t launch_set_vec3(asd_handle* h, double* dst, float* dstf, const double v[3]) {
    Dyn3 d;
    for (int k = 0; k < 3; k++) d.v[k] = v[k];
    set_vec3_k<<<1, 32, 0, h->stream>>>(dst, dstf, d);
    h->launches += 1;
    return cudaGetLastError();
}

cudaError_t launch_set_scalar(asd_handle* h, double* dst, double v) {
    set_scalar_k<<<1, 1, 0, h->stream>>>(dst, v);
    h->launches += 1;
    return cudaGetLastError();
}

// Two-temperature model, one step (src/laser_heating.cpp:884-895), then the spin bath
// temperature of every replica.
__global__ void ttm_step_k(TtmDev* s, const uint64_t* step_base, uint64_t t, uint32_t nrep, double* sq,
                           float* sqf) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const uint64_t step = step_base ? *step_base + t : t;
    const double time = (double)(step - s->t0) * s->dt;
    double P = 0.0;
    for (uint32_t p = 0; p < s->np; p++) {
        const double x = (time - s->delay[p]) / s->tau;
        P += s->P * s->scale[p] * exp(-(x * x));
    }
    const double Te = s->Te, Tl = s->Tl;
    const double Ten = (-s->G * (Te - Tl) + P) * s->dt / (s->ge * Te) + Te;
    const double Tln = (s->G * (Ten - Tl) - s->Cl * (Tl - s->T0) / s->ct) * s->dt / s->Cl + Tl;
    s->Te = Ten;
    s->Tl = Tln;
    const double r = sqrt(s->bath_e ? Ten : Tln);
    for (uint32_t q = 0; q < nrep; q++) { sq[q] = r; sqf[q] = (float)r; }
}

cudaError_t launch_ttm_step(asd_handle* h, const uint64_t* step_base, uint64_t t) {
    ttm_step_k<<<1, 32, 0, h->stream>>>(h->d_ttm, step_base, t, h->nrep, h->d_rep_sqrtT, h->d_rep_sqrtT_f);
    h->launches += 1;
    return cudaGetLastError();
}

cudaError_t launch_mag_push(asd_handle* h) {
    const uint32_t m = h->nrep * h->nsub;
    mag_push_k<<<nb(m, 128), 128, 0, h->stream>>>(m, h->d_mag, h->d_stats);
    h->launches += 1;
    return cudaGetLastError();
}

cudaError_t launch_set_scalar_f(asd_handle* h, float* dst, float v) {
    set_scalar_f_k<<<1, 1, 0, h->stream>>>(dst, v);
    h->launches += 1;
    return cudaGetLastError();
}

cudaError_t launch_field_only(asd_handle* h, double* d_out) {
    if (h->p.precision == ASD_FP64_PLAIN) return launch_plain_field(h, d_out);
    if (h->p.precision == ASD_FP32) return field_t<float>(h, d_out);
    return field_t<double>(h, d_out);
}

cudaError_t launch_magnetisation(asd_handle* h) {
    const uint32_t nsub = h->nsub;
    uint32_t maxrep = 0;
    for (uint32_t r = 0; r < h->nrep; r++) maxrep = std::max(maxrep, h->h_rep_off[r + 1] - h->h_rep_off[r]);
    const uint32_t nchunk = (maxrep + MAG_CHUNK - 1) / MAG_CHUNK;
    dim3 grid(nchunk ? nchunk : 1, h->nrep);
    const uint32_t* sub_of_atom = h->d_sub_of_atom;
    const double* inv_count = h->d_inv_count;
    // few outputs: the last partial block forms the means (one launch); else mag_final does
    const uint32_t nq = h->nrep * nsub * 3;
    const MagFinish f{nq <= 12 ? h->d_magcnt : nullptr, h->nrep, inv_count, h->d_mag};
    if (h->p.precision == ASD_FP64_PLAIN) {
        mag_partial_aos<<<grid, MAG_BLOCK, 0, h->stream>>>(h->sc, nsub, sub_of_atom, h->p_s, grid.x, h->d_magpart, f);
    } else if (h->p.precision == ASD_FP32) {
        const bool comp = (h->p.flags & ASD_FLAG_COMPENSATED) != 0;
        const float* lo[3] = {comp ? h->sl[0] : nullptr, comp ? h->sl[1] : nullptr, comp ? h->sl[2] : nullptr};
        if (nsub == 1)
            mag_partial_ns<float, 1><<<grid, MAG_BLOCK, 0, h->stream>>>(h->sc, nsub, sub_of_atom, h->sf[0], h->sf[1],
                                                                        h->sf[2], lo[0], lo[1], lo[2], grid.x, h->d_magpart, f);
        else if (nsub == 2)
            mag_partial_ns<float, 2><<<grid, MAG_BLOCK, 0, h->stream>>>(h->sc, nsub, sub_of_atom, h->sf[0], h->sf[1],
                                                                        h->sf[2], lo[0], lo[1], lo[2], grid.x, h->d_magpart, f);
        else if (nsub <= 4)
            mag_partial_ns<float, 4><<<grid, MAG_BLOCK, 0, h->stream>>>(h->sc, nsub, sub_of_atom, h->sf[0], h->sf[1],
                                                                        h->sf[2], lo[0], lo[1], lo[2], grid.x, h->d_magpart, f);
        else
            mag_partial<float><<<grid, MAG_BLOCK, 0, h->stream>>>(h->sc, nsub, sub_of_atom, h->sf[0], h->sf[1], h->sf[2],
                                                                 lo[0], lo[1], lo[2], grid.x, h->d_magpart, f);
    } else {
        mag_partial<double><<<grid, MAG_BLOCK, 0, h->stream>>>(h->sc, nsub, sub_of_atom, h->sd[0], h->sd[1], h->sd[2],
                                                              nullptr, nullptr, nullptr, grid.x, h->d_magpart, f);
    }
    h->launches += 1;
    if (!f.cnt) {
        mag_final<<<nq, 128, 0, h->stream>>>(h->nrep, nsub, grid.x, h->d_magpart, inv_count, h->d_mag);
        h->launches += 1;
    }
    return cudaGetLastError();
}

cudaError_t raise_smem_limit(const void* kernel, size_t bytes) {
    if (bytes <= 48 * 1024) return cudaSuccess;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    static std::mutex mu;
    static std::map<std::pair<int, const void*>, size_t> raised;
    std::lock_guard<std::mutex> lock(mu);
    size_t& have = raised[{dev, kernel}];
    if (bytes <= have) return cudaSuccess;
    e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e == cudaSuccess) have = bytes;
    return e;
}

cudaError_t launch_check_spins(asd_handle* h, const double* d_aos, unsigned long long* d_check) {
    cudaError_t e = cudaMemsetAsync(d_check, 0xff, 2 * sizeof(unsigned long long), h->stream);
    if (e != cudaSuccess) return e;
    spins_check_k<<<nb(h->n, 256), 256, 0, h->stream>>>(h->n, d_aos, d_check);
    h->launches += 1;
    return cudaGetLastError();
}

cudaError_t launch_convert_spins_in(asd_handle* h, const double* d_aos) {
    const unsigned g = nb(h->n, 256);
    if (h->p.precision == ASD_FP64_PLAIN) {
        spins_in_plain_k<<<g, 256, 0, h->stream>>>(h->n, d_aos, h->p_s);
    } else if (h->p.precision == ASD_FP32) {
        const bool comp = (h->p.flags & ASD_FLAG_COMPENSATED) != 0;
        spins_in_k<float><<<g, 256, 0, h->stream>>>(h->n, d_aos, h->sf[0], h->sf[1], h->sf[2], comp ? h->sl[0] : nullptr,
                                                     comp ? h->sl[1] : nullptr, comp ? h->sl[2] : nullptr);
    } else {
        spins_in_k<double><<<g, 256, 0, h->stream>>>(h->n, d_aos, h->sd[0], h->sd[1], h->sd[2], nullptr, nullptr, nullptr);
    }
    h->launches += 1;
    return cudaGetLastError();
}

// what: 0 spins, 1 det field
cudaError_t launch_convert_out(asd_handle* h, int what, double* d_aos) {
    const unsigned g = nb(h->n, 256);
    if (h->p.precision == ASD_FP32) {
        const bool comp = what == 0 && (h->p.flags & ASD_FLAG_COMPENSATED) != 0;
        float* const* s = what == 0 ? h->sf : h->detf;
        soa_out_k<float><<<g, 256, 0, h->stream>>>(h->n, s[0], s[1], s[2], comp ? h->sl[0] : nullptr,
                                                   comp ? h->sl[1] : nullptr, comp ? h->sl[2] : nullptr, d_aos);
    } else {
        double* const* s = what == 0 ? h->sd : h->detd;
        soa_out_k<double><<<g, 256, 0, h->stream>>>(h->n, s[0], s[1], s[2], nullptr, nullptr, nullptr, d_aos);
    }
    h->launches += 1;
    return cudaGetLastError();
}

}  // namespace asd
