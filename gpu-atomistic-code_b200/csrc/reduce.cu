// Magnetisation reduction, layout conversions at the host boundary, and the
// field-only evaluation behind asd_get_field.
#include "gather.cuh"
#include <algorithm>
#include <map>
#include <mutex>
#include <tuple>

namespace asd {
namespace {

inline unsigned nb(size_t n, int b) { return (unsigned)((n + b - 1) / b); }
constexpr int MAG_BLOCK = 256;

// Sums N values over the block together (one shared-memory round for all N); the totals are
// valid in thread 0.  The order is fixed, so the result does not depend on timing.  sm holds
// N * 32 doubles.
template <int N>
__device__ __forceinline__ void block_sum_n(double (&v)[N], double* sm) {
#pragma unroll
    for (int k = 0; k < N; k++)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], o);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31, nw = blockDim.x >> 5;
    __syncthreads();
    if (l == 0) {
#pragma unroll
        for (int k = 0; k < N; k++) sm[k * 32 + w] = v[k];
    }
    __syncthreads();
    if (w == 0) {
#pragma unroll
        for (int k = 0; k < N; k++) {
            double r = l < nw ? sm[k * 32 + l] : 0.0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) r += __shfl_down_sync(0xffffffffu, r, o);
            v[k] = r;
        }
    }
}

// Outputs the last partial block forms by itself (more: a separate mag_final launch).
constexpr uint32_t MAG_FINISH_MAX = 12;

struct MagFinish {
    uint32_t* cnt;              // block ticket counter (nullptr: mag_final forms the means)
    uint32_t nrep;
    const double* inv_count;    // 1 / spins per (replica, sublattice)
    double* out;                // means [nrep][nsub][3]
    double* hout;               // the caller's page-locked host buffer (device address), or nullptr
};

// The means from the chunk partials, by one block: thread t adds the words t, t + blockDim, ...
// of each replica's [chunk][sublattice][component] run of partials to the accumulator of the
// word's output (NQ accumulators, at least nrep * nsub * 3), then one block sum of them all.
template <int NQ>
__device__ __forceinline__ void mag_sum_outputs(const MagFinish& f, uint32_t nsub, uint32_t nchunk,
                                                const double* part, double* sm) {
    double acc[NQ];
#pragma unroll
    for (int k = 0; k < NQ; k++) acc[k] = 0.0;
    const uint32_t w = nsub * 3, m = nchunk * w;
    for (uint32_t r = 0; r < f.nrep; r++) {
        const double* p = part + (size_t)r * m;
#pragma unroll 4
        for (uint32_t e = threadIdx.x; e < m; e += blockDim.x) {
            const double v = __ldcg(p + e);
            const uint32_t q = r * w + e % w;
#pragma unroll
            for (uint32_t k = 0; k < (uint32_t)NQ; k++)
                if (k == q) acc[k] += v;
        }
    }
    block_sum_n<NQ>(acc, sm);
    if (threadIdx.x == 0) {
        const uint32_t nq = f.nrep * w;
#pragma unroll
        for (uint32_t k = 0; k < (uint32_t)NQ; k++) {
            if (k < nq) {
                const double mq = acc[k] * f.inv_count[k / 3];
                f.out[k] = mq;
                if (f.hout) f.hout[k] = mq;
            }
        }
    }
}

// The last block of a partial-sum launch to finish (ticket on *cnt) also forms the means:
// out[q] = inv_count * (the chunk partials of output q summed by the block in a fixed order),
// the same whatever the order the blocks finish in; it then rearms the counter.  Every caller
// stores its block's partials from thread 0.
__device__ __forceinline__ void mag_finish_last(const MagFinish& f, uint32_t nblocks, uint32_t nsub, uint32_t nchunk,
                                                const double* part, double* sm) {
    if (!f.cnt) return;
    __shared__ uint32_t last;
    // thread 0 stored this block's partials: its ticket, a release-acquire add, orders them
    // before the count and, in the last block, every earlier block's partials before the reads
    // below (the block barrier passes that on to the other threads)
    if (threadIdx.x == 0) {
        uint32_t old;
        asm volatile("atom.add.acq_rel.gpu.u32 %0, [%1], 1;" : "=r"(old) : "l"(f.cnt) : "memory");
        last = old == nblocks - 1 ? 1u : 0u;
    }
    __syncthreads();
    if (!last) return;
    const uint32_t nq = f.nrep * nsub * 3;
    if (nq <= 3) mag_sum_outputs<3>(f, nsub, nchunk, part, sm);
    else if (nq <= 6) mag_sum_outputs<6>(f, nsub, nchunk, part, sm);
    else mag_sum_outputs<MAG_FINISH_MAX>(f, nsub, nchunk, part, sm);
    if (threadIdx.x == 0) *f.cnt = 0;
}

// Sixteen-byte vector of spin components: 4 floats or 2 doubles.
template <typename R> struct Vec16;
template <> struct Vec16<float> {
    static constexpr uint32_t n = 4;
    __device__ static void load(const float* p, double (&o)[4]) {
        const float4 v = __ldg(reinterpret_cast<const float4*>(p));
        o[0] = v.x; o[1] = v.y; o[2] = v.z; o[3] = v.w;
    }
};
template <> struct Vec16<double> {
    static constexpr uint32_t n = 2;
    __device__ static void load(const double* p, double (&o)[2]) {
        const double2 v = __ldg(reinterpret_cast<const double2*>(p));
        o[0] = v.x; o[1] = v.y;
    }
};

// Partial sums of S over one chunk of one replica for NS >= nsub sublattices in one pass,
// in FP64 and a fixed order (deterministic): part[((r*nchunk + c)*nsub + s)*3 + comp].  A
// whole chunk that starts on a 16-byte boundary is read with one vector load per array and
// thread per round (all of a thread's loads in flight together); other chunks spin by spin.
template <typename R, int NS>
__global__ void __launch_bounds__(MAG_BLOCK, 4)
    mag_partial_ns(StepConst c, uint32_t nsub, const uint32_t* __restrict__ sub_of_atom, const R* __restrict__ sx,
                   const R* __restrict__ sy, const R* __restrict__ sz, const float* __restrict__ lx,
                   const float* __restrict__ ly, const float* __restrict__ lz, uint32_t nchunk,
                   double* __restrict__ part, MagFinish f) {
    __shared__ double sm[MAG_FINISH_MAX * 32];
    const uint32_t r = blockIdx.y, ch = blockIdx.x;
    const uint32_t beg = c.rep_off[r] + ch * MAG_CHUNK;
    const uint32_t end = min(c.rep_off[r + 1], beg + MAG_CHUNK);
    double a[3 * NS];
#pragma unroll
    for (int k = 0; k < 3 * NS; k++) a[k] = 0.0;
    auto add = [&](uint32_t i, double v0, double v1, double v2) {
        const uint32_t s = NS == 1 ? 0u : sub_of_atom[atom_of(c, i)];
#pragma unroll
        for (int q = 0; q < NS; q++)
            if (s == (uint32_t)q) { a[3 * q] += v0; a[3 * q + 1] += v1; a[3 * q + 2] += v2; }
    };
    constexpr uint32_t V = Vec16<R>::n;
    constexpr uint32_t ROUNDS = MAG_CHUNK / (V * MAG_BLOCK);
    static_assert(ROUNDS * V * MAG_BLOCK == MAG_CHUNK, "a chunk is a whole number of vector rounds");
    const uintptr_t ptrs = reinterpret_cast<uintptr_t>(sx) | reinterpret_cast<uintptr_t>(sy) |
                           reinterpret_cast<uintptr_t>(sz) | reinterpret_cast<uintptr_t>(lx) |
                           reinterpret_cast<uintptr_t>(ly) | reinterpret_cast<uintptr_t>(lz);
    if (end - beg == MAG_CHUNK && beg % V == 0 && (ptrs & 15u) == 0 && blockDim.x == MAG_BLOCK) {
#pragma unroll
        for (uint32_t k = 0; k < ROUNDS; k++) {
            const uint32_t i = beg + V * (threadIdx.x + k * MAG_BLOCK);
            double x[V], y[V], z[V];
            Vec16<R>::load(sx + i, x); Vec16<R>::load(sy + i, y); Vec16<R>::load(sz + i, z);
            if constexpr (sizeof(R) == 4) {
                if (lx) {       // the low words of the compensated FP32 form
                    double u[V], v[V], w[V];
                    Vec16<float>::load(lx + i, u); Vec16<float>::load(ly + i, v); Vec16<float>::load(lz + i, w);
#pragma unroll
                    for (uint32_t j = 0; j < V; j++) { x[j] += u[j]; y[j] += v[j]; z[j] += w[j]; }
                }
            }
#pragma unroll
            for (uint32_t j = 0; j < V; j++) add(i + j, x[j], y[j], z[j]);
        }
    } else {
        for (uint32_t i = beg + threadIdx.x; i < end; i += blockDim.x) {
            double v0 = (double)sx[i], v1 = (double)sy[i], v2 = (double)sz[i];
            if (lx) { v0 += (double)lx[i]; v1 += (double)ly[i]; v2 += (double)lz[i]; }
            add(i, v0, v1, v2);
        }
    }
    block_sum_n<3 * NS>(a, sm);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int q = 0; q < NS; q++) {
            if ((uint32_t)q < nsub) {
                double* o = part + (((size_t)r * nchunk + ch) * nsub + q) * 3;
                o[0] = a[3 * q]; o[1] = a[3 * q + 1]; o[2] = a[3 * q + 2];
            }
        }
    }
    mag_finish_last(f, gridDim.x * gridDim.y, nsub, nchunk, part, sm);
}

// Any number of sublattices: one pass over the chunk per sublattice.
template <typename R>
__global__ void __launch_bounds__(MAG_BLOCK)
    mag_partial(StepConst c, uint32_t nsub, const uint32_t* __restrict__ sub_of_atom, const R* __restrict__ sx,
                const R* __restrict__ sy, const R* __restrict__ sz, const float* __restrict__ lx,
                const float* __restrict__ ly, const float* __restrict__ lz, uint32_t nchunk,
                double* __restrict__ part, MagFinish f) {
    __shared__ double sm[MAG_FINISH_MAX * 32];
    const uint32_t r = blockIdx.y, ch = blockIdx.x;
    const uint32_t beg = c.rep_off[r] + ch * MAG_CHUNK;
    const uint32_t end = min(c.rep_off[r + 1], beg + MAG_CHUNK);
    for (uint32_t s = 0; s < nsub; s++) {
        double a[3] = {0.0, 0.0, 0.0};
        for (uint32_t i = beg + threadIdx.x; i < end; i += blockDim.x) {
            if (sub_of_atom[atom_of(c, i)] != s) continue;
            a[0] += (double)sx[i]; a[1] += (double)sy[i]; a[2] += (double)sz[i];
            if (lx) { a[0] += (double)lx[i]; a[1] += (double)ly[i]; a[2] += (double)lz[i]; }
        }
        block_sum_n<3>(a, sm);
        if (threadIdx.x == 0) {
            double* o = part + (((size_t)r * nchunk + ch) * nsub + s) * 3;
            o[0] = a[0]; o[1] = a[1]; o[2] = a[2];
        }
    }
    mag_finish_last(f, gridDim.x * gridDim.y, nsub, nchunk, part, sm);
}

// Plain form: AoS doubles.
__global__ void __launch_bounds__(MAG_BLOCK)
    mag_partial_aos(StepConst c, uint32_t nsub, const uint32_t* __restrict__ sub_of_atom,
                    const double* __restrict__ s3, uint32_t nchunk, double* __restrict__ part, MagFinish f) {
    __shared__ double sm[MAG_FINISH_MAX * 32];
    const uint32_t r = blockIdx.y, ch = blockIdx.x;
    const uint32_t beg = c.rep_off[r] + ch * MAG_CHUNK;
    const uint32_t end = min(c.rep_off[r + 1], beg + MAG_CHUNK);
    for (uint32_t s = 0; s < nsub; s++) {
        double a[3] = {0.0, 0.0, 0.0};
        for (uint32_t i = beg + threadIdx.x; i < end; i += blockDim.x) {
            if (sub_of_atom[atom_of(c, i)] != s) continue;
            a[0] += s3[3 * (size_t)i]; a[1] += s3[3 * (size_t)i + 1]; a[2] += s3[3 * (size_t)i + 2];
        }
        block_sum_n<3>(a, sm);
        if (threadIdx.x == 0) {
            double* o = part + (((size_t)r * nchunk + ch) * nsub + s) * 3;
            o[0] = a[0]; o[1] = a[1]; o[2] = a[2];
        }
    }
    mag_finish_last(f, gridDim.x * gridDim.y, nsub, nchunk, part, sm);
}

__global__ void mag_final(uint32_t nrep, uint32_t nsub, uint32_t nchunk, const double* __restrict__ part,
                          const double* __restrict__ inv_count, double* __restrict__ out, double* hout) {
    // one block per (replica, sublattice, component): its threads stride over the chunks, then a
    // block sum (fixed order, so the result does not depend on timing)
    __shared__ double sm[32];
    const uint32_t q = blockIdx.x;
    if (q >= nrep * nsub * 3) return;
    const uint32_t comp = q % 3, s = (q / 3) % nsub, r = q / (3 * nsub);
    double acc[1] = {0.0};
    for (uint32_t ch = threadIdx.x; ch < nchunk; ch += blockDim.x)
        acc[0] += part[(((size_t)r * nchunk + ch) * nsub + s) * 3 + comp];
    block_sum_n<1>(acc, sm);
    if (threadIdx.x == 0) {
        const double mq = acc[0] * inv_count[r * nsub + s];
        out[q] = mq;
        if (hout) hout[q] = mq;
    }
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

template <typename R>
void launch_mag_partial(asd_handle* h, dim3 grid, R* const s[3], const float* lx, const float* ly, const float* lz,
                        const MagFinish& f) {
    const uint32_t nsub = h->nsub;
    const uint32_t* sub = h->d_sub_of_atom;
    if (nsub == 1)
        mag_partial_ns<R, 1><<<grid, MAG_BLOCK, 0, h->stream>>>(h->sc, nsub, sub, s[0], s[1], s[2], lx, ly, lz, grid.x,
                                                                h->d_magpart, f);
    else if (nsub == 2)
        mag_partial_ns<R, 2><<<grid, MAG_BLOCK, 0, h->stream>>>(h->sc, nsub, sub, s[0], s[1], s[2], lx, ly, lz, grid.x,
                                                                h->d_magpart, f);
    else if (nsub <= 4)
        mag_partial_ns<R, 4><<<grid, MAG_BLOCK, 0, h->stream>>>(h->sc, nsub, sub, s[0], s[1], s[2], lx, ly, lz, grid.x,
                                                                h->d_magpart, f);
    else
        mag_partial<R><<<grid, MAG_BLOCK, 0, h->stream>>>(h->sc, nsub, sub, s[0], s[1], s[2], lx, ly, lz, grid.x,
                                                          h->d_magpart, f);
}

cudaError_t launch_magnetisation(asd_handle* h, double* hout) {
    const uint32_t nsub = h->nsub;
    uint32_t maxrep = 0;
    for (uint32_t r = 0; r < h->nrep; r++) maxrep = std::max(maxrep, h->h_rep_off[r + 1] - h->h_rep_off[r]);
    const uint32_t nchunk = (maxrep + MAG_CHUNK - 1) / MAG_CHUNK;
    dim3 grid(nchunk ? nchunk : 1, h->nrep);
    const double* inv_count = h->d_inv_count;
    // few outputs: the last partial block forms the means (one launch); else mag_final does
    const uint32_t nq = h->nrep * nsub * 3;
    const MagFinish f{nq <= MAG_FINISH_MAX ? h->d_magcnt : nullptr, h->nrep, inv_count, h->d_mag, hout};
    if (h->p.precision == ASD_FP64_PLAIN) {
        mag_partial_aos<<<grid, MAG_BLOCK, 0, h->stream>>>(h->sc, nsub, h->d_sub_of_atom, h->p_s, grid.x,
                                                           h->d_magpart, f);
    } else if (h->p.precision == ASD_FP32) {
        const bool comp = (h->p.flags & ASD_FLAG_COMPENSATED) != 0;
        launch_mag_partial<float>(h, grid, h->sf, comp ? h->sl[0] : nullptr, comp ? h->sl[1] : nullptr,
                                  comp ? h->sl[2] : nullptr, f);
    } else {
        launch_mag_partial<double>(h, grid, h->sd, nullptr, nullptr, nullptr, f);
    }
    h->launches += 1;
    if (!f.cnt) {
        mag_final<<<nq, 128, 0, h->stream>>>(h->nrep, nsub, grid.x, h->d_magpart, inv_count, h->d_mag, hout);
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

cudaError_t resident_grid(const void* kernel, uint32_t block, size_t smem, uint32_t work, uint32_t* grid) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    static std::mutex mu;
    static std::map<std::tuple<const void*, uint32_t, size_t, int>, uint32_t> cache;
    const auto key = std::make_tuple(kernel, block, smem, dev);
    std::lock_guard<std::mutex> lock(mu);
    auto it = cache.find(key);
    if (it == cache.end()) {
        int per_sm = 0, sms = 0;
        if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, (int)block, smem)) != cudaSuccess)
            return e;
        if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
        it = cache.emplace(key, (uint32_t)std::max(1, per_sm) * (uint32_t)std::max(1, sms)).first;
    }
    *grid = std::max(1u, std::min(work, it->second));
    return cudaSuccess;
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
