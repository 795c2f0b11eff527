// Exchange-field gathers shared by the stage kernels and the field read-back.
//
// Two device layouts per storage scheme:
//  * streamed values: each matrix entry carries its tensor (SELL-32 float4/float2 packing or
//    component-major doubles; DIA component-major values);
//  * typed: each entry carries a small tensor id into a table of the distinct tensors of the
//    matrix (the reference builds every value from a per-(sublattice pair, shell) tensor,
//    src/exch_unitcell.cpp:399, so a lattice has few); SELL entries pack (column, id) into
//    one 32-bit word, DIA stores one id byte per (diagonal, row); id 0 is the zero tensor.
//    The table is staged in shared memory, component-major [c][ntypes].
#pragma once
#include "internal.h"

namespace asd {

template <typename R>
struct Vec3 { R* p[3]; };
template <typename R>
struct CVec3 { const R* p[3]; };

template <typename T>
__device__ __forceinline__ T ldcs(const T* p) { return __ldcs(p); }

// ---- bulk (TMA) staging of a block's typed SELL words into shared memory
// One thread arms an mbarrier with the byte count and issues one cp.async.bulk global->shared
// copy (16-byte aligned source, destination and size); every thread later waits on the
// barrier's phase 0 with a bounded number of try_wait polls.
__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// L2 prefetch of a 16-byte-aligned range (a hint: no completion to wait for).
__device__ __forceinline__ void bulk_prefetch_l2(const void* src, uint32_t bytes) {
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(src), "r"(bytes) : "memory");
}

// The one arrival of the barrier's phase, announcing the bytes all copies will deliver.
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
}

// Streamed data (read once per launch): evict-first in L2.
__device__ __forceinline__ void bulk_copy_stream(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    uint64_t policy;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(policy));
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], %4;" ::"r"(
            smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar)), "l"(policy)
        : "memory");
}

// Reused data (neighbour spins other blocks read too): default L2 policy.
__device__ __forceinline__ void bulk_copy(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_addr(dst)),
                 "l"(src), "r"(bytes), "r"(smem_addr(bar))
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait for phase 0: false after `limit` polls (each poll may suspend the warp briefly).
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t limit) {
    for (uint32_t it = 0; it < limit; it++)
        if (mbar_try_wait(bar, 0)) return true;
    return false;
}
// Orders this thread's earlier generic-proxy shared-memory accesses (and, after a block barrier,
// the block's) before its later bulk copies into the same memory.
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// The same for phase `parity` of a barrier that completes once per item of a loop.
__device__ __forceinline__ bool mbar_wait_parity_bounded(uint64_t* bar, uint32_t parity, uint32_t limit) {
    for (uint32_t it = 0; it < limit; it++)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}
constexpr uint32_t STAGE_WAIT_POLLS = 1u << 22;
constexpr uint32_t ERR_STAGE_TIMEOUT = 1u;

// Copy the tensor table (ncomp x ntypes) into shared memory; all threads of the block take part.
template <typename R>
__device__ __forceinline__ void load_table(const R* __restrict__ tab, uint32_t count, R* smem) {
    for (uint32_t q = threadIdx.x; q < count; q += blockDim.x) smem[q] = tab[q];
    __syncthreads();
}

template <typename R>
__device__ __forceinline__ const R* table_of(const SellDev& m) {
    if constexpr (sizeof(R) == 4) return m.tab_f; else return m.tab_d;
}
template <typename R>
__device__ __forceinline__ const R* table_of(const DiaDev& m) {
    if constexpr (sizeof(R) == 4) return m.tab_f; else return m.tab_d;
}

// Table row stride: 4 (xx, yy, zz, 0) for the diagonal form, 12 (9 + 3 zeros) for full tensors.
template <bool FULL>
__host__ __device__ constexpr uint32_t table_stride() { return FULL ? 12u : 4u; }

// h += J_t (x, y, z) for tensor id t of the shared-memory table (type-major rows).
template <typename R, bool FULL>
__device__ __forceinline__ void accumulate_typed(const R* tab, uint32_t t, R x, R y, R z, R h[3]) {
    if constexpr (sizeof(R) == 4) {
        const float4* T = reinterpret_cast<const float4*>(tab) + t * (FULL ? 3 : 1);
        const float4 a = T[0];
        if (!FULL) {
            h[0] = fmaf(a.x, x, h[0]);
            h[1] = fmaf(a.y, y, h[1]);
            h[2] = fmaf(a.z, z, h[2]);
        } else {
            const float4 b = T[1];
            const float4 c = T[2];
            h[0] = fmaf(a.x, x, fmaf(a.y, y, fmaf(a.z, z, h[0])));
            h[1] = fmaf(a.w, x, fmaf(b.x, y, fmaf(b.y, z, h[1])));
            h[2] = fmaf(b.z, x, fmaf(b.w, y, fmaf(c.x, z, h[2])));
        }
    } else {
        const R* T = tab + t * table_stride<FULL>();
        if (!FULL) {
            h[0] += T[0] * x; h[1] += T[1] * y; h[2] += T[2] * z;
        } else {
            h[0] += T[0] * x + T[1] * y + T[2] * z;
            h[1] += T[3] * x + T[4] * y + T[5] * z;
            h[2] += T[6] * x + T[7] * y + T[8] * z;
        }
    }
}

// h += sum over the row's entries of J_e S_col(e), SELL-32 layout (one warp per slice).
template <typename R, bool FULL>
__device__ __forceinline__ void gather_sell(const SellDev& m, uint32_t i, const CVec3<R>& s, const R* tab, R h[3],
                                            const uint32_t* staged = nullptr, uint32_t wbase = 0,
                                            const R* sspin = nullptr, const uint16_t* staged16 = nullptr) {
    const uint32_t sl = i >> 5, lane = i & 31u;
    const uint32_t p0 = __ldg(m.slice_ptr + sl), p1 = __ldg(m.slice_ptr + sl + 1);
    if (m.typed && staged16 && sspin) {
        // 16-bit words: slot | id << lbits into the staged neighbour spins [3][spin_slots]
        const uint32_t mask = (1u << m.lbits) - 1u, cb = m.lbits, ns = m.spin_slots;
#pragma unroll 4
        for (uint32_t e = p0 - wbase + lane; e < p1 - wbase; e += 32) {
            const uint32_t w = staged16[e];
            const uint32_t j = w & mask, t = w >> cb;
            accumulate_typed<R, FULL>(tab, t, sspin[j], sspin[ns + j], sspin[2 * ns + j], h);
        }
        return;
    }
    if (m.typed && staged && sspin) {
        // words carry block-local slots into the staged neighbour spins [3][spin_slots]
        const uint32_t mask = (1u << m.colbits) - 1u, cb = m.colbits, ns = m.spin_slots;
#pragma unroll 4
        for (uint32_t e = p0 - wbase + lane; e < p1 - wbase; e += 32) {
            const uint32_t w = staged[e];
            const uint32_t j = w & mask, t = w >> cb;
            accumulate_typed<R, FULL>(tab, t, sspin[j], sspin[ns + j], sspin[2 * ns + j], h);
        }
        return;
    }
    if (m.typed && staged) {
        // this block's words are in shared memory, indexed from the block's first entry
        const uint32_t mask = (1u << m.colbits) - 1u, cb = m.colbits;
#pragma unroll 4
        for (uint32_t e = p0 - wbase + lane; e < p1 - wbase; e += 32) {
            const uint32_t w = staged[e];
            const uint32_t j = w & mask, t = w >> cb;
            const R x = __ldg(s.p[0] + j), y = __ldg(s.p[1] + j), z = __ldg(s.p[2] + j);
            accumulate_typed<R, FULL>(tab, t, x, y, z, h);
        }
        return;
    }
    if (m.typed) {
        const uint32_t mask = (1u << m.colbits) - 1u, cb = m.colbits;
#pragma unroll 4
        for (uint32_t e = p0 + lane; e < p1; e += 32) {
            const uint32_t w = ldcs(m.typed + e);
            const uint32_t j = w & mask, t = w >> cb;
            const R x = __ldg(s.p[0] + j), y = __ldg(s.p[1] + j), z = __ldg(s.p[2] + j);
            accumulate_typed<R, FULL>(tab, t, x, y, z, h);
        }
        return;
    }
    if constexpr (sizeof(R) == 4) {
#pragma unroll 2
        for (uint32_t e = p0 + lane; e < p1; e += 32) {
            const float4 a = ldcs(m.a + e);
            const int j = __float_as_int(a.x);
            const float x = __ldg(s.p[0] + j), y = __ldg(s.p[1] + j), z = __ldg(s.p[2] + j);
            if (!FULL) {
                h[0] = fmaf(a.y, x, h[0]);
                h[1] = fmaf(a.z, y, h[1]);
                h[2] = fmaf(a.w, z, h[2]);
            } else {
                const float4 b = ldcs(m.b + e);
                const float2 c = ldcs(m.c + e);
                h[0] = fmaf(a.y, x, fmaf(a.z, y, fmaf(a.w, z, h[0])));
                h[1] = fmaf(b.x, x, fmaf(b.y, y, fmaf(b.z, z, h[1])));
                h[2] = fmaf(b.w, x, fmaf(c.x, y, fmaf(c.y, z, h[2])));
            }
        }
    } else {
        const uint32_t E = m.entries;
        for (uint32_t e = p0 + lane; e < p1; e += 32) {
            const int j = ldcs(m.col + e);
            const double x = __ldg(s.p[0] + j), y = __ldg(s.p[1] + j), z = __ldg(s.p[2] + j);
            const double* v = m.val;
            if (!FULL) {
                h[0] += ldcs(v + e) * x;
                h[1] += ldcs(v + E + e) * y;
                h[2] += ldcs(v + 2 * (size_t)E + e) * z;
            } else {
                h[0] += ldcs(v + e) * x + ldcs(v + E + e) * y + ldcs(v + 2 * (size_t)E + e) * z;
                h[1] += ldcs(v + 3 * (size_t)E + e) * x + ldcs(v + 4 * (size_t)E + e) * y + ldcs(v + 5 * (size_t)E + e) * z;
                h[2] += ldcs(v + 6 * (size_t)E + e) * x + ldcs(v + 7 * (size_t)E + e) * y + ldcs(v + 8 * (size_t)E + e) * z;
            }
        }
    }
}

// h += sum over diagonals d with 0 <= i+off[d] < n of J_{d,i} S_{i+off[d]}, row-aligned DIA.
template <typename R, bool FULL>
__device__ __forceinline__ void gather_dia(const DiaDev& m, uint32_t n, uint32_t i, const CVec3<R>& s, const R* tab,
                                           R h[3]) {
    // the warp walks its tile's active diagonals (warp-uniform list)
    const uint32_t k0 = __ldg(m.tile_ptr + (i >> 5)), k1 = __ldg(m.tile_ptr + (i >> 5) + 1);
    if (m.dtype) {
        for (uint32_t k = k0; k < k1; k++) {
            const uint32_t d = __ldg(m.tile_diag + k);
            const int64_t col = (int64_t)i + __ldg(m.off + d);
            if (col < 0 || col >= (int64_t)n) continue;
            const uint32_t t = ldcs(m.dtype + (size_t)d * n + i);
            if (t == 0) continue;
            const R x = __ldg(s.p[0] + col), y = __ldg(s.p[1] + col), z = __ldg(s.p[2] + col);
            accumulate_typed<R, FULL>(tab, t, x, y, z, h);
        }
        return;
    }
    const size_t ND = (size_t)m.ndiag * n;
    const R* v;
    if constexpr (sizeof(R) == 4) v = m.valf; else v = m.vald;
    for (uint32_t k = k0; k < k1; k++) {
        const uint32_t d = __ldg(m.tile_diag + k);
        const int64_t col = (int64_t)i + __ldg(m.off + d);
        if (col < 0 || col >= (int64_t)n) continue;
        const size_t a = (size_t)d * n + i;
        const R x = __ldg(s.p[0] + col), y = __ldg(s.p[1] + col), z = __ldg(s.p[2] + col);
        if (!FULL) {
            h[0] += ldcs(v + a) * x;
            h[1] += ldcs(v + ND + a) * y;
            h[2] += ldcs(v + 2 * ND + a) * z;
        } else {
            h[0] += ldcs(v + a) * x + ldcs(v + ND + a) * y + ldcs(v + 2 * ND + a) * z;
            h[1] += ldcs(v + 3 * ND + a) * x + ldcs(v + 4 * ND + a) * y + ldcs(v + 5 * ND + a) * z;
            h[2] += ldcs(v + 6 * ND + a) * x + ldcs(v + 7 * ND + a) * y + ldcs(v + 8 * ND + a) * z;
        }
    }
}

}  // namespace asd
