// Long-range field, FP32 form: the zero-padded convolution H = IFFT(N_k FFT(M)) in three kernels
// of this library, pruned to the spins' bounding box (replaces the reference's zero / copy /
// cufftExecC2C / CFConv / cufftExecC2C / copy sequence, src/cufields.cu:248-462,
// src/cuda_util.cu:76,97,245,250, and the two 2D cuFFT passes of the earlier pruned path).
//
//  plane_zy_fwd  (one block per box row x and component): real FFT along z of the box rows
//                (the spectrum kept in shared memory, transposed), then the FFT along y of
//                every kz: Y[c][kz][ky-tile][x][j], x and y counted from the box origin.
//  plane_x_conv  (one block per (kz, tile of T ky columns)): its Y tile of all three components
//                and its N_k tile arrive by bulk copy; FFT along x, the 3x3 product with N_k,
//                the inverse FFT along x, box rows only, written back in place by bulk copy.
//  plane_yz_inv  (one block per box row x and component): inverse FFT along y of every kz
//                (box columns only, into shared memory), then the inverse real FFT along z of
//                the box rows into H_r.
//
// Shifting the box to the origin along x and y does not change the cyclic convolution (it
// depends on mesh differences only), and lets every pass skip the zero half of its input and
// the discarded half of its output.  The transforms are unnormalised like cuFFT's: the stage
// kernels multiply the gathered field by 1/P.
#include "fft_dev.cuh"
#include "gather.cuh"
#include <algorithm>
#include <cooperative_groups.h>
#include <cstring>

namespace asd {
namespace {
using namespace fftd;
namespace cg = cooperative_groups;

inline unsigned nbk(size_t n, int b) { return (unsigned)((n + b - 1) / b); }

constexpr uint32_t PT = 8;                 // ky tile width of the spectrum and N_k layouts

struct PlaneArgs {
    uint32_t m0;                     // mesh x (y and z are compile-time in the kernels)
    uint32_t bx0, by0;               // box origin (x, y)
    uint32_t zs, nz;                 // z rows: float2 pairs [zs, zs + nz) hold data, nz <= N/2
    uint32_t bx, by;                 // box extents along x (<= m0/2) and y (<= m1/2)
    uint32_t ntile;                  // ky tiles (m1 / PT)
    uint32_t kzb;                    // kz values per y-pass round (rounds balanced)
    uint32_t scr;                    // scratch (float2) of the z/y passes
    uint32_t nkx;                    // kx rows of the N_k tile: m0 (full) or m0/2 + 1 (kx parity used)
    uint32_t odd;                    // bit q: component q of N_k is odd in kx (N(-kx) = -N(kx))
    size_t P;                        // padded real points
    const float2* twt;               // twiddles: z (N), z split (N + 1), y (m1), x (m0)
    uint32_t twx_off;                // offset of the x twiddles in twt (2N + 1 + m1)
    uint32_t* err;                   // device error bits
    uint32_t wait_once;              // test aid: the bulk-copy wait gives up at once (ASD_FLAG_WAIT_TIMEOUT)
    uint32_t* xq;                    // x-pass item counters (zero between launches): next item, finished blocks
};

constexpr uint32_t ERR_FFT_TIMEOUT = 2u;

__device__ __forceinline__ void bulk_store(void* gdst, const void* ssrc, uint32_t bytes) {
    asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(gdst), "r"(smem_addr(ssrc)),
                 "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void bulk_commit_wait_read() {
    asm volatile("cp.async.bulk.commit_group;" ::: "memory");
    asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
}

// Y element (c, kz, x, ky) in the tiled spectrum layout [c][kz][ky / PT][x][ky % PT].
__device__ __forceinline__ size_t yk_index(const PlaneArgs& A, uint32_t Kz, uint32_t c, uint32_t kz, uint32_t x,
                                           uint32_t ky) {
    return ((((size_t)c * Kz + kz) * A.ntile + (ky / PT)) * A.bx + x) * PT + (ky % PT);
}

// The elements ky = m + R1 q (q < R2) of one (c, kz, x) column that y-pass thread m touches, as a
// pointer and a per-q stride: with R1 a multiple of PT, ky / PT = m / PT + q R1 / PT and
// ky % PT = m % PT, so the column needs one multiply-add per element instead of the full index.
template <int R1>
struct YkCol {
    static_assert(R1 % PT == 0, "the y transform's first factor is a multiple of the ky tile");
    float2* p;
    uint32_t qs;
    __device__ __forceinline__ YkCol(float2* yk, const PlaneArgs& A, uint32_t Kz, uint32_t c, uint32_t kz, uint32_t x,
                                     uint32_t m) {
        const uint32_t tile = A.bx * PT;              // float2 per ky tile of one (c, kz)
        p = yk + ((size_t)c * Kz + kz) * A.ntile * tile + (size_t)x * PT + (m / PT) * tile + (m % PT);
        qs = (R1 / PT) * tile;
    }
    __device__ __forceinline__ float2& operator[](uint32_t q) const { return p[q * qs]; }
};

// Compile-time geometry of the z/y kernels: z rows of N = Z1 Z2 complex points (mesh z = 2N),
// y transforms of M1 = R1 R2 points.  A (component, box row x) is shared by a cluster of CL
// blocks: block `rank` transforms the z rows y in [rank HY, rank HY + HY) (the box's y extent
// is at most M1/2 = CL HY) and the kz in [rank HK, rank HK + HK); the transposed z spectrum of
// its rows, Zs[KZ][LDZ], is read and written across the cluster in distributed shared memory.
// HY is a multiple of R2, so the block owning row t + R2 k of a y pass is k / (HY / R2).
template <int Z1, int Z2, int R1, int R2>
struct ZYGeom {
    static constexpr uint32_t N = Z1 * Z2, KZ = N + 1;
    static constexpr uint32_t TY = 256 / (Z1 > Z2 ? Z1 : Z2);         // z rows per round
    static constexpr uint32_t LD = fft2pass_pitch(N, Z1, Z2);          // z row pitch
    static constexpr uint32_t M1 = R1 * R2;
    static constexpr uint32_t CL = M1 >= 32 ? 4 : 1;
    static constexpr uint32_t HY = M1 >= 32 ? M1 / 8 : M1 / 2;
    static constexpr uint32_t KPB = HY / R2;                           // k values per owner block
    static constexpr uint32_t LDZ = HY | 1u;
    // the real kz = 0 and kz = N planes share one complex y transform (slot 0): N slots in all
    static constexpr uint32_t HK = N / CL;
    static_assert(CL == 1 || HY % R2 == 0, "cluster rows must be whole y-pass columns");
    static_assert(N % CL == 0, "y-pass slots split evenly over the cluster");
};
__host__ __device__ constexpr uint32_t zy_cl(uint32_t m1) { return m1 >= 32 ? 4 : 1; }
__host__ __device__ constexpr uint32_t zy_hy(uint32_t m1) { return m1 >= 32 ? m1 / 8 : m1 / 2; }

// z and y twiddles from the table into shared memory (they are contiguous in both)
__device__ __forceinline__ void copy_tw(float2* dst, const float2* __restrict__ src, uint32_t n) {
    for (uint32_t j = threadIdx.x; j < n; j += blockDim.x) dst[j] = __ldg(src + j);
}

// Split cluster barrier: arrive (release: this thread's earlier shared-memory accesses, local
// and remote, are ordered before it) and wait (acquire).  A block that only has to outlive its
// peers' reads of its shared memory arrives as soon as its own remote reads are done and waits
// at its end, so the wait does not hold its global stores behind a fence.
__device__ __forceinline__ void cluster_arrive() { asm volatile("barrier.cluster.arrive.release.aligned;" ::: "memory"); }
__device__ __forceinline__ void cluster_wait() { asm volatile("barrier.cluster.wait.acquire.aligned;" ::: "memory"); }
// Arrive without ordering any memory access: the start-of-kernel handshake (every block of the
// cluster is running before any block touches a peer's shared memory), waited for just before
// the first remote access.
__device__ __forceinline__ void cluster_arrive_relaxed() { asm volatile("barrier.cluster.arrive.relaxed.aligned;" ::: "memory"); }

// The threads that handle a set of z rows: with warp-local rows (rows_warp_local<Z1, Z2>) warp w
// loads, transforms and stores its own RW = 32 / Z2 rows of the TY, else the whole block
// handles all TY rows.
template <bool WL, uint32_t TY, uint32_t RW>
struct RowGroup {
    uint32_t r0, nr, t, nt;        // first row, rows, thread index in the group, group size
    __device__ __forceinline__ RowGroup() {
        if constexpr (WL) { r0 = (threadIdx.x >> 5) * RW; nr = RW; t = threadIdx.x & 31u; nt = 32; }
        else { r0 = 0; nr = TY; t = threadIdx.x; nt = blockDim.x; }
    }
};

// ---------------------------------------------------------------- forward: z (R2C) then y
template <int Z1, int Z2, int R1, int R2>
__global__ void __launch_bounds__(256, (Z1 > 8 ? 3 : 4)) plane_zy_fwd(const float* __restrict__ mr, float2* __restrict__ yk,
                                                       const PlaneArgs A) {
    using G = ZYGeom<Z1, Z2, R1, R2>;
    constexpr uint32_t N = G::N, KZ = G::KZ, TY = G::TY, LD = G::LD, M1 = G::M1;
    constexpr uint32_t CL = G::CL, HY = G::HY, LDZ = G::LDZ, HK = G::HK, KPB = G::KPB;
    constexpr bool WLZ = rows_warp_local<Z1, Z2>();    // z rows warp-local
    constexpr bool WLY = R1 == R2 && 32 % R1 == 0;     // a kz slot's y passes inside one warp
    extern __shared__ __align__(16) float2 sm[];
    cg::cluster_group cl = cg::this_cluster();
    float2* Zs = sm;                                   // [KZ][LDZ]: this block's z rows
    float2* scr = Zs + (size_t)KZ * LDZ;               // z rows [TY][LD] | y exchange [kzb][R1][R2+1]
    float2* twz = scr + A.scr;                         // N + (N + 1) z twiddles
    float2* twy = twz + 2 * N + 1;                     // M1 y twiddles
    const uint32_t rank = cl.block_rank();
    const uint32_t xl = blockIdx.x / CL, c = blockIdx.y, x = A.bx0 + xl;
    copy_tw(twz, A.twt, 2 * N + 1 + M1);               // set-up data: before the wait
    pdl_enter();
    __syncthreads();
    // the box row x of component c from its y = by0 row on: pair n of row yl at rowx[yl N + n]
    const float2* rowx = reinterpret_cast<const float2*>(mr + (size_t)c * A.P) + A.zs + ((size_t)x * M1 + A.by0) * N;
    const float2* ws = twz + N;
    const uint32_t ry0 = rank * HY, ry1 = min(A.by, ry0 + HY);
    const RowGroup<WLZ, TY, 32 / Z2> g;
    for (uint32_t y0 = ry0; y0 < ry1; y0 += TY) {
        group_sync<WLZ>();
        // rows shifted to the z pair zs; pairs n >= N/2 are zero and not read by the pruned pass
        for (uint32_t e = g.t; e < g.nr * (N / 2); e += g.nt) {
            const uint32_t r = g.r0 + e / (N / 2), n = e % (N / 2), yl = y0 + r;
            float2 v = make_float2(0.f, 0.f);
            if (yl < ry1 && n < A.nz) v = rowx[yl * N + n];
            scr[r * LD + n] = v;
        }
        group_sync<WLZ>();
        fft2pass<Z1, Z2, false, true, false>(scr, LD, twz, TY);
        // X_k and X_{N-k} from the same two values Z_k, Z_{N-k}
        constexpr uint32_t NH = N / 2 + 1;
        auto split = [&](uint32_t r, uint32_t k) {
            const float2 zk = scr[r * LD + (k & (N - 1))], zm = scr[r * LD + ((N - k) & (N - 1))];
            float2* zc = Zs + (y0 + r - ry0);
            zc[k * LDZ] = r2c_split(zk, zm, ws[k]);
            if (k != N / 2) zc[(N - k) * LDZ] = r2c_split(zm, zk, ws[N - k]);
        };
        if constexpr (WLZ) {
            // the warp's own rows one by one, k across the lanes (no division by NH)
            for (uint32_t rr = 0; rr < g.nr; rr++)
                if (y0 + g.r0 + rr < ry1)
                    for (uint32_t k = g.t; k < NH; k += 32) split(g.r0 + rr, k);
        } else {
            for (uint32_t e = g.t; e < NH * g.nr; e += g.nt) {
                const uint32_t r = g.r0 + e / NH, k = e % NH;
                if (y0 + r < ry1) split(r, k);
            }
        }
    }
    cl.sync();                                         // every block's rows are in its Zs
    const float2* zb[CL];
#pragma unroll
    for (uint32_t o = 0; o < CL; o++) zb[o] = cl.map_shared_rank(Zs, o);
    // y transforms of this block's slots: slot s >= 1 is the plane kz = s; slot 0 carries the two
    // real planes kz = 0 and kz = N as P = X_0 + i X_N, whose transform C gives
    // F_0(ky) = (C(ky) + conj C(-ky)) / 2 and F_N(ky) = (C(ky) - conj C(-ky)) / 2i
    float2* cpk = scr + A.kzb * R1 * (R2 + 1);         // [M1]: C of slot 0
    const uint32_t s_lo = rank * HK, s_hi = s_lo + HK;
    for (uint32_t s0 = s_lo; s0 < s_hi; s0 += A.kzb) {
        {
            const uint32_t kzl = threadIdx.x / R2, t = threadIdx.x % R2, sl = s0 + kzl;
            if (kzl < A.kzb && sl < s_hi) {
                float2 v[R1];
#pragma unroll
                for (int k = 0; k < R1 / 2; k++) {     // rows y >= M1/2 are zero
                    const uint32_t yy = t + R2 * k;
                    constexpr uint32_t kpb = CL == 1 ? R1 : KPB;
                    const uint32_t off = t + R2 * (k % kpb);
                    v[k] = make_float2(0.f, 0.f);
                    if (yy < A.by) {
                        if (sl) v[k] = zb[k / kpb][sl * LDZ + off];
                        else v[k] = make_float2(zb[k / kpb][off].x, zb[k / kpb][N * LDZ + off].x);
                    }
                }
                dftp<R1, false, true, false>(v);
#pragma unroll
                for (int m = 1; m < R1; m++) v[m] = cmul(v[m], twy[t * m]);
#pragma unroll
                for (int m = 0; m < R1; m++) scr[(kzl * R1 + m) * (R2 + 1) + t] = v[m];
            }
        }
        // the last round has read every peer row this block needs: arrive on the cluster
        // barrier whose wait ends the kernel
        if (s0 + A.kzb >= s_hi) cluster_arrive();
        group_sync<WLY>();
        const bool packed = s0 == 0;                   // block-uniform: slot 0 is in this round
        {
            const uint32_t kzl = threadIdx.x / R1, m = threadIdx.x % R1, sl = s0 + kzl;
            if (kzl < A.kzb && sl < s_hi) {
                float2 u[R2];
#pragma unroll
                for (int t = 0; t < R2; t++) u[t] = scr[(kzl * R1 + m) * (R2 + 1) + t];
                dft<R2, false>(u);
                if (sl) {
                    if constexpr (R1 % PT == 0) {
                        const YkCol<R1> col(yk, A, KZ, c, sl, xl, m);
#pragma unroll
                        for (int q = 0; q < R2; q++) col[q] = u[q];
                    } else {
#pragma unroll
                        for (int q = 0; q < R2; q++) yk[yk_index(A, KZ, c, sl, xl, m + R1 * q)] = u[q];
                    }
                } else {
#pragma unroll
                    for (int q = 0; q < R2; q++) cpk[m + R1 * q] = u[q];
                }
            }
        }
        if (packed) {
            // slot 0's pass-2 threads are the first R1 of the block: warp 0 (WLY) splits C
            group_sync<WLY>();
            if (!WLY || threadIdx.x < 32)
                for (uint32_t ky = threadIdx.x; ky < M1; ky += WLY ? 32u : blockDim.x) {
                    const float2 a = cpk[ky], b = cpk[(M1 - ky) & (M1 - 1)];
                    yk[yk_index(A, KZ, c, 0, xl, ky)] = make_float2(0.5f * (a.x + b.x), 0.5f * (a.y - b.y));
                    yk[yk_index(A, KZ, c, N, xl, ky)] = make_float2(0.5f * (a.y + b.y), -0.5f * (a.x - b.x));
                }
        }
        group_sync<WLY>();
    }
    cluster_wait();                                    // no block retires while a peer reads its Zs
}

// ---------------------------------------------------------------- x, N_k product, inverse x
// Shared memory: Ys [3][bx][PT] (input), Ns (N_k tile: 6 x nkx x PT floats or 9 x M0 x PT
// float2), E (exchange, R1 x (R2 PT + 8) float2), twx [M0].  A real N_k whose every component is
// even or odd in kx is stored for kx <= M0/2 only (nkx = M0/2 + 1 rows); the rows kx > M0/2 are
// read at M0 - kx with the component's sign.
//
// Persistent: block b starts with the (kz, tile) item b (item = kz * ntile + tile) and takes
// each further item from a counter (blocks that started late, behind the previous kernel's
// last blocks, take fewer).  The next item's spectrum is copied into Ys as soon as the forward
// transform has read it, and its N_k tile into Ns once the product has read that, so both
// copies run under the product and the inverse transform; the inverse writes its box rows
// straight to global memory.  One mbarrier, one phase per item.  The last block to finish
// zeroes the counters for the next launch.
template <int R1, int R2, bool CPLX>
__global__ void __launch_bounds__(PT * R1, CPLX ? 1 : 3) plane_x_conv(float2* __restrict__ yk,
                                                                      const void* __restrict__ nkt, const uint32_t Kz,
                                                                      const PlaneArgs A) {
    extern __shared__ __align__(16) unsigned char smraw[];
    __shared__ __align__(8) uint64_t bar;
    constexpr uint32_t T = PT;
    constexpr uint32_t M0 = R1 * R2;
    constexpr uint32_t NQ = CPLX ? 9 : 6;
    constexpr uint32_t NB = CPLX ? 8 : 4;             // bytes per N_k component value
    constexpr uint32_t EP = R2 * T + 8;               // exchange pitch per m (padded: no bank conflicts)
    const uint32_t nitems = A.ntile * Kz;
    float2* Ys = reinterpret_cast<float2*>(smraw);
    const uint32_t ys_bytes = 3u * A.bx * T * 8u;
    unsigned char* Nsb = smraw + ((ys_bytes + 15u) & ~15u);
    const uint32_t ns_bytes = NQ * A.nkx * T * NB;
    float2* E = reinterpret_cast<float2*>(Nsb + ns_bytes);
    float2* twx = E + R1 * EP;
    const uint32_t tid = threadIdx.x, j = tid % T, r = tid / T;
    const uint32_t slab = A.bx * T;                   // float2 per (c, kz, tile) slab
    // slab of component c of item it: [c][kz][tile] with it = kz * ntile + tile
    auto slab_of = [&](uint32_t it, uint32_t c) {
        return yk + ((size_t)c * Kz * A.ntile + it) * slab;
    };
    auto nk_of = [&](uint32_t it) { return static_cast<const unsigned char*>(nkt) + (size_t)it * ns_bytes; };
    const uint32_t polls = A.wait_once ? 0u : STAGE_WAIT_POLLS;
    __shared__ uint32_t next_item;
    uint32_t item = blockIdx.x;                       // < nitems: the grid is at most the item count
    // the N_k tile and the twiddles are set-up data: copied before the wait, the spectrum after
    if (tid == 0) {
        mbar_init(&bar, 1);
        mbar_arrive_expect_tx(&bar, ys_bytes + ns_bytes);
        bulk_copy_stream(Nsb, nk_of(item), ns_bytes, &bar);
    }
    copy_tw(twx, A.twt + A.twx_off, M0);
    pdl_enter();
    if (tid == 0)
        for (uint32_t c = 0; c < 3; c++) bulk_copy_stream(Ys + c * slab, slab_of(item, c), slab * 8u, &bar);
    __syncthreads();
    for (uint32_t phase = 0; item < nitems; phase ^= 1u) {
        if (__syncthreads_or(!mbar_wait_parity_bounded(&bar, phase, polls))) {
            // the copies did not land in time for some thread: the whole block flags it, leaves
            // this item untransformed, and stops taking items once the copies into shared memory
            // have finished (bounded again)
            if (tid == 0) atomicOr(A.err, ERR_FFT_TIMEOUT);
            mbar_wait_parity_bounded(&bar, phase, STAGE_WAIT_POLLS);
            break;
        }
        // forward x transform of the three components; thread (j, m) keeps X[c][m + R1 q]
        float2 X[3][R2];
#pragma unroll
        for (int c = 0; c < 3; c++) {
            if (r < R2) {
                const uint32_t t = r;
                float2 v[R1];
#pragma unroll
                for (int k = 0; k < R1 / 2; k++) {         // rows x >= M0/2 are zero
                    const uint32_t xx = t + R2 * k;
                    v[k] = xx < A.bx ? Ys[(c * A.bx + xx) * T + j] : make_float2(0.f, 0.f);
                }
                dftp<R1, false, true, false>(v);
#pragma unroll
                for (int m = 1; m < R1; m++) v[m] = cmul(v[m], twx[t * m]);
#pragma unroll
                for (int m = 0; m < R1; m++) E[m * EP + t * T + j] = v[m];
            }
            __syncthreads();
            {
                const uint32_t m = r;
#pragma unroll
                for (int t = 0; t < R2; t++) X[c][t] = E[m * EP + t * T + j];
                dft<R2, false>(X[c]);
            }
            __syncthreads();
        }
        // the forward transform has read Ys (the barrier that ends its last component): the next
        // item's spectrum goes there, the expected bytes counting its N_k tile too
        if (tid == 0) {
            const uint32_t nx = gridDim.x + atomicAdd(A.xq, 1u);
            next_item = nx;
            if (nx < nitems) {
                fence_async_smem();
                mbar_arrive_expect_tx(&bar, ys_bytes + ns_bytes);
                for (uint32_t c = 0; c < 3; c++) bulk_copy_stream(Ys + c * slab, slab_of(nx, c), slab * 8u, &bar);
            }
        }
        // H_k = N_k M_k at kx = m + R1 q
        {
            const uint32_t m = r;
#pragma unroll
            for (int q = 0; q < R2; q++) {
                const uint32_t kx = m + R1 * q;
                const float2 a = X[0][q], b = X[1][q], cc = X[2][q];
                if constexpr (!CPLX) {
                    const float* Ns = reinterpret_cast<const float*>(Nsb);
                    const bool mir = kx >= A.nkx;                  // kx > M0/2 in the half layout
                    const uint32_t row = mir ? M0 - kx : kx, nk = A.nkx;
                    const uint32_t neg = mir ? A.odd : 0u;
                    float n6[6];
#pragma unroll
                    for (int q6 = 0; q6 < 6; q6++) {
                        const float v = Ns[(q6 * nk + row) * T + j];
                        n6[q6] = (neg >> q6) & 1u ? -v : v;
                    }
                    X[0][q] = make_float2(n6[0] * a.x + n6[1] * b.x + n6[2] * cc.x, n6[0] * a.y + n6[1] * b.y + n6[2] * cc.y);
                    X[1][q] = make_float2(n6[1] * a.x + n6[3] * b.x + n6[4] * cc.x, n6[1] * a.y + n6[3] * b.y + n6[4] * cc.y);
                    X[2][q] = make_float2(n6[2] * a.x + n6[4] * b.x + n6[5] * cc.x, n6[2] * a.y + n6[4] * b.y + n6[5] * cc.y);
                } else {
                    const float2* Ns = reinterpret_cast<const float2*>(Nsb);
                    const float2 v[3] = {a, b, cc};
#pragma unroll
                    for (int al = 0; al < 3; al++) {
                        float2 o = make_float2(0.f, 0.f);
#pragma unroll
                        for (int be = 0; be < 3; be++) o = cadd(o, cmul(Ns[((3 * al + be) * M0 + kx) * T + j], v[be]));
                        X[al][q] = o;
                    }
                }
            }
        }
        __syncthreads();                              // every thread has read its N_k values
        const uint32_t next = next_item;
        if (next < nitems && tid == 0) {
            fence_async_smem();
            bulk_copy_stream(Nsb, nk_of(next), ns_bytes, &bar);
        }
        // inverse x transform, box rows only, straight to the item's slabs in global memory
#pragma unroll
        for (int c = 0; c < 3; c++) {
            {
                const uint32_t m = r;
                dft<R2, true>(X[c]);
#pragma unroll
                for (int t = 0; t < R2; t++) E[m * EP + t * T + j] = t ? cmulc(X[c][t], twx[t * m]) : X[c][t];
            }
            __syncthreads();
            if (r < R2) {
                const uint32_t t = r;
                float2 w[R1];
#pragma unroll
                for (int m = 0; m < R1; m++) w[m] = E[m * EP + t * T + j];
                dftp<R1, true, false, true>(w);        // the rows x < M0/2 only
                float2* gy = slab_of(item, c);
#pragma unroll
                for (int k = 0; k < R1 / 2; k++) {
                    const uint32_t xx = t + R2 * k;
                    if (xx < A.bx) gy[xx * T + j] = w[k];
                }
            }
            __syncthreads();
        }
        item = next;
    }
    // every block has taken its last item once all have finished: the last one rearms the counters
    if (tid == 0) {
        uint32_t done;
        asm volatile("atom.add.acq_rel.gpu.u32 %0, [%1], 1;" : "=r"(done) : "l"(A.xq + 1) : "memory");
        if (done == gridDim.x - 1) { A.xq[0] = 0u; A.xq[1] = 0u; }
    }
}

// ---------------------------------------------------------------- inverse: y then z (C2R)
// 4 blocks per SM (64 registers, no spill) where the z rows are at most 64 points (8 × 8), 3
// for the longer rows, whose passes spill at 64; like the forward kernel.
template <int Z1, int Z2, int R1, int R2>
__global__ void __launch_bounds__(256, (Z1 > 8 ? 3 : 4)) plane_yz_inv(const float2* __restrict__ yk, float* __restrict__ hr,
                                                       const PlaneArgs A) {
    using G = ZYGeom<Z1, Z2, R1, R2>;
    constexpr uint32_t N = G::N, KZ = G::KZ, TY = G::TY, LD = G::LD, M1 = G::M1;
    constexpr uint32_t CL = G::CL, HY = G::HY, LDZ = G::LDZ, HK = G::HK, KPB = G::KPB;
    constexpr bool WLZ = rows_warp_local<Z1, Z2>();
    constexpr bool WLY = R1 == R2 && 32 % R1 == 0;
    extern __shared__ __align__(16) float2 sm[];
    cg::cluster_group cl = cg::this_cluster();
    float2* Zs = sm;
    float2* scr = Zs + (size_t)KZ * LDZ;
    float2* twz = scr + A.scr;
    float2* twy = twz + 2 * N + 1;
    const uint32_t rank = cl.block_rank();
    const uint32_t xl = blockIdx.x / CL, c = blockIdx.y, x = A.bx0 + xl;
    copy_tw(twz, A.twt, 2 * N + 1 + M1);               // set-up data: before the wait
    cluster_arrive_relaxed();
    float2* zb[CL];
#pragma unroll
    for (uint32_t o = 0; o < CL; o++) zb[o] = cl.map_shared_rank(Zs, o);
    pdl_enter();
    __syncthreads();
    // inverse y of this block's slots (slot 0: D = G_0 + i G_N of the real planes kz = 0 and N,
    // whose inverse is g_0 + i g_N); every box row's value goes to the Zs of the block owning it
    const uint32_t s_lo = rank * HK, s_hi = s_lo + HK;
    for (uint32_t s0 = s_lo; s0 < s_hi; s0 += A.kzb) {
        {
            const uint32_t kzl = threadIdx.x / R1, m = threadIdx.x % R1, sl = s0 + kzl;
            if (kzl < A.kzb && sl < s_hi) {
                float2 u[R2];
                if (sl) {
                    // (the full index per element: with a per-q stride the loads are hoisted
                    // together and the kernel no longer fits its register cap)
#pragma unroll
                    for (int q = 0; q < R2; q++) u[q] = yk[yk_index(A, KZ, c, sl, xl, m + R1 * q)];
                } else {
#pragma unroll
                    for (int q = 0; q < R2; q++) {
                        const float2 g0 = yk[yk_index(A, KZ, c, 0, xl, m + R1 * q)];
                        const float2 gn = yk[yk_index(A, KZ, c, N, xl, m + R1 * q)];
                        u[q] = make_float2(g0.x - gn.y, g0.y + gn.x);
                    }
                }
                dft<R2, true>(u);
#pragma unroll
                for (int t = 0; t < R2; t++)
                    scr[(kzl * R1 + m) * (R2 + 1) + t] = t ? cmulc(u[t], twy[t * m]) : u[t];
            }
        }
        if (s0 == s_lo) cluster_wait();                // every peer is running: remote stores may start
        group_sync<WLY>();
        {
            const uint32_t kzl = threadIdx.x / R2, t = threadIdx.x % R2, sl = s0 + kzl;
            if (kzl < A.kzb && sl < s_hi) {
                float2 w[R1];
#pragma unroll
                for (int m = 0; m < R1; m++) w[m] = scr[(kzl * R1 + m) * (R2 + 1) + t];
                dftp<R1, true, false, true>(w);        // the rows y < M1/2 only
#pragma unroll
                for (int k = 0; k < R1 / 2; k++) {
                    const uint32_t yy = t + R2 * k;
                    constexpr uint32_t kpb = CL == 1 ? R1 : KPB;
                    const uint32_t off = t + R2 * (k % kpb);
                    if (yy < A.by) {
                        if (sl) {
                            zb[k / kpb][sl * LDZ + off] = w[k];
                        } else {
                            zb[k / kpb][off] = make_float2(w[k].x, 0.f);
                            zb[k / kpb][N * LDZ + off] = make_float2(w[k].y, 0.f);
                        }
                    }
                }
            }
        }
        group_sync<WLY>();
    }
    cl.sync();                                         // every row of every block's Zs is written
    const float2* ws = twz + N;
    float2* out0 = reinterpret_cast<float2*>(hr + (size_t)c * A.P) + A.zs;
    const uint32_t ry0 = rank * HY, ry1 = min(A.by, ry0 + HY);
    const RowGroup<WLZ, TY, 32 / Z2> g;
    float2* outx = out0 + ((size_t)x * M1 + A.by0) * N;   // pair n of row yl at outx[yl N + n]
    constexpr uint32_t half = N / 2, nh = half + 1;
    // Z'_k and Z'_{N-k} of row r from X_k, X_{N-k}, in place
    auto pre = [&](uint32_t r, uint32_t k) {
        const float2 xk = scr[r * LD + k], xm = scr[r * LD + (N - k)];
        const float2 zk = c2r_pre(xk, xm, ws[k]);
        if (k != 0 && k != half) scr[r * LD + (N - k)] = c2r_pre(xm, xk, ws[N - k]);
        scr[r * LD + k] = zk;
    };
    for (uint32_t y0 = ry0; y0 < ry1; y0 += TY) {
        if constexpr (WLZ) {
            // the warp's own rows one by one, k across the lanes (no division by KZ or nh)
            for (uint32_t rr = 0; rr < g.nr; rr++) {
                const uint32_t r = g.r0 + rr, yl = y0 + r;
                for (uint32_t k = g.t; k < KZ; k += 32)
                    scr[r * LD + k] = yl < ry1 ? Zs[k * LDZ + (yl - ry0)] : make_float2(0.f, 0.f);
            }
            __syncwarp();
            for (uint32_t rr = 0; rr < g.nr; rr++)
                for (uint32_t k = g.t; k < nh; k += 32) pre(g.r0 + rr, k);
        } else {
            for (uint32_t e = g.t; e < KZ * g.nr; e += g.nt) {
                const uint32_t r = g.r0 + e / KZ, k = e % KZ, yl = y0 + r;
                scr[r * LD + k] = yl < ry1 ? Zs[k * LDZ + (yl - ry0)] : make_float2(0.f, 0.f);
            }
            __syncthreads();
            for (uint32_t e = g.t; e < g.nr * nh; e += g.nt) {
                const uint32_t r = g.r0 + e / nh, k = e % nh;
                pre(r, k);
            }
        }
        group_sync<WLZ>();
        fft2pass<Z1, Z2, true, false, true>(scr, LD, twz, TY);   // pairs n < N/2 only
        for (uint32_t e = g.t; e < g.nr * (N / 2); e += g.nt) {
            const uint32_t r = g.r0 + e / (N / 2), n = e % (N / 2), yl = y0 + r;
            if (yl >= ry1 || n >= A.nz) continue;
            outx[yl * N + n] = scr[r * LD + n];
        }
        group_sync<WLZ>();
    }
}

// ---------------------------------------------------------------- N_k in the tiled layout
// From the FP64 half spectrum z[q][x][y][kz] (cuFFT D2Z of N_r) to
// nkt[kz][tile][q][kx][j] (real: float, kx < nkx; complex: float2, kx < m0), ky = tile T + j.
__global__ void nk_tile_real(size_t Pk, uint32_t nkx, uint32_t m1, uint32_t Kz, uint32_t T,
                             const double2* __restrict__ z, float* __restrict__ out, size_t total) {
    const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= total) return;
    const uint32_t j = (uint32_t)(e % T);
    size_t rest = e / T;
    const uint32_t kx = (uint32_t)(rest % nkx); rest /= nkx;
    const uint32_t q = (uint32_t)(rest % 6); rest /= 6;
    const uint32_t tile = (uint32_t)(rest % (m1 / T));
    const uint32_t kz = (uint32_t)(rest / (m1 / T));
    const uint32_t ky = tile * T + j;
    out[e] = (float)z[(size_t)q * Pk + ((size_t)kx * m1 + ky) * Kz + kz].x;
}

__global__ void nk_tile_cplx(size_t Pk, uint32_t m0, uint32_t m1, uint32_t Kz, uint32_t T,
                             const double2* __restrict__ z, float2* __restrict__ out) {
    const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= Pk * 9) return;
    const uint32_t j = (uint32_t)(e % T);
    size_t rest = e / T;
    const uint32_t kx = (uint32_t)(rest % m0); rest /= m0;
    const uint32_t q = (uint32_t)(rest % 9); rest /= 9;
    const uint32_t tile = (uint32_t)(rest % (m1 / T));
    const uint32_t kz = (uint32_t)(rest / (m1 / T));
    const uint32_t ky = tile * T + j;
    const double2 v = z[(size_t)q * Pk + ((size_t)kx * m1 + ky) * Kz + kz];
    out[e] = make_float2((float)v.x, (float)v.y);
}

// Largest |N(kx) - N(m0-kx)| and |N(kx) + N(m0-kx)| (real parts) of each of the 6 components:
// dev[2q] (even test), dev[2q+1] (odd test); non-negative doubles compare like their bits.
__global__ void nk_parity_x(size_t Pk, uint32_t m0, uint32_t m1, uint32_t Kz, const double2* __restrict__ z,
                            unsigned long long* dev) {
    double de[6] = {0, 0, 0, 0, 0, 0}, dodd[6] = {0, 0, 0, 0, 0, 0};
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < Pk; i += (size_t)gridDim.x * blockDim.x) {
        const uint32_t kx = (uint32_t)(i / ((size_t)m1 * Kz));
        const size_t rest = i % ((size_t)m1 * Kz);
        const size_t mi = (size_t)((m0 - kx) % m0) * m1 * Kz + rest;
#pragma unroll
        for (int q = 0; q < 6; q++) {
            const double a = z[(size_t)q * Pk + i].x, b = z[(size_t)q * Pk + mi].x;
            de[q] = fmax(de[q], fabs(a - b));
            dodd[q] = fmax(dodd[q], fabs(a + b));
        }
    }
#pragma unroll
    for (int q = 0; q < 6; q++) {
        for (int o = 16; o > 0; o >>= 1) {
            de[q] = fmax(de[q], __shfl_xor_sync(0xffffffffu, de[q], o));
            dodd[q] = fmax(dodd[q], __shfl_xor_sync(0xffffffffu, dodd[q], o));
        }
        if ((threadIdx.x & 31) == 0) {
            atomicMax(dev + 2 * q, (unsigned long long)__double_as_longlong(de[q]));
            atomicMax(dev + 2 * q + 1, (unsigned long long)__double_as_longlong(dodd[q]));
        }
    }
}

// Twiddle table of the plane kernels, rounded from double precision: exp(-2 pi i j / N) (j < N),
// exp(-i pi k / N) (k <= N), exp(-2 pi i j / m1) (j < m1), exp(-2 pi i j / m0) (j < m0).
__global__ void tw_table_k(uint32_t N, uint32_t m1, uint32_t m0, float2* __restrict__ t) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t n1 = 2 * N + 1, n2 = n1 + m1, n3 = n2 + m0;
    if (i >= n3) return;
    double a;
    if (i < N) a = -2.0 * (double)i / (double)N;
    else if (i < n1) a = -(double)(i - N) / (double)N;
    else if (i < n2) a = -2.0 * (double)(i - n1) / (double)m1;
    else a = -2.0 * (double)(i - n2) / (double)m0;
    double sn, cs;
    sincospi(a, &sn, &cs);
    t[i] = make_float2((float)cs, (float)sn);
}

uint32_t ilog2(uint32_t v) {
    uint32_t l = 0;
    while ((1u << l) < v) l++;
    return l;
}

PlaneArgs plane_args(const LongRange& L) {
    PlaneArgs A{};
    const uint32_t m1 = L.mesh[1], N = L.mesh[2] / 2, Kz = N + 1;
    const int z1 = split_r1((int)N), z2 = split_r2((int)N);
    const uint32_t TY = 256 / (uint32_t)std::max(z1, z2);
    const uint32_t LD = fft2pass_pitch(N, (uint32_t)z1, (uint32_t)z2);
    A.m0 = L.mesh[0];
    A.bx0 = L.box0[0]; A.by0 = L.box0[1];
    A.zs = L.box0[2] / 2;
    A.nz = L.box1[2] / 2 - A.zs + 1;
    A.bx = L.box1[0] - L.box0[0] + 1;
    A.by = L.box1[1] - L.box0[1] + 1;
    A.ntile = m1 / PT;
    const uint32_t CL = zy_cl(m1), hk = N / CL;       // y-pass slots per block
    const int r1 = split_r1((int)m1), r2 = split_r2((int)m1);
    const uint32_t kzmax = 256 / (uint32_t)std::max(r1, r2);
    const uint32_t rounds = (hk + kzmax - 1) / kzmax;
    A.kzb = (hk + rounds - 1) / rounds;                // equal rounds of at most kzmax kz
    A.scr = std::max<uint32_t>(TY * LD, A.kzb * (uint32_t)r1 * (uint32_t)(r2 + 1) + m1);
    A.nkx = L.nk_nkx ? L.nk_nkx : A.m0;
    A.odd = L.nk_odd;
    A.P = L.P;
    A.twt = L.twt;
    A.twx_off = 2 * N + 1 + m1;
    A.xq = L.xq;
    return A;
}

size_t zy_smem(const LongRange& L, const PlaneArgs& A) {
    const uint32_t N = L.mesh[2] / 2, ldz = zy_hy(L.mesh[1]) | 1u;
    return sizeof(float2) * ((size_t)(N + 1) * ldz + A.scr + 2 * N + 1 + L.mesh[1]);
}

size_t xconv_smem(const PlaneArgs& A, bool cplx) {
    const size_t ys = ((3u * A.bx * PT * 8u) + 15u) & ~(size_t)15u;
    const size_t ns = cplx ? (size_t)9 * A.m0 * PT * 8 : (size_t)6 * A.nkx * PT * 4;
    const uint32_t r1 = (uint32_t)split_r1((int)A.m0), r2 = (uint32_t)split_r2((int)A.m0);
    return ys + ns + sizeof(float2) * ((size_t)r1 * (r2 * PT + 8) + A.m0);
}

template <typename K>
cudaError_t set_smem(K kern, size_t bytes) {
    return raise_smem_limit(reinterpret_cast<const void*>(kern), bytes);
}

// z split x y split instantiations: z N in {4..256}, y mesh in {8..256}
#define ASD_ZY_CASES(M, Z1, Z2)                                                                           \
    switch (M) {                                                                                          \
    case 8: ASD_ZY_CALL(Z1, Z2, 4, 2) break;                                                              \
    case 16: ASD_ZY_CALL(Z1, Z2, 4, 4) break;                                                             \
    case 32: ASD_ZY_CALL(Z1, Z2, 8, 4) break;                                                             \
    case 64: ASD_ZY_CALL(Z1, Z2, 8, 8) break;                                                             \
    case 128: ASD_ZY_CALL(Z1, Z2, 16, 8) break;                                                           \
    case 256: ASD_ZY_CALL(Z1, Z2, 16, 16) break;                                                          \
    default: return cudaErrorInvalidValue;                                                                \
    }

#define ASD_Z_CASES(N, M)                                                                                 \
    switch (N) {                                                                                          \
    case 4: ASD_ZY_CASES(M, 2, 2) break;                                                                  \
    case 8: ASD_ZY_CASES(M, 4, 2) break;                                                                  \
    case 16: ASD_ZY_CASES(M, 4, 4) break;                                                                 \
    case 32: ASD_ZY_CASES(M, 8, 4) break;                                                                 \
    case 64: ASD_ZY_CASES(M, 8, 8) break;                                                                 \
    case 128: ASD_ZY_CASES(M, 16, 8) break;                                                               \
    case 256: ASD_ZY_CASES(M, 16, 16) break;                                                              \
    default: return cudaErrorInvalidValue;                                                                \
    }

cudaError_t run_zy(const LongRange& L, const PlaneArgs& A, bool inverse, cudaStream_t st, bool pdl) {
    const size_t sm = zy_smem(L, A);
    const uint32_t CL = zy_cl(L.mesh[1]);
    const dim3 grid(A.bx * CL, 3);
    const float* mr = L.r;
    float* hr = L.r + 3 * L.P;
    float2* yk = L.yk;
    const float2* ykc = L.yk;
    cudaError_t e = cudaSuccess;
#define ASD_ZY_CALL(Z1, Z2, R1, R2)                                                                       \
    if (inverse) {                                                                                        \
        if ((e = set_smem(plane_yz_inv<Z1, Z2, R1, R2>, sm)) != cudaSuccess) return e;                    \
        e = launch_step_kernel(plane_yz_inv<Z1, Z2, R1, R2>, grid, dim3(256), sm, st, CL, pdl, ykc, hr, A); \
    } else {                                                                                              \
        if ((e = set_smem(plane_zy_fwd<Z1, Z2, R1, R2>, sm)) != cudaSuccess) return e;                    \
        e = launch_step_kernel(plane_zy_fwd<Z1, Z2, R1, R2>, grid, dim3(256), sm, st, CL, pdl, mr, yk, A);  \
    }
    ASD_Z_CASES(L.mesh[2] / 2, L.mesh[1])
#undef ASD_ZY_CALL
    return e != cudaSuccess ? e : cudaGetLastError();
}

template <int R1, int R2, bool CPLX>
cudaError_t run_xconv_k(const LongRange& L, const PlaneArgs& A, cudaStream_t st, bool pdl) {
    const uint32_t Kz = L.mesh[2] / 2 + 1;
    const size_t sm = xconv_smem(A, CPLX);
    const uint32_t block = PT * R1;
    cudaError_t e;
    uint32_t grid = 0;
    if ((e = set_smem(plane_x_conv<R1, R2, CPLX>, sm)) != cudaSuccess) return e;
    if ((e = resident_grid(reinterpret_cast<const void*>(plane_x_conv<R1, R2, CPLX>), block, sm, A.ntile * Kz, &grid)) !=
        cudaSuccess)
        return e;
    const void* nkt = L.nkt;
    e = launch_step_kernel(plane_x_conv<R1, R2, CPLX>, dim3(grid), dim3(block), sm, st, 1, pdl, L.yk, nkt, Kz, A);
    return e != cudaSuccess ? e : cudaGetLastError();
}

template <int R1, int R2>
cudaError_t run_xconv_t(const LongRange& L, const PlaneArgs& A, bool cplx, cudaStream_t st, bool pdl) {
    return cplx ? run_xconv_k<R1, R2, true>(L, A, st, pdl) : run_xconv_k<R1, R2, false>(L, A, st, pdl);
}

cudaError_t run_xconv(const LongRange& L, const PlaneArgs& A, bool cplx, cudaStream_t st, bool pdl) {
    switch (A.m0) {
    case 4: return run_xconv_t<2, 2>(L, A, cplx, st, pdl);
    case 8: return run_xconv_t<4, 2>(L, A, cplx, st, pdl);
    case 16: return run_xconv_t<4, 4>(L, A, cplx, st, pdl);
    case 32: return run_xconv_t<8, 4>(L, A, cplx, st, pdl);
    case 64: return run_xconv_t<8, 8>(L, A, cplx, st, pdl);
    case 128: return run_xconv_t<16, 8>(L, A, cplx, st, pdl);
    case 256: return run_xconv_t<16, 16>(L, A, cplx, st, pdl);
    default: return cudaErrorInvalidValue;
    }
}

}  // namespace

// The plane path applies when every mesh axis is a power of two (x 4..256, y 8..256, z 8..512:
// the register transforms' sizes), the spins' box spans at most half the mesh along x and y and
// its z pairs fit in half a row (so every forward pass skips the zero half of its input and
// every inverse pass forms only the box half of its output), and the shared memory fits.
bool plane_path_fits(const LongRange& L, bool cplx) {
    auto p2 = [](uint32_t v) { return v >= 2 && (v & (v - 1)) == 0; };
    if (!p2(L.mesh[0]) || !p2(L.mesh[1]) || !p2(L.mesh[2])) return false;
    if (L.mesh[0] < 4 || L.mesh[0] > 256 || L.mesh[1] < 8 || L.mesh[1] > 256 || L.mesh[2] < 8 || L.mesh[2] > 512)
        return false;
    LongRange t = L;
    t.nk_nkx = L.mesh[0];                              // the larger N_k tile bounds the shared memory
    const PlaneArgs A = plane_args(t);
    const uint32_t N = L.mesh[2] / 2;
    if (2 * A.bx > L.mesh[0] || 2 * A.by > L.mesh[1] || 2 * A.nz > N) return false;
    return zy_smem(L, A) <= 200 * 1024 && xconv_smem(A, cplx) <= 220 * 1024;
}

size_t plane_spectrum_elems(const LongRange& L) {
    const PlaneArgs A = plane_args(L);
    return 3 * (size_t)(L.mesh[2] / 2 + 1) * A.ntile * A.bx * PT;
}

// Tiled N_k from the FP64 half spectrum z[ncomp][m0][m1][Kz] (device); allocates L.nkt.  A real
// N_k whose 6 components are each even or odd in kx (the point dipole and symmetric exchange on
// a lattice with mirror symmetry in x) keeps only kx <= m0/2.
cudaError_t build_nk_tiles(asd_handle* h, const double2* z, uint32_t ncomp, bool cplx) {
    LongRange& L = h->lr;
    const uint32_t Kz = L.mesh[2] / 2 + 1;
    const size_t Pk = (size_t)L.mesh[0] * L.mesh[1] * Kz;
    cudaError_t e;
    if (!cplx) {
        unsigned long long* dev = nullptr;
        if ((e = cudaMalloc(&dev, 12 * sizeof(unsigned long long))) != cudaSuccess) return e;
        cudaMemsetAsync(dev, 0, 12 * sizeof(unsigned long long), h->stream);
        nk_parity_x<<<std::min<unsigned>(nbk(Pk, 256), 148 * 8), 256, 0, h->stream>>>(Pk, L.mesh[0], L.mesh[1], Kz,
                                                                                         z, dev);
        unsigned long long hb[12];
        cudaMemcpyAsync(hb, dev, sizeof(hb), cudaMemcpyDeviceToHost, h->stream);
        e = cudaStreamSynchronize(h->stream);
        cudaFree(dev);
        if (e != cudaSuccess) return e;
        double d[12], big = 0.0;
        for (int q = 0; q < 12; q++) { memcpy(&d[q], &hb[q], 8); big = std::max(big, d[q]); }
        // tolerance: FP64 transform rounding relative to the spectrum's scale (big >= max |N_k|)
        const double tol = 1e-11 * big;
        uint32_t odd = 0;
        bool ok = L.mesh[0] >= 2;
        for (int q = 0; q < 6 && ok; q++) {
            if (d[2 * q] <= tol) continue;                 // even
            if (d[2 * q + 1] <= tol) { odd |= 1u << q; continue; }
            ok = false;
        }
        L.nk_nkx = ok ? L.mesh[0] / 2 + 1 : L.mesh[0];
        L.nk_odd = ok ? odd : 0;
        const size_t total = (size_t)6 * L.nk_nkx * L.mesh[1] * Kz;
        float* t = nullptr;
        if ((e = cudaMalloc(&t, sizeof(float) * total)) != cudaSuccess) return e;
        nk_tile_real<<<nbk(total, 256), 256, 0, h->stream>>>(Pk, L.nk_nkx, L.mesh[1], Kz, PT, z, t, total);
        L.nkt = t;
    } else {
        float2* t = nullptr;
        if ((e = cudaMalloc(&t, sizeof(float2) * 9 * Pk)) != cudaSuccess) return e;
        (void)ncomp;
        L.nk_nkx = L.mesh[0];
        L.nk_odd = 0;
        nk_tile_cplx<<<nbk(9 * Pk, 256), 256, 0, h->stream>>>(Pk, L.mesh[0], L.mesh[1], Kz, PT, z, t);
        L.nkt = t;
    }
    return cudaGetLastError();
}

// Twiddle table of the plane kernels (allocates L.twt) and the x pass's item counters (L.xq,
// zeroed).
cudaError_t build_plane_twiddles(asd_handle* h) {
    LongRange& L = h->lr;
    const uint32_t N = L.mesh[2] / 2, n = 2 * N + 1 + L.mesh[1] + L.mesh[0];
    cudaError_t e = cudaMalloc(&L.twt, sizeof(float2) * n);
    if (e != cudaSuccess) return e;
    if ((e = cudaMalloc(&L.xq, 2 * sizeof(uint32_t))) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(L.xq, 0, 2 * sizeof(uint32_t), h->stream)) != cudaSuccess) return e;
    tw_table_k<<<nbk(n, 256), 256, 0, h->stream>>>(N, L.mesh[1], L.mesh[0], L.twt);
    return cudaGetLastError();
}

// M_r -> H_r through the three plane kernels.
// Algorithmic bytes per launch: the box rows of M_r or H_r (3 components, the z pairs that hold
// data), the spectrum (3 x (N+1) x m1 x box x float2) read and/or written once, N_k read once.
cudaError_t launch_lr_planes(asd_handle* h) {
    LongRange& L = h->lr;
    PlaneArgs A = plane_args(L);
    A.err = h->d_err;
    A.wait_once = (h->p.flags & ASD_FLAG_WAIT_TIMEOUT) ? 1u : 0u;
    const bool cplx = !(L.ncomp == 6 && L.nk_real);
    const double rows = 3.0 * A.bx * A.by * 2.0 * A.nz * 4.0;
    const double spec = 8.0 * (double)plane_spectrum_elems(L);
    const double nkb = cplx ? 9.0 * 8.0 * L.mesh[0] * L.mesh[1] * (L.mesh[2] / 2 + 1)
                            : 6.0 * 4.0 * A.nkx * L.mesh[1] * (L.mesh[2] / 2 + 1);
    cudaError_t e;
    timer_begin(h);
    const bool pdl = step_pdl(h);
    if ((e = run_zy(L, A, false, h->stream, pdl)) != cudaSuccess) return e;
    timer_end(h, "plane_zy_fwd (z R2C + y FFT)", rows + spec);
    timer_begin(h);
    if ((e = run_xconv(L, A, cplx, h->stream, pdl)) != cudaSuccess) return e;
    timer_end(h, "plane_x_conv (x FFT, N_k product, inverse x FFT)", 2.0 * spec + nkb);
    timer_begin(h);
    if ((e = run_zy(L, A, true, h->stream, pdl)) != cudaSuccess) return e;
    timer_end(h, "plane_yz_inv (inverse y FFT + z C2R)", spec + rows);
    h->launches += 3;
    return cudaSuccess;
}

}  // namespace asd
