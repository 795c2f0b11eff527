// Long-range (dipolar / FFT-exchange) field on the zero-padded mesh.
//
// FP32 form: the padded real spin arrays M_r[3][P] (zero outside the spin
// sites, written once) are transformed R2C to the half spectrum, multiplied
// point-wise by N_k in place, and transformed C2R into H_r[3][P]; the stage
// kernels gather H_r/P at the spin sites and scatter their output spins into
// M_r, so no zeroing or copy kernels run per evaluation (the reference zeroes
// and copies four full-size complex arrays per evaluation:
// src/cuda.cu:47-60, src/cufields.cu:248-462).
//
// N_k is built on the device in FP64 (D2Z of the FP64 real-space matrix) and
// stored in FP32: 6 real components when N_r is symmetric and even (point
// dipole + symmetric exchange), else 9 complex.
#include "internal.h"
#include <algorithm>
#include <cstdio>

namespace asd {
namespace {

inline unsigned nb(size_t n, int b) { return (unsigned)((n + b - 1) / b); }

// H_k[a] = sum_b N_k[a][b] M_k[b] at one half-spectrum point, in place.
// Real symmetric N_k: components xx, xy, xz, yy, yz, zz.
__global__ void kconv6r(size_t Pk, const float* __restrict__ nk, float2* __restrict__ m) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= Pk) return;
    const float2 x = m[i], y = m[Pk + i], z = m[2 * Pk + i];
    const float nxx = __ldcs(nk + i), nxy = __ldcs(nk + Pk + i), nxz = __ldcs(nk + 2 * Pk + i);
    const float nyy = __ldcs(nk + 3 * Pk + i), nyz = __ldcs(nk + 4 * Pk + i), nzz = __ldcs(nk + 5 * Pk + i);
    m[i] = make_float2(nxx * x.x + nxy * y.x + nxz * z.x, nxx * x.y + nxy * y.y + nxz * z.y);
    m[Pk + i] = make_float2(nxy * x.x + nyy * y.x + nyz * z.x, nxy * x.y + nyy * y.y + nyz * z.y);
    m[2 * Pk + i] = make_float2(nxz * x.x + nyz * y.x + nzz * z.x, nxz * x.y + nyz * y.y + nzz * z.y);
}

// General N_k: 9 complex components (a,b) row-major.
__global__ void kconv9c(size_t Pk, const float2* __restrict__ nk, float2* __restrict__ m) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= Pk) return;
    const float2 v[3] = {m[i], m[Pk + i], m[2 * Pk + i]};
    float2 o[3];
#pragma unroll
    for (int a = 0; a < 3; a++) {
        float re = 0.f, im = 0.f;
#pragma unroll
        for (int b = 0; b < 3; b++) {
            const float2 nn = __ldcs(nk + (size_t)(3 * a + b) * Pk + i);
            re += nn.x * v[b].x - nn.y * v[b].y;
            im += nn.x * v[b].y + nn.y * v[b].x;
        }
        o[a] = make_float2(re, im);
    }
    m[i] = o[0]; m[Pk + i] = o[1]; m[2 * Pk + i] = o[2];
}

template <typename R>
__global__ void scatter_k(uint32_t n, size_t P, const R* __restrict__ sx, const R* __restrict__ sy,
                          const R* __restrict__ sz, const float* __restrict__ w, const uint32_t* __restrict__ idx,
                          float* __restrict__ mr) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t m = idx[i];
    const float wv = w[i];
    mr[m] = (float)sx[i] * wv;
    mr[P + m] = (float)sy[i] * wv;
    mr[2 * P + m] = (float)sz[i] * wv;
}

// Largest |Re| and |Im| of the FP64 half spectrum (non-negative doubles order like their bits):
// grid-stride per thread, warp and block maxima, one atomic per block.
__global__ void nk_extent(size_t m, const double2* __restrict__ z, unsigned long long* mx) {
    __shared__ double sre[32], sim[32];
    double re = 0.0, im = 0.0;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (size_t)gridDim.x * blockDim.x) {
        re = fmax(re, fabs(z[i].x));
        im = fmax(im, fabs(z[i].y));
    }
    for (int o = 16; o > 0; o >>= 1) {
        re = fmax(re, __shfl_xor_sync(0xffffffffu, re, o));
        im = fmax(im, __shfl_xor_sync(0xffffffffu, im, o));
    }
    if ((threadIdx.x & 31) == 0) { sre[threadIdx.x >> 5] = re; sim[threadIdx.x >> 5] = im; }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (uint32_t w = 1; w < blockDim.x / 32; w++) { re = fmax(re, sre[w]); im = fmax(im, sim[w]); }
        atomicMax(mx, (unsigned long long)__double_as_longlong(re));
        atomicMax(mx + 1, (unsigned long long)__double_as_longlong(im));
    }
}

__global__ void nk_pack_real(size_t Pk, uint32_t ncomp, const double2* __restrict__ z, const int* comp_map,
                             float* __restrict__ out, int* __restrict__ dummy) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= Pk * ncomp) return;
    (void)comp_map; (void)dummy;
    out[i] = (float)z[i].x;
}

__global__ void nk_pack_cplx(size_t m, const double2* __restrict__ z, float2* __restrict__ out) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    out[i] = make_float2((float)z[i].x, (float)z[i].y);
}

__global__ void real_to_cplx(size_t m, const double* __restrict__ r, double2* __restrict__ z) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    z[i] = make_double2(r[i], 0.0);
}

// ---- pruned transform along z: M = mesh[2] = 2N real points per row, N complex points
// z_n = x_2n + i x_2n+1 per row.  N = N1 * N2 in {4, ..., 256} runs as two register passes
// (Cooley-Tukey: N1-point DFTs of the N2 strided subsequences, twiddle, N2-point DFTs); other
// sizes use a radix-2 pass per stage in shared memory.
struct ZPass {
    uint32_t m0, m1, mz, N, logN, Kz, TY, logTY;
    uint32_t bx0, by0, by1, bz0, bz1;   // box: x from bx0 (grid y), y in [by0, by1], z in [bz0, bz1]
    size_t P, Pk;                       // padded real points; spectrum points Kz*m0*m1
};

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// tw[j] = exp(-2 pi i j / N) for j < N, then the split twiddles ws[k] = exp(-i pi k / N) for
// k <= N at tw + N.
__device__ __forceinline__ void load_twiddles(float2* tw, uint32_t N) {
    for (uint32_t j = threadIdx.x; j < N; j += blockDim.x) {
        float sn, cs;
        sincospif(-2.0f * (float)j / (float)N, &sn, &cs);
        tw[j] = make_float2(cs, sn);
    }
    for (uint32_t k = threadIdx.x; k <= N; k += blockDim.x) {
        float sn, cs;
        sincospif(-(float)k / (float)N, &sn, &cs);
        tw[N + k] = make_float2(cs, sn);
    }
}

// In-place radix-2 FFT of TY rows of N points (stride ld) already in bit-reversed order.
template <bool INV>
__device__ __forceinline__ void smem_fft(float2* s, uint32_t ld, const float2* tw, const ZPass& A) {
    const uint32_t half_n = A.N / 2, lhn = A.logN - 1;
    for (uint32_t len = 2, lg = 1; len <= A.N; len <<= 1, lg++) {
        const uint32_t half = len >> 1, step = A.N >> lg;
        for (uint32_t b = threadIdx.x; b < A.TY * half_n; b += blockDim.x) {
            const uint32_t r = b >> lhn, q = b & (half_n - 1);
            const uint32_t g = q >> (lg - 1), j = q & (half - 1);
            const uint32_t i0 = r * ld + g * len + j, i1 = i0 + half;
            float2 w = tw[j * step];
            if (INV) w.y = -w.y;
            const float2 u = s[i0], v = cmul(s[i1], w);
            s[i0] = make_float2(u.x + v.x, u.y + v.y);
            s[i1] = make_float2(u.x - v.x, u.y - v.y);
        }
        __syncthreads();
    }
}

template <int R>
__device__ __forceinline__ constexpr int brev_c(int k) {
    int r = 0;
    for (int b = 1, o = R >> 1; b < R; b <<= 1, o >>= 1)
        if (k & b) r |= o;
    return r;
}

// R-point DFT in registers (radix-2, decimation in time); the twiddle of a length-len
// butterfly is w_len^j = tw[j N / len].
template <int R, bool INV>
__device__ __forceinline__ void reg_dft(float2 (&v)[R], const float2* tw, uint32_t N) {
    float2 a[R];
#pragma unroll
    for (int k = 0; k < R; k++) a[brev_c<R>(k)] = v[k];
#pragma unroll
    for (int len = 2; len <= R; len <<= 1) {
        const uint32_t step = N / (uint32_t)len;
#pragma unroll
        for (int g = 0; g < R; g += len)
#pragma unroll
            for (int j = 0; j < len / 2; j++) {
                float2 t = a[g + j + len / 2];
                if (j != 0) {
                    float2 w = tw[j * step];
                    if (INV) w.y = -w.y;
                    t = cmul(t, w);
                }
                const float2 u = a[g + j];
                a[g + j] = make_float2(u.x + t.x, u.y + t.y);
                a[g + j + len / 2] = make_float2(u.x - t.x, u.y - t.y);
            }
    }
#pragma unroll
    for (int k = 0; k < R; k++) v[k] = a[k];
}

// N = N1 N2 point DFT of TY rows (natural order in and out, in place), TY * max(N1, N2) <= 256:
// X[m + N1 q] = sum_t w_N2^{t q} w_N^{t m} sum_k w_N1^{k m} z[t + N2 k].
template <int N1, int N2, bool INV>
__device__ __forceinline__ void fft2pass(float2* s, uint32_t ld, const float2* tw, uint32_t TY) {
    constexpr uint32_t N = N1 * N2;
    {
        const uint32_t it = threadIdx.x, r = it / N2, t = it % N2;
        const bool act = it < TY * N2;
        float2 v[N1];
        if (act) {
#pragma unroll
            for (int k = 0; k < N1; k++) v[k] = s[r * ld + t + N2 * k];
            reg_dft<N1, INV>(v, tw, N);
#pragma unroll
            for (int m = 1; m < N1; m++) {
                float2 w = tw[t * m];
                if (INV) w.y = -w.y;
                v[m] = cmul(v[m], w);
            }
        }
        __syncthreads();
        if (act) {
#pragma unroll
            for (int m = 0; m < N1; m++) s[r * ld + m * N2 + t] = v[m];
        }
        __syncthreads();
    }
    {
        const uint32_t it = threadIdx.x, r = it / N1, m = it % N1;
        const bool act = it < TY * N1;
        float2 u[N2];
        if (act) {
#pragma unroll
            for (int t = 0; t < N2; t++) u[t] = s[r * ld + m * N2 + t];
            reg_dft<N2, INV>(u, tw, N);
        }
        __syncthreads();
        if (act) {
#pragma unroll
            for (int q = 0; q < N2; q++) s[r * ld + m + N1 * q] = u[q];
        }
        __syncthreads();
    }
}

// M_r rows (c, x, y in the box) -> half spectrum k1[c][kz][x][y], kz = 0..N.
// grid: (y tiles of TY rows, box rows in x, 3 components).  N1 = 0: radix-2 fallback.
template <int N1, int N2>
__global__ void zpass_r2c(const float* __restrict__ mr, float2* __restrict__ k1, const ZPass A) {
    extern __shared__ float2 zs[];
    const uint32_t ld = A.N + 2;
    float2* tw = zs + A.TY * ld;
    const uint32_t c = blockIdx.z, x = A.bx0 + blockIdx.y, y0 = A.by0 + blockIdx.x * A.TY;
    load_twiddles(tw, A.N);
    const float2* row0 = reinterpret_cast<const float2*>(mr + (size_t)c * A.P);
    for (uint32_t e = threadIdx.x; e < A.TY * A.N; e += blockDim.x) {
        const uint32_t r = e >> A.logN, n = e & (A.N - 1), y = y0 + r;
        float2 v = make_float2(0.f, 0.f);
        if (y <= A.by1 && 2 * n + 1 >= A.bz0 && 2 * n <= A.bz1)
            v = row0[(((size_t)x * A.m1 + y) * A.mz) / 2 + n];
        if constexpr (N1 > 0) zs[r * ld + n] = v;
        else zs[r * ld + (__brev(n) >> (32 - A.logN))] = v;
    }
    __syncthreads();
    if constexpr (N1 > 0) fft2pass<N1, N2, false>(zs, ld, tw, A.TY);
    else smem_fft<false>(zs, ld, tw, A);
    // X_k = E_k + w^k O_k, E = (Z_k + conj Z_{N-k}) / 2, O = -i (Z_k - conj Z_{N-k}) / 2, w = e^{-i pi / N}
    const float2* ws = tw + A.N;
    for (uint32_t e = threadIdx.x; e < (A.N + 1) * A.TY; e += blockDim.x) {
        const uint32_t k = e >> A.logTY, r = e & (A.TY - 1), y = y0 + r;
        if (y > A.by1) continue;
        const float2 zk = zs[r * ld + (k & (A.N - 1))], zm = zs[r * ld + ((A.N - k) & (A.N - 1))];
        const float2 E = make_float2(0.5f * (zk.x + zm.x), 0.5f * (zk.y - zm.y));
        const float2 O = make_float2(0.5f * (zk.y + zm.y), -0.5f * (zk.x - zm.x));
        const float2 wo = cmul(ws[k], O);
        k1[(((size_t)c * A.Kz + k) * A.m0 + x) * A.m1 + y] = make_float2(E.x + wo.x, E.y + wo.y);
    }
}

// Z'_k = (X_k + conj X_{N-k}) + i e^{+i pi k / N} (X_k - conj X_{N-k}): twice the spectrum of
// z_n = x_2n + i x_2n+1, so that the unnormalised inverse gives 2N x (cuFFT's C2R scaling).
__device__ __forceinline__ float2 c2r_pre(float2 xk, float2 xm, float2 wsk) {
    const float2 sp = make_float2(xk.x + xm.x, xk.y - xm.y);
    const float2 df = make_float2(xk.x - xm.x, xk.y + xm.y);
    const float2 t = cmul(make_float2(wsk.x, -wsk.y), df);
    return make_float2(sp.x - t.y, sp.y + t.x);
}

// Spectrum k2[c][kz][x][y] of the box rows -> H_r rows, unnormalised like cuFFT's C2R.
template <int N1, int N2>
__global__ void zpass_c2r(const float2* __restrict__ k2, float* __restrict__ hr, const ZPass A) {
    extern __shared__ float2 zs[];
    const uint32_t ld = A.N + 2;
    const uint32_t c = blockIdx.z, x = A.bx0 + blockIdx.y, y0 = A.by0 + blockIdx.x * A.TY;
    float2* s = zs;                          // [TY][N+2]: spectrum rows, then Z' in place
    float2* xs2 = zs + A.TY * ld;            // fallback only: [TY][N+1] bit-reversed Z'
    float2* tw = N1 > 0 ? xs2 : xs2 + A.TY * (A.N + 1);
    load_twiddles(tw, A.N);
    for (uint32_t e = threadIdx.x; e < (A.N + 1) * A.TY; e += blockDim.x) {
        const uint32_t k = e >> A.logTY, r = e & (A.TY - 1), y = y0 + r;
        s[r * ld + k] = y <= A.by1 ? k2[(((size_t)c * A.Kz + k) * A.m0 + x) * A.m1 + y] : make_float2(0.f, 0.f);
    }
    __syncthreads();
    const float2* ws = tw + A.N;
    if constexpr (N1 > 0) {
        // pairwise in place: thread (r, k) for k in [0, N/2] writes Z'_k and Z'_{N-k}
        const uint32_t half = A.N / 2, nh = half + 1;
        for (uint32_t e = threadIdx.x; e < A.TY * nh; e += blockDim.x) {
            const uint32_t r = e / nh, k = e % nh;
            const float2 xk = s[r * ld + k], xm = s[r * ld + (A.N - k)];
            const float2 zk = c2r_pre(xk, xm, ws[k]);
            if (k != 0 && k != half) s[r * ld + (A.N - k)] = c2r_pre(xm, xk, ws[A.N - k]);
            s[r * ld + k] = zk;
        }
        __syncthreads();
        fft2pass<N1, N2, true>(s, ld, tw, A.TY);
    } else {
        const uint32_t ld2 = A.N + 1;
        for (uint32_t e = threadIdx.x; e < A.TY * A.N; e += blockDim.x) {
            const uint32_t r = e >> A.logN, k = e & (A.N - 1);
            xs2[r * ld2 + (__brev(k) >> (32 - A.logN))] = c2r_pre(s[r * ld + k], s[r * ld + (A.N - k)], ws[k]);
        }
        __syncthreads();
        smem_fft<true>(xs2, ld2, tw, A);
        s = xs2;
    }
    const uint32_t lds = N1 > 0 ? ld : A.N + 1;
    float2* out0 = reinterpret_cast<float2*>(hr + (size_t)c * A.P);
    for (uint32_t e = threadIdx.x; e < A.TY * A.N; e += blockDim.x) {
        const uint32_t r = e >> A.logN, n = e & (A.N - 1), y = y0 + r;
        if (y > A.by1 || 2 * n + 1 < A.bz0 || 2 * n > A.bz1) continue;
        out0[(((size_t)x * A.m1 + y) * A.mz) / 2 + n] = s[r * lds + n];
    }
}

// [comp][x][y][kz] -> [comp][kz][x][y] for the pruned spectrum layout.
template <typename T>
__global__ void permute_nk(size_t Pk, uint32_t ncomp, uint32_t m0, uint32_t m1, uint32_t Kz, const T* __restrict__ in,
                           T* __restrict__ out) {
    const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= Pk * ncomp) return;
    const size_t q = e / Pk, i = e % Pk;
    const uint32_t kz = (uint32_t)(i % Kz);
    const size_t xy = i / Kz;                       // x * m1 + y
    out[q * Pk + (size_t)kz * m0 * m1 + xy] = in[e];
}

// (N1, N2) of the two-pass transform for N complex points, (0, 0) for the radix-2 fallback.
void zpass_split(uint32_t N, int* n1, int* n2) {
    static const int tab[][3] = {{4, 2, 2}, {8, 4, 2}, {16, 4, 4}, {32, 8, 4}, {64, 8, 8}, {128, 16, 8}, {256, 16, 16}};
    *n1 = 0; *n2 = 0;
    for (const auto& t : tab)
        if ((uint32_t)t[0] == N) { *n1 = t[1]; *n2 = t[2]; }
}

ZPass zpass_args(const LongRange& L) {
    ZPass A{};
    A.m0 = L.mesh[0]; A.m1 = L.mesh[1]; A.mz = L.mesh[2]; A.N = A.mz / 2;
    A.logN = 0;
    while ((1u << A.logN) < A.N) A.logN++;
    A.Kz = A.N + 1;
    int n1, n2;
    zpass_split(A.N, &n1, &n2);
    if (n1) A.TY = 256 / (uint32_t)std::max(n1, n2);             // every thread busy in both passes
    else A.TY = A.N >= 2048 ? 1 : std::min<uint32_t>(32, 2048 / A.N);
    A.logTY = 0;
    while ((1u << A.logTY) < A.TY) A.logTY++;
    A.bx0 = L.box0[0]; A.by0 = L.box0[1]; A.by1 = L.box1[1]; A.bz0 = L.box0[2]; A.bz1 = L.box1[2];
    A.P = L.P; A.Pk = (size_t)A.Kz * A.m0 * A.m1;
    return A;
}

}  // namespace

// Pruned-transform sizes: shared memory of the two z-pass kernels.
size_t zpass_smem(const LongRange& L, bool inverse) {
    const ZPass A = zpass_args(L);
    int n1, n2;
    zpass_split(A.N, &n1, &n2);
    const size_t tws = 2 * (size_t)A.N + 1;                 // FFT twiddles + split twiddles
    const size_t rows = (size_t)A.TY * (A.N + 2);
    if (!inverse || n1) return sizeof(float2) * (rows + tws);
    return sizeof(float2) * (rows + (size_t)A.TY * (A.N + 1) + tws);
}

// Launch the z-pass of the right (N1, N2) instantiation.
static cudaError_t zpass_run(asd_handle* h, bool inverse) {
    LongRange& L = h->lr;
    const ZPass A = zpass_args(L);
    int n1, n2;
    zpass_split(A.N, &n1, &n2);
    const dim3 grid((A.by1 - A.by0 + A.TY) / A.TY, L.box1[0] - L.box0[0] + 1, 3);
    const size_t sm = zpass_smem(L, inverse);
    float* hr = L.r + 3 * L.P;
#define ZP(a, b)                                                                                      \
    if (inverse) zpass_c2r<a, b><<<grid, 256, sm, h->stream>>>(L.k2, hr, A);                          \
    else zpass_r2c<a, b><<<grid, 256, sm, h->stream>>>(L.r, L.k1, A);
    switch (A.N) {
    case 4: ZP(2, 2) break;
    case 8: ZP(4, 2) break;
    case 16: ZP(4, 4) break;
    case 32: ZP(8, 4) break;
    case 64: ZP(8, 8) break;
    case 128: ZP(16, 8) break;
    case 256: ZP(16, 16) break;
    default: ZP(0, 0) break;
    }
#undef ZP
    h->launches += 1;
    return cudaGetLastError();
}

cudaError_t permute_nk_pruned(asd_handle* h) {
    LongRange& L = h->lr;
    const ZPass A = zpass_args(L);
    cudaError_t e;
    if (L.ncomp == 6 && L.nk_real) {
        float* t = nullptr;
        if ((e = cudaMalloc(&t, sizeof(float) * 6 * A.Pk)) != cudaSuccess) return e;
        permute_nk<float><<<nb(6 * A.Pk, 256), 256, 0, h->stream>>>(A.Pk, 6, A.m0, A.m1, A.Kz, L.nkr, t);
        cudaStreamSynchronize(h->stream);
        cudaFree(L.nkr);
        L.nkr = t;
    } else {
        float2* t = nullptr;
        if ((e = cudaMalloc(&t, sizeof(float2) * 9 * A.Pk)) != cudaSuccess) return e;
        permute_nk<float2><<<nb(9 * A.Pk, 256), 256, 0, h->stream>>>(A.Pk, 9, A.m0, A.m1, A.Kz, L.nkc, t);
        cudaStreamSynchronize(h->stream);
        cudaFree(L.nkc);
        L.nkc = t;
    }
    return cudaGetLastError();
}

// The handle's spins (FP32 or fused FP64) times their weight into the padded M_r.
cudaError_t launch_lr_scatter(asd_handle* h) {
    LongRange& L = h->lr;
    if (h->p.precision == ASD_FP32)
        scatter_k<float><<<nb(h->n, 256), 256, 0, h->stream>>>(h->n, L.P, h->sf[0], h->sf[1], h->sf[2], L.w, L.mesh_idx, L.r);
    else
        scatter_k<double><<<nb(h->n, 256), 256, 0, h->stream>>>(h->n, L.P, h->sd[0], h->sd[1], h->sd[2], L.w, L.mesh_idx, L.r);
    h->launches += 1;
    return cudaGetLastError();
}

// M_r -> (R2C) -> N_k . M_k -> (C2R) -> H_r
cudaError_t launch_lr_eval_f32(asd_handle* h) {
    LongRange& L = h->lr;
    if (L.planes) return launch_lr_planes(h);
    if (L.pruned) {
        const ZPass A = zpass_args(L);
        cudaError_t e = zpass_run(h, false);
        if (e != cudaSuccess) return e;
        if (cufftExecC2C(L.c2c, (cufftComplex*)L.k1, (cufftComplex*)L.k2, CUFFT_FORWARD) != CUFFT_SUCCESS)
            return cudaErrorUnknown;
        if (L.ncomp == 6 && L.nk_real) kconv6r<<<nb(A.Pk, 256), 256, 0, h->stream>>>(A.Pk, L.nkr, L.k2);
        else kconv9c<<<nb(A.Pk, 256), 256, 0, h->stream>>>(A.Pk, L.nkc, L.k2);
        h->launches += 1;
        if (cufftExecC2C(L.c2c, (cufftComplex*)L.k2, (cufftComplex*)L.k2, CUFFT_INVERSE) != CUFFT_SUCCESS)
            return cudaErrorUnknown;
        return zpass_run(h, true);
    }
    if (cufftExecR2C(L.r2c, (cufftReal*)L.r, (cufftComplex*)L.k) != CUFFT_SUCCESS) return cudaErrorUnknown;
    if (L.ncomp == 6 && L.nk_real) kconv6r<<<nb(L.Pk, 256), 256, 0, h->stream>>>(L.Pk, L.nkr, L.k);
    else kconv9c<<<nb(L.Pk, 256), 256, 0, h->stream>>>(L.Pk, L.nkc, L.k);
    h->launches += 1;
    if (cufftExecC2R(L.c2r, (cufftComplex*)L.k, (cufftReal*)(L.r + 3 * L.P)) != CUFFT_SUCCESS) return cudaErrorUnknown;
    return cudaGetLastError();
}

// Build the FP32 half-spectrum N_k from the FP64 real-space matrix d_nr[9][P] (device).
cudaError_t build_nk_f32(asd_handle* h, const double* d_nr) {
    LongRange& L = h->lr;
    int dims[3] = {(int)L.mesh[0], (int)L.mesh[1], (int)L.mesh[2]};
    const uint32_t nc = L.ncomp;
    static const int map6[6] = {0, 1, 2, 4, 5, 8};
    double* src = nullptr;
    double2* z = nullptr;
    cudaError_t e;
    if ((e = cudaMalloc(&src, sizeof(double) * nc * L.P)) != cudaSuccess) return e;
    if ((e = cudaMalloc(&z, sizeof(double2) * nc * L.Pk)) != cudaSuccess) { cudaFree(src); return e; }
    for (uint32_t q = 0; q < nc; q++) {
        const int comp = nc == 6 ? map6[q] : (int)q;
        cudaMemcpyAsync(src + q * L.P, d_nr + comp * L.P, sizeof(double) * L.P, cudaMemcpyDeviceToDevice, h->stream);
    }
    cufftHandle plan;
    if (cufftPlanMany(&plan, 3, dims, nullptr, 1, (int)L.P, nullptr, 1, (int)L.Pk, CUFFT_D2Z, (int)nc) != CUFFT_SUCCESS) {
        cudaFree(src); cudaFree(z);
        return cudaErrorMemoryAllocation;
    }
    cufftSetStream(plan, h->stream);
    if (cufftExecD2Z(plan, src, (cufftDoubleComplex*)z) != CUFFT_SUCCESS) {
        cufftDestroy(plan); cudaFree(src); cudaFree(z);
        return cudaErrorUnknown;
    }
    unsigned long long* mx = nullptr;
    cudaMalloc(&mx, 2 * sizeof(unsigned long long));
    cudaMemsetAsync(mx, 0, 2 * sizeof(unsigned long long), h->stream);
    nk_extent<<<std::min<unsigned>(nb(nc * L.Pk, 256), 148 * 8), 256, 0, h->stream>>>(nc * L.Pk, z, mx);
    unsigned long long hm[2] = {0, 0};
    cudaMemcpyAsync(hm, mx, sizeof(hm), cudaMemcpyDeviceToHost, h->stream);
    cudaStreamSynchronize(h->stream);
    double re, im;
    memcpy(&re, &hm[0], 8); memcpy(&im, &hm[1], 8);
    L.nk_real = (im <= 1e-9 * re) ? 1 : 0;
    if (L.planes) {
        // the plane kernels read N_k tiled per (kz, ky tile); a general N_k takes 9 complex
        // components (a symmetric set expanded first)
        const bool cplx = !(nc == 6 && L.nk_real);
        double2* z9 = z;
        if (cplx && nc == 6) {
            cudaMalloc(&z9, sizeof(double2) * 9 * L.Pk);
            static const int inv6[9] = {0, 1, 2, 1, 3, 4, 2, 4, 5};
            for (int q = 0; q < 9; q++)
                cudaMemcpyAsync(z9 + q * L.Pk, z + inv6[q] * L.Pk, sizeof(double2) * L.Pk, cudaMemcpyDeviceToDevice, h->stream);
        }
        if (cplx) L.ncomp = 9;
        e = build_nk_tiles(h, z9, cplx ? 9 : 6, cplx);
        cudaError_t e2 = cudaStreamSynchronize(h->stream);
        if (z9 != z) cudaFree(z9);
        cufftDestroy(plan);
        cudaFree(mx); cudaFree(src); cudaFree(z);
        if (e != cudaSuccess) return e;
        if (e2 != cudaSuccess) return e2;
        e = cudaMalloc(&L.yk, sizeof(float2) * plane_spectrum_elems(L));
        return e == cudaSuccess ? cudaGetLastError() : e;
    }
    if (nc == 6 && L.nk_real) {
        cudaMalloc(&L.nkr, sizeof(float) * 6 * L.Pk);
        nk_pack_real<<<nb(6 * L.Pk, 256), 256, 0, h->stream>>>(L.Pk, 6, z, nullptr, L.nkr, nullptr);
    } else {
        // general path stores all 9 components; expand a symmetric set first
        double2* z9 = z;
        if (nc == 6) {
            cudaMalloc(&z9, sizeof(double2) * 9 * L.Pk);
            static const int inv[9] = {0, 1, 2, 1, 3, 4, 2, 4, 5};
            for (int q = 0; q < 9; q++)
                cudaMemcpyAsync(z9 + q * L.Pk, z + inv[q] * L.Pk, sizeof(double2) * L.Pk, cudaMemcpyDeviceToDevice, h->stream);
        }
        cudaMalloc(&L.nkc, sizeof(float2) * 9 * L.Pk);
        nk_pack_cplx<<<nb(9 * L.Pk, 256), 256, 0, h->stream>>>(9 * L.Pk, z9, L.nkc);
        if (z9 != z) { cudaStreamSynchronize(h->stream); cudaFree(z9); }
        L.ncomp = 9;
    }
    e = cudaStreamSynchronize(h->stream);
    cufftDestroy(plan);
    cudaFree(mx); cudaFree(src); cudaFree(z);
    return e == cudaSuccess ? cudaGetLastError() : e;
}

// FP64 plain: complex N_k[9][P] by Z2Z forward of N_r (as the reference's FFTW
// forward of the complex Nrab, src/intmat.cpp:332-398).
cudaError_t build_nk_plain(asd_handle* h, const double* d_nr) {
    LongRange& L = h->lr;
    int dims[3] = {(int)L.mesh[0], (int)L.mesh[1], (int)L.mesh[2]};
    double2* zin = nullptr;
    cudaError_t e;
    if ((e = cudaMalloc(&zin, sizeof(double2) * 9 * L.P)) != cudaSuccess) return e;
    real_to_cplx<<<nb(9 * L.P, 256), 256, 0, h->stream>>>(9 * L.P, d_nr, zin);
    cufftHandle plan;
    if (cufftPlanMany(&plan, 3, dims, nullptr, 1, (int)L.P, nullptr, 1, (int)L.P, CUFFT_Z2Z, 9) != CUFFT_SUCCESS) {
        cudaFree(zin);
        return cudaErrorMemoryAllocation;
    }
    cufftSetStream(plan, h->stream);
    if (cufftExecZ2Z(plan, (cufftDoubleComplex*)zin, (cufftDoubleComplex*)L.znk, CUFFT_FORWARD) != CUFFT_SUCCESS) {
        cufftDestroy(plan); cudaFree(zin);
        return cudaErrorUnknown;
    }
    e = cudaStreamSynchronize(h->stream);
    cufftDestroy(plan);
    cudaFree(zin);
    return e;
}

}  // namespace asd
