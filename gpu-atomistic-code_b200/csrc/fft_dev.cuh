// Device building blocks of the long-range-field transforms (FP32, power-of-two sizes).
//
//  * dft<R, INV>: R-point DFT (R <= 16) of a register array, natural order in and out,
//    radix-4/radix-2 with compile-time twiddles (multiplications by +-1, +-i are free).
//  * The "four-step" split N = R1 R2 used by the plane kernels:
//        X[m + R1 q] = sum_t w_R2^{t q} w_N^{t m} sum_k w_R1^{k m} x[t + R2 k]
//    pass 1: one thread per t runs the R1-point DFT over k and multiplies by w_N^{t m};
//    pass 2: one thread per m runs the R2-point DFT over t.  The inverse runs the same passes
//    in reverse order with conjugate twiddles (unnormalised, like cuFFT).
//  * The z-axis real transform (R2C / C2R through an N-point complex FFT of
//    z_n = x_2n + i x_2n+1 plus the split) with its shared-memory two-pass FFT.
#pragma once
#include <cstdint>

namespace asd {
namespace fftd {

__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// a * conj(b)
__device__ __forceinline__ float2 cmulc(float2 a, float2 b) {
    return make_float2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}

// a * w_16^e (forward, w = exp(-2 pi i / 16)) or a * conj(w_16^e) (inverse); e is a compile-time
// constant after unrolling, so the switch folds to the one expression.
template <bool INV>
__device__ __forceinline__ float2 tw16(float2 a, int e) {
    constexpr float C1 = 0.92387953251128676f;   // cos(pi/8)
    constexpr float S1 = 0.38268343236508977f;   // sin(pi/8)
    constexpr float H = 0.70710678118654752f;    // sqrt(1/2)
    const float sg = INV ? 1.0f : -1.0f;         // sign of the imaginary part of w_16^1
    switch (e & 15) {
    case 0: return a;
    case 4: return INV ? make_float2(-a.y, a.x) : make_float2(a.y, -a.x);
    case 8: return make_float2(-a.x, -a.y);
    case 12: return INV ? make_float2(a.y, -a.x) : make_float2(-a.y, a.x);
    case 2: return cmul(a, make_float2(H, sg * H));
    case 6: return cmul(a, make_float2(-H, sg * H));
    case 10: return cmul(a, make_float2(-H, -sg * H));
    case 14: return cmul(a, make_float2(H, -sg * H));
    case 1: return cmul(a, make_float2(C1, sg * S1));
    case 3: return cmul(a, make_float2(S1, sg * C1));
    case 5: return cmul(a, make_float2(-S1, sg * C1));
    case 7: return cmul(a, make_float2(-C1, sg * S1));
    case 9: return cmul(a, make_float2(-C1, -sg * S1));
    case 11: return cmul(a, make_float2(-S1, -sg * C1));
    case 13: return cmul(a, make_float2(S1, -sg * C1));
    default: return cmul(a, make_float2(C1, -sg * S1));   // 15
    }
}

// a * (-i) forward, a * (+i) inverse
template <bool INV>
__device__ __forceinline__ float2 mul_mi(float2 a) {
    return INV ? make_float2(-a.y, a.x) : make_float2(a.y, -a.x);
}

template <int R, bool INV>
struct Dft;

template <bool INV>
struct Dft<1, INV> {
    static __device__ __forceinline__ void run(float2*) {}
};

template <bool INV>
struct Dft<2, INV> {
    static __device__ __forceinline__ void run(float2* v) {
        const float2 a = v[0], b = v[1];
        v[0] = cadd(a, b);
        v[1] = csub(a, b);
    }
};

template <bool INV>
struct Dft<4, INV> {
    static __device__ __forceinline__ void run(float2* v) {
        const float2 t0 = cadd(v[0], v[2]), t1 = csub(v[0], v[2]);
        const float2 t2 = cadd(v[1], v[3]), t3 = mul_mi<INV>(csub(v[1], v[3]));
        v[0] = cadd(t0, t2);
        v[2] = csub(t0, t2);
        v[1] = cadd(t1, t3);
        v[3] = csub(t1, t3);
    }
};

// R = 4 Q (Q = 2 or 4): four-step with N1 = 4, N2 = Q in registers.
template <int R, bool INV>
struct Dft {
    static_assert(R == 8 || R == 16, "register DFT sizes are 1, 2, 4, 8, 16");
    static __device__ __forceinline__ void run(float2* v) {
        constexpr int Q = R / 4;
        float2 a[Q][4];
#pragma unroll
        for (int t = 0; t < Q; t++) {
#pragma unroll
            for (int k = 0; k < 4; k++) a[t][k] = v[t + Q * k];
            Dft<4, INV>::run(a[t]);
#pragma unroll
            for (int m = 1; m < 4; m++) a[t][m] = tw16<INV>(a[t][m], (t * m) * (16 / R));
        }
#pragma unroll
        for (int m = 0; m < 4; m++) {
            float2 b[Q];
#pragma unroll
            for (int t = 0; t < Q; t++) b[t] = a[t][m];
            Dft<Q, INV>::run(b);
#pragma unroll
            for (int q = 0; q < Q; q++) v[m + 4 * q] = b[q];
        }
    }
};

template <int R, bool INV>
__device__ __forceinline__ void dft(float2 (&v)[R]) {
    Dft<R, INV>::run(v);
}

// Pruned R-point DFT: inputs v[NIN..R) are zero (not read), and only the outputs v[0..NOUT)
// are formed (the others are left undefined).  NIN, NOUT in {R/2, R}, R in {2, 4, 8, 16}.
template <int R, bool INV, int NIN, int NOUT>
struct DftP;

template <bool INV, int NIN, int NOUT>
struct DftP<2, INV, NIN, NOUT> {
    static __device__ __forceinline__ void run(float2* v) {
        if constexpr (NIN == 1) {
            v[1] = v[0];
        } else if constexpr (NOUT == 1) {
            v[0] = cadd(v[0], v[1]);
        } else {
            Dft<2, INV>::run(v);
        }
    }
};

template <bool INV, int NIN, int NOUT>
struct DftP<4, INV, NIN, NOUT> {
    static __device__ __forceinline__ void run(float2* v) {
        float2 t0, t1, t2, t3;
        if constexpr (NIN == 2) {
            t0 = v[0]; t1 = v[0]; t2 = v[1]; t3 = mul_mi<INV>(v[1]);
        } else {
            t0 = cadd(v[0], v[2]); t1 = csub(v[0], v[2]);
            t2 = cadd(v[1], v[3]); t3 = mul_mi<INV>(csub(v[1], v[3]));
        }
        v[0] = cadd(t0, t2);
        v[1] = cadd(t1, t3);
        if constexpr (NOUT == 4) {
            v[2] = csub(t0, t2);
            v[3] = csub(t1, t3);
        }
    }
};

// R = 4 Q: the inputs t + Q k < NIN = R/2 are the k < 2; the outputs m + 4 q < NOUT = R/2 are the
// q < Q/2.
template <int R, bool INV, int NIN, int NOUT>
struct DftP {
    static_assert(R == 8 || R == 16, "pruned DFT sizes are 2, 4, 8, 16");
    static __device__ __forceinline__ void run(float2* v) {
        constexpr int Q = R / 4;
        float2 a[Q][4];
#pragma unroll
        for (int t = 0; t < Q; t++) {
#pragma unroll
            for (int k = 0; k < 4; k++) a[t][k] = (NIN == R || k < 2) ? v[t + Q * k] : make_float2(0.f, 0.f);
            DftP<4, INV, (NIN == R ? 4 : 2), 4>::run(a[t]);
#pragma unroll
            for (int m = 1; m < 4; m++) a[t][m] = tw16<INV>(a[t][m], (t * m) * (16 / R));
        }
#pragma unroll
        for (int m = 0; m < 4; m++) {
            float2 b[Q];
#pragma unroll
            for (int t = 0; t < Q; t++) b[t] = a[t][m];
            if constexpr (NOUT == R) Dft<Q, INV>::run(b);
            else DftP<Q, INV, Q, Q / 2>::run(b);
#pragma unroll
            for (int q = 0; q < (NOUT == R ? Q : Q / 2); q++) v[m + 4 * q] = b[q];
        }
    }
};

// The R-point DFT with the upper half of the inputs zero (HIN) and/or only the lower half of the
// outputs formed (HOUT).
template <int R, bool INV, bool HIN, bool HOUT>
__device__ __forceinline__ void dftp(float2 (&v)[R]) {
    if constexpr (!HIN && !HOUT) Dft<R, INV>::run(v);
    else DftP<R, INV, HIN ? R / 2 : R, HOUT ? R / 2 : R>::run(v);
}

// (R1, R2) of the four-step split of a power-of-two N <= 256 (R1 >= R2).
__host__ __device__ constexpr int split_r1(int N) { return N <= 2 ? N : N <= 8 ? (N == 8 ? 4 : 2) : N <= 32 ? (N == 32 ? 8 : 4) : N <= 128 ? (N == 128 ? 16 : 8) : 16; }
__host__ __device__ constexpr int split_r2(int N) { return N / split_r1(N); }
__host__ __device__ constexpr uint32_t ilog2c(uint32_t v) { return v <= 1 ? 0 : 1 + ilog2c(v / 2); }

// tw[j] = exp(-2 pi i j / N), j < N.
__device__ __forceinline__ void load_tw(float2* tw, uint32_t N) {
    for (uint32_t j = threadIdx.x; j < N; j += blockDim.x) {
        float sn, cs;
        sincospif(-2.0f * (float)j / (float)N, &sn, &cs);
        tw[j] = make_float2(cs, sn);
    }
}

// tw[j] = exp(-2 pi i j / N) for j < N, then the split twiddles ws[k] = exp(-i pi k / N) for
// k <= N at tw + N.
__device__ __forceinline__ void load_twiddles(float2* tw, uint32_t N) {
    load_tw(tw, N);
    for (uint32_t k = threadIdx.x; k <= N; k += blockDim.x) {
        float sn, cs;
        sincospif(-(float)k / (float)N, &sn, &cs);
        tw[N + k] = make_float2(cs, sn);
    }
}

// Barrier of a group of threads that shares rows of shared memory: the warp when every row's
// threads lie in one warp (WL), else the block.
template <bool WL>
__device__ __forceinline__ void group_sync() {
    if constexpr (WL) __syncwarp(); else __syncthreads();
}

// True when fft2pass<N1, N2> keeps every row inside one warp: both passes give row r the
// threads [r N2, (r + 1) N2), so warp w owns the rows [w 32 / N2, (w + 1) 32 / N2).
template <int N1, int N2>
__host__ __device__ constexpr bool rows_warp_local() { return N1 == N2 && 32 % N2 == 0; }

// N = N1 * N2 point DFT of TY rows of shared memory (row pitch ld, natural order in and out, in
// place), TY * max(N1, N2) <= blockDim.x; N1, N2 <= 16.  The intermediate between the passes is
// stored with pitch N2 + 1 per m, so ld >= N1 (N2 + 1); with ld = N2 (mod 16) the accesses of
// both passes are free of bank conflicts.  Ends with a barrier: the warp's when
// rows_warp_local<N1, N2>() (the caller then writes and reads each row from the warp owning
// it), else the block's.
template <int N1, int N2, bool INV, bool HIN = false, bool HOUT = false>
__device__ __forceinline__ void fft2pass(float2* s, uint32_t ld, const float2* tw, uint32_t TY) {
    // HIN: the row's inputs N/2..N are zero (pass 1 reads k < N1/2 only); HOUT: only the outputs
    // 0..N/2 are formed (pass 2 writes q < N2/2 only)
    constexpr bool WL = rows_warp_local<N1, N2>();
    {
        const uint32_t it = threadIdx.x, r = it / N2, t = it % N2;
        const bool act = it < TY * N2;
        float2 v[N1];
        if (act) {
#pragma unroll
            for (int k = 0; k < N1; k++) v[k] = (!HIN || k < N1 / 2) ? s[r * ld + t + N2 * k] : make_float2(0.f, 0.f);
            dftp<N1, INV, HIN, false>(v);
#pragma unroll
            for (int m = 1; m < N1; m++) v[m] = INV ? cmulc(v[m], tw[t * m]) : cmul(v[m], tw[t * m]);
        }
        group_sync<WL>();
        if (act) {
#pragma unroll
            for (int m = 0; m < N1; m++) s[r * ld + m * (N2 + 1) + t] = v[m];
        }
        group_sync<WL>();
    }
    {
        const uint32_t it = threadIdx.x, r = it / N1, m = it % N1;
        const bool act = it < TY * N1;
        float2 u[N2];
        if (act) {
#pragma unroll
            for (int t = 0; t < N2; t++) u[t] = s[r * ld + m * (N2 + 1) + t];
            dftp<N2, INV, false, HOUT>(u);
        }
        group_sync<WL>();
        if (act) {
#pragma unroll
            for (int q = 0; q < (HOUT ? N2 / 2 : N2); q++) s[r * ld + m + N1 * q] = u[q];
        }
        group_sync<WL>();
    }
}

// Row pitch for fft2pass on N = N1 N2 points with room for index N: the smallest
// ld >= max(N + 1, N1 (N2 + 1)) with ld = N2 (mod 16).
__host__ __device__ constexpr uint32_t fft2pass_pitch(uint32_t N, uint32_t N1, uint32_t N2) {
    uint32_t need = N + 1 > N1 * (N2 + 1) ? N + 1 : N1 * (N2 + 1);
    uint32_t ld = need;
    while (ld % 16 != N2 % 16) ld++;
    return ld;
}

// R2C split: X_k = E_k + w^k O_k, E = (Z_k + conj Z_{N-k}) / 2, O = -i (Z_k - conj Z_{N-k}) / 2,
// w = e^{-i pi / N}, from the N-point spectrum Z of z_n = x_2n + i x_2n+1.
__device__ __forceinline__ float2 r2c_split(float2 zk, float2 zm, float2 wsk) {
    const float2 E = make_float2(0.5f * (zk.x + zm.x), 0.5f * (zk.y - zm.y));
    const float2 O = make_float2(0.5f * (zk.y + zm.y), -0.5f * (zk.x - zm.x));
    const float2 wo = cmul(wsk, O);
    return make_float2(E.x + wo.x, E.y + wo.y);
}

// C2R pre-processing: Z'_k = (X_k + conj X_{N-k}) + i e^{+i pi k / N} (X_k - conj X_{N-k}): twice
// the spectrum of z_n = x_2n + i x_2n+1, so that the unnormalised inverse gives 2N x (cuFFT's C2R
// scaling).
__device__ __forceinline__ float2 c2r_pre(float2 xk, float2 xm, float2 wsk) {
    const float2 sp = make_float2(xk.x + xm.x, xk.y - xm.y);
    const float2 df = make_float2(xk.x - xm.x, xk.y + xm.y);
    const float2 t = cmul(make_float2(wsk.x, -wsk.y), df);
    return make_float2(sp.x - t.y, sp.y + t.x);
}

}  // namespace fftd
}  // namespace asd
