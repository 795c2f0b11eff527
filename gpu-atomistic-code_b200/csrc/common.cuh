// Shared device definitions: parameter blocks, the thermal-noise generator and
// the per-spin field/torque arithmetic used by every stage kernel.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#define ASD_MAX_MAT 16
#define ASD_MAX_SUB 16

namespace asd {

// Per unit-cell atom constants (the reference expands these to per-spin arrays
// Csigma/Cllgpf/Clambda/Ck1u/Ck1udir, src/cuda_util.cu:497-527; the fused
// kernels read them from the parameter block instead).
struct MatConst {
    double llgpf;    // -1/(1+lambda^2)          (src/llg.cpp:592, 629)
    double lambda;
    double sigma;    // sqrt(2 kB lambda/(mu muB dt gamma gyro))  (src/llg.cpp:591)
    double k1u;      // 2K/(mu muB)               (src/geom.cpp:244)
    double k1udir[3];
    uint32_t sub;
    uint32_t pad;
    // single-precision copies for the FP32 form (no per-thread conversions)
    float llgpf_f, lambda_f, sigma_f, k1u_f, k1udir_f[3], pad_f;
};

// Kernel parameter block shared by all stage kernels (passed by value).
struct StepConst {
    uint32_t n;         // spins in the handle (all replicas)
    uint32_t nmat;
    uint32_t nrep;
    uint32_t flags;
    MatConst mat[ASD_MAX_MAT];
    double rdt;         // dt * gyro (src/llg.cpp:306)
    double dt;          // [s]
    double k2perp_f, k2perpdir[3], k2par_f, k2pardir[3];   // 2K/basemm (src/cuint.cu:99)
    double k4perp_f, k4perpdirs[9], k4par_f, k4pardirs[9];
    uint64_t seed;
    const uint32_t* atom;      // per-spin unit-cell atom or nullptr (-> i % nmat)
    const uint32_t* rep_off;   // nrep+1
    const uint32_t* rep_of_tile; // replica of the first spin of every 32-spin tile
    const uint32_t* q4_ptr;      // four-spin quartets of spin i: q4_jkl[q4_ptr[i] .. q4_ptr[i+1])
    const uint4* q4_jkl;         // (j, k, l, 0)
    double q4_jq;                // JQ [T]
    float q4_jq_f;               // JQ (/3 when divided) for the FP32 form
    int q4_div3;                 // the GPU path's division by 3
    const double* rep_sqrtT;   // nrep: sqrt(T) per replica
    const uint32_t* rep_stream;
    const double* dyn;         // mutable scalars, see DYN_*
    const uint64_t* step_base; // device step counter
    // single-precision copies for the FP32 form
    float rdt_f;
    float k2perp_ff, k2par_ff, k4perp_ff, k4par_ff;
    float k2perpdir_f[3], k2pardir_f[3], k4perpdirs_f[9], k4pardirs_f[9];
    const float* rep_sqrtT_f;  // nrep
    const float* dynf;         // float copy of the mutable scalars
};

// Layout of the mutable scalar block (device memory, updated between launches).
enum {
    DYN_APPLIED = 0, DYN_STAG_SCALE = 3, DYN_DET_STEP = 4,
    DYN_PULSE_AMP = 5, DYN_PULSE_T0 = 6, DYN_PULSE_ISIG = 7,   // site-field envelope
    DYN_COUNT = 8
};

// Site-field multiplier at step t: rv, times amp exp(-((t dt - t0)/sigma)^2/2) when amp != 0.
__device__ __forceinline__ float site_scale_f(const float* dynf, const double* dyn, uint64_t t, double dt) {
    float sc = dynf[DYN_STAG_SCALE];
    if (dynf[DYN_PULSE_AMP] != 0.0f) {
        const float x = (float)(((double)t * dt - dyn[DYN_PULSE_T0]) * dyn[DYN_PULSE_ISIG]);
        sc *= dynf[DYN_PULSE_AMP] * expf(-0.5f * x * x);
    }
    return sc;
}
__device__ __forceinline__ double site_scale_d(const double* dyn, uint64_t t, double dt) {
    double sc = dyn[DYN_STAG_SCALE];
    if (dyn[DYN_PULSE_AMP] != 0.0) {
        const double x = ((double)t * dt - dyn[DYN_PULSE_T0]) * dyn[DYN_PULSE_ISIG];
        sc *= dyn[DYN_PULSE_AMP] * exp(-0.5 * x * x);
    }
    return sc;
}

// Programmatic dependent launch, in every step kernel before its first access to memory that
// an earlier kernel of the stream writes or reads: wait until the previous kernel has completed
// and its memory is visible (a no-op for a kernel launched without the attribute), then let the
// next kernel's blocks launch (they wait the same way).  Before it a kernel touches only
// set-up data - twiddles, N_k tiles, the exchange words, tables and spans, the mesh index -
// which are written at creation and complete (synchronous uploads, a device-wide free) before
// the first step, so its prologue overlaps the previous kernel's last blocks.
__device__ __forceinline__ void pdl_enter() {
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

__device__ __forceinline__ uint32_t atom_of(const StepConst& c, uint32_t i) {
    return c.atom ? c.atom[i] : (c.nmat == 1 ? 0u : i % c.nmat);
}

// Four-spin field of spin i, accumulated from zero in quartet order (src/cufields.cu:59-90);
// get(j, v) loads spin j.
template <typename R, typename Get>
__device__ __forceinline__ void four_spin(const StepConst& c, uint32_t i, Get get, R h4[3]) {
    h4[0] = h4[1] = h4[2] = R(0);
    const uint32_t q0 = __ldg(c.q4_ptr + i), q1 = __ldg(c.q4_ptr + i + 1);
    for (uint32_t q = q0; q < q1; q++) {
        const uint4 jkl = __ldg(c.q4_jkl + q);
        R sj[3], sk[3], sl[3];
        get(jkl.x, sj); get(jkl.y, sk); get(jkl.z, sl);
        const R skdotsl = sk[0] * sl[0] + sk[1] * sl[1] + sk[2] * sl[2];
        const R sjdotsl = sj[0] * sl[0] + sj[1] * sl[1] + sj[2] * sl[2];
        const R skdotsj = sk[0] * sj[0] + sk[1] * sj[1] + sk[2] * sj[2];
        for (int a = 0; a < 3; a++) {
            const R v = sj[a] * skdotsl + sk[a] * sjdotsl + sl[a] * skdotsj;
            if constexpr (sizeof(R) == 8) h4[a] -= c.q4_div3 ? (c.q4_jq * v) / 3.0 : c.q4_jq * v;
            else h4[a] -= c.q4_jq_f * v;
        }
    }
}

// Replica of spin i: the replica of its 32-spin tile's first spin, advanced past the replica
// boundaries that lie inside the tile (none unless a replica is shorter than the tile).
__device__ __forceinline__ uint32_t replica_of(const StepConst& c, uint32_t i) {
    if (c.nrep == 1) return 0;
    uint32_t r = __ldg(c.rep_of_tile + (i >> 5));
    while (r + 1 < c.nrep && __ldg(c.rep_off + r + 1) <= i) r++;
    return r;
}

// ---------------------------------------------------------------------------
// Thermal noise.  Philox4x32-10 (Salmon et al., SC'11) keyed by the seed with
// counter (spin-in-replica, step_lo, step_hi, stream), then Box-Muller on
// (u0,u1) and (u2,u3).  log and sincos(2 pi u) are evaluated from their
// series with correctly rounded intrinsics only (no contraction), so the
// deviates are bit-identical on any IEEE-754 implementation of the same steps.

__device__ __forceinline__ void philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1) {
#pragma unroll
    for (int r = 0; r < 10; r++) {
        const uint32_t lo0 = 0xD2511F53u * c[0];
        const uint32_t hi0 = __umulhi(0xD2511F53u, c[0]);
        const uint32_t lo1 = 0xCD9E8D57u * c[2];
        const uint32_t hi1 = __umulhi(0xCD9E8D57u, c[2]);
        const uint32_t n0 = hi1 ^ c[1] ^ k0;
        const uint32_t n2 = hi0 ^ c[3] ^ k1;
        c[0] = n0; c[1] = lo1; c[2] = n2; c[3] = lo0;
        k0 += 0x9E3779B9u; k1 += 0xBB67AE85u;
    }
}

// ln x for x in (0,1]: x = m 2^e, m in [sqrt(1/2), sqrt(2)), ln m = 2 atanh(f), f=(m-1)/(m+1).
__device__ __forceinline__ double series_log(double x) {
    int e;
    double m = frexp(x, &e);
    if (m < 0x1.6a09e667f3bcdp-1) { m = __dmul_rn(m, 2.0); e = e - 1; }
    const double f = __ddiv_rn(__dsub_rn(m, 1.0), __dadd_rn(m, 1.0));
    const double f2 = __dmul_rn(f, f);
    double p = 0x1.642c8590b2164p-5;            // 1/23
    p = __fma_rn(p, f2, 0x1.8618618618618p-5);  // 1/21
    p = __fma_rn(p, f2, 0x1.af286bca1af28p-5);  // 1/19
    p = __fma_rn(p, f2, 0x1.e1e1e1e1e1e1ep-5);  // 1/17
    p = __fma_rn(p, f2, 0x1.1111111111111p-4);  // 1/15
    p = __fma_rn(p, f2, 0x1.3b13b13b13b14p-4);  // 1/13
    p = __fma_rn(p, f2, 0x1.745d1745d1746p-4);  // 1/11
    p = __fma_rn(p, f2, 0x1.c71c71c71c71cp-4);  // 1/9
    p = __fma_rn(p, f2, 0x1.2492492492492p-3);  // 1/7
    p = __fma_rn(p, f2, 0x1.999999999999ap-3);  // 1/5
    p = __fma_rn(p, f2, 0x1.5555555555555p-2);  // 1/3
    p = __fma_rn(p, f2, 1.0);
    const double lnm = __dmul_rn(2.0, __dmul_rn(f, p));
    return __fma_rn((double)e, 0x1.62e42fefa39efp-1, lnm);
}

// (sin, cos) of the angle from those of its reduced argument in octant q, without branches:
// q in {1,2,5,6} swaps the pair, q in {4..7} negates sin, q in {2..5} negates cos.
template <typename T>
__device__ __forceinline__ void octant_select(int q, T s, T c, T& sn, T& cs) {
    const bool swap = ((q + 1) >> 1) & 1;
    const T a = swap ? c : s, b = swap ? s : c;
    sn = (q >> 2) & 1 ? -a : a;
    cs = ((q + 2) >> 2) & 1 ? -b : b;
}

// sin, cos of 2 pi (x+0.5)/2^32: exact octant reduction, Taylor series on [0, pi/4].
__device__ __forceinline__ void series_sincos_2pi(uint32_t x, double& sn, double& cs) {
    const double v = __dmul_rn(__dadd_rn((double)x, 0.5), 0x1p-29);
    const double qd = floor(v);
    const int q = (int)qd;
    const double r = __dsub_rn(v, qd);
    const double psi = __dmul_rn((q & 1) ? __dsub_rn(1.0, r) : r, 0x1.921fb54442d18p-1);
    const double p2 = __dmul_rn(psi, psi);
    const double mp2 = -p2;
    double sp = 0x1.2f49b46814157p-57;            // 1/19!
    sp = __fma_rn(sp, mp2, 0x1.952c77030ad4ap-49); // 1/17!
    sp = __fma_rn(sp, mp2, 0x1.ae7f3e733b81fp-41); // 1/15!
    sp = __fma_rn(sp, mp2, 0x1.6124613a86d09p-33); // 1/13!
    sp = __fma_rn(sp, mp2, 0x1.ae64567f544e4p-26); // 1/11!
    sp = __fma_rn(sp, mp2, 0x1.71de3a556c734p-19); // 1/9!
    sp = __fma_rn(sp, mp2, 0x1.a01a01a01a01ap-13); // 1/7!
    sp = __fma_rn(sp, mp2, 0x1.1111111111111p-7);  // 1/5!
    sp = __fma_rn(sp, mp2, 0x1.5555555555555p-3);  // 1/3!
    sp = __fma_rn(sp, mp2, 1.0);
    const double s = __dmul_rn(psi, sp);
    double cp = 0x1.6827863b97d97p-53;            // 1/18!
    cp = __fma_rn(cp, mp2, 0x1.ae7f3e733b81fp-45); // 1/16!
    cp = __fma_rn(cp, mp2, 0x1.93974a8c07c9dp-37); // 1/14!
    cp = __fma_rn(cp, mp2, 0x1.1eed8eff8d898p-29); // 1/12!
    cp = __fma_rn(cp, mp2, 0x1.27e4fb7789f5cp-22); // 1/10!
    cp = __fma_rn(cp, mp2, 0x1.a01a01a01a01ap-16); // 1/8!
    cp = __fma_rn(cp, mp2, 0x1.6c16c16c16c17p-10); // 1/6!
    cp = __fma_rn(cp, mp2, 0x1.5555555555555p-5);  // 1/4!
    cp = __fma_rn(cp, mp2, 0x1.0000000000000p-1);  // 1/2!
    const double c = __fma_rn(cp, mp2, 1.0);
    octant_select(q, s, c, sn, cs);
}

__device__ __forceinline__ void thermal_normals(uint64_t seed, uint32_t stream, uint32_t spin, uint64_t step,
                                                double out[3]) {
    uint32_t c[4] = {spin, (uint32_t)step, (uint32_t)(step >> 32), stream};
    philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
    const double u0 = __dmul_rn(__dadd_rn((double)c[0], 0.5), 0x1p-32);
    const double u2 = __dmul_rn(__dadd_rn((double)c[2], 0.5), 0x1p-32);
    const double r0 = __dsqrt_rn(__dmul_rn(-2.0, series_log(u0)));
    const double r2 = __dsqrt_rn(__dmul_rn(-2.0, series_log(u2)));
    double s1, c1, s3, c3;
    series_sincos_2pi(c[1], s1, c1);
    series_sincos_2pi(c[3], s3, c3);
    out[0] = __dmul_rn(r0, c1);
    out[1] = __dmul_rn(r0, s1);
    out[2] = __dmul_rn(r2, c3);
}

// Single-precision variant for the FP32 form: the same Philox draw, uniforms
// u = (float(x) + 0.5) 2^-32 (float(x) rounded to nearest, so small u keep their
// relative precision and the tail follows the double draw), the sin/cos octant taken
// exactly from the top 3 bits of x, and shorter series evaluated with correctly rounded
// float operations (ln: terms to f^11; sin to psi^11, cos to psi^12), accurate to a few
// float ulps and reproducible on any IEEE-754 float implementation.
__device__ __forceinline__ float series_logf(float x) {
    int e;
    float m = frexpf(x, &e);
    if (m < 0x1.6a09e6p-1f) { m = __fmul_rn(m, 2.0f); e = e - 1; }
    const float f = __fdiv_rn(__fsub_rn(m, 1.0f), __fadd_rn(m, 1.0f));
    const float f2 = __fmul_rn(f, f);
    float p = 0x1.745d18p-4f;               // 1/11
    p = __fmaf_rn(p, f2, 0x1.c71c72p-4f);   // 1/9
    p = __fmaf_rn(p, f2, 0x1.24924ap-3f);   // 1/7
    p = __fmaf_rn(p, f2, 0x1.99999ap-3f);   // 1/5
    p = __fmaf_rn(p, f2, 0x1.555556p-2f);   // 1/3
    p = __fmaf_rn(p, f2, 1.0f);
    const float lnm = __fmul_rn(2.0f, __fmul_rn(f, p));
    return __fmaf_rn((float)e, 0x1.62e430p-1f, lnm);
}

__device__ __forceinline__ void series_sincos_2pi_f(uint32_t x, float& sn, float& cs) {
    const int q = (int)(x >> 29);                                                          // octant
    const float r = __fmul_rn(__fadd_rn(__uint2float_rn(x & 0x1FFFFFFFu), 0.5f), 0x1p-29f); // in (0, 1]
    const float psi = __fmul_rn((q & 1) ? __fsub_rn(1.0f, r) : r, 0x1.921fb6p-1f);
    const float mp2 = -__fmul_rn(psi, psi);
    float sp = 0x1.ae6456p-26f;               // 1/11!
    sp = __fmaf_rn(sp, mp2, 0x1.71de3ap-19f); // 1/9!
    sp = __fmaf_rn(sp, mp2, 0x1.a01a02p-13f); // 1/7!
    sp = __fmaf_rn(sp, mp2, 0x1.111112p-7f);  // 1/5!
    sp = __fmaf_rn(sp, mp2, 0x1.555556p-3f);  // 1/3!
    sp = __fmaf_rn(sp, mp2, 1.0f);
    const float s = __fmul_rn(psi, sp);
    float cp = 0x1.1eed8ep-29f;               // 1/12!
    cp = __fmaf_rn(cp, mp2, 0x1.27e4fcp-22f); // 1/10!
    cp = __fmaf_rn(cp, mp2, 0x1.a01a02p-16f); // 1/8!
    cp = __fmaf_rn(cp, mp2, 0x1.6c16c2p-10f); // 1/6!
    cp = __fmaf_rn(cp, mp2, 0x1.555556p-5f);  // 1/4!
    cp = __fmaf_rn(cp, mp2, 0x1.000000p-1f);  // 1/2!
    const float c = __fmaf_rn(cp, mp2, 1.0f);
    octant_select(q, s, c, sn, cs);
}

__device__ __forceinline__ void thermal_normals_f(uint64_t seed, uint32_t stream, uint32_t spin, uint64_t step,
                                                  float out[3]) {
    uint32_t c[4] = {spin, (uint32_t)step, (uint32_t)(step >> 32), stream};
    philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
    const float u0 = __fmul_rn(__fadd_rn(__uint2float_rn(c[0]), 0.5f), 0x1p-32f);   // in (0, 1]
    const float u2 = __fmul_rn(__fadd_rn(__uint2float_rn(c[2]), 0.5f), 0x1p-32f);
    const float r0 = __fsqrt_rn(__fmul_rn(-2.0f, series_logf(u0)));
    const float r2 = __fsqrt_rn(__fmul_rn(-2.0f, series_logf(u2)));
    float s1, c1, s3, c3;
    series_sincos_2pi_f(c[1], s1, c1);
    series_sincos_2pi_f(c[3], s3, c3);
    out[0] = __fmul_rn(r0, c1);
    out[1] = __fmul_rn(r0, s1);
    out[2] = __fmul_rn(r2, c3);
}

}  // namespace asd
