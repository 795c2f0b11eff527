// FP64 "plain" form of the step: one thread per spin, AoS doubles [3i+c],
// per-spin parameter arrays and separate noise / field / stage launches -
// the structure of the reference CUDA Heun (src/cuda.cu:43-258) and RK
// (src/cudaRK4.cu:38-233, src/cudaRK5.cu) pipelines, written anew.
//
// This file is compiled with --fmad=false: every expression is evaluated
// in the written order with correctly rounded operations, so the results
// reproduce, bit for bit, an FP64 scalar CPU evaluation in the same order.
#include "internal.h"
#include <cmath>

namespace asd {
namespace {

__global__ void plain_noise_k(StepConst c, uint64_t step, double* __restrict__ rnd) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= c.n) return;
    const uint32_t r = replica_of(c, i);
    double xi[3];
    thermal_normals(c.seed, c.rep_stream[r], i - c.rep_off[r], step, xi);
    rnd[3 * i] = xi[0];
    rnd[3 * i + 1] = xi[1];
    rnd[3 * i + 2] = xi[2];
}

// CH = HDemag + sum_j J_ij S_j  (overwrite; src/cufields.cu:180-246 semantics)
template <bool FULL>
__global__ void plain_spmv_csr(uint32_t n, const uint32_t* __restrict__ xadj, const uint32_t* __restrict__ adj,
                               PlainExch ex, const double* __restrict__ s, const double* __restrict__ hd,
                               double* __restrict__ ch, int zz_from_yy) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double dot[3] = {0.0, 0.0, 0.0};
    const double* vzz = zz_from_yy ? ex.v[4] : ex.v[8];
    for (uint32_t k = xadj[i]; k < xadj[i + 1]; k++) {
        const uint32_t j = adj[k];
        if (!FULL) {
            dot[0] += ex.v[0][k] * s[3 * j];
            dot[1] += ex.v[4][k] * s[3 * j + 1];
            dot[2] += vzz[k] * s[3 * j + 2];
        } else {
            const double m[9] = {ex.v[0][k], ex.v[1][k], ex.v[2][k], ex.v[3][k], ex.v[4][k],
                                 ex.v[5][k], ex.v[6][k], ex.v[7][k], vzz[k]};
#pragma unroll
            for (int co = 0; co < 3; co++)
#pragma unroll
                for (int ro = 0; ro < 3; ro++) dot[co] += m[3 * co + ro] * s[3 * j + ro];
        }
    }
    ch[3 * i] = hd[3 * i] + dot[0];
    ch[3 * i + 1] = hd[3 * i + 1] + dot[1];
    ch[3 * i + 2] = hd[3 * i + 2] + dot[2];
}

// Row-aligned DIA, values v[c][d*N+row], bounds-checked column (src/cufields.cu:97-178 semantics).
template <bool FULL>
__global__ void plain_spmv_dia(uint32_t n, uint32_t ndiag, const int32_t* __restrict__ off, PlainExch ex,
                               const double* __restrict__ s, const double* __restrict__ hd,
                               double* __restrict__ ch, int zz_from_yy) {
    const uint32_t row = blockIdx.x * blockDim.x + threadIdx.x;
    if (row >= n) return;
    double dot[3] = {0.0, 0.0, 0.0};
    const double* vzz = zz_from_yy ? ex.v[4] : ex.v[8];
    for (uint32_t d = 0; d < ndiag; d++) {
        const int64_t col = (int64_t)row + off[d];
        const size_t a = (size_t)d * n + row;
        if (col < 0 || col >= (int64_t)n) continue;
        if (!FULL) {
            dot[0] += ex.v[0][a] * s[3 * col];
            dot[1] += ex.v[4][a] * s[3 * col + 1];
            dot[2] += vzz[a] * s[3 * col + 2];
        } else {
            const double m[9] = {ex.v[0][a], ex.v[1][a], ex.v[2][a], ex.v[3][a], ex.v[4][a],
                                 ex.v[5][a], ex.v[6][a], ex.v[7][a], vzz[a]};
#pragma unroll
            for (int co = 0; co < 3; co++)
#pragma unroll
                for (int ro = 0; ro < 3; ro++) dot[co] += m[3 * co + ro] * s[3 * col + ro];
        }
    }
    ch[3 * row] = hd[3 * row] + dot[0];
    ch[3 * row + 1] = hd[3 * row + 1] + dot[1];
    ch[3 * row + 2] = hd[3 * row + 2] + dot[2];
}

struct PlainSpin {
    const double *sigma, *llgpf, *lambda, *k1u, *k1udir, *hstg;
};

// Total field of one spin (src/cuint.cu:66-137 order): CH + site + thermal + applied + anisotropy.
__device__ __forceinline__ void plain_total_field(const StepConst& c, const PlainSpin& ps, uint32_t i,
                                                  const double* ch, const double* rnd, const double s[3],
                                                  double h[3], double lrn[3]) {
    const uint32_t r = replica_of(c, i);
    const double TP = c.rep_sqrtT[r] * ps.sigma[i];
    lrn[0] = rnd[3 * i] * TP;
    lrn[1] = rnd[3 * i + 1] * TP;
    lrn[2] = rnd[3 * i + 2] * TP;
    const double* ap = c.dyn + DYN_APPLIED;
    h[0] = ch[3 * i] + ps.hstg[3 * i] + lrn[0] + ap[0];
    h[1] = ch[3 * i + 1] + ps.hstg[3 * i + 1] + lrn[1] + ap[1];
    h[2] = ch[3 * i + 2] + ps.hstg[3 * i + 2] + lrn[2] + ap[2];
    const double d[3] = {ps.k1udir[3 * i], ps.k1udir[3 * i + 1], ps.k1udir[3 * i + 2]};
    const double k1u = ps.k1u[i];
    const double sdn = s[0] * d[0] + s[1] * d[1] + s[2] * d[2];
    h[0] += (k1u * sdn * d[0]);
    h[1] += (k1u * sdn * d[1]);
    h[2] += (k1u * sdn * d[2]);
    const double sdk2perp = s[0] * c.k2perpdir[0] + s[1] * c.k2perpdir[1] + s[2] * c.k2perpdir[2];
    for (int a = 0; a < 3; a++) h[a] += c.k2perp_f * sdk2perp * c.k2perpdir[a];
    const double sdk2par = s[0] * c.k2pardir[0] + s[1] * c.k2pardir[1] + s[2] * c.k2pardir[2];
    for (int a = 0; a < 3; a++) h[a] += c.k2par_f * sdk2par * c.k2pardir[a];
    for (int dir = 0; dir < 3; dir++) {
        const double* pd = c.k4perpdirs + 3 * dir;
        const double* qd = c.k4pardirs + 3 * dir;
        const double sdk4perp = s[0] * pd[0] + s[1] * pd[1] + s[2] * pd[2];
        const double sdk4par = s[0] * qd[0] + s[1] * qd[1] + s[2] * qd[2];
        for (int a = 0; a < 3; a++) h[a] += c.k4perp_f * sdk4perp * pd[a];
        for (int a = 0; a < 3; a++) h[a] += c.k4par_f * sdk4par * qd[a];
    }
}

__device__ __forceinline__ void plain_torque(double scale, double llgpf, double lambda, const double s[3],
                                             const double h[3], double f[3]) {
    const double sxh[3] = {s[1] * h[2] - s[2] * h[1], s[2] * h[0] - s[0] * h[2], s[0] * h[1] - s[1] * h[0]};
    const double sxsxh[3] = {s[1] * sxh[2] - s[2] * sxh[1], s[2] * sxh[0] - s[0] * sxh[2],
                             s[0] * sxh[1] - s[1] * sxh[0]};
    for (int j = 0; j < 3; j++) {
        if (scale == 1.0) f[j] = llgpf * (sxh[j] + lambda * sxsxh[j]);
        else f[j] = scale * llgpf * (sxh[j] + lambda * sxsxh[j]);
    }
}

__device__ __forceinline__ void plain_normalise(double v[3]) {
    const double mods = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    v[0] /= mods; v[1] /= mods; v[2] /= mods;
}

// Heun predictor (src/cuint.cu:60-163 semantics).
__global__ void plain_heun1(StepConst c, PlainSpin ps, const double* __restrict__ ch, const double* __restrict__ sp,
                            double* __restrict__ es, const double* __restrict__ rnd, double* __restrict__ fn) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= c.n) return;
    const double s[3] = {sp[3 * i], sp[3 * i + 1], sp[3 * i + 2]};
    double h[3], lrn[3], f[3], e[3];
    plain_total_field(c, ps, i, ch, rnd, s, h, lrn);
    plain_torque(1.0, ps.llgpf[i], ps.lambda[i], s, h, f);
    for (int j = 0; j < 3; j++) { fn[3 * i + j] = f[j]; e[j] = s[j] + f[j] * c.rdt; }
    plain_normalise(e);
    es[3 * i] = e[0]; es[3 * i + 1] = e[1]; es[3 * i + 2] = e[2];
}

// Heun corrector + det field (src/cuint.cu:165-242 semantics).
__global__ void plain_heun2(StepConst c, PlainSpin ps, const double* __restrict__ ch, double* __restrict__ sp,
                            const double* __restrict__ es, const double* __restrict__ rnd,
                            const double* __restrict__ fn, double* __restrict__ det) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= c.n) return;
    const double e[3] = {es[3 * i], es[3 * i + 1], es[3 * i + 2]};
    double h[3], lrn[3], f[3], p[3];
    plain_total_field(c, ps, i, ch, rnd, e, h, lrn);
    plain_torque(1.0, ps.llgpf[i], ps.lambda[i], e, h, f);
    for (int j = 0; j < 3; j++) p[j] = sp[3 * i + j] + (0.5 * (fn[3 * i + j] + f[j]) * c.rdt);
    plain_normalise(p);
    for (int j = 0; j < 3; j++) {
        sp[3 * i + j] = p[j];
        det[3 * i + j] = h[j] - lrn[j];
    }
}

struct RkBufs {
    double* k[6];
};

__constant__ double RK5B[5][5] = {
    {0.2, 0, 0, 0, 0},
    {3.0 / 40.0, 9.0 / 40.0, 0, 0, 0},
    {0.3, -0.9, 1.2, 0, 0},
    {-11.0 / 54, 2.5, -70.0 / 27.0, 35.0 / 27.0, 0},
    {1631.0 / 55296.0, 175.0 / 512.0, 575.0 / 13824.0, 44275.0 / 110592.0, 253.0 / 4096.0}};
__constant__ double RK5C[6] = {37.0 / 378.0, 0.0, 250.0 / 621.0, 125.0 / 594.0, 0.0, 512.0 / 1771.0};

// One RK stage: k_st = rdt f(stage spin, H), next stage spin (src/cuintRK4.cu:62-434,
// src/cuintRK5.cu:79-628 semantics; quirks selected by flags).
__global__ void plain_rk_stage(StepConst c, PlainSpin ps, int nst, int st, const double* __restrict__ ch,
                               const double* __restrict__ sp, double* __restrict__ es,
                               const double* __restrict__ rnd, RkBufs kb) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= c.n) return;
    const bool dbl = (c.flags & ASD_FLAG_RK_DOUBLE_RDT) != 0;
    const bool mixed = (c.flags & ASD_FLAG_RK_STAGE_SPIN_MIXED) != 0;
    const double S[3] = {sp[3 * i], sp[3 * i + 1], sp[3 * i + 2]};
    double sv[3];
    if (st == 0) { sv[0] = S[0]; sv[1] = S[1]; sv[2] = S[2]; }
    else if (mixed) { sv[0] = es[3 * i]; sv[1] = S[1]; sv[2] = es[3 * i + 2]; }
    else { sv[0] = es[3 * i]; sv[1] = es[3 * i + 1]; sv[2] = es[3 * i + 2]; }
    double h[3], lrn[3], k[3];
    plain_total_field(c, ps, i, ch, rnd, sv, h, lrn);
    plain_torque(c.rdt, ps.llgpf[i], ps.lambda[i], sv, h, k);
    for (int j = 0; j < 3; j++) kb.k[st][3 * i + j] = k[j];
    if (st == nst - 1) return;
    double e[3];
    for (int j = 0; j < 3; j++) {
        double inc;
        const size_t q = 3 * (size_t)i + j;
        if (nst == 4) {
            if (dbl) inc = st == 2 ? c.rdt * k[j] : c.rdt * k[j] * 0.5;
            else inc = k[j] * (st == 2 ? 1.0 : 0.5);
        } else {
            double sum;
            if (st == 0) sum = RK5B[0][0] * k[j];
            else if (st == 1) sum = RK5B[1][0] * kb.k[0][q] + RK5B[1][1] * k[j];
            else if (st == 2) sum = RK5B[2][0] * kb.k[0][q] + RK5B[2][1] * kb.k[1][q] + RK5B[2][2] * k[j];
            else if (st == 3)
                sum = RK5B[3][0] * kb.k[0][q] + RK5B[3][1] * kb.k[1][q] + RK5B[3][2] * kb.k[2][q] + RK5B[3][3] * k[j];
            else
                sum = RK5B[4][0] * kb.k[0][q] + RK5B[4][1] * kb.k[1][q] + RK5B[4][2] * kb.k[2][q] +
                      RK5B[4][3] * kb.k[3][q] + RK5B[4][4] * k[j];
            inc = dbl ? c.rdt * sum : sum;
        }
        e[j] = S[j] + inc;
    }
    plain_normalise(e);
    es[3 * i] = e[0]; es[3 * i + 1] = e[1]; es[3 * i + 2] = e[2];
}

// Final combination + renormalisation (CdetSnp1, src/cuintRK4.cu:436-456, src/cuintRK5.cu:630-649).
__global__ void plain_rk_final(uint32_t n, int nst, double* __restrict__ sp, RkBufs kb) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double ls[3];
    for (int j = 0; j < 3; j++) {
        const size_t q = 3 * (size_t)i + j;
        if (nst == 4)
            ls[j] = sp[q] + kb.k[0][q] * (1.0 / 6.0) + kb.k[1][q] * (1.0 / 3.0) + kb.k[2][q] * (1.0 / 3.0) +
                    kb.k[3][q] * (1.0 / 6.0);
        else
            ls[j] = sp[q] + kb.k[0][q] * RK5C[0] + kb.k[1][q] * RK5C[1] + kb.k[2][q] * RK5C[2] +
                    kb.k[3][q] * RK5C[3] + kb.k[4][q] * RK5C[4] + kb.k[5][q] * RK5C[5];
    }
    plain_normalise(ls);
    sp[3 * i] = ls[0]; sp[3 * i + 1] = ls[1]; sp[3 * i + 2] = ls[2];
}

// Site field ramp (CincStagFields, src/cufields.cu:46-56).
__global__ void plain_ramp(uint32_t n, double rv, const double* __restrict__ init, double* __restrict__ hs) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= 3 * n) return;
    hs[i] = rv * init[i];
}

// ---- long-range field, reference-structured FP64 complex pipeline ----
__global__ void plain_zero_c(size_t m, double2* __restrict__ a) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < m) a[i] = make_double2(0.0, 0.0);
}

__global__ void plain_scatter(uint32_t n, size_t P, const double* __restrict__ s, const float* __restrict__ w,
                              const uint32_t* __restrict__ midx, double2* __restrict__ zr) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const size_t m = midx[i];
    const double wi = (double)w[i];
    for (int c = 0; c < 3; c++) zr[c * P + m].x = s[3 * i + c] * wi;
}

// H_k[a] = sum_b N_k[a][b] S_k[b], complex, 9 components (src/cufields.cu:294-330 semantics).
__global__ void plain_kconv9(size_t P, const double2* __restrict__ nk, const double2* __restrict__ sk,
                             double2* __restrict__ hk) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P) return;
    for (int a = 0; a < 3; a++) {
        double2 acc = make_double2(0.0, 0.0);
        for (int b = 0; b < 3; b++) {
            const double2 nn = nk[(size_t)(3 * a + b) * P + i];
            const double2 ss = sk[(size_t)b * P + i];
            acc.x += (nn.x * ss.x - nn.y * ss.y);
            acc.y += (nn.x * ss.y + nn.y * ss.x);
        }
        hk[(size_t)a * P + i] = acc;
    }
}

__global__ void plain_gather(uint32_t n, size_t P, const double2* __restrict__ zr, const uint32_t* __restrict__ midx,
                             double* __restrict__ out, int as_float) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const size_t m = midx[i];
    for (int c = 0; c < 3; c++) {
        double v = zr[c * P + m].x / (double)P;
        if (as_float) v = (double)(float)v;
        out[3 * i + c] = v;
    }
}

inline unsigned nb(size_t n, int b) { return (unsigned)((n + b - 1) / b); }

}  // namespace

// Long-range field of spins s into out (3N AoS) via the padded FP64 complex FFTs.
cudaError_t launch_lr_eval_plain(asd_handle* h, const double* s, double* out, bool as_demag) {
    LongRange& L = h->lr;
    const int B = 256;
    cudaStream_t st = h->stream;
    plain_zero_c<<<nb(3 * L.P, B), B, 0, st>>>(3 * L.P, L.zr);
    plain_scatter<<<nb(h->n, B), B, 0, st>>>(h->n, L.P, s, L.w, L.mesh_idx, L.zr);
    h->launches += 2;
    if (cufftExecZ2Z(L.z2z, (cufftDoubleComplex*)L.zr, (cufftDoubleComplex*)L.zk, CUFFT_FORWARD) != CUFFT_SUCCESS)
        return cudaErrorUnknown;
    plain_kconv9<<<nb(L.P, B), B, 0, st>>>(L.P, L.znk, L.zk, L.zh);
    h->launches += 1;
    if (cufftExecZ2Z(L.z2z, (cufftDoubleComplex*)L.zh, (cufftDoubleComplex*)L.zr, CUFFT_INVERSE) != CUFFT_SUCCESS)
        return cudaErrorUnknown;
    const int as_float = as_demag && (h->p.flags & ASD_FLAG_GPU_HDEMAG_FP32) ? 1 : 0;
    plain_gather<<<nb(h->n, B), B, 0, st>>>(h->n, L.P, L.zr, L.mesh_idx, out, as_float);
    h->launches += 1;
    return cudaGetLastError();
}

// CH += four-spin field (src/cufields.cu:59-90; launched after the SpMV as src/cuda.cu:143-146).
__global__ void plain_four_spin(const StepConst c, const double* __restrict__ s, double* __restrict__ ch) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= c.n) return;
    double h4[3];
    four_spin<double>(c, i, [&](uint32_t j, double v[3]) { v[0] = s[3 * (size_t)j]; v[1] = s[3 * (size_t)j + 1]; v[2] = s[3 * (size_t)j + 2]; }, h4);
    ch[3 * (size_t)i] += h4[0];
    ch[3 * (size_t)i + 1] += h4[1];
    ch[3 * (size_t)i + 2] += h4[2];
}

static cudaError_t plain_field_exch(asd_handle* h, const double* s, double* ch);

static cudaError_t plain_field(asd_handle* h, const double* s, double* ch) {
    cudaError_t e = plain_field_exch(h, s, ch);
    if (e != cudaSuccess || !h->sc.q4_ptr) return e;
    plain_four_spin<<<nb(h->n, 256), 256, 0, h->stream>>>(h->sc, s, ch);
    h->launches += 1;
    return cudaGetLastError();
}

static cudaError_t plain_field_exch(asd_handle* h, const double* s, double* ch) {
    const int B = 256;
    cudaStream_t st = h->stream;
    const int zz = (h->p.flags & ASD_FLAG_GPU_DZZ_FROM_DYY) ? 1 : 0;
    if (h->lr.mode == ASD_LR_FFT) return launch_lr_eval_plain(h, s, ch, false);
    if (h->exch == ASD_EXCH_CSR) {
        if (h->full) plain_spmv_csr<true><<<nb(h->n, B), B, 0, st>>>(h->n, h->pex.xadj, h->pex.adjncy, h->pex, s, h->p_hdemag, ch, zz);
        else plain_spmv_csr<false><<<nb(h->n, B), B, 0, st>>>(h->n, h->pex.xadj, h->pex.adjncy, h->pex, s, h->p_hdemag, ch, zz);
    } else if (h->exch == ASD_EXCH_DIA) {
        if (h->full) plain_spmv_dia<true><<<nb(h->n, B), B, 0, st>>>(h->n, h->pex.ndiag, h->pex.off, h->pex, s, h->p_hdemag, ch, zz);
        else plain_spmv_dia<false><<<nb(h->n, B), B, 0, st>>>(h->n, h->pex.ndiag, h->pex.off, h->pex, s, h->p_hdemag, ch, zz);
    } else {
        cudaMemcpyAsync(ch, h->p_hdemag, 3 * (size_t)h->n * sizeof(double), cudaMemcpyDeviceToDevice, st);
        return cudaGetLastError();
    }
    h->launches += 1;
    return cudaGetLastError();
}

cudaError_t launch_plain_step(asd_handle* h, uint64_t t) {
    const int B = 256;
    cudaStream_t st = h->stream;
    cudaError_t e;
    PlainSpin ps{h->p_sigma, h->p_llgpf, h->p_lambda, h->p_k1u, h->p_k1udir, h->p_hstg};
    const uint32_t upd = h->p.update ? h->p.update : 1;
    const bool dip_refresh = h->lr.mode == ASD_LR_DIPOLE && (t % upd) == 0;
    if (h->d_ttm && (e = launch_ttm_step(h, nullptr, t)) != cudaSuccess) return e;
    if (h->pulse_amp != 0.0 && h->has_site) {
        // the driver-side rampStag of every step (src/cuda.cu:38-41) with the pulse envelope
        const double x = ((double)t * h->p.dt - h->pulse_t0) / h->pulse_sigma;
        const double f = h->pulse_amp * exp(-0.5 * x * x);
        if ((e = launch_plain_ramp(h, h->stag_rv * f)) != cudaSuccess) return e;
    }
    if (h->p.integrator == ASD_HEUN) {
        if (dip_refresh && (e = launch_lr_eval_plain(h, h->p_s, h->p_hdemag, true)) != cudaSuccess) return e;
        if ((e = plain_field(h, h->p_s, h->p_ch)) != cudaSuccess) return e;
        plain_noise_k<<<nb(h->n, B), B, 0, st>>>(h->sc, t, h->p_rand);
        plain_heun1<<<nb(h->n, B), B, 0, st>>>(h->sc, ps, h->p_ch, h->p_s, h->p_es, h->p_rand, h->p_fn);
        h->launches += 2;
        const bool stale = (h->p.flags & ASD_FLAG_GPU_CSR_DIP_STALE) && h->lr.mode == ASD_LR_DIPOLE &&
                           h->exch == ASD_EXCH_CSR && !h->full;
        if (!stale && (e = plain_field(h, h->p_es, h->p_ch)) != cudaSuccess) return e;
        plain_heun2<<<nb(h->n, B), B, 0, st>>>(h->sc, ps, h->p_ch, h->p_s, h->p_es, h->p_rand, h->p_fn, h->p_det);
        h->launches += 1;
        return cudaGetLastError();
    }
    const int nst = h->p.integrator == ASD_RK4 ? 4 : 6;
    RkBufs kb;
    for (int q = 0; q < 6; q++) kb.k[q] = h->p_k[q];
    plain_noise_k<<<nb(h->n, B), B, 0, st>>>(h->sc, t, h->p_rand);
    h->launches += 1;
    if (dip_refresh && (e = launch_lr_eval_plain(h, h->p_s, h->p_hdemag, true)) != cudaSuccess) return e;
    for (int s = 0; s < nst; s++) {
        if ((e = plain_field(h, s == 0 ? h->p_s : h->p_es, h->p_ch)) != cudaSuccess) return e;
        plain_rk_stage<<<nb(h->n, B), B, 0, st>>>(h->sc, ps, nst, s, h->p_ch, h->p_s, h->p_es, h->p_rand, kb);
        h->launches += 1;
    }
    plain_rk_final<<<nb(h->n, B), B, 0, st>>>(h->n, nst, h->p_s, kb);
    h->launches += 1;
    return cudaGetLastError();
}

cudaError_t launch_plain_ramp(asd_handle* h, double rv) {
    plain_ramp<<<nb(3 * (size_t)h->n, 256), 256, 0, h->stream>>>(h->n, rv, h->p_hinit, h->p_hstg);
    h->launches += 1;
    return cudaGetLastError();
}

// Field of the current spins with the long-range part as currently held (CHDemag semantics).
cudaError_t launch_plain_field(asd_handle* h, double* out) { return plain_field(h, h->p_s, out); }

__global__ void normals_k(uint64_t seed, uint32_t stream, uint64_t step, uint32_t n, double* out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double xi[3];
    thermal_normals(seed, stream, i, step, xi);
    out[3 * i] = xi[0]; out[3 * i + 1] = xi[1]; out[3 * i + 2] = xi[2];
}

cudaError_t launch_thermal_normals(uint64_t seed, uint32_t stream, uint64_t step, uint32_t n, double* d_out,
                                   cudaStream_t st) {
    normals_k<<<nb(n, 256), 256, 0, st>>>(seed, stream, step, n, d_out);
    return cudaGetLastError();
}

__global__ void normals_f_k(uint64_t seed, uint32_t stream, uint64_t step, uint32_t n, float* out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float xi[3];
    thermal_normals_f(seed, stream, i, step, xi);
    out[3 * i] = xi[0]; out[3 * i + 1] = xi[1]; out[3 * i + 2] = xi[2];
}

cudaError_t launch_thermal_normals_f(uint64_t seed, uint32_t stream, uint64_t step, uint32_t n, float* d_out,
                                     cudaStream_t st) {
    normals_f_k<<<nb(n, 256), 256, 0, st>>>(seed, stream, step, n, d_out);
    return cudaGetLastError();
}

}  // namespace asd
