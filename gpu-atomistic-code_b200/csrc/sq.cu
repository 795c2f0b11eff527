// In-situ S(q,t) sampler: the spin-map transform of the reference's timeseries driver
// (src/timeseries.cpp:274-330).  Each sample forms psi(r) = uo_a S_a + i uo_b S_b on the
// lattice mesh, with (a, b) the axes transverse to the quantisation axis and uo the
// per-sublattice sign (src/sf_glob.cpp), transforms it forward in 3D (cuFFT Z2Z, the sign
// convention of FFTW_FORWARD) and appends psi_k at the chosen k-points to a series kept in
// device memory; the host reads the series once at the end.
#include "internal.h"

namespace asd {
namespace {

inline unsigned nb(size_t n, int b) { return (unsigned)((n + b - 1) / b); }

template <typename R>
__global__ void sq_scatter(uint32_t n, const R* __restrict__ sx, const R* __restrict__ sy, const R* __restrict__ sz,
                           const float* __restrict__ lx, const float* __restrict__ ly, const float* __restrict__ lz,
                           const double* __restrict__ aos, const uint32_t* __restrict__ idx,
                           const uint32_t* __restrict__ sub_of_spin, const double* __restrict__ uo, int a, int b,
                           double2* __restrict__ grid) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double s[3];
    if (aos) {
        s[0] = aos[3 * (size_t)i]; s[1] = aos[3 * (size_t)i + 1]; s[2] = aos[3 * (size_t)i + 2];
    } else {
        s[0] = (double)sx[i]; s[1] = (double)sy[i]; s[2] = (double)sz[i];
        if (lx) { s[0] += (double)lx[i]; s[1] += (double)ly[i]; s[2] += (double)lz[i]; }
    }
    const uint32_t sl = sub_of_spin[i];
    grid[idx[i]] = make_double2(s[a] * uo[3 * sl + a], s[b] * uo[3 * sl + b]);
}

__global__ void sq_gather(uint32_t nk, const uint32_t* __restrict__ kidx, const double2* __restrict__ grid,
                          double2* __restrict__ row) {
    const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q < nk) row[q] = grid[kidx[q]];
}

}  // namespace

cudaError_t launch_sq_sample(asd_handle* h) {
    SqSampler& S = h->sq;
    cudaError_t e = cudaMemsetAsync(S.grid, 0, sizeof(double2) * S.P, h->stream);
    if (e != cudaSuccess) return e;
    const int a = S.qaxis == 0 ? 1 : 0, b = S.qaxis == 2 ? 1 : 2;
    const unsigned g = nb(h->n, 256);
    if (h->p.precision == ASD_FP64_PLAIN) {
        sq_scatter<double><<<g, 256, 0, h->stream>>>(h->n, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, h->p_s,
                                                      S.idx, S.sub, S.uo, a, b, S.grid);
    } else if (h->p.precision == ASD_FP32) {
        const bool comp = (h->p.flags & ASD_FLAG_COMPENSATED) != 0;
        sq_scatter<float><<<g, 256, 0, h->stream>>>(h->n, h->sf[0], h->sf[1], h->sf[2], comp ? h->sl[0] : nullptr,
                                                     comp ? h->sl[1] : nullptr, comp ? h->sl[2] : nullptr, nullptr,
                                                     S.idx, S.sub, S.uo, a, b, S.grid);
    } else {
        sq_scatter<double><<<g, 256, 0, h->stream>>>(h->n, h->sd[0], h->sd[1], h->sd[2], nullptr, nullptr, nullptr,
                                                      nullptr, S.idx, S.sub, S.uo, a, b, S.grid);
    }
    h->launches += 1;
    if (cufftExecZ2Z(S.plan, (cufftDoubleComplex*)S.grid, (cufftDoubleComplex*)S.grid, CUFFT_FORWARD) != CUFFT_SUCCESS)
        return cudaErrorUnknown;
    sq_gather<<<nb(S.nk, 128), 128, 0, h->stream>>>(S.nk, S.kidx, S.grid, S.series + (size_t)S.nsamples * S.nk);
    h->launches += 1;
    S.nsamples++;
    return cudaGetLastError();
}

}  // namespace asd

namespace asd {
namespace {

// Windowed copy of the series, laid out [k][t] so each k-point is one contiguous FFT batch.
__global__ void sq_window_k(uint32_t ns, uint32_t nk, const double2* __restrict__ series, int window, double alpha,
                            double beta, double2* __restrict__ out) {
    const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (size_t)ns * nk) return;
    const uint32_t t = (uint32_t)(e / nk), k = (uint32_t)(e % nk);
    double2 v = series[e];
    if (window == 1) {
        const double w = alpha - beta * cos(2.0 * M_PI * (double)t / ((double)ns - 1.0));
        v.x *= w;
        v.y *= w;
    }
    out[(size_t)k * ns + t] = v;
}

// One-sided PSD with the time-series tool's pairing of w with ns-1-w.
__global__ void sq_psd(uint32_t ns, uint32_t nk, const double2* __restrict__ X, double norm, double* __restrict__ raw) {
    const uint32_t half = ns / 2;
    const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (size_t)half * nk) return;
    const uint32_t k = (uint32_t)(e / half), w = (uint32_t)(e % half);
    const double2 a = X[(size_t)k * ns + w], b = X[(size_t)k * ns + (ns - 1 - w)];
    const double ax = a.x / norm, ay = a.y / norm, bx = b.x / norm, by = b.y / norm;
    raw[e] = (ax * ax + ay * ay) + (bx * bx + by * by);
}

// Recursive Gaussian (Alvarez and Mazorra, SIAM J. Numer. Anal. 31, 590 (1994)) and the peak
// search, one thread per k-point: the recursion is sequential along the frequency axis.
__global__ void sq_smooth_peaks(uint32_t half, uint32_t nk, const double* __restrict__ raw, double* __restrict__ sm,
                                double sigma, int nsteps, double wscale, double flo, double fhi,
                                uint32_t* __restrict__ praw, uint32_t* __restrict__ psm) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nk) return;
    const double* r = raw + (size_t)k * half;
    double* d = sm + (size_t)k * half;
    for (uint32_t i = 0; i < half; i++) d[i] = r[i];
    const double lam = (sigma * sigma) / (2.0 * nsteps);
    const double nu = (1.0 + 2.0 * lam - sqrt(1.0 + 4.0 * lam)) / (2.0 * lam);
    const double bscale = 1.0 / (1.0 - nu), post = pow(nu / lam, (double)nsteps);
    for (int s = 0; s < nsteps; s++) {
        d[0] *= bscale;
        for (uint32_t i = 1; i < half; i++) d[i] += nu * d[i - 1];
        d[half - 1] *= bscale;
        for (uint32_t i = half - 1; i > 0; i--) d[i - 1] += nu * d[i];
    }
    for (uint32_t i = 0; i < half; i++) d[i] *= post;
    double mr = 0.0, ms = 0.0;
    uint32_t ir = 0, is = 0;
    for (uint32_t w = 0; w < half; w++) {
        const double f = (double)w * wscale;
        const bool in = f > flo && f < fhi;
        if (d[w] > ms && in) { ms = d[w]; is = w; }
        if (r[w] > mr && w > 1 && in) { mr = r[w]; ir = w; }
    }
    praw[k] = ir;
    psm[k] = is;
}

}  // namespace

cudaError_t launch_sq_spectrum(asd_handle* h, int window, double alpha, double beta, uint32_t pixelwidth,
                               double sample_dt, double flo, double fhi, double* d_raw, double* d_smooth,
                               uint32_t* d_peaks) {
    SqSampler& S = h->sq;
    const uint32_t ns = S.nsamples, nk = S.nk, half = ns / 2;
    double2* X = nullptr;
    cudaError_t e = cudaMalloc(&X, sizeof(double2) * (size_t)ns * nk);
    if (e != cudaSuccess) return e;
    cufftHandle plan = 0;
    int n1[1] = {(int)ns};
    bool ok = cufftPlanMany(&plan, 1, n1, nullptr, 1, (int)ns, nullptr, 1, (int)ns, CUFFT_Z2Z, (int)nk) ==
                  CUFFT_SUCCESS &&
              cufftSetStream(plan, h->stream) == CUFFT_SUCCESS;
    if (ok) {
        sq_window_k<<<nb((size_t)ns * nk, 256), 256, 0, h->stream>>>(ns, nk, S.series, window, alpha, beta, X);
        ok = cufftExecZ2Z(plan, (cufftDoubleComplex*)X, (cufftDoubleComplex*)X, CUFFT_FORWARD) == CUFFT_SUCCESS;
    }
    if (ok) {
        sq_psd<<<nb((size_t)half * nk, 256), 256, 0, h->stream>>>(ns, nk, X, (double)S.P * (double)ns, d_raw);
        sq_smooth_peaks<<<nb(nk, 64), 64, 0, h->stream>>>(half, nk, d_raw, d_smooth, (double)pixelwidth, 10,
                                                          2.0 * M_PI / ((double)ns * sample_dt), flo, fhi, d_peaks,
                                                          d_peaks + nk);
        h->launches += 3;
    }
    const cudaError_t le = cudaGetLastError();
    const cudaError_t se = cudaStreamSynchronize(h->stream);   // the plan's work area is in use until here
    if (plan) cufftDestroy(plan);
    cudaFree(X);
    if (!ok) return cudaErrorUnknown;
    return le != cudaSuccess ? le : se;
}

}  // namespace asd
