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
