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

__global__ void scatter_k(uint32_t n, size_t P, const float* __restrict__ sx, const float* __restrict__ sy,
                          const float* __restrict__ sz, const float* __restrict__ w, const uint32_t* __restrict__ idx,
                          float* __restrict__ mr) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t m = idx[i];
    const float wv = w[i];
    mr[m] = sx[i] * wv;
    mr[P + m] = sy[i] * wv;
    mr[2 * P + m] = sz[i] * wv;
}

// Largest |Re| and |Im| of the FP64 half spectrum (non-negative doubles order like their bits).
__global__ void nk_extent(size_t m, const double2* __restrict__ z, unsigned long long* mx) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    double re = 0.0, im = 0.0;
    if (i < m) { re = fabs(z[i].x); im = fabs(z[i].y); }
    for (int o = 16; o > 0; o >>= 1) {
        re = fmax(re, __shfl_xor_sync(0xffffffffu, re, o));
        im = fmax(im, __shfl_xor_sync(0xffffffffu, im, o));
    }
    if ((threadIdx.x & 31) == 0) {
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

}  // namespace

cudaError_t launch_lr_scatter_f32(asd_handle* h, const float* const s[3]) {
    LongRange& L = h->lr;
    scatter_k<<<nb(h->n, 256), 256, 0, h->stream>>>(h->n, L.P, s[0], s[1], s[2], L.w, L.mesh_idx, L.r);
    h->launches += 1;
    return cudaGetLastError();
}

// M_r -> (R2C) -> N_k . M_k -> (C2R) -> H_r
cudaError_t launch_lr_eval_f32(asd_handle* h) {
    LongRange& L = h->lr;
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
    const int* n = nullptr; (void)n;
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
    nk_extent<<<nb(nc * L.Pk, 256), 256, 0, h->stream>>>(nc * L.Pk, z, mx);
    unsigned long long hm[2] = {0, 0};
    cudaMemcpyAsync(hm, mx, sizeof(hm), cudaMemcpyDeviceToHost, h->stream);
    cudaStreamSynchronize(h->stream);
    double re, im;
    memcpy(&re, &hm[0], 8); memcpy(&im, &hm[1], 8);
    L.nk_real = (im <= 1e-9 * re) ? 1 : 0;
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
