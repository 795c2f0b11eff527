// Test-infrastructure harness around the reference's own CUDA step kernels.
//
// Compiled together with the reference sources src/cuint.cu (CHeun1/CHeun2),
// src/cufields.cu (CSpMV_CSR/_OffDiag, CSpMV_DIA/_OffDiag, CSpMV_CSR_FourSpin),
// src/cuintRK4.cu and src/cuintRK5.cu exactly where they lie in the reference
// tree (see oracle/Makefile), and with ref_harness.cpp (+ the reference's
// llgCPU sources it needs), whose refh_* calls fill the namespace globals the
// reference's copyConstData() functions read.  This file allocates the device
// arrays the reference's cuda_util.cu would allocate (same layouts: AoS
// [3*i+c] doubles for spins/fields, per-spin sigma/llgpf/lambda/k1u, float
// Crand of 3N rounded up to even, float CHDemag) and replays the launch
// sequences of cullg::llgGPU (src/cuda.cu:43-258, branch exchm>0 without the
// FFT dipole), cullg::llgGPURK4 (src/cudaRK4.cu:38-233) and cullg::llgGPURK5
// (src/cudaRK5.cu).  The noise comes from the caller (Crand), not cuRAND.
// It is a parity pin for the product and the oracle; nothing in the product
// links it.
#include <cuda_runtime.h>
#include <cufft.h>
#include <curand.h>
#include <libconfig.h++>
#include "../inc/arrays.h"
#include "../inc/exch.h"
#include "../inc/config.h"
#include "../inc/geom.h"
#include "../inc/fields.h"
#include "../inc/spins.h"
#include "../inc/llg.h"
#include "../inc/anis.h"
#include "../inc/cuint.h"
#include "../inc/cufields.h"
#include "../inc/cuintRK4.h"
#include "../inc/cuintRK5.h"
#include <cstring>
#include <vector>

// Read by cufields::copyConstData (src/cufields.cu:31-43); only the FFT kernels use them.
namespace geom {
unsigned int zpdim[3] = {0, 0, 0};
Array<unsigned int> Nk;
}

namespace {
struct Dev {
    unsigned n = 0, block = 128, curand_n = 0;
    double *spin = nullptr, *espin = nullptr, *h = nullptr, *fn = nullptr, *det = nullptr, *hstg = nullptr;
    double *sigma = nullptr, *llgpf = nullptr, *lambda = nullptr, *k1u = nullptr, *k1udir = nullptr;
    double *rk[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
    float *rand = nullptr, *hdemag = nullptr;
    unsigned *xadj = nullptr, *adjncy = nullptr;
    int *offset = nullptr;
    double *d[9] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
    unsigned *q_xadj = nullptr, *q_j = nullptr, *q_k = nullptr, *q_l = nullptr;
    std::vector<void*> owned;
};
Dev g;
curandGenerator_t gen = nullptr;   // set: every step draws Crand as src/cuda.cu:148 does

template <class T>
T* upload(const T* src, size_t n) {
    T* p = nullptr;
    if (cudaMalloc((void**)&p, (n ? n : 1) * sizeof(T)) != cudaSuccess) p = nullptr;
    g.owned.push_back(p);  // a failed allocation is recorded as nullptr and fails refg_init
    if (!p) return nullptr;
    if (src) cudaMemcpy(p, src, n * sizeof(T), cudaMemcpyHostToDevice);
    else cudaMemset(p, 0, (n ? n : 1) * sizeof(T));
    return p;
}

std::vector<double> aos(const Array<double>& x, const Array<double>& y, const Array<double>& z, unsigned n) {
    std::vector<double> v(3 * (size_t)n);
    for (unsigned i = 0; i < n; i++) { v[3 * i] = x[i]; v[3 * i + 1] = y[i]; v[3 * i + 2] = z[i]; }
    return v;
}

void release() {
    for (void* p : g.owned)
        if (p) cudaFree(p);
    g = Dev();
}

int status() {
    cudaError_t e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaGetLastError();
    return e == cudaSuccess ? 0 : -(int)e;
}

// The exchange SpMV of src/cuda.cu:118-140 on spins s (overwrites CH with CHDemag + J.s).
void spmv(double* s) {
    const unsigned nb = (g.n + g.block - 1) / g.block;
    if (config::exchm == 1) {
        if (!config::offdiag)
            cufields::CSpMV_DIA<<<nb, g.block>>>(g.n, g.offset, g.d[0], g.d[4], g.d[8], s, g.hdemag, g.h);
        else
            cufields::CSpMV_DIA_OffDiag<<<nb, g.block>>>(g.n, g.offset, g.d[0], g.d[1], g.d[2], g.d[3], g.d[4], g.d[5],
                                                         g.d[6], g.d[7], g.d[8], s, g.hdemag, g.h);
    } else {
        if (!config::offdiag)
            cufields::CSpMV_CSR<<<nb, g.block>>>(g.n, g.xadj, g.adjncy, g.d[0], g.d[4], g.d[8], s, g.hdemag, g.h);
        else
            cufields::CSpMV_CSR_OffDiag<<<nb, g.block>>>(g.n, g.xadj, g.adjncy, g.d[0], g.d[1], g.d[2], g.d[3], g.d[4],
                                                         g.d[5], g.d[6], g.d[7], g.d[8], s, g.hdemag, g.h);
    }
}
}  // namespace

extern "C" {

// Upload the state the refh_* calls left in the namespace globals, as
// cullg::allocate_memory_on_card (src/cuda_util.cu:261-520) would, and copy the
// constant-memory data of the four kernel files.  dzz_from_dyy reproduces the
// reference upload of Cdzz from datayy (src/cuda_util.cu:308-312,373-377).
int refg_init(unsigned block, int dzz_from_dyy) {
    release();
    const unsigned n = geom::nspins;
    if (n == 0 || block == 0 || block > 1024) return -1;
    g.n = n;
    g.block = block;
    std::vector<double> s = aos(spins::Sx, spins::Sy, spins::Sz, n);
    g.spin = upload(s.data(), s.size());
    g.espin = upload<double>(nullptr, 3 * (size_t)n);
    g.h = upload<double>(nullptr, 3 * (size_t)n);
    g.fn = upload<double>(nullptr, 3 * (size_t)n);
    g.det = upload<double>(nullptr, 3 * (size_t)n);
    for (int k = 0; k < 6; k++) g.rk[k] = upload<double>(nullptr, 3 * (size_t)n);
    std::vector<double> hs = aos(fields::Hstagx, fields::Hstagy, fields::Hstagz, n);
    g.hstg = upload(hs.data(), hs.size());
    std::vector<double> hd = aos(fields::HDemagx, fields::HDemagy, fields::HDemagz, n);
    std::vector<float> hdf(hd.begin(), hd.end());
    g.hdemag = upload(hdf.data(), hdf.size());
    g.curand_n = 3 * n + ((3 * n) % 2);
    g.rand = upload<float>(nullptr, g.curand_n);
    g.sigma = upload(geom::sigma.ptr(), n);
    g.llgpf = upload(geom::llgpf.ptr(), n);
    g.lambda = upload(geom::lambda.ptr(), n);
    g.k1u = upload(anis::k1u.ptr(), n);
    std::vector<double> kd(3 * (size_t)n);
    for (unsigned i = 0; i < n; i++)
        for (int c = 0; c < 3; c++) kd[3 * i + c] = anis::k1udir(i, c);
    g.k1udir = upload(kd.data(), kd.size());
    Array<double>* d[9] = {&exch::dataxx, &exch::dataxy, &exch::dataxz, &exch::datayx, &exch::datayy,
                           &exch::datayz, &exch::datazx, &exch::datazy, &exch::datazz};
    for (int c = 0; c < 9; c++) {
        Array<double>& src = (c == 8 && dzz_from_dyy) ? exch::datayy : *d[c];
        g.d[c] = upload(src.ptr(), src.size());
    }
    if (config::exchm == 2) {
        g.xadj = upload(exch::xadj.ptr(), exch::xadj.size());
        g.adjncy = upload(exch::adjncy.ptr(), exch::adjncy.size());
    } else {
        g.offset = upload(exch::diagoffset.ptr(), exch::diagoffset.size());
    }
    if (exch::inc4spin) {
        g.q_xadj = upload(exch::xadj_j.ptr(), exch::xadj_j.size());
        g.q_j = upload(exch::adjncy_j.ptr(), exch::adjncy_j.size());
        g.q_k = upload(exch::adjncy_k.ptr(), exch::adjncy_k.size());
        g.q_l = upload(exch::adjncy_l.ptr(), exch::adjncy_l.size());
    }
    for (void* p : g.owned)
        if (!p) { release(); return -2; }
    geom::Nk.resize(3);
    for (int c = 0; c < 3; c++) geom::Nk[c] = 0;
    cuint::copyConstData();
    cufields::copyConstData();
    cuintRK4::copyConstData();
    cuintRK5::copyConstData();
    return status();
}

// The normals the next steps read (Crand, float, [3*i+c]); n <= 3N.
int refg_set_noise(const float* xi, size_t n) {
    if (!g.rand || n > g.curand_n) return -1;
    cudaMemcpy(g.rand, xi, n * sizeof(float), cudaMemcpyHostToDevice);
    return status();
}

// nsteps steps of integrator 0 (Heun, src/cuda.cu:43-258), 1 (RK4,
// src/cudaRK4.cu:38-233) or 2 (RK5, src/cudaRK5.cu), every step reading the
// same Crand (the reference draws a new one per step; the caller sets it).
int refg_run(int integrator, unsigned nsteps) {
    if (!g.spin) return -1;
    const unsigned nb = (g.n + g.block - 1) / g.block;
    const double T = llg::T, ax = llg::applied[0], ay = llg::applied[1], az = llg::applied[2];
    for (unsigned t = 0; t < nsteps; t++) {
        if (integrator != 0 && gen) curandGenerateNormal(gen, g.rand, g.curand_n, 0.0f, 1.0f);  // src/cudaRK4.cu:41
        if (integrator == 0) {
            spmv(g.spin);
            if (exch::inc4spin)
                cufields::CSpMV_CSR_FourSpin<<<nb, g.block>>>(g.n, g.q_xadj, g.q_j, g.q_k, g.q_l, g.h, g.spin);
            if (gen) curandGenerateNormal(gen, g.rand, g.curand_n, 0.0f, 1.0f);                  // src/cuda.cu:148
            cuint::CHeun1<<<nb, g.block>>>(g.n, T, ax, ay, az, g.h, g.spin, g.espin, g.rand, g.fn, g.sigma, g.llgpf,
                                           g.lambda, g.k1u, g.k1udir, g.hstg);
            spmv(g.espin);
            if (exch::inc4spin)
                cufields::CSpMV_CSR_FourSpin<<<nb, g.block>>>(g.n, g.q_xadj, g.q_j, g.q_k, g.q_l, g.h, g.espin);
            cuint::CHeun2<<<nb, g.block>>>(g.n, T, ax, ay, az, g.h, g.spin, g.espin, g.rand, g.fn, g.sigma, g.llgpf,
                                           g.lambda, g.k1u, g.k1udir, g.det, g.hstg);
        } else if (integrator == 1) {
            spmv(g.spin);
            cuintRK4::CdetRK4k1<<<nb, g.block>>>(g.n, T, ax, ay, az, g.h, g.spin, g.espin, g.rk[0], g.rand, g.sigma,
                                                 g.llgpf, g.lambda, g.k1u, g.k1udir, g.hstg);
            spmv(g.espin);
            cuintRK4::CdetRK4k2<<<nb, g.block>>>(g.n, T, ax, ay, az, g.h, g.spin, g.espin, g.rk[1], g.rand, g.sigma,
                                                 g.llgpf, g.lambda, g.k1u, g.k1udir, g.hstg);
            spmv(g.espin);
            cuintRK4::CdetRK4k3<<<nb, g.block>>>(g.n, T, ax, ay, az, g.h, g.spin, g.espin, g.rk[2], g.rand, g.sigma,
                                                 g.llgpf, g.lambda, g.k1u, g.k1udir, g.hstg);
            spmv(g.espin);
            cuintRK4::CdetRK4k4<<<nb, g.block>>>(g.n, T, ax, ay, az, g.h, g.spin, g.espin, g.rk[3], g.rand, g.sigma,
                                                 g.llgpf, g.lambda, g.k1u, g.k1udir, g.hstg);
            cuintRK4::CdetSnp1<<<nb, g.block>>>(g.n, g.spin, g.rk[0], g.rk[1], g.rk[2], g.rk[3]);
        } else if (integrator == 2) {
            double** k = g.rk;
            spmv(g.spin);
            cuintRK5::CdetRK5k1<<<nb, g.block>>>(g.n, T, ax, ay, az, g.h, g.spin, g.espin, k[0], g.rand, g.sigma,
                                                 g.llgpf, g.lambda, g.k1u, g.k1udir, g.hstg);
            spmv(g.espin);
            cuintRK5::CdetRK5k2<<<nb, g.block>>>(g.n, T, ax, ay, az, g.h, g.spin, g.espin, k[1], k[0], g.rand,
                                                 g.sigma, g.llgpf, g.lambda, g.k1u, g.k1udir, g.hstg);
            spmv(g.espin);
            cuintRK5::CdetRK5k3<<<nb, g.block>>>(g.n, T, ax, ay, az, g.h, g.spin, g.espin, k[2], k[1], k[0], g.rand,
                                                 g.sigma, g.llgpf, g.lambda, g.k1u, g.k1udir, g.hstg);
            spmv(g.espin);
            cuintRK5::CdetRK5k4<<<nb, g.block>>>(g.n, T, ax, ay, az, g.h, g.spin, g.espin, k[3], k[2], k[1], k[0],
                                                 g.rand, g.sigma, g.llgpf, g.lambda, g.k1u, g.k1udir, g.hstg);
            spmv(g.espin);
            cuintRK5::CdetRK5k5<<<nb, g.block>>>(g.n, T, ax, ay, az, g.h, g.spin, g.espin, k[4], k[3], k[2], k[1],
                                                 k[0], g.rand, g.sigma, g.llgpf, g.lambda, g.k1u, g.k1udir, g.hstg);
            spmv(g.espin);
            cuintRK5::CdetRK5k6<<<nb, g.block>>>(g.n, T, ax, ay, az, g.h, g.spin, g.espin, k[5], k[4], k[3], k[2],
                                                 k[1], k[0], g.rand, g.sigma, g.llgpf, g.lambda, g.k1u, g.k1udir,
                                                 g.hstg);
            cuintRK5::CdetSnp1<<<nb, g.block>>>(g.n, g.spin, k[0], k[1], k[2], k[3], k[4], k[5]);
        } else {
            return -1;
        }
    }
    return status();
}

// cuRAND XORWOW seeded as cullg::cuinit does (src/cuda.cu:345-368); from then on every step
// draws its own Crand like the reference instead of reading the caller's.
int refg_enable_curand(unsigned long long seed) {
    if (gen) { curandDestroyGenerator(gen); gen = nullptr; }
    if (curandCreateGenerator(&gen, CURAND_RNG_PSEUDO_DEFAULT) != CURAND_STATUS_SUCCESS) { gen = nullptr; return -1; }
    if (curandSetPseudoRandomGeneratorSeed(gen, seed) != CURAND_STATUS_SUCCESS) return -1;
    if (curandGenerateSeeds(gen) != CURAND_STATUS_SUCCESS) return -1;
    return status();
}

// Device time of nsteps steps, each preceded by an untimed write of flush_bytes (the L2
// flushed as the library's cold timers do) and bracketed by its own CUDA events.
int refg_time_steps(int integrator, unsigned nsteps, size_t flush_bytes, double* ms) {
    if (!g.spin || !ms) return -1;
    void* flush = nullptr;
    if (flush_bytes && cudaMalloc(&flush, flush_bytes) != cudaSuccess) return -2;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    double total = 0.0;
    int rc = 0;
    for (unsigned t = 0; t < nsteps && rc == 0; t++) {
        if (flush) cudaMemset(flush, t & 0xFF, flush_bytes);
        cudaEventRecord(e0, 0);
        const unsigned nb = (g.n + g.block - 1) / g.block;
        // one step, without the synchronising status() of refg_run
        const double T = llg::T, ax = llg::applied[0], ay = llg::applied[1], az = llg::applied[2];
        if (integrator == 0) {
            spmv(g.spin);
            if (exch::inc4spin)
                cufields::CSpMV_CSR_FourSpin<<<nb, g.block>>>(g.n, g.q_xadj, g.q_j, g.q_k, g.q_l, g.h, g.spin);
            if (gen) curandGenerateNormal(gen, g.rand, g.curand_n, 0.0f, 1.0f);
            cuint::CHeun1<<<nb, g.block>>>(g.n, T, ax, ay, az, g.h, g.spin, g.espin, g.rand, g.fn, g.sigma, g.llgpf,
                                           g.lambda, g.k1u, g.k1udir, g.hstg);
            spmv(g.espin);
            if (exch::inc4spin)
                cufields::CSpMV_CSR_FourSpin<<<nb, g.block>>>(g.n, g.q_xadj, g.q_j, g.q_k, g.q_l, g.h, g.espin);
            cuint::CHeun2<<<nb, g.block>>>(g.n, T, ax, ay, az, g.h, g.spin, g.espin, g.rand, g.fn, g.sigma, g.llgpf,
                                           g.lambda, g.k1u, g.k1udir, g.det, g.hstg);
        } else {
            rc = -1;
        }
        cudaEventRecord(e1, 0);
        if (cudaEventSynchronize(e1) != cudaSuccess) rc = -3;
        float m = 0.f;
        cudaEventElapsedTime(&m, e0, e1);
        total += m;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (flush) cudaFree(flush);
    *ms = total;
    const int st = status();
    return rc ? rc : st;
}

int refg_get_spins(double* out) {
    if (!g.spin) return -1;
    cudaMemcpy(out, g.spin, 3 * (size_t)g.n * sizeof(double), cudaMemcpyDeviceToHost);
    return status();
}

// A work array after the last step: 0..5 CRKk1..CRKk6, 6 Cespin, 7 CH (3N doubles each).
int refg_get_buffer(int which, double* out) {
    if (!g.spin || which < 0 || which > 7) return -1;
    const double* src = which < 6 ? g.rk[which] : which == 6 ? g.espin : g.h;
    cudaMemcpy(out, src, 3 * (size_t)g.n * sizeof(double), cudaMemcpyDeviceToHost);
    return status();
}

// CDetFields: the Heun corrector's total field less the thermal term (src/cuint.cu:238).
int refg_get_det_field(double* out) {
    if (!g.det) return -1;
    cudaMemcpy(out, g.det, 3 * (size_t)g.n * sizeof(double), cudaMemcpyDeviceToHost);
    return status();
}

void refg_free() {
    release();
    if (gen) { curandDestroyGenerator(gen); gen = nullptr; }
}
}
