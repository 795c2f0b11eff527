// Test-infrastructure harness around the reference's own CPU Heun step.
//
// This file is compiled together with the reference sources
//   src/llgCPU.cpp, src/matrix_mul_cpu.cpp and (unless ASD_REF_REPLAY) src/random.cpp
// exactly where they lie in the reference tree (see oracle/Makefile).  It
// defines the namespace globals those sources read (geom::, spins::, fields::,
// exch::, anis::, llg::, config::) and exposes a small C API so that the
// Python tests and bench.py can drive llgCPU::llgCPU(t) (src/llgCPU.cpp:56-361)
// on inputs they build themselves.  It is the CPU baseline and a parity pin
// for the oracle; nothing in the product links it.
//
// With -DASD_REF_REPLAY the reference RNG (src/random.cpp) is replaced at link
// time by Random::normal() reading a caller-supplied buffer, so that recorded
// noise can be fed to llgCPU (the reference draws 3N normals per step, x,y,z
// per spin in spin order, src/llgCPU.cpp:131-138).
#include <libconfig.h++>
#include "../inc/arrays.h"
#include "../inc/exch.h"
#include "../inc/config.h"
#include "../inc/geom.h"
#include "../inc/fields.h"
#include "../inc/spins.h"
#include "../inc/llg.h"
#include "../inc/llgCPU.h"
#include "../inc/random.h"
#include "../inc/anis.h"
#include <cmath>
#include <cstring>
#include <cstdio>
#include <vector>
#include <sstream>
#include <string>

namespace geom {
unsigned int nspins = 0;
Array<double> lambda, llgpf, sigma;
unitCellMembers ucm;
}
namespace spins {
Array<double> Sx, Sy, Sz, eSx, eSy, eSz;
unsigned int update = 1;
}
namespace fields {
Array<double> Hstagx, Hstagy, Hstagz, Hx, Hy, Hz, Hthx, Hthy, Hthz, HDemagx, HDemagy, HDemagz, H4sx, H4sy, H4sz;
static int fft_called = 0;
void ftdip() { fft_called++; }
void eftdip() { fft_called++; }
void dipftdip() { fft_called++; }
}
namespace exch {
Array<int> diagoffset, offdiagoffset;
Array<unsigned int> xadj, adjncy, xadj_j, adjncy_j, adjncy_k, adjncy_l;
Array<double> dataxx, dataxy, dataxz, datayx, datayy, datayz, datazx, datazy, datazz;
Array<double> JQ;
unsigned int diagnumdiag = 0, offdiagnumdiag = 0;
bool inc4spin = false;
}
namespace anis {
Array<double> k1u;
Array2D<double> k1udir;
double k2par = 0, k2perp = 0, k4par = 0, k4perp = 0;
Array<double> k2perpdir, k2pardir;
Array2D<double> k4perpdirs, k4pardirs;
}
namespace llg {
// Same constant values as src/llg.cpp:25.
double applied[3] = {0, 0, 0}, T = 0, dt = 1e-16, rdt = 0, gyro = 1.76e11, muB = 9.27e-24, kB = 1.38e-23;
}
namespace config {
std::ofstream Info, Log;
unsigned int exchm = 2, dipm = 0;
bool inc_dip = false, offdiag = false;
void printline(std::ofstream&) {}
}
// error::errMessage exits in the reference (src/error.cpp:19-28); here it records the message
// for refh_last_error and returns.
static std::string g_last_error;
namespace error {
void errPreamble(std::string, int) {}
void errWarnPreamble(std::string, int) {}
void errMessage(std::string m) { g_last_error = m; }
void errMessage(std::stringstream& m) { g_last_error = m.str(); }
void errWarning(std::string) {}
}

#ifdef ASD_REF_REPLAY
namespace Random {
static std::vector<double> g_noise;
static size_t g_pos = 0;
bool ri = true;
void seed(const unsigned int, const unsigned int) {}
double rand() { return 0.0; }
double normal() {
    if (g_noise.empty()) return 0.0;
    double v = g_noise[g_pos];
    g_pos = (g_pos + 1) % g_noise.size();
    return v;
}
}
#endif

static void fill3(Array<double>& a, Array<double>& b, Array<double>& c, const double* src, unsigned n) {
    a.resize(n); b.resize(n); c.resize(n);
    for (unsigned i = 0; i < n; i++) {
        a[i] = src ? src[3 * i] : 0.0;
        b[i] = src ? src[3 * i + 1] : 0.0;
        c[i] = src ? src[3 * i + 2] : 0.0;
    }
}

extern "C" {

// Per-unit-cell-atom material (mu in muB, damping, relative gamma) and the
// unit-cell atom of every spin (geom::lu(i,4)).  Prefactors follow
// src/llg.cpp:591-592 and src/llg.cpp:626-631; rdt follows src/llg.cpp:306.
int refh_init(unsigned n, unsigned nauc, const double* mu, const double* lam, const double* gam,
              const unsigned* atom_of_spin, double dt, double T, const double* applied) {
    geom::nspins = n;
    geom::ucm.init(nauc, nauc);
    for (unsigned t = 0; t < nauc; t++) {
        geom::ucm.SetMu(mu[t], t);
        geom::ucm.SetDamping(lam[t], t);
        geom::ucm.SetGamma(gam[t], t);
    }
    llg::dt = dt;
    llg::rdt = dt * llg::gyro;
    llg::T = T;
    for (int c = 0; c < 3; c++) llg::applied[c] = applied ? applied[c] : 0.0;
    geom::lambda.resize(n); geom::llgpf.resize(n); geom::sigma.resize(n);
    for (unsigned i = 0; i < n; i++) {
        unsigned t = atom_of_spin[i];
        geom::lambda[i] = lam[t];
        geom::llgpf[i] = -1. / (1.0 + lam[t] * lam[t]);
        geom::sigma[i] = sqrt(2.0 * llg::kB * lam[t] / (mu[t] * llg::muB * dt * gam[t] * llg::gyro));
    }
    spins::Sx.resize(n); spins::Sy.resize(n); spins::Sz.resize(n);
    // llgCPU's own work arrays (fn, eS, Hth) are sized here (src/llgCPU.cpp:32-54)
    llgCPU::initLLG();
    fill3(fields::Hx, fields::Hy, fields::Hz, nullptr, n);
    fill3(fields::Hthx, fields::Hthy, fields::Hthz, nullptr, n);
    fill3(fields::HDemagx, fields::HDemagy, fields::HDemagz, nullptr, n);
    fill3(fields::H4sx, fields::H4sy, fields::H4sz, nullptr, n);
    fill3(fields::Hstagx, fields::Hstagy, fields::Hstagz, nullptr, n);
    anis::k1u.resize(n);
    anis::k1udir.resize(n, 3);
    for (unsigned i = 0; i < n; i++) { anis::k1u[i] = 0; for (int c = 0; c < 3; c++) anis::k1udir(i, c) = 0; }
    anis::k2perpdir.resize(3); anis::k2pardir.resize(3);
    anis::k4perpdirs.resize(3, 3); anis::k4pardirs.resize(3, 3);
    for (int a = 0; a < 3; a++) {
        anis::k2perpdir[a] = 0; anis::k2pardir[a] = 0;
        for (int b = 0; b < 3; b++) { anis::k4perpdirs(a, b) = 0; anis::k4pardirs(a, b) = 0; }
    }
    anis::k2par = anis::k2perp = anis::k4par = anis::k4perp = 0;
    exch::inc4spin = false;
    config::inc_dip = false;
    return 0;
}

void refh_set_temperature(double T) { llg::T = T; }

// The last message passed to error::errMessage ("" if none), then cleared.
const char* refh_last_error() {
    static std::string out;
    out = g_last_error;
    g_last_error.clear();
    return out.c_str();
}

// k1u per spin already scaled as in src/geom.cpp:244 (2K/(mu muB)).
int refh_set_anis(const double* k1u, const double* k1udir, double k2perp, const double* k2perpdir,
                  double k2par, const double* k2pardir, double k4perp, const double* k4perpdirs,
                  double k4par, const double* k4pardirs) {
    unsigned n = geom::nspins;
    for (unsigned i = 0; i < n; i++) {
        anis::k1u[i] = k1u ? k1u[i] : 0.0;
        for (int c = 0; c < 3; c++) anis::k1udir(i, c) = k1udir ? k1udir[3 * i + c] : 0.0;
    }
    anis::k2perp = k2perp; anis::k2par = k2par; anis::k4perp = k4perp; anis::k4par = k4par;
    for (int a = 0; a < 3; a++) {
        anis::k2perpdir[a] = k2perpdir ? k2perpdir[a] : 0.0;
        anis::k2pardir[a] = k2pardir ? k2pardir[a] : 0.0;
        for (int b = 0; b < 3; b++) {
            anis::k4perpdirs(a, b) = k4perpdirs ? k4perpdirs[3 * a + b] : 0.0;
            anis::k4pardirs(a, b) = k4pardirs ? k4pardirs[3 * a + b] : 0.0;
        }
    }
    return 0;
}

// CSR exchange: values are J/(mu_i muB) [T], nnz x 9 row-major (alpha,beta).
int refh_set_csr(int offdiag, unsigned nnz, const unsigned* xadj, const unsigned* adjncy, const double* data9) {
    unsigned n = geom::nspins;
    config::exchm = 2;
    config::offdiag = offdiag != 0;
    exch::xadj.resize(n + 1);
    for (unsigned i = 0; i <= n; i++) exch::xadj[i] = xadj[i];
    exch::adjncy.resize(nnz);
    Array<double>* d[9] = {&exch::dataxx, &exch::dataxy, &exch::dataxz, &exch::datayx, &exch::datayy,
                           &exch::datayz, &exch::datazx, &exch::datazy, &exch::datazz};
    for (int c = 0; c < 9; c++) d[c]->resize(nnz);
    for (unsigned k = 0; k < nnz; k++) {
        exch::adjncy[k] = adjncy[k];
        for (int c = 0; c < 9; c++) (*d[c])[k] = data9[9 * k + c];
    }
    return 0;
}

// Row-aligned DIA exchange (data[c][n*N+row], src/matrix_conv.cpp:28-141):
// ndiag offsets, 9 x ndiag x N values.  llgCPU's off-diagonal DIA path reads
// exch::offdiagnumdiag (src/llgCPU.cpp:95,261) which the reference never sets
// (src/exch.cpp:23); the caller chooses it through offdiag_numdiag.
int refh_set_dia(int offdiag, unsigned ndiag, const int* offsets, const double* data9, unsigned offdiag_numdiag) {
    unsigned n = geom::nspins;
    config::exchm = 1;
    config::offdiag = offdiag != 0;
    exch::diagnumdiag = ndiag;
    exch::offdiagnumdiag = offdiag_numdiag;
    exch::diagoffset.resize(ndiag);
    exch::offdiagoffset.resize(ndiag);
    for (unsigned k = 0; k < ndiag; k++) { exch::diagoffset[k] = offsets[k]; exch::offdiagoffset[k] = offsets[k]; }
    Array<double>* d[9] = {&exch::dataxx, &exch::dataxy, &exch::dataxz, &exch::datayx, &exch::datayy,
                           &exch::datayz, &exch::datazx, &exch::datazy, &exch::datazz};
    size_t m = (size_t)ndiag * n;
    for (int c = 0; c < 9; c++) {
        d[c]->resize(m);
        for (size_t k = 0; k < m; k++) (*d[c])[k] = data9[(size_t)c * m + k];
    }
    return 0;
}

// Four-spin quartets (exch::xadj_j / adjncy_j,k,l, src/exch_read_4_spin.cpp:147-270) and the
// constant JQ(0) in T; llgCPU adds -JQ (Sj (Sk.Sl) + Sk (Sj.Sl) + Sl (Sk.Sj)) per quartet
// (src/llgCPU.cpp:148-170).
int refh_set_four_spin(unsigned nq, const unsigned* xadj_jkl, const unsigned* adj_j, const unsigned* adj_k,
                       const unsigned* adj_l, double jq) {
    unsigned n = geom::nspins;
    exch::inc4spin = true;
    exch::xadj_j.resize(n + 1);
    for (unsigned i = 0; i <= n; i++) exch::xadj_j[i] = xadj_jkl[i];
    exch::adjncy_j.resize(nq); exch::adjncy_k.resize(nq); exch::adjncy_l.resize(nq);
    for (unsigned q = 0; q < nq; q++) {
        exch::adjncy_j[q] = adj_j[q]; exch::adjncy_k[q] = adj_k[q]; exch::adjncy_l[q] = adj_l[q];
    }
    exch::JQ.resize(1);
    exch::JQ[0] = jq;
    return 0;
}

int refh_set_site_fields(const double* hstag, const double* hdemag) {
    unsigned n = geom::nspins;
    fill3(fields::Hstagx, fields::Hstagy, fields::Hstagz, hstag, n);
    fill3(fields::HDemagx, fields::HDemagy, fields::HDemagz, hdemag, n);
    return 0;
}

// Initial spins as the reference's restart_text reader stores them: each
// vector divided by its length (src/spins.cpp:384-392).
int refh_set_spins(const double* s) {
    for (unsigned i = 0; i < geom::nspins; i++) {
        spins::Sx[i] = s[3 * i]; spins::Sy[i] = s[3 * i + 1]; spins::Sz[i] = s[3 * i + 2];
        const double mods = sqrt(spins::Sx[i] * spins::Sx[i] + spins::Sy[i] * spins::Sy[i] + spins::Sz[i] * spins::Sz[i]);
        spins::Sx[i] /= mods; spins::Sy[i] /= mods; spins::Sz[i] /= mods;
    }
    return 0;
}

int refh_get_spins(double* s) {
    for (unsigned i = 0; i < geom::nspins; i++) {
        s[3 * i] = spins::Sx[i]; s[3 * i + 1] = spins::Sy[i]; s[3 * i + 2] = spins::Sz[i];
    }
    return 0;
}

// fields::H after a step: the accumulated exchange field (see src/llgCPU.cpp:58-60).
int refh_get_field(double* h) {
    for (unsigned i = 0; i < geom::nspins; i++) {
        h[3 * i] = fields::Hx[i]; h[3 * i + 1] = fields::Hy[i]; h[3 * i + 2] = fields::Hz[i];
    }
    return 0;
}

int refh_get_thermal(double* h) {
    for (unsigned i = 0; i < geom::nspins; i++) {
        h[3 * i] = fields::Hthx[i]; h[3 * i + 1] = fields::Hthy[i]; h[3 * i + 2] = fields::Hthz[i];
    }
    return 0;
}

void refh_seed(unsigned a, unsigned b) { Random::seed(a, b); }

double refh_normal() { return Random::normal(); }

double refh_rand() { return Random::rand(); }

#ifdef ASD_REF_REPLAY
int refh_set_noise(const double* xi, size_t n) {
    Random::g_noise.assign(xi, xi + n);
    Random::g_pos = 0;
    return 0;
}
#endif

// Advance nsteps reference CPU Heun steps starting at step t0.
int refh_run(unsigned t0, unsigned nsteps) {
    for (unsigned t = t0; t < t0 + nsteps; t++) llgCPU::llgCPU(t);
    return fields::fft_called ? -1 : 0;
}

}
