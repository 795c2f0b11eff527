// cullg_asd.cpp — drop-in replacement for the reference's GPU integrator layer.
//
// Dropped into the reference's src/ in place of src/cuda.cu, src/cudaRK4.cu, src/cudaRK5.cu and
// src/cuda_util.cu, it defines the cullg:: functions of inc/cuda.h:62-70 on top of the C ABI of
// libasd_b200 (include/asd.h).  It reads the same namespace globals the old files read
// (geom::, exch::, anis::, llg::, spins::, fields::, config::), so llg::integrate
// (src/llg.cpp:639-664) and every driver above it (src/simple.cpp, src/mvt.cpp, ...) stay as
// they are.  Build: add this file to the reference's object list and link -lasd_b200.
#include <libconfig.h++>
#include "../inc/arrays.h"
#include "../inc/cuda.h"
#include "../inc/geom.h"
#include "../inc/exch.h"
#include "../inc/spins.h"
#include "../inc/fields.h"
#include "../inc/llg.h"
#include "../inc/anis.h"
#include "../inc/config.h"
#include "../inc/error.h"
#include "asd.h"
#include <vector>

namespace cullg {
namespace {
asd_handle* H = nullptr;
uint32_t precision = ASD_FP32;          // ASD_FP64_PLAIN reproduces the reference arithmetic
uint32_t extra_flags = 0;               // e.g. the reference's GPU quirks, ASD_FLAG_GPU_*

std::vector<double> aos(Array<double>& x, Array<double>& y, Array<double>& z) {
    std::vector<double> v(3 * (size_t)geom::nspins);
    for (unsigned i = 0; i < geom::nspins; i++) { v[3 * i] = x[i]; v[3 * i + 1] = y[i]; v[3 * i + 2] = z[i]; }
    return v;
}

void fail(const char* what) {
    error::errPreamble(__FILE__, __LINE__);
    error::errMessage(std::string(what) + ": " + asd_last_error(H));
}
}  // namespace

// Precision and extra flags of the next cuinit (not part of the reference interface).
void asd_configure(uint32_t prec, uint32_t flags) { precision = prec; extra_flags = flags; }

void cuinit() {                                                   // src/cuda.cu:261-402
    asd_params p{};
    p.integrator = llg::intscheme;                                // 0 heun, 1 rk4, 2 rk5
    p.precision = precision;
    p.flags = (precision == ASD_FP32 ? ASD_FLAG_COMPENSATED : 0u) | extra_flags;
    p.dt = llg::dt;
    p.gyro = llg::gyro; p.muB = llg::muB; p.kB = llg::kB;
    for (int a = 0; a < 3; a++) p.applied[a] = llg::applied[a];
    p.k2perp = anis::k2perp; p.k2par = anis::k2par; p.k4perp = anis::k4perp; p.k4par = anis::k4par;
    for (int a = 0; a < 3; a++) { p.k2perpdir[a] = anis::k2perpdir[a]; p.k2pardir[a] = anis::k2pardir[a]; }
    for (int a = 0; a < 9; a++) { p.k4perpdirs[a] = anis::k4perpdirs.ptr()[a]; p.k4pardirs[a] = anis::k4pardirs.ptr()[a]; }
    p.seed = config::seed;
    p.update = spins::update;
    std::vector<asd_material> mats(geom::ucm.NumAtomsUnitCell());
    for (unsigned t = 0; t < mats.size(); t++)
        mats[t] = {geom::ucm.GetMu(t), geom::ucm.GetDamping(t), geom::ucm.GetGamma(t), geom::ucm.GetK1U(t),
                   {geom::ucm.GetK1UDir(t, 0), geom::ucm.GetK1UDir(t, 1), geom::ucm.GetK1UDir(t, 2)},
                   geom::ucm.GetSublattice(t)};
    std::vector<uint32_t> atom(geom::nspins);
    for (unsigned i = 0; i < geom::nspins; i++) atom[i] = geom::lu(i, 4);
    asd_system s{};
    s.nspins = geom::nspins; s.nmat = (uint32_t)mats.size(); s.mat = mats.data(); s.atom = atom.data();
    s.exch = config::exchm; s.exch_full = config::offdiag ? 1 : 0;
    Array<double>* d[9] = {&exch::dataxx, &exch::dataxy, &exch::dataxz, &exch::datayx, &exch::datayy,
                           &exch::datayz, &exch::datazx, &exch::datazy, &exch::datazz};
    const int diag_comp[3] = {0, 4, 8};
    std::vector<double> val;
    if (config::exchm == 2) {                                     // CSR: nnz x 9, row-major
        const unsigned nnz = exch::adjncy.size();
        val.assign(9 * (size_t)nnz, 0.0);
        for (unsigned k = 0; k < nnz; k++)
            for (int q = 0; q < 9; q++)
                if (d[q]->size() >= nnz) val[9 * (size_t)k + q] = (*d[q])[k];
        s.xadj = exch::xadj.ptr(); s.adjncy = exch::adjncy.ptr(); s.nnz = nnz; s.csr_val = val.data();
    } else if (config::exchm == 1) {                              // DIA: c x ndiag x N
        const size_t m = (size_t)exch::diagnumdiag * geom::nspins;
        const int nc = config::offdiag ? 9 : 3;
        val.assign(nc * m, 0.0);
        for (int c = 0; c < nc; c++) {
            Array<double>& src = *d[config::offdiag ? c : diag_comp[c]];
            for (size_t k = 0; k < m && k < src.size(); k++) val[c * m + k] = src[k];
        }
        s.ndiag = exch::diagnumdiag; s.dia_offset = exch::diagoffset.ptr(); s.dia_val = val.data();
    }
    // dipole (config::inc_dip): s.lr = ASD_LR_DIPOLE, s.mesh = geom::zpdim x Nk, s.mesh_xyz =
    // geom::lu(i, 0..2), s.nr = the real-space intmat::dipNrab before its FFT
    s.temperature = llg::T;
    std::vector<double> hst = aos(fields::Hstagx, fields::Hstagy, fields::Hstagz);
    s.site_field = hst.data();
    if (asd_create(&p, &s, 1, &H) != ASD_OK) fail("asd_create");
    std::vector<double> s3 = aos(spins::Sx, spins::Sy, spins::Sz);
    if (asd_set_spins(H, s3.data(), geom::nspins) != ASD_OK) fail("asd_set_spins");
}

static void step_and_mirror(unsigned int& t) {                    // src/cuda.cu:43-258
    if (asd_set_temperature(H, ASD_ALL_REPLICAS, llg::T) != ASD_OK) fail("asd_set_temperature");
    if (asd_set_applied(H, llg::applied) != ASD_OK) fail("asd_set_applied");
    if (asd_step(H, 1) != ASD_OK) fail("asd_step");
    if (t % spins::update == 0) {                                 // the D2H mirror of src/cuda.cu:234-256
        std::vector<double> s3(3 * (size_t)geom::nspins), h3(3 * (size_t)geom::nspins);
        asd_get_spins(H, s3.data(), geom::nspins);
        asd_get_det_field(H, h3.data(), geom::nspins);
        for (unsigned i = 0; i < geom::nspins; i++) {
            spins::Sx[i] = s3[3 * i]; spins::Sy[i] = s3[3 * i + 1]; spins::Sz[i] = s3[3 * i + 2];
            fields::Hx[i] = h3[3 * i]; fields::Hy[i] = h3[3 * i + 1]; fields::Hz[i] = h3[3 * i + 2];
        }
    }
}
void llgGPU(unsigned int& t) { step_and_mirror(t); }
void llgGPURK4(unsigned int& t) { step_and_mirror(t); }
void llgGPURK5(unsigned int& t) { step_and_mirror(t); }
void rampStag(double rv) { asd_set_site_field_scale(H, rv); }                 // src/cuda.cu:38-41
void CsetStagFields() {                                                       // src/cuda_util.cu:563-575
    std::vector<double> h = aos(fields::Hstagx, fields::Hstagy, fields::Hstagz);
    asd_set_site_field(H, h.data(), geom::nspins);
}
void CsetStagFieldsZero() { asd_set_site_field(H, nullptr, 0); }             // src/cuda_util.cu:576-588
void deallocate_cuda_memory() { asd_destroy(H); H = nullptr; }               // src/cuda_util.cu:186-242
}  // namespace cullg
