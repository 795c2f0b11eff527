// Test-infrastructure harness around the reference's own set-up code:
//   exch::exchunitcell        (src/exch_unitcell.cpp:265-489)  CSR assembly from unit-cell shells
//   matconv::csr_to_dia_diag / csr_to_dia_offdiag (src/matrix_conv.cpp:28-272)  CSR -> DIA
// compiled where they lie in the reference tree (see oracle/Makefile).  It defines the
// namespace globals those functions read and exposes a C API for the tests, which compare the
// library's asd_build_csr / asd_csr_to_dia against them.  Nothing in the product links it.
//
// checkdiag is sized 2N here where the reference sizes it 2N-1 (src/exch_unitcell.cpp:27):
// a bond at offset N-1 makes exchunitcell increment checkdiag[2N-1] (src/exch_unitcell.cpp:375-384),
// one past the reference's array; the extra slot keeps that write in bounds, and the conversion
// still scans only the first 2N-1 entries, as the reference does.
#include <libconfig.h++>
#include "../inc/arrays.h"
#include "../inc/exch.h"
#include "../inc/config.h"
#include "../inc/geom.h"
#include "../inc/llg.h"
#include "../inc/matrix_conv.h"
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>

namespace geom {
unsigned int dim[3] = {0, 0, 0}, nspins = 0;
Array2D<int> lu;
Array2D<double> rprim;
Array<double> mu, rx, ry, rz;
Array4D<unsigned int> atnolu;
unitCellMembers ucm;
}
namespace exch {
Array<int> diagoffset, offdiagoffset, checkdiag;
Array<unsigned int> xadj, adjncy;
Array<double> dataxx, dataxy, dataxz, datayx, datayy, datayz, datazx, datazy, datazz;
Array2D<unsigned int> shell_list;
Array4D<double> exchvec;
Array5D<double> J;
unsigned int diagnumdiag = 0, offdiagnumdiag = 0;
bool outputJ = false, oem = false, cutexch = false;
double rcut = 0.0;
void get_exch_unitcell(int, char**) {}
}
namespace config {
std::ofstream Info, Log;
bool pbc[3] = {true, true, true}, offdiag = false;
unsigned int exchm = 2;
void printline(std::ofstream&) {}
void openLogFile() {}
}
namespace llg {
double muB = 9.27e-24;   // src/llg.cpp:25
}
namespace error {
void errPreamble(std::string, int) {}
void errWarnPreamble(std::string, int) {}
void errMessage(std::string) {}
void errMessage(std::stringstream&) {}
void errWarning(std::string) {}
}

extern "C" {

// Lattice dim[0] x dim[1] x dim[2] cells of nauc atoms (spin numbering of src/geom.cpp:190-245);
// shells[s1*nauc+s2] interactions between atom s1 and atom s2 with cell offsets
// vec[((s1*nauc+s2)*maxsh+k)*3+c] and tensors Jt[((s1*nauc+s2)*maxsh+k)*9+ab] [J].
// Two calls: xadj == NULL returns *nnz only.
int refb_exchunitcell(const unsigned* dim, const int* pbc, unsigned nauc, const double* mu, const unsigned* shells,
                      unsigned maxsh, const double* vec, const double* Jt, int offdiag, unsigned* nnz,
                      unsigned* xadj, unsigned* adjncy, double* val9, unsigned cap) {
    for (int c = 0; c < 3; c++) { geom::dim[c] = dim[c]; config::pbc[c] = pbc[c] != 0; }
    const unsigned n = dim[0] * dim[1] * dim[2] * nauc;
    geom::nspins = n;
    geom::ucm.init(nauc, nauc);
    for (unsigned t = 0; t < nauc; t++) {
        geom::ucm.SetMu(mu[t], t);
        geom::ucm.SetSublattice(t, t);
        geom::ucm.SetXred(0.0, 0.0, 0.0, t);
    }
    geom::lu.resize(n, 8);
    geom::lu.IFill(0);
    geom::mu.resize(n); geom::rx.resize(n); geom::ry.resize(n); geom::rz.resize(n);
    geom::rprim.resize(3, 3);
    geom::rprim.IFill(0);
    for (int c = 0; c < 3; c++) geom::rprim(c, c) = 1.0;
    geom::atnolu.resize(dim[0], dim[1], dim[2], nauc);
    unsigned a = 0;
    for (unsigned i = 0; i < dim[0]; i++)
        for (unsigned j = 0; j < dim[1]; j++)
            for (unsigned k = 0; k < dim[2]; k++)
                for (unsigned t = 0; t < nauc; t++, a++) {
                    geom::lu(a, 3) = t; geom::lu(a, 4) = t;
                    geom::lu(a, 5) = i; geom::lu(a, 6) = j; geom::lu(a, 7) = k;
                    geom::mu[a] = mu[t];
                    geom::rx[a] = i; geom::ry[a] = j; geom::rz[a] = k;
                    geom::atnolu(i, j, k, t) = a;
                }
    exch::shell_list.resize(nauc, nauc);
    exch::exchvec.resize(nauc, nauc, maxsh ? maxsh : 1, 3);
    exch::J.resize(nauc, nauc, maxsh ? maxsh : 1, 3, 3);
    for (unsigned s1 = 0; s1 < nauc; s1++)
        for (unsigned s2 = 0; s2 < nauc; s2++) {
            exch::shell_list(s1, s2) = shells[s1 * nauc + s2];
            for (unsigned k = 0; k < shells[s1 * nauc + s2]; k++) {
                const size_t b = ((size_t)(s1 * nauc + s2) * maxsh + k);
                for (int c = 0; c < 3; c++) exch::exchvec(s1, s2, k, c) = vec[3 * b + c];
                for (int p = 0; p < 3; p++)
                    for (int q = 0; q < 3; q++) exch::J(s1, s2, k, p, q) = Jt[9 * b + 3 * p + q];
            }
        }
    exch::checkdiag.resize(2 * n);
    exch::checkdiag.IFill(0);
    config::offdiag = offdiag != 0;
    exch::exchunitcell();
    const unsigned m = exch::xadj[n];
    *nnz = m;
    if (!xadj) return 0;
    if (cap < m) return 1;
    for (unsigned i = 0; i <= n; i++) xadj[i] = exch::xadj[i];
    Array<double>* d[9] = {&exch::dataxx, &exch::dataxy, &exch::dataxz, &exch::datayx, &exch::datayy,
                           &exch::datayz, &exch::datazx, &exch::datazy, &exch::datazz};
    for (unsigned k = 0; k < m; k++) {
        adjncy[k] = exch::adjncy[k];
        for (int q = 0; q < 9; q++) val9[9 * (size_t)k + q] = d[q]->size() ? (*d[q])[k] : 0.0;
    }
    return 0;
}

// CSR -> DIA through the reference's conversion: diagonal occupancy as exchunitcell records it,
// numdiag counted over the first 2N-1 slots (src/exch_unitcell.cpp:424-428), then
// csr_to_dia_diag (and csr_to_dia_offdiag when offdiag).  Outputs data9[c][d*N+row] for all 9
// components (zeros where not converted).  offsets == NULL: *ndiag only.
int refb_csr_to_dia(unsigned n, const unsigned* xadj, const unsigned* adjncy, const double* val9, int offdiag,
                    unsigned* ndiag, int* offsets, double* data9, unsigned cap) {
    exch::checkdiag.resize(2 * n);
    exch::checkdiag.IFill(0);
    for (unsigned i = 0; i < n; i++)
        for (unsigned k = xadj[i]; k < xadj[i + 1]; k++) {
            const unsigned j = adjncy[k];
            if (i > j) exch::checkdiag[n - (i - j)]++;
            else if (i == j) exch::checkdiag[n]++;
            else exch::checkdiag[n + (j - i)]++;
        }
    unsigned nd = 0;
    for (unsigned i = 0; i < 2 * n - 1; i++)
        if (exch::checkdiag[i] > 0) nd++;
    *ndiag = nd;
    if (!offsets) return 0;
    if (cap < nd) return 1;
    exch::xadj.resize(n + 1);
    for (unsigned i = 0; i <= n; i++) exch::xadj[i] = xadj[i];
    const unsigned m = xadj[n];
    exch::adjncy.resize(m);
    Array<double>* d[9] = {&exch::dataxx, &exch::dataxy, &exch::dataxz, &exch::datayx, &exch::datayy,
                           &exch::datayz, &exch::datazx, &exch::datazy, &exch::datazz};
    for (int q = 0; q < 9; q++) d[q]->resize(m);
    for (unsigned k = 0; k < m; k++) {
        exch::adjncy[k] = adjncy[k];
        for (int q = 0; q < 9; q++) (*d[q])[k] = val9[9 * (size_t)k + q];
    }
    unsigned N = n;
    if (offdiag) {
        // the offdiagonal conversion reads the offsets the diagonal one writes
        matconv::csr_to_dia_diag(N, exch::xadj, exch::adjncy, exch::diagoffset, nd, exch::checkdiag, exch::dataxx,
                                 exch::datayy, exch::datazz);
        matconv::csr_to_dia_offdiag(N, exch::xadj, exch::adjncy, exch::diagoffset, nd, exch::checkdiag, exch::dataxy,
                                    exch::dataxz, exch::datayx, exch::datayz, exch::datazx, exch::datazy);
    } else {
        matconv::csr_to_dia_diag(N, exch::xadj, exch::adjncy, exch::diagoffset, nd, exch::checkdiag, exch::dataxx,
                                 exch::datayy, exch::datazz);
    }
    for (unsigned q = 0; q < nd; q++) offsets[q] = exch::diagoffset[q];
    std::memset(data9, 0, sizeof(double) * 9 * (size_t)nd * n);
    for (int q = 0; q < 9; q++) {
        const bool diag = q == 0 || q == 4 || q == 8;
        if (!diag && !offdiag) continue;
        for (size_t e = 0; e < (size_t)nd * n; e++) data9[(size_t)q * nd * n + e] = (*d[q])[e];
    }
    return 0;
}

}  // extern "C"
