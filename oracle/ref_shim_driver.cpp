// Test-infrastructure driver of the reference-side binding gpu-atomistic-code_b200/shim/cullg_asd.cpp.
//
// Linked with ref_harness.cpp (whose refh_* calls fill the reference's namespace globals) and the
// shim itself, both compiled against the reference's own headers (see oracle/Makefile), and with
// libasd_b200.so.  It defines the few globals the shim reads that the CPU harness does not
// (geom::lu, llg::intscheme, config::seed) and drives cullg::cuinit / cullg::llgGPU* the way
// llg::integrate does (src/llg.cpp:639-664), so a test can run the library through the
// reference's own data contract and compare with the reference's kernels and the oracle.
#include <libconfig.h++>
#include "../inc/arrays.h"
#include "../inc/cuda.h"
#include "../inc/geom.h"
#include "../inc/llg.h"
#include "../inc/spins.h"
#include "../inc/config.h"
#include <cstdint>

namespace geom {
Array2D<int> lu;
}
namespace llg {
unsigned int intscheme = 0;
}
namespace config {
unsigned int seed = 1;
}
namespace cullg {
void asd_configure(uint32_t prec, uint32_t flags);
}

extern "C" {

// geom::lu(i, 0..2) = cell coordinates, lu(i, 4) = unit-cell atom (src/geom.cpp:214-266).
int refs_set_lu(unsigned n, const unsigned* atom, const int* coords) {
    geom::lu.resize(n, 5);
    for (unsigned i = 0; i < n; i++) {
        for (int c = 0; c < 3; c++) geom::lu(i, c) = coords ? coords[3 * i + c] : 0;
        geom::lu(i, 3) = (int)atom[i];
        geom::lu(i, 4) = (int)atom[i];
    }
    return 0;
}

// The unit cell's K1U [J] and axis per atom, and its species (read by the shim's cuinit).
int refs_set_ucm(unsigned nauc, const double* k1u, const double* dir, const unsigned* sublattice) {
    for (unsigned t = 0; t < nauc; t++) {
        geom::ucm.SetK1U(t, k1u[t], dir[3 * t], dir[3 * t + 1], dir[3 * t + 2]);
        geom::ucm.SetSublattice(sublattice[t], t);
    }
    return 0;
}

int refs_configure(unsigned intscheme, unsigned seed, unsigned update, unsigned precision, unsigned flags) {
    llg::intscheme = intscheme;
    config::seed = seed;
    spins::update = update;
    cullg::asd_configure(precision, flags);
    return 0;
}

int refs_cuinit() { cullg::cuinit(); return 0; }

// nsteps calls of the integrator llg::integrate would pick (src/llg.cpp:647-659).
int refs_run(unsigned t0, unsigned nsteps) {
    for (unsigned t = t0; t < t0 + nsteps; t++) {
        if (llg::intscheme == 0) cullg::llgGPU(t);
        else if (llg::intscheme == 1) cullg::llgGPURK4(t);
        else cullg::llgGPURK5(t);
    }
    return 0;
}

int refs_free() { cullg::deallocate_cuda_memory(); return 0; }
}
