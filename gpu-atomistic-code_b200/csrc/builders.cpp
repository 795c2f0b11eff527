// Set-up builders (host, FP64): bond list -> CSR, CSR -> row-aligned DIA,
// point-dipole interaction matrix on the padded mesh, exchange fold.
#include "../../include/asd.h"
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

extern "C" {

// Spins are numbered ((i*d1 + j)*d2 + k)*nauc + t (src/geom.cpp:214-266).  For every
// spin of unit-cell atom a and every bond b with bond_atom[b]==a, the neighbour is
// atom bond_to[b] in cell (i,j,k)+bond_vec[b], wrapped on periodic axes and dropped on
// open ones (src/exch_unitcell.cpp:293-351); value J_b/(mu_a muB) (src/exch_unitcell.cpp:399).
// Bonds are taken in list order, which fixes the CSR column order of each row.
int asd_build_csr(const uint32_t dim[3], const int pbc[3], uint32_t nauc, const double* mu, uint32_t nbond,
                  const uint32_t* bond_atom, const uint32_t* bond_to, const int32_t* bond_vec, const double* bond_J,
                  double muB, uint32_t* xadj, uint32_t* adjncy, double* val, uint32_t* nnz_out) {
    if (!dim || !pbc || !mu || nauc == 0 || !nnz_out) return ASD_EINVAL;
    if (nbond && (!bond_atom || !bond_to || !bond_vec || !bond_J)) return ASD_EINVAL;
    for (uint32_t b = 0; b < nbond; b++)
        if (bond_atom[b] >= nauc || bond_to[b] >= nauc) return ASD_EINVAL;
    if (muB == 0) muB = 9.27e-24;
    const uint64_t n64 = (uint64_t)dim[0] * dim[1] * dim[2] * nauc;
    if (n64 == 0 || n64 >= (1ull << 31)) return ASD_EINVAL;
    const uint32_t n = (uint32_t)n64;
    const bool fill = xadj && adjncy && val;
    uint64_t nnz = 0;
    if (fill) xadj[0] = 0;
    uint32_t row = 0;
    for (uint32_t i = 0; i < dim[0]; i++)
        for (uint32_t j = 0; j < dim[1]; j++)
            for (uint32_t k = 0; k < dim[2]; k++)
                for (uint32_t t = 0; t < nauc; t++, row++) {
                    const int ucc[3] = {(int)i, (int)j, (int)k};
                    for (uint32_t b = 0; b < nbond; b++) {
                        if (bond_atom[b] != t) continue;
                        int lv[3];
                        bool ok = true;
                        for (int x = 0; x < 3; x++) {
                            lv[x] = ucc[x] + bond_vec[3 * b + x];
                            const int d = (int)dim[x];
                            if (lv[x] < 0 || lv[x] >= d) {
                                if (!pbc[x]) { ok = false; break; }
                                lv[x] = ((lv[x] % d) + d) % d;
                            }
                        }
                        if (!ok) continue;
                        const uint32_t col = (((uint32_t)lv[0] * dim[1] + (uint32_t)lv[1]) * dim[2] + (uint32_t)lv[2]) * nauc + bond_to[b];
                        if (fill) {
                            adjncy[nnz] = col;
                            for (int q = 0; q < 9; q++) val[9 * nnz + q] = bond_J[9 * (size_t)b + q] / (mu[t] * muB);
                        }
                        nnz++;
                        if (nnz >= (1ull << 32)) return ASD_EINVAL;
                    }
                    if (fill) xadj[row + 1] = (uint32_t)nnz;
                }
    (void)n;
    *nnz_out = (uint32_t)nnz;
    return ASD_OK;
}

// Row-aligned DIA (data[c][d*N+row] = A[row][row+off[d]]), offsets ascending, built from
// the occupied diagonals of the CSR pattern (src/matrix_conv.cpp:28-272,
// src/exch_unitcell.cpp:374-391).  The reference's diagonal scan stops before offset N-1
// (src/matrix_conv.cpp:43, src/exch_unitcell.cpp:413) and so drops that diagonal; it is kept here.
int asd_csr_to_dia(uint32_t n, const uint32_t* xadj, const uint32_t* adjncy, const double* val9, uint32_t ncomp,
                   int32_t* offsets, double* data9, uint32_t* ndiag_out) {
    if (!xadj || !adjncy || !ndiag_out || n == 0 || (ncomp != 3 && ncomp != 9)) return ASD_EINVAL;
    static const int q3[3] = {0, 4, 8};
    std::vector<uint32_t> occ(2 * (size_t)n, 0);
    for (uint32_t i = 0; i < n; i++)
        for (uint32_t k = xadj[i]; k < xadj[i + 1]; k++) {
            if (adjncy[k] >= n) return ASD_EINVAL;
            occ[(size_t)n + adjncy[k] - i]++;
        }
    std::vector<int32_t> off;
    for (size_t q = 0; q < 2 * (size_t)n; q++)
        if (occ[q]) off.push_back((int32_t)((int64_t)q - n));
    *ndiag_out = (uint32_t)off.size();
    if (!offsets) return ASD_OK;
    if (!data9 || !val9) return ASD_EINVAL;
    memcpy(offsets, off.data(), off.size() * sizeof(int32_t));
    const size_t m = off.size() * (size_t)n;
    memset(data9, 0, ncomp * m * sizeof(double));
    std::vector<int32_t> slot(2 * (size_t)n, -1);
    for (size_t d = 0; d < off.size(); d++) slot[(size_t)((int64_t)off[d] + n)] = (int32_t)d;
    for (uint32_t i = 0; i < n; i++)
        for (uint32_t k = xadj[i]; k < xadj[i + 1]; k++) {
            const size_t d = (size_t)slot[(size_t)n + adjncy[k] - i];
            // a later entry for the same column replaces an earlier one (as the reference scan does)
            for (uint32_t q = 0; q < ncomp; q++)
                data9[(size_t)q * m + d * n + i] = val9[9 * (size_t)k + (ncomp == 3 ? q3[q] : (int)q)];
        }
    return ASD_OK;
}

// nr[(3a+b)*P + cell] += 1e-7 (3 e_a e_b - d_ab)/r^3 * mu_scale * muB for every mesh
// displacement except 0; displacement of index m along an axis of length L=dim*nk is m
// for m <= L and m-2L above (src/intmat.cpp:250-331).  Axes with L < 2 contribute only m=0.
int asd_build_dipole_nr(const uint32_t dim[3], const uint32_t nk[3], const double abc[3], double muB, double mu_scale,
                        double* nr) {
    if (!dim || !nk || !abc || !nr) return ASD_EINVAL;
    if (muB == 0) muB = 9.27e-24;
    uint32_t L[3], M[3];
    bool mono[3];
    for (int l = 0; l < 3; l++) {
        if (!dim[l] || !nk[l]) return ASD_EINVAL;
        L[l] = dim[l] * nk[l];
        M[l] = 2 * L[l];
        mono[l] = L[l] < 2;
    }
    const size_t P = (size_t)M[0] * M[1] * M[2];
    const int I[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
    for (uint32_t i = 0; i < M[0]; i++)
        for (uint32_t j = 0; j < M[1]; j++)
            for (uint32_t k = 0; k < M[2]; k++) {
                if (i == 0 && j == 0 && k == 0) continue;
                const uint32_t m[3] = {i, j, k};
                if ((m[0] && mono[0]) || (m[1] && mono[1]) || (m[2] && mono[2])) continue;
                double r[3];
                for (int l = 0; l < 3; l++) {
                    const int disp = m[l] > L[l] ? (int)m[l] - (int)M[l] : (int)m[l];
                    r[l] = (double)disp * abc[l] / (double)nk[l];
                }
                const double mr = sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
                const double inv3 = 1. / (mr * mr * mr);
                const double e[3] = {r[0] / mr, r[1] / mr, r[2] / mr};
                const size_t cell = ((size_t)i * M[1] + j) * M[2] + k;
                for (int a = 0; a < 3; a++)
                    for (int b = 0; b < 3; b++)
                        nr[(size_t)(3 * a + b) * P + cell] += 1e-7 * ((3.0 * e[a] * e[b]) - I[a][b]) * inv3 * mu_scale * muB;
            }
    return ASD_OK;
}

// Every image of each shell vector under axis permutation and sign change gets the
// shell tensor J/(mu muB) once (src/exch_intmat.cpp:45-140).
int asd_fold_exchange_nr(const uint32_t mesh[3], uint32_t nshell, const int32_t* shell_vec, const double* J9,
                         double mu_muB, double* nr, uint32_t* count) {
    if (!mesh || !nr || (nshell && (!shell_vec || !J9)) || mu_muB == 0) return ASD_EINVAL;
    const size_t P = (size_t)mesh[0] * mesh[1] * mesh[2];
    std::vector<unsigned char> seen(P, 0);
    uint32_t total = 0;
    static const int perm[6][3] = {{0, 1, 2}, {0, 2, 1}, {1, 2, 0}, {1, 0, 2}, {2, 0, 1}, {2, 1, 0}};
    for (uint32_t s = 0; s < nshell; s++) {
        const int32_t* v = shell_vec + 3 * s;
        std::vector<unsigned char> seen_shell(0);
        for (int pq = 0; pq < 6; pq++) {
            const int rc[3] = {v[perm[pq][0]], v[perm[pq][1]], v[perm[pq][2]]};
            for (int sg = 0; sg < 8; sg++) {
                int w[3] = {(sg & 4) ? rc[0] : -rc[0], (sg & 2) ? rc[1] : -rc[1], (sg & 1) ? rc[2] : -rc[2]};
                for (int x = 0; x < 3; x++) {
                    if (std::abs(w[x]) >= (int)mesh[x]) return ASD_EINVAL;
                    if (w[x] < 0) w[x] += (int)mesh[x];
                }
                const size_t cell = ((size_t)w[0] * mesh[1] + w[1]) * mesh[2] + w[2];
                if (seen[cell]) continue;
                for (int q = 0; q < 9; q++) nr[(size_t)q * P + cell] += J9[9 * (size_t)s + q] / mu_muB;
                seen[cell] = 1;
                total++;
            }
        }
    }
    if (count) *count = total;
    return ASD_OK;
}

}  // extern "C"

// ---- initial spins
extern "C" int asd_spins_random(uint32_t n, uint32_t mwc[2], double* out) {
    if (!mwc || !out || mwc[0] == 0 || mwc[1] == 0) return ASD_EINVAL;
    uint32_t x = mwc[0], y = mwc[1];
    // multiply-with-carry pair of 16-bit lags 18000 and 30903, scaled by 1/(2^32-1)
    auto next = [&]() -> double {
        x = 18000u * (x & 0xFFFFu) + (x >> 16);
        y = 30903u * (y & 0xFFFFu) + (y >> 16);
        return (double)((x << 16) + (y & 0xFFFFu)) * (1.0 / 4294967295.0);
    };
    for (uint32_t i = 0; i < n; i++) {
        double v1 = 0.0, v2 = 0.0, s = 2.0;
        while (s > 1.0) {
            v1 = 2.0 * next() - 1.0;
            v2 = 2.0 * next() - 1.0;
            s = v1 * v1 + v2 * v2;
        }
        const double ss = std::sqrt(1.0 - s);
        out[3 * (size_t)i] = 2.0 * v1 * ss;
        out[3 * (size_t)i + 1] = 2.0 * v2 * ss;
        out[3 * (size_t)i + 2] = 1.0 - 2.0 * s;
    }
    mwc[0] = x; mwc[1] = y;
    return ASD_OK;
}

extern "C" int asd_spins_pattern(uint32_t n, uint32_t axis, const int32_t* coords, const uint32_t* atom_of_spin,
                                 const double* init_spin, double* out) {
    if (!out || axis > 3) return ASD_EINVAL;
    if (axis < 3 && !coords) return ASD_EINVAL;
    if (axis == 3 && (!atom_of_spin || !init_spin)) return ASD_EINVAL;
    for (uint32_t i = 0; i < n; i++) {
        double* o = out + 3 * (size_t)i;
        if (axis == 3) {
            for (int c = 0; c < 3; c++) o[c] = init_spin[3 * (size_t)atom_of_spin[i] + c];
        } else {
            const int32_t* r = coords + 3 * (size_t)i;
            o[0] = o[1] = o[2] = 0.0;
            o[axis] = ((r[0] + r[1] + r[2]) % 2 == 0) ? 1.0 : -1.0;
        }
    }
    return ASD_OK;
}

// ---- neighbour-spin staging plan of the fused stage kernel
namespace {
constexpr uint32_t SPIN_SMEM_MAX = 64 * 1024;   // bytes of staged spins (3 components) per block
constexpr uint32_t SPANS_MAX = 24;               // spans per block (one bulk copy per span and component)
constexpr uint32_t SPAN_GAP = 32;                // columns closer than this share one span
constexpr uint32_t SPIN_PAD_ELEMS = 8;           // zeroed elements after each spin array in the library
}  // namespace

int asd_plan_spin_spans(uint32_t n, uint32_t nslices, const uint32_t* slice_ptr, const uint32_t* words,
                        uint32_t colbits, uint32_t elem_bytes, uint32_t block, uint32_t* span_ptr, uint32_t* spans,
                        uint32_t spans_cap, uint32_t* local_words, uint32_t* nspans_out, uint32_t* slots_out) {
    if (!slice_ptr || !words || !span_ptr || !nspans_out || !slots_out || n == 0 || nslices == 0) return ASD_EINVAL;
    if ((elem_bytes != 4 && elem_bytes != 8) || block < 32 || block % 32 || colbits == 0 || colbits > 32)
        return ASD_EINVAL;
    if ((uint64_t)nslices * 32 < n || (uint64_t)nslices * 32 >= (uint64_t)n + 32) return ASD_EINVAL;
    const bool fill = spans != nullptr;
    if (fill && !local_words) return ASD_EINVAL;
    const uint32_t align = 16 / elem_bytes;
    const uint32_t slots_cap = (SPIN_SMEM_MAX / (3 * elem_bytes)) & ~(align - 1);
    const uint32_t mask = colbits >= 32 ? 0xFFFFFFFFu : (1u << colbits) - 1u;
    if (slots_cap > mask) return ASD_ENOTSUP;
    const uint32_t spb = block / 32, nblk = (nslices + spb - 1) / spb;
    const uint64_t limit = (uint64_t)n + SPIN_PAD_ELEMS;
    std::vector<uint32_t> cols;
    std::vector<uint32_t> bs;   // (start, len) pairs of the current block
    uint32_t total_spans = 0, slots_max = 0;
    span_ptr[0] = 0;
    for (uint32_t b = 0; b < nblk; b++) {
        const uint32_t e0 = slice_ptr[b * spb], e1 = slice_ptr[std::min((b + 1) * spb, nslices)];
        if (e1 < e0) return ASD_EINVAL;
        cols.clear();
        for (uint32_t e = e0; e < e1; e++) {
            const uint32_t c = words[e] & mask;
            if (c >= n) return ASD_EINVAL;
            cols.push_back(c);
        }
        std::sort(cols.begin(), cols.end());
        cols.erase(std::unique(cols.begin(), cols.end()), cols.end());
        bs.clear();
        uint32_t total = 0;
        bool fits = !cols.empty();
        for (size_t q = 0; q < cols.size() && fits;) {
            uint32_t hi = cols[q];
            size_t r = q + 1;
            while (r < cols.size() && cols[r] - hi <= SPAN_GAP) hi = cols[r++];
            const uint32_t a0 = cols[q] & ~(align - 1);
            // hi <= n-1, so the aligned end is at most n+align-1 < n+SPIN_PAD_ELEMS; checked all the same
            const uint64_t a1 = ((uint64_t)hi + align) & ~(uint64_t)(align - 1);
            if (a1 > limit) { fits = false; break; }
            if (!bs.empty() && a0 < bs[bs.size() - 2] + bs.back()) {      // aligned spans touch: merge
                const uint32_t end = std::max<uint32_t>(bs[bs.size() - 2] + bs.back(), (uint32_t)a1);
                total += end - (bs[bs.size() - 2] + bs.back());
                bs.back() = end - bs[bs.size() - 2];
            } else {
                bs.push_back(a0);
                bs.push_back((uint32_t)(a1 - a0));
                total += (uint32_t)(a1 - a0);
            }
            if (bs.size() / 2 > SPANS_MAX || total > slots_cap) fits = false;
            q = r;
        }
        const uint32_t nb = fits ? (uint32_t)(bs.size() / 2) : 0;
        if (fill) {
            if (total_spans + nb > spans_cap) return ASD_EINVAL;
            uint32_t off = 0;
            for (uint32_t k = 0; k < nb; k++) {
                uint32_t* t = spans + 4 * (size_t)(total_spans + k);
                t[0] = bs[2 * k]; t[1] = bs[2 * k + 1]; t[2] = off; t[3] = 0;
                off += bs[2 * k + 1];
            }
            for (uint32_t e = e0; e < e1; e++) {
                if (!nb) { local_words[e] = words[e]; continue; }
                const uint32_t c = words[e] & mask;
                uint32_t k = 0, o = 0;
                while (!(c >= bs[2 * k] && c < bs[2 * k] + bs[2 * k + 1])) { o += bs[2 * k + 1]; k++; }
                local_words[e] = (o + (c - bs[2 * k])) | (words[e] & ~mask);
            }
        }
        if (nb) slots_max = std::max(slots_max, total);
        total_spans += nb;
        span_ptr[b + 1] = total_spans;
    }
    *nspans_out = total_spans;
    *slots_out = (slots_max + align - 1) & ~(align - 1);
    return ASD_OK;
}
