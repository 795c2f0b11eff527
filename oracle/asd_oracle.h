/* FP64 CPU oracle for the stochastic-LLG time step of the atomistic
 * spin-dynamics reference (tomostler13/gpu-atomistic-code).
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / reference legs of bench.py may load this library; the
 * product never links or calls it.
 *
 * Parity pinning: the reference ships no tests, golden vectors or fixtures.
 * This restatement is pinned against the reference's own src/llgCPU.cpp,
 * src/matrix_mul_cpu.cpp and src/random.cpp compiled from source
 * (oracle/_ref, see oracle/Makefile), and the GPU-only parts (RK4/RK5,
 * FFT convolution) against their analytic properties; see tests/.
 *
 * Default semantics are the reference CUDA path (src/cuda.cu, src/cuint.cu,
 * src/cufields.cu, src/cuintRK4.cu, src/cuintRK5.cu) with its arithmetic in
 * FP64 and renormalisation as s/|s| (src/llgCPU.cpp:236-239).  The ORC_*
 * flags switch on the reference's documented quirks one by one.
 */
#ifndef ASD_ORACLE_H
#define ASD_ORACLE_H
#include <stdint.h>
#include <stddef.h>
#ifdef __cplusplus
extern "C" {
#endif

/* Quirk flags (bitmask). */
#define ORC_CPU_CORRECTOR_ACCUM   (1u << 0)  /* src/llgCPU.cpp:58-60,253-274: corrector exchange = H(S)+H(S') */
#define ORC_CPU_THERMAL_Z_FROM_X  (1u << 1)  /* src/llgCPU.cpp:180,302: z thermal uses Hthx */
#define ORC_RK_DOUBLE_RDT         (1u << 2)  /* src/cuintRK4.cu:141-142, src/cuintRK5.cu:158-159: stage uses rdt*k with k incl. rdt */
#define ORC_RK_STAGE_SPIN_MIXED   (1u << 3)  /* src/cuintRK4.cu:172,266,359; src/cuintRK5.cu:189,283,376,468,560: es={eS.x,S.y,eS.z} */
#define ORC_GPU_CSR_DIP_STALE     (1u << 4)  /* src/cuda.cu:192-199: CSR+dipole+diag corrector keeps the predictor field */
#define ORC_CPU_SUM_ORDER         (1u << 5)  /* src/llgCPU.cpp:180,302: llgCPU order of the field terms */
#define ORC_GPU_DZZ_FROM_DYY      (1u << 6)  /* src/cuda_util.cu:308-312,373-377: zz exchange from yy */
#define ORC_GPU_HDEMAG_FP32       (1u << 7)  /* src/cuda_glob.cu: CHDemag stored as float */

/* Exchange storage. */
#define ORC_EXCH_NONE 0
#define ORC_EXCH_DIA  1
#define ORC_EXCH_CSR  2

/* Long-range field. */
#define ORC_LR_NONE   0
#define ORC_LR_DIPOLE 1   /* exchm>0 + Include_dipole: refreshed every `update` steps at stage 1 */
#define ORC_LR_FFT    2   /* exchm==0: full field from the interaction matrix at every stage */

/* Integrators (llg::intscheme, src/llg.cpp:322-333). */
#define ORC_HEUN 0
#define ORC_RK4  1
#define ORC_RK5  2

/* Noise sources. */
#define ORC_NOISE_PHILOX 0  /* the product's generator: Philox4x32-10 + Box-Muller */
#define ORC_NOISE_MWC    1  /* the reference CPU generator: MWC1616 + Marsaglia polar */
#define ORC_NOISE_BUFFER 2  /* caller-supplied normals, 3 per spin per step */

typedef struct orc_ctx orc_ctx;

orc_ctx* orc_create(uint32_t n);
void orc_destroy(orc_ctx* c);

/* Per-spin material, already expanded: llgpf, lambda, sigma (src/llg.cpp:591-592,626-631),
 * k1u as 2K/(mu muB) and its unit axis (src/geom.cpp:244-247). */
int orc_set_material(orc_ctx* c, const double* llgpf, const double* lambda, const double* sigma,
                     const double* k1u, const double* k1udir);
/* Global K2/K4 terms (src/cuint.cu:32-41); basemm = mu(atom 0)*muB. */
int orc_set_global_anis(orc_ctx* c, double k2perp, const double* k2perpdir, double k2par, const double* k2pardir,
                        double k4perp, const double* k4perpdirs, double k4par, const double* k4pardirs, double basemm);
int orc_set_dynamics(orc_ctx* c, int integrator, double rdt, const double* applied);
/* Replicas: contiguous spin ranges [off[r],off[r+1]) with their own temperature and Philox stream. */
int orc_set_replicas(orc_ctx* c, uint32_t nrep, const uint32_t* off, const double* T, const uint32_t* stream);
/* CSR with nnz x 9 values (alpha,beta row-major, [T]); full=0 uses xx,yy,zz only. */
int orc_set_csr(orc_ctx* c, int full, uint32_t nnz, const uint32_t* xadj, const uint32_t* adjncy, const double* val9);
/* Row-aligned DIA: data[comp][n*N+row] for 9 comps (src/matrix_conv.cpp:28-272). */
int orc_set_dia(orc_ctx* c, int full, uint32_t ndiag, const int32_t* offsets, const double* val9);
int orc_set_site_field(orc_ctx* c, const double* hstag, double scale);
/* Gaussian time envelope of the site field: multiplier amp exp(-((t dt - t0)/sigma)^2 / 2). */
int orc_set_pulse(orc_ctx* c, double amp, double t0, double sigma, double dt);
/* Four-spin quartets (CSR over spins, ptr[n+1]; j, k, l) with JQ [T]; div3 selects the GPU
 * path's division by 3 (src/cufields.cu:76-78).  ptr NULL removes the term. */
int orc_set_four_spin(orc_ctx* c, const uint32_t* ptr, const uint32_t* j, const uint32_t* k, const uint32_t* l,
                      double jq, int div3);
/* Long-range field by direct summation on the periodic padded mesh:
 * H_i = sum_j Nr[s_i][s_j][a][b][(x_i-x_j) mod n] * w_j * S_j[b], with w_j = mu_j for
 * ORC_LR_DIPOLE (src/cufields.cu:355) and 1 for ORC_LR_FFT (src/cufields.cu:381).
 * nr is [nspec][nspec][3][3][n0][n1][n2]; mesh is 3 ints per spin; spec per spin (or NULL). */
int orc_set_longrange(orc_ctx* c, int mode, const uint32_t* mesh_dims, const uint32_t* mesh_xyz,
                      uint32_t nspec, const uint32_t* spec, const double* nr, const double* w, uint32_t update);
int orc_set_flags(orc_ctx* c, uint32_t flags);
int orc_set_noise(orc_ctx* c, int mode, uint64_t seed, uint32_t mwc_a, uint32_t mwc_b,
                  const double* buf, size_t buf_len);
int orc_set_spins(orc_ctx* c, const double* s);
int orc_get_spins(const orc_ctx* c, double* s);
int orc_get_det_field(const orc_ctx* c, double* h);
/* The exchange + long-range field of the current spins (what CH holds after the stage-1 SpMV). */
int orc_field(orc_ctx* c, double* h);
int orc_run(orc_ctx* c, uint64_t t0, uint64_t nsteps);
/* Sublattice mean per replica (src/util_mag.cpp:44-65): out[(r*nsub+s)*3+c]. */
int orc_magnetisation(const orc_ctx* c, uint32_t nsub, const uint32_t* sublattice, double* out);

/* Noise generators, exposed for known-answer tests. */
void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
void orc_thermal_normals(uint64_t seed, uint32_t stream, uint32_t spin, uint64_t step, double out[3]);
void orc_thermal_normals_f(uint64_t seed, uint32_t stream, uint32_t spin, uint64_t step, float out[3]);
double orc_log(double x);
void orc_sincos_2pi(uint32_t x, double* s, double* co);
void orc_mwc_seed(uint32_t a, uint32_t b);
double orc_mwc_rand(void);
double orc_mwc_normal(void);

/* Setup-time restatements used to check the product's builders. */
/* CSR -> row-aligned DIA (src/matrix_conv.cpp:28-272); returns ndiag; offsets/data sized by caller
 * (data 9 x ndiag x n).  Pass offsets=NULL to count only. */
int orc_csr_to_dia(uint32_t n, const uint32_t* xadj, const uint32_t* adjncy, const double* val9,
                   int32_t* offsets, double* data9);
/* Point-dipole interaction matrix on the padded mesh (src/intmat.cpp:188-331), FP64, one species:
 * nr[3][3][n0][n1][n2] += 1e-7*(3 e_a e_b - d_ab)/r^3 * muB * mu_scale. dim = lattice cells,
 * nk = mesh points per cell, abc = lattice constants [m]; mesh = 2*dim*nk per axis. */
int orc_build_dipole_nr(const uint32_t* dim, const uint32_t* nk, const double* abc, double muB,
                        double mu_scale, double* nr);
/* Exchange fold (src/exch_intmat.cpp:28-163) for one species pair: every sign/permutation
 * image of each shell vector (in mesh units) gets J/(mu muB) once. */
int orc_fold_exchange_nr(const uint32_t* mesh, uint32_t nshell, const int32_t* shell_vec,
                         const double* J9, double mu_muB, double* nr);

#ifdef __cplusplus
}
#endif
#endif
