/*
 * asd.h - C ABI of the B200-native stochastic Landau-Lifshitz-Gilbert step.
 *
 * Drop-in replacement for the integrator layer of tomostler13/gpu-atomistic-code
 * (the reference).  Every entry point below names the reference interface it
 * replaces (path:line inside the reference project).  Signatures use plain C
 * types, pointers and sizes only; no C++ or PyTorch types cross this boundary.
 *
 * Conventions
 *  - Spins, fields and other per-spin vectors cross the boundary as host arrays
 *    of doubles in spin-major order [3*i+c], the layout of the reference's device
 *    arrays (src/cuda.cu:239-252).  Replicas are concatenated in the order given
 *    to asd_create.
 *  - Every call returns ASD_OK (0) or a positive ASD_E* code and never exits the
 *    process (the reference calls exit(0) on errors, src/error.cpp:19-28).  After
 *    a failure asd_last_error() returns a message.
 *  - A handle owns one CUDA stream on the device current at asd_create; calls on
 *    one handle are not thread-safe, distinct handles are independent.
 */
#ifndef ASD_H
#define ASD_H
#include <stddef.h>
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

/* Status codes */
#define ASD_OK        0
#define ASD_EINVAL    1  /* bad argument or inconsistent input */
#define ASD_ECUDA     2  /* CUDA runtime error (message has the CUDA string) */
#define ASD_ENOMEM    3  /* device allocation failed */
#define ASD_ETIMEOUT  4  /* a bounded device-side wait ran out */
#define ASD_ESTATE    5  /* call not valid in the handle's state */
#define ASD_ECUFFT    6  /* cuFFT error */
#define ASD_ENOTSUP   7  /* combination not supported */
#define ASD_ENOTFINITE 8 /* a non-finite spin was produced or supplied */

/* Integrators: llg::intscheme (src/llg.cpp:309-341). */
#define ASD_HEUN 0
#define ASD_RK4  1
#define ASD_RK5  2

/* Arithmetic forms of the step. */
#define ASD_FP64_PLAIN 0  /* FP64, one thread per spin, separate noise/SpMV/stage launches (reference-structured) */
#define ASD_FP32       1  /* FP32 state and fields, FP64 renormalisation, fused stage kernels, CUDA graph */
#define ASD_FP64_FUSED 2  /* the fused stage kernels instantiated in FP64 */

/* Exchange storage: config::exchm (src/config.cpp:139-159) plus "none". */
#define ASD_EXCH_FFT  0   /* exchange folded into the k-space interaction matrix */
#define ASD_EXCH_DIA  1
#define ASD_EXCH_CSR  2
#define ASD_EXCH_NONE 3

/* Long-range (dipolar) field. */
#define ASD_LR_NONE   0
#define ASD_LR_DIPOLE 1   /* Include_dipole with CSR/DIA exchange, refreshed every `update` steps */
#define ASD_LR_FFT    2   /* exchm==0: the whole field from the interaction matrix at every stage */

/* Reference-compatibility switches (asd_params.flags).  Default 0 = the CUDA
 * path's physics with its bugs fixed. */
#define ASD_FLAG_RK_DOUBLE_RDT       (1u << 2)  /* src/cuintRK4.cu:141-142, src/cuintRK5.cu:158-159 */
#define ASD_FLAG_RK_STAGE_SPIN_MIXED (1u << 3)  /* src/cuintRK4.cu:172: es={Cespin[3i],Cspin[3i+1],Cespin[3i+2]} */
#define ASD_FLAG_GPU_CSR_DIP_STALE   (1u << 4)  /* src/cuda.cu:192-199 */
#define ASD_FLAG_GPU_DZZ_FROM_DYY    (1u << 6)  /* src/cuda_util.cu:308-312,373-377 */
#define ASD_FLAG_GPU_HDEMAG_FP32     (1u << 7)  /* CHDemag stored as float (src/cuda_glob.cu) */
#define ASD_FLAG_COMPENSATED         (1u << 16) /* FP32 form: spins kept as float hi+lo pairs */
#define ASD_FLAG_AUTOTUNE            (1u << 17) /* FP32 form: time block shapes at create */
#define ASD_FLAG_STREAMED_EXCHANGE   (1u << 18) /* fused forms: keep every tensor in the matrix stream
                                                   instead of the typed (column, tensor-id) layout */
#define ASD_FLAG_CUFFT_PLANES        (1u << 19) /* fused forms: run the (x, y) passes of the long-range
                                                   transform through cuFFT instead of the library's
                                                   plane kernels (comparison aid) */
#define ASD_FLAG_WAIT_TIMEOUT           (1u << 20) /* test aid: the device-side waits for bulk copies give
                                                   up at once and take their time-out path (the stage
                                                   kernels then read global memory, results unchanged;
                                                   the x transform leaves its tile, an invalid field);
                                                   the wait before a block retires keeps its bound;
                                                   asd_sync reports ASD_ETIMEOUT */
#define ASD_FLAG_SERIAL_LAUNCH       (1u << 21) /* fused forms: launch the step kernels strictly one
                                                   after another (no programmatic dependent launch:
                                                   a comparison aid) */

#define ASD_ALL_REPLICAS 0xFFFFFFFFu

/* Per unit-cell atom (the reference's unitCellMembers, inc/unitcell.h). */
typedef struct asd_material {
    double mu;          /* moment [muB] (GetMu) */
    double lambda;      /* Gilbert damping (GetDamping) */
    double gamma;       /* gyromagnetic ratio relative to 1.76e11 (GetGamma) */
    double k1u;         /* first-order uniaxial constant [J/atom] (GetK1U) */
    double k1u_dir[3];  /* its unit axis (GetK1UDir) */
    uint32_t sublattice;/* magnetic species (GetSublattice) */
} asd_material;

/* Run parameters: the llg{} and anis{} settings plus the RNG seed. */
typedef struct asd_params {
    uint32_t integrator;   /* ASD_HEUN / ASD_RK4 / ASD_RK5 */
    uint32_t precision;    /* ASD_FP64_PLAIN / ASD_FP32 / ASD_FP64_FUSED */
    double dt;             /* time step [s] (llg.dt) */
    double applied[3];     /* applied field [T] (llg.applied) */
    double k2perp, k2perpdir[3], k2par, k2pardir[3];        /* [J], unit axes (anis.*) */
    double k4perp, k4perpdirs[9], k4par, k4pardirs[9];      /* 3 axes each, row-major */
    uint64_t seed;         /* Philox key for the thermal field */
    uint32_t update;       /* dipole refresh period in steps (llg.update); 0 -> 1 */
    uint32_t flags;        /* ASD_FLAG_* */
    double gyro, muB, kB;  /* 0 -> the reference constants 1.76e11, 9.27e-24, 1.38e-23 (src/llg.cpp:25) */
} asd_params;

/* One lattice (replica) and its interactions. */
typedef struct asd_system {
    uint32_t nspins;
    uint32_t nmat;                  /* unit-cell atoms described by mat[] */
    const asd_material* mat;
    const uint32_t* atom;           /* unit-cell atom of each spin (geom::lu(i,4)); NULL -> i % nmat */
    uint32_t exch;                  /* ASD_EXCH_* */
    uint32_t exch_full;             /* 0: xx,yy,zz only; 1: full 3x3 (config::offdiag) */
    /* CSR (exch == ASD_EXCH_CSR): exch::xadj / adjncy / data** */
    const uint32_t* xadj;           /* nspins+1 */
    const uint32_t* adjncy;         /* nnz */
    uint32_t nnz;
    const double* csr_val;          /* nnz x 9 [T], row-major (alpha,beta); diagonal form reads 0,4,8 */
    /* DIA (exch == ASD_EXCH_DIA): exch::diagoffset / data**, row-aligned data[c][n*N+row] */
    uint32_t ndiag;
    const int32_t* dia_offset;      /* ndiag */
    const double* dia_val;          /* c x ndiag x nspins [T]: c=3 (xx,yy,zz) if !exch_full, else 9 */
    /* Long-range field on the zero-padded mesh (intmat::dipNrab / Nrab before the FFT). */
    uint32_t lr;                    /* ASD_LR_* */
    uint32_t mesh[3];               /* padded mesh 2*dim*Nm per axis */
    const uint32_t* mesh_xyz;       /* 3 per spin: geom::lu(i,0..2) */
    const double* nr;               /* real-space matrix [3][3][mesh0][mesh1][mesh2], FP64 */
    double temperature;             /* [K] (llg::T) */
    uint32_t stream;                /* Philox stream of this replica */
    const double* site_field;       /* 3N staggered/site field [T] (fields::Hstag*), or NULL */
} asd_system;

typedef struct asd_handle asd_handle;

/* cullg::cuinit (src/cuda.cu:261-402) + llg::initLLG prefactors (src/llg.cpp:585-631):
 * uploads nsys replicas, derives sigma / llgpf / k1u per atom, builds device layouts,
 * FFT plans and N_k. */
int asd_create(const asd_params* p, const asd_system* sys, uint32_t nsys, asd_handle** out);
/* cullg::deallocate_cuda_memory (src/cuda_util.cu:186-242). */
int asd_destroy(asd_handle* h);
/* Message of the last failure on h; with h == NULL, of the calling thread's last failed asd_create. */
const char* asd_last_error(const asd_handle* h);
const char* asd_version(void);

/* Initial spins (spins::Sx/Sy/Sz uploaded in allocate_memory_on_card, src/cuda_util.cu:536-537);
 * s: 3*nspins_total doubles, normalised on upload. */
int asd_set_spins(asd_handle* h, const double* s, size_t n_spins);
/* Spin read-back (the D2H copy of src/cuda.cu:239-246). */
int asd_get_spins(asd_handle* h, double* s, size_t n_spins);
/* CDetFields read-back (src/cuda.cu:247-252): total field minus thermal at the last corrector. */
int asd_get_det_field(asd_handle* h, double* hout, size_t n_spins);
/* The field of the current spins without thermal, anisotropy, applied and site terms
 * (CH after the stage-1 field kernels, src/cufields.cu:201-203, 405). */
int asd_get_field(asd_handle* h, double* hout, size_t n_spins);

/* llg::integrate(t) x nsteps (src/llg.cpp:639-664 -> cullg::llgGPU / llgGPURK4 / llgGPURK5). */
int asd_step(asd_handle* h, uint64_t nsteps);
int asd_get_step(const asd_handle* h, uint64_t* t);
int asd_set_step(asd_handle* h, uint64_t t);
int asd_sync(asd_handle* h);

/* Exact state for checkpoint and restart, the binary counterpart of the reference's restart
 * files (spins::restart_text, src/spins.cpp:342-398, which print the spins as text): the spins in
 * the form's own storage (FP32 hi+lo pairs, or FP64), the step counter, the replicas' bath
 * temperatures and the two-temperature model's state.  buf == NULL: *len = the size needed.
 * Parameters (applied field, site-field ramp, flags) are the caller's and are not included. */
int asd_get_state(asd_handle* h, void* buf, size_t* len);
/* Restore a state taken from a handle created with the same parameters and lattice (and the
 * two-temperature model started when the state carries one): no renormalisation, so the next
 * steps are bit-identical to those of the run the state was taken from. */
int asd_set_state(asd_handle* h, const void* buf, size_t len);

/* llg::T (passed per launch, src/cuda.cu:159); replica ASD_ALL_REPLICAS sets all. */
int asd_set_temperature(asd_handle* h, uint32_t replica, double T);
/* llg::applied (src/cuda.cu:159), in effect from the next step.  In the fused forms a following
 * asd_step(h, 1) carries it in its one-step graph (no launch of its own); any other call that
 * reads it on the device sends it first. */
int asd_set_applied(asd_handle* h, const double applied[3]);
/* cullg::CsetStagFields / CsetStagFieldsZero (src/cuda_util.cu:563-588): profile 3N [T], NULL zeroes it. */
int asd_set_site_field(asd_handle* h, const double* profile, size_t n_spins);
/* cullg::rampStag(rv) (src/cuda.cu:38-41): site field = rv * profile. */
int asd_set_site_field_scale(asd_handle* h, double rv);

/* Time envelope of the site field, the in-step form of a driver calling rampStag every step
 * (src/cuda.cu:38-41, src/ramp_stag.cpp): site field = rv * amp * exp(-(t-t0)^2/(2 sigma^2)) *
 * profile with t = step*dt [s]; amp = 0 switches the envelope off (site field = rv * profile). */
int asd_set_site_field_pulse(asd_handle* h, double amp, double t0, double sigma);

/* util::calc_mag method 0 (src/util_mag.cpp:44-65) per replica: out[(r*nsub+s)*3+c], FP64 sums.
 * A page-locked `out` (cudaHostAlloc / cudaHostRegister) that this device can address receives
 * the means from the reduction kernel itself; any other buffer by a copy.  Returns after both. */
int asd_magnetisation(asd_handle* h, double* out, size_t out_len);
/* Sublattice-mean magnetisation of spins that already sit in device memory, without any
 * device allocation.  No counterpart in the reference: it exists for callers that cannot call
 * cudaMalloc/cudaFree where they need the result - a host that hands all device memory to its
 * own pool allocator and runs at its limit, or a loop that must avoid cudaFree's device-wide
 * synchronisation.
 *   d_spins: 3*nspins doubles [3i+c] on the current device; d_sublattice: nspins sublattice
 *   indices on the device, or NULL for one sublattice (spins whose index is nsub or more are
 *   left out of every sum); d_out: nsub*3 doubles on the device; stream: a cudaStream_t
 *   (NULL = legacy default stream).  Work is enqueued on the stream; the call returns without
 *   waiting.
 * Scratch is a static device array of ASD_NOALLOC_MAX_BLOCKS x ASD_NOALLOC_MAX_SUBLATTICES x 4
 * doubles (1 MiB) that every GPU loading the library keeps until exit; nsub above
 * ASD_NOALLOC_MAX_SUBLATTICES is rejected with ASD_EINVAL.  The first call on a device looks
 * up the array's device address (kept for the process; a device reset invalidates it, so do
 * not call this on a device after cudaDeviceReset) and should come before any stream capture.
 * All calls share the array: calls that overlap on the GPU (different streams, no ordering)
 * race. */
#define ASD_NOALLOC_MAX_BLOCKS 2048
#define ASD_NOALLOC_MAX_SUBLATTICES 16
int asd_magnetisation_noalloc(const double* d_spins, uint32_t nspins, const uint32_t* d_sublattice, uint32_t nsub,
                              double* d_out, void* stream);
/* M(T) statistics kept on the device, the RunningStat of sim::MvT (src/mvt.cpp:258-275,
 * inc/util.h:22-75): each sample computes every replica's sublattice means and pushes
 * |m_s| into a Welford accumulator per (replica, sublattice).  Sampling enqueues work on
 * the handle's stream and returns without a host synchronisation. */
int asd_sample_magnetisation(asd_handle* h);
/* out[(r*nsub+s)*4 + k], k = 0: samples, 1: mean |m_s|, 2: variance (n-1 normalised),
 * 3: the mean before the last sample (MvT's convergence test uses both means). */
int asd_magnetisation_stats(asd_handle* h, double* out, size_t out_len);
int asd_reset_magnetisation_stats(asd_handle* h);
/* In-situ S(q,t) sampling, the spin-map transform of sim::timeseries (src/timeseries.cpp:274-330):
 * psi(r) = uo_a S_a + i uo_b S_b with (a,b) the axes transverse to qaxis (0: y,z; 1: x,z; 2: x,y),
 * uo[s*3+c] per sublattice (NULL: all 1), forward 3D FFT on the lattice mesh mesh[3] with each
 * spin at mesh_xyz (3 per spin), psi_k kept on the device for the nk k-points kpoints (3 mesh
 * indices each) per sample, up to max_samples samples.  One replica per handle. */
int asd_sq_setup(asd_handle* h, uint32_t qaxis, const double* uo, const uint32_t mesh[3], const uint32_t* mesh_xyz,
                 uint32_t nk, const uint32_t* kpoints, uint32_t max_samples);
/* Record psi_k of the current spins (enqueued on the handle's stream, no host synchronisation). */
int asd_sq_sample(asd_handle* h);
/* Copy the recorded series out: out[(sample*nk + k)*2 + {re, im}]; *nsamples = samples recorded. */
int asd_sq_get(asd_handle* h, double* out, size_t out_len, uint32_t* nsamples);
/* Four-spin exchange, cufields::CSpMV_CSR_FourSpin (src/cufields.cu:59-90) and llgCPU
 * (src/llgCPU.cpp:142-170): for each quartet (j, k, l) of spin i, listed CSR-style in
 * adj_j/adj_k/adj_l[xadj_jkl[i] .. xadj_jkl[i+1]),
 *   H_i -= JQ (S_j (S_k.S_l) + S_k (S_j.S_l) + S_l (S_k.S_j))    [/ 3 on the GPU path: divide_by_3]
 * added to the exchange field at every field evaluation.  JQ in tesla.  xadj_jkl == NULL removes
 * the term. */
int asd_set_four_spin(asd_handle* h, const uint32_t* xadj_jkl, const uint32_t* adj_j, const uint32_t* adj_k,
                      const uint32_t* adj_l, double JQ, int divide_by_3);

/* Two-temperature model of the laser-heating driver (src/laser_heating.cpp:648-676, CalcTe at
 * :884-895): every step, before integrating it, the electron and lattice temperatures advance as
 *   P  = fluence * sum_p scale_p exp(-((t - delay_p) / pump_time)^2),  t = (step - start) dt
 *   Te = (-G (Te - Tl) + P) dt / (gamma_e Te) + Te
 *   Tl = ( G (Te - Tl) - Cl (Tl - T0) / cooling_time) dt / Cl + Tl      (with the new Te)
 * and every replica's spin bath takes Te (bath_is_electrons) or Tl.  Runs on the device inside
 * the step, so the temperature never crosses to the host. */
#define ASD_TTM_MAX_PULSES 16
typedef struct asd_ttm {
    double gamma_e;        /* Ce(Te) = gamma_e Te */
    double Cl;             /* lattice specific heat */
    double G_ep;           /* electron-phonon coupling */
    double pump_time;      /* Gaussian width tau [s] */
    double pump_fluence;   /* laser power */
    double cooling_time;   /* [s] */
    double initial_T;      /* T0 = Te = Tl at the start [K], > 1e-5 */
    uint32_t npulses;      /* <= ASD_TTM_MAX_PULSES */
    uint32_t bath_is_electrons;
    double pulse_scale[ASD_TTM_MAX_PULSES];
    double pulse_delay[ASD_TTM_MAX_PULSES];
} asd_ttm;
/* Start the two-temperature model at the current step (NULL stops it; the spin bath keeps the
 * last temperature). */
int asd_set_ttm(asd_handle* h, const asd_ttm* ttm);
/* Current electron and lattice temperatures of the model. */
int asd_get_ttm_temperatures(asd_handle* h, double* Te, double* Tl);

/* Dynamic structure factor of the recorded series, per k-point, on the device: replaces the
 * time-series analysis tool fourier_space_analysis/src/timeseries.cpp:142-275.
 *   window 0: none; 1: generalised Hamming alpha - beta cos(2 pi t / (ns - 1))   (:185-189)
 *   forward FFT in time, divided by mesh points x ns                             (:143, :124, :198-203)
 *   one-sided PSD raw[w] = |X(w)|^2 + |X(ns - 1 - w)|^2, w < ns/2                (:225-235)
 *   smooth = Alvarez-Mazorra recursive Gaussian of raw, 10 passes,
 *            width round(width_hz * ns * sample_dt) bins                         (:153, :237, :289-325)
 *   peaks: argmax of smooth (w >= 0) and of raw (w > 1) with fcut_lo < w 2 pi / (ns sample_dt) < fcut_hi (:242-256)
 * raw and smooth are [nk][ns/2] (either may be NULL); peak_raw / peak_smooth are [nk] bin indices
 * (0 when no bin qualifies).  ASD_EINVAL when fewer than 2 samples or the width rounds to 0 bins. */
int asd_sq_spectrum(asd_handle* h, uint32_t window, double alpha, double beta, double width_hz, double sample_dt,
                    double fcut_lo, double fcut_hi, double* raw, double* smooth, size_t len, uint32_t* peak_raw,
                    uint32_t* peak_smooth);
/* Number of sublattices (GetNMS) of the handle. */
int asd_num_sublattices(const asd_handle* h, uint32_t* nsub);

/* Time nsteps asd_step calls on the device with CUDA events on the handle's stream;
 * *ms = elapsed milliseconds, *launches = kernels this library launched. */
int asd_time_steps(asd_handle* h, uint64_t nsteps, double* ms, uint64_t* launches);
/* Advance nsteps with direct (un-graphed) launches, bracketing every fused stage-kernel and
 * long-range plane-kernel launch with CUDA events on the handle's stream; results via
 * asd_kernel_stats / asd_kernel_table.
 * Measurement aid with no reference counterpart. */
int asd_time_kernels(asd_handle* h, uint64_t nsteps);
/* As asd_time_kernels, with a device buffer of flush_bytes written before every timed launch so
 * each launch starts with a cold L2 (flush_bytes > L2 size). */
int asd_time_kernels_cold(asd_handle* h, uint64_t nsteps, uint64_t flush_bytes);
/* Device time of nsteps steps, each preceded by an untimed write of flush_bytes (> L2 size) and
 * bracketed by its own CUDA events; *ms = sum over the steps.  Measurement aid. */
int asd_time_steps_cold(asd_handle* h, uint64_t nsteps, uint64_t flush_bytes, double* ms, uint64_t* launches);
/* Device time of the dominant kernel of the last asd_time_kernels (the one with the largest
 * summed time over its launches): average ms per launch, launch count and algorithmic bytes per
 * launch.  Measurement aid. */
int asd_kernel_stats(const asd_handle* h, char* name, size_t name_len, double* avg_ms, uint64_t* count,
                     double* bytes_per_launch);
/* Every kernel timed in the last asd_time_kernels, one line each: "name|avg_ms|count|bytes\n";
 * ASD_EINVAL when out_len is too small.  Measurement aid. */
int asd_kernel_table(const asd_handle* h, char* out, size_t out_len);
/* Launch shape of the fused stage kernel chosen at create (block size, shared-memory staging of
 * the typed exchange words), with ASD_FLAG_AUTOTUNE the autotuner's timings, and the transform
 * path of the long-range field. */
int asd_tuning(const asd_handle* h, char* out, size_t out_len);
/* Set the fused stage kernel's launch shape by hand: block in {64, 128, 256}; staging 1 stages
 * each block's typed exchange words in shared memory by bulk copy, staging 2 also the spans of
 * neighbour spins its rows read (each falls back to the lower mode where the layout is not
 * typed SELL or the data do not fit).  Results do not depend on the shape. */
int asd_set_launch_shape(asd_handle* h, uint32_t block, uint32_t staging);
/* Device layout of the fused kernels: for a DIA matrix ASD_EXCH_DIA (row-aligned diagonals, the
 * reference's layout) or ASD_EXCH_CSR (the same entries as SELL-32, summed in the same order);
 * for a CSR matrix of one replica whose entries lie on at most 32 diagonals (a regular lattice)
 * ASD_EXCH_CSR (SELL-32) or ASD_EXCH_DIA (typed diagonals, summed in ascending diagonal order).
 * The autotuner chooses between them.  Measurement and tuning aid. */
int asd_set_device_layout(asd_handle* h, uint32_t layout);

/* The thermal normals the step uses for (seed, stream, step): 3 per spin for spins
 * [0, nspins), computed by the device generator (Philox4x32-10 + Box-Muller). */
int asd_thermal_normals(uint64_t seed, uint32_t stream, uint64_t step, uint32_t nspins, double* out);
/* The FP32 form's normals for the same (seed, stream, step): the same Philox draw through
 * the single-precision Box-Muller series. */
int asd_thermal_normals_f32(uint64_t seed, uint32_t stream, uint64_t step, uint32_t nspins, float* out);

/* --- set-up builders (host C++, FP64) ---------------------------------------- */
/* Bond list -> CSR as exch::exchunitcell does (src/exch_unitcell.cpp:265-489): spins ordered
 * (i,j,k,t) with t innermost (src/geom.cpp:214-266); bond b of unit-cell atom a_b to atom
 * t_b in the cell offset vec_b (3 ints) with tensor J_b (9 doubles [J]); value J/(mu_a muB).
 * Pass xadj/adjncy/val = NULL to get *nnz only. */
int asd_build_csr(const uint32_t dim[3], const int pbc[3], uint32_t nauc, const double* mu,
                  uint32_t nbond, const uint32_t* bond_atom, const uint32_t* bond_to, const int32_t* bond_vec,
                  const double* bond_J, double muB, uint32_t* xadj, uint32_t* adjncy, double* val, uint32_t* nnz);
/* matconv::csr_to_dia_diag / csr_to_dia_offdiag (src/matrix_conv.cpp:28-272): returns ndiag in
 * *ndiag; data is ncomp x ndiag x n with ncomp 3 (xx,yy,zz) or 9; pass offsets/data = NULL to
 * count only. */
int asd_csr_to_dia(uint32_t n, const uint32_t* xadj, const uint32_t* adjncy, const double* val9, uint32_t ncomp,
                   int32_t* offsets, double* data, uint32_t* ndiag);
/* intmat::fillDipIntmat / fillIntmat (src/intmat.cpp:188-331): nr[3][3][2dim*nk] (+=). */
int asd_build_dipole_nr(const uint32_t dim[3], const uint32_t nk[3], const double abc[3], double muB,
                        double mu_scale, double* nr);
/* exch::fft (src/exch_intmat.cpp:28-163): fold shell tensors into nr (+=); returns images in *count. */
int asd_fold_exchange_nr(const uint32_t mesh[3], uint32_t nshell, const int32_t* shell_vec,
                         const double* J9, double mu_muB, double* nr, uint32_t* count);

/* Initial spins of the reference's spin-config modes (host only), n x 3 doubles out.
 * random: spins::setSpinsRandom (src/spins.cpp:265-281), Marsaglia's (1972) point on the sphere
 * from Random::rand of the MWC1616 stream (src/random.cpp:17-40) whose state (x, y) is taken
 * from and returned in mwc[2] (both non-zero, as Random::seed demands). */
int asd_spins_random(uint32_t n, uint32_t mwc[2], double* out);
/* chequer: spins::setSpinsChequerX/Y/Z (src/spins.cpp:282-341): +e_axis where the cell
 * coordinates (geom::lu(i,0..2), n x 3) sum to an even number, -e_axis elsewhere; axis 0..2.
 * config (axis 3): spins::setSpinsConfig (src/spins.cpp:254-264), the initial spin of each
 * spin's unit-cell atom, init_spin[3 * atom_of_spin[i] + c] (coords unused). */
int asd_spins_pattern(uint32_t n, uint32_t axis, const int32_t* coords, const uint32_t* atom_of_spin,
                      const double* init_spin, double* out);

/* Neighbour-spin staging plan of the fused stage kernel (host only, no device needed).  For
 * SELL-32 slices (nslices, slice_ptr[nslices+1]) of typed words (column in the low colbits bits)
 * and blocks of `block` rows: each block's distinct columns are merged into spans (gaps of at
 * most 32 joined), widened to 16-byte boundaries of elem_bytes-sized elements and given
 * consecutive shared-memory slots.  A block whose spans exceed 24 or 64 KB of 3-component spins
 * gets none and keeps global columns.  Outputs span_ptr[nblocks+1], spans[4*k] = (start, len,
 * slot offset, 0), local_words[E] (column replaced by the slot), *nspans and *slots (largest
 * block's slots).  spans == NULL: counts only (span_ptr still filled). */
int asd_plan_spin_spans(uint32_t n, uint32_t nslices, const uint32_t* slice_ptr, const uint32_t* words,
                        uint32_t colbits, uint32_t elem_bytes, uint32_t block, uint32_t* span_ptr, uint32_t* spans,
                        uint32_t spans_cap, uint32_t* local_words, uint32_t* nspans, uint32_t* slots);

/* ---- input files of the reference (no libconfig needed); messages go to err[err_len] ---- */
/* One atom of a unit-cell (.ucf) file. */
typedef struct asd_ucf_atom {
    uint32_t sublattice;       /* magnetic species */
    double xred[3];            /* reduced coordinates */
    int32_t mesh_point[3];     /* position on the unit cell's k-mesh (only when mesh_points) */
    double mu, damping, gamma; /* [muB], Gilbert damping, relative to 1.76e11 */
    char element[16];
    double init_spin[3];
    double k1u;                /* [J] */
    double k1u_dir[3];
} asd_ucf_atom;
/* .ucf reader, geom::readGlobalGeom (src/geom_glob.cpp:190-295): "nms nauc", then per atom
 * "sl x y z [mx my mz] mu damping gamma element sx sy sz K1U dx dy dz" (mesh point present when
 * the k-mesh is set, mesh_points != 0), with the reference's checks on mu, gamma, the K1U axis
 * and per-species moments (src/unitcell.h:131-218).  atoms == NULL: counts only. */
int asd_read_ucf(const char* path, int mesh_points, uint32_t* nms, uint32_t* nauc, asd_ucf_atom* atoms,
                 uint32_t cap, char* err, size_t err_len);
/* .exch reader for the unitcell method, exch::get_exch_unitcell
 * (src/exch_determine_exchange_matrix.cpp:27-144): groups exchange_<s1>_<s2> with
 * Num_Interactions, units and UnitCell<i> / J<i>_<row> arrays.  Bonds come out in file order
 * per (s1, s2): species, cell offset rounded half away from zero (src/exch_unitcell.cpp:303-327),
 * J in joules, 3x3 row-major.  bond arrays NULL: *nbonds only.  Feeds asd_build_csr. */
int asd_read_exch(const char* path, uint32_t nms, uint32_t* nbonds, uint32_t* bond_s1, uint32_t* bond_s2,
                  int32_t* bond_vec, double* bond_J, uint32_t cap, char* err, size_t err_len);
/* csr_exch_mat.dat reader (src/exch.cpp:63-133): "N", "nnz", xadj[N+1], then per entry
 * "col xx yy zz" [T]; val9 is nnz x 9 with only the diagonal filled.  xadj NULL: *nnz only. */
int asd_read_csr_exch(const char* path, uint32_t nspins, uint32_t* nnz, uint32_t* xadj, uint32_t* adjncy,
                      double* val9, uint32_t cap, char* err, size_t err_len);
/* csr_exch_mat.dat writer in the layout src/exch_unitcell.cpp:36-63 writes (diagonal
 * components; 17 significant digits where the reference prints 6). */
int asd_write_csr_exch(const char* path, uint32_t nspins, const uint32_t* xadj, const uint32_t* adjncy,
                       const double* val9);

#ifdef __cplusplus
}
#endif
#endif /* ASD_H */
