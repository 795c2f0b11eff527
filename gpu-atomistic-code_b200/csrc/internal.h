// Host-side handle and the launch interface between api.cpp and the kernels.
#pragma once
#include "../../include/asd.h"
#include "common.cuh"
#include <cufft.h>
#include <string>
#include <utility>
#include <vector>

namespace asd {

// Device layouts of the exchange matrix.
//  SELL-32 (sliced ELLPACK, slice height = warp size) for CSR input: rows are
//  grouped in slices of 32; entry (slice s, k, lane) sits at slice_ptr[s] + 32k + lane,
//  so one warp reads 32 consecutive entries per k.  Padding entries point at the
//  row itself with zero tensor.
//  Float: diagonal form packs (col, xx, yy, zz) in one float4; full form packs
//  (col, m00, m01, m02), (m10, m11, m12, m20), (m21, m22) in float4+float4+float2.
//  Double: col[E] plus component-major values val[c][E].
struct SellDev {
    uint32_t nslices = 0, entries = 0;
    uint32_t* slice_ptr = nullptr;
    float4* a = nullptr;
    float4* b = nullptr;
    float2* c = nullptr;
    int32_t* col = nullptr;
    double* val = nullptr;
    // typed layout: entry word = col | id << colbits; table [ncomp][ntypes]
    uint32_t* typed = nullptr;
    uint32_t colbits = 0, ntypes = 0;
    float* tab_f = nullptr;
    double* tab_d = nullptr;
    // bulk staging in shared memory at the launch block size: stage 1 copies each block's typed
    // words, stage 2 also the neighbour spins its rows read (spin_block = block size the local
    // words were built for); stage_words / spin_slots size the buffers; err collects device
    // error bits
    uint32_t stage = 0, stage_words = 0;
    uint32_t* err = nullptr;
    // neighbour-spin staging: per block, spans [start, start+len) of the spin arrays land at
    // slot offset off in shared memory ([3][spin_slots] components); lwords are the typed words
    // with the column replaced by the slot (blocks without spans keep global columns)
    uint32_t* lwords = nullptr;
    // the same local words packed to 16 bits (slot | id << lbits) when the largest block's slots
    // and the tensor ids fit; blocks without spans then read their global words unstaged
    uint16_t* lwords16 = nullptr;
    uint32_t lbits = 0;
    uint32_t* span_ptr = nullptr;
    uint4* spans = nullptr;          // (start, len, off, 0) in elements
    uint32_t spin_slots = 0, spin_block = 0;
};
constexpr uint32_t MAG_CHUNK = 2048;  // spins per block of the magnetisation reduction
constexpr uint32_t SPIN_PAD = 8;     // zeroed elements after every gather-source spin array

// Row-aligned DIA, values component-major val[c][d*N+row], c = 3 (diag) or 9;
// typed layout: one id byte per (diagonal, row), table [ncomp][ntypes].
struct DiaDev {
    uint32_t ndiag = 0;
    int32_t* off = nullptr;
    float* valf = nullptr;
    double* vald = nullptr;
    uint8_t* dtype = nullptr;
    uint32_t ntypes = 0;
    float* tab_f = nullptr;
    double* tab_d = nullptr;
    // per warp tile (32 rows): the diagonals with a nonzero entry in the tile's rows,
    // tile_diag[tile_ptr[w] .. tile_ptr[w+1]) in ascending order
    uint32_t* tile_ptr = nullptr;
    uint32_t* tile_diag = nullptr;
};

// Reference-structured CSR / DIA for the FP64 plain form (separate component arrays).
struct PlainExch {
    uint32_t* xadj = nullptr;
    uint32_t* adjncy = nullptr;
    double* v[9] = {nullptr};
    uint32_t ndiag = 0;
    int32_t* off = nullptr;
};

// Long-range field buffers (zero-padded mesh, FP32 R2C/C2R or FP64 C2C plain).
struct LongRange {
    int mode = ASD_LR_NONE;
    uint32_t mesh[3] = {0, 0, 0};
    size_t P = 0, Pk = 0;          // padded real sites, half-spectrum points
    uint32_t ncomp = 6;            // 6 (symmetric) or 9 components of N_k
    int nk_real = 1;               // N_k purely real (even N_r)
    uint32_t* mesh_idx = nullptr;  // per spin linear mesh index
    float* w = nullptr;            // per spin weight (mu for dipole, 1 for FFT exchange)
    float* r = nullptr;            // [3][P] padded real input / output
    float2* k = nullptr;           // [3][Pk]
    float* nkr = nullptr;          // [ncomp][Pk] real N_k
    float2* nkc = nullptr;         // [ncomp][Pk] complex N_k
    cufftHandle r2c = 0, c2r = 0;
    // pruned transform (power-of-two last mesh axis): own real FFT along z for the rows of the
    // spins' bounding box box0..box1 (inclusive), then 2D C2C over the (x, y) planes; spectra
    // in the transposed layout [c][kz][x][y]; k1 stays zero outside the box rows
    int pruned = 0;
    uint32_t box0[3] = {0, 0, 0}, box1[3] = {0, 0, 0};
    float2* k1 = nullptr;
    float2* k2 = nullptr;
    cufftHandle c2c = 0;
    // plane path (every axis a power of two, x and y <= 256): the library's own three kernels
    // (z+y forward, x + N_k product + inverse x, inverse y+z); the spectrum yk is
    // [c][kz][ky tile][box x][8] and N_k is tiled to match ([kz][tile][comp][kx][8])
    int planes = 0;
    uint32_t nk_nkx = 0, nk_odd = 0;   // kx rows of the tiled N_k and its odd components (bits)
    float2* yk = nullptr;
    void* nkt = nullptr;
    float2* twt = nullptr;          // twiddle table of the plane kernels
    uint32_t* xq = nullptr;           // x-pass item counters: next item, finished blocks
    // FP64 plain: complex padded arrays [3][P] and full complex N_k [9][P]
    double2 *zr = nullptr, *zk = nullptr, *zh = nullptr, *znk = nullptr;
    cufftHandle z2z = 0;
};

// In-situ S(q,t) sampler state (lattice mesh, complex FP64 grid, k-point series).
struct SqSampler {
    bool on = false;
    uint32_t qaxis = 2, nk = 0, max_samples = 0, nsamples = 0;
    size_t P = 0;
    uint32_t* idx = nullptr;     // per-spin mesh index
    uint32_t* sub = nullptr;     // per-spin sublattice
    double* uo = nullptr;        // nsub x 3 signs
    uint32_t* kidx = nullptr;    // per-k mesh index
    double2* grid = nullptr;     // [P]
    double2* series = nullptr;   // [max_samples][nk]
    cufftHandle plan = 0;
};

// Two-temperature model state and parameters (device copy; Te, Tl advance in place).
struct TtmDev {
    double Te, Tl;
    double G, Cl, ge, dt, T0, ct, tau, P;
    uint64_t t0;                 // step at which the model started
    uint32_t np, bath_e;
    double scale[ASD_TTM_MAX_PULSES], delay[ASD_TTM_MAX_PULSES];
};

struct KernelTimer {
    std::string name;
    double total_ms = 0.0;
    uint64_t count = 0;
    double bytes = 0.0;
};

}  // namespace asd

struct asd_handle {
    asd_params p{};
    std::string err;
    int device = 0;
    cudaStream_t stream = nullptr;
    uint32_t n = 0, nrep = 0, nmat = 0, nsub = 1;
    uint32_t exch = ASD_EXCH_NONE, full = 0;
    uint32_t dexch = ASD_EXCH_NONE;      // device layout of the fused kernels (DIA input may run as SELL)
    bool dia_alt = false;                // a CSR matrix also held as typed DIA (few diagonals)
    uint64_t step = 0;
    uint64_t launches = 0;
    asd::StepConst sc{};
    std::vector<uint32_t> h_rep_off;
    std::vector<double> h_rep_T;
    std::vector<uint32_t> h_atom;      // empty -> i % nmat
    std::vector<uint32_t> h_sub_of_mat;
    // device: replica tables, atoms, mutable scalars
    uint32_t *d_rep_off = nullptr, *d_rep_stream = nullptr, *d_atom = nullptr;
    double *d_rep_sqrtT = nullptr, *d_dyn = nullptr;
    float *d_rep_sqrtT_f = nullptr, *d_dynf = nullptr;
    uint64_t* d_step = nullptr;
    // FP32 / FP64-fused state, SoA
    float *sf[3] = {nullptr}, *sl[3] = {nullptr}, *esf[3] = {nullptr}, *fnf[3] = {nullptr};
    float *kf[6][3] = {{nullptr}};
    float *detf[3] = {nullptr}, *stagf[3] = {nullptr};
    double *sd[3] = {nullptr}, *esd[3] = {nullptr}, *fnd[3] = {nullptr}, *kd[6][3] = {{nullptr}};
    float* nzf[3] = {nullptr};           // this step's thermal field sigma sqrt(T) xi (fused forms)
    double* nzd[3] = {nullptr};
    double *detd[3] = {nullptr}, *stagd[3] = {nullptr};
    asd::SellDev sell;
    asd::DiaDev dia;
    // FP64 plain (AoS [3i+c], reference-structured)
    double *p_s = nullptr, *p_es = nullptr, *p_fn = nullptr, *p_ch = nullptr, *p_hdemag = nullptr, *p_rand = nullptr,
           *p_det = nullptr, *p_hstg = nullptr, *p_hinit = nullptr, *p_k[6] = {nullptr};
    double *p_sigma = nullptr, *p_llgpf = nullptr, *p_lambda = nullptr, *p_k1u = nullptr, *p_k1udir = nullptr;
    asd::PlainExch pex;
    asd::LongRange lr;
    // reductions
    double* d_magpart = nullptr;
    size_t magpart_len = 0;
    double* d_mag = nullptr;
    uint32_t* d_magcnt = nullptr;        // block ticket of the one-launch magnetisation (rearmed to 0)
    double* d_inv_count = nullptr;
    uint32_t* d_sub_of_atom = nullptr;
    uint64_t graph_launches = 0;
    std::vector<uint32_t> h_slice_ptr;   // SELL slice offsets (host copy, for staging capacity)
    std::vector<uint32_t> h_words;       // typed SELL words (host copy, for the local words)
    uint32_t* d_err = nullptr;           // device error bits (staging wait timeouts)
    uint32_t* h_err = nullptr;           // page-locked host word the error bits are read into
    double* d_aos = nullptr;             // [3N] staging buffer of the spin / field transfers
    unsigned long long* d_check = nullptr; // [2] first non-finite component, first zero-length spin
    uint32_t* d_rep_of_tile = nullptr;   // replica of each 32-spin tile's first spin
    asd::TtmDev* d_ttm = nullptr;        // two-temperature model (null: off)
    uint32_t* d_q4ptr = nullptr;         // four-spin quartet offsets [N+1]
    uint4* d_q4jkl = nullptr;            // four-spin quartets (j, k, l, 0)
    std::string tune;                    // autotuner result, "B=.. stage=.. (ms ...)"
    bool lr_scattered = false;
    double nnz_per_row = 0.0;
    // site-field ramp value and time envelope (host copies; the plain form ramps from the host)
    double stag_rv = 1.0, pulse_amp = 0.0, pulse_t0 = 0.0, pulse_sigma = 1.0;
    bool has_site = false;
    // M(T) running statistics per (replica, sublattice): n, mean, M2, previous mean
    double* d_stats = nullptr;
    asd::SqSampler sq;
    // CUDA graph of a chunk of FP32 steps
    cudaGraphExec_t graph = nullptr;
    uint32_t graph_steps = 0;
    cudaGraphExec_t graph1 = nullptr;    // one step (single-step calls)
    cudaGraph_t graph1_src = nullptr;    // its captured graph (kept: its det node is updated in place)
    cudaGraphNode_t det_node = nullptr;  // the one-step graph's det_here_k, which also writes the applied field
    bool applied_pending = false;        // the applied field awaits the next one-step graph or a flush
    uint64_t graph1_launches = 0;
    int block = 256;
    // timing of the dominant kernel
    bool timing = false;
    void* flush_buf = nullptr;           // written before each timed stage launch (cold L2)
    size_t flush_bytes = 0;
    std::vector<asd::KernelTimer> ktab;  // per kernel (name) of the last asd_time_kernels
    cudaEvent_t kev[2] = {nullptr, nullptr};
};

namespace asd {
// Timed launches (asd_time_kernels): before the launch, an optional L2 flush and an event on the
// handle's stream; after it, the event pair's device time accumulated under `name` with the
// launch's algorithmic bytes.
// Step kernels launch with programmatic dependent launch unless kernels are timed one by one or
// ASD_FLAG_SERIAL_LAUNCH asks for strict order.
inline bool step_pdl(const asd_handle* h) { return !h->timing && !(h->p.flags & ASD_FLAG_SERIAL_LAUNCH); }

inline void timer_begin(asd_handle* h) {
    if (!h->timing) return;
    if (h->flush_buf) cudaMemsetAsync(h->flush_buf, 0, h->flush_bytes, h->stream);
    cudaEventRecord(h->kev[0], h->stream);
}
inline void timer_end(asd_handle* h, const std::string& name, double bytes) {
    if (!h->timing) return;
    cudaEventRecord(h->kev[1], h->stream);
    cudaEventSynchronize(h->kev[1]);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, h->kev[0], h->kev[1]);
    KernelTimer* kt = nullptr;
    for (auto& k : h->ktab)
        if (k.name == name) kt = &k;
    if (!kt) {
        h->ktab.push_back(KernelTimer{name, 0.0, 0, 0.0});
        kt = &h->ktab.back();
    }
    kt->bytes = (kt->bytes * kt->count + bytes) / (double)(kt->count + 1);
    kt->total_ms += ms;
    kt->count += 1;
}
}  // namespace asd

namespace asd {
// launchers implemented in the .cu files; all return cudaError_t of the launch
cudaError_t launch_plain_step(asd_handle* h, uint64_t t);
cudaError_t launch_fused_step(asd_handle* h, uint32_t rel, bool in_capture);
cudaError_t launch_step_advance(asd_handle* h, uint32_t nsteps);
cudaError_t launch_det_here(asd_handle* h);
// The one-step graph's det_here_k node with the applied field h->p.applied (no launch).
cudaError_t update_det_applied(asd_handle* h);
const void* det_here_kernel();
cudaError_t launch_lr_eval_f32(asd_handle* h);
cudaError_t launch_lr_scatter(asd_handle* h);
cudaError_t launch_lr_planes(asd_handle* h);
cudaError_t build_plane_twiddles(asd_handle* h);
bool plane_path_fits(const LongRange& L, bool cplx);
size_t plane_spectrum_elems(const LongRange& L);
cudaError_t build_nk_tiles(asd_handle* h, const double2* z, uint32_t ncomp, bool cplx);
cudaError_t launch_lr_eval_plain(asd_handle* h, const double* s, double* out, bool overwrite_with_demag);
cudaError_t launch_field_only(asd_handle* h, double* d_out);
cudaError_t launch_plain_field(asd_handle* h, double* d_out);
cudaError_t launch_plain_ramp(asd_handle* h, double rv);
cudaError_t launch_set_scalar(asd_handle* h, double* dst, double v);
cudaError_t launch_set_vec3(asd_handle* h, double* dst, float* dstf, const double v[3]);
cudaError_t launch_set_scalar_f(asd_handle* h, float* dst, float v);
cudaError_t launch_mag_push(asd_handle* h);
// one two-temperature-model step for step t (device counter + rel when step_base is set, else t)
cudaError_t launch_ttm_step(asd_handle* h, const uint64_t* step_base, uint64_t t);
cudaError_t time_first_stage(asd_handle* h, int warm, int reps, float* ms);
cudaError_t launch_sq_sample(asd_handle* h);
cudaError_t launch_sq_spectrum(asd_handle* h, int window, double alpha, double beta, uint32_t pixelwidth,
                               double sample_dt, double flo, double fhi, double* d_raw, double* d_smooth,
                               uint32_t* d_peaks);
// hout: the device address of a page-locked host buffer the means are also written to (the
// kernel stores them there itself, so no copy follows), or nullptr.
cudaError_t launch_magnetisation(asd_handle* h, double* hout = nullptr);
cudaError_t launch_thermal_normals(uint64_t seed, uint32_t stream, uint64_t step, uint32_t n, double* d_out,
                                   cudaStream_t st);
cudaError_t launch_thermal_normals_f(uint64_t seed, uint32_t stream, uint64_t step, uint32_t n, float* d_out,
                                     cudaStream_t st);
cudaError_t launch_convert_spins_in(asd_handle* h, const double* d_aos);
// Raise a kernel's dynamic shared-memory limit on the current device to at least `bytes`,
// calling cudaFuncSetAttribute only when this (device, kernel) has not been raised that far.
cudaError_t raise_smem_limit(const void* kernel, size_t bytes);
// Blocks of a persistent kernel: as many as are resident on the device at once (cached per
// kernel, block size, shared memory and device), at most `work` (and at least 1).
cudaError_t resident_grid(const void* kernel, uint32_t block, size_t smem, uint32_t work, uint32_t* grid);

// Launch of a step kernel (one that starts with pdl_enter): with `pdl` its blocks may become
// resident while the previous kernel of the stream finishes (programmatic dependent launch);
// `cluster` > 1 groups the blocks into thread-block clusters along x.
template <typename... KArgs, typename... Args>
cudaError_t launch_step_kernel(void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st,
                               uint32_t cluster, bool pdl, Args&&... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[2];
    unsigned n = 0;
    if (cluster > 1) {
        attr[n].id = cudaLaunchAttributeClusterDimension;
        attr[n].val.clusterDim.x = cluster;
        attr[n].val.clusterDim.y = 1;
        attr[n].val.clusterDim.z = 1;
        n++;
    }
    if (pdl) {
        attr[n].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        attr[n].val.programmaticStreamSerializationAllowed = 1;
        n++;
    }
    cfg.attrs = attr;
    cfg.numAttrs = n;
    return cudaLaunchKernelEx(&cfg, kern, std::forward<Args>(args)...);
}
cudaError_t launch_check_spins(asd_handle* h, const double* d_aos, unsigned long long* d_check);
cudaError_t launch_convert_out(asd_handle* h, int what, double* d_aos);
cudaError_t build_nk_f32(asd_handle* h, const double* d_nr);
cudaError_t permute_nk_pruned(asd_handle* h);
cudaError_t build_nk_plain(asd_handle* h, const double* d_nr);
}  // namespace asd
