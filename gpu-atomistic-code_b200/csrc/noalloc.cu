// Sublattice magnetisation of spins already in device memory, with no device
// allocation at all: the partial sums live in a fixed file-scope device array.
//
// Who needs this: code that cannot call cudaMalloc/cudaFree at the point it
// wants a magnetisation - a host that hands all device memory to its own pool
// allocator and runs at its limit, or a time-critical loop that must not hit
// cudaFree's implicit device-wide synchronisation.  asd_magnetisation() on a
// handle allocates its scratch once at asd_create; this entry point needs
// neither a handle nor an allocation.
#include "../../include/asd.h"
#include <cuda_runtime.h>
#include <mutex>

namespace {

constexpr uint32_t NA_MAX_BLOCKS = ASD_NOALLOC_MAX_BLOCKS;
constexpr uint32_t NA_MAX_SUB = ASD_NOALLOC_MAX_SUBLATTICES;
constexpr uint32_t NA_BLOCK = 256;

// 4 doubles (sum x, sum y, sum z, count) per (block, sublattice): 2048*16*4*8 B = 1 MiB.
// Every GPU that loads the library holds this array until the process exits.
static __device__ __align__(256) double g_partials[NA_MAX_BLOCKS * NA_MAX_SUB * 4];

// Host-side address of g_partials on each device, looked up once per device.
std::mutex g_mu;
void* g_addr[128] = {nullptr};

__device__ __forceinline__ double na_block_sum(double v, double* sm) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) sm[w] = v;
    __syncthreads();
    double r = 0.0;
    if (w == 0) {
        r = l < (int)(blockDim.x >> 5) ? sm[l] : 0.0;
        for (int o = 16; o > 0; o >>= 1) r += __shfl_down_sync(0xffffffffu, r, o);
    }
    return r;
}

// Block b sums the spins of [b*chunk, (b+1)*chunk) per sublattice in one pass (register
// accumulators for NS >= nsub sublattices, each thread in a fixed order) and writes every slot
// (b, s) it owns, so nothing left from an earlier call is ever read.  Spins whose sublattice
// id is nsub or more are left out of every sum.
template <uint32_t NS>
__global__ void na_partial(const double* __restrict__ s3, uint32_t n, const uint32_t* __restrict__ sub,
                           uint32_t nsub, uint32_t chunk, double* __restrict__ part) {
    __shared__ double sm[32];
    const uint32_t b = blockIdx.x;
    const size_t beg = (size_t)b * chunk;
    const size_t end = beg + chunk < n ? beg + chunk : n;
    double acc[NS][4];
#pragma unroll
    for (uint32_t q = 0; q < NS; q++) acc[q][0] = acc[q][1] = acc[q][2] = acc[q][3] = 0.0;
    for (size_t i = beg + threadIdx.x; i < end; i += blockDim.x) {
        const uint32_t s = sub ? sub[i] : 0u;
        const double x = s3[3 * i], y = s3[3 * i + 1], z = s3[3 * i + 2];
#pragma unroll
        for (uint32_t q = 0; q < NS; q++)
            if (q == s) { acc[q][0] += x; acc[q][1] += y; acc[q][2] += z; acc[q][3] += 1.0; }
    }
#pragma unroll
    for (uint32_t q = 0; q < NS; q++) {
        if (q >= nsub) break;
        double t[4];
#pragma unroll
        for (int k = 0; k < 4; k++) t[k] = na_block_sum(acc[q][k], sm);
        if (threadIdx.x == 0) {
            double* o = part + ((size_t)b * nsub + q) * 4;
            o[0] = t[0]; o[1] = t[1]; o[2] = t[2]; o[3] = t[3];
        }
    }
}

// One thread per (sublattice, component): fixed-order sum over the blocks.
__global__ void na_final(uint32_t nblocks, uint32_t nsub, const double* __restrict__ part, double* __restrict__ out) {
    const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= nsub * 3) return;
    const uint32_t s = q / 3, c = q % 3;
    double acc = 0.0, cnt = 0.0;
    for (uint32_t b = 0; b < nblocks; b++) {
        acc += part[((size_t)b * nsub + s) * 4 + c];
        cnt += part[((size_t)b * nsub + s) * 4 + 3];
    }
    out[q] = cnt > 0.0 ? acc * (1.0 / cnt) : 0.0;
}

}  // namespace

extern "C" int asd_magnetisation_noalloc(const double* d_spins, uint32_t nspins, const uint32_t* d_sublattice,
                                         uint32_t nsub, double* d_out, void* stream) {
    if (!d_spins || !d_out || nspins == 0 || nspins > 0x7FFFFFFFu) return ASD_EINVAL;
    if (nsub == 0 || nsub > NA_MAX_SUB) return ASD_EINVAL;  // beyond the static scratch
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 128) return ASD_ECUDA;
    void* part = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_mu);
        if (!g_addr[dev]) {
            // first call on this device: look up the device address of the static array
            if (cudaGetSymbolAddress(&g_addr[dev], g_partials) != cudaSuccess) {
                g_addr[dev] = nullptr;
                return ASD_ECUDA;
            }
        }
        part = g_addr[dev];
    }
    uint32_t nblocks = (nspins + NA_BLOCK - 1) / NA_BLOCK;
    if (nblocks > NA_MAX_BLOCKS) nblocks = NA_MAX_BLOCKS;
    const uint32_t chunk = (nspins + nblocks - 1) / nblocks;
    nblocks = (nspins + chunk - 1) / chunk;
    cudaStream_t st = (cudaStream_t)stream;
    double* pp = (double*)part;
    if (nsub == 1) na_partial<1><<<nblocks, NA_BLOCK, 0, st>>>(d_spins, nspins, d_sublattice, nsub, chunk, pp);
    else if (nsub == 2) na_partial<2><<<nblocks, NA_BLOCK, 0, st>>>(d_spins, nspins, d_sublattice, nsub, chunk, pp);
    else if (nsub <= 4) na_partial<4><<<nblocks, NA_BLOCK, 0, st>>>(d_spins, nspins, d_sublattice, nsub, chunk, pp);
    else if (nsub <= 8) na_partial<8><<<nblocks, NA_BLOCK, 0, st>>>(d_spins, nspins, d_sublattice, nsub, chunk, pp);
    else na_partial<16><<<nblocks, NA_BLOCK, 0, st>>>(d_spins, nspins, d_sublattice, nsub, chunk, pp);
    na_final<<<1, 64, 0, st>>>(nblocks, nsub, (const double*)part, d_out);
    return cudaGetLastError() == cudaSuccess ? ASD_OK : ASD_ECUDA;
}
