// sph_noalloc.cu — the cell sort (hash, stable counting sort, cell ranges)
// for callers that cannot allocate device memory.
//
// Some callers cannot call cudaMalloc: a host program whose device memory is
// owned by another allocator (an engine or framework that reserves the whole
// budget up front and forbids outside allocations), or a latency-critical
// loop where cudaMalloc's implicit device synchronisation is not acceptable.
// sph_sort_cells_noalloc serves them: the caller passes device inputs and
// outputs, and every scratch buffer lives in one file-scope __device__ array
// of fixed size (SPH_NOALLOC_MAX_PARTICLES particles, SPH_NOALLOC_MAX_CELLS
// cells, about 3.7 MB), which every GPU that loads this library holds until
// the process exits.
//
// Host code must not use g_noalloc_scratch's name as a device address: on the
// host it names a stand-in, and a kernel given it would fault or, where the
// GPU can reach host memory, silently touch the wrong memory.  The first call
// on each device therefore looks up the real device address with
// cudaGetSymbolAddress (with that device current) and caches it; make that
// first call before any stream capture begins.  The cached address lives as
// long as the process; cudaDeviceReset unloads the module that holds the array,
// after which the cached address is stale and this entry point must not be
// called on that device again.  All calls share the array and
// it keeps the last call's contents: the counters that must start at zero are
// cleared by every call, and calls that overlap on the GPU (two streams, or
// two host threads) race on it.
#include "../../include/sph/sph.h"
#include "sph_scan.cuh"

#include <cuda_runtime.h>
#include <algorithm>
#include <cstdio>
#include <mutex>

namespace {

using sph::kScanBlocks;
using sph::kScanThreads;
using sph::scan_phase1;
using sph::scan_phase2;
using sph::scan_phase3;

constexpr int kThreads = 256;

__device__ __forceinline__ uint32_t grid_stride_start() { return blockIdx.x * blockDim.x + threadIdx.x; }
__device__ __forceinline__ uint32_t grid_stride() { return gridDim.x * blockDim.x; }

// (uint)floor(x / cell) in FP32 round-to-nearest, clamped to the grid: the
// same cell the step's hash computes.
__device__ __forceinline__ uint32_t cell_coord(float x, float cs, uint32_t n)
{
    float f = floorf(__fdiv_rn(x, cs));
    if (!(f >= 0.0f)) return 0u;
    if (f >= (float)n) return n - 1u;
    return (uint32_t)f;
}

constexpr uint32_t kMaxP = SPH_NOALLOC_MAX_PARTICLES;
constexpr uint32_t kMaxC = SPH_NOALLOC_MAX_CELLS;

// word offsets inside the scratch array
constexpr size_t kOffCount = 0;                      // [kMaxC + 1] per-cell counts
constexpr size_t kOffCellOff = kOffCount + kMaxC + 1; // [kMaxC + 1] exclusive scan of counts
constexpr size_t kOffKey = kOffCellOff + kMaxC + 1;  // [kMaxP] key per particle
constexpr size_t kOffSlot = kOffKey + kMaxP;         // [kMaxP] arrival slot inside the cell
constexpr size_t kOffTmp = kOffSlot + kMaxP;         // [kMaxP] unstable cell order
constexpr size_t kOffBlocks = kOffTmp + kMaxP;       // [kScanBlocks] scan block totals
constexpr size_t kOffGrand = kOffBlocks + kScanBlocks;
constexpr size_t kWords = kOffGrand + 4;

__device__ __align__(256) uint32_t g_noalloc_scratch[kWords];

constexpr int kMaxDevices = 64;
uint32_t *g_dev_scratch[kMaxDevices] = {};
std::mutex g_setup_mutex;

// Device address of the scratch array on the current device (set-up on the
// first call per device).
uint32_t *scratch_for_current_device(int *err)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        *err = SPH_ERR_NO_DEVICE;
        return nullptr;
    }
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_dev_scratch[dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            fprintf(stderr, "sph_sort_cells_noalloc: cudaGetSymbolAddress failed: %s\n", cudaGetErrorString(e));
            *err = SPH_ERR_CUDA;
            return nullptr;
        }
        g_dev_scratch[dev] = (uint32_t *)p;
    }
    return g_dev_scratch[dev];
}

template <int DIM>
__global__ void __launch_bounds__(kThreads) na_hash(sph_config c, uint32_t n, const float *__restrict__ pos,
                                                   uint32_t *__restrict__ key, uint32_t *__restrict__ slot,
                                                   uint32_t *__restrict__ count)
{
    for (uint32_t i = grid_stride_start(); i < n; i += grid_stride()) {
        const uint32_t x = cell_coord(pos[(size_t)i * DIM], c.cell_size, c.ncell[0]);
        const uint32_t y = cell_coord(pos[(size_t)i * DIM + 1], c.cell_size, c.ncell[1]);
        const uint32_t z = DIM == 3 ? cell_coord(pos[(size_t)i * DIM + 2], c.cell_size, c.ncell[2]) : 0u;
        const uint32_t k = z * c.ncell[0] * c.ncell[1] + y * c.ncell[0] + x;
        key[i] = k;
        slot[i] = atomicAdd(count + k, 1u);
    }
}

__global__ void __launch_bounds__(kThreads) na_scatter(uint32_t n, const uint32_t *__restrict__ key,
                                                      const uint32_t *__restrict__ slot,
                                                      const uint32_t *__restrict__ off, uint32_t *__restrict__ tmp)
{
    for (uint32_t i = grid_stride_start(); i < n; i += grid_stride()) tmp[off[key[i]] + slot[i]] = i;
}

// stable order inside each cell: rank by particle index among the cell's members.
// A particle compares itself with every member of its cell, so the cost is
// quadratic in a cell's population; with at most SPH_NOALLOC_MAX_PARTICLES
// particles and cells of an SPH kernel length (tens of members) that stays
// small, but a caller that piles many particles into one cell pays for it.
__global__ void __launch_bounds__(kThreads) na_rank(uint32_t n, const uint32_t *__restrict__ key,
                                                   const uint32_t *__restrict__ off, const uint32_t *__restrict__ tmp,
                                                   uint32_t *__restrict__ key_out, uint32_t *__restrict__ index_out)
{
    for (uint32_t s = grid_stride_start(); s < n; s += grid_stride()) {
        const uint32_t i = tmp[s], k = key[i];
        const uint32_t b = off[k], e = off[k + 1];
        uint32_t r = 0;
        for (uint32_t t = b; t < e; ++t) r += tmp[t] < i;
        key_out[b + r] = k;
        index_out[b + r] = i;
    }
}

// cell_start / cell_end in the reference's format from the offsets
__global__ void __launch_bounds__(kThreads) na_ranges(const uint32_t *__restrict__ off, uint32_t nc,
                                                     uint32_t *__restrict__ start, uint32_t *__restrict__ end)
{
    for (uint32_t q = grid_stride_start(); q < nc; q += grid_stride()) {
        const uint32_t b = off[q], e = off[q + 1];
        start[q] = e > b ? b : 0xffffffffu;
        end[q] = e > b ? e : 0u;
    }
}

}  // namespace

extern "C" int sph_sort_cells_noalloc(const sph_config *cfg, uint32_t n, const float *pos_dev, uint32_t *key_dev,
                                      uint32_t *index_dev, uint32_t *cell_start_dev, uint32_t *cell_end_dev,
                                      void *stream)
{
    if (!cfg || (cfg->dim != 2 && cfg->dim != 3)) return SPH_ERR_INVALID;
    if (!(cfg->cell_size > 0.0f) || cfg->ncell[0] == 0 || cfg->ncell[1] == 0 || (cfg->dim == 3 && cfg->ncell[2] == 0))
        return SPH_ERR_INVALID;
    const uint64_t C = (uint64_t)cfg->ncell[0] * cfg->ncell[1] * (cfg->dim == 3 ? cfg->ncell[2] : 1u);
    if (n > kMaxP || C > kMaxC) {
        fprintf(stderr,
                "sph_sort_cells_noalloc: %u particles / %llu cells exceed the fixed maximum of %u particles / %u cells\n",
                n, (unsigned long long)C, kMaxP, kMaxC);
        return SPH_ERR_RANGE;
    }
    if (!cell_start_dev || !cell_end_dev || (n && (!pos_dev || !key_dev || !index_dev))) return SPH_ERR_INVALID;
    int err = SPH_OK;
    uint32_t *sc = scratch_for_current_device(&err);
    if (!sc) return err;
    cudaStream_t s = (cudaStream_t)stream;
    uint32_t *count = sc + kOffCount, *off = sc + kOffCellOff, *key = sc + kOffKey, *slot = sc + kOffSlot;
    uint32_t *tmp = sc + kOffTmp, *blocks = sc + kOffBlocks, *grand = sc + kOffGrand;
    const uint32_t nc = (uint32_t)C;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const uint32_t G = std::max(1u, std::min((n + kThreads - 1) / kThreads, (uint32_t)sms * 8u));
    const uint32_t GC = std::max(1u, std::min((nc + kThreads - 1) / kThreads, (uint32_t)sms * 8u));

    cudaMemsetAsync(count, 0, sizeof(uint32_t) * (nc + 1), s);   // counts start at zero every call
    if (cfg->dim == 3) na_hash<3><<<G, kThreads, 0, s>>>(*cfg, n, pos_dev, key, slot, count);
    else na_hash<2><<<G, kThreads, 0, s>>>(*cfg, n, pos_dev, key, slot, count);
    scan_phase1<uint32_t><<<kScanBlocks, kScanThreads, 0, s>>>(count, nullptr, nc, blocks);
    scan_phase2<uint32_t><<<1, kScanBlocks, 0, s>>>(blocks, grand);
    scan_phase3<uint32_t><<<kScanBlocks, kScanThreads, 0, s>>>(count, off, nullptr, nc, blocks, grand, 1, nullptr);
    na_scatter<<<G, kThreads, 0, s>>>(n, key, slot, off, tmp);
    na_rank<<<G, kThreads, 0, s>>>(n, key, off, tmp, key_dev, index_dev);
    na_ranges<<<GC, kThreads, 0, s>>>(off, nc, cell_start_dev, cell_end_dev);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        fprintf(stderr, "sph_sort_cells_noalloc: %s\n", cudaGetErrorString(e));
        return SPH_ERR_CUDA;
    }
    return SPH_OK;
}
