// sph_scan.cuh — device-wide exclusive prefix sums whose length is read from
// device memory, so a step that changes its particle count on the device
// never needs the host to learn the count (the reference syncs on two
// thrust::reduce calls per step, SPH-3D-2/sph_system.cu:1639,1836).
//
// Two launches: per-block chunk totals, then per-block rescans, each block
// summing the block totals before its own (scan_phase23).  The grid is fixed
// at launch (kScanBlocks); each block takes a contiguous chunk of
// ceil(len/kScanBlocks) elements, so the traffic is two reads and one write
// of the input.  (The three-launch form, with one block scanning the totals
// in between, remains for the no-allocation sort.)
#pragma once
#include <cstdint>

namespace sph {

constexpr int kScanBlocks = 1024;   // fixed grid of the scan phases (== threads of phase 2)
constexpr int kScanThreads = 256;

template <typename T> struct Add {
    __device__ __forceinline__ T operator()(T a, T b) const { return a + b; }
};
__device__ __forceinline__ uint2 operator+(uint2 a, uint2 b) { return make_uint2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ uint2 operator-(uint2 a, uint2 b) { return make_uint2(a.x - b.x, a.y - b.y); }

template <typename T> __device__ __forceinline__ T zero_of();
template <> __device__ __forceinline__ uint32_t zero_of<uint32_t>() { return 0u; }
template <> __device__ __forceinline__ uint2 zero_of<uint2>() { return make_uint2(0u, 0u); }

template <typename T> __device__ __forceinline__ T shfl_up(T v, int d)
{
    return __shfl_up_sync(0xffffffffu, v, d);
}
template <> __device__ __forceinline__ uint2 shfl_up<uint2>(uint2 v, int d)
{
    return make_uint2(__shfl_up_sync(0xffffffffu, v.x, d), __shfl_up_sync(0xffffffffu, v.y, d));
}

// Inclusive scan across the block; returns the thread's inclusive value and
// writes the block total to *total.
template <typename T>
__device__ __forceinline__ T block_inclusive_scan(T v, T *warp_tot, T *total)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int d = 1; d < 32; d <<= 1) {
        T o = shfl_up(v, d);
        if (lane >= d) v = v + o;
    }
    if (lane == 31) warp_tot[warp] = v;
    __syncthreads();
    if (warp == 0) {
        const int nw = blockDim.x >> 5;
        T w = lane < nw ? warp_tot[lane] : zero_of<T>();
        for (int d = 1; d < 32; d <<= 1) {
            T o = shfl_up(w, d);
            if (lane >= d) w = w + o;
        }
        if (lane < nw) warp_tot[lane] = w;
    }
    __syncthreads();
    if (warp > 0) v = v + warp_tot[warp - 1];
    *total = warp_tot[(blockDim.x >> 5) - 1];
    __syncthreads();
    return v;
}

__device__ __forceinline__ void chunk_of(uint32_t len, uint32_t &b, uint32_t &e)
{
    uint32_t chunk = (len + gridDim.x - 1) / gridDim.x;
    b = min(len, blockIdx.x * chunk);
    e = min(len, b + chunk);
}

// The phases as device bodies over the launch's blocks (gridDim.x of them,
// at most kScanBlocks; blockDim.x at most kScanThreads), shared by the three
// launches below and by the persistent step kernel, which runs them between
// grid-wide barriers.
template <typename T>
__device__ __forceinline__ void scan_phase1_body(const T *in, uint32_t len, T *block_tot)
{
    __shared__ T wt[kScanThreads / 32];
    uint32_t b, e;
    chunk_of(len, b, e);
    T acc = zero_of<T>();
    for (uint32_t i = b + threadIdx.x; i < e; i += blockDim.x) acc = acc + in[i];
    T tot;
    block_inclusive_scan(acc, wt, &tot);
    if (threadIdx.x == 0) block_tot[blockIdx.x] = tot;
}

// skip_if_zero (optional): a count of the nonzero inputs; at 0 the scan is
// all zeros, which scan_phase23 writes without reading the input.
template <typename T>
__global__ void __launch_bounds__(kScanThreads) scan_phase1(const T *__restrict__ in, const uint32_t *len_ptr,
                                                           uint32_t len_const, T *__restrict__ block_tot,
                                                           const uint32_t *skip_if_zero = nullptr)
{
    if (skip_if_zero && *skip_if_zero == 0u) return;
    scan_phase1_body<T>(in, len_ptr ? *len_ptr : len_const, block_tot);
}

// Exclusive scan of nb block totals by one block of any size (each thread
// takes a contiguous run); grand total to *grand (if non-null).
template <typename T>
__device__ __forceinline__ void scan_phase2_body(T *block_tot, uint32_t nb, T *grand)
{
    __shared__ T wt[kScanThreads / 32];
    const uint32_t per = (nb + blockDim.x - 1) / blockDim.x;
    const uint32_t b = min(nb, threadIdx.x * per), e = min(nb, b + per);
    T acc = zero_of<T>();
    for (uint32_t i = b; i < e; ++i) acc = acc + block_tot[i];
    T tot;
    T run = block_inclusive_scan(acc, wt, &tot) - acc;
    for (uint32_t i = b; i < e; ++i) {
        const T v = block_tot[i];
        block_tot[i] = run;
        run = run + v;
    }
    if (threadIdx.x == 0 && grand) *grand = tot;
}

// One block of kScanBlocks threads: exclusive scan of the block totals;
// grand total to *grand (if non-null).
template <typename T>
__global__ void __launch_bounds__(kScanBlocks) scan_phase2(T *block_tot, T *grand)
{
    __shared__ T wt[kScanBlocks / 32];
    T v = block_tot[threadIdx.x];
    T tot;
    T inc = block_inclusive_scan(v, wt, &tot);
    block_tot[threadIdx.x] = inc - v;
    if (threadIdx.x == 0 && grand) *grand = tot;
}

// Exclusive scan of each chunk plus its block offset.  If out_total_at_len,
// out[len] receives the grand total (used for cell offsets, out[C]).
// If list != nullptr (T = uint32_t flags only), list[out[i]] = i for in[i]==1.
template <typename T>
__device__ __forceinline__ void scan_phase3_body(const T *in, T *out, uint32_t len, const T *block_off,
                                                 const T *grand, int out_total_at_len, uint32_t *list)
{
    __shared__ T wt[kScanThreads / 32];
    uint32_t b, e;
    chunk_of(len, b, e);
    T carry = block_off[blockIdx.x];
    for (uint32_t base = b; base < e; base += blockDim.x) {
        uint32_t i = base + threadIdx.x;
        T v = i < e ? in[i] : zero_of<T>();
        T tot;
        T inc = block_inclusive_scan(v, wt, &tot);
        if (i < e) {
            T ex = carry + inc - v;
            out[i] = ex;
            if constexpr (sizeof(T) == 4) {
                if (list && v) list[ex] = i;
            }
        }
        carry = carry + tot;
    }
    if (out_total_at_len && blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) out[len] = *grand;
}

// Phases 2 and 3 in one: every block sums the nb block totals itself (its
// exclusive offset and the grand total), then rescans its chunk.  For a grid
// whose blocks meet at barriers (the persistent step), this saves the barrier
// after a separate phase 2.  Block 0 writes the grand total to *grand.
template <typename T>
__device__ __forceinline__ void scan_phase23_body(const T *in, T *out, uint32_t len, const T *block_tot,
                                                  T *grand, int out_total_at_len, uint32_t *list)
{
    __shared__ T wt[kScanThreads / 32];
    __shared__ T s_off, s_all;
    T pre = zero_of<T>(), all = zero_of<T>();
    for (uint32_t i = threadIdx.x; i < gridDim.x; i += blockDim.x) {
        const T v = block_tot[i];
        all = all + v;
        if (i < blockIdx.x) pre = pre + v;
    }
    T tot;
    block_inclusive_scan(pre, wt, &tot);
    if (threadIdx.x == 0) s_off = tot;
    block_inclusive_scan(all, wt, &tot);
    if (threadIdx.x == 0) s_all = tot;
    __syncthreads();
    const T off = s_off, total = s_all;
    uint32_t b, e;
    chunk_of(len, b, e);
    T carry = off;
    for (uint32_t base = b; base < e; base += blockDim.x) {
        uint32_t i = base + threadIdx.x;
        T v = i < e ? in[i] : zero_of<T>();
        T t2;
        T inc = block_inclusive_scan(v, wt, &t2);
        if (i < e) {
            T ex = carry + inc - v;
            out[i] = ex;
            if constexpr (sizeof(T) == 4) {
                if (list && v) list[ex] = i;
            }
        }
        carry = carry + t2;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0 && grand) *grand = total;
    if (out_total_at_len && blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) out[len] = total;
}

// The whole scan in one phase, for inputs of at most PER elements per
// thread of one block (len <= PER * blockDim.x): every block sums all the
// elements before its chunk itself (PER independent loads per thread, in
// flight together), so no barrier separates the block totals from the
// rescan.  The last block (whose chunk ends at len) writes the grand total to
// *grand (if non-null) and, if out_total_at_len, to out[len].
template <typename T, int PER>
__device__ __forceinline__ void scan_onepass_body(const T *in, T *out, uint32_t len, T *grand, int out_total_at_len)
{
    __shared__ T wt[kScanThreads / 32];
    uint32_t b, e;
    chunk_of(len, b, e);
    T part[PER];
#pragma unroll
    for (int u = 0; u < PER; ++u) {
        const uint32_t i = threadIdx.x + (uint32_t)u * blockDim.x;
        part[u] = i < b ? in[i] : zero_of<T>();
    }
    T pre = zero_of<T>();
#pragma unroll
    for (int u = 0; u < PER; ++u) pre = pre + part[u];
    T carry;
    block_inclusive_scan(pre, wt, &carry);
    for (uint32_t base = b; base < e; base += blockDim.x) {
        uint32_t i = base + threadIdx.x;
        T v = i < e ? in[i] : zero_of<T>();
        T t2;
        T inc = block_inclusive_scan(v, wt, &t2);
        if (i < e) out[i] = carry + inc - v;
        carry = carry + t2;
    }
    if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) {
        if (grand) *grand = carry;
        if (out_total_at_len) out[len] = carry;
    }
}

// Phases 2 and 3 as one launch (after scan_phase1 over the same grid).
template <typename T>
__global__ void __launch_bounds__(kScanThreads) scan_phase23(const T *__restrict__ in, T *__restrict__ out,
                                                            const uint32_t *len_ptr, uint32_t len_const,
                                                            const T *__restrict__ block_tot, T *grand,
                                                            int out_total_at_len, uint32_t *list,
                                                            const uint32_t *skip_if_zero = nullptr)
{
    const uint32_t len = len_ptr ? *len_ptr : len_const;
    if (skip_if_zero && *skip_if_zero == 0u) {   // every input is zero: so is every output
        for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < len; i += gridDim.x * blockDim.x)
            out[i] = zero_of<T>();
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            if (grand) *grand = zero_of<T>();
            if (out_total_at_len) out[len] = zero_of<T>();
        }
        return;
    }
    scan_phase23_body<T>(in, out, len, block_tot, grand, out_total_at_len, list);
}

template <typename T>
__global__ void __launch_bounds__(kScanThreads) scan_phase3(const T *__restrict__ in, T *__restrict__ out,
                                                           const uint32_t *len_ptr, uint32_t len_const,
                                                           const T *__restrict__ block_off,
                                                           const T *grand, int out_total_at_len,
                                                           uint32_t *list)
{
    scan_phase3_body<T>(in, out, len_ptr ? *len_ptr : len_const, block_off, grand, out_total_at_len, list);
}

}  // namespace sph
