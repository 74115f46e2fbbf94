// sort.cu — spatial ordering of the particles (a permutation, never a move).
//
// The deposit and the gather touch one cell of each of k grids per particle.
// When the particles a warp processes are scattered over the box, those
// touches land on as many cells as there are lanes: shared-memory bank
// conflicts in the gather and one shared atomic per (particle, grid) in the
// deposit.  Processing particles in the order of a space-filling curve makes
// neighbouring lanes, and the consecutive particles of one thread, fall into
// the same cells, so gathers broadcast and deposits merge before the atomic.
//
// The permutation is built by a counting sort over 32^3 world cells keyed by
// their Morton index: count (warp-merged global atomics), one-CTA exclusive
// scan, scatter.  The caller's arrays keep their order; kernels read
// particle perm[s] for slot s.  Order within a bin is whatever the atomics
// give; no result depends on it (integer mass sums are order-free and every
// particle's force is summed over grids in index order by one thread).
#include "mog_internal.h"

namespace mog {

namespace {

constexpr int kBinBits = 5;               // 32 cells per axis
constexpr int kBins = 1 << (3 * kBinBits);

__device__ __forceinline__ uint32_t spread3(uint32_t v) {
    // bit i of v -> bit 3i
    v &= 0x3ff;
    v = (v | (v << 16)) & 0x030000ff;
    v = (v | (v << 8)) & 0x0300f00f;
    v = (v | (v << 4)) & 0x030c30c3;
    v = (v | (v << 2)) & 0x09249249;
    return v;
}

__device__ __forceinline__ uint32_t bin_of(float4 P, float inv_cell) {
    const int m = (1 << kBinBits) - 1;
    const int x = min(max(__float2int_rd(P.x * inv_cell), 0), m);
    const int y = min(max(__float2int_rd(P.y * inv_cell), 0), m);
    const int z = min(max(__float2int_rd(P.z * inv_cell), 0), m);
    return spread3(x) | (spread3(y) << 1) | (spread3(z) << 2);
}

__global__ void __launch_bounds__(256) sort_count_kernel(const float4* __restrict__ pos,
                                                         int64_t n, float inv_cell,
                                                         unsigned* __restrict__ count) {
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = p < n;
    const uint32_t key = valid ? bin_of(pos[p], inv_cell) : 0xffffffffu;
    const unsigned m = __match_any_sync(kFull, key);
    if (valid && (threadIdx.x & 31) == __ffs(m) - 1) atomicAdd(count + key, (unsigned)__popc(m));
}

// Exclusive scan of kBins counts by one CTA of 1024 threads (32 bins each).
__global__ void __launch_bounds__(1024) sort_scan_kernel(const unsigned* __restrict__ count,
                                                         unsigned* __restrict__ cursor) {
    constexpr int kPer = kBins / 1024;
    __shared__ unsigned warp_tot[32];
    const int t = threadIdx.x;
    unsigned local[kPer];
    unsigned sum = 0;
#pragma unroll
    for (int i = 0; i < kPer; ++i) {
        local[i] = sum;
        sum += count[t * kPer + i];
    }
    // inclusive scan of per-thread sums
    unsigned incl = sum;
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned v = __shfl_up_sync(kFull, incl, o);
        if ((t & 31) >= o) incl += v;
    }
    if ((t & 31) == 31) warp_tot[t >> 5] = incl;
    __syncthreads();
    if (t < 32) {
        unsigned w = warp_tot[t];
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned v = __shfl_up_sync(kFull, w, o);
            if (t >= o) w += v;
        }
        warp_tot[t] = w;  // inclusive over warps
    }
    __syncthreads();
    const unsigned before = (incl - sum) + ((t >> 5) ? warp_tot[(t >> 5) - 1] : 0u);
#pragma unroll
    for (int i = 0; i < kPer; ++i) cursor[t * kPer + i] = before + local[i];
}

__global__ void __launch_bounds__(256) sort_scatter_kernel(const float4* __restrict__ pos,
                                                           int64_t n, float inv_cell,
                                                           unsigned* __restrict__ cursor,
                                                           int* __restrict__ perm,
                                                           unsigned* flags) {
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = p < n;
    const uint32_t key = valid ? bin_of(pos[p], inv_cell) : 0xffffffffu;
    const unsigned m = __match_any_sync(kFull, key);
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(m) - 1;
    unsigned base = 0;
    if (valid && lane == leader) base = atomicAdd(cursor + key, (unsigned)__popc(m));
    base = __shfl_sync(kFull, base, leader);
    if (valid) {
        const unsigned rank = __popc(m & ((1u << lane) - 1u));
        if (in_bounds(flags, (uint64_t)base + rank, (uint64_t)n)) perm[base + rank] = (int)p;
    }
}

__global__ void __launch_bounds__(256) gather_sorted_kernel(const float4* __restrict__ pos,
                                                            const int* __restrict__ perm,
                                                            int64_t n, float4* __restrict__ out) {
    const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s < n) out[s] = pos[__ldg(perm + s)];
}

}  // namespace

cudaError_t launch_gather_sorted(const float4* pos, const int* perm, int64_t n, float4* out,
                                 cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    gather_sorted_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(pos, perm, n, out);
    return cudaGetLastError();
}

size_t sort_scratch_bytes() { return 2 * (size_t)kBins * sizeof(unsigned); }

cudaError_t launch_sort(const float4* pos, int64_t n, float world, void* scratch, int* perm,
                        unsigned* flags, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    unsigned* count = static_cast<unsigned*>(scratch);
    unsigned* cursor = count + kBins;
    const float inv_cell = (float)(1 << kBinBits) / world;
    cudaError_t err = cudaMemsetAsync(count, 0, sizeof(unsigned) * kBins, s);
    if (err != cudaSuccess) return err;
    const unsigned blocks = (unsigned)((n + 255) / 256);
    sort_count_kernel<<<blocks, 256, 0, s>>>(pos, n, inv_cell, count);
    sort_scan_kernel<<<1, 1024, 0, s>>>(count, cursor);
    sort_scatter_kernel<<<blocks, 256, 0, s>>>(pos, n, inv_cell, cursor, perm, flags);
    return cudaGetLastError();
}

}  // namespace mog
