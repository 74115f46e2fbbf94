// deposit.cu — K1: rotate + offset + NGP mass deposit into all k grids.
//
// Replaces mass.glsl:27-55 (one thread per particle looping over k grids,
// one global uint32 atomic per (particle, grid)) and the per-step host
// upload of zeros in clear_mass (main.py:558-562).
//
// Design: a CTA owns `gpc` grids (or one slab of one grid when g^3 cells do
// not fit shared memory) and a chunk of particles.  It accumulates a
// private fixed-point histogram in shared memory with 32/64-bit shared
// atomics, then flushes the non-zero cells to the global grid with one
// global atomic each.  Integer addition is associative, so the result is
// bit-identical whatever the schedule.  When all particles of a warp carry
// the same quantised mass (the equal-mass case of every benchmark
// configuration) lanes that hit the same cell are merged with
// __match_any_sync and a single add of popc * q, which removes the
// shared-atomic serialisation in dense regions.
#include <algorithm>

#include "mog_internal.h"

namespace mog {

namespace {

template <typename Acc>
struct Quant;
template <>
struct Quant<unsigned long long> {
    static __device__ __forceinline__ unsigned long long q(float m, float scale, unsigned& bad) {
        return quantize_u64(m, scale, bad);
    }
};
template <>
struct Quant<unsigned> {
    static __device__ __forceinline__ unsigned q(float m, float, unsigned& bad) {
        return quantize_u32(m, bad);
    }
};

constexpr uint32_t kNoCell = 0xffffffffu;

// Shared-memory histogram deposit.  blockIdx.x: particle chunk; blockIdx.y:
// group of `gpc` grids; blockIdx.z: slab of (1 << slab_lg) consecutive
// cells of each grid (slab_lg == 3*lg means the whole grid).
template <typename Acc, int IDX, bool AGG>
__global__ void __launch_bounds__(1024) deposit_smem_kernel(const float4* __restrict__ pos,
                                                            int64_t n, int64_t chunk,
                                                            Ensemble e, int gpc, int slab_lg,
                                                            Acc* __restrict__ mass) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int lg = e.lg;
    const uint32_t slab_cells = 1u << slab_lg;
    const uint32_t slab_lo = (uint32_t)blockIdx.z << slab_lg;
    const int g0 = blockIdx.y * gpc;
    const int ng = min(gpc, e.k - g0);

    // shared layout: [transforms: gpc * 16 floats][histogram: gpc * slab_cells]
    float* xf = reinterpret_cast<float*>(smem_raw);
    Acc* hist = reinterpret_cast<Acc*>(smem_raw + (size_t)gpc * 16 * sizeof(float));

    for (int i = threadIdx.x; i < ng * 16; i += blockDim.x) {
        const int j = i >> 4, w = i & 15;
        float v;
        if (IDX == 0) {
            v = (w < 12) ? reinterpret_cast<const float*>(e.fast + g0 + j)[w] : 0.f;
        } else {
            v = (w < 12) ? e.rot12[(g0 + j) * 12 + w] : e.off4[(g0 + j) * 4 + (w - 12)];
        }
        xf[i] = v;
    }
    for (uint32_t i = threadIdx.x; i < (uint32_t)ng * slab_cells; i += blockDim.x) hist[i] = 0;
    __syncthreads();

    const IndexParams ip = e.index_params();
    const int64_t lo = (int64_t)blockIdx.x * chunk;
    const int64_t hi = min(n, lo + chunk);
    const int lane = threadIdx.x & 31;
    unsigned bad = 0;
    double qsum = 0.0;

    for (int64_t base = lo; base < hi; base += blockDim.x) {
        const int64_t p = base + threadIdx.x;
        const bool valid = p < hi;
        float4 P = valid ? __ldg(pos + p) : make_float4(0.f, 0.f, 0.f, 0.f);
        Acc q = valid ? Quant<Acc>::q(P.w, e.scale, bad) : Acc(0);
        qsum += (double)q;
        const float cx = __fsub_rn(P.x, ip.half_l);
        const float cy = __fsub_rn(P.y, ip.half_l);
        const float cz = __fsub_rn(P.z, ip.half_l);

        bool uni = false;
        Acc q0 = q;
        if (AGG) {
            const unsigned vmask = __ballot_sync(kFull, valid);
            q0 = __shfl_sync(kFull, q, vmask ? __ffs(vmask) - 1 : 0);
            uni = __all_sync(kFull, !valid || q == q0);
        }
#pragma unroll 2
        for (int j = 0; j < ng; ++j) {
            uint32_t cell;
            if (IDX == 0) {
                const float4* r = reinterpret_cast<const float4*>(xf + j * 16);
                cell = cell_fast(r[0], r[1], r[2], cx, cy, cz, lg);
            } else {
                cell = cell_exact(xf + j * 16, xf + j * 16 + 12, cx, cy, cz, ip);
            }
            uint32_t local = cell - slab_lo;
            const bool hit = valid && local < slab_cells;
            Acc* h = hist + (size_t)j * slab_cells;
            if (AGG && uni) {
                const uint32_t key = hit ? local : kNoCell;
                const unsigned m = __match_any_sync(kFull, key);
                if (hit && lane == __ffs(m) - 1) atomicAdd(h + local, q0 * (Acc)__popc(m));
            } else if (hit) {
                atomicAdd(h + local, q);
            }
        }
    }

    // Overflow bookkeeping: every grid receives every particle's q, so the
    // total of one grid bounds every cell; the first grid group counts it.
    if (blockIdx.y == 0 && blockIdx.z == 0 && sizeof(Acc) == 8) {
        for (int o = 16; o > 0; o >>= 1) qsum += __shfl_xor_sync(kFull, qsum, o);
        if (lane == 0 && qsum != 0.0) atomicAdd(e.mass_total, qsum);
    }
    if (bad) raise_flags(e.flags, bad);
    __syncthreads();

    const size_t gcells = (size_t)1 << (3 * lg);
    for (uint32_t i = threadIdx.x; i < (uint32_t)ng * slab_cells; i += blockDim.x) {
        const Acc v = hist[i];
        if (v) {
            const uint32_t j = i >> slab_lg, c = i & (slab_cells - 1);
            atomicAdd(mass + (size_t)(g0 + j) * gcells + slab_lo + c, v);
        }
    }
}

// Direct global-atomic deposit (any g): one thread per particle, all grids.
template <typename Acc, int IDX>
__global__ void __launch_bounds__(256) deposit_global_kernel(const float4* __restrict__ pos,
                                                             int64_t n, Ensemble e,
                                                             Acc* __restrict__ mass) {
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = p < n;
    const IndexParams ip = e.index_params();
    unsigned bad = 0;
    const float4 P = valid ? __ldg(pos + p) : make_float4(0.f, 0.f, 0.f, 0.f);
    const Acc q = valid ? Quant<Acc>::q(P.w, e.scale, bad) : Acc(0);
    const float cx = __fsub_rn(P.x, ip.half_l);
    const float cy = __fsub_rn(P.y, ip.half_l);
    const float cz = __fsub_rn(P.z, ip.half_l);
    const size_t gcells = (size_t)1 << (3 * e.lg);
    for (int i = 0; valid && i < e.k; ++i) {
        uint32_t cell;
        if (IDX == 0) {
            const FastXf f = e.fast[i];
            cell = cell_fast(f.row[0], f.row[1], f.row[2], cx, cy, cz, e.lg);
        } else {
            cell = cell_exact(e.rot12 + 12 * i, e.off4 + 4 * i, cx, cy, cz, ip);
        }
        if (q) atomicAdd(mass + (size_t)i * gcells + cell, q);
    }
    if (sizeof(Acc) == 8) {
        double qs = (double)q;  // blocks are whole warps, so every lane is present
        for (int o = 16; o > 0; o >>= 1) qs += __shfl_xor_sync(kFull, qs, o);
        if ((threadIdx.x & 31) == 0 && qs != 0.0) atomicAdd(e.mass_total, qs);
    }
    if (bad) raise_flags(e.flags, bad);
}

}  // namespace

template <typename Acc, int IDX>
static cudaError_t deposit_typed(const Ensemble& e, const float4* pos, int64_t n, Acc* mass,
                                 const DepositShape& sh, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    const int cells_lg = 3 * e.lg;
    const size_t grid_bytes = sizeof(Acc) << cells_lg;
    const size_t budget = 100 * 1024;  // two CTAs per SM
    if (sh.grids_per_cta < 0) {
        const int threads = 256;
        const int64_t blocks = (n + threads - 1) / threads;
        deposit_global_kernel<Acc, IDX><<<(unsigned)blocks, threads, 0, s>>>(pos, n, e, mass);
        return cudaGetLastError();
    }
    int gpc = sh.grids_per_cta;
    int slab_lg = cells_lg;
    if (gpc == 0) {
        if (grid_bytes <= budget) {
            gpc = (int)std::min<size_t>((size_t)e.k, budget / grid_bytes);
        } else {
            gpc = 1;
            while (((size_t)sizeof(Acc) << slab_lg) > 128 * 1024) --slab_lg;
        }
    } else if (grid_bytes * gpc > 200 * 1024) {
        gpc = 1;
        while (((size_t)sizeof(Acc) << slab_lg) > 128 * 1024) --slab_lg;
    }
    gpc = std::max(1, std::min(gpc, e.k));
    const size_t smem = (size_t)gpc * 16 * sizeof(float) + ((size_t)gpc * sizeof(Acc) << slab_lg);
    auto launch = [&](auto kern) -> cudaError_t {
        cudaError_t err = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               (int)smem);
        if (err != cudaSuccess) return err;
        const int groups = (e.k + gpc - 1) / gpc;
        const int slabs = 1 << (cells_lg - slab_lg);
        int chunks = sh.chunks;
        if (chunks <= 0) {
            const int per_sm = smem > 110 * 1024 ? 1 : 2;
            const int64_t target = (int64_t)num_sms() * per_sm * 4;
            int64_t c = (target + (int64_t)groups * slabs - 1) / ((int64_t)groups * slabs);
            const int64_t max_c = (n + 2047) / 2048;
            chunks = (int)std::max<int64_t>(1, std::min<int64_t>(c, max_c));
        }
        const int64_t chunk = (n + chunks - 1) / chunks;
        dim3 grid(chunks, groups, slabs);
        kern<<<grid, sh.threads, smem, s>>>(pos, n, chunk, e, gpc, slab_lg, mass);
        return cudaGetLastError();
    };
    if (sh.aggregate) return launch(deposit_smem_kernel<Acc, IDX, true>);
    return launch(deposit_smem_kernel<Acc, IDX, false>);
}

cudaError_t launch_deposit(const Ensemble& e, const float4* pos, int64_t n, void* mass,
                           const DepositShape& shape, cudaStream_t s) {
    if (e.mass_mode == 0) {
        auto* m = static_cast<unsigned long long*>(mass);
        return e.index_mode == 0 ? deposit_typed<unsigned long long, 0>(e, pos, n, m, shape, s)
                                 : deposit_typed<unsigned long long, 1>(e, pos, n, m, shape, s);
    }
    auto* m = static_cast<unsigned*>(mass);
    return e.index_mode == 0 ? deposit_typed<unsigned, 0>(e, pos, n, m, shape, s)
                             : deposit_typed<unsigned, 1>(e, pos, n, m, shape, s);
}

}  // namespace mog
