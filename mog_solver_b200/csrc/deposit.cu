// deposit.cu — K1: rotate + offset + NGP mass deposit into all k grids.
//
// Replaces mass.glsl:27-55 (one thread per particle looping over k grids,
// one global uint32 atomic per (particle, grid)) and the per-step host
// upload of zeros in clear_mass (main.py:558-562).
//
// Design: a CTA owns `gpc` grids (or one slab of one grid when g^3 cells do
// not fit shared memory) and a chunk of particles.  It accumulates a
// private fixed-point histogram in shared memory with 32-bit shared
// atomics, then flushes the non-zero cells to the global grid with one
// global atomic each.  Integer addition is associative, so the result is
// bit-identical whatever the schedule.
#include <algorithm>

#include "../../include/mog.h"
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

// Shared histograms are 32-bit words: 64-bit shared atomics are several
// times slower on this part, and 32-bit adds to one address from many
// lanes are merged by the hardware.  MODE 0 (u32 x1000 grids): one word
// per cell, wrapping mod 2^32 like the reference's uint atomicAdd.
// MODE 1 (u64 fixed point): a low and a high word per cell; q is split into
// halves, the low add returns the previous value so its carry is counted
// exactly once, and the cell's 64-bit value is (hi << 32) + lo.  Equal
// power-of-two masses have an all-zero low half and cost one add.
template <int MODE>
struct SmemHist;
template <>
struct SmemHist<0> {
    using Acc = unsigned;
    static constexpr int kWords = 1;
    static __device__ __forceinline__ void add(unsigned* lo, unsigned*, uint32_t c, Acc q) {
        atomicAdd(lo + c, q);
    }
    static __device__ __forceinline__ Acc read(const unsigned* lo, const unsigned*, uint32_t c) {
        return lo[c];
    }
};
template <>
struct SmemHist<1> {
    using Acc = unsigned long long;
    static constexpr int kWords = 2;
    static __device__ __forceinline__ void add(unsigned* lo, unsigned* hi, uint32_t c, Acc q) {
        const unsigned ql = (unsigned)q;
        unsigned qh = (unsigned)(q >> 32);
        if (ql) {
            const unsigned old = atomicAdd(lo + c, ql);
            qh += (old > ~ql) ? 1u : 0u;  // old + ql wrapped past 2^32
        }
        if (qh) atomicAdd(hi + c, qh);
    }
    static __device__ __forceinline__ Acc read(const unsigned* lo, const unsigned* hi, uint32_t c) {
        return ((Acc)hi[c] << 32) | lo[c];
    }
};

// Sharded deposits (SHARD kernels): `mass` points at the step's
// ShardTargets, and v is added to cell `cell` (index in the k g^3 layout)
// of the owning rank's accumulation buffer with a system-scope atomic
// (several GPUs add to one cell over NVLink).
template <typename Acc>
__device__ __forceinline__ void shard_add(const Ensemble& e, Acc* mass, uint64_t cell, Acc v) {
    const ShardTargets* t = reinterpret_cast<const ShardTargets*>(mass);
    const int grid = (int)(cell >> (3 * e.lg));
    Acc* base = static_cast<Acc*>(t->base[shard_owner(grid, e.k, t->world)]);
    atomicAdd_system(base + cell, v);
}

// A sharded deposit's CTA makes its remote adds visible system-wide before
// it exits (the step's signal follows the kernel): the barrier orders every
// thread's adds before thread 0's system-scope fence.  Every thread of the
// CTA must reach it.
template <bool SHARD>
__device__ __forceinline__ void shard_release() {
    if constexpr (SHARD) {
        __syncthreads();
        if (threadIdx.x == 0) __threadfence_system();
    }
}

// Shared-memory histogram deposit.  blockIdx.x: particle chunk; blockIdx.y:
// group of `gpc` grids; blockIdx.z: slab of (1 << slab_lg) consecutive
// cells of each grid (slab_lg == 3*lg means the whole grid).  Each thread
// carries PPT particles through the grid loop, so the grid's cell-index
// rows are loaded once per PPT particles and the PPT index computations
// and shared adds overlap.  With AGG (used when the particles come in
// spatial order) the lanes of a warp merge runs of equal cells with a
// ballot of run heads, so a run costs one shared add.
template <int MODE, int IDX, int PPT, bool AGG, bool SHARD = false>
__global__ void __launch_bounds__(1024) deposit_smem_kernel(const float4* __restrict__ pos,
                                                            const int* __restrict__ perm,
                                                            int64_t n, int64_t chunk,
                                                            Ensemble e, int gpc, int slab_lg,
                                                            typename SmemHist<MODE>::Acc* __restrict__ mass) {
    using H = SmemHist<MODE>;
    using Acc = typename H::Acc;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int lg = e.lg;
    const uint32_t slab_cells = 1u << slab_lg;
    const uint32_t slab_lo = (uint32_t)blockIdx.z << slab_lg;
    const int g0 = blockIdx.y * gpc;
    const int ng = min(gpc, e.k - g0);
    const uint32_t words = (uint32_t)ng * slab_cells;

    // shared layout: [transforms: gpc * 16 floats][lo words][hi words]
    float* xf = reinterpret_cast<float*>(smem_raw);
    unsigned* lo_w = reinterpret_cast<unsigned*>(smem_raw + (size_t)gpc * 16 * sizeof(float));
    unsigned* hi_w = lo_w + (size_t)gpc * slab_cells;

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
    for (uint32_t i = threadIdx.x; i < words; i += blockDim.x) {
        lo_w[i] = 0u;
        if (H::kWords == 2) hi_w[i] = 0u;
    }
    __syncthreads();

    const IndexParams ip = e.index_params();
    const int64_t lo = (int64_t)blockIdx.x * chunk;
    const int64_t hi = min(n, lo + chunk);
    const int T = blockDim.x;
    unsigned bad = 0;
    double qsum = 0.0;

    const int lane = threadIdx.x & 31;
    for (int64_t base = lo; base < hi; base += (int64_t)T * PPT) {
        float cx[PPT], cy[PPT], cz[PPT];
        Acc q[PPT];
        bool valid[PPT];
#pragma unroll
        for (int u = 0; u < PPT; ++u) {
            // the 32 lanes of a warp take 32 consecutive slots, so with a
            // spatial ordering they are neighbours and share cells
            const int64_t slot = base + (int64_t)u * T + threadIdx.x;
            valid[u] = slot < hi;
            float4 P = make_float4(0.f, 0.f, 0.f, 0.f);
            if (valid[u]) {
                const int64_t src = perm ? (int64_t)__ldg(perm + slot) : slot;
                if (in_bounds(e.flags, (uint64_t)src, (uint64_t)n)) P = __ldg(pos + src);
            }
            unsigned b = 0;
            if (MODE == 1)
                q[u] = valid[u] ? quantize_u64(P.w, e.scale, b) : 0ull;
            else
                q[u] = valid[u] ? quantize_u32(P.w, b) : 0u;
            bad |= b;
            qsum += (double)q[u];
            cx[u] = __fsub_rn(P.x, ip.half_l);
            cy[u] = __fsub_rn(P.y, ip.half_l);
            cz[u] = __fsub_rn(P.z, ip.half_l);
        }
        // equal masses across the warp (checked once per batch) let a run
        // of lanes on one cell add q * (run length) without a scan
        bool uni[PPT];
        if (AGG) {
#pragma unroll
            for (int u = 0; u < PPT; ++u) {
                const unsigned vm = __ballot_sync(kFull, valid[u]);
                const Acc q0 = __shfl_sync(kFull, q[u], vm ? __ffs(vm) - 1 : 0);
                uni[u] = __all_sync(kFull, !valid[u] || q[u] == q0);
            }
        }
        for (int j = 0; j < ng; ++j) {
            unsigned* lw = lo_w + (size_t)j * slab_cells;
            unsigned* hw = hi_w + (size_t)j * slab_cells;
            const float4* r = reinterpret_cast<const float4*>(xf + j * 16);
            float4 r0, r1, r2;
            if (IDX == 0) {
                r0 = r[0];
                r1 = r[1];
                r2 = r[2];
            }
#pragma unroll
            for (int u = 0; u < PPT; ++u) {
                uint32_t local;
                if (IDX == 0)
                    local = cell_fast(r0, r1, r2, cx[u], cy[u], cz[u], lg) - slab_lo;
                else
                    local = cell_exact(xf + j * 16, xf + j * 16 + 12, cx[u], cy[u], cz[u], ip) - slab_lo;
                const uint32_t key = (valid[u] && local < slab_cells) ? local : 0xffffffffu;
                if (!AGG) {
                    if (key != 0xffffffffu) H::add(lw, hw, key, q[u]);
                    continue;
                }
                // warp-segmented merge of runs of equal keys (sorted input)
                const uint32_t prev = __shfl_up_sync(kFull, key, 1);
                const unsigned heads = __ballot_sync(kFull, lane == 0 || key != prev);
                const int start = 31 - __clz(heads & (0xffffffffu >> (31 - lane)));
                const bool tail = lane == 31 || ((heads >> (lane + 1)) & 1u);
                Acc v = q[u];
                if (uni[u]) {
                    v = q[u] * (Acc)(lane - start + 1);
                } else {
#pragma unroll
                    for (int d = 1; d < 32; d <<= 1) {
                        const Acc o = __shfl_up_sync(kFull, v, d);
                        if (lane - d >= start) v += o;
                    }
                }
                if (tail && key != 0xffffffffu) H::add(lw, hw, key, v);
            }
        }
    }

    // Overflow bookkeeping: every grid receives every particle's q, so the
    // total of one grid bounds every cell; the first grid group counts it.
    if (MODE == 1 && blockIdx.y == 0 && blockIdx.z == 0) {
        for (int o = 16; o > 0; o >>= 1) qsum += __shfl_xor_sync(kFull, qsum, o);
        if ((threadIdx.x & 31) == 0 && qsum != 0.0) atomicAdd(e.mass_total, qsum);
    }
    if (bad) raise_flags(e.flags, bad);
    __syncthreads();

    const size_t gcells = (size_t)1 << (3 * lg);
    for (uint32_t i = threadIdx.x; i < words; i += blockDim.x) {
        const Acc v = H::read(lo_w, hi_w, i);
        if (v) {
            const uint32_t j = i >> slab_lg, c = i & (slab_cells - 1);
            const size_t cell = (size_t)(g0 + j) * gcells + slab_lo + c;
            if (in_bounds(e.flags, cell, (uint64_t)e.cells())) {
                if constexpr (SHARD)
                    shard_add(e, mass, cell, v);
                else
                    atomicAdd(mass + cell, v);
            }
        }
    }
    shard_release<SHARD>();
}

// Specialised deposit for the common case: g <= 16 known at compile time,
// FAST cell indices, whole grids in shared memory.  Cell offsets use
// compile-time masks and shifts, shared adds are red.shared.add.u32 on
// 32-bit shared addresses, full batches run without bounds checks, and
// when every lane of a warp has a zero low word (equal power-of-two
// fixed-point masses) the 64-bit add is a single add of the high word.
__device__ __forceinline__ void red_shared(uint32_t addr, unsigned v) {
    asm volatile("red.shared.add.u32 [%0], %1;" ::"r"(addr), "r"(v) : "memory");
}
__device__ __forceinline__ unsigned atom_shared(uint32_t addr, unsigned v) {
    unsigned old;
    asm volatile("atom.shared.add.u32 %0, [%1], %2;" : "=r"(old) : "r"(addr), "r"(v) : "memory");
    return old;
}

// Shared-histogram word of a grid word w: the low 5 bits (the bank) XORed
// with bits 5-9.  Cells of a compact region (a thin disk seen in a rotated
// grid covers few distinct x) then spread over all 32 banks instead of the
// few that their low x and y bits name.  An involution (bits 5 and up are
// left alone), so the flush maps a word back to its cell with the same
// function.  hist_swizzle_bytes is the same map on byte offsets (4 w).
__device__ __forceinline__ uint32_t hist_swizzle(uint32_t w) {
    return w ^ ((w >> 5) & 31u);
}
__device__ __forceinline__ uint32_t hist_swizzle_bytes(uint32_t b) {
    return b ^ ((b >> 5) & 124u);
}

// A grid's FAST index rows as the deposit keeps them in shared memory:
// p0 = (r0.x, r1.x, r0.y, r1.y), p1 = (r0.z, r1.z, r0.w, r1.w), p2 = r2, so
// that tx and ty come from paired FMAs (fma.rn.f32x2: two IEEE FMAs, each
// rounded as the scalar one, in cell_fast's order).
struct DepositRows {
    float4 p0, p1, p2;
};
__device__ __forceinline__ DepositRows deposit_rows(const FastXf& f) {
    const float4 r0 = f.row[0], r1 = f.row[1];
    return {make_float4(r0.x, r1.x, r0.y, r1.y), make_float4(r0.z, r1.z, r0.w, r1.w), f.row[2]};
}

// 4 * (x | y << LG | z << 2 LG) of cell_fast's cell; cc[a] = the centred
// coordinate a, duplicated into a pair.
template <int LG>
__device__ __forceinline__ uint32_t cell_byte_offset(const DepositRows& r, const float2 (&cc)[3]) {
    constexpr uint32_t M = (1u << LG) - 1u;
    constexpr float kMagic = 12582912.0f;  // 1.5 * 2^23, as floor_mod_pow2
    const float2 txy =
        __ffma2_rn(make_float2(r.p1.x, r.p1.y), cc[2],
                   __ffma2_rn(make_float2(r.p0.z, r.p0.w), cc[1],
                              __ffma2_rn(make_float2(r.p0.x, r.p0.y), cc[0], make_float2(r.p1.z, r.p1.w))));
    const float tz =
        __fmaf_rn(r.p2.z, cc[2].x, __fmaf_rn(r.p2.y, cc[1].x, __fmaf_rn(r.p2.x, cc[0].x, r.p2.w)));
    const float2 bxy = __fadd2_rd(txy, make_float2(kMagic, kMagic));
    const uint32_t bx = __float_as_uint(bxy.x), by = __float_as_uint(bxy.y);
    const uint32_t bz = __float_as_uint(__fadd_rd(tz, kMagic));
    return ((bx & M) << 2) | ((by & M) << (LG + 2)) | ((bz & M) << (2 * LG + 2));
}

//
// SPLIT (u64 mode, for grids whose two words per cell do not fit shared
// memory, g = 32): only the high words live in shared memory; a non-zero
// low half goes straight to the global 64-bit cell with one global atomic
// (equal power-of-two masses have none).
//
// One tile: every thread of the CTA deposits particles [lo, hi) into grids
// [g0, g0 + ng) through the shared histogram at smem_raw (gpc * 3 float4
// rows, then the words).  count_total: add the tile's q to e.mass_total
// (done by the tiles of the first grid group, which see every particle
// once).  Returns after the flush, without a closing barrier.
// COUNT (u64, uniform masses): one word per cell counts the particles whose
// fixed-point mass equals the tile's first particle's, q_ref; the flush adds
// count * q_ref.  A particle with another mass (only when the masses are not
// all equal) goes straight to its global cell with one 64-bit atomic.
template <int LG, int MODE, int PPT, bool SPLIT, bool SHARD, bool COUNT = false>
__device__ __forceinline__ void deposit_fast_tile(const float4* __restrict__ pos, int64_t lo,
                                                  int64_t hi, const Ensemble& e, int gpc, int g0,
                                                  int ng, bool count_total,
                                                  typename SmemHist<MODE>::Acc* __restrict__ mass,
                                                  unsigned char* smem_raw) {
    using H = SmemHist<MODE>;
    using Acc = typename H::Acc;
    static_assert(!SPLIT || MODE == 1, "the split histogram is for u64 grids");
    static_assert(!COUNT || (MODE == 1 && !SPLIT && !SHARD), "the count histogram is for u64 grids");
    constexpr bool ONE = SPLIT || COUNT;  // one shared word per cell
    constexpr int G3 = 1 << (3 * LG);
    static_assert(sizeof(DepositRows) == 48, "DepositRows layout");
    const uint32_t words = (uint32_t)ng * G3;
    DepositRows* rows = reinterpret_cast<DepositRows*>(smem_raw);              // gpc rows
    unsigned* lo_w = reinterpret_cast<unsigned*>(smem_raw + (size_t)gpc * 48);
    unsigned* hi_w = ONE ? lo_w : lo_w + (size_t)gpc * G3;
    const uint32_t lo_base = (uint32_t)__cvta_generic_to_shared(lo_w);
    const uint32_t hi_base = (uint32_t)__cvta_generic_to_shared(hi_w);

    for (int i = threadIdx.x; i < ng; i += blockDim.x) rows[i] = deposit_rows(e.fast[g0 + i]);
    for (uint32_t i = threadIdx.x; i < words; i += blockDim.x) {
        lo_w[i] = 0u;
        if (H::kWords == 2 && !ONE) hi_w[i] = 0u;
    }
    __syncthreads();

    Acc q_ref = 0;
    if (COUNT && lo < hi) {
        unsigned b = 0;
        q_ref = (Acc)quantize_u64(__ldg(pos + lo).w, e.scale, b);
    }
    const unsigned rl = (unsigned)q_ref, rh = (unsigned)((unsigned long long)q_ref >> 32);
    const float half_l = e.world * 0.5f;
    const int T = blockDim.x;
    unsigned bad = 0;
    double qsum = 0.0;
    for (int64_t base = lo; base < hi; base += (int64_t)T * PPT) {
        const bool full = base + (int64_t)T * PPT <= hi;  // block-uniform
        float2 cc[PPT][3];
        unsigned ql[PPT], qh[PPT];
        bool live[PPT];
#pragma unroll
        for (int u = 0; u < PPT; ++u) {
            const int64_t slot = base + (int64_t)u * T + threadIdx.x;
            const bool valid = full || slot < hi;
            live[u] = valid;
            const float4 P = valid ? __ldg(pos + slot) : make_float4(0.f, 0.f, 0.f, 0.f);
            unsigned b = 0;
            Acc q;
            if (MODE == 1)
                q = valid ? quantize_u64(P.w, e.scale, b) : 0ull;
            else
                q = valid ? quantize_u32(P.w, b) : 0u;
            bad |= b;
            qsum += (double)q;
            ql[u] = (unsigned)q;
            qh[u] = MODE == 1 ? (unsigned)((unsigned long long)q >> 32) : 0u;
            const float cx = __fsub_rn(P.x, half_l), cy = __fsub_rn(P.y, half_l),
                        cz = __fsub_rn(P.z, half_l);
            cc[u][0] = make_float2(cx, cx);
            cc[u][1] = make_float2(cy, cy);
            cc[u][2] = make_float2(cz, cz);
        }
        if constexpr (COUNT) {
            // one vote per batch: does every particle of the warp have q_ref?
            unsigned odd = 0;
#pragma unroll
            for (int u = 0; u < PPT; ++u) odd |= (live[u] && (ql[u] != rl || qh[u] != rh)) ? 1u : 0u;
            if (__all_sync(kFull, odd == 0u)) {
                // the whole warp counts: one add of 1 per particle and grid
                // (full batches need no per-particle test)
                for (int j = 0; j < ng; ++j) {
                    const DepositRows r = rows[j];
                    const uint32_t gbyte = (uint32_t)j * (G3 * 4u);
                    const uint32_t base_j = hi_base + gbyte;
#pragma unroll
                    for (int u = 0; u < PPT; ++u) {
                        const uint32_t off = cell_byte_offset<LG>(r, cc[u]);
                        if (!in_bounds(e.flags, (gbyte + off) >> 2, words)) continue;
                        const uint32_t addr = LG >= 4 ? base_j + hist_swizzle_bytes(off)
                                                      : hi_base + hist_swizzle_bytes(gbyte + off);
                        if (full || live[u]) red_shared(addr, 1u);
                    }
                }
                continue;
            }
            for (int j = 0; j < ng; ++j) {
                const DepositRows r = rows[j];
                const uint32_t gbyte = (uint32_t)j * (G3 * 4u);
#pragma unroll
                for (int u = 0; u < PPT; ++u) {
                    const uint32_t off = gbyte + cell_byte_offset<LG>(r, cc[u]);
                    if (!in_bounds(e.flags, off >> 2, words)) continue;
                    if (!live[u]) continue;
                    if (ql[u] == rl && qh[u] == rh)
                        red_shared(hi_base + hist_swizzle_bytes(off), 1u);
                    else if (ql[u] | qh[u])
                        atomicAdd(mass + (size_t)g0 * G3 + (off >> 2), ((Acc)qh[u] << 32) | (Acc)ql[u]);
                }
            }
            continue;
        }
        // one vote per batch: can the low words be skipped for the whole warp?
        bool hi_only = false;
        if (MODE == 1) {
            unsigned any_lo = 0;
#pragma unroll
            for (int u = 0; u < PPT; ++u) any_lo |= ql[u];
            hi_only = __all_sync(kFull, any_lo == 0u);
        }
        // the common case (equal power-of-two masses): one add of the high
        // word per particle and grid, in a loop of its own (in the split
        // layout as well: there are no low halves to send to global memory)
        if (MODE == 1 && hi_only) {
            for (int j = 0; j < ng; ++j) {
                const DepositRows r = rows[j];
                const uint32_t gbyte = (uint32_t)j * (G3 * 4u);
                const uint32_t base_j = hi_base + gbyte;
#pragma unroll
                for (int u = 0; u < PPT; ++u) {
                    const uint32_t off = cell_byte_offset<LG>(r, cc[u]);
                    if (!in_bounds(e.flags, (gbyte + off) >> 2, words)) continue;
                    // for g >= 16 the grid's byte offset (bit 14 and up) lies
                    // above the bits the swizzle reads and writes
                    const uint32_t addr = LG >= 4 ? base_j + hist_swizzle_bytes(off)
                                                  : hi_base + hist_swizzle_bytes(gbyte + off);
                    if (qh[u]) red_shared(addr, qh[u]);
                }
            }
            continue;
        }
        for (int j = 0; j < ng; ++j) {
            const DepositRows r = rows[j];
            const uint32_t gbyte = (uint32_t)j * (G3 * 4u);
#pragma unroll
            for (int u = 0; u < PPT; ++u) {
                const uint32_t off = gbyte + cell_byte_offset<LG>(r, cc[u]);
                if (!in_bounds(e.flags, off >> 2, words)) continue;
                const uint32_t soff = hist_swizzle_bytes(off);  // the shared word's bytes
                if (MODE == 0) {
                    if (ql[u]) red_shared(lo_base + soff, ql[u]);   // zero for padding lanes
                } else if (SPLIT) {
                    if (ql[u]) {
                        if constexpr (SHARD)
                            shard_add(e, mass, (uint64_t)g0 * G3 + (off >> 2), (Acc)ql[u]);
                        else
                            atomicAdd(mass + (size_t)g0 * G3 + (off >> 2), (Acc)ql[u]);
                    }
                    if (qh[u]) red_shared(hi_base + soff, qh[u]);
                } else if (hi_only) {
                    if (qh[u]) red_shared(hi_base + soff, qh[u]);
                } else {
                    unsigned h = qh[u];
                    if (ql[u]) {
                        const unsigned old = atom_shared(lo_base + soff, ql[u]);
                        h += (old > ~ql[u]) ? 1u : 0u;
                    }
                    if (h) red_shared(hi_base + soff, h);
                }
            }
        }
    }
    if (MODE == 1 && count_total) {
        for (int o = 16; o > 0; o >>= 1) qsum += __shfl_xor_sync(kFull, qsum, o);
        if ((threadIdx.x & 31) == 0 && qsum != 0.0) atomicAdd(e.mass_total, qsum);
    }
    if (bad) raise_flags(e.flags, bad);
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < words; i += blockDim.x) {
        const Acc v = COUNT ? (Acc)hi_w[i] * q_ref : (SPLIT ? (Acc)hi_w[i] << 32 : H::read(lo_w, hi_w, i));
        const uint32_t w = hist_swizzle(i);  // the grid word this shared word holds
        if (v && in_bounds(e.flags, (size_t)g0 * G3 + w, (uint64_t)e.cells())) {
            if constexpr (SHARD)
                shard_add(e, mass, (uint64_t)g0 * G3 + w, v);
            else
                atomicAdd(mass + (size_t)g0 * G3 + w, v);
        }
    }
}

template <int LG, int MODE, int PPT, bool SPLIT = false, bool SHARD = false, bool COUNT = false>
__global__ void __launch_bounds__(1024) deposit_fast_kernel(const float4* __restrict__ pos,
                                                            int64_t n, int64_t chunk, Ensemble e,
                                                            int gpc,
                                                            typename SmemHist<MODE>::Acc* __restrict__ mass) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int g0 = blockIdx.y * gpc;
    const int64_t lo = (int64_t)blockIdx.x * chunk;
    deposit_fast_tile<LG, MODE, PPT, SPLIT, SHARD, COUNT>(pos, lo, min(n, lo + chunk), e, gpc, g0,
                                                   min(gpc, e.k - g0), blockIdx.y == 0, mass,
                                                   smem_raw);
    shard_release<SHARD>();
}

// Batched ensemble, one persistent launch for every simulation of a batch:
// each CTA pops tiles (simulation, grid group, particle chunk) from the
// host-built list with an atomic counter until it runs out, and deposits
// each through the same tile body as deposit_fast_kernel.  The histogram
// layout follows the tile's own grid count and grid size; at g = 32 in u64
// mode it is the split (high-word) histogram, as in the single launch;
// LAYOUT 1: the split histogram at g = 8 and 16 as well; LAYOUT 2: the count
// histogram (uniform masses) at every grid size.
template <int MODE, int LAYOUT>
__global__ void __launch_bounds__(1024, 1) deposit_queue_kernel(const BatchSim* __restrict__ sims,
                                                               const DepositTile* __restrict__ tiles,
                                                               int ntiles, unsigned* __restrict__ counter) {
    using Acc = typename SmemHist<MODE>::Acc;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ int s_tile;
    for (;;) {
        if (threadIdx.x == 0) s_tile = (int)atomicAdd(counter, 1u);
        __syncthreads();
        const int t = s_tile;
        if (t >= ntiles) return;  // block-uniform
        const DepositTile tile = tiles[t];
        const BatchSim& S = sims[tile.sim];
        const Ensemble e = S.e;
        const float4* pos = S.pos;
        Acc* mass = static_cast<Acc*>(S.mass);
        const bool first = tile.g0 == 0;
        constexpr bool CNT = MODE == 1 && LAYOUT == 2;
        constexpr bool SPL = MODE == 1 && LAYOUT == 1;
        if (e.lg == 3)
            deposit_fast_tile<3, MODE, 4, SPL, false, CNT>(pos, tile.lo, tile.hi, e, tile.ng, tile.g0,
                                                           tile.ng, first, mass, smem_raw);
        else if (e.lg == 4)
            deposit_fast_tile<4, MODE, 4, SPL, false, CNT>(pos, tile.lo, tile.hi, e, tile.ng, tile.g0,
                                                           tile.ng, first, mass, smem_raw);
        else
            deposit_fast_tile<5, MODE, 4, MODE == 1 && !CNT, false, CNT>(pos, tile.lo, tile.hi, e,
                                                                        tile.ng, tile.g0, tile.ng,
                                                                        first, mass, smem_raw);
        __syncthreads();  // the next tile reuses the histogram and s_tile
    }
}

// Direct global-atomic deposit (any g): one thread per particle, all grids.
template <typename Acc, int IDX, bool SHARD = false>
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
        if (q && in_bounds(e.flags, (size_t)i * gcells + cell, (uint64_t)e.cells())) {
            if constexpr (SHARD)
                shard_add(e, mass, (uint64_t)i * gcells + cell, q);
            else
                atomicAdd(mass + (size_t)i * gcells + cell, q);
        }
    }
    shard_release<SHARD>();
    if (sizeof(Acc) == 8) {
        double qs = (double)q;  // blocks are whole warps, so every lane is present
        for (int o = 16; o > 0; o >>= 1) qs += __shfl_xor_sync(kFull, qs, o);
        if ((threadIdx.x & 31) == 0 && qs != 0.0) atomicAdd(e.mass_total, qs);
    }
    if (bad) raise_flags(e.flags, bad);
}

}  // namespace

// Particle chunks per grid group.  Every chunk costs one histogram flush
// (gpc * g^3 global atomics), so chunks stay few, but the CTAs (groups x
// chunks, `per_sm` resident per SM) should fill whole waves: one wave for
// up to 4 groups (each SM flushes once), 2 for up to 16, 3 for up to 64, 13
// beyond (measured on k = 16 / 32 / 240, g = 16, and k = 240, g = 32: k = 32
// in 4 groups takes 49 us in one wave against 53 in two; in 8 groups, 60 us
// in two against 62 in one; k = 240 in 20 groups 264 us in three against
// 269 in five and 273 in two; k = 240 at g = 32, one grid a group, 706 us in
// 13 waves against 748 in five and 721 to 740 in 10 to 26).  At least 2048
// particles per chunk.
static int auto_chunks(int64_t n, int64_t groups, int per_sm) {
    const int64_t waves = groups <= 4 ? 1 : (groups <= 16 ? 2 : (groups <= 64 ? 3 : 13));
    const int64_t c = waves * num_sms() * per_sm / std::max<int64_t>(groups, 1);
    const int64_t max_c = (n + 2047) / 2048;
    return (int)std::max<int64_t>(1, std::min<int64_t>(c, max_c));
}

template <int MODE, int IDX, bool SHARD>
static cudaError_t deposit_typed(const Ensemble& e, const float4* pos, const int* perm, int64_t n,
                                 bool ordered, void* mass_v, const DepositShape& sh,
                                 cudaStream_t s) {
    using H = SmemHist<MODE>;
    using Acc = typename H::Acc;
    Acc* mass = static_cast<Acc*>(mass_v);
    if (n <= 0) return cudaSuccess;
    const int cells_lg = 3 * e.lg;
    const size_t word_bytes = 4 * H::kWords;
    const size_t grid_bytes = word_bytes << cells_lg;
    const size_t budget = 200 * 1024;  // one CTA of up to 1024 threads per SM
    if (sh.grids_per_cta < 0) {
        const int threads = 256;
        const int64_t blocks = (n + threads - 1) / threads;
        deposit_global_kernel<Acc, IDX, SHARD><<<(unsigned)blocks, threads, 0, s>>>(pos, n, e, mass);
        return cudaGetLastError();
    }
    int gpc = sh.grids_per_cta;
    int slab_lg = cells_lg;
    if (gpc == 0) {
        // as many grids as fit, lowered to a divisor of k when one is at
        // least half that, so every grid group carries the same work
        const int most = (int)std::max<size_t>(1, std::min<size_t>((size_t)e.k, budget / grid_bytes));
        gpc = most;
        for (int d = most; d * 2 >= most && d >= 1; --d)
            if (e.k % d == 0) {
                gpc = d;
                break;
            }
    }
    if (grid_bytes * gpc > budget) {
        gpc = 1;
        while ((word_bytes << slab_lg) > 128 * 1024) --slab_lg;
    }
    gpc = std::max(1, std::min(gpc, e.k));
    const size_t smem = (size_t)gpc * 16 * sizeof(float) + ((size_t)gpc * word_bytes << slab_lg);
    // the sharded deposit is built for 4 particles per thread only
    const int ppt = SHARD ? 4 : (sh.ppt == 1 || sh.ppt == 2 || sh.ppt == 4 ? sh.ppt : 4);
    const bool agg = sh.aggregate < 0 ? ordered : sh.aggregate != 0;
    // The split histogram (u64, high words only, 4 bytes a cell; low halves
    // go to the global cells, and equal power-of-two masses have none).  At
    // g = 32 it fits one grid per CTA where the two-word one needs two
    // slabs (the default); at g = 8 and 16 (tuning deposit_split = 1) it
    // fits twice the grids per CTA.
    // The count histogram (u64, tuning deposit_split = 2, for uniform masses):
    // one word per cell at g = 8, 16 and 32 counting the particles of the
    // tile's first mass, whatever that mass is.
    const bool count = !SHARD && MODE == 1 && sh.split == 2 && (e.g == 8 || e.g == 16 || e.g == 32);
    const bool split32 = !count && MODE == 1 && e.g == 32 && sh.grids_per_cta <= 1 && sh.split >= 0;
    const bool split_small = !count && !SHARD && MODE == 1 && (e.g == 8 || e.g == 16) && sh.split == 1;
    const bool split = split32 || split_small || count;
    if (split && IDX == 0 && !agg && !perm && sh.fast != 0) {
        const int fit = (int)std::max<size_t>(1, budget / ((size_t)4 << cells_lg));
        if (split32 || (count && e.g == 32 && sh.grids_per_cta <= 1)) {
            gpc = 1;
        } else if (sh.grids_per_cta > 0) {
            gpc = std::min(sh.grids_per_cta, fit);
        } else {
            const int most = std::min(e.k, fit);
            gpc = most;
            for (int d = most; d * 2 >= most && d >= 1; --d)
                if (e.k % d == 0) {
                    gpc = d;
                    break;
                }
        }
        slab_lg = cells_lg;
    }
    if (IDX == 0 && !agg && !perm && slab_lg == cells_lg && (e.g == 8 || e.g == 16 || e.g == 32) &&
        sh.fast != 0) {
        auto launch_fast = [&](auto kern) -> cudaError_t {
            const size_t fsmem = (size_t)gpc * 48 + ((size_t)gpc * (split ? 4 : word_bytes) << cells_lg);
            cudaError_t err = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                   (int)fsmem);
            if (err != cudaSuccess) return err;
            const int groups = (e.k + gpc - 1) / gpc;
            int chunks = sh.chunks;
            if (chunks <= 0) chunks = auto_chunks(n, groups, fsmem > 110 * 1024 ? 1 : 2);
            const int64_t chunk = (n + chunks - 1) / chunks;
            kern<<<dim3(chunks, groups, 1), sh.threads, fsmem, s>>>(pos, n, chunk, e, gpc, mass);
            return cudaGetLastError();
        };
        if constexpr (SHARD) {
            if (e.g == 32) return launch_fast(deposit_fast_kernel<5, MODE, 4, MODE == 1, true>);
            if (e.g == 16) return launch_fast(deposit_fast_kernel<4, MODE, 4, false, true>);
            return launch_fast(deposit_fast_kernel<3, MODE, 4, false, true>);
        } else {
            if constexpr (MODE == 1) {
                if (count && e.g == 32) return launch_fast(deposit_fast_kernel<5, 1, 4, false, false, true>);
            }
            if (e.g == 32) {
                if constexpr (MODE == 1) {
                    if (ppt == 1) return launch_fast(deposit_fast_kernel<5, 1, 1, true>);
                    if (ppt == 2) return launch_fast(deposit_fast_kernel<5, 1, 2, true>);
                    return launch_fast(deposit_fast_kernel<5, 1, 4, true>);
                } else {
                    if (ppt == 1) return launch_fast(deposit_fast_kernel<5, MODE, 1>);
                    if (ppt == 2) return launch_fast(deposit_fast_kernel<5, MODE, 2>);
                    return launch_fast(deposit_fast_kernel<5, MODE, 4>);
                }
            }
            if constexpr (MODE == 1) {
                if (count && e.g == 16) return launch_fast(deposit_fast_kernel<4, 1, 4, false, false, true>);
                if (count) return launch_fast(deposit_fast_kernel<3, 1, 4, false, false, true>);
                if (split_small && e.g == 16) return launch_fast(deposit_fast_kernel<4, 1, 4, true>);
                if (split_small) return launch_fast(deposit_fast_kernel<3, 1, 4, true>);
            }
            if (e.g == 16) {
                if (ppt == 1) return launch_fast(deposit_fast_kernel<4, MODE, 1>);
                if (ppt == 2) return launch_fast(deposit_fast_kernel<4, MODE, 2>);
                return launch_fast(deposit_fast_kernel<4, MODE, 4>);
            }
            if (ppt == 1) return launch_fast(deposit_fast_kernel<3, MODE, 1>);
            if (ppt == 2) return launch_fast(deposit_fast_kernel<3, MODE, 2>);
            return launch_fast(deposit_fast_kernel<3, MODE, 4>);
        }
    }
    auto launch = [&](auto kern) -> cudaError_t {
        cudaError_t err = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               (int)smem);
        if (err != cudaSuccess) return err;
        const int groups = (e.k + gpc - 1) / gpc;
        const int slabs = 1 << (cells_lg - slab_lg);
        int chunks = sh.chunks;
        if (chunks <= 0) chunks = auto_chunks(n, groups * slabs, smem > 110 * 1024 ? 1 : 2);
        const int64_t chunk = (n + chunks - 1) / chunks;
        dim3 grid(chunks, groups, slabs);
        kern<<<grid, sh.threads, smem, s>>>(pos, perm, n, chunk, e, gpc, slab_lg, mass);
        return cudaGetLastError();
    };
    if constexpr (SHARD) {
        if (agg) return launch(deposit_smem_kernel<MODE, IDX, 4, true, true>);
        return launch(deposit_smem_kernel<MODE, IDX, 4, false, true>);
    } else {
        if (agg) {
            if (ppt == 1) return launch(deposit_smem_kernel<MODE, IDX, 1, true>);
            if (ppt == 4) return launch(deposit_smem_kernel<MODE, IDX, 4, true>);
            return launch(deposit_smem_kernel<MODE, IDX, 2, true>);
        }
        if (ppt == 1) return launch(deposit_smem_kernel<MODE, IDX, 1, false>);
        if (ppt == 4) return launch(deposit_smem_kernel<MODE, IDX, 4, false>);
        return launch(deposit_smem_kernel<MODE, IDX, 2, false>);
    }
}

// Work-queue deposit tiles hold whole grids: two words a cell in u64 mode
// at g <= 16, the split histogram's one word at g = 32, one word in u32
// mode; as many grids as fit 200 KB, lowered to a divisor of k when one is
// at least half of that (equal work per grid group).
int queue_deposit_grids(int g, int mass_mode, int k, bool split) {
    const size_t words = (mass_mode == MOG_MASS_U64_FIXED && g <= 16 && !split) ? 2 : 1;
    const size_t grid_bytes = 4 * words * (size_t)g * g * g + 48;
    const int most = (int)std::max<size_t>(1, std::min<size_t>((size_t)k, (200 * 1024) / grid_bytes));
    for (int d = most; d * 2 >= most && d >= 1; --d)
        if (k % d == 0) return d;
    return most;
}

size_t queue_deposit_smem(int g, int mass_mode, int ng, bool split) {
    const size_t words = (mass_mode == MOG_MASS_U64_FIXED && g <= 16 && !split) ? 2 : 1;
    return (size_t)ng * 48 + 4 * words * (size_t)ng * g * g * g;
}

cudaError_t launch_deposit_queue(int mass_mode, int layout, const BatchSim* sims,
                                 const DepositTile* tiles, int ntiles, unsigned* counter, size_t smem,
                                 cudaStream_t s) {
    if (ntiles <= 0) return cudaSuccess;
    auto go = [&](auto kern) -> cudaError_t {
        cudaError_t err = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               (int)smem);
        if (err != cudaSuccess) return err;
        const int ctas = std::min(ntiles, num_sms() * (smem > 110 * 1024 ? 1 : 2));
        kern<<<ctas, 1024, smem, s>>>(sims, tiles, ntiles, counter);
        return cudaGetLastError();
    };
    if (mass_mode != MOG_MASS_U64_FIXED) return go(deposit_queue_kernel<0, 0>);
    if (layout == 2) return go(deposit_queue_kernel<1, 2>);
    return layout == 1 ? go(deposit_queue_kernel<1, 1>) : go(deposit_queue_kernel<1, 0>);
}

cudaError_t launch_deposit(const Ensemble& e, const float4* pos, const int* perm, int64_t n,
                           bool ordered, void* mass, const DepositShape& shape, cudaStream_t s,
                           bool shard) {
    if (shard) {
        if (e.mass_mode == 0)
            return e.index_mode == 0 ? deposit_typed<1, 0, true>(e, pos, perm, n, ordered, mass, shape, s)
                                     : deposit_typed<1, 1, true>(e, pos, perm, n, ordered, mass, shape, s);
        return e.index_mode == 0 ? deposit_typed<0, 0, true>(e, pos, perm, n, ordered, mass, shape, s)
                                 : deposit_typed<0, 1, true>(e, pos, perm, n, ordered, mass, shape, s);
    }
    if (e.mass_mode == 0)
        return e.index_mode == 0 ? deposit_typed<1, 0, false>(e, pos, perm, n, ordered, mass, shape, s)
                                 : deposit_typed<1, 1, false>(e, pos, perm, n, ordered, mass, shape, s);
    return e.index_mode == 0 ? deposit_typed<0, 0, false>(e, pos, perm, n, ordered, mass, shape, s)
                             : deposit_typed<0, 1, false>(e, pos, perm, n, ordered, mass, shape, s);
}

}  // namespace mog
