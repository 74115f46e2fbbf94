// update.cu — K3: force gather over all k grids, ensemble average and the
// damped leapfrog update.
//
// Replaces update.glsl:53-89 (one thread per particle, k image loads and
// k 3x3 transposed-rotation products).  Two changes make it cheap:
//  * the spectral epilogue already stored every grid's force rotated back
//    into the world frame (M_i F_i(cell), the very product update.glsl:77
//    forms, with the same FP32 operations), so a (particle, grid) touch is
//    one cell index + one float4 load + three adds; it stored cell c at
//    force_slot(c) (x XORed with (2y ^ 4z) mod 8), so that the cells a
//    warp's particles fall in, and their y and z neighbours, spread over
//    the 16-byte bank quads of a staged grid instead of sharing one;
//  * for large particle counts each CTA stages grid i's whole force field
//    (g^3 float4, 64 KB at g = 16) in shared memory with one bulk async
//    copy (cp.async.bulk + mbarrier), three stages deep, and every
//    particle the CTA owns gathers from shared memory.  The per-particle
//    state (centred position, running force) stays in registers across all
//    k grids, so HBM sees each particle once for reading and once for
//    writing.
// The force accumulates grid by grid in index order, like the shader's
// loop, so the result is bit-identical to a sequential FP32 evaluation.
#include <algorithm>

#include "mog_internal.h"

namespace mog {

namespace {

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}
__device__ __forceinline__ void mbar_fence_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes,
                                         uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// One 16-byte shared load (ld.shared.v4) at a shared-window address.  A
// volatile asm is neither repeated nor moved across the mbarrier waits, so
// the grid rows loaded with it stay in registers for the whole grid instead
// of being reloaded for every particle.
__device__ __forceinline__ float4 ld_shared_f4_at(uint32_t addr) {
    float4 v;
    asm volatile("ld.shared.v4.f32 {%0, %1, %2, %3}, [%4];"
                 : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
                 : "r"(addr));
    return v;
}
// Orders this thread's generic-proxy shared-memory accesses before its
// later bulk (async-proxy) copies into the same memory.
__device__ __forceinline__ void fence_proxy_async_shared() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
// Bounded wait: gives up after ~2^31 SM cycles (about a second) and
// reports false; the caller then abandons the launch with MOG_FLAG_TIMEOUT.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, unsigned parity) {
    const long long t0 = clock64();
    while (!mbar_try_wait(bar, parity)) {
        if (clock64() - t0 > (1ll << 31)) return false;
    }
    return true;
}

// Shared epilogue: average, then update.glsl:81-89 with IEEE ops.
template <bool ACC_OUT>
__device__ __forceinline__ void finish_particle(int64_t p, float4 P, float ax, float ay, float az,
                                                float4* __restrict__ pos, float4* __restrict__ vel,
                                                float4* __restrict__ acc_out, float kf, float dt,
                                                float damp, float world, unsigned& bad) {
    ax = __fdiv_rn(ax, kf);
    ay = __fdiv_rn(ay, kf);
    az = __fdiv_rn(az, kf);
    if (ACC_OUT) {
        acc_out[p] = make_float4(ax, ay, az, 0.f);
        return;
    }
    const float4 V = vel[p];
    float vx = __fsub_rn(V.x, __fmul_rn(ax, dt));
    float vy = __fsub_rn(V.y, __fmul_rn(ay, dt));
    float vz = __fsub_rn(V.z, __fmul_rn(az, dt));
    vx = __fmul_rn(vx, damp);
    vy = __fmul_rn(vy, damp);
    vz = __fmul_rn(vz, damp);
    float px = glsl_mod(__fadd_rn(P.x, __fmul_rn(vx, dt)), world);
    float py = glsl_mod(__fadd_rn(P.y, __fmul_rn(vy, dt)), world);
    float pz = glsl_mod(__fadd_rn(P.z, __fmul_rn(vz, dt)), world);
    if (!(isfinite(px) && isfinite(py) && isfinite(pz))) bad |= 1u;
    pos[p] = make_float4(px, py, pz, P.w);
    vel[p] = make_float4(vx, vy, vz, 0.f);
}

// One grid's gathers for a thread's PPT particles from the staged grid at
// shared address F (xf: the grid's 16 transform floats there, r0..r2 its
// FAST rows already in registers): slot, one 16-byte shared load, the
// running force (x, y as a pair, one add.f32x2: two IEEE adds) in grid
// order.  FULL: every slot is live (no per-particle test).  LG > 0: g = 2^LG
// at compile time.
template <int IDX, int PPT, int LG, bool FULL>
__device__ __forceinline__ void gather_grid(uint32_t F, const float* x, const float4& r0,
                                            const float4& r1, const float4& r2,
                                            const float (&cx)[PPT], const float (&cy)[PPT],
                                            const float (&cz)[PPT], float2 (&axy)[PPT],
                                            float (&az)[PPT], int cnt, const IndexParams& ip,
                                            unsigned* flags) {
    const int lg = LG > 0 ? LG : ip.lg;
    const uint32_t G3 = 1u << (3 * lg);
#pragma unroll
    for (int j = 0; j < PPT; ++j) {
        if (FULL || j < cnt) {
            uint32_t c = IDX == 0 ? slot_fast(r0, r1, r2, cx[j], cy[j], cz[j], lg)
                                  : force_slot(cell_exact(x, x + 12, cx[j], cy[j], cz[j], ip), lg);
            if (!in_bounds(flags, c, (uint64_t)G3)) c = 0;
            const float4 f = ld_shared_f4_at(F + (c << 4));
            axy[j] = __fadd2_rn(axy[j], make_float2(f.x, f.y));
            az[j] = __fadd_rn(az[j], f.z);
        }
    }
}

// Particle in slot `slot` (slot < n).  A checked build redirects a
// permutation entry outside [0, n) to the slot itself and flags it.
__device__ __forceinline__ int64_t particle_of(const int* __restrict__ perm, int64_t slot,
                                               int64_t n, unsigned* flags) {
    if (!perm) return slot;
    const int64_t p = (int64_t)__ldg(perm + slot);
    return in_bounds(flags, (uint64_t)p, (uint64_t)n) ? p : slot;
}

// Copy grid i's force field (or the z-slabs of it that the CTA's particles
// can reach) into a stage.  t_z = a . c + b is affine in the centred
// position, so over the CTA's bounding box of c it is extremal at the
// corners; every particle's z cell lies in [floor(min t_z), floor(max t_z)]
// (a 0.01-cell margin covers the rounding of either index mode).
__device__ __forceinline__ void issue_grid(int i, int s, const float4* __restrict__ W,
                                           float4* stage, uint64_t* full, int lg,
                                           const float* box, bool sparse, const float* xf,
                                           int idx_mode, const IndexParams& ip) {
    const int g = 1 << lg;
    const int G3 = 1 << (3 * lg);
    const unsigned slab = (unsigned)g * g;  // float4 per z-slab
    const float4* src = W + (size_t)i * G3;
    float4* dst = stage + (size_t)s * G3;
    int z0 = 0, nz = g;
    if (sparse) {
        float a0, a1, a2, b, inv = 1.0f;
        const float* x = xf + i * 16;
        if (idx_mode == 0) {
            a0 = x[8];
            a1 = x[9];
            a2 = x[10];
            b = x[11];
        } else {  // rotated_z = R[2] c.x + R[6] c.y + R[10] c.z, t_z = (rotated_z + L/2 - off_z) / h
            a0 = x[2];
            a1 = x[6];
            a2 = x[10];
            b = ip.half_l - x[14];
            inv = 1.0f / ip.voxel;
        }
        float tmin = 3.0e38f, tmax = -3.0e38f;
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const float cx = box[(q & 1) ? 3 : 0], cy = box[(q & 2) ? 4 : 1], cz = box[(q & 4) ? 5 : 2];
            const float t = (a0 * cx + a1 * cy + a2 * cz + b) * inv;
            tmin = fminf(tmin, t);
            tmax = fmaxf(tmax, t);
        }
        if (isfinite(tmin) && isfinite(tmax) && tmax - tmin < (float)(g - 2)) {
            const int zlo = __float2int_rd(tmin - 0.01f);
            const int zhi = __float2int_rd(tmax + 0.01f);
            nz = zhi - zlo + 1;
            z0 = zlo & (g - 1);
        }
    }
    if (nz >= g) {
        mbar_expect_tx(full + s, (unsigned)G3 * 16u);
        bulk_g2s(dst, src, (unsigned)G3 * 16u, full + s);
        return;
    }
    mbar_expect_tx(full + s, (unsigned)nz * slab * 16u);
    const int first = min(nz, g - z0);
    bulk_g2s(dst + (size_t)z0 * slab, src + (size_t)z0 * slab, (unsigned)first * slab * 16u, full + s);
    if (nz > first)
        bulk_g2s(dst, src, (unsigned)(nz - first) * slab * 16u, full + s);
}

// Staged gather.  Launch: one CTA per SM (shared-memory bound).  The CTA
// owns slots [lo, hi); thread t owns slots lo + t + j * blockDim, so the
// 32 lanes of a warp always hold consecutive slots: with a spatial
// ordering they fall in the same few cells and their shared-memory loads
// broadcast instead of conflicting, and the CTA's particles occupy a small
// box, so only the z-slabs of each grid that the box reaches are staged.
template <int IDX, int PPT, bool ACC_OUT, int THREADS, int LG = 0, int FULLP = 0>
__global__ void __launch_bounds__(THREADS, 1)
    update_staged_kernel(float4* __restrict__ pos, float4* __restrict__ vel,
                         const float4* __restrict__ pos_s, const int* __restrict__ perm,
                         int64_t n, int64_t per_cta, const float4* __restrict__ W, Ensemble e,
                         float dt, float damp, float4* __restrict__ acc_out, int nstage,
                         int sparse) {
    extern __shared__ __align__(128) unsigned char smem[];
    const int G3 = 1 << (3 * e.lg);
    const size_t grid_bytes = (size_t)G3 * 16u;
    float4* stage = reinterpret_cast<float4*>(smem);
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + (size_t)nstage * grid_bytes);
    float* xf = reinterpret_cast<float*>(full + 8);
    __shared__ int abort_flag;
    __shared__ float box[6];        // min c.xyz, max c.xyz of the CTA's particles
    __shared__ float wbox[THREADS / 32][6];   // per-warp partial boxes
    __shared__ unsigned stage_done[8];        // warps done with a stage's current grid
    __shared__ int stage_grid[8];             // grid last copied into a stage

    const int tid = threadIdx.x;
    const int T = blockDim.x;
    if (tid == 0) {
        abort_flag = 0;
        for (int s = 0; s < nstage; ++s) {
            mbar_init(full + s, 1);
            stage_done[s] = 0u;
            stage_grid[s] = s < e.k ? s : -1;
        }
        mbar_fence_init();
    }
    for (int i = tid; i < e.k * 16; i += T) {
        const int j = i >> 4, w = i & 15;
        float v;
        if (IDX == 0)
            v = (w < 12) ? reinterpret_cast<const float*>(e.fast + j)[w] : 0.f;
        else
            v = (w < 12) ? e.rot12[j * 12 + w] : e.off4[j * 4 + (w - 12)];
        xf[i] = v;
    }

    const IndexParams ip = e.index_params();
    const int64_t lo = (int64_t)blockIdx.x * per_cta;
    const int64_t hi = min(n, lo + per_cta);
    const int64_t first = lo + tid;
    const int64_t mine = hi - first;
    const int64_t slots = (mine + T - 1) / T;
    const int cnt = mine <= 0 ? 0 : (int)(slots < PPT ? slots : PPT);
    float cx[PPT], cy[PPT], cz[PPT], az[PPT];
    float2 axy[PPT];
    float bmin[3] = {3.0e38f, 3.0e38f, 3.0e38f}, bmax[3] = {-3.0e38f, -3.0e38f, -3.0e38f};
#pragma unroll
    for (int j = 0; j < PPT; ++j) {
        float4 P = make_float4(0.f, 0.f, 0.f, 0.f);
        if (j < cnt) {
            const int64_t slot = first + (int64_t)j * T;
            P = pos_s ? pos_s[slot] : pos[particle_of(perm, slot, n, e.flags)];
        }
        cx[j] = __fsub_rn(P.x, ip.half_l);
        cy[j] = __fsub_rn(P.y, ip.half_l);
        cz[j] = __fsub_rn(P.z, ip.half_l);
        axy[j] = make_float2(0.f, 0.f);
        az[j] = 0.f;
        if (j < cnt) {
            bmin[0] = fminf(bmin[0], cx[j]);
            bmin[1] = fminf(bmin[1], cy[j]);
            bmin[2] = fminf(bmin[2], cz[j]);
            bmax[0] = fmaxf(bmax[0], cx[j]);
            bmax[1] = fmaxf(bmax[1], cy[j]);
            bmax[2] = fmaxf(bmax[2], cz[j]);
        }
    }
    if (sparse) {
        for (int o = 16; o > 0; o >>= 1)
            for (int a = 0; a < 3; ++a) {
                bmin[a] = fminf(bmin[a], __shfl_xor_sync(kFull, bmin[a], o));
                bmax[a] = fmaxf(bmax[a], __shfl_xor_sync(kFull, bmax[a], o));
            }
        if ((tid & 31) == 0)
            for (int a = 0; a < 3; ++a) {
                wbox[tid >> 5][a] = bmin[a];
                wbox[tid >> 5][3 + a] = bmax[a];
            }
    }
    __syncthreads();
    if (tid == 0) {
        if (sparse) {
            for (int a = 0; a < 3; ++a) {
                float mn = 3.0e38f, mx = -3.0e38f;
                for (int w = 0; w < (T >> 5); ++w) {
                    mn = fminf(mn, wbox[w][a]);
                    mx = fmaxf(mx, wbox[w][3 + a]);
                }
                box[a] = mn;
                box[3 + a] = mx;
            }
        }
        for (int s = 0; s < nstage && s < e.k; ++s)
            issue_grid(s, s, W, stage, full, e.lg, box, sparse && box[0] <= box[3], xf, IDX, ip);
    }

    // No block-wide barrier per grid: each warp waits for the grid's copy,
    // gathers, and counts itself done with the stage; the last warp to finish
    // grid i refills the stage with grid i + nstage.  Warps drift up to
    // nstage grids apart instead of waiting for the slowest one every grid.
    const unsigned nwarps = (unsigned)(T >> 5);
    const uint32_t stage_s = smem_u32(stage);
    bool aborted = false;
    for (int i = 0; i < e.k; ++i) {
        const int s = i % nstage;
        const unsigned parity = (unsigned)((i / nstage) & 1);
        if (!__all_sync(kFull, mbar_wait_bounded(full + s, parity))) {
            aborted = true;  // warp-uniform
            break;
        }
        const uint32_t F = stage_s + (uint32_t)s * (uint32_t)G3 * 16u;
        const float* x = xf + i * 16;
        float4 r0 = make_float4(0.f, 0.f, 0.f, 0.f), r1 = r0, r2 = r0;
        if (IDX == 0) {  // the grid's FAST rows, once per grid
            const uint32_t xa = smem_u32(x);
            r0 = ld_shared_f4_at(xa);
            r1 = ld_shared_f4_at(xa + 16);
            r2 = ld_shared_f4_at(xa + 32);
        }
        if (FULLP && cnt == PPT)
            gather_grid<IDX, PPT, LG, true>(F, x, r0, r1, r2, cx, cy, cz, axy, az, cnt, ip, e.flags);
        else
            gather_grid<IDX, PPT, LG, false>(F, x, r0, r1, r2, cx, cy, cz, axy, az, cnt, ip, e.flags);
        // every lane's loads of the stage have returned (their values are
        // summed) before the warp counts itself done
        __syncwarp();
        if ((tid & 31) == 0) {
            __threadfence_block();
            if (atomicAdd(&stage_done[s], 1u) == nwarps - 1) {
                stage_done[s] = 0u;
                __threadfence_block();
                if (i + nstage < e.k) {
                    stage_grid[s] = i + nstage;
                    fence_proxy_async_shared();
                    issue_grid(i + nstage, s, W, stage, full, e.lg, box, sparse && box[0] <= box[3],
                               xf, IDX, ip);
                }
            }
        }
    }
    if (aborted && (tid & 31) == 0) abort_flag = 1;
    __syncthreads();
    if (abort_flag) {
        // A copy never landed.  The copy issued last into each stage may
        // still be in flight: let it land (bounded as well) before the CTA's
        // shared memory is released, then report and leave.
        if (tid == 0) {
            atomicOr(e.flags, 4u);
            for (int q = 0; q < nstage; ++q) {
                const int j = stage_grid[q];
                if (j >= 0) (void)mbar_wait_bounded(full + q, (unsigned)((j / nstage) & 1));
            }
        }
        return;
    }

    unsigned bad = 0;
    const float kf = (float)e.k;
#pragma unroll
    for (int j = 0; j < PPT; ++j) {
        if (j < cnt) {
            const int64_t slot = first + (int64_t)j * T;
            const int64_t p = particle_of(perm, slot, n, e.flags);
            const float4 P = pos_s ? pos_s[slot] : pos[p];
            finish_particle<ACC_OUT>(p, P, axy[j].x, axy[j].y, az[j], pos, vel, acc_out, kf, dt,
                                     damp, e.world, bad);
        }
    }
    if (bad) raise_flags(e.flags, bad);
}

// Batched ensemble, one persistent launch for every simulation of a batch:
// each CTA pops tiles (simulation, particle chunk of THREADS * PPT) from
// the host-built list with an atomic counter.  A tile of a simulation with
// g <= 16 stages its grids one by one in shared memory exactly as
// update_staged_kernel does (bulk copies into `nstage` stages of 64 KB on
// mbarriers); a tile with g = 32 (512 KB a grid) gathers from L2.  The
// copy count runs on across tiles, so each stage's mbarrier parity is that
// count's round.  Per particle the force is summed grid by grid in index
// order, so every simulation's result is bit-identical to its own step.
template <int PPT, int THREADS>
__global__ void __launch_bounds__(THREADS, 1)
    gather_queue_kernel(const BatchSim* __restrict__ sims, const GatherTile* __restrict__ tiles,
                        int ntiles, unsigned* __restrict__ counter, int nstage) {
    extern __shared__ __align__(128) unsigned char smem[];
    constexpr size_t kStageBytes = (size_t)16 << 12;  // one g = 16 grid of float4
    float4* stage = reinterpret_cast<float4*>(smem);
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + (size_t)nstage * kStageBytes);
    float* xf = reinterpret_cast<float*>(full + 8);
    __shared__ int s_tile;
    __shared__ int abort_flag;
    const int tid = threadIdx.x;
    if (tid == 0) {
        abort_flag = 0;
        for (int q = 0; q < nstage; ++q) mbar_init(full + q, 1);
        mbar_fence_init();
    }
    __syncthreads();
    const float no_box[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    uint32_t issued = 0;  // bulk copies this CTA has issued (the same in every thread)
    for (;;) {
        if (tid == 0) s_tile = (int)atomicAdd(counter, 1u);
        __syncthreads();
        const int t = s_tile;
        if (t >= ntiles) return;  // block-uniform
        const GatherTile tile = tiles[t];
        const BatchSim& S = sims[tile.sim];
        const Ensemble e = S.e;
        const float4* W = S.force;
        float4* pos = S.pos;
        const IndexParams ip = e.index_params();
        const int G3 = 1 << (3 * e.lg);
        const int64_t first = tile.lo + tid;
        const int64_t mine = tile.hi - first;
        const int cnt = mine <= 0 ? 0 : (int)((mine + THREADS - 1) / THREADS < PPT ? (mine + THREADS - 1) / THREADS : PPT);
        float cx[PPT], cy[PPT], cz[PPT], az[PPT];
        float2 axy[PPT];
#pragma unroll
        for (int j = 0; j < PPT; ++j) {
            const float4 P = j < cnt ? pos[first + (int64_t)j * THREADS] : make_float4(0.f, 0.f, 0.f, 0.f);
            cx[j] = __fsub_rn(P.x, ip.half_l);
            cy[j] = __fsub_rn(P.y, ip.half_l);
            cz[j] = __fsub_rn(P.z, ip.half_l);
            axy[j] = make_float2(0.f, 0.f);
            az[j] = 0.f;
        }
        if (e.lg <= 4) {
            for (int i = tid; i < e.k * 16; i += THREADS) {
                const int j = i >> 4, w = i & 15;
                xf[i] = (w < 12) ? reinterpret_cast<const float*>(e.fast + j)[w] : 0.f;
            }
            __syncthreads();
            if (tid == 0)
                for (int q = 0; q < nstage && q < e.k; ++q)
                    issue_grid(q, (int)((issued + q) % nstage), W, stage, full, e.lg, no_box, false,
                               xf, 0, ip);
            for (int i = 0; i < e.k; ++i) {
                const uint32_t c = issued + (uint32_t)i;
                const int q = (int)(c % nstage);
                if (!mbar_wait_bounded(full + q, (c / nstage) & 1u)) abort_flag = 1;
                const uint32_t F = smem_u32(stage) + (uint32_t)q * (uint32_t)G3 * 16u;
                const uint32_t xa = smem_u32(xf + i * 16);
                const float4 r0 = ld_shared_f4_at(xa), r1 = ld_shared_f4_at(xa + 16),
                             r2 = ld_shared_f4_at(xa + 32);
                if (e.lg == 4)  // g = 16 with compile-time shifts and masks
                    gather_grid<0, PPT, 4, false>(F, nullptr, r0, r1, r2, cx, cy, cz, axy, az, cnt,
                                                  ip, e.flags);
                else
                    gather_grid<0, PPT, 0, false>(F, nullptr, r0, r1, r2, cx, cy, cz, axy, az, cnt,
                                                  ip, e.flags);
                __syncthreads();
                if (abort_flag) {
                    // let the copies still in flight land (bounded) before the
                    // CTA's shared memory is released, then report and leave
                    if (tid == 0) {
                        atomicOr(e.flags, 4u);
                        for (int j = i; j < i + nstage && j < e.k; ++j) {
                            const uint32_t cj = issued + (uint32_t)j;
                            (void)mbar_wait_bounded(full + cj % nstage, (cj / nstage) & 1u);
                        }
                    }
                    return;
                }
                if (tid == 0 && i + nstage < e.k)
                    issue_grid(i + nstage, q, W, stage, full, e.lg, no_box, false, xf, 0, ip);
            }
            issued += (uint32_t)e.k;
        } else {
            for (int i = 0; i < e.k; ++i) {
                const FastXf xr = e.fast[i];
                const float4* F = W + (size_t)i * G3;
                uint32_t prev = 0xffffffffu;
                float4 f = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
                for (int j = 0; j < PPT; ++j) {
                    if (j < cnt) {
                        uint32_t cell = slot_fast(xr.row[0], xr.row[1], xr.row[2], cx[j], cy[j], cz[j], ip.lg);
                        if (!in_bounds(e.flags, cell, (uint64_t)G3)) cell = 0;
                        if (cell != prev) f = __ldg(F + cell);
                        prev = cell;
                        axy[j] = __fadd2_rn(axy[j], make_float2(f.x, f.y));
                        az[j] = __fadd_rn(az[j], f.z);
                    }
                }
            }
        }
        unsigned bad = 0;
#pragma unroll
        for (int j = 0; j < PPT; ++j) {
            if (j < cnt) {
                const int64_t p = first + (int64_t)j * THREADS;
                finish_particle<false>(p, pos[p], axy[j].x, axy[j].y, az[j], pos, S.vel, nullptr,
                                       (float)e.k, S.dt, S.damping, e.world, bad);
            }
        }
        if (bad) raise_flags(e.flags, bad);
        __syncthreads();  // the next tile reuses xf, the stages and s_tile
    }
}

// Direct gather from L1/L2, any g: each thread owns DPPT consecutive slots
// and reuses a force value when consecutive particles share a cell.
template <int IDX, int DPPT, bool ACC_OUT>
__global__ void __launch_bounds__(256) update_direct_kernel(float4* __restrict__ pos,
                                                            float4* __restrict__ vel,
                                                            const float4* __restrict__ pos_s,
                                                            const int* __restrict__ perm,
                                                            int64_t n,
                                                            const float4* __restrict__ W,
                                                            Ensemble e, float dt, float damp,
                                                            float4* __restrict__ acc_out) {
    const int64_t first = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) * DPPT;
    if (first >= n) return;
    const int cnt = (int)(n - first < DPPT ? n - first : DPPT);
    const IndexParams ip = e.index_params();
    float cx[DPPT], cy[DPPT], cz[DPPT], ax[DPPT], ay[DPPT], az[DPPT];
#pragma unroll
    for (int j = 0; j < DPPT; ++j) {
        float4 P = make_float4(0.f, 0.f, 0.f, 0.f);
        if (j < cnt) P = pos_s ? pos_s[first + j] : pos[particle_of(perm, first + j, n, e.flags)];
        cx[j] = __fsub_rn(P.x, ip.half_l);
        cy[j] = __fsub_rn(P.y, ip.half_l);
        cz[j] = __fsub_rn(P.z, ip.half_l);
        ax[j] = ay[j] = az[j] = 0.f;
    }
    const int G3 = 1 << (3 * e.lg);
    for (int i = 0; i < e.k; ++i) {
        const float4* F = W + (size_t)i * G3;
        uint32_t prev = 0xffffffffu;
        float4 f = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
        for (int j = 0; j < DPPT; ++j) {
            if (j < cnt) {
                uint32_t c;
                if (IDX == 0) {
                    const FastXf x = e.fast[i];
                    c = slot_fast(x.row[0], x.row[1], x.row[2], cx[j], cy[j], cz[j], ip.lg);
                } else {
                    c = force_slot(cell_exact(e.rot12 + 12 * i, e.off4 + 4 * i, cx[j], cy[j], cz[j], ip),
                                   ip.lg);
                }
                if (!in_bounds(e.flags, c, (uint64_t)G3)) c = 0;
                if (c != prev) f = __ldg(F + c);
                prev = c;
                ax[j] = __fadd_rn(ax[j], f.x);
                ay[j] = __fadd_rn(ay[j], f.y);
                az[j] = __fadd_rn(az[j], f.z);
            }
        }
    }
    unsigned bad = 0;
#pragma unroll
    for (int j = 0; j < DPPT; ++j) {
        if (j < cnt) {
            const int64_t p = particle_of(perm, first + j, n, e.flags);
            finish_particle<ACC_OUT>(p, pos_s ? pos_s[first + j] : pos[p], ax[j], ay[j], az[j], pos, vel, acc_out,
                                     (float)e.k, dt, damp, e.world, bad);
        }
    }
    if (bad) raise_flags(e.flags, bad);
}

template <int IDX, int PPT, bool ACC, int THREADS>
cudaError_t launch_staged(const Ensemble& e, float4* pos, float4* vel, const float4* pos_s,
                          const int* perm, int64_t n, const float4* W, float dt, float damp,
                          float4* acc, int ctas, int nstage, size_t smem, int sparse,
                          cudaStream_t s) {
    // g = 16 (the staged grids are g <= 16) with compile-time shifts and
    // masks; a check-free copy of the particle loop where the registers
    // leave room for it (PPT <= 8)
    auto kern = (IDX == 0 && e.lg == 4)
                    ? update_staged_kernel<IDX, PPT, ACC, THREADS, 4, (PPT <= 8 ? 1 : 0)>
                    : update_staged_kernel<IDX, PPT, ACC, THREADS, 0, 0>;
    const int threads = THREADS;
    cudaError_t err =
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (err != cudaSuccess) return err;
    const int64_t per_cta = (n + ctas - 1) / ctas;
    kern<<<ctas, threads, smem, s>>>(pos, vel, pos_s, perm, n, per_cta, W, e, dt, damp, acc, nstage,
                                     sparse);
    return cudaGetLastError();
}

template <int IDX, bool ACC>
cudaError_t update_mode(const Ensemble& e, float4* pos, float4* vel, const float4* pos_s,
                        const int* perm, int64_t n, const float4* W, float dt, float damp,
                        float4* acc, const UpdateShape& sh, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    const size_t grid_bytes = (size_t)16 << (3 * e.lg);
    const int sms = num_sms();
    const int threads = 512;  // minimum staged launch, for the auto choice below
    const int nstage = 3;
    const size_t smem = nstage * grid_bytes + 8 * sizeof(uint64_t) + (size_t)e.k * 16 * sizeof(float);
    bool staged;
    if (sh.staged >= 0)
        staged = sh.staged != 0;
    else
        staged = e.g <= 16 && n >= (int64_t)sms * threads * 2 && smem <= 220 * 1024;
    if (staged && smem > 220 * 1024) staged = false;
    if (!staged) {
        // auto (0): 4 particles a thread (cell reuse, loads in flight) once
        // there are enough threads to fill the SMs, else 1
        const int dppt = sh.direct_ppt == 1 || sh.direct_ppt == 2 || sh.direct_ppt == 4
                             ? sh.direct_ppt
                             : (n >= (int64_t)sms * 256 * 8 ? 4 : 1);
        const int64_t threads_needed = (n + dppt - 1) / dppt;
        const unsigned blocks = (unsigned)((threads_needed + 255) / 256);
        if (dppt == 1)
            update_direct_kernel<IDX, 1, ACC><<<blocks, 256, 0, s>>>(pos, vel, pos_s, perm, n, W, e, dt,
                                                                     damp, acc);
        else if (dppt == 2)
            update_direct_kernel<IDX, 2, ACC><<<blocks, 256, 0, s>>>(pos, vel, pos_s, perm, n, W, e, dt,
                                                                     damp, acc);
        else
            update_direct_kernel<IDX, 4, ACC><<<blocks, 256, 0, s>>>(pos, vel, pos_s, perm, n, W, e, dt,
                                                                     damp, acc);
        return cudaGetLastError();
    }
    // Sparse staging only pays when the CTAs' particles are spatially compact.
    const int sparse = (pos_s || perm) ? 1 : 0;
    // Block size (occupancy) against particles per thread (registers): the
    // launch bounds give 512 threads ~128 registers, 768 ~85, 1024 64.  Auto
    // (0) is 512: measured at c2 (N = 2^20, k = 240) 0.456 ms against 0.518
    // ms for 1024 threads of 7 particles.
    const int T = sh.threads == 768 || sh.threads == 1024 ? sh.threads : 512;
    const int max_ppt = T == 512 ? 16 : (T == 768 ? 10 : 7);
    int ctas = sh.ctas > 0 ? sh.ctas : sms;
    const int64_t per_thread = (n + (int64_t)ctas * T - 1) / ((int64_t)ctas * T);
    if (per_thread > max_ppt) ctas = (int)((n + (int64_t)max_ppt * T - 1) / ((int64_t)max_ppt * T));
    const int64_t ppt = (n + (int64_t)ctas * T - 1) / ((int64_t)ctas * T);
#define MOG_STAGED(P, TH) \
    return launch_staged<IDX, P, ACC, TH>(e, pos, vel, pos_s, perm, n, W, dt, damp, acc, ctas, nstage, smem, sparse, s)
    if (T == 1024) {
        if (ppt <= 4) MOG_STAGED(4, 1024);
        MOG_STAGED(7, 1024);
    }
    if (T == 768) {
        if (ppt <= 4) MOG_STAGED(4, 768);
        if (ppt <= 8) MOG_STAGED(8, 768);
        MOG_STAGED(10, 768);
    }
    if (ppt <= 4) MOG_STAGED(4, 512);
    if (ppt <= 8) MOG_STAGED(8, 512);
    if (ppt <= 12) MOG_STAGED(12, 512);
    if (ppt <= 14) MOG_STAGED(14, 512);
    MOG_STAGED(16, 512);
#undef MOG_STAGED
}

// One bounded wait that nothing satisfies: a fresh mbarrier expecting one
// arrival, waited on by thread 0 with the gather's own mbar_wait_bounded.
// It gives up after its budget and raises MOG_FLAG_TIMEOUT (4), exactly as
// the staged gather does when a bulk copy never lands.
__global__ void __launch_bounds__(32) wait_timeout_selftest_kernel(unsigned* flags) {
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        mbar_fence_init();
    }
    __syncthreads();
    if (threadIdx.x == 0 && !mbar_wait_bounded(&bar, 0)) atomicOr(flags, 4u);
}

}  // namespace

cudaError_t launch_wait_timeout_selftest(unsigned* flags, cudaStream_t s) {
    wait_timeout_selftest_kernel<<<1, 32, 0, s>>>(flags);
    return cudaGetLastError();
}

cudaError_t launch_gather_queue(const BatchSim* sims, const GatherTile* tiles, int ntiles,
                                unsigned* counter, int kmax, cudaStream_t s) {
    if (ntiles <= 0) return cudaSuccess;
    constexpr int nstage = 3;
    const size_t smem = nstage * ((size_t)16 << 12) + 8 * sizeof(uint64_t) +
                        (size_t)std::max(kmax, 1) * 16 * sizeof(float);
    if (smem > 227 * 1024) return cudaErrorInvalidValue;
    auto kern = gather_queue_kernel<kQueueGatherPPT, kQueueGatherThreads>;
    cudaError_t err = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (err != cudaSuccess) return err;
    kern<<<std::min(ntiles, num_sms()), kQueueGatherThreads, smem, s>>>(sims, tiles, ntiles, counter,
                                                                        nstage);
    return cudaGetLastError();
}

cudaError_t launch_update(const Ensemble& e, float4* pos, float4* vel, const float4* pos_s,
                          const int* perm, int64_t n, const float4* force_world, float dt,
                          float damping, float4* acc_out, const UpdateShape& shape, cudaStream_t s) {
    if (acc_out)
        return e.index_mode == 0 ? update_mode<0, true>(e, pos, vel, pos_s, perm, n, force_world,
                                                        dt, damping, acc_out, shape, s)
                                 : update_mode<1, true>(e, pos, vel, pos_s, perm, n, force_world,
                                                        dt, damping, acc_out, shape, s);
    return e.index_mode == 0 ? update_mode<0, false>(e, pos, vel, pos_s, perm, n, force_world, dt,
                                                     damping, nullptr, shape, s)
                             : update_mode<1, false>(e, pos, vel, pos_s, perm, n, force_world, dt,
                                                     damping, nullptr, shape, s);
}

}  // namespace mog
