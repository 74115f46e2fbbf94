// render.cu — headless particle renderer: the reference's particle draw
// (main.py:359-423, on_render main.py:678-703) as CUDA kernels writing an
// image into device memory.  The per-point and per-pixel arithmetic is
// render_math.cuh, shared with the host twin at the end of this file.
//
// GL blends the fragments of one pixel in primitive order, so the image
// depends on the order of the particles.  The kernels keep that order
// without per-pixel locks:
//   1. vertex:    one thread per particle: clip, window position, size,
//                 colour; the number of 16 x 16 pixel tiles its square may
//                 touch;
//   2. scan:      exclusive prefix sum of the counts (the (particle, tile)
//                 pair offsets, in particle order);
//   3. expand:    each particle writes its (tile, particle) pairs at its
//                 offset, so the pair list is in particle order;
//   4. sort:      stable LSD radix sort of the pairs by tile, 8 bits a pass:
//                 within a tile the particles stay in index order;
//   5. bounds:    first and one-past-last pair of every tile;
//   6. composite: one CTA per tile, one thread per pixel: the tile's
//                 particles are staged in shared memory 256 at a time with
//                 their pixel boxes, and every thread blends its pixel
//                 through the ones whose box holds it, in order.
// The result is the sequential GL blend, bit for bit (the host twin is
// that sequential loop).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <new>

#include "../../include/mog.h"
#include "mog_internal.h"
#include "render_math.cuh"

namespace mog {
namespace {

using rnd::Params;
using rnd::Splat;

constexpr int kTile = 16;                 // tile edge in pixels; composite CTA = kTile^2 threads
constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanBlock = kScanThreads * kScanItems;   // elements per scan block
constexpr int kSortThreads = 256;
constexpr int kSortWarps = kSortThreads / 32;
constexpr int kSortItems = 8;                           // entries per thread
constexpr int kSortBlock = kSortThreads * kSortItems;   // entries per sort block
constexpr int kRadix = 256;

// ---- 1. vertex -----------------------------------------------------------
__global__ void __launch_bounds__(256) render_vertex_kernel(const float4* __restrict__ pos,
                                                            const float4* __restrict__ vel,
                                                            int64_t n, Params R,
                                                            Splat* __restrict__ splats,
                                                            uint32_t* __restrict__ counts) {
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    const float4 P = pos[p], V = vel[p];
    Splat s;
    uint32_t c = 0;
    if (rnd::vertex(P.x, P.y, P.z, V.x, V.y, V.z, R, s)) {
        int i0, i1, j0, j1;
        if (rnd::pixel_range(s, R, i0, i1, j0, j1))
            c = (uint32_t)((i1 / kTile - i0 / kTile + 1) * (j1 / kTile - j0 / kTile + 1));
        splats[p] = s;
    }
    counts[p] = c;
}

// ---- 2. exclusive scan (any length; 2048 elements a block) -----------------
template <typename In, typename Out>
__global__ void __launch_bounds__(kScanThreads) scan_block_kernel(const In* __restrict__ in,
                                                                  Out* __restrict__ out, int64_t n,
                                                                  Out* __restrict__ sums,
                                                                  Out* __restrict__ total) {
    __shared__ Out warp_sum[kScanThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int64_t base = (int64_t)blockIdx.x * kScanBlock + (int64_t)threadIdx.x * kScanItems;
    Out v[kScanItems];
    Out s = 0;
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
        v[i] = base + i < n ? (Out)in[base + i] : (Out)0;
        s += v[i];
    }
    Out incl = s;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const Out t = __shfl_up_sync(kFull, incl, o);
        if (lane >= o) incl += t;
    }
    if (lane == 31) warp_sum[warp] = incl;
    __syncthreads();
    if (threadIdx.x == 0) {
        Out run = 0;
        for (int w = 0; w < kScanThreads / 32; ++w) {
            const Out t = warp_sum[w];
            warp_sum[w] = run;
            run += t;
        }
        if (sums) sums[blockIdx.x] = run;
        if (total && gridDim.x == 1) *total = run;
    }
    __syncthreads();
    Out run = warp_sum[warp] + incl - s;
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
        if (base + i < n) out[base + i] = run;
        run += v[i];
    }
}

template <typename T>
__global__ void __launch_bounds__(256) scan_add_kernel(T* __restrict__ out, int64_t n,
                                                       const T* __restrict__ offs) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] += offs[i / kScanBlock];
}

// Elements of scratch a scan of n elements needs (sums and their scan, per level).
int64_t scan_scratch(int64_t n) {
    int64_t total = 0;
    for (int64_t m = (n + kScanBlock - 1) / kScanBlock; m > 1; m = (m + kScanBlock - 1) / kScanBlock)
        total += 2 * m;
    return total;
}

// Kernel launches of scan_exclusive over n elements.
int scan_launches(int64_t n) {
    const int64_t nb = (n + kScanBlock - 1) / kScanBlock;
    return nb <= 1 ? 1 : 2 + scan_launches(nb);
}

// out[i] = in[0] + ... + in[i-1]; *total = the sum of all n (if non-null).
template <typename In, typename Out>
cudaError_t scan_exclusive(const In* in, Out* out, int64_t n, Out* scratch, Out* total,
                           cudaStream_t s) {
    const int64_t nb = (n + kScanBlock - 1) / kScanBlock;
    if (nb <= 1) {
        scan_block_kernel<In, Out><<<1, kScanThreads, 0, s>>>(in, out, n, nullptr, total);
        return cudaGetLastError();
    }
    Out* sums = scratch;
    Out* sums_scanned = scratch + nb;
    scan_block_kernel<In, Out><<<(unsigned)nb, kScanThreads, 0, s>>>(in, out, n, sums, nullptr);
    cudaError_t err = scan_exclusive<Out, Out>(sums, sums_scanned, nb, scratch + 2 * nb, total, s);
    if (err != cudaSuccess) return err;
    scan_add_kernel<Out><<<(unsigned)((n + 255) / 256), 256, 0, s>>>(out, n, sums_scanned);
    return cudaGetLastError();
}

// ---- 3. expand -------------------------------------------------------------
__global__ void __launch_bounds__(256) render_expand_kernel(const Splat* __restrict__ splats,
                                                            const uint32_t* __restrict__ counts,
                                                            const uint64_t* __restrict__ offsets,
                                                            int64_t n, Params R, int tiles_x,
                                                            uint32_t* __restrict__ keys,
                                                            uint32_t* __restrict__ vals) {
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n || counts[p] == 0) return;
    const Splat s = splats[p];
    int i0, i1, j0, j1;
    rnd::pixel_range(s, R, i0, i1, j0, j1);  // non-empty: counts[p] > 0
    uint64_t o = offsets[p];
    for (int ty = j0 / kTile; ty <= j1 / kTile; ++ty)
        for (int tx = i0 / kTile; tx <= i1 / kTile; ++tx) {
            keys[o] = (uint32_t)(ty * tiles_x + tx);
            vals[o] = (uint32_t)p;
            ++o;
        }
}

// ---- 4. stable radix sort by tile -------------------------------------------
// Pass over digit (key >> shift) & 255.  Block b holds entries
// [b * 2048, (b + 1) * 2048); warp w of it the 256 entries from b * 2048 +
// w * 256, taken 32 at a time in order.  counts[d * nblocks + b] = entries
// of block b with digit d.
__global__ void __launch_bounds__(kSortThreads) sort_hist_kernel(const uint32_t* __restrict__ keys,
                                                                 int64_t m, int shift,
                                                                 uint32_t* __restrict__ counts,
                                                                 int64_t nblocks) {
    __shared__ uint32_t hist[kRadix];
    hist[threadIdx.x] = 0;
    __syncthreads();
    const int64_t base = (int64_t)blockIdx.x * kSortBlock;
    for (int i = threadIdx.x; i < kSortBlock; i += kSortThreads)
        if (base + i < m) atomicAdd(&hist[(keys[base + i] >> shift) & (kRadix - 1)], 1u);
    __syncthreads();
    counts[(int64_t)threadIdx.x * nblocks + blockIdx.x] = hist[threadIdx.x];
}

// offsets = exclusive scan of counts (digit-major): where block b's first
// entry with digit d goes.  Each warp ranks its entries among equal digits
// with __match_any_sync, in entry order, so equal keys keep their order.
__global__ void __launch_bounds__(kSortThreads) sort_scatter_kernel(
    const uint32_t* __restrict__ keys_in, const uint32_t* __restrict__ vals_in, int64_t m,
    int shift, const uint32_t* __restrict__ offsets, int64_t nblocks,
    uint32_t* __restrict__ keys_out, uint32_t* __restrict__ vals_out) {
    __shared__ uint32_t wcount[kSortWarps][kRadix];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int w = 0; w < kSortWarps; ++w) wcount[w][threadIdx.x] = 0;
    __syncthreads();
    const int64_t first = (int64_t)blockIdx.x * kSortBlock + (int64_t)warp * (kSortBlock / kSortWarps);
    const unsigned lt = (1u << lane) - 1u;
    // per-warp digit counts
    for (int step = 0; step < kSortBlock / kSortWarps / 32; ++step) {
        const int64_t i = first + step * 32 + lane;
        const bool valid = i < m;
        const uint32_t d = valid ? (keys_in[i] >> shift) & (kRadix - 1) : kRadix;
        const unsigned same = __match_any_sync(kFull, d);
        if (valid && (same & lt) == 0) wcount[warp][d] += (uint32_t)__popc(same);
        __syncwarp();
    }
    __syncthreads();
    // thread d: exclusive prefix of digit d over the warps, from the global offset
    {
        const int d = threadIdx.x;
        uint32_t run = offsets[(int64_t)d * nblocks + blockIdx.x];
        for (int w = 0; w < kSortWarps; ++w) {
            const uint32_t c = wcount[w][d];
            wcount[w][d] = run;
            run += c;
        }
    }
    __syncthreads();
    for (int step = 0; step < kSortBlock / kSortWarps / 32; ++step) {
        const int64_t i = first + step * 32 + lane;
        const bool valid = i < m;
        const uint32_t key = valid ? keys_in[i] : 0u;
        const uint32_t d = valid ? (key >> shift) & (kRadix - 1) : kRadix;
        const unsigned same = __match_any_sync(kFull, d);
        if (valid) {
            const uint32_t dst = wcount[warp][d] + (uint32_t)__popc(same & lt);
            keys_out[dst] = key;
            vals_out[dst] = vals_in[i];
        }
        __syncwarp();
        if (valid && (same & lt) == 0) wcount[warp][d] += (uint32_t)__popc(same);
        __syncwarp();
    }
}

// ---- 5. tile bounds ----------------------------------------------------------
__global__ void __launch_bounds__(256) tile_bounds_kernel(const uint32_t* __restrict__ keys,
                                                          int64_t m, uint32_t* __restrict__ start,
                                                          uint32_t* __restrict__ end) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    const uint32_t k = keys[i];
    if (i == 0 || keys[i - 1] != k) start[k] = (uint32_t)i;
    if (i == m - 1 || keys[i + 1] != k) end[k] = (uint32_t)(i + 1);
}

// ---- 6. composite --------------------------------------------------------------
__global__ void __launch_bounds__(kTile* kTile) render_composite_kernel(
    const Splat* __restrict__ splats, const uint32_t* __restrict__ vals,
    const uint32_t* __restrict__ start, const uint32_t* __restrict__ end, Params R, int tiles_x,
    void* __restrict__ image) {
    __shared__ Splat stage[kTile * kTile];
    __shared__ int4 box[kTile * kTile];  // pixel_range of each staged splat (a superset of its pixels)
    const int tile = blockIdx.x;
    const int px = (tile % tiles_x) * kTile + (threadIdx.x % kTile);
    const int py = (tile / tiles_x) * kTile + (threadIdx.x / kTile);
    const bool inside = px < R.width && py < R.height;
    const float xc = (float)px + 0.5f, yc = (float)py + 0.5f;
    rnd::Pixel pix;
    rnd::clear_pixel(R, pix);
    const uint32_t lo = start[tile], hi = end[tile];
    for (uint32_t b = lo; b < hi; b += kTile * kTile) {
        const uint32_t cnt = min((uint32_t)(kTile * kTile), hi - b);
        if (threadIdx.x < cnt) {
            const Splat sp = splats[vals[b + threadIdx.x]];
            int i0, i1, j0, j1;
            rnd::pixel_range(sp, R, i0, i1, j0, j1);
            stage[threadIdx.x] = sp;
            box[threadIdx.x] = make_int4(i0, i1, j0, j1);
        }
        __syncthreads();
        if (inside) {
            for (uint32_t j = 0; j < cnt; ++j) {
                // most splats miss most pixels: reject on the integer box
                // before the exact test
                const int4 bx = box[j];
                if (px < bx.x || px > bx.y || py < bx.z || py > bx.w) continue;
                float a;
                if (rnd::fragment(stage[j], xc, yc, a)) rnd::blend_pixel(R, stage[j], a, pix);
            }
        }
        __syncthreads();
    }
    if (!inside) return;
    const size_t o = ((size_t)(R.height - 1 - py) * R.width + px) * 4;
    if (R.format == MOG_RENDER_RGBA8) {
        uchar4 q = make_uchar4((unsigned char)pix.c[0], (unsigned char)pix.c[1],
                               (unsigned char)pix.c[2], (unsigned char)pix.c[3]);
        reinterpret_cast<uchar4*>(image)[o / 4] = q;
    } else {
        reinterpret_cast<float4*>(image)[o / 4] = make_float4(pix.c[0], pix.c[1], pix.c[2], pix.c[3]);
    }
}

// ---- host side -------------------------------------------------------------------
const char* check_params(const mog_render_params* p) {
    if (!p) return "null render parameters";
    if (p->width < 1 || p->height < 1 || p->width > 16384 || p->height > 16384)
        return "image size must be 1..16384 in each direction";
    if (!std::isfinite(p->world_size) || p->world_size <= 0.f) return "world_size must be > 0";
    if (!std::isfinite(p->speed_scale)) return "speed_scale must be finite";
    for (int i = 0; i < 16; ++i)
        if (!std::isfinite(p->m_view[i]) || !std::isfinite(p->m_proj[i]))
            return "camera matrices must be finite";
    for (int i = 0; i < 4; ++i)
        if (!std::isfinite(p->clear[i])) return "clear colour must be finite";
    if (p->point_mode != 0 && p->point_mode != 1) return "point_mode must be 0 or 1";
    if (!(p->point_size >= 1.f && p->point_size <= 65536.f)) return "point_size must be in [1, 65536]";
    if (!(p->max_point_size >= 1.f && p->max_point_size <= 65536.f))
        return "max_point_size must be in [1, 65536]";
    if (p->format != MOG_RENDER_RGBA8 && p->format != MOG_RENDER_RGBA32F)
        return "format must be MOG_RENDER_RGBA8 or MOG_RENDER_RGBA32F";
    return nullptr;
}

Params make_params(const mog_render_params* p) {
    Params R;
    rnd::mat_mul(p->m_proj, p->m_view, R.M);  // GLSL m_proj * m_view
    R.world = p->world_size;
    R.speed_scale = p->speed_scale;
    R.half_w = (float)p->width * 0.5f;
    R.half_h = (float)p->height * 0.5f;
    R.width = p->width;
    R.height = p->height;
    R.program_size = p->point_mode;
    R.point_size = p->point_size;
    R.max_point_size = p->max_point_size;
    for (int i = 0; i < 4; ++i) R.clear[i] = p->clear[i];
    R.format = p->format;
    R.tile = kTile;
    return R;
}

}  // namespace
}  // namespace mog

struct mog_renderer {
    int device = 0;
    void* buf[9] = {};
    size_t cap[9] = {};
    uint64_t* host_total = nullptr;  // pinned
    int64_t last_pairs = 0;          // (point, tile) pairs of the last frame
    int32_t last_launches = 0;       // kernels the last frame launched
};

namespace {

// Device buffer slot `i` with at least `bytes`; contents are not kept.
cudaError_t grow(mog_renderer* r, int i, size_t bytes, void** out) {
    if (bytes == 0) bytes = 16;
    if (r->cap[i] < bytes) {
        if (r->buf[i]) {
            cudaError_t e = cudaFree(r->buf[i]);
            r->buf[i] = nullptr;
            r->cap[i] = 0;
            if (e != cudaSuccess) return e;
        }
        const size_t want = bytes + bytes / 4;
        cudaError_t e = cudaMalloc(&r->buf[i], want);
        if (e != cudaSuccess) return e;
        r->cap[i] = want;
    }
    *out = r->buf[i];
    return cudaSuccess;
}

int cuda_error(cudaError_t e, const char* where) {
    static thread_local char msg[256];
    snprintf(msg, sizeof msg, "%s: %s", where, cudaGetErrorString(e));
    return mog::report_error(MOG_ERR_CUDA, msg);
}

}  // namespace

extern "C" {

void mog_render_params_default(mog_render_params* p) {
    if (!p) return;
    std::memset(p, 0, sizeof *p);
    p->width = 2560;
    p->height = 1440;
    p->world_size = 100.f;
    p->speed_scale = 0.f;
    for (int i = 0; i < 4; ++i) p->m_view[5 * i] = p->m_proj[5 * i] = 1.f;
    p->clear[0] = 0.01f;
    p->clear[1] = 0.01f;
    p->clear[2] = 0.02f;
    p->clear[3] = 0.f;
    p->point_mode = 0;
    p->point_size = 1.f;
    p->max_point_size = 2047.f;
    p->format = MOG_RENDER_RGBA8;
}

int mog_renderer_create(mog_renderer** out) {
    if (!out) return mog::report_error(MOG_ERR_ARG, "null output pointer");
    *out = nullptr;
    mog_renderer* r = new (std::nothrow) mog_renderer();
    if (!r) return mog::report_error(MOG_ERR_ARG, "out of host memory");
    cudaError_t e = cudaGetDevice(&r->device);
    if (e == cudaSuccess) e = cudaMallocHost(&r->host_total, sizeof(uint64_t));
    if (e != cudaSuccess) {
        delete r;
        return cuda_error(e, "mog_renderer_create");
    }
    *out = r;
    return MOG_OK;
}

int mog_renderer_destroy(mog_renderer* r) {
    if (!r) return MOG_OK;
    for (void* b : r->buf)
        if (b) cudaFree(b);
    if (r->host_total) cudaFreeHost(r->host_total);
    delete r;
    return MOG_OK;
}

int mog_render(mog_renderer* r, const mog_render_params* p, const float* pos4, const float* vel4,
               int64_t n, void* image, void* stream) {
    using namespace mog;
    if (const char* why = check_params(p)) return report_error(MOG_ERR_ARG, why);
    if (!r || !image || n < 0 || n > 0xFFFFFFFFll || (n > 0 && (!pos4 || !vel4)))
        return report_error(MOG_ERR_ARG, "bad renderer, image, particle buffers or count");
    if (reinterpret_cast<uintptr_t>(image) % (p->format == MOG_RENDER_RGBA8 ? 4 : 16) != 0 ||
        reinterpret_cast<uintptr_t>(pos4) % 16 != 0 || reinterpret_cast<uintptr_t>(vel4) % 16 != 0)
        return report_error(MOG_ERR_ARG, "image must be 4-byte (RGBA8) or 16-byte (RGBA32F) "
                                         "aligned, particle buffers 16-byte aligned");
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev != r->device)
        return report_error(MOG_ERR_ARG, "the renderer was created on another device");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    r->last_pairs = 0;
    r->last_launches = 0;
    const Params R = make_params(p);
    const int tiles_x = (p->width + kTile - 1) / kTile;
    const int tiles_y = (p->height + kTile - 1) / kTile;
    const int64_t tiles = (int64_t)tiles_x * tiles_y;
    cudaError_t e;
    void *splats, *counts, *offsets, *scan_tmp, *bounds;
#define MOG_R(call, where)                              \
    do {                                                \
        if ((e = (call)) != cudaSuccess) return cuda_error(e, where); \
    } while (0)
    const int64_t nn = n > 0 ? n : 1;
    MOG_R(grow(r, 0, sizeof(Splat) * nn, &splats), "render buffers");
    MOG_R(grow(r, 1, sizeof(uint32_t) * nn, &counts), "render buffers");
    MOG_R(grow(r, 2, sizeof(uint64_t) * (nn + 1), &offsets), "render buffers");
    MOG_R(grow(r, 3, sizeof(uint64_t) * (scan_scratch(nn) + 1), &scan_tmp), "render buffers");
    MOG_R(grow(r, 4, sizeof(uint32_t) * 2 * tiles, &bounds), "render buffers");
    uint32_t* start = static_cast<uint32_t*>(bounds);
    uint32_t* end = start + tiles;
    uint64_t* total = static_cast<uint64_t*>(offsets) + nn;
    MOG_R(cudaMemsetAsync(bounds, 0, sizeof(uint32_t) * 2 * tiles, s), "render clear bounds");
    MOG_R(cudaMemsetAsync(total, 0, sizeof(uint64_t), s), "render clear total");
    if (n > 0) {
        const unsigned blocks = (unsigned)((n + 255) / 256);
        render_vertex_kernel<<<blocks, 256, 0, s>>>(reinterpret_cast<const float4*>(pos4),
                                                    reinterpret_cast<const float4*>(vel4), n, R,
                                                    static_cast<Splat*>(splats),
                                                    static_cast<uint32_t*>(counts));
        MOG_R(cudaGetLastError(), "render vertex");
        r->last_launches += 1 + scan_launches(n);
        MOG_R((scan_exclusive<uint32_t, uint64_t>(static_cast<uint32_t*>(counts),
                                                  static_cast<uint64_t*>(offsets), n,
                                                  static_cast<uint64_t*>(scan_tmp), total, s)),
              "render scan");
    }
    MOG_R(cudaMemcpyAsync(r->host_total, total, sizeof(uint64_t), cudaMemcpyDeviceToHost, s),
          "render read pair count");
    MOG_R(cudaStreamSynchronize(s), "render read pair count");
    const uint64_t m = *r->host_total;
    r->last_pairs = (int64_t)m;
    if (m > 0x7FFFFFFFull)
        return report_error(MOG_ERR_UNSUPPORTED, "the points touch more than 2^31 - 1 (point, tile) pairs");
    if (m > 0) {
        void *k0, *v0, *k1, *v1, *hist;
        MOG_R(grow(r, 5, sizeof(uint32_t) * m, &k0), "render pair buffers");
        MOG_R(grow(r, 6, sizeof(uint32_t) * m, &v0), "render pair buffers");
        MOG_R(grow(r, 7, sizeof(uint32_t) * 2 * m, &k1), "render pair buffers");
        v1 = static_cast<uint32_t*>(k1) + m;
        const int64_t nblocks = ((int64_t)m + kSortBlock - 1) / kSortBlock;
        const int64_t hn = nblocks * kRadix;
        MOG_R(grow(r, 8, sizeof(uint32_t) * (2 * hn + scan_scratch(hn) + 1), &hist), "render sort buffers");
        uint32_t* hcount = static_cast<uint32_t*>(hist);
        uint32_t* hoff = hcount + hn;
        uint32_t* htmp = hoff + hn;
        render_expand_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(
            static_cast<Splat*>(splats), static_cast<uint32_t*>(counts),
            static_cast<uint64_t*>(offsets), n, R, tiles_x, static_cast<uint32_t*>(k0),
            static_cast<uint32_t*>(v0));
        MOG_R(cudaGetLastError(), "render expand");
        int bits = 0;
        while (((int64_t)1 << bits) < tiles) ++bits;
        uint32_t *kin = static_cast<uint32_t*>(k0), *vin = static_cast<uint32_t*>(v0);
        uint32_t *kout = static_cast<uint32_t*>(k1), *vout = static_cast<uint32_t*>(v1);
        for (int shift = 0; shift < bits; shift += 8) {
            sort_hist_kernel<<<(unsigned)nblocks, kSortThreads, 0, s>>>(kin, (int64_t)m, shift,
                                                                         hcount, nblocks);
            MOG_R(cudaGetLastError(), "render sort");
            MOG_R((scan_exclusive<uint32_t, uint32_t>(hcount, hoff, hn, htmp, nullptr, s)),
                  "render sort scan");
            sort_scatter_kernel<<<(unsigned)nblocks, kSortThreads, 0, s>>>(
                kin, vin, (int64_t)m, shift, hoff, nblocks, kout, vout);
            MOG_R(cudaGetLastError(), "render sort");
            std::swap(kin, kout);
            std::swap(vin, vout);
            r->last_launches += 2 + scan_launches(hn);
        }
        tile_bounds_kernel<<<(unsigned)(((int64_t)m + 255) / 256), 256, 0, s>>>(kin, (int64_t)m,
                                                                                 start, end);
        MOG_R(cudaGetLastError(), "render bounds");
        render_composite_kernel<<<(unsigned)tiles, kTile * kTile, 0, s>>>(
            static_cast<Splat*>(splats), vin, start, end, R, tiles_x, image);
        r->last_launches += 3;  // expand, bounds, composite
    } else {
        render_composite_kernel<<<(unsigned)tiles, kTile * kTile, 0, s>>>(
            static_cast<Splat*>(splats), nullptr, start, end, R, tiles_x, image);
        r->last_launches += 1;
    }
    MOG_R(cudaGetLastError(), "render composite");
#undef MOG_R
    return MOG_OK;
}

int mog_renderer_stats(const mog_renderer* r, int64_t* pairs, int32_t* launches) {
    if (!r) return mog::report_error(MOG_ERR_ARG, "null renderer");
    if (pairs) *pairs = r->last_pairs;
    if (launches) *launches = r->last_launches;
    return MOG_OK;
}

int mog_render_host(const mog_render_params* p, const float* pos4, const float* vel4, int64_t n,
                    void* image) {
    using namespace mog;
    if (const char* why = check_params(p)) return report_error(MOG_ERR_ARG, why);
    if (!image || n < 0 || n > 0xFFFFFFFFll || (n > 0 && (!pos4 || !vel4)))
        return report_error(MOG_ERR_ARG, "bad image, particle buffers or count");
    const Params R = make_params(p);
    const int W = p->width, H = p->height;
    rnd::Pixel* fb = new (std::nothrow) rnd::Pixel[(size_t)W * H];
    if (!fb) return report_error(MOG_ERR_ARG, "out of host memory");
    for (size_t i = 0; i < (size_t)W * H; ++i) rnd::clear_pixel(R, fb[i]);
    for (int64_t q = 0; q < n; ++q) {
        const float* P = pos4 + 4 * q;
        const float* V = vel4 + 4 * q;
        Splat s;
        int i0, i1, j0, j1;
        if (!rnd::vertex(P[0], P[1], P[2], V[0], V[1], V[2], R, s)) continue;
        if (!rnd::pixel_range(s, R, i0, i1, j0, j1)) continue;
        for (int j = j0; j <= j1; ++j)
            for (int i = i0; i <= i1; ++i) {
                float a;
                if (rnd::fragment(s, (float)i + 0.5f, (float)j + 0.5f, a))
                    rnd::blend_pixel(R, s, a, fb[(size_t)j * W + i]);
            }
    }
    for (int j = 0; j < H; ++j)
        for (int i = 0; i < W; ++i) {
            const rnd::Pixel& px = fb[(size_t)j * W + i];
            const size_t o = ((size_t)(H - 1 - j) * W + i) * 4;
            for (int k = 0; k < 4; ++k) {
                if (p->format == MOG_RENDER_RGBA8)
                    static_cast<unsigned char*>(image)[o + k] = (unsigned char)px.c[k];
                else
                    static_cast<float*>(image)[o + k] = px.c[k];
            }
        }
    delete[] fb;
    return MOG_OK;
}

}  // extern "C"
