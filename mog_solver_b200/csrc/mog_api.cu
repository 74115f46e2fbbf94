// mog_api.cu — the C ABI of include/mog.h.
//
// Replaces the reference's Simulation set-up and step orchestration
// (main.py:108-248 for buffers, textures, shaders and transforms;
// main.py:558-672 for clear_mass / step_fft / step).  The reference issues
// a host upload of zeros plus about 65 dispatches with a memory barrier
// after each (g = 16); one step here is three kernels on the caller's
// stream (deposit, spectral solve, gather + update), and mog_step_n
// replays a captured CUDA graph of that step.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/mog.h"
#include "mog_internal.h"

namespace {

thread_local std::string g_last_error;

int fail(int code, const std::string& msg) {
    g_last_error = msg;
    return code;
}
int cuda_fail(cudaError_t err, const char* where) {
    std::string m = std::string(where) + ": " + cudaGetErrorName(err) + " (" +
                    cudaGetErrorString(err) + ")";
    return fail(MOG_ERR_CUDA, m);
}

}  // namespace

namespace mog {
// Sets the calling thread's mog_last_error() text; returns code.
int report_error(int code, const char* msg) { return fail(code, msg); }
}  // namespace mog

namespace {

#define MOG_CUDA(call, where)                          \
    do {                                               \
        cudaError_t err__ = (call);                    \
        if (err__ != cudaSuccess) return cuda_fail(err__, where); \
    } while (0)

}  // namespace

namespace mog {

int num_sms() {
    static int cached[64] = {0};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) return 148;
    if (cached[dev] == 0) {
        int v = 0;
        if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v <= 0)
            v = 148;
        cached[dev] = v;
    }
    return cached[dev];
}

namespace {

__global__ void check_total_kernel(Ensemble e) {
    if (e.mass_mode == 0 && e.mass_total) {
        if (*e.mass_total >= 18446744073709551616.0) atomicOr(e.flags, 2u);
        *e.mass_total = 0.0;
    }
}

// FP64 reductions: per-block partial sums, then a fixed-order final sum, so
// the result does not depend on scheduling.
__global__ void __launch_bounds__(256) diag_partial_kernel(const float4* __restrict__ pos,
                                                           const float4* __restrict__ vel,
                                                           int64_t n, double* __restrict__ partial) {
    double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n;
         p += (int64_t)gridDim.x * blockDim.x) {
        const float4 P = pos[p];
        const float4 V = vel[p];
        const double m = P.w, vx = V.x, vy = V.y, vz = V.z;
        acc[0] += m * vx;
        acc[1] += m * vy;
        acc[2] += m * vz;
        acc[3] += 0.5 * m * (vx * vx + vy * vy + vz * vz);
        acc[4] += m;
        acc[5] += m * (double)P.x;
        acc[6] += m * (double)P.y;
        acc[7] += m * (double)P.z;
    }
    __shared__ double red[8][256];
    for (int q = 0; q < 8; ++q) red[q][threadIdx.x] = acc[q];
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w)
            for (int q = 0; q < 8; ++q) red[q][threadIdx.x] += red[q][threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x < 8) partial[blockIdx.x * 8 + threadIdx.x] = red[threadIdx.x][0];
}

__global__ void diag_final_kernel(const double* __restrict__ partial, int nblocks,
                                  double* __restrict__ out8) {
    if (threadIdx.x != 0) return;
    double s[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int b = 0; b < nblocks; ++b)
        for (int q = 0; q < 8; ++q) s[q] += partial[b * 8 + q];
    for (int q = 0; q < 5; ++q) out8[q] = s[q];
    const double m = s[4];
    for (int q = 0; q < 3; ++q) out8[5 + q] = m != 0.0 ? s[5 + q] / m : 0.0;
}

}  // namespace

cudaError_t launch_diagnostics(const float4* pos, const float4* vel, int64_t n, double* partial,
                               int nblocks, double* out8, cudaStream_t s) {
    diag_partial_kernel<<<nblocks, 256, 0, s>>>(pos, vel, n, partial);
    diag_final_kernel<<<1, 32, 0, s>>>(partial, nblocks, out8);
    return cudaGetLastError();
}

}  // namespace mog

struct GraphEntry {
    float* pos = nullptr;
    float* vel = nullptr;
    int64_t n = 0;
    float dt = 0.f;
    bool sorts = false;       // whether the captured step re-orders the particles
    cudaGraphExec_t exec = nullptr;
};

struct mog_model {
    int device = 0;
    float* d_params = nullptr;
    float* d_m = nullptr;
    float* d_v = nullptr;
    float* d_grad = nullptr;
    void* d_frags = nullptr;
    float* d_partial = nullptr;
    float* d_loss = nullptr;
    int partial_ctas = 0;
    int step = 0;
    mog::ModelNorm norm{};
};

// A handle's part in a sharded step over peer memory (mog_shard_*).
struct ShardState {
    int rank = 0;
    int world = 0;                   // 0: not sharded
    void* d_accum = nullptr;         // this rank's accumulation buffer: 3 slots of k g^3 cells
    uint64_t* d_flags = nullptr;     // this rank's flag words, one per rank
    mog::ShardTargets* d_targets = nullptr;  // every rank's buffer for each of the 3 slots
    mog::ShardView view;             // every rank's buffers (this rank's included)
    bool ipc[mog::kMaxShardRanks] = {};  // rank q's buffers were opened from IPC handles
    bool connected = false;
    uint64_t epoch = 0;              // steps deposited (the flags' value)
};

struct mog_handle {
    mog_config cfg{};
    int device = 0;
    mog::Ensemble e;
    mog::DepositShape dshape;
    mog::UpdateShape ushape;
    float* d_rot12 = nullptr;
    float* d_off4 = nullptr;
    mog::FastXf* d_fast = nullptr;
    float* d_green = nullptr;
    float* d_ktab = nullptr;
    float4* d_conv = nullptr;
    unsigned* d_flags = nullptr;
    double* d_total = nullptr;
    void* d_mass = nullptr;      // k g^3 (u64 or u32)
    float4* d_force = nullptr;   // k g^3 world-frame forces
    float4* d_force2 = nullptr;  // stage-update staging (lazy)
    void* d_scratch = nullptr;   // spectral scratch (g >= 32, or tensor-core DFT passes)
    void* d_dft = nullptr;       // DFT matrices of the tensor-core passes
    double* d_diag = nullptr;    // diagnostics partials + result
    int* d_perm = nullptr;       // spatial order of the particles (slot -> particle)
    float4* d_pos_s = nullptr;   // positions in spatial order (refreshed every step)
    void* d_sort = nullptr;      // counting-sort scratch
    int64_t perm_cap = 0;        // capacity of d_perm
    int64_t perm_n = -1;         // n the permutation was built for
    int sort_every = 0;          // re-order every this many steps (0 = never)
    int learned_fold = 1;        // learned step: cell masses written by the solve's epilogue
    int learned_ctas = 2;        // learned kernel CTAs per SM (2 or 3)
    int solve_split = 0;         // g = 8/16 fft solve on 3-CTA clusters: 0 auto, 1, -1
    uint64_t step_count = 0;     // steps issued (decides when to re-order)
    std::vector<GraphEntry> graphs;
    std::vector<mog::GridRows> rows;  // learned-gather rows of the k grids (host)
    float* d_spread = nullptr;        // per-CTA (spread, |mean force|) sums of the last learned step
    int spread_cap = 0;               // CTAs d_spread has room for
    int spread_blocks = 0;
    int64_t spread_n = 0;
    ShardState shard;
    // steps over host-memory particles (mog_step_host, mog_learned_step_host):
    // device copies of the records, a copy-in and a copy-out stream, and the
    // events that order each chunk's copies against its kernels
    float4* d_hpos = nullptr;
    float4* d_hvel = nullptr;
    int64_t host_cap = 0;
    cudaStream_t s_in = nullptr;
    cudaStream_t s_out = nullptr;
    cudaEvent_t ev_start = nullptr;
    cudaEvent_t ev_out = nullptr;
    std::vector<cudaEvent_t> ev_pos, ev_vel, ev_done;
};

namespace {

constexpr int kDiagBlocks = 296;

bool is_pow2(int v) { return v > 0 && (v & (v - 1)) == 0; }

int validate(const mog_config& c) {
    if (c.n_grids <= 0) return fail(MOG_ERR_CONFIG, "n_grids must be positive");
    if (c.n_grids > 4096) return fail(MOG_ERR_CONFIG, "n_grids must be <= 4096");
    if (!is_pow2(c.grid_size) || c.grid_size < 2 || c.grid_size > 64)
        return fail(MOG_ERR_CONFIG, "grid_size must be a power of two in [2, 64]");
    if (!(std::isfinite(c.world_size) && c.world_size > 0.f))
        return fail(MOG_ERR_CONFIG, "world_size must be finite and positive");
    if (!std::isfinite(c.G)) return fail(MOG_ERR_CONFIG, "G must be finite");
    if (!std::isfinite(c.dt)) return fail(MOG_ERR_CONFIG, "dt must be finite");
    if (!std::isfinite(c.damping)) return fail(MOG_ERR_CONFIG, "damping must be finite");
    if (c.solver != MOG_SOLVER_FFT && c.solver != MOG_SOLVER_CONVOLUTION)
        return fail(MOG_ERR_CONFIG, "solver must be fft (0) or convolution (1)");
    if (c.solver == MOG_SOLVER_CONVOLUTION && c.grid_size > 32)
        return fail(MOG_ERR_UNSUPPORTED, "convolution solver supports grid_size <= 32");
    if (c.mass_mode != MOG_MASS_U64_FIXED && c.mass_mode != MOG_MASS_U32_X1000)
        return fail(MOG_ERR_CONFIG, "mass_mode must be 0 (u64 fixed) or 1 (u32 x1000)");
    if (c.scale_bits < 0 || c.scale_bits > 100)
        return fail(MOG_ERR_CONFIG, "scale_bits must be in [0, 100]");
    if (c.index_mode != MOG_INDEX_FAST && c.index_mode != MOG_INDEX_EXACT)
        return fail(MOG_ERR_CONFIG, "index_mode must be 0 (fast) or 1 (exact)");
    if (c.dft_prec != MOG_DFT_FFT32 && c.dft_prec != MOG_DFT_TC_BF16X3)
        return fail(MOG_ERR_CONFIG, "dft_prec must be 0 (fp32 fft) or 1 (tensor-core bf16x3)");
    if (c.num_particles < 0) return fail(MOG_ERR_CONFIG, "num_particles must be >= 0");
    if (c.compat_flags & ~MOG_COMPAT_FFT_TEXTURE_ALIAS)
        return fail(MOG_ERR_CONFIG, "unknown compat_flags bits");
    if (!(std::isfinite(c.softening) && c.softening >= 0.f))
        return fail(MOG_ERR_CONFIG, "softening must be finite and >= 0");
    if (c.softening > 0.f && c.solver != MOG_SOLVER_FFT)
        return fail(MOG_ERR_CONFIG, "softening applies to the fft solver only");
    return MOG_OK;
}

// Green's factors on [kz][ky][kx] (greens.glsl:17-47): FP64 values, the
// reference's FP32 k^2 > 1e-4 test for which bins are kept.
std::vector<float> green_table(int g, float world, float G, float softening) {
    std::vector<float> out((size_t)g * g * g, 0.f);
    auto shift = [g](int i) { return i <= g / 2 ? i : i - g; };
    volatile float two_pi_f = 2.0f * 3.14159265359f;  // the shader's TWO_PI
    const float step_f = two_pi_f / world;
    const double two_pi = 6.283185307179586476925286766559;
    const double step = two_pi / (double)world;
    const double a = (double)softening * (double)world / (double)g;
    for (int iz = 0; iz < g; ++iz)
        for (int iy = 0; iy < g; ++iy)
            for (int ix = 0; ix < g; ++ix) {
                volatile float kxf = (float)shift(ix) * step_f, kyf = (float)shift(iy) * step_f,
                               kzf = (float)shift(iz) * step_f;
                volatile float kxx = kxf * kxf, kyy = kyf * kyf, kzz = kzf * kzf;
                volatile float k2xy = kxx + kyy;
                const float k2f = k2xy + kzz;
                if (!(k2f > 1e-4f)) continue;
                const double kx = shift(ix) * step, ky = shift(iy) * step, kz = shift(iz) * step;
                const double k2 = kx * kx + ky * ky + kz * kz;
                const double v = softening > 0.f ? -2.0 * two_pi * (double)G * std::exp(-k2 * a * a) / k2
                                                 : -two_pi * (double)G / k2;
                out[((size_t)iz * g + iy) * g + ix] = (float)v;
            }
    return out;
}

// Real-space kernel of init_greens_kernel (main.py:250-278), FP64 then f4,
// same operation order so the table matches the reference's bit for bit.
std::vector<float> conv_kernel_table(int g, double voxel) {
    std::vector<float> k((size_t)g * g * g * 4, 0.f);
    const double pi = 3.141592653589793;
    for (int iz = 0; iz < g; ++iz)
        for (int iy = 0; iy < g; ++iy)
            for (int ix = 0; ix < g; ++ix) {
                const int dx = ix <= g / 2 ? ix : ix - g;
                const int dy = iy <= g / 2 ? iy : iy - g;
                const int dz = iz <= g / 2 ? iz : iz - g;
                const double rx = dx * voxel, ry = dy * voxel, rz = dz * voxel;
                const double r2 = rx * rx + ry * ry + rz * rz;
                const double r = std::sqrt(r2);
                if (r > 1e-10) {
                    const double f = 1.0 / (4.0 * pi * r2 * r);
                    float* o = &k[(((size_t)iz * g + iy) * g + ix) * 4];
                    o[0] = (float)(rx * f);
                    o[1] = (float)(ry * f);
                    o[2] = (float)(rz * f);
                }
            }
    return k;
}

int set_device(mog_handle* h) {
    int cur = -1;
    MOG_CUDA(cudaGetDevice(&cur), "cudaGetDevice");
    if (cur != h->device) MOG_CUDA(cudaSetDevice(h->device), "cudaSetDevice");
    return MOG_OK;
}

int check_particles(mog_handle* h, const void* pos, const void* vel, int64_t n, bool need_vel) {
    if (n < 0) return fail(MOG_ERR_ARG, "n must be >= 0");
    if (n > 0 && !pos) return fail(MOG_ERR_ARG, "pos4 is null");
    if (n > 0 && need_vel && !vel) return fail(MOG_ERR_ARG, "vel4 is null");
    if (((uintptr_t)pos & 15) || ((uintptr_t)vel & 15))
        return fail(MOG_ERR_ARG, "pos4/vel4 must be 16-byte aligned");
    if (h->cfg.num_particles > 0 && n > h->cfg.num_particles)
        return fail(MOG_ERR_ARG, "n exceeds the handle's num_particles capacity");
    return MOG_OK;
}

// Whether the next step re-orders the particles (a permutation of [0, n)
// must exist for this n before any kernel reads it).
bool wants_sort(const mog_handle* h, int64_t n) {
    if (h->sort_every <= 0 || n <= 0) return false;
    return h->perm_n != n || h->step_count % (uint64_t)h->sort_every == 0;
}

// Spatial ordering.  When ordering is on, (re)build the permutation if
// `sort`, then gather the positions into spatial order (every step: they
// move); *perm and *pos_s are what the kernels read, or null when off.
int order_particles(mog_handle* h, const float4* pos, int64_t n, bool sort, cudaStream_t s,
                    const int** perm, const float4** pos_s) {
    *perm = nullptr;
    *pos_s = nullptr;
    if (h->sort_every <= 0 || n <= 0) return MOG_OK;
    if (n > h->perm_cap) {
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        cudaStreamIsCapturing(s, &cs);
        if (cs != cudaStreamCaptureStatusNone)
            return fail(MOG_ERR_ARG, "n exceeds num_particles inside a captured step");
        if (h->d_perm) cudaFree(h->d_perm);
        if (h->d_pos_s) cudaFree(h->d_pos_s);
        h->d_perm = nullptr;
        h->d_pos_s = nullptr;
        h->perm_n = -1;
        MOG_CUDA(cudaMalloc((void**)&h->d_perm, sizeof(int) * n), "cudaMalloc perm");
        MOG_CUDA(cudaMalloc((void**)&h->d_pos_s, sizeof(float4) * n), "cudaMalloc sorted positions");
        h->perm_cap = n;
    }
    if (sort || h->perm_n != n) {
        cudaError_t err = mog::launch_sort(pos, n, h->e.world, h->d_sort, h->d_perm, h->d_flags, s);
        if (err != cudaSuccess) return cuda_fail(err, "spatial order");
        h->perm_n = n;
    }
    cudaError_t err = mog::launch_gather_sorted(pos, h->d_perm, n, h->d_pos_s, s);
    if (err != cudaSuccess) return cuda_fail(err, "gather sorted positions");
    *perm = h->d_perm;
    *pos_s = h->d_pos_s;
    return MOG_OK;
}

// The kernels of one step (or of a force evaluation when acc != null).
int run_pipeline(mog_handle* h, float4* pos, float4* vel, int64_t n, float dt, float4* acc,
                 cudaStream_t s, bool sort) {
    const mog::Ensemble& e = h->e;
    const int* perm = nullptr;
    const float4* pos_s = nullptr;
    int rc = order_particles(h, pos, n, sort, s, &perm, &pos_s);
    if (rc) return rc;
    // The mass grid does not depend on the order; shared atomics from
    // spatially ordered lanes collide on one address, so by default the
    // deposit keeps the caller's order and only the gather uses the ordering.
    const bool dep_sorted = pos_s && h->dshape.sorted_input;
    cudaError_t err = dep_sorted
                          ? mog::launch_deposit(e, pos_s, nullptr, n, true, h->d_mass, h->dshape, s)
                          : mog::launch_deposit(e, pos, nullptr, n, false, h->d_mass, h->dshape, s);
    if (err != cudaSuccess) return cuda_fail(err, "deposit");
    if (h->cfg.solver == MOG_SOLVER_FFT)
        err = mog::launch_spectral(e, h->d_mass, h->d_force, mog::kFrameWorldSlot, true, h->d_scratch, s, h->solve_split);
    else
        err = mog::launch_convolution(e, h->d_mass, h->d_force, mog::kFrameWorldSlot, true, s);
    if (err != cudaSuccess) return cuda_fail(err, "solve");
    err = mog::launch_update(e, pos, vel, pos_s, perm, n, h->d_force, dt, h->cfg.damping, acc,
                             h->ushape, s);
    if (err != cudaSuccess) return cuda_fail(err, "update");
    return MOG_OK;
}

size_t mass_bytes(const mog_handle* h) {
    return (size_t)h->e.cells() * (h->cfg.mass_mode == MOG_MASS_U64_FIXED ? 8 : 4);
}

void release_shard(mog_handle* h) {
    ShardState& sh = h->shard;
    for (int q = 0; q < mog::kMaxShardRanks; ++q)
        if (sh.ipc[q]) {
            if (sh.view.accum[q]) cudaIpcCloseMemHandle(sh.view.accum[q]);
            if (sh.view.flags_peer[q]) cudaIpcCloseMemHandle(sh.view.flags_peer[q]);
        }
    if (sh.d_accum) cudaFree(sh.d_accum);
    if (sh.d_flags) cudaFree(sh.d_flags);
    if (sh.d_targets) cudaFree(sh.d_targets);
    sh = ShardState();
}

void release(mog_handle* h) {
    release_shard(h);
    for (auto& g : h->graphs)
        if (g.exec) cudaGraphExecDestroy(g.exec);
    h->graphs.clear();
    void* ptrs[] = {h->d_rot12, h->d_off4, h->d_fast, h->d_green, h->d_ktab, h->d_conv,
                    h->d_flags, h->d_total, h->d_mass, h->d_force, h->d_force2, h->d_scratch,
                    h->d_diag, h->d_perm, h->d_sort, h->d_pos_s, h->d_spread, h->d_dft,
                    h->d_hpos, h->d_hvel};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    for (auto* evs : {&h->ev_pos, &h->ev_vel, &h->ev_done})
        for (cudaEvent_t x : *evs)
            if (x) cudaEventDestroy(x);
    if (h->ev_start) cudaEventDestroy(h->ev_start);
    if (h->ev_out) cudaEventDestroy(h->ev_out);
    if (h->s_in) cudaStreamDestroy(h->s_in);
    if (h->s_out) cudaStreamDestroy(h->s_out);
}

}  // namespace

extern "C" {

int mog_config_default(mog_config* c) {
    if (!c) return fail(MOG_ERR_ARG, "cfg is null");
    std::memset(c, 0, sizeof(*c));
    // main.py:179-189 (no config.yaml) and main.py:667 (damping default)
    c->n_grids = 16;
    c->grid_size = 16;
    c->world_size = 100.0f;
    c->G = 1.0f;
    c->dt = 0.00001f;
    c->damping = 1.0f;
    c->solver = MOG_SOLVER_FFT;
    c->mass_mode = MOG_MASS_U64_FIXED;
    c->scale_bits = 32;
    c->index_mode = MOG_INDEX_FAST;
    c->dft_prec = MOG_DFT_FFT32;
    c->num_particles = 100000;
    return MOG_OK;
}

int mog_create(const mog_config* cfg, const float* rot12, const float* off4, mog_handle** out) {
    if (!cfg || !rot12 || !off4 || !out) return fail(MOG_ERR_ARG, "null argument to mog_create");
    *out = nullptr;
    int rc = validate(*cfg);
    if (rc) return rc;
    if (cfg->dft_prec == MOG_DFT_TC_BF16X3 &&
        (cfg->solver != MOG_SOLVER_FFT || (cfg->grid_size != 16 && cfg->grid_size != 32)))
        return fail(MOG_ERR_UNSUPPORTED, "tensor-core DFT precision needs the fft solver and grid_size 16 or 32");
    for (int i = 0; i < cfg->n_grids * 12; ++i)
        if (!std::isfinite(rot12[i])) return fail(MOG_ERR_CONFIG, "rotation entries must be finite");
    for (int i = 0; i < cfg->n_grids * 4; ++i)
        if (!std::isfinite(off4[i])) return fail(MOG_ERR_CONFIG, "offset entries must be finite");

    mog_handle* h = new mog_handle();
    h->cfg = *cfg;
    cudaGetDevice(&h->device);
    const int k = cfg->n_grids, g = cfg->grid_size;
    int lg = 0;
    while ((1 << lg) < g) ++lg;
    mog::Ensemble& e = h->e;
    e.k = k;
    e.g = g;
    e.lg = lg;
    e.mass_mode = cfg->mass_mode;
    e.index_mode = cfg->index_mode;
    e.world = cfg->world_size;
    // voxel = world / grid in double, passed to the shaders as a float
    // uniform (main.py:118, mass.glsl:17)
    e.voxel = (float)((double)cfg->world_size / (double)g);
    e.G = cfg->G;
    e.scale = std::ldexp(1.0f, cfg->scale_bits);
    e.inv_scale = std::ldexp(1.0f, -cfg->scale_bits);
    // the reference's ping-pong leaves the result in its scratch texture
    // after an odd number of passes, 3 (log2 g + 1)
    e.alias_xz = (cfg->compat_flags & MOG_COMPAT_FFT_TEXTURE_ALIAS) && ((3 * (lg + 1)) & 1) ? 1 : 0;
    e.dft_tc = cfg->dft_prec == MOG_DFT_TC_BF16X3 ? 1 : 0;

    // FAST-mode rows: t_r = sum_j (M[j][r] / h) c_j + (L/2 - off_r) / h
    std::vector<mog::FastXf> fast(k);
    const double hv = (double)e.voxel;
    const double half_l = (double)(cfg->world_size * 0.5f);
    for (int i = 0; i < k; ++i) {
        const float* R = rot12 + 12 * i;
        float* rows = reinterpret_cast<float*>(&fast[i]);
        for (int r = 0; r < 3; ++r) {
            for (int j = 0; j < 3; ++j) rows[4 * r + j] = (float)((double)R[4 * j + r] / hv);
            rows[4 * r + 3] = (float)((half_l - (double)off4[4 * i + r]) / hv);
        }
    }
    h->rows.resize(k);
    for (int i = 0; i < k; ++i) h->rows[i] = mog::make_grid_rows(fast[i], rot12 + 12 * i, e.voxel);
    const size_t cells = (size_t)e.cells();
    const size_t g3 = (size_t)g * g * g;
    auto fail_free = [&](cudaError_t err, const char* where) {
        release(h);
        delete h;
        return cuda_fail(err, where);
    };
#define ALLOC(ptr, bytes)                                                     \
    do {                                                                      \
        cudaError_t err__ = cudaMalloc((void**)&(ptr), (bytes));              \
        if (err__ != cudaSuccess) return fail_free(err__, "cudaMalloc " #ptr); \
    } while (0)
    ALLOC(h->d_rot12, sizeof(float) * 12 * k);
    ALLOC(h->d_off4, sizeof(float) * 4 * k);
    ALLOC(h->d_fast, sizeof(mog::FastXf) * k);
    ALLOC(h->d_green, sizeof(float) * g3);
    ALLOC(h->d_ktab, sizeof(float) * g);
    ALLOC(h->d_conv, sizeof(float4) * g3);
    ALLOC(h->d_flags, sizeof(unsigned) * 4);
    ALLOC(h->d_total, sizeof(double) * 2);
    ALLOC(h->d_mass, cells * (cfg->mass_mode == MOG_MASS_U64_FIXED ? 8 : 4));
    ALLOC(h->d_force, sizeof(float4) * cells);
    ALLOC(h->d_diag, sizeof(double) * (kDiagBlocks * 8 + 8));
    std::vector<uint16_t> dft_tab;
    if (e.dft_tc) {
        dft_tab = mog::dft_tc_tables(g);
        ALLOC(h->d_dft, sizeof(uint16_t) * dft_tab.size());
    }
    const size_t scratch = mog::spectral_scratch_bytes(e);
    if (scratch) ALLOC(h->d_scratch, scratch);
    // spatial-order buffers for the declared capacity (no allocation may
    // happen later inside a captured step)
    if (cfg->num_particles > 0) {
        ALLOC(h->d_perm, sizeof(int) * cfg->num_particles);
        ALLOC(h->d_pos_s, sizeof(float4) * cfg->num_particles);
        h->perm_cap = cfg->num_particles;
    }
    ALLOC(h->d_sort, mog::sort_scratch_bytes());
    // room for the CTAs of a whole learned step even when the host-buffer
    // step launches its kernel once per chunk
    h->spread_cap = mog::num_sms() * 32;
    ALLOC(h->d_spread, sizeof(float) * 2 * h->spread_cap);
#undef ALLOC
    cudaError_t err;
    std::vector<float> convk = conv_kernel_table(g, hv);
    if ((err = cudaMemcpy(h->d_rot12, rot12, sizeof(float) * 12 * k, cudaMemcpyHostToDevice)) ||
        (err = cudaMemcpy(h->d_off4, off4, sizeof(float) * 4 * k, cudaMemcpyHostToDevice)) ||
        (err = cudaMemcpy(h->d_fast, fast.data(), sizeof(mog::FastXf) * k, cudaMemcpyHostToDevice)) ||
        (err = cudaMemcpy(h->d_conv, convk.data(), sizeof(float) * convk.size(), cudaMemcpyHostToDevice)) ||
        (err = cudaMemset(h->d_flags, 0, sizeof(unsigned) * 4)) ||
        (err = cudaMemset(h->d_total, 0, sizeof(double) * 2)) ||
        (err = cudaMemset(h->d_mass, 0, mass_bytes(h))) ||
        (e.dft_tc && (err = cudaMemcpy(h->d_dft, dft_tab.data(), sizeof(uint16_t) * dft_tab.size(),
                                       cudaMemcpyHostToDevice))))
        return fail_free(err, "mog_create upload");
    e.dft_tables = h->d_dft;
    e.rot12 = h->d_rot12;
    e.off4 = h->d_off4;
    e.fast = h->d_fast;
    e.green = h->d_green;
    e.ktab = h->d_ktab;
    e.conv_kernel = h->d_conv;
    e.flags = h->d_flags;
    e.mass_total = h->d_total;
    if ((err = mog::launch_build_tables(g, cfg->world_size, cfg->G, h->d_green, h->d_ktab, 0)) ||
        (err = cudaDeviceSynchronize()))
        return fail_free(err, "Green's table build");
    if (cfg->softening > 0.f) {
        // the softened variant's factors, built on the host in FP64
        const std::vector<float> gt = green_table(g, cfg->world_size, cfg->G, cfg->softening);
        if ((err = cudaMemcpy(h->d_green, gt.data(), sizeof(float) * gt.size(), cudaMemcpyHostToDevice)))
            return fail_free(err, "softened Green's table upload");
    }
    *out = h;
    return MOG_OK;
}

int mog_destroy(mog_handle* h) {
    if (!h) return MOG_OK;
    set_device(h);
    release(h);
    delete h;
    return MOG_OK;
}

int mog_step(mog_handle* h, float* pos4, float* vel4, int64_t n, float dt_eff, void* stream) {
    if (!h) return fail(MOG_ERR_ARG, "handle is null");
    int rc = check_particles(h, pos4, vel4, n, true);
    if (rc) return rc;
    if (!std::isfinite(dt_eff)) return fail(MOG_ERR_ARG, "dt_eff must be finite");
    if ((rc = set_device(h))) return rc;
    rc = run_pipeline(h, reinterpret_cast<float4*>(pos4), reinterpret_cast<float4*>(vel4), n,
                      dt_eff, nullptr, static_cast<cudaStream_t>(stream), wants_sort(h, n));
    if (!rc) ++h->step_count;
    return rc;
}

int mog_step_n(mog_handle* h, float* pos4, float* vel4, int64_t n, float dt_eff, int32_t n_steps,
               void* stream) {
    if (!h) return fail(MOG_ERR_ARG, "handle is null");
    int rc = check_particles(h, pos4, vel4, n, true);
    if (rc) return rc;
    if (n_steps < 0) return fail(MOG_ERR_ARG, "n_steps must be >= 0");
    if (!std::isfinite(dt_eff)) return fail(MOG_ERR_ARG, "dt_eff must be finite");
    if ((rc = set_device(h))) return rc;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (n_steps == 0 || n == 0) return MOG_OK;
    // The legacy default stream cannot be captured: run the steps directly.
    if (s == nullptr || s == cudaStreamLegacy) {
        for (int i = 0; i < n_steps; ++i) {
            if ((rc = run_pipeline(h, reinterpret_cast<float4*>(pos4),
                                   reinterpret_cast<float4*>(vel4), n, dt_eff, nullptr, s,
                                   wants_sort(h, n))))
                return rc;
            ++h->step_count;
        }
        return MOG_OK;
    }
    for (int i = 0; i < n_steps; ++i) {
        // Two graphs per particle set: with and without the re-ordering.
        const bool sorts = wants_sort(h, n);
        if (h->perm_n != n && h->sort_every > 0 && !sorts) return fail(MOG_ERR_ARG, "internal: no order");
        GraphEntry* ge = nullptr;
        for (auto& g : h->graphs)
            if (g.pos == pos4 && g.vel == vel4 && g.n == n && g.dt == dt_eff && g.sorts == sorts)
                ge = &g;
        if (!ge) {
            cudaGraph_t graph = nullptr;
            MOG_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal), "begin capture");
            rc = run_pipeline(h, reinterpret_cast<float4*>(pos4), reinterpret_cast<float4*>(vel4), n,
                              dt_eff, nullptr, s, sorts);
            cudaError_t end = cudaStreamEndCapture(s, &graph);
            if (rc) {
                if (graph) cudaGraphDestroy(graph);
                return rc;
            }
            if (end != cudaSuccess) return cuda_fail(end, "end capture");
            GraphEntry entry;
            entry.pos = pos4;
            entry.vel = vel4;
            entry.n = n;
            entry.dt = dt_eff;
            entry.sorts = sorts;
            cudaError_t err = cudaGraphInstantiate(&entry.exec, graph, 0);
            cudaGraphDestroy(graph);
            if (err != cudaSuccess) return cuda_fail(err, "graph instantiate");
            if (h->graphs.size() >= 8) {
                cudaGraphExecDestroy(h->graphs.front().exec);
                h->graphs.erase(h->graphs.begin());
            }
            h->graphs.push_back(entry);
            ge = &h->graphs.back();
        }
        MOG_CUDA(cudaGraphLaunch(ge->exec, s), "graph launch");
        ++h->step_count;
    }
    return MOG_OK;
}

int mog_step_profiled(mog_handle* h, float* pos4, float* vel4, int64_t n, float dt_eff,
                      float* phase_ms, void* stream) {
    if (!h || !phase_ms) return fail(MOG_ERR_ARG, "null argument");
    int rc = check_particles(h, pos4, vel4, n, true);
    if (rc) return rc;
    if (!std::isfinite(dt_eff)) return fail(MOG_ERR_ARG, "dt_eff must be finite");
    if ((rc = set_device(h))) return rc;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    cudaEvent_t ev[5];
    for (auto& e : ev) MOG_CUDA(cudaEventCreate(&e), "event create");
    const mog::Ensemble& e = h->e;
    float4* pos = reinterpret_cast<float4*>(pos4);
    float4* vel = reinterpret_cast<float4*>(vel4);
    const int* perm = nullptr;
    const float4* pos_s = nullptr;
    cudaError_t err = cudaEventRecord(ev[0], s);
    if (!err) {
        rc = order_particles(h, pos, n, wants_sort(h, n), s, &perm, &pos_s);
        if (rc) {
            for (auto& x : ev) cudaEventDestroy(x);
            return rc;
        }
    }
    if (!err) err = cudaEventRecord(ev[1], s);
    if (!err)
        err = (pos_s && h->dshape.sorted_input)
                  ? mog::launch_deposit(e, pos_s, nullptr, n, true, h->d_mass, h->dshape, s)
                  : mog::launch_deposit(e, pos, nullptr, n, false, h->d_mass, h->dshape, s);
    if (!err) err = cudaEventRecord(ev[2], s);
    if (!err)
        err = h->cfg.solver == MOG_SOLVER_FFT
                  ? mog::launch_spectral(e, h->d_mass, h->d_force, mog::kFrameWorldSlot, true, h->d_scratch, s, h->solve_split)
                  : mog::launch_convolution(e, h->d_mass, h->d_force, mog::kFrameWorldSlot, true, s);
    if (!err) err = cudaEventRecord(ev[3], s);
    if (!err)
        err = mog::launch_update(e, pos, vel, pos_s, perm, n, h->d_force, dt_eff, h->cfg.damping,
                                 nullptr, h->ushape, s);
    if (!err) err = cudaEventRecord(ev[4], s);
    if (!err) err = cudaEventSynchronize(ev[4]);
    for (int i = 0; i < 4 && !err; ++i) err = cudaEventElapsedTime(&phase_ms[i], ev[i], ev[i + 1]);
    for (auto& x : ev) cudaEventDestroy(x);
    if (err) return cuda_fail(err, "profiled step");
    ++h->step_count;
    return MOG_OK;
}

int mog_forces(mog_handle* h, const float* pos4, float* acc4, int64_t n, void* stream) {
    if (!h) return fail(MOG_ERR_ARG, "handle is null");
    int rc = check_particles(h, pos4, acc4, n, true);
    if (rc) return rc;
    if ((rc = set_device(h))) return rc;
    return run_pipeline(h, const_cast<float4*>(reinterpret_cast<const float4*>(pos4)), nullptr, n,
                        0.f, reinterpret_cast<float4*>(acc4), static_cast<cudaStream_t>(stream),
                        h->sort_every > 0);
}

int mog_deposit(mog_handle* h, const float* pos4, int64_t n, void* mass_out, void* stream) {
    if (!h) return fail(MOG_ERR_ARG, "handle is null");
    int rc = check_particles(h, pos4, nullptr, n, false);
    if (rc) return rc;
    if (!mass_out) return fail(MOG_ERR_ARG, "mass_out is null");
    if ((rc = set_device(h))) return rc;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    MOG_CUDA(cudaMemsetAsync(mass_out, 0, mass_bytes(h), s), "clear mass");
    const int* perm = nullptr;
    const float4* pos_s = nullptr;
    if ((rc = order_particles(h, reinterpret_cast<const float4*>(pos4), n, h->sort_every > 0, s,
                              &perm, &pos_s)))
        return rc;
    cudaError_t err =
        (pos_s && h->dshape.sorted_input)
            ? mog::launch_deposit(h->e, pos_s, nullptr, n, true, mass_out, h->dshape, s)
            : mog::launch_deposit(h->e, reinterpret_cast<const float4*>(pos4), nullptr, n, false,
                                  mass_out, h->dshape, s);
    if (err != cudaSuccess) return cuda_fail(err, "deposit");
    mog::check_total_kernel<<<1, 1, 0, s>>>(h->e);
    MOG_CUDA(cudaGetLastError(), "check total");
    return MOG_OK;
}

int mog_solve(mog_handle* h, const void* mass_in, float* force4_out, void* stream) {
    if (!h) return fail(MOG_ERR_ARG, "handle is null");
    if (!mass_in || !force4_out) return fail(MOG_ERR_ARG, "null buffer");
    if ((uintptr_t)force4_out & 15) return fail(MOG_ERR_ARG, "force4_out must be 16-byte aligned");
    int rc = set_device(h);
    if (rc) return rc;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    cudaError_t err;
    if (h->cfg.solver == MOG_SOLVER_FFT)
        err = mog::launch_spectral(h->e, const_cast<void*>(mass_in),
                                   reinterpret_cast<float4*>(force4_out), mog::kFrameGrid, false,
                                   h->d_scratch, s, h->solve_split);
    else
        err = mog::launch_convolution(h->e, const_cast<void*>(mass_in),
                                      reinterpret_cast<float4*>(force4_out), mog::kFrameGrid, false, s);
    if (err != cudaSuccess) return cuda_fail(err, "solve");
    return MOG_OK;
}

int mog_update(mog_handle* h, float* pos4, float* vel4, int64_t n, const float* force4_in,
               float dt_eff, void* stream) {
    if (!h) return fail(MOG_ERR_ARG, "handle is null");
    int rc = check_particles(h, pos4, vel4, n, true);
    if (rc) return rc;
    if (!force4_in) return fail(MOG_ERR_ARG, "force4_in is null");
    if ((rc = set_device(h))) return rc;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (!h->d_force2) MOG_CUDA(cudaMalloc((void**)&h->d_force2, sizeof(float4) * h->e.cells()), "cudaMalloc force2");
    cudaError_t err = mog::launch_prerotate(h->e, reinterpret_cast<const float4*>(force4_in), h->d_force2, s);
    if (err != cudaSuccess) return cuda_fail(err, "prerotate");
    const int* perm = nullptr;
    const float4* pos_s = nullptr;
    if ((rc = order_particles(h, reinterpret_cast<const float4*>(pos4), n, h->sort_every > 0, s,
                              &perm, &pos_s)))
        return rc;
    err = mog::launch_update(h->e, reinterpret_cast<float4*>(pos4), reinterpret_cast<float4*>(vel4),
                             pos_s, perm, n, h->d_force2, dt_eff, h->cfg.damping, nullptr, h->ushape, s);
    if (err != cudaSuccess) return cuda_fail(err, "update");
    return MOG_OK;
}

int mog_get_tuning(const mog_handle* h, mog_tuning* out) {
    if (!h || !out) return fail(MOG_ERR_ARG, "null argument");
    std::memset(out, 0, sizeof(*out));
    out->deposit_threads = h->dshape.threads;
    out->deposit_grids_per_cta = h->dshape.grids_per_cta;
    out->deposit_chunks = h->dshape.chunks;
    out->deposit_ppt = h->dshape.ppt;
    out->update_staged = h->ushape.staged;
    out->update_ctas = h->ushape.ctas;
    out->sort_every = h->sort_every;
    out->deposit_aggregate = h->dshape.aggregate;
    out->deposit_generic = h->dshape.fast ? 0 : 1;
    out->deposit_sorted = h->dshape.sorted_input;
    out->update_threads = h->ushape.threads;
    out->update_direct_ppt = h->ushape.direct_ppt;
    out->deposit_split = h->dshape.split;
    out->learned_fold = h->learned_fold ? 1 : -1;
    out->learned_ctas_per_sm = h->learned_ctas;
    out->solve_split = h->solve_split;
    return MOG_OK;
}

int mog_set_tuning(mog_handle* h, const mog_tuning* t) {
    if (!h || !t) return fail(MOG_ERR_ARG, "null argument");
    if (t->deposit_threads && (t->deposit_threads < 64 || t->deposit_threads > 1024 ||
                               t->deposit_threads % 32))
        return fail(MOG_ERR_ARG, "deposit_threads must be a multiple of 32 in [64, 1024]");
    if (t->deposit_grids_per_cta < -1 || t->deposit_chunks < 0 || t->update_ctas < 0 ||
        t->update_staged < -1 || t->update_staged > 1 ||
        (t->deposit_ppt != 0 && t->deposit_ppt != 1 && t->deposit_ppt != 2 && t->deposit_ppt != 4) ||
        t->sort_every < -1 || t->deposit_aggregate < -1 || t->deposit_aggregate > 1 ||
        (t->update_threads != 0 && t->update_threads != 512 && t->update_threads != 768 &&
         t->update_threads != 1024) ||
        (t->update_direct_ppt != 0 && t->update_direct_ppt != 1 && t->update_direct_ppt != 2 &&
         t->update_direct_ppt != 4) ||
        t->deposit_split < -1 || t->deposit_split > 2 || t->learned_fold < -1 ||
        t->learned_fold > 1 ||
        (t->learned_ctas_per_sm != 0 && t->learned_ctas_per_sm != 2 && t->learned_ctas_per_sm != 3) ||
        t->solve_split < -1 || t->solve_split > 1)
        return fail(MOG_ERR_ARG, "tuning value out of range");
    h->dshape.threads = t->deposit_threads ? t->deposit_threads : 1024;
    h->dshape.grids_per_cta = t->deposit_grids_per_cta;
    h->dshape.chunks = t->deposit_chunks;
    h->dshape.ppt = t->deposit_ppt ? t->deposit_ppt : 4;
    h->ushape.staged = t->update_staged;
    h->ushape.ctas = t->update_ctas;
    h->ushape.direct_ppt = t->update_direct_ppt;
    h->sort_every = t->sort_every < 0 ? 0 : t->sort_every;
    h->dshape.aggregate = t->deposit_aggregate;
    h->dshape.fast = t->deposit_generic ? 0 : 1;
    h->dshape.sorted_input = t->deposit_sorted ? 1 : 0;
    h->ushape.threads = t->update_threads;
    h->dshape.split = t->deposit_split;
    h->learned_fold = t->learned_fold >= 0 ? 1 : 0;
    h->learned_ctas = t->learned_ctas_per_sm ? t->learned_ctas_per_sm : 2;
    h->solve_split = t->solve_split;
    for (auto& g : h->graphs)
        if (g.exec) cudaGraphExecDestroy(g.exec);
    h->graphs.clear();
    return MOG_OK;
}

int mog_get_status(mog_handle* h, uint32_t* flags, void* stream) {
    if (!h || !flags) return fail(MOG_ERR_ARG, "null argument");
    int rc = set_device(h);
    if (rc) return rc;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    unsigned v = 0;
    MOG_CUDA(cudaMemcpyAsync(&v, h->d_flags, sizeof(unsigned), cudaMemcpyDeviceToHost, s), "read flags");
    MOG_CUDA(cudaMemsetAsync(h->d_flags, 0, sizeof(unsigned), s), "clear flags");
    MOG_CUDA(cudaStreamSynchronize(s), "sync");
    *flags = v;
    return MOG_OK;
}

// The deposit's per-slot target tables, from the connected view.
static int upload_targets(mog_handle* h) {
    ShardState& sh = h->shard;
    mog::ShardTargets t[3];
    for (int slot = 0; slot < 3; ++slot) {
        for (int q = 0; q < mog::kMaxShardRanks; ++q)
            t[slot].base[q] = q < sh.world ? static_cast<char*>(sh.view.accum[q]) + (size_t)slot * mass_bytes(h)
                                           : nullptr;
        t[slot].world = sh.world;
    }
    MOG_CUDA(cudaMemcpy(sh.d_targets, t, sizeof t, cudaMemcpyHostToDevice), "shard targets upload");
    sh.connected = true;
    return MOG_OK;
}

int mog_shard_init(mog_handle* h, int32_t rank, int32_t world) {
    if (!h) return fail(MOG_ERR_ARG, "null handle");
    if (world < 1 || world > mog::kMaxShardRanks)
        return fail(MOG_ERR_ARG, "world must be 1..8");
    if (rank < 0 || rank >= world) return fail(MOG_ERR_ARG, "rank must be in [0, world)");
    int rc = set_device(h);
    if (rc) return rc;
    release_shard(h);
    ShardState& sh = h->shard;
    const size_t bytes = 3 * mass_bytes(h);
    MOG_CUDA(cudaMalloc(&sh.d_accum, bytes), "cudaMalloc shard accumulation");
    MOG_CUDA(cudaMalloc((void**)&sh.d_flags, sizeof(uint64_t) * world), "cudaMalloc shard flags");
    MOG_CUDA(cudaMalloc((void**)&sh.d_targets, sizeof(mog::ShardTargets) * 3), "cudaMalloc shard targets");
    MOG_CUDA(cudaMemset(sh.d_accum, 0, bytes), "clear shard accumulation");
    MOG_CUDA(cudaMemset(sh.d_flags, 0, sizeof(uint64_t) * world), "clear shard flags");
    MOG_CUDA(cudaDeviceSynchronize(), "shard init");
    sh.rank = rank;
    sh.world = world;
    return MOG_OK;
}

int mog_shard_export(const mog_handle* h, uint8_t* accum_ipc, uint8_t* flags_ipc) {
    if (!h || !accum_ipc || !flags_ipc) return fail(MOG_ERR_ARG, "null argument");
    if (!h->shard.world) return fail(MOG_ERR_ARG, "mog_shard_init first");
    static_assert(sizeof(cudaIpcMemHandle_t) == 64, "IPC handles are 64 bytes");
    cudaIpcMemHandle_t a, f;
    MOG_CUDA(cudaIpcGetMemHandle(&a, h->shard.d_accum), "cudaIpcGetMemHandle");
    MOG_CUDA(cudaIpcGetMemHandle(&f, h->shard.d_flags), "cudaIpcGetMemHandle");
    std::memcpy(accum_ipc, &a, 64);
    std::memcpy(flags_ipc, &f, 64);
    return MOG_OK;
}

int mog_shard_connect(mog_handle* h, const uint8_t* accum_ipcs, const uint8_t* flags_ipcs) {
    if (!h || !accum_ipcs || !flags_ipcs) return fail(MOG_ERR_ARG, "null argument");
    ShardState& sh = h->shard;
    if (!sh.world) return fail(MOG_ERR_ARG, "mog_shard_init first");
    if (sh.connected) return fail(MOG_ERR_ARG, "already connected");
    int rc = set_device(h);
    if (rc) return rc;
    for (int q = 0; q < sh.world; ++q) {
        if (q == sh.rank) {
            sh.view.accum[q] = sh.d_accum;
            sh.view.flags_peer[q] = sh.d_flags;
            continue;
        }
        cudaIpcMemHandle_t a, f;
        std::memcpy(&a, accum_ipcs + 64 * q, 64);
        std::memcpy(&f, flags_ipcs + 64 * q, 64);
        void *pa = nullptr, *pf = nullptr;
        cudaError_t err = cudaIpcOpenMemHandle(&pa, a, cudaIpcMemLazyEnablePeerAccess);
        if (err == cudaSuccess) {
            err = cudaIpcOpenMemHandle(&pf, f, cudaIpcMemLazyEnablePeerAccess);
            if (err != cudaSuccess) cudaIpcCloseMemHandle(pa);
        }
        if (err != cudaSuccess) {
            release_shard(h);
            return cuda_fail(err, "cudaIpcOpenMemHandle (peer buffers)");
        }
        sh.view.accum[q] = pa;
        sh.view.flags_peer[q] = static_cast<uint64_t*>(pf);
        sh.ipc[q] = true;
    }
    sh.view.flags_local = sh.d_flags;
    sh.view.rank = sh.rank;
    sh.view.world = sh.world;
    return upload_targets(h);
}

int mog_shard_connect_local(mog_handle* h, mog_handle* const* peers) {
    if (!h || !peers) return fail(MOG_ERR_ARG, "null argument");
    ShardState& sh = h->shard;
    if (!sh.world) return fail(MOG_ERR_ARG, "mog_shard_init first");
    if (sh.connected) return fail(MOG_ERR_ARG, "already connected");
    int rc = set_device(h);
    if (rc) return rc;
    for (int q = 0; q < sh.world; ++q) {
        const mog_handle* p = peers[q];
        if (!p || p->shard.world != sh.world || p->shard.rank != q)
            return fail(MOG_ERR_ARG, "peers[q] must be rank q of the same world (mog_shard_init)");
        if (p->cfg.n_grids != h->cfg.n_grids || p->cfg.grid_size != h->cfg.grid_size ||
            p->cfg.mass_mode != h->cfg.mass_mode)
            return fail(MOG_ERR_ARG, "every rank needs the same n_grids, grid_size and mass_mode");
        if (q == sh.rank && p != h) return fail(MOG_ERR_ARG, "peers[rank] must be this handle");
        if (p->device != h->device) {
            int can = 0;
            MOG_CUDA(cudaDeviceCanAccessPeer(&can, h->device, p->device), "cudaDeviceCanAccessPeer");
            if (!can) return fail(MOG_ERR_UNSUPPORTED, "no peer access between the ranks' devices");
            cudaError_t err = cudaDeviceEnablePeerAccess(p->device, 0);
            if (err == cudaErrorPeerAccessAlreadyEnabled)
                cudaGetLastError();
            else if (err != cudaSuccess)
                return cuda_fail(err, "cudaDeviceEnablePeerAccess");
        }
        sh.view.accum[q] = p->shard.d_accum;
        sh.view.flags_peer[q] = p->shard.d_flags;
    }
    sh.view.flags_local = sh.d_flags;
    sh.view.rank = sh.rank;
    sh.view.world = sh.world;
    return upload_targets(h);
}

int mog_shard_deposit(mog_handle* h, const float* pos4, int64_t n, void* stream) {
    if (!h) return fail(MOG_ERR_ARG, "null handle");
    ShardState& sh = h->shard;
    if (!sh.connected) return fail(MOG_ERR_ARG, "connect the shard first");
    int rc = check_particles(h, pos4, nullptr, n, false);
    if (rc) return rc;
    if ((rc = set_device(h))) return rc;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const uint64_t epoch = sh.epoch + 1;
    const int slot = (int)(epoch % 3);
    MOG_CUDA(mog::launch_deposit(h->e, reinterpret_cast<const float4*>(pos4), nullptr, n, false,
                                 sh.d_targets + slot, h->dshape, s, true),
             "sharded deposit");
    MOG_CUDA(mog::launch_shard_signal(sh.view, epoch, s), "shard signal");
    sh.epoch = epoch;
    return MOG_OK;
}

int mog_shard_exchange(mog_handle* h, void* stream) {
    if (!h) return fail(MOG_ERR_ARG, "null handle");
    ShardState& sh = h->shard;
    if (!sh.connected || sh.epoch == 0) return fail(MOG_ERR_ARG, "mog_shard_deposit first");
    int rc = set_device(h);
    if (rc) return rc;
    MOG_CUDA(mog::launch_shard_exchange(h->e, sh.view, sh.epoch, (int)(sh.epoch % 3), h->d_mass,
                                        static_cast<cudaStream_t>(stream)),
             "shard exchange");
    return MOG_OK;
}

int mog_shard_finish(mog_handle* h, float* pos4, float* vel4, int64_t n, float dt_eff,
                     void* stream) {
    if (!h) return fail(MOG_ERR_ARG, "null handle");
    if (!h->shard.connected) return fail(MOG_ERR_ARG, "connect the shard first");
    int rc = check_particles(h, pos4, vel4, n, true);
    if (rc) return rc;
    if (!std::isfinite(dt_eff)) return fail(MOG_ERR_ARG, "dt_eff must be finite");
    if ((rc = set_device(h))) return rc;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    float4* pos = reinterpret_cast<float4*>(pos4);
    const int* perm = nullptr;
    const float4* pos_s = nullptr;
    if ((rc = order_particles(h, pos, n, wants_sort(h, n), s, &perm, &pos_s))) return rc;
    const mog::Ensemble& e = h->e;
    cudaError_t err = h->cfg.solver == MOG_SOLVER_FFT
                          ? mog::launch_spectral(e, h->d_mass, h->d_force, mog::kFrameWorldSlot, true, h->d_scratch, s, h->solve_split)
                          : mog::launch_convolution(e, h->d_mass, h->d_force, mog::kFrameWorldSlot, true, s);
    if (err != cudaSuccess) return cuda_fail(err, "solve");
    err = mog::launch_update(e, pos, reinterpret_cast<float4*>(vel4), pos_s, perm, n, h->d_force,
                             dt_eff, h->cfg.damping, nullptr, h->ushape, s);
    if (err != cudaSuccess) return cuda_fail(err, "update");
    ++h->step_count;
    return MOG_OK;
}

int mog_shard_step(mog_handle* h, float* pos4, float* vel4, int64_t n, float dt_eff, void* stream) {
    int rc = mog_shard_deposit(h, pos4, n, stream);
    if (!rc) rc = mog_shard_exchange(h, stream);
    if (!rc) rc = mog_shard_finish(h, pos4, vel4, n, dt_eff, stream);
    return rc;
}

int mog_selftest_wait_timeout(mog_handle* h, void* stream) {
    if (!h) return fail(MOG_ERR_ARG, "null argument");
    int rc = set_device(h);
    if (rc) return rc;
    MOG_CUDA(mog::launch_wait_timeout_selftest(h->d_flags, static_cast<cudaStream_t>(stream)),
             "wait self-test");
    return MOG_OK;
}

int mog_diagnostics(mog_handle* h, const float* pos4, const float* vel4, int64_t n, double* out8,
                    void* stream) {
    if (!h || !out8) return fail(MOG_ERR_ARG, "null argument");
    int rc = check_particles(h, pos4, vel4, n, true);
    if (rc) return rc;
    if ((rc = set_device(h))) return rc;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    double* res = h->d_diag + kDiagBlocks * 8;
    cudaError_t err = mog::launch_diagnostics(reinterpret_cast<const float4*>(pos4),
                                              reinterpret_cast<const float4*>(vel4), n, h->d_diag,
                                              kDiagBlocks, res, s);
    if (err != cudaSuccess) return cuda_fail(err, "diagnostics");
    MOG_CUDA(cudaMemcpyAsync(out8, res, 8 * sizeof(double), cudaMemcpyDeviceToHost, s), "read diagnostics");
    MOG_CUDA(cudaStreamSynchronize(s), "sync");
    return MOG_OK;
}

int mog_direct_sum(const float* targets4, int64_t nt, const float* sources4, int64_t ns,
                   double world, double g_eff, double soft, double* out3, void* stream) {
    if (nt < 0 || ns < 0) return fail(MOG_ERR_ARG, "negative size");
    if ((nt && (!targets4 || !out3)) || (ns && !sources4)) return fail(MOG_ERR_ARG, "null buffer");
    if (!(world > 0.0) || !std::isfinite(g_eff) || !(soft >= 0.0))
        return fail(MOG_ERR_ARG, "world must be positive, g_eff finite, soft >= 0");
    if (nt == 0) return MOG_OK;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int chunks = (int)std::max<int64_t>(1, std::min<int64_t>(32, (ns + 8191) / 8192));
    double* partial = nullptr;
    MOG_CUDA(cudaMallocAsync((void**)&partial, sizeof(double) * 3 * nt * chunks, s), "alloc partial");
    cudaError_t err = mog::launch_direct_sum(reinterpret_cast<const float4*>(targets4), nt,
                                             reinterpret_cast<const float4*>(sources4), ns, world,
                                             g_eff, soft, partial, chunks, out3, s);
    cudaFreeAsync(partial, s);
    if (err != cudaSuccess) return cuda_fail(err, "direct sum");
    return MOG_OK;
}

int mog_direct_sum_noalloc(const float* targets4, int64_t nt, const float* sources4, int64_t ns,
                           double world, double g_eff, double soft, double* out3, void* stream) {
    if (nt < 0 || ns < 0) return fail(MOG_ERR_ARG, "negative size");
    if ((nt && (!targets4 || !out3)) || (ns && !sources4)) return fail(MOG_ERR_ARG, "null buffer");
    if (!(world > 0.0) || !std::isfinite(g_eff) || !(soft >= 0.0))
        return fail(MOG_ERR_ARG, "world must be positive, g_eff finite, soft >= 0");
    if (nt == 0) return MOG_OK;
    // same source chunking as mog_direct_sum, so the two agree bit for bit
    const int chunks = (int)std::max<int64_t>(1, std::min<int64_t>(32, (ns + 8191) / 8192));
    if (nt > mog::kDirectScratchPairs / chunks)
        return fail(MOG_ERR_ARG, "mog_direct_sum_noalloc: " + std::to_string(nt) + " targets x " +
                                     std::to_string(chunks) + " source chunks exceeds the fixed scratch of " +
                                     std::to_string(mog::kDirectScratchPairs) +
                                     " target-chunk pairs (at most " +
                                     std::to_string(mog::kDirectScratchPairs / chunks) +
                                     " targets for this source count)");
    double* partial = nullptr;
    cudaError_t err = mog::direct_sum_scratch(&partial);
    if (err != cudaSuccess) return cuda_fail(err, "direct-sum scratch address");
    err = mog::launch_direct_sum(reinterpret_cast<const float4*>(targets4), nt,
                                 reinterpret_cast<const float4*>(sources4), ns, world, g_eff, soft,
                                 partial, chunks, out3, static_cast<cudaStream_t>(stream));
    if (err != cudaSuccess) return cuda_fail(err, "direct sum");
    return MOG_OK;
}

int mog_green_table(int32_t g, float world, float G, float softening, float* out) {
    if (!out) return fail(MOG_ERR_ARG, "out is null");
    if (!is_pow2(g) || g < 2 || g > 64) return fail(MOG_ERR_ARG, "g must be a power of two in [2, 64]");
    if (!(std::isfinite(world) && world > 0.f) || !std::isfinite(G) ||
        !(std::isfinite(softening) && softening >= 0.f))
        return fail(MOG_ERR_ARG, "world must be positive, G finite, softening >= 0");
    const std::vector<float> t = green_table(g, world, G, softening);
    std::memcpy(out, t.data(), sizeof(float) * t.size());
    return MOG_OK;
}

const char* mog_strerror(int code) {
    switch (code) {
        case MOG_OK: return "ok";
        case MOG_ERR_CONFIG: return "invalid configuration";
        case MOG_ERR_CUDA: return "CUDA error";
        case MOG_ERR_OVERFLOW: return "fixed-point mass overflow";
        case MOG_ERR_NONFINITE: return "non-finite particle state";
        case MOG_ERR_TIMEOUT: return "bounded device wait timed out";
        case MOG_ERR_ARG: return "invalid argument";
        case MOG_ERR_UNSUPPORTED: return "unsupported configuration";
        default: return "unknown status";
    }
}

const char* mog_last_error(void) { return g_last_error.c_str(); }

const char* mog_version(void) { return "mog-b200 0.1 (sm_100a)"; }

}  // extern "C"

// ---- learned correction ---------------------------------------------------

// Deposit + world-frame solve with the handle's ensemble, then the cell
// masses into the force grid's .w lane (the mass grid is cleared for the
// next deposit), then the learned kernel, which gathers everything from
// that grid.  ev (optional): 5 events recorded around the deposit, the
// solve, the cell-mass pass and the learned kernel.
static int run_learned(mog_handle* h, const mog_model* m, int out_mode, float* pos4, float* vel4,
                       int64_t n, float dt, float4* out4, float* feat, cudaStream_t s,
                       cudaEvent_t* ev = nullptr) {
    const mog::Ensemble& e = h->e;
    const float4* pos = reinterpret_cast<const float4*>(pos4);
    cudaError_t err = ev ? cudaEventRecord(ev[0], s) : cudaSuccess;
    if (!err) err = mog::launch_deposit(e, pos, nullptr, n, false, h->d_mass, h->dshape, s);
    if (err != cudaSuccess) return cuda_fail(err, "deposit");
    if (ev && (err = cudaEventRecord(ev[1], s))) return cuda_fail(err, "event");
    if (h->cfg.solver == MOG_SOLVER_FFT && h->learned_fold) {
        // the solve's epilogue leaves the cell masses in the force grid's .w
        // (a separate pass where the fused kernel does not apply)
        err = mog::launch_spectral_density(e, h->d_mass, h->d_force, h->d_scratch, s, h->solve_split);
        if (err != cudaSuccess) return cuda_fail(err, "solve");
        if (ev && (err = cudaEventRecord(ev[2], s))) return cuda_fail(err, "event");
    } else {
        if (h->cfg.solver == MOG_SOLVER_FFT)
            err = mog::launch_spectral(e, h->d_mass, h->d_force, mog::kFrameWorld, false, h->d_scratch, s, h->solve_split);
        else
            err = mog::launch_convolution(e, h->d_mass, h->d_force, mog::kFrameWorld, false, s);
        if (err != cudaSuccess) return cuda_fail(err, "solve");
        if (ev && (err = cudaEventRecord(ev[2], s))) return cuda_fail(err, "event");
        err = mog::launch_density_w(e, h->d_mass, h->d_force, s);
        if (err != cudaSuccess) return cuda_fail(err, "cell masses");
    }
    if (ev && (err = cudaEventRecord(ev[3], s))) return cuda_fail(err, "event");
    mog::LearnedOut out;
    out.out4 = out4;
    out.feat = feat;
    if (out_mode == 0) {
        out.spread = h->d_spread;
        out.spread_cap = h->spread_cap;
    }
    err = mog::launch_learned(out_mode, e, h->rows.data(), reinterpret_cast<float4*>(pos4),
                              reinterpret_cast<float4*>(vel4), n, h->d_force, m->norm, m->d_frags,
                              m->d_params, dt, h->cfg.damping, out, s, h->learned_ctas);
    if (err != cudaSuccess) return cuda_fail(err, "learned kernel");
    if (ev && (err = cudaEventRecord(ev[4], s))) return cuda_fail(err, "event");
    if (out_mode == 0) {
        h->spread_blocks = out.blocks;
        h->spread_n = n;
    }
    return MOG_OK;
}

// Device copies, streams and per-chunk events of the host-buffer steps.
static int ensure_host_step(mog_handle* h, int64_t n, int chunks) {
    if (n > h->host_cap) {
        if (h->d_hpos) cudaFree(h->d_hpos);
        if (h->d_hvel) cudaFree(h->d_hvel);
        h->d_hpos = h->d_hvel = nullptr;
        h->host_cap = 0;
        MOG_CUDA(cudaMalloc((void**)&h->d_hpos, sizeof(float4) * n), "host step buffers");
        MOG_CUDA(cudaMalloc((void**)&h->d_hvel, sizeof(float4) * n), "host step buffers");
        h->host_cap = n;
    }
    if (!h->s_in) {
        MOG_CUDA(cudaStreamCreateWithFlags(&h->s_in, cudaStreamNonBlocking), "copy stream");
        MOG_CUDA(cudaStreamCreateWithFlags(&h->s_out, cudaStreamNonBlocking), "copy stream");
        MOG_CUDA(cudaEventCreateWithFlags(&h->ev_start, cudaEventDisableTiming), "event");
        MOG_CUDA(cudaEventCreateWithFlags(&h->ev_out, cudaEventDisableTiming), "event");
    }
    while ((int)h->ev_done.size() < chunks) {
        cudaEvent_t a, b, c;
        MOG_CUDA(cudaEventCreateWithFlags(&a, cudaEventDisableTiming), "event");
        MOG_CUDA(cudaEventCreateWithFlags(&b, cudaEventDisableTiming), "event");
        MOG_CUDA(cudaEventCreateWithFlags(&c, cudaEventDisableTiming), "event");
        h->ev_pos.push_back(a);
        h->ev_vel.push_back(b);
        h->ev_done.push_back(c);
    }
    return MOG_OK;
}

// One step over host-memory particles, in `chunks` pieces of whole 256-
// particle blocks.  Copy-in stream: every position chunk, then every
// velocity chunk.  Caller's stream: each chunk's deposit as soon as its
// positions have landed; the solve; then each chunk's update (the learned
// kernel, or the gather + leapfrog), each as soon as its velocities have
// landed.  Copy-out stream: each chunk's records as soon as its update is
// done.  The caller's stream finally waits for the last copy out.  The
// plain update stages every grid once per launch, so it runs as one launch
// (its copies out still go chunk by chunk).  Integer deposits and
// per-particle updates make the result bit-identical to the device step.
static int run_host_step(mog_handle* h, const mog_model* m, float* pos_host, float* vel_host,
                         int64_t n, float dt, int chunks, cudaStream_t s) {
    const mog::Ensemble& e = h->e;
    int64_t per = (n + chunks - 1) / chunks;
    per = std::max<int64_t>(256, (per + 255) / 256 * 256);
    chunks = (int)((n + per - 1) / per);
    int rc = ensure_host_step(h, n, chunks);
    if (rc) return rc;
    auto lo_of = [&](int c) { return (int64_t)c * per; };
    auto n_of = [&](int c) { return std::min<int64_t>(n, lo_of(c) + per) - lo_of(c); };
    const float4* hp = reinterpret_cast<const float4*>(pos_host);
    const float4* hv = reinterpret_cast<const float4*>(vel_host);
    MOG_CUDA(cudaEventRecord(h->ev_start, s), "event");
    MOG_CUDA(cudaStreamWaitEvent(h->s_in, h->ev_start, 0), "wait");
    for (int c = 0; c < chunks; ++c) {
        MOG_CUDA(cudaMemcpyAsync(h->d_hpos + lo_of(c), hp + lo_of(c), sizeof(float4) * n_of(c),
                                 cudaMemcpyHostToDevice, h->s_in), "positions in");
        MOG_CUDA(cudaEventRecord(h->ev_pos[c], h->s_in), "event");
    }
    for (int c = 0; c < chunks; ++c) {
        MOG_CUDA(cudaMemcpyAsync(h->d_hvel + lo_of(c), hv + lo_of(c), sizeof(float4) * n_of(c),
                                 cudaMemcpyHostToDevice, h->s_in), "velocities in");
        MOG_CUDA(cudaEventRecord(h->ev_vel[c], h->s_in), "event");
    }
    cudaError_t err = cudaSuccess;
    for (int c = 0; c < chunks && !err; ++c) {
        err = cudaStreamWaitEvent(s, h->ev_pos[c], 0);
        if (!err)
            err = mog::launch_deposit(e, h->d_hpos + lo_of(c), nullptr, n_of(c), false, h->d_mass,
                                      h->dshape, s);
    }
    if (err) return cuda_fail(err, "deposit");
    if (m) {
        if (h->cfg.solver == MOG_SOLVER_FFT && h->learned_fold) {
            err = mog::launch_spectral_density(e, h->d_mass, h->d_force, h->d_scratch, s, h->solve_split);
        } else {
            err = h->cfg.solver == MOG_SOLVER_FFT
                      ? mog::launch_spectral(e, h->d_mass, h->d_force, mog::kFrameWorld, false, h->d_scratch, s, h->solve_split)
                      : mog::launch_convolution(e, h->d_mass, h->d_force, mog::kFrameWorld, false, s);
            if (!err) err = mog::launch_density_w(e, h->d_mass, h->d_force, s);
        }
    } else {
        err = h->cfg.solver == MOG_SOLVER_FFT
                  ? mog::launch_spectral(e, h->d_mass, h->d_force, mog::kFrameWorldSlot, true, h->d_scratch, s, h->solve_split)
                  : mog::launch_convolution(e, h->d_mass, h->d_force, mog::kFrameWorldSlot, true, s);
    }
    if (err) return cuda_fail(err, "solve");
    int used = 0;  // spread partial sums written so far (one per learned CTA)
    const int upd_chunks = m ? chunks : 1;
    for (int c = 0; c < chunks && !err; ++c) {
        if (c < upd_chunks) {
            const int last = m ? c : chunks - 1;  // velocities this launch needs
            for (int v = m ? c : 0; v <= last && !err; ++v) err = cudaStreamWaitEvent(s, h->ev_vel[v], 0);
            const int64_t lo = m ? lo_of(c) : 0, cnt = m ? n_of(c) : n;
            if (!err && m) {
                mog::LearnedOut out;
                out.spread = h->d_spread + 2 * used;
                out.spread_cap = h->spread_cap - used;
                err = mog::launch_learned(0, e, h->rows.data(), h->d_hpos + lo, h->d_hvel + lo, cnt,
                                          h->d_force, m->norm, m->d_frags, m->d_params, dt,
                                          h->cfg.damping, out, s, h->learned_ctas);
                used += out.blocks;
            } else if (!err) {
                err = mog::launch_update(e, h->d_hpos, h->d_hvel, nullptr, nullptr, n, h->d_force, dt,
                                         h->cfg.damping, nullptr, h->ushape, s);
            }
            if (!err) err = cudaEventRecord(h->ev_done[c], s);
        }
        const int done_ev = std::min(c, upd_chunks - 1);
        if (!err) err = cudaStreamWaitEvent(h->s_out, h->ev_done[done_ev], 0);
        if (!err)
            err = cudaMemcpyAsync(pos_host + 4 * lo_of(c), h->d_hpos + lo_of(c),
                                  sizeof(float4) * n_of(c), cudaMemcpyDeviceToHost, h->s_out);
        if (!err)
            err = cudaMemcpyAsync(vel_host + 4 * lo_of(c), h->d_hvel + lo_of(c),
                                  sizeof(float4) * n_of(c), cudaMemcpyDeviceToHost, h->s_out);
    }
    if (err) return cuda_fail(err, "host step");
    MOG_CUDA(cudaEventRecord(h->ev_out, h->s_out), "event");
    MOG_CUDA(cudaStreamWaitEvent(s, h->ev_out, 0), "wait");
    if (m) {
        h->spread_blocks = used;
        h->spread_n = n;
    }
    return MOG_OK;
}

extern "C" {

int mog_model_create(mog_model** out) {
    if (!out) return fail(MOG_ERR_ARG, "null argument");
    *out = nullptr;
    mog_model* m = new mog_model();
    cudaGetDevice(&m->device);
    const size_t pb = sizeof(float) * mog::mlp_param_count();
    cudaError_t err;
    if ((err = cudaMalloc((void**)&m->d_params, pb)) || (err = cudaMalloc((void**)&m->d_m, pb)) ||
        (err = cudaMalloc((void**)&m->d_v, pb)) || (err = cudaMalloc((void**)&m->d_grad, pb)) ||
        (err = cudaMalloc(&m->d_frags, mog::mlp_fragment_bytes())) ||
        (err = cudaMemset(m->d_params, 0, pb)) || (err = cudaMemset(m->d_m, 0, pb)) ||
        (err = cudaMemset(m->d_v, 0, pb))) {
        mog_model_destroy(m);
        return cuda_fail(err, "mog_model_create");
    }
    for (int j = 0; j < mog::kModelIn; ++j) m->norm.inv_sigma[j] = 1.f;
    m->norm.force_scale = m->norm.rho_ref = m->norm.out_scale = 1.f;
    *out = m;
    return MOG_OK;
}

int mog_model_destroy(mog_model* m) {
    if (!m) return MOG_OK;
    void* ptrs[] = {m->d_params, m->d_m, m->d_v, m->d_grad, m->d_frags, m->d_partial, m->d_loss};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    delete m;
    return MOG_OK;
}

int mog_model_set(mog_model* m, const float* params, const float* norm) {
    if (!m || !params || !norm) return fail(MOG_ERR_ARG, "null argument");
    for (int i = 0; i < MOG_MODEL_NORM; ++i)
        if (!std::isfinite(norm[i])) return fail(MOG_ERR_ARG, "norm must be finite");
    if (!(norm[24] > 0.f) || !(norm[25] > 0.f))
        return fail(MOG_ERR_ARG, "force_scale and rho_ref must be positive");
    if (norm[27] != 0.f && norm[27] != 1.f) return fail(MOG_ERR_ARG, "norm[27] (base mode) must be 0 or 1");
    const size_t pb = sizeof(float) * mog::mlp_param_count();
    MOG_CUDA(cudaMemcpy(m->d_params, params, pb, cudaMemcpyHostToDevice), "upload params");
    MOG_CUDA(cudaMemset(m->d_m, 0, pb), "reset adam");
    MOG_CUDA(cudaMemset(m->d_v, 0, pb), "reset adam");
    std::memcpy(&m->norm, norm, sizeof(mog::ModelNorm));
    m->step = 0;
    MOG_CUDA(mog::launch_pack_fragments(m->d_params, m->d_frags, 0), "pack fragments");
    MOG_CUDA(cudaDeviceSynchronize(), "sync");
    return MOG_OK;
}

int mog_model_get(const mog_model* m, float* params, float* norm) {
    if (!m || !params || !norm) return fail(MOG_ERR_ARG, "null argument");
    MOG_CUDA(cudaDeviceSynchronize(), "sync");
    MOG_CUDA(cudaMemcpy(params, m->d_params, sizeof(float) * mog::mlp_param_count(),
                        cudaMemcpyDeviceToHost), "download params");
    std::memcpy(norm, &m->norm, sizeof(mog::ModelNorm));
    return MOG_OK;
}

int mog_model_train_step(mog_model* m, const float* feat16, const float* target4, const int* idx,
                         int32_t batch, float lr, float* loss_out, float* grad_out, void* stream) {
    if (!m || !feat16 || !target4 || !idx) return fail(MOG_ERR_ARG, "null argument");
    if (batch <= 0) return fail(MOG_ERR_ARG, "batch must be positive");
    if (!std::isfinite(lr) || lr < 0.f) return fail(MOG_ERR_ARG, "lr must be finite and >= 0");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int ctas = (batch + 127) / 128;
    if (ctas > m->partial_ctas) {
        MOG_CUDA(cudaStreamSynchronize(s), "sync");
        cudaFree(m->d_partial);
        cudaFree(m->d_loss);
        m->d_partial = nullptr;
        m->d_loss = nullptr;
        MOG_CUDA(cudaMalloc((void**)&m->d_partial, sizeof(float) * mog::mlp_param_count() * ctas), "partials");
        MOG_CUDA(cudaMalloc((void**)&m->d_loss, sizeof(float) * ctas), "loss partials");
        m->partial_ctas = ctas;
    }
    if (lr > 0.f) ++m->step;
    cudaError_t err = mog::launch_mlp_train_step(feat16, target4, idx, batch, m->d_params,
                                                 m->d_partial, m->d_loss, m->d_grad, m->d_m,
                                                 m->d_v, lr, m->step, s);
    if (err != cudaSuccess) return cuda_fail(err, "train step");
    if (lr > 0.f) {
        err = mog::launch_pack_fragments(m->d_params, m->d_frags, s);
        if (err != cudaSuccess) return cuda_fail(err, "pack fragments");
    }
    if (grad_out)
        MOG_CUDA(cudaMemcpyAsync(grad_out, m->d_grad, sizeof(float) * mog::mlp_param_count(),
                                 cudaMemcpyDeviceToDevice, s), "copy grad");
    if (loss_out) {
        std::vector<float> l(ctas);
        MOG_CUDA(cudaMemcpyAsync(l.data(), m->d_loss, sizeof(float) * ctas, cudaMemcpyDeviceToHost, s),
                 "read loss");
        MOG_CUDA(cudaStreamSynchronize(s), "sync");
        double tot = 0;
        for (float v : l) tot += v;
        *loss_out = (float)(tot / batch);
    }
    return MOG_OK;
}

int mog_features(mog_handle* h, const mog_model* m, const float* pos4, int64_t n, float* mean4_out,
                 float* feat16_out, void* stream) {
    if (!h || !m) return fail(MOG_ERR_ARG, "null argument");
    int rc = check_particles(h, pos4, mean4_out, n, true);
    if (rc) return rc;
    if (n > 0 && !feat16_out) return fail(MOG_ERR_ARG, "feat16_out is null");
    if ((rc = set_device(h))) return rc;
    return run_learned(h, m, 2, const_cast<float*>(pos4), nullptr, n, 0.f,
                       reinterpret_cast<float4*>(mean4_out), feat16_out,
                       static_cast<cudaStream_t>(stream));
}

int mog_learned_forces(mog_handle* h, const mog_model* m, const float* pos4, float* acc4, int64_t n,
                       void* stream) {
    if (!h || !m) return fail(MOG_ERR_ARG, "null argument");
    int rc = check_particles(h, pos4, acc4, n, true);
    if (rc) return rc;
    if ((rc = set_device(h))) return rc;
    return run_learned(h, m, 1, const_cast<float*>(pos4), nullptr, n, 0.f,
                       reinterpret_cast<float4*>(acc4), nullptr, static_cast<cudaStream_t>(stream));
}

int mog_learned_step(mog_handle* h, const mog_model* m, float* pos4, float* vel4, int64_t n,
                     float dt_eff, void* stream) {
    if (!h || !m) return fail(MOG_ERR_ARG, "null argument");
    int rc = check_particles(h, pos4, vel4, n, true);
    if (rc) return rc;
    if (!std::isfinite(dt_eff)) return fail(MOG_ERR_ARG, "dt_eff must be finite");
    if ((rc = set_device(h))) return rc;
    if ((rc = run_learned(h, m, 0, pos4, vel4, n, dt_eff, nullptr, nullptr,
                          static_cast<cudaStream_t>(stream))))
        return rc;
    ++h->step_count;
    return MOG_OK;
}

int mog_learned_step_profiled(mog_handle* h, const mog_model* m, float* pos4, float* vel4,
                              int64_t n, float dt_eff, float* phase_ms, void* stream) {
    if (!h || !m || !phase_ms) return fail(MOG_ERR_ARG, "null argument");
    int rc = check_particles(h, pos4, vel4, n, true);
    if (rc) return rc;
    if (!std::isfinite(dt_eff)) return fail(MOG_ERR_ARG, "dt_eff must be finite");
    if ((rc = set_device(h))) return rc;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    cudaEvent_t ev[5];
    for (auto& x : ev) MOG_CUDA(cudaEventCreate(&x), "event create");
    rc = run_learned(h, m, 0, pos4, vel4, n, dt_eff, nullptr, nullptr, s, ev);
    cudaError_t err = rc ? cudaSuccess : cudaEventSynchronize(ev[4]);
    for (int i = 0; i < 4 && !rc && !err; ++i) err = cudaEventElapsedTime(&phase_ms[i], ev[i], ev[i + 1]);
    for (auto& x : ev) cudaEventDestroy(x);
    if (rc) return rc;
    if (err) return cuda_fail(err, "profiled learned step");
    ++h->step_count;
    return MOG_OK;
}

int mog_learned_spread(mog_handle* h, double* out2, void* stream) {
    if (!h || !out2) return fail(MOG_ERR_ARG, "null argument");
    int rc = set_device(h);
    if (rc) return rc;
    out2[0] = out2[1] = 0.0;
    if (h->spread_blocks <= 0 || h->spread_n <= 0) return MOG_OK;
    std::vector<float> part(2 * (size_t)h->spread_blocks);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    MOG_CUDA(cudaMemcpyAsync(part.data(), h->d_spread, sizeof(float) * part.size(),
                             cudaMemcpyDeviceToHost, s), "read spread");
    MOG_CUDA(cudaStreamSynchronize(s), "sync");
    double a = 0.0, b = 0.0;
    for (int i = 0; i < h->spread_blocks; ++i) {
        a += part[2 * i];
        b += part[2 * i + 1];
    }
    out2[0] = a / (double)h->spread_n;
    out2[1] = b / (double)h->spread_n;
    return MOG_OK;
}

static int host_step_args(mog_handle* h, float* pos4_host, float* vel4_host, int64_t n,
                          float dt_eff, int32_t chunks) {
    int rc = check_particles(h, pos4_host, vel4_host, n, true);
    if (rc) return rc;
    if (!std::isfinite(dt_eff)) return fail(MOG_ERR_ARG, "dt_eff must be finite");
    if (chunks < 1 || chunks > 64) return fail(MOG_ERR_ARG, "chunks must be in [1, 64]");
    return set_device(h);
}

int mog_step_host(mog_handle* h, float* pos4_host, float* vel4_host, int64_t n, float dt_eff,
                  int32_t chunks, void* stream) {
    if (!h) return fail(MOG_ERR_ARG, "handle is null");
    int rc = host_step_args(h, pos4_host, vel4_host, n, dt_eff, chunks);
    if (rc || n == 0) return rc;
    if ((rc = run_host_step(h, nullptr, pos4_host, vel4_host, n, dt_eff, chunks,
                            static_cast<cudaStream_t>(stream))))
        return rc;
    ++h->step_count;
    return MOG_OK;
}

int mog_learned_step_host(mog_handle* h, const mog_model* m, float* pos4_host, float* vel4_host,
                          int64_t n, float dt_eff, int32_t chunks, void* stream) {
    if (!h || !m) return fail(MOG_ERR_ARG, "null argument");
    int rc = host_step_args(h, pos4_host, vel4_host, n, dt_eff, chunks);
    if (rc || n == 0) return rc;
    if ((rc = run_host_step(h, m, pos4_host, vel4_host, n, dt_eff, chunks,
                            static_cast<cudaStream_t>(stream))))
        return rc;
    ++h->step_count;
    return MOG_OK;
}

}  // extern "C"

// ---- batched simulations -------------------------------------------------

struct mog_batch {
    std::vector<mog_handle*> sims;
    int device = 0;
    cudaStream_t cap = nullptr;
    std::vector<cudaStream_t> branch;
    std::vector<cudaEvent_t> done;
    cudaEvent_t fork = nullptr;
    mog_batch_tuning tuning{1, 0, 0, 0};
    struct Entry {
        std::vector<float*> pos, vel;
        std::vector<int64_t> n;
        std::vector<float> dt;
        cudaGraphExec_t exec = nullptr;
        // work-queue mode: the simulation records, both tile lists and the
        // two queue counters (device memory owned by the entry)
        void* d_queue = nullptr;
        int queue = 0;
    };
    std::vector<Entry> graphs;
};

namespace {

void release_entry(mog_batch::Entry& g) {
    if (g.exec) cudaGraphExecDestroy(g.exec);
    if (g.d_queue) cudaFree(g.d_queue);
    g.exec = nullptr;
    g.d_queue = nullptr;
}

// Whether the batch can run as the two persistent work-queue launches:
// every simulation uses the FFT solver, FAST cell indices, no spatial
// re-ordering and g of 8, 16 or 32, and all share one mass mode.
bool queue_eligible(const mog_batch* b) {
    const int mm = b->sims[0]->cfg.mass_mode;
    for (const mog_handle* h : b->sims) {
        const int g = h->cfg.grid_size;
        if (h->cfg.solver != MOG_SOLVER_FFT || h->cfg.index_mode != MOG_INDEX_FAST ||
            h->sort_every != 0 || h->cfg.mass_mode != mm || (g != 8 && g != 16 && g != 32))
            return false;
    }
    return true;
}

// Tile lists of one ensemble step, largest first (so the last tiles to
// be popped are the short ones).  Deposit tiles: whole grid groups of
// queue_deposit_grids grids over `chunk` particles; gather tiles:
// kQueueGatherTile particles over all of a simulation's grids.  A g = 32
// gather reads L2 instead of shared memory and counts double.
void build_tiles(const mog_batch* b, const int64_t* n, int64_t chunk,
                 std::vector<mog::DepositTile>& dep, std::vector<mog::GatherTile>& gat) {
    std::vector<std::pair<double, mog::DepositTile>> d;
    std::vector<std::pair<double, mog::GatherTile>> q;
    for (int i = 0; i < (int)b->sims.size(); ++i) {
        const mog_handle* h = b->sims[i];
        const int k = h->cfg.n_grids, g = h->cfg.grid_size;
        const int gpc = mog::queue_deposit_grids(g, h->cfg.mass_mode, k, b->tuning.deposit_split > 0);
        for (int g0 = 0; g0 < k; g0 += gpc)
            for (int64_t lo = 0; lo < n[i]; lo += chunk) {
                mog::DepositTile t{i, g0, std::min(gpc, k - g0), 0, lo, std::min(n[i], lo + chunk)};
                d.push_back({(double)(t.hi - t.lo) * t.ng, t});
            }
        for (int64_t lo = 0; lo < n[i]; lo += mog::kQueueGatherTile) {
            mog::GatherTile t{i, 0, lo, std::min(n[i], lo + mog::kQueueGatherTile)};
            q.push_back({(double)(t.hi - t.lo) * k * (g > 16 ? 2.0 : 1.0), t});
        }
    }
    auto by_cost = [](const auto& a, const auto& b2) { return a.first > b2.first; };
    std::stable_sort(d.begin(), d.end(), by_cost);
    std::stable_sort(q.begin(), q.end(), by_cost);
    dep.clear();
    gat.clear();
    for (auto& x : d) dep.push_back(x.second);
    for (auto& x : q) gat.push_back(x.second);
}

// Capture one ensemble step as: clear the two queue counters, the
// work-queue deposit of every simulation, every simulation's solve on its
// own branch, the work-queue gather + update of every simulation.
int capture_queue_step(mog_batch* b, float* const* pos4, float* const* vel4, const int64_t* n,
                       const float* dt_eff, mog_batch::Entry& entry, cudaGraph_t* graph) {
    const int count = (int)b->sims.size();
    const int64_t chunk = b->tuning.deposit_chunk > 0 ? b->tuning.deposit_chunk : 393216;
    std::vector<mog::DepositTile> dep;
    std::vector<mog::GatherTile> gat;
    build_tiles(b, n, chunk, dep, gat);
    std::vector<mog::BatchSim> recs(count);
    size_t smem = 0;
    int kmax = 1;
    for (int i = 0; i < count; ++i) {
        mog_handle* h = b->sims[i];
        recs[i].e = h->e;
        recs[i].pos = reinterpret_cast<float4*>(pos4[i]);
        recs[i].vel = reinterpret_cast<float4*>(vel4[i]);
        recs[i].n = n[i];
        recs[i].mass = h->d_mass;
        recs[i].force = h->d_force;
        recs[i].dt = dt_eff[i];
        recs[i].damping = h->cfg.damping;
        const int g = h->cfg.grid_size;
        const bool split = b->tuning.deposit_split > 0;
        smem = std::max(smem, mog::queue_deposit_smem(
                                  g, h->cfg.mass_mode,
                                  mog::queue_deposit_grids(g, h->cfg.mass_mode, h->cfg.n_grids, split),
                                  split));
        kmax = std::max(kmax, h->cfg.n_grids);
    }
    const size_t sims_b = sizeof(mog::BatchSim) * count;
    const size_t dep_b = sizeof(mog::DepositTile) * dep.size();
    const size_t gat_b = sizeof(mog::GatherTile) * gat.size();
    auto up = [](size_t x) { return (x + 255) & ~(size_t)255; };
    const size_t total = up(sims_b) + up(dep_b) + up(gat_b) + 256;
    char* base = nullptr;
    MOG_CUDA(cudaMalloc((void**)&base, total), "batch queue buffers");
    entry.d_queue = base;
    auto* d_sims = reinterpret_cast<mog::BatchSim*>(base);
    auto* d_dep = reinterpret_cast<mog::DepositTile*>(base + up(sims_b));
    auto* d_gat = reinterpret_cast<mog::GatherTile*>(base + up(sims_b) + up(dep_b));
    auto* d_cnt = reinterpret_cast<unsigned*>(base + up(sims_b) + up(dep_b) + up(gat_b));
    MOG_CUDA(cudaMemcpy(d_sims, recs.data(), sims_b, cudaMemcpyHostToDevice), "batch records");
    if (dep_b) MOG_CUDA(cudaMemcpy(d_dep, dep.data(), dep_b, cudaMemcpyHostToDevice), "deposit tiles");
    if (gat_b) MOG_CUDA(cudaMemcpy(d_gat, gat.data(), gat_b, cudaMemcpyHostToDevice), "gather tiles");

    int rc = MOG_OK;
    MOG_CUDA(cudaStreamBeginCapture(b->cap, cudaStreamCaptureModeThreadLocal), "begin capture");
    cudaError_t err = cudaMemsetAsync(d_cnt, 0, 2 * sizeof(unsigned), b->cap);
    if (!err) err = mog::launch_deposit_queue(b->sims[0]->cfg.mass_mode, b->tuning.deposit_split,
                                              d_sims, d_dep, (int)dep.size(), d_cnt, smem, b->cap);
    if (!err) err = cudaEventRecord(b->fork, b->cap);
    for (int i = 0; i < count && !err; ++i) {
        mog_handle* h = b->sims[i];
        err = cudaStreamWaitEvent(b->branch[i], b->fork, 0);
        if (!err) err = mog::launch_spectral(h->e, h->d_mass, h->d_force, mog::kFrameWorldSlot, true, h->d_scratch,
                                             b->branch[i], h->solve_split);
        if (!err) err = cudaEventRecord(b->done[i], b->branch[i]);
        if (!err) err = cudaStreamWaitEvent(b->cap, b->done[i], 0);
    }
    if (!err) err = mog::launch_gather_queue(d_sims, d_gat, (int)gat.size(), d_cnt + 1, kmax, b->cap);
    cudaError_t end = cudaStreamEndCapture(b->cap, graph);
    if (err || end) {
        if (*graph) cudaGraphDestroy(*graph);
        *graph = nullptr;
        rc = cuda_fail(err ? err : end, "batch work-queue capture");
    }
    entry.queue = 1;
    return rc;
}

}  // namespace

extern "C" {

int mog_batch_set_tuning(mog_batch* b, const mog_batch_tuning* t) {
    if (!b || !t) return fail(MOG_ERR_ARG, "null argument");
    if (t->work_queue < 0 || t->work_queue > 1 || t->deposit_chunk < 0 ||
        (t->deposit_chunk > 0 && t->deposit_chunk < 1024) || t->deposit_split < 0 ||
        t->deposit_split > 2)
        return fail(MOG_ERR_ARG, "batch tuning value out of range");
    b->tuning = *t;
    for (auto& g : b->graphs) release_entry(g);
    b->graphs.clear();
    return MOG_OK;
}

int mog_batch_get_tuning(const mog_batch* b, mog_batch_tuning* t) {
    if (!b || !t) return fail(MOG_ERR_ARG, "null argument");
    *t = b->tuning;
    t->active_work_queue = (b->tuning.work_queue && queue_eligible(b)) ? 1 : 0;
    return MOG_OK;
}

int mog_batch_destroy(mog_batch* b) {
    if (!b) return MOG_OK;
    for (auto& g : b->graphs) release_entry(g);
    for (auto s : b->branch)
        if (s) cudaStreamDestroy(s);
    for (auto e : b->done)
        if (e) cudaEventDestroy(e);
    if (b->fork) cudaEventDestroy(b->fork);
    if (b->cap) cudaStreamDestroy(b->cap);
    delete b;
    return MOG_OK;
}

int mog_batch_create(mog_handle* const* handles, int32_t count, mog_batch** out) {
    if (!handles || !out || count <= 0) return fail(MOG_ERR_ARG, "need handles and count > 0");
    *out = nullptr;
    mog_batch* b = new mog_batch();
    b->device = handles[0] ? handles[0]->device : 0;
    for (int i = 0; i < count; ++i) {
        if (!handles[i]) {
            mog_batch_destroy(b);
            return fail(MOG_ERR_ARG, "null handle in batch");
        }
        if (handles[i]->device != b->device) {
            mog_batch_destroy(b);
            return fail(MOG_ERR_ARG, "all handles of a batch must be on one device");
        }
        for (int j = 0; j < i; ++j)
            if (handles[j] == handles[i]) {
                mog_batch_destroy(b);
                return fail(MOG_ERR_ARG, "a handle appears twice in the batch");
            }
        b->sims.push_back(handles[i]);
    }
    cudaError_t err = cudaStreamCreateWithFlags(&b->cap, cudaStreamNonBlocking);
    if (!err) err = cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming);
    b->branch.assign(count, nullptr);
    b->done.assign(count, nullptr);
    for (int i = 0; i < count && !err; ++i) {
        err = cudaStreamCreateWithFlags(&b->branch[i], cudaStreamNonBlocking);
        if (!err) err = cudaEventCreateWithFlags(&b->done[i], cudaEventDisableTiming);
    }
    if (err) {
        mog_batch_destroy(b);
        return cuda_fail(err, "mog_batch_create");
    }
    *out = b;
    return MOG_OK;
}

int mog_batch_step(mog_batch* b, float* const* pos4, float* const* vel4, const int64_t* n,
                   const float* dt_eff, int32_t n_steps, void* stream) {
    if (!b || !pos4 || !vel4 || !n || !dt_eff) return fail(MOG_ERR_ARG, "null argument");
    if (n_steps < 0) return fail(MOG_ERR_ARG, "n_steps must be >= 0");
    const int count = (int)b->sims.size();
    for (int i = 0; i < count; ++i) {
        int rc = check_particles(b->sims[i], pos4[i], vel4[i], n[i], true);
        if (rc) return rc;
        if (!std::isfinite(dt_eff[i])) return fail(MOG_ERR_ARG, "dt_eff must be finite");
    }
    if (n_steps == 0) return MOG_OK;
    int rc = set_device(b->sims[0]);
    if (rc) return rc;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    mog_batch::Entry* ge = nullptr;
    for (auto& g : b->graphs) {
        bool same = true;
        for (int i = 0; i < count && same; ++i)
            same = g.pos[i] == pos4[i] && g.vel[i] == vel4[i] && g.n[i] == n[i] && g.dt[i] == dt_eff[i];
        if (same) ge = &g;
    }
    if (!ge && b->tuning.work_queue && queue_eligible(b)) {
        mog_batch::Entry entry;
        cudaGraph_t graph = nullptr;
        rc = capture_queue_step(b, pos4, vel4, n, dt_eff, entry, &graph);
        cudaError_t err = rc ? cudaSuccess : cudaGraphInstantiate(&entry.exec, graph, 0);
        if (graph) cudaGraphDestroy(graph);
        if (rc || err) {
            release_entry(entry);
            return rc ? rc : cuda_fail(err, "batch graph instantiate");
        }
        entry.pos.assign(pos4, pos4 + count);
        entry.vel.assign(vel4, vel4 + count);
        entry.n.assign(n, n + count);
        entry.dt.assign(dt_eff, dt_eff + count);
        if (b->graphs.size() >= 4) {
            release_entry(b->graphs.front());
            b->graphs.erase(b->graphs.begin());
        }
        b->graphs.push_back(std::move(entry));
        ge = &b->graphs.back();
    }
    if (!ge) {
        // buffers that a captured step cannot allocate
        for (int i = 0; i < count; ++i) {
            mog_handle* h = b->sims[i];
            if (h->sort_every == 1 && n[i] > h->perm_cap)
                return fail(MOG_ERR_ARG, "batch: n exceeds a handle's num_particles");
        }
        cudaGraph_t graph = nullptr;
        MOG_CUDA(cudaStreamBeginCapture(b->cap, cudaStreamCaptureModeThreadLocal), "begin capture");
        cudaError_t err = cudaEventRecord(b->fork, b->cap);
        for (int i = 0; i < count && !err && !rc; ++i) {
            err = cudaStreamWaitEvent(b->branch[i], b->fork, 0);
            if (err) break;
            mog_handle* h = b->sims[i];
            rc = run_pipeline(h, reinterpret_cast<float4*>(pos4[i]), reinterpret_cast<float4*>(vel4[i]),
                              n[i], dt_eff[i], nullptr, b->branch[i], h->sort_every == 1);
            if (!rc) err = cudaEventRecord(b->done[i], b->branch[i]);
            if (!err && !rc) err = cudaStreamWaitEvent(b->cap, b->done[i], 0);
        }
        cudaError_t end = cudaStreamEndCapture(b->cap, &graph);
        if (rc || err || end) {
            if (graph) cudaGraphDestroy(graph);
            if (rc) return rc;
            return cuda_fail(err ? err : end, "batch capture");
        }
        mog_batch::Entry entry;
        entry.pos.assign(pos4, pos4 + count);
        entry.vel.assign(vel4, vel4 + count);
        entry.n.assign(n, n + count);
        entry.dt.assign(dt_eff, dt_eff + count);
        err = cudaGraphInstantiate(&entry.exec, graph, 0);
        cudaGraphDestroy(graph);
        if (err) return cuda_fail(err, "batch graph instantiate");
        if (b->graphs.size() >= 4) {
            release_entry(b->graphs.front());
            b->graphs.erase(b->graphs.begin());
        }
        b->graphs.push_back(std::move(entry));
        ge = &b->graphs.back();
    }
    for (int t = 0; t < n_steps; ++t) MOG_CUDA(cudaGraphLaunch(ge->exec, s), "batch graph launch");
    for (auto* h : b->sims) h->step_count += (uint64_t)n_steps;
    return MOG_OK;
}

}  // extern "C"

