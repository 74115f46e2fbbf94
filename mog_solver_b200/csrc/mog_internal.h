// mog_internal.h — host-side launcher interface between the C ABI layer
// (mog_api.cu) and the kernel translation units.
#pragma once

#include <algorithm>
#include <cstdint>
#include <vector>
#include <cuda_runtime.h>

#include "mog_device.cuh"

namespace mog {

// Ranks of a sharded step over peer memory (at most this many).
constexpr int kMaxShardRanks = 8;

// Grid ownership of a sharded step: grid i belongs to rank
// floor(i * world / k), so rank r owns the grids
// [ceil(r k / world), ceil((r + 1) k / world)) (none when world > k and the
// range is empty).  The owner accumulates the grid's cells from every rank.
__host__ __device__ inline int shard_owner(int grid, int k, int world) {
    return (int)(((int64_t)grid * world) / k);
}
__host__ __device__ inline int shard_first_grid(int rank, int k, int world) {
    return (int)(((int64_t)rank * k + world - 1) / world);
}

// Where a sharded deposit sends each grid's cells (device memory, one per
// slot): base[q] is rank q's accumulation buffer for the slot, in the full
// k g^3 layout (only the grids q owns are written).
struct ShardTargets {
    void* base[kMaxShardRanks];
    int world;
};

// Everything about one grid ensemble that the kernels read.  All pointers
// are device memory owned by the handle.
struct Ensemble {
    int k = 0;             // number of grids
    int g = 0;             // cells per axis (power of two)
    int lg = 0;            // log2 g
    int mass_mode = 0;     // MOG_MASS_*
    int index_mode = 0;    // MOG_INDEX_*
    int alias_xz = 0;      // reproduce the reference's x <- z force aliasing
    float world = 0.f;     // L
    float voxel = 0.f;     // h
    float G = 0.f;
    float scale = 0.f;     // 2^scale_bits (u64 mode)
    float inv_scale = 0.f; // 2^-scale_bits
    const float* rot12 = nullptr;   // k x 12 (reference packing)
    const float* off4 = nullptr;    // k x 4
    const FastXf* fast = nullptr;   // k FAST-mode rows
    const float* green = nullptr;   // g^3 Green's factors -2 pi G / k^2 (0 when k^2 <= 1e-4)
    const float* ktab = nullptr;    // g wave numbers 2 pi shift(i) / L
    const float4* conv_kernel = nullptr;  // g^3 real-space kernel r/(4 pi r^3) (main.py:250-278)
    int dft_tc = 0;                 // axis passes on the tensor cores (MOG_DFT_TC_BF16X3)
    const void* dft_tables = nullptr;  // their DFT matrices (dft_tc_tables layout)
    unsigned* flags = nullptr;      // device status word
    double* mass_total = nullptr;   // running sum of q for the overflow check

    __host__ __device__ int64_t cells() const { return (int64_t)k << (3 * lg); }
    __host__ __device__ IndexParams index_params() const {
        IndexParams ip;
        ip.half_l = world * 0.5f;
        ip.world = world;
        ip.voxel = voxel;
        ip.lg = lg;
        return ip;
    }
};

// Launch-shape knobs (chosen by the autotuner or by defaults).
struct DepositShape {
    int threads = 1024;
    int grids_per_cta = 0;  // 0 = default for (g, mass mode); -1 = global atomics
    int chunks = 0;         // particle chunks; 0 = derived from n
    int ppt = 4;            // particles per thread carried through the grid loop
    int aggregate = -1;     // warp-merge runs of equal cells: -1 auto (when ordered), 0, 1
    int fast = 1;           // use the specialised kernel where it applies
    int sorted_input = 0;   // read the spatially ordered copy (else the caller's order)
    int split = 0;          // u64 one-word histogram: 0 auto (high words, g = 32), 1 high words also g = 8/16, 2 counts (uniform masses), -1 never
};
struct UpdateShape {
    int threads = 0;        // staged gather block size: 512, 768 or 1024; 0 auto
    int staged = -1;        // -1 auto, 0 global gathers, 1 smem-staged grids
    int ctas = 0;           // staged kernel CTAs; 0 = one per SM
    int direct_ppt = 0;     // particles per thread of the direct gather; 0 auto
};

int num_sms();

// mass grid (u64 or u32 per mode) <- particles.  Zeroes nothing: the
// caller provides a zeroed grid.  shard: `mass` is instead a device
// ShardTargets, and each cell goes to its owning rank's buffer.
// perm (nullable): slot s processes particle perm[s].  ordered: the
// particles arrive in spatial order (pos already permuted, or perm set), so
// warp merging of equal cells pays off.
cudaError_t launch_deposit(const Ensemble& e, const float4* pos, const int* perm, int64_t n,
                           bool ordered, void* mass, const DepositShape& shape, cudaStream_t s,
                           bool shard = false);

// Layout of a solve's force grid (float4 per cell).
//   kFrameGrid      (fx, fy, fz, |f|) in each grid's own frame at cell c
//                   (the reference's gradient texture, the stage entry points);
//   kFrameWorld     M_i f as (x, y, z, 0) at cell c (the learned path's
//                   gather, which reads it from L1/L2);
//   kFrameWorldSlot M_i f as (x, y, z, 0) at force_slot(c) (the plain
//                   gathers, which stage whole grids in shared memory).
constexpr int kFrameGrid = 0;
constexpr int kFrameWorld = 1;
constexpr int kFrameWorldSlot = 2;

// force grid <- mass grid in the layout `frame` names.  zero_mass clears
// the input for the next step.  scratch: device memory of
// spectral_scratch_bytes(e) bytes.  split: the g = 8/16 fft solve on
// clusters of three CTAs per grid pair, 0 auto, 1 always, -1 never (same
// forces; kept out of Ensemble, whose size shapes every kernel's
// parameter block).
cudaError_t launch_spectral(const Ensemble& e, void* mass, float4* force, int frame,
                            bool zero_mass, void* scratch, cudaStream_t s, int split = 0);
size_t spectral_scratch_bytes(const Ensemble& e);

cudaError_t launch_convolution(const Ensemble& e, void* mass, float4* force, int frame,
                               bool zero_mass, cudaStream_t s);

// Tensor-core DFT passes (dft_tc.cu), g = 16 or 32: host-built B tables
// (forward hi, lo, inverse hi, lo; BF16 bits) and one in-place axis pass
// over the lines of nf fields of pairs x g^3 complex values.
std::vector<uint16_t> dft_tc_tables(int g);
cudaError_t launch_dft_tc(int g, float2* f0, float2* f1, float2* f2, int nf, int axis, int pairs,
                          bool inverse, const void* tables, unsigned* flags, cudaStream_t s);
// World-frame spectral solve that also leaves each cell's mass in the
// force grid's .w lane and clears the mass grid (the learned path).
cudaError_t launch_spectral_density(const Ensemble& e, void* mass, float4* force, void* scratch,
                                    cudaStream_t s, int split = 0);
// Rotate a grid-frame force grid (kFrameGrid) into the world frame, stored
// as kFrameWorldSlot for launch_update (the stage entry point mog_update).
cudaError_t launch_prerotate(const Ensemble& e, const float4* force_grid, float4* force_world,
                             cudaStream_t s);

// Gather + average + (optionally) leapfrog from a kFrameWorldSlot grid.
// When acc_out is non-null the averaged force is written there and pos/vel
// are left untouched.
// pos_sorted (nullable): pos[perm[s]] for every slot s, from which the
// cells are computed; the caller's pos/vel are read and written once per
// particle through perm.
cudaError_t launch_update(const Ensemble& e, float4* pos, float4* vel, const float4* pos_sorted,
                          const int* perm, int64_t n, const float4* force_world, float dt,
                          float damping, float4* acc_out, const UpdateShape& shape, cudaStream_t s);

// ---- batched ensemble work queue (deposit.cu, update.cu) -----------------
// One simulation of a batch as the work-queue kernels read it (device
// memory, one record per simulation).
struct BatchSim {
    Ensemble e;
    float4* pos = nullptr;
    float4* vel = nullptr;
    int64_t n = 0;
    void* mass = nullptr;           // its mass grid (zeroed by its previous solve)
    const float4* force = nullptr;  // its world-frame force grid
    float dt = 0.f;
    float damping = 1.f;
};
// Deposit tile: particles [lo, hi) of simulation `sim` into its grids
// [g0, g0 + ng).  Gather tile: particles [lo, hi) over all its grids.
struct DepositTile {
    int32_t sim, g0, ng, pad;
    int64_t lo, hi;
};
struct GatherTile {
    int32_t sim, pad;
    int64_t lo, hi;
};
// Grids per deposit tile for a simulation (whole grids in shared memory),
// the tile's shared-memory bytes, and the particles of one gather tile.
// split: u64 grids keep one word per cell in shared memory at every g (high
// words, or counts for uniform masses; at g = 32 they always do).
int queue_deposit_grids(int g, int mass_mode, int k, bool split);
size_t queue_deposit_smem(int g, int mass_mode, int ng, bool split);
constexpr int kQueueGatherThreads = 512;
constexpr int kQueueGatherPPT = 14;
constexpr int64_t kQueueGatherTile = (int64_t)kQueueGatherThreads * kQueueGatherPPT;
// Persistent launches over a host-built tile list (largest first): every
// CTA pops tiles with an atomic counter (*counter must be 0 at launch)
// until the list runs out.  All simulations use FAST cell indices and
// share the mass mode; g is 8, 16 or 32.  kmax: the most grids of any
// simulation (the gather stages their index rows in shared memory).
cudaError_t launch_deposit_queue(int mass_mode, int layout, const BatchSim* sims,
                                 const DepositTile* tiles, int ntiles, unsigned* counter, size_t smem,
                                 cudaStream_t s);
cudaError_t launch_gather_queue(const BatchSim* sims, const GatherTile* tiles, int ntiles,
                                unsigned* counter, int kmax, cudaStream_t s);

// Spatial ordering: perm <- particles sorted by the Morton index of their
// 32^3 world cell.  scratch: sort_scratch_bytes() bytes.
size_t sort_scratch_bytes();
// out[s] = pos[perm[s]]: the positions in spatial order, read coalesced by
// the deposit and the gather.
// One bounded device wait that nothing satisfies (update.cu); raises
// MOG_FLAG_TIMEOUT in *flags after about a second.
cudaError_t launch_wait_timeout_selftest(unsigned* flags, cudaStream_t s);

// Sharded step over peer memory (shard.cu).  accum[q]: rank q's
// accumulation buffer (3 slots of k g^3 cells), flags_local: this rank's
// world epoch words, flags_peer[q]: rank q's.
struct ShardView {
    void* accum[kMaxShardRanks] = {};
    uint64_t* flags_peer[kMaxShardRanks] = {};
    uint64_t* flags_local = nullptr;
    int rank = 0;
    int world = 0;
};
// This rank's deposit for `epoch` is complete: store epoch into word
// `rank` of every rank's flags (system-scope release).
cudaError_t launch_shard_signal(const ShardView& v, uint64_t epoch, cudaStream_t s);
// Wait (bounded) until every rank has signalled `epoch`, copy every
// owner's slice of slot `slot` into the local grid `local` (k g^3 cells),
// then clear this rank's slice of the previous step's slot.  A wait that
// runs out raises MOG_FLAG_TIMEOUT in e.flags and copies nothing.
cudaError_t launch_shard_exchange(const Ensemble& e, const ShardView& v, uint64_t epoch, int slot,
                                  void* local, cudaStream_t s);

// Sets the calling thread's mog_last_error() text (mog_api.cu); returns code.
int report_error(int code, const char* msg);

cudaError_t launch_gather_sorted(const float4* pos, const int* perm, int64_t n, float4* out,
                                 cudaStream_t s);
cudaError_t launch_sort(const float4* pos, int64_t n, float world, void* scratch, int* perm,
                        unsigned* flags, cudaStream_t s);

// Green's-function and wave-number tables (FP64 arithmetic on the device).
cudaError_t launch_build_tables(int g, float world, float G, float* green, float* ktab,
                                cudaStream_t s);

// FP64 momentum / energy / mass / centre-of-mass reduction.
cudaError_t launch_diagnostics(const float4* pos, const float4* vel, int64_t n, double* partial,
                               int nblocks, double* out8, cudaStream_t s);

// FP64 direct-sum yardstick: out3[t] = g_eff * sum_j m_j d / (|d|^2 + soft^2)^1.5
// over minimum-image separations.  partial: chunks * nt * 3 doubles.
cudaError_t launch_direct_sum(const float4* targets, int64_t nt, const float4* sources, int64_t ns,
                              double world, double g_eff, double soft, double* partial, int chunks,
                              double* out3, cudaStream_t s);
// Scratch of the allocation-free direct sum (diagnostics.cu): room for
// kDirectScratchPairs (target, chunk) partial sums of 3 doubles.
constexpr int64_t kDirectScratchPairs = int64_t(1) << 19;
cudaError_t direct_sum_scratch(double** out);

// ---- learned correction (learned.cu) ------------------------------------
constexpr int kModelIn = 12;
// Per-model normalisation: x = (f - mu) / sigma, out = y * out_scale.
struct ModelNorm {
    float mu[kModelIn];
    float inv_sigma[kModelIn];
    float force_scale;   // s: forces enter the features as F / s
    float rho_ref;       // mean cell mass (total mass / g^3)
    float out_scale;     // residual = y * out_scale
    float base_mode;     // 0: residual to the plain mean; 1: to mean + regression correction
};


// Per-grid data of the learned gather: the pre-scaled index rows (t = A c
// + b, cell = floor(t), as cell_fast), the grid's rotation times the voxel
// size and the cell-centre shift, so that the world-frame offset from the
// cell centre is
//     (h M) (t - floor(t) - 1/2) = (h M) frac(t) + o,  o = -(h M) (1/2, 1/2, 1/2).
// The x and y index rows are stored interleaved, t01[j] = (row0[j], row1[j]),
// so that tx and ty are computed together by paired FP32 FMAs (fma.rn.f32x2).
struct GridRows {
    float2 t01[4];  // (row 0, row 1) coefficients of c.x, c.y, c.z and the constant
    float4 t2;      // row 2: coefficients of c.x, c.y, c.z and the constant
    float m[9];
    float o[3];
};
static_assert(sizeof(GridRows) == 96, "GridRows layout");
// rows[i] for grid i of an ensemble (host), from its FAST rows and rotation.
GridRows make_grid_rows(const FastXf& fast, const float* rot12, float voxel);

int mlp_param_count();
size_t mlp_fragment_bytes();
size_t mlp_train_smem();
// Cell masses into W's .w lane (and the mass grid cleared) after a
// world-frame solve; then the fused gather + features + network + update
// (out_mode 0: step pos/vel; 1: corrected force into out4; 2: features,
// out4 = plain mean force, feat = n x 16).
cudaError_t launch_density_w(const Ensemble& e, void* mass, float4* W, cudaStream_t s);
// Outputs of the learned kernel: out4 / feat as out_mode says; spread (if
// not null, room for 2 * spread_cap floats) receives per-CTA sums of the
// particles' mean grid-to-grid force spread (mean of features 6-8) and of
// their mean-force magnitude (feature 10), both in units of the model's
// force scale, for `blocks` CTAs.
struct LearnedOut {
    float4* out4 = nullptr;
    float* feat = nullptr;
    float* spread = nullptr;
    int spread_cap = 0;
    int blocks = 0;
};
// rows: the ensemble's k GridRows in host memory (they travel in the launch
// parameters when k is one of the compiled ensemble sizes).
cudaError_t launch_learned(int out_mode, const Ensemble& e, const GridRows* rows, float4* pos,
                           float4* vel, int64_t n, const float4* W, const ModelNorm& norm,
                           const void* frags, const float* params, float dt, float damp,
                           LearnedOut& out, cudaStream_t s, int ctas_per_sm = 2);
cudaError_t launch_pack_fragments(const float* params, void* frags, cudaStream_t s);
cudaError_t launch_mlp_train_step(const float* feat, const float* target, const int* idx,
                                  int batch, float* params, float* partial, float* loss_partial,
                                  float* grad, float* m, float* v, float lr, int t,
                                  cudaStream_t s);

}  // namespace mog
