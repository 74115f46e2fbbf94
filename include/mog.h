/*
 * mog.h — C ABI of the B200 (sm_100a) Mixture-of-Grids force-and-step library.
 *
 * The reference (tbmo/mog-solver) runs one particle-mesh gravity step as a
 * sequence of GLSL compute dispatches issued from Python through moderngl
 * (main.py:592-669).  Its state lives in GL buffers owned by the
 * `Simulation` object.  This header is the drop-in boundary that replaces
 * that pipeline: the caller owns the particle buffers (device memory,
 * 16-byte float4 records exactly like the reference's std430 `vec4`
 * SSBOs), the library owns the grids, spectra, tables and graphs.
 *
 * Conventions
 *  - Every pointer named pos4 / vel4 / acc4 is device memory holding n
 *    float4 records (x, y, z, w); pos.w is the particle mass, vel.w is 0
 *    (update.glsl:88-89).
 *  - `stream` is a cudaStream_t passed as void* (0 = legacy default stream).
 *    All work is stream ordered; no entry point synchronises the host
 *    except mog_create, mog_get_status, mog_step_profiled,
 *    mog_diagnostics and mog_render.
 *  - Every entry point returns MOG_OK (0) or an error code; the text of the
 *    last error on the calling thread is available from mog_last_error().
 */
#ifndef MOG_H
#define MOG_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes --------------------------------------------------- */
#define MOG_OK              0
#define MOG_ERR_CONFIG      1  /* invalid configuration value             */
#define MOG_ERR_CUDA        2  /* a CUDA runtime call failed              */
#define MOG_ERR_OVERFLOW    3  /* fixed-point mass total left u64 range   */
#define MOG_ERR_NONFINITE   4  /* a particle position became NaN/Inf      */
#define MOG_ERR_TIMEOUT     5  /* a bounded device wait gave up           */
#define MOG_ERR_ARG         6  /* bad pointer / size argument             */
#define MOG_ERR_UNSUPPORTED 7  /* combination not built (e.g. g > 64)     */

/* ---- enumerations ----------------------------------------------------- */
/* solver switch, config.yaml `solver: fft|convolution` (main.py:125-126)  */
#define MOG_SOLVER_FFT          0
#define MOG_SOLVER_CONVOLUTION  1
/* mass fixed point: u64 with scale 2^scale_bits (deterministic, exact),  */
/* or the reference's uint32(m*1000) truncation (mass.glsl:52-54)          */
#define MOG_MASS_U64_FIXED      0
#define MOG_MASS_U32_X1000      1
/* cell-index arithmetic: FAST = floor((R^T c)/h + (L/2-off)/h) mod g with */
/* a pre-scaled matrix and fused multiply-adds; EXACT = the shader's own   */
/* op sequence (mass.glsl:42-50) with IEEE division and no contraction     */
#define MOG_INDEX_FAST          0
#define MOG_INDEX_EXACT         1
/* spectral transform precision                                             */
#define MOG_DFT_FFT32           0  /* FP32 radix-2 FFT in shared memory      */
#define MOG_DFT_TC_BF16X3       1  /* DFT stages on tcgen05, bf16 hi+lo x3   */
/* MOG_DFT_TC_BF16X3 (fft solver, grid_size 16 or 32): every axis pass of
 * the spectral solve (fft_batched.glsl:45-132) is a dense g-point DFT done
 * as a GEMM on the tensor cores: lines x (2g reals) times the real form of
 * the DFT matrix, inputs split into BF16 hi + lo, three products
 * accumulated in FP32.  About 6e-6 relative L2 from FP64 on the
 * colliding-disk set at k = 240, g = 32 (the FP32 FFT: 2e-7).  Other sizes
 * return MOG_ERR_UNSUPPORTED. */

/* compatibility flags (mog_config.compat_flags) */
/* Reproduce the reference's texture aliasing in run_fft_3d_batched        */
/* (main.py:564-590, 638-646): when 3 (log2 g + 1) is odd (g = 4, 16, 64)  */
/* the z inverse transform reuses the texture holding the finished x       */
/* result, so pack.glsl reads the z-gradient as the x force.  Off by       */
/* default: the library computes the gradient the shaders intend.          */
#define MOG_COMPAT_FFT_TEXTURE_ALIAS 1

/* device status flag bits returned by mog_get_status */
#define MOG_FLAG_NONFINITE  1u
#define MOG_FLAG_OVERFLOW   2u
#define MOG_FLAG_TIMEOUT    4u
#define MOG_FLAG_BADMASS    8u
/* an index outside its buffer was caught and the access skipped; raised
   only by a library built with -DMOG_CHECK (python -m mog_solver_b200.build
   --check), whose kernels bounds-check their scatter and gather indices */
#define MOG_FLAG_BOUNDS    16u

/*
 * Configuration.  Field names follow config.yaml (config.yaml:2-18) and
 * the reference's parse (main.py:115-126); the last block holds the keys
 * this library adds.
 */
typedef struct mog_config {
    int32_t n_grids;        /* k  (config `n_grids`,  main.py:115)          */
    int32_t grid_size;      /* g  (config `grid_size`, main.py:116); 2..64, power of 2 */
    float   world_size;     /* L  (config `world_size`, main.py:117)        */
    float   G;              /* config `G` (main.py:120)                     */
    float   dt;             /* config `dt` (main.py:121)                    */
    float   damping;        /* config `damping`, default 1.0 (main.py:667)  */
    int32_t solver;         /* MOG_SOLVER_*                                 */
    int32_t mass_mode;      /* MOG_MASS_*                                   */
    int32_t scale_bits;     /* u64 mode: q = trunc(m * 2^scale_bits), 0..100 */
    int32_t index_mode;     /* MOG_INDEX_*                                  */
    int32_t dft_prec;       /* MOG_DFT_*                                    */
    int32_t compat_flags;   /* MOG_COMPAT_* bits                            */
    int64_t num_particles;  /* capacity: largest n passed to the step calls */
    float   softening;      /* fft solver: spectral softening radius a in voxels; 0 = the
                               live greens.glsl:17-61 (-2 pi G / k^2); > 0 = the variant
                               commented out in greens.glsl:63-115:
                               -4 pi G exp(-k^2 a^2) / k^2                   */
} mog_config;

typedef struct mog_handle mog_handle;

/*
 * Launch-shape knobs: the interface of the project's autotuner
 * (mog_solver_b200/autotune.py).  No counterpart in the reference, whose
 * dispatch shapes are fixed in main.py:596-668.  Zero means "library
 * default" for every field except update_staged (-1 = automatic).
 */
typedef struct mog_tuning {
    int32_t deposit_threads;        /* threads per deposit CTA, 64..1024, multiple of 32 */
    int32_t deposit_grids_per_cta;  /* grids per CTA histogram; -1 = global atomics        */
    int32_t deposit_chunks;         /* particle chunks per grid group                       */
    int32_t deposit_ppt;            /* particles per thread in the deposit: 1, 2 or 4       */
    int32_t update_staged;          /* -1 auto, 0 gathers from L2, 1 shared-memory staged    */
    int32_t update_ctas;            /* CTAs of the staged gather (0 = one per SM)            */
    int32_t sort_every;             /* spatial re-ordering period in steps; 0 = never (default) */
    int32_t update_direct_ppt;      /* particles per thread of the L2-gather update: 1, 2, 4;
                                       0 auto (4 from 8 x 256 threads per SM, else 1)       */
    int32_t deposit_aggregate;      /* warp-merge runs of equal cells: -1 auto, 0 off, 1 on  */
    int32_t deposit_generic;        /* 1: never use the specialised g <= 16 deposit kernel    */
    int32_t deposit_sorted;         /* 1: deposit from the spatially ordered copy too         */
    int32_t update_threads;         /* staged gather block: 512, 768 or 1024; 0 auto (512)   */
    int32_t deposit_split;          /* u64 shared histogram of high words only (low halves as
                                       global atomics; none for equal power-of-two masses):
                                       0 auto (g = 32), 1 also at g = 8 and 16, -1 never;
                                       2 = one word per cell counting the particles of a CTA's
                                       first mass (uniform masses of any value; any other mass
                                       takes a global atomic), at g = 8, 16 and 32            */
    int32_t learned_fold;           /* learned step: 0 (default) or 1 = the fft solve's epilogue
                                       writes the cell masses (one launch fewer at g = 8, 16),
                                       -1 = a separate pass                                     */
    int32_t learned_ctas_per_sm;    /* learned kernel occupancy: 0 auto (2), 2 or 3 CTAs of 256
                                       threads per SM (register budget 128, or 80 with spills) */
    int32_t solve_split;            /* g = 8, 16 fft solve: 1 = a cluster of 3 CTAs per grid pair
                                       (one gradient field each), -1 = one CTA per pair, 0 auto
                                       (clusters while 3 x pairs <= SMs); same forces either way */
} mog_tuning;

/* Fill a config with the reference's in-code defaults (main.py:179-189). */
int mog_config_default(mog_config* cfg);

/*
 * Create a solver.  rot12 is k x 12 floats, off4 is k x 4 floats, both in
 * host memory, packed exactly as the reference's compute_transforms
 * (main.py:157-172): rotations[i][4j..4j+2] = row j of the rotation
 * matrix M_i, offsets[i][0..2] = offset of grid i.  Replaces
 * Simulation.__init__ buffer/texture/shader set-up (main.py:191-248).
 */
int mog_create(const mog_config* cfg, const float* rot12, const float* off4,
               mog_handle** out);

/* Release every device resource of the handle. */
int mog_destroy(mog_handle* h);

/*
 * One step: deposit -> spectral solve -> gather/rotate/average ->
 * leapfrog with damping, in place on pos4/vel4.  Replaces
 * Simulation.step / step_fft (main.py:592-672).  dt_eff is the step's
 * deltaTime = dt * timescale (main.py:662); negative values run backwards.
 */
int mog_step(mog_handle* h, float* pos4, float* vel4, int64_t n,
             float dt_eff, void* stream);

/*
 * n_steps steps replayed from a CUDA graph captured once per
 * (pos4, vel4, n, dt_eff) combination.  Same result as n_steps calls of
 * mog_step (the frame loop of main.py:674-676, without rendering).
 */
int mog_step_n(mog_handle* h, float* pos4, float* vel4, int64_t n,
               float dt_eff, int32_t n_steps, void* stream);

/*
 * Ensemble-averaged force at every particle (the avgForce of
 * update.glsl:81) without moving anything: acc4[p] = (Fx, Fy, Fz, 0).
 * Used for accuracy measurements and by the learned correction.
 */
int mog_forces(mog_handle* h, const float* pos4, float* acc4, int64_t n,
               void* stream);

/*
 * Stage entry points (parity testing and custom pipelines).
 *
 * mog_deposit: mass.glsl:27-55 into a caller buffer of k*g^3 cells
 *   (uint64 in MOG_MASS_U64_FIXED mode, uint32 in MOG_MASS_U32_X1000 mode).
 *   The buffer is zeroed first (main.py:558-562).
 * mog_solve: complex.glsl + fft_batched.glsl + fourier.glsl + greens.glsl
 *   + pack.glsl from a caller mass grid to a caller force grid of k*g^3
 *   float4 (fx, fy, fz, |f|) in each grid's own frame (the reference's
 *   gradient texture layout, pack.glsl:23-29).
 * mog_update: update.glsl:53-89 from a caller force grid in that same
 *   layout.
 */
int mog_deposit(mog_handle* h, const float* pos4, int64_t n, void* mass_out,
                void* stream);
int mog_solve(mog_handle* h, const void* mass_in, float* force4_out,
              void* stream);
int mog_update(mog_handle* h, float* pos4, float* vel4, int64_t n,
               const float* force4_in, float dt_eff, void* stream);

/*
 * mog_step with CUDA events recorded on `stream` between its kernels;
 * phase_ms[0..3] receive the device time of the spatial ordering (0 when
 * this step does not re-order), the deposit, the solve and the
 * gather/update.  Synchronises the stream (measurement only).
 */
int mog_step_profiled(mog_handle* h, float* pos4, float* vel4, int64_t n,
                      float dt_eff, float* phase_ms, void* stream);

/* Read / replace the handle's launch shapes (drops cached CUDA graphs). */
int mog_get_tuning(const mog_handle* h, mog_tuning* out);
int mog_set_tuning(mog_handle* h, const mog_tuning* t);

/*
 * Reads (and clears) the device status word: OR of MOG_FLAG_* bits raised
 * since the last call.  Synchronises the handle's work on `stream`.
 */
int mog_get_status(mog_handle* h, uint32_t* flags, void* stream);

/* ---- sharded step over peer memory --------------------------------------
 * One simulation's particles split over `world` GPUs (<= 8), one handle per
 * rank, every handle created with the same config, transforms and
 * scale_bits (no counterpart in the reference, which runs on one GL
 * context).  Grid i belongs to rank floor(i * world / k).  The deposit
 * adds each rank's cells straight into the owner's accumulation buffer with
 * system-scope atomics over NVLink; the exchange waits (bounded) for every
 * rank's deposit and copies the owners' slices into the local grid.  The
 * integer total is exact, so the trajectory is bit-identical to one handle
 * stepping all particles, for any split.  Every rank must make the same
 * calls in the same order.
 *
 * mog_shard_init       allocate this rank's accumulation (3 x k g^3 cells)
 *                      and flags; synchronises.
 * mog_shard_export     64-byte CUDA IPC handles of those two buffers.
 * mog_shard_connect    open the other ranks' handles (world x 64 bytes
 *                      each, in rank order; this rank's entry is ignored).
 * mog_shard_connect_local  the same for ranks held in this process
 *                      (peers[q] = rank q's handle; peer access is enabled
 *                      between different devices).
 * mog_shard_deposit    deposit this rank's particles, then signal.
 * mog_shard_exchange   wait for all ranks, gather the total grid.  A wait
 *                      that runs out raises MOG_FLAG_TIMEOUT.
 * mog_shard_finish     solve and update this rank's particles.
 * mog_shard_step       the last three in order.
 * Destroy the handles only after every rank has finished its last step.
 */
int mog_shard_init(mog_handle* h, int32_t rank, int32_t world);
int mog_shard_export(const mog_handle* h, uint8_t* accum_ipc, uint8_t* flags_ipc);
int mog_shard_connect(mog_handle* h, const uint8_t* accum_ipcs, const uint8_t* flags_ipcs);
int mog_shard_connect_local(mog_handle* h, mog_handle* const* peers);
int mog_shard_deposit(mog_handle* h, const float* pos4, int64_t n, void* stream);
int mog_shard_exchange(mog_handle* h, void* stream);
int mog_shard_finish(mog_handle* h, float* pos4, float* vel4, int64_t n, float dt_eff,
                     void* stream);
int mog_shard_step(mog_handle* h, float* pos4, float* vel4, int64_t n, float dt_eff, void* stream);

/*
 * Failure-detection self-test (no counterpart in the reference): one
 * device wait that nothing satisfies, bounded like every wait in the
 * library's kernels (about 2^31 SM cycles, a second).  It gives up, raises
 * MOG_FLAG_TIMEOUT in the handle's status word and returns, leaving the
 * context usable; mog_get_status then reports it.  Stream ordered.
 */
int mog_selftest_wait_timeout(mog_handle* h, void* stream);

/*
 * FP64 diagnostics of a particle set: out[0..2] = total momentum
 * sum(m v), out[3] = kinetic energy sum(m |v|^2 / 2), out[4] = total
 * mass, out[5..7] = centre of mass.  No counterpart in the reference,
 * which prints nothing but its configuration (main.py:147-155).
 */
int mog_diagnostics(mog_handle* h, const float* pos4, const float* vel4,
                    int64_t n, double* out8, void* stream);

/*
 * FP64 direct-sum yardstick of force accuracy (no counterpart in the
 * reference).  For each of nt target records (device float4, w ignored)
 * sums over ns source records (device float4, w = mass):
 *     out3[t] = g_eff * sum_j m_j d / (|d|^2 + soft^2)^(3/2),
 * d = target - source wrapped to the minimum image of a periodic box of
 * side `world`.  With g_eff = G h^3 / 2 this is the Newtonian field in the
 * solver's units (greens.glsl:40, pack.glsl:21).  out3: device, nt x 3
 * doubles.  Deterministic (fixed-order reduction); synchronous-free.
 */
int mog_direct_sum(const float* targets4, int64_t nt, const float* sources4, int64_t ns,
                   double world, double g_eff, double soft, double* out3, void* stream);

/*
 * mog_direct_sum without any device allocation.  No counterpart in the
 * reference.  mog_direct_sum takes its partial sums from a stream-ordered
 * allocation, which some callers cannot make: a process whose device memory
 * is already held by its own caching allocator (a framework that has grown
 * its pool to fill the GPU), or a device or driver without stream-ordered
 * memory pools.  This entry point writes the partial sums into a fixed
 * 12 MiB scratch that is part of the library image on each device instead,
 * and returns the same result as mog_direct_sum bit for bit (same source
 * chunking, same summation order).
 *
 * Limit: nt * chunks <= 524288, chunks = min(32, ceil(ns / 8192)) (at least
 * 1); so at most 16384 targets once ns > 253952.  Larger requests return
 * MOG_ERR_ARG with the limit in mog_last_error() and launch nothing.
 * The first call on each device does a one-time set-up (it looks up the
 * scratch's device address); make that first call before any stream
 * capture begins.  The looked-up address is kept for the life of the
 * process, so the device's primary context must not be reset in between
 * (cudaDeviceReset would unload the library's module and leave the kept
 * address pointing at freed memory).  Nothing in the scratch needs to start at zero: every
 * partial sum a call reads was written earlier in the same call.  All
 * calls on one device share the one scratch, so calls that overlap in time
 * (other streams, other threads) race with one another and must be
 * serialised by the caller.
 */
int mog_direct_sum_noalloc(const float* targets4, int64_t nt, const float* sources4,
                           int64_t ns, double world, double g_eff, double soft, double* out3,
                           void* stream);

/*
 * Batched independent simulations (the "batched uneven
 * ensemble"; no counterpart in the reference, which runs one simulation per
 * window).  A batch groups `count` handles on one device.  mog_batch_step
 * advances every simulation n_steps steps; each ensemble step is ONE CUDA
 * graph launch in which every simulation's kernels run on its own branch,
 * so small and large simulations overlap on the GPU.  The graph is captured
 * once per combination of (pos4[i], vel4[i], n[i], dt_eff[i]).  Spatial
 * re-ordering inside a batch happens on every step when a handle's
 * sort_every is 1 and never otherwise.
 */
typedef struct mog_batch mog_batch;
int mog_batch_create(mog_handle* const* handles, int32_t count, mog_batch** out);
int mog_batch_step(mog_batch* b, float* const* pos4, float* const* vel4, const int64_t* n,
                   const float* dt_eff, int32_t n_steps, void* stream);
int mog_batch_destroy(mog_batch* b);

/*
 * Launch shapes of a batch.  work_queue = 1 (default): when every
 * simulation uses the FFT solver, FAST cell indices, no spatial
 * re-ordering, g = 8, 16 or 32 and one shared mass mode, an ensemble step
 * is ONE persistent work-queue deposit over all simulations, each
 * simulation's solve on its own graph branch, and ONE persistent
 * work-queue gather + update over all simulations; every CTA pops tiles
 * (simulation, grid group, particle chunk) / (simulation, particle chunk)
 * from a largest-first list until it runs out.  Otherwise (or with
 * work_queue = 0) each simulation's three kernels run on their own branch.
 * deposit_chunk: particles per deposit tile (0 = 393216; else >= 1024).
 * deposit_split: 1 = u64 grids keep only their high words in the work-queue
 * deposit's shared memory at g = 8 and 16 too (twice the grids per tile;
 * pays when every mass has a zero fixed-point low half, which then needs no
 * global atomic), 0 = only at g = 32; 2 = one word per cell counting the
 * particles of a tile's first mass at every g (uniform masses of any value;
 * any other mass takes a global atomic).
 * The result never depends on these.  mog_batch_get_tuning also reports
 * whether the work-queue launches apply (active_work_queue, read only).
 */
typedef struct mog_batch_tuning {
    int32_t work_queue;
    int32_t deposit_chunk;
    int32_t active_work_queue;
    int32_t deposit_split;
} mog_batch_tuning;
int mog_batch_set_tuning(mog_batch* b, const mog_batch_tuning* t);
int mog_batch_get_tuning(const mog_batch* b, mog_batch_tuning* t);

/*
 * Learned correction of a cheap ensemble (no counterpart in the reference,
 * whose force is always the plain k-grid average, update.glsl:67-81).
 * A model is a 12 -> 64 -> 64 -> 3 GELU network predicting, from per-particle
 * statistics of the handle's ensemble, the residual to a larger ensemble.
 *   params: MOG_MODEL_PARAMS floats, W1[64][12] b1[64] W2[64][64] b2[64]
 *           W3[3][64] b3[3] (FP32 master copy; inference runs in FP16).
 *   norm:   MOG_MODEL_NORM floats, mu[12] inv_sigma[12] force_scale
 *           rho_ref out_scale base_mode — features are (f - mu) * inv_sigma
 *           with forces divided by force_scale and densities by rho_ref;
 *           the predicted residual is y * out_scale, added to the plain
 *           ensemble mean (base_mode 0) or to the mean plus the per-particle
 *           least-squares correction carried in feature slots 12-14
 *           (base_mode 1).
 */
#define MOG_MODEL_PARAMS 5187
#define MOG_MODEL_NORM 28
typedef struct mog_model mog_model;
int mog_model_create(mog_model** out);
int mog_model_destroy(mog_model* m);
/* Upload parameters and normalisation (host memory); resets Adam state. */
int mog_model_set(mog_model* m, const float* params, const float* norm);
/* Download parameters and normalisation to host memory (synchronises). */
int mog_model_get(const mog_model* m, float* params, float* norm);
/*
 * One Adam step (lr; betas 0.9, 0.999) on the mean squared error of the
 * `batch` samples idx[0..batch) of feat16 (device, rows of 16 floats, the
 * first 12 used) against target4 (device, rows of 4 floats, 3 used).
 * Optional outputs: *loss_out (host; synchronises) and grad_out (device,
 * MOG_MODEL_PARAMS floats).  lr = 0 computes the gradient only.
 */
int mog_model_train_step(mog_model* m, const float* feat16, const float* target4,
                         const int* idx, int32_t batch, float lr, float* loss_out,
                         float* grad_out, void* stream);
/*
 * Deposit + solve with the handle's ensemble, then per-particle features:
 * mean4_out (device n float4, the plain ensemble force) and feat16_out
 * (device n x 16 floats: 0-11 standardised with m's norm, 12-14 the
 * least-squares correction in force units, 15 zero).
 */
int mog_features(mog_handle* h, const mog_model* m, const float* pos4, int64_t n,
                 float* mean4_out, float* feat16_out, void* stream);
/* Corrected force (base force of m's base_mode + predicted residual) at every
 * particle, and one damped leapfrog step with it (update.glsl:83-89). */
int mog_learned_forces(mog_handle* h, const mog_model* m, const float* pos4, float* acc4,
                       int64_t n, void* stream);
int mog_learned_step(mog_handle* h, const mog_model* m, float* pos4, float* vel4, int64_t n,
                     float dt_eff, void* stream);
/*
 * mog_learned_step with CUDA events between its kernels: phase_ms[0..3]
 * receive the device time of the deposit, the solve, the cell-mass pass and
 * the fused gather + network + update kernel.  Synchronises the stream.
 */
int mog_learned_step_profiled(mog_handle* h, const mog_model* m, float* pos4, float* vel4,
                              int64_t n, float dt_eff, float* phase_ms, void* stream);
/*
 * Statistics of the particles of the last mog_learned_step, summed per CTA
 * by that step's own kernel in a fixed order: out2[0] = the mean over
 * particles of their grid-to-grid force spread (mean of features 6-8
 * before standardisation), out2[1] = the mean of their ensemble-mean force
 * magnitude (feature 10); both in units of the model's force_scale.  The
 * variance gate of the learned path compares their ratio with the one of
 * its training data.  Zeros before the first learned step.  Synchronises
 * the stream.
 */
int mog_learned_spread(mog_handle* h, double* out2, void* stream);

/*
 * mog_step / mog_learned_step over particles held in HOST memory, for a
 * caller whose particle state lives on the host between steps (the
 * reference's Simulation.step with its buffers read back every frame,
 * main.py:592-676).  pos4_host / vel4_host: n float4 records in host
 * memory, page-locked (cudaHostAlloc / cudaHostRegister) for the copies to
 * run asynchronously; pageable memory works but serialises them.  The
 * particles travel in `chunks` pieces (1..64; 4 to 8 overlap best): each
 * chunk's positions are deposited as soon as they land, and after the
 * solve each chunk is updated (the learned kernel; the plain gather runs
 * as one launch) and copied back while later chunks still compute, so the
 * copies in both directions overlap the kernels.  The handle keeps device
 * copies of the records (2 n float4, allocated on the first call and when
 * n grows) and two copy streams.  Everything is queued on `stream`; the
 * host buffers hold the stepped particles once `stream` reaches the end of
 * the call (synchronise it before reading them).  The result is bit-identical
 * to copying the records to the device, stepping there and copying back.
 * The variance-gate statistics of mog_learned_spread cover the whole step.
 */
int mog_step_host(mog_handle* h, float* pos4_host, float* vel4_host, int64_t n, float dt_eff,
                  int32_t chunks, void* stream);
int mog_learned_step_host(mog_handle* h, const mog_model* m, float* pos4_host, float* vel4_host,
                          int64_t n, float dt_eff, int32_t chunks, void* stream);

/*
 * The Green's factor table the spectral solve multiplies by, g^3 floats in
 * [kz][ky][kx] order, written to host memory `out`: -2 pi G / k^2
 * (softening 0) or -4 pi G exp(-k^2 a^2) / k^2 with a = softening * L / g,
 * in FP64 then rounded to FP32; 0 where the reference's FP32 k^2 <= 1e-4
 * (greens.glsl:17-47).  Host only, no GPU needed.  No counterpart in the
 * reference (it builds the factor per bin in the shader).  For softening 0
 * the library builds the same table on the GPU, equal to this one up to the
 * last bit of k^2.
 */
int mog_green_table(int32_t g, float world, float G, float softening, float* out);

/*
 * The reference's initial-condition sampler, init_particles.glsl (DIM 3) as
 * init_particles_gpu dispatches it (main.py:283-310): particle i draws
 * candidates from an integer hash of seed + 12345 i (inside a sphere,
 * shape 1, or a cube, shape 0, of the world shrunk by spawn_buffer * L on
 * every side), keeps the first whose random threshold falls below
 * clamp(fbm + 1/2, 0, 1)^contrast (4-octave Perlin noise at
 * noise_scale / L), falls back to a uniform draw after 64 tries, and gets
 * a velocity uniform in [-L/2, L/2)^3.  pos4 / vel4: n float4 records
 * (x, y, z, mass) and (vx, vy, vz, 0); n < 2^32.  The reference's default
 * call is noise_scale 4, contrast 2, seed 12345, spawn_buffer 0.1, shape 1.
 * mog_init_particles: device buffers, on `stream` (no synchronisation).
 * mog_init_particles_host: host buffers, on the host (no GPU needed); the
 * same arithmetic, with the host math library's cos, sin, acos and pow.
 */
int mog_init_particles(float* pos4, float* vel4, int64_t n, float world, float noise_scale,
                       float contrast, uint32_t seed, float mass, float spawn_buffer,
                       int32_t shape, void* stream);
int mog_init_particles_host(float* pos4, float* vel4, int64_t n, float world, float noise_scale,
                            float contrast, uint32_t seed, float mass, float spawn_buffer,
                            int32_t shape);

/*
 * The reference's two-galaxy initialiser, Simulation.init_particles2
 * (main.py:312-357), on the GPU.  Two spherical exponential blobs (scale
 * 0.08 L) at L/2 -/+ 0.2 L along x with bulk velocities +/-(0.3, 0.1, 0),
 * each spinning about its own axis with speed 0.3 sqrt(r / L + 0.01); the
 * first n/2 records form galaxy 0, the next n/2 galaxy 1, an odd last
 * record stays zero.  The reference draws from NumPy's sequential global
 * generator; here particle i takes its three uniforms from a counter-based
 * generator keyed by `seed` (SplitMix64), so the particle set has the
 * reference's distribution but not its exact draws (for those, use the
 * host routine ics.reference_two_galaxies).  Formulas in FP64, stored as
 * FP32 records (x, y, z, mass) / (vx, vy, vz, 0).
 * mog_init_two_galaxies: device buffers, on `stream`.
 * mog_init_two_galaxies_host: host buffers, the same function on the host
 * (the host math library's log, sin, cos, acos, sqrt).
 */
int mog_init_two_galaxies(float* pos4, float* vel4, int64_t n, float world, float mass,
                          uint64_t seed, void* stream);
int mog_init_two_galaxies_host(float* pos4, float* vel4, int64_t n, float world, float mass,
                               uint64_t seed);

/* ---- headless particle renderer ---------------------------------------
 * Replaces the reference's particle draw (vertex and fragment shaders,
 * main.py:359-423; on_render, main.py:678-703) with CUDA kernels writing
 * an image into a device buffer, under OpenGL's rules for points: clip to
 * the view volume, square points, gl_PointCoord, and SRC_ALPHA /
 * ONE_MINUS_SRC_ALPHA blending in particle index order on every pixel.
 * The reference never enables GL_PROGRAM_POINT_SIZE, so its points have
 * the fixed size 1; point_mode 1 uses the shader's 800 / (w + 0.1).
 * Rows are stored top row first; each pixel is 4 channels, RGBA. */
#define MOG_RENDER_RGBA8   0  /* 8-bit target: round(clamp(c) * 255) after every blend */
#define MOG_RENDER_RGBA32F 1  /* float target: no rounding, no clamping */

typedef struct mog_render_params {
    int32_t width, height;   /* pixels (the reference's window is 2560 x 1440, main.py:104) */
    float   world_size;      /* the world_size uniform */
    float   speed_scale;     /* the speed_scale uniform (main.py:419 sets 0.0) */
    float   m_view[16];      /* the m_view uniform, column-major: the bytes on_render writes */
    float   m_proj[16];      /* the m_proj uniform, column-major */
    float   clear[4];        /* clear colour (main.py:681: 0.01, 0.01, 0.02; alpha 0) */
    int32_t point_mode;      /* 0: every point point_size pixels wide; 1: the shader's size */
    float   point_size;      /* 1.0, the GL default */
    float   max_point_size;  /* sizes are clamped to [1, max_point_size] */
    int32_t format;          /* MOG_RENDER_RGBA8 or MOG_RENDER_RGBA32F */
} mog_render_params;

typedef struct mog_renderer mog_renderer;

/* Defaults: the reference's uniforms and GL state, 2560 x 1440, identity
 * matrices (the caller writes the camera's). */
void mog_render_params_default(mog_render_params* p);

/* A renderer owns its device scratch (grown on demand). */
int mog_renderer_create(mog_renderer** out);
int mog_renderer_destroy(mog_renderer* r);

/*
 * Draws n particles (device pos4 / vel4, as the step uses them) into the
 * device buffer `image` (width x height x 4 bytes for RGBA8, x 4 floats
 * for RGBA32F), on `stream`.  It waits for the stream once, to size the
 * tile lists.  MOG_ERR_UNSUPPORTED if the points touch more than 2^31 - 1
 * (point, tile) pairs.
 */
int mog_render(mog_renderer* r, const mog_render_params* p, const float* pos4,
               const float* vel4, int64_t n, void* image, void* stream);

/* The last frame's (point, tile) pair count and number of kernel launches. */
int mog_renderer_stats(const mog_renderer* r, int64_t* pairs, int32_t* launches);

/* The same image from host buffers, on the host (no GPU needed), bit for bit. */
int mog_render_host(const mog_render_params* p, const float* pos4, const float* vel4,
                    int64_t n, void* image);

/* Human-readable text for a status code, and the calling thread's last
 * error message. */
const char* mog_strerror(int code);
const char* mog_last_error(void);

/* Library version string. */
const char* mog_version(void);

#ifdef __cplusplus
}
#endif

#endif /* MOG_H */
