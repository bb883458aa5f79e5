/*
 * phix_b200.h -- C ABI of the B200-native PhiX time-step library
 * (libphix_b200.so, built from phix_b200/csrc for sm_100a).
 *
 * Every entry point takes plain device pointers, sizes and POD descriptors,
 * never throws, and returns PHIX_OK (0) or a negative status; the message of
 * the last failure on the calling thread is available from phix_last_error().
 * The C++ drop-in API (include/phix/...) turns a negative status into the
 * exception type the reference throws (std::runtime_error for CUDA failures,
 * std::invalid_argument for shape and argument errors).
 *
 * Field layout.  A field is the reference's ghost-padded stored array
 * (ScalarField.h:15-27): stored dims n[a] + 2*ghost on every axis, unused
 * axes of 1-D/2-D meshes included, x fastest, FP64.  Kernels write physical
 * cells; ghost cells are only ever filled the way the reference fills them.
 *
 * Streams.  `stream` arguments are cudaStream_t values passed as void*;
 * NULL means the legacy default stream.  Calls are asynchronous unless the
 * name says otherwise.
 */
#ifndef PHIX_B200_H
#define PHIX_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PHIX_ABI_VERSION 1

/* status codes */
#define PHIX_OK 0
#define PHIX_ERR_ARG (-1)         /* bad argument / shape (std::invalid_argument) */
#define PHIX_ERR_CUDA (-2)        /* CUDA runtime failure (std::runtime_error)     */
#define PHIX_ERR_UNSUPPORTED (-3) /* combination not built                        */
#define PHIX_ERR_NONFINITE (-4)   /* diagnostics found NaN/Inf in a field         */
#define PHIX_ERR_TIMEOUT (-5)     /* a bounded device-side wait gave up           */

/* boundary condition kinds, per axis side (Boundary.cu:95-195) */
#define PHIX_BC_NONE 0     /* ghost cells left as stored                    */
#define PHIX_BC_PERIODIC 1 /* PeriodicBC: ghost <- opposite physical layer  */
#define PHIX_BC_NOFLUX 2   /* NoFluxBC: ghost <- nearest physical cell      */
#define PHIX_BC_FIXED 3    /* FixedBC: ghost <- constant bc_val             */

/* built-in physics (right-hand sides of the reference's drivers) */
#define PHIX_PHYS_AC 0   /* prm = [L, kappa]:  L*kappa*lap(phi) + L*pw(phi, p - p^3)          */
#define PHIX_PHYS_CH 1   /* prm = [M, kappa, rho, ca, cb]:  M*lap(f'(c) - kappa*lap(c), bcs),
                            f'(c) = 2 rho (c-ca)(c-cb)(2c-ca-cb)                               */
#define PHIX_PHYS_CHAC 2 /* prm = [M, L, kappa_c, kappa_eta, lambda]; fields (c, eta):
                            c  : M*lap(f_c(c,eta) - kappa_c*lap(c), bcs)
                            eta: (-L)*f_eta(eta,c) + (L*kappa_eta)*lap(eta)
                            f = c^2(1-c)^2 + eta^2(1-eta)^2 + lambda c^2 eta^2                 */

/* time schemes (Solver.h:17-20) */
#define PHIX_EULER 0
#define PHIX_RK4 1
/* Multi-step Euler of the shipped Cahn-Hilliard app (PHIX_PHYS_CH only, 1-D/2-D,
 * ghost 1): fields (c, mu); per step mu = f'(c) - kappa*lap(c) (STEADY) and
 * c += dt*M*lap(mu) (TRANSIENT), one launch.  Replaces Solver(steps, dt) with
 * {&c, bcs, &eqMu, STEADY}, {&mu, bcs, &eqC, TRANSIENT} (Solver.cu:112-144,
 * :317-340).  mu always stays in the caller's / first buffer. */
#define PHIX_MULTISTEP 2

/* arithmetic of the stencil kernels */
#define PHIX_F64 0
#define PHIX_F32 1

/* Mesh + boundary description.  n[a] = 1 and d[a] = 1 for unused axes. */
typedef struct {
    int32_t dim;        /* 1, 2 or 3                                   */
    int32_t n[3];       /* physical cells per axis                     */
    int32_t ghost;      /* ghost layers of the stored layout (>= 1)    */
    int32_t bc_type[6]; /* [2*axis + side], side 0 = low, 1 = high     */
    int32_t reserved;   /* must be 0                                   */
    double d[3];        /* spacing                                     */
    double bc_val[6];   /* value for PHIX_BC_FIXED sides               */
} phix_grid_t;

typedef struct phix_stepper phix_stepper_t;

/* ---- library ---------------------------------------------------------- */
int phix_abi_version(void);
const char* phix_last_error(void);
/* Number of kernel launches this library has issued in this process. */
long long phix_launch_count(void);

/* ---- single operators (replace the reference's per-term kernels) ------- */

/* Ghost refresh with every BC of `g`, in buildBCs order.
 * Replaces PeriodicBC/NoFluxBC/FixedBC::applyOnGPU (Boundary.cu:224-351). */
int phix_bc_apply(double* field, const phix_grid_t* g, void* stream);

/* rhs += coeff * lap(src) on physical cells.
 * Replaces kernel_lap_accumulate + lap(f) (Equation.cu:40-80, :130-183). */
int phix_lap_accumulate(double* rhs, const double* src, double coeff, const phix_grid_t* g, void* stream);

/* rhs += coeff * d(src)/dx_axis, central difference.
 * Replaces kernel_grad_accumulate + grad(f, axis) (Equation.cu:89-124, :185-240). */
int phix_grad_accumulate(double* rhs, const double* src, double coeff, int axis, const phix_grid_t* g,
                         void* stream);

/* Built-in pointwise functors for phix_pointwise_accumulate. */
#define PHIX_PW_IDENT 0  /* f(a)    = a                                   */
#define PHIX_PW_AC 1     /* f(a)    = a - a^3   (tutorials/quickstart)    */
#define PHIX_PW_DW 2     /* f(a)    = 2 rho (a-ca)(a-cb)(2a-ca-cb), prm = physics CH prm */
#define PHIX_PW_CHAC_C 3 /* f(c,e)  = f_c of PHIX_PHYS_CHAC, prm[4] = lambda              */
#define PHIX_PW_CHAC_E 4 /* f(e,c)  = f_eta of PHIX_PHYS_CHAC, prm[4] = lambda            */
#define PHIX_PW_MUL 5    /* f(a,b)  = a*b                                 */

/* rhs += coeff * f(s1[, s2]) on physical cells.
 * Replaces kernel_pw_accumulate / kernel_pw2_accumulate (TermPW.inl:18-63)
 * for the functors above (user functors are instantiated by the C++ API). */
int phix_pointwise_accumulate(double* rhs, const double* s1, const double* s2, double coeff, int func,
                              const double* prm, const phix_grid_t* g, void* stream);

/* rhs += coeff * s1 * s2 on physical cells.
 * Replaces kernel_mul_accumulate (Equation.cu:386-404). */
int phix_mul_accumulate(double* rhs, const double* s1, const double* s2, double coeff, const phix_grid_t* g,
                        void* stream);

/* dst[i] += coeff * src[i] over n stored elements.
 * Replaces kernel_axpy (Solver.cu:30-35). */
int phix_axpy(double* dst, const double* src, double coeff, size_t n, void* stream);

/* ---- fused time stepper (Solver / VectorSolver replacement) ------------ */

/* Create a stepper for one built-in physics.  It owns the stage buffers
 * (RK4: k1..k3 per field), a second state buffer per field, an internal
 * stream and any captured CUDA graphs.  precision = PHIX_F64 works on the
 * reference layout in FP64; PHIX_F32 keeps an FP32 copy of the state and
 * runs the stencil arithmetic in FP32.
 * Replaces Solver(Equation&, bcs, dt, scheme) (Solver.cu:86-107) and
 * VectorSolver (VectorSolver.cu:77-100). */
int phix_stepper_create(phix_stepper_t** out, int phys, int scheme, int precision, const double* prm, double dt,
                        const phix_grid_t* g);
int phix_stepper_destroy(phix_stepper_t* h);
int phix_stepper_nfields(const phix_stepper_t* h);

/* Copy the state in from / out to FP64 stored device arrays (one per field),
 * converting precision when the stepper is FP32.  Ordered on `stream`. */
int phix_stepper_load(phix_stepper_t* h, const double* const* fields, void* stream);
int phix_stepper_store(phix_stepper_t* h, double* const* fields, void* stream);

/* Advance nsteps time steps on `stream`.  Each step is one launch per RK
 * stage (4 for RK4, 1 for Euler) with the BCs, the stage combination and the
 * final update fused in; a single-field 2-D RK4 step whose sides are all
 * periodic or zero-flux is one launch for all four stages, and a 3-D RK4 step
 * of CH or CH+AC with z periodic and x, y periodic or zero-flux is two
 * launches of two fused stages each, input planes staged by TMA (see
 * phix_stepper_set_fusion).  When steps_per_graph > 0 (see
 * phix_stepper_set_graph) whole groups of steps replay as one CUDA graph.
 * Replaces Solver::advance / VectorSolver::advance (Solver.cu:366-382;
 * VectorSolver.cu:186-228). */
int phix_stepper_advance(phix_stepper_t* h, int nsteps, void* stream);

/* Reads and clears the stepper's device error flag: PHIX_ERR_TIMEOUT if a
 * fused 3-D step gave up waiting (2 s) for a plane copy since the last check
 * (its CTA returned without writing that part of the step), else PHIX_OK.
 * Synchronous on `stream`.  No reference counterpart. */
int phix_stepper_status(phix_stepper_t* h, void* stream);

/* Replay groups of `steps_per_graph` steps from a captured CUDA graph
 * (0 disables graphs).  Replaces the driver step loop (Solver::run,
 * Solver.cu:405-414) between callbacks. */
int phix_stepper_set_graph(phix_stepper_t* h, int steps_per_graph);

/* 1: where supported, run each RK4 step as one launch that keeps the four
 * stage states in shared memory and recomputes the tile halos; 0: one launch
 * per stage.  Both give the same bits.  Default: 1 for FP32 steppers and for
 * FP64 CH steppers whose four sides are periodic (the pair kernels), else 0
 * (the faster of the two on B200 for each).  PHIX_MULTISTEP steppers on 2-D
 * grids with four periodic sides: 1 (default) runs the pair-layout step,
 * 0 the box-tile step; one launch per step either way, same bits.  No
 * reference counterpart (the reference runs each term and stage as its own
 * kernels). */
int phix_stepper_set_fusion(phix_stepper_t* h, int one_launch_per_step);
/* (3-D CH / CH+AC RK4: 1 = the two-launch fused step, 0 = one launch per
 * stage; same bits.) */

/* Kernel launches one time step takes with the current settings (per launch
 * when one launch advances several steps, see phix_stepper_depth). */
int phix_stepper_launches_per_step(const phix_stepper_t* h);
/* Temporal-block depth of the current settings: time steps one launch
 * advances (2 for the temporally blocked pair tiles of phix_stepper_set_tiles,
 * else 1).  No reference counterpart. */
int phix_stepper_depth(const phix_stepper_t* h);

/* Tile shape of the 2-D kernels.  One launch per stage: -1 the box tiles
 * (64x16, 256 threads, flat cell loops), 0..3 column-walking tiles (TX x TY =
 * 64x16, 64x32, 128x16, 32x16 with 4, 4, 2, 8 row groups; 256 threads).  One
 * launch per RK4 step: 0..5 cell-per-thread tiles of 64x16, 64x32, 128x16,
 * 128x32 (512 threads), 128x64 and 256x32 (1024 threads; FP32 only);
 * 6..15 pair tiles (CH with four periodic sides; two cells per thread) of
 * 128x64, 128x32, 128x32, 128x16, 64x32, 64x64, 256x32, 128x28, 64x28, 64x16
 * with 8, 8, 4, 4, 8, 8, 4, 8, 8, 4 row blocks; 16..19 temporally blocked
 * pair tiles (two RK4 steps per launch on a 16-cell halo, see
 * phix_stepper_depth) of 64x32, 64x16, 128x16, 64x28 with 8, 4, 4, 8 row
 * blocks.  Shapes that do not fit in
 * shared memory for the precision are refused when the step runs.
 * PHIX_MULTISTEP steppers with the pair-layout step: 0..5 pair tiles of
 * 128x32, 64x32, 128x16, 64x16, 64x64, 256x16 with 8, 8, 4, 4, 8, 4 row
 * blocks (threads = (TX/2 + 2) x row blocks).  3-D steppers: with one launch
 * per stage, -1 (and 0, 1) streams CH / CH+AC grids (z periodic; x, y
 * periodic or zero-flux) through the TMA-staged kernel on its default tile,
 * 3..5 pick that kernel's tile variants (FP32: 32x8 with one row per thread,
 * 32x16 with four, 32x6 with one; FP64: 32x6 with one, 32x8 with two and
 * with one), and 2 selects the marching kernel without TMA; on the fused
 * two-stage RK4 path 0 (the default) or 1 pick two tile variants (the second
 * puts the stages-3-4 launch on 32x8 tiles).  -1 picks by grid (see
 * phix_stepper_autotune for a measured choice).  All give the same bits.
 * No reference counterpart. */
int phix_stepper_set_tiles(phix_stepper_t* h, int tile_cfg);

/* The current launch form (1: one launch per RK4 step) and tile shape. */
int phix_stepper_get_tiles(const phix_stepper_t* h, int* one_launch_per_step, int* tile_cfg);

/* Time every launch form (one launch per stage or per RK4 step; for
 * PHIX_MULTISTEP the box-tile and the pair-layout step) and tile shape this
 * stepper's grid can take, twice on trial_steps steps of its current state,
 * keep the fastest (state, mu included, saved and restored); *best_ms = ms
 * per step.  No reference counterpart. */
int phix_stepper_autotune(phix_stepper_t* h, int trial_steps, double* best_ms);

/* FP64 only: run directly on caller-owned buffers, no copies.  fields[f] is
 * the current state and alt[f] a second stored array of the same size.
 * After phix_stepper_advance, phix_stepper_current() reports which of the two
 * holds the newest state (0: fields, 1: alt); the drop-in Solver swaps
 * ScalarField::d_curr / d_prev accordingly. */
int phix_stepper_bind(phix_stepper_t* h, double* const* fields, double* const* alt);
int phix_stepper_current(const phix_stepper_t* h);

/* End-to-end convenience: host FP64 stored arrays in, nsteps, host arrays
 * out (host->device copy, advance, device->host copy, synchronise). */
int phix_stepper_run_host(phix_stepper_t* h, const double* const* host_in, double* const* host_out, int nsteps);

/* ---- batched engine: many independent 2-D fields in one launch per stage */

typedef struct phix_batch phix_batch_t;

/* ninst independent 2-D simulations of one single-field physics (AC or CH),
 * each with its own grid (size, spacing, BCs) and its own prm[8*i .. 8*i+7],
 * advanced in lockstep with time step dt.  Each RK4 step of all instances is
 * one launch (phix_batch_set_fusion), else each stage is one persistent
 * kernel over a shared tile list; state and stage buffers come from one
 * device pool.  No reference counterpart: the reference runs one
 * Solver per field (Solver.cu:86-107), i.e. instances one after another. */
int phix_batch_create(phix_batch_t** out, int phys, int scheme, int precision, int ninst, const phix_grid_t* grids,
                      const double* prm, double dt);
int phix_batch_destroy(phix_batch_t* b);

/* 1: run each RK4 step of the whole batch as one launch (one CTA per tile,
 * the four stage states in shared memory, tile halos recomputed; the pair
 * kernels with 128x32 (FP32) or 64x32 (FP64) tiles when every instance is
 * CH with four periodic sides, else 128x32 cell-per-thread tiles);
 * needs RK4 and periodic or zero-flux sides on every instance, else
 * PHIX_ERR_UNSUPPORTED.  0: one launch per stage.  Both give the same bits.
 * Default: 1 wherever it is possible (the faster on B200 in both
 * precisions).  No reference counterpart. */
int phix_batch_set_fusion(phix_batch_t* b, int one_launch_per_step);
/* Temporal-block depth of the one-launch step: 2 runs two RK4 steps per
 * launch (the pair kernels on tiles with a 16-cell halo, the first step's
 * update kept in shared memory; an odd remaining step runs alone), 1 (the
 * default) one.  Depth 2 needs the pair kernels, else PHIX_ERR_UNSUPPORTED.
 * Same bits either way.  phix_batch_depth: the depth in effect.  No
 * reference counterpart. */
int phix_batch_set_depth(phix_batch_t* b, int depth);
int phix_batch_depth(const phix_batch_t* b);

/* Kernel launches one batched time step takes with the current settings. */
int phix_batch_launches_per_step(const phix_batch_t* b);
/* Copy one instance's FP64 stored array in / out (device, or host when
 * from_host / to_host is non-zero; host copies are synchronous). */
int phix_batch_load(phix_batch_t* b, int inst, const double* field, int from_host, void* stream);
int phix_batch_store(phix_batch_t* b, int inst, double* field, int to_host, void* stream);
int phix_batch_advance(phix_batch_t* b, int nsteps, void* stream);
int phix_batch_set_graph(phix_batch_t* b, int steps_per_graph);
/* Tile shape id (0..5: 64x16, 32x16, 128x8, 64x8, 32x32, 128x16) and resident
 * CTAs per SM of the persistent launches (0 = occupancy limit). */
int phix_batch_set_tiles(phix_batch_t* b, int tile_cfg, int ctas_per_sm);
int phix_batch_get_tiles(const phix_batch_t* b, int* tile_cfg, int* ctas_per_sm, int* ntiles);
/* Time every tile shape x CTA count of the one-launch-per-stage kernels, and
 * the one-launch step at temporal-block depths 1 and 2 where possible, on
 * trial_steps steps of the real batch (state saved and restored); keep the
 * fastest; *best_ms = ms per step. */
int phix_batch_autotune(phix_batch_t* b, int trial_steps, double* best_ms);
/* FP64 mass (sum of u * dV over physical cells) per instance; synchronous. */
int phix_batch_mass(phix_batch_t* b, double* masses);

/* ---- learned surrogate (Cahn-Hilliard, 50 FD steps per call) ----------- */

/* A 4-layer 3x3 CNN (1 -> 32 -> 32 -> 32 -> 1, GELU, circular padding) that
 * predicts c(t + 50 dt) - c(t) from c(t), followed by an exact FP64
 * mean-mass projection.  The 32 -> 32 layers (forward, data gradient and
 * weight gradient) run as BF16 implicit GEMMs on the tcgen05 tensor cores
 * with FP32 accumulation in TMEM; the fused inference step runs the 1 -> 32
 * and 32 -> 1 layers as UMMAs as well.  States are compact [B][H][W] FP64 device
 * arrays; W must be a multiple of 128.  No reference counterpart: the
 * reference only has the FD solver (Solver.cu). */
typedef struct phix_surrogate phix_surrogate_t;
int phix_surrogate_create(phix_surrogate_t** out, int H, int W, int batch_max, double in_shift, double in_scale,
                          double out_scale);
int phix_surrogate_destroy(phix_surrogate_t* s);
/* Number of FP32 parameters: W1[32][9] b1[32] W2[32][9][32] b2[32]
 * W3[32][9][32] b3[32] W4[9][32] b4[1], W[n][tap][ci] with tap = 3*ky + kx. */
int phix_surrogate_nparams(void);
int phix_surrogate_set_params(phix_surrogate_t* s, const float* host_params);
int phix_surrogate_get_params(phix_surrogate_t* s, float* host_params, float* host_grads);
/* c_out = c + out_scale * net(c), then c_out += mean(c) - mean(c_out).  By
 * default one fused kernel (all four layers on the tensor cores, layers 1
 * and 4 as UMMAs too, activations never leaving shared memory) plus the
 * projection; c and c_out must not overlap. */
int phix_surrogate_step(phix_surrogate_t* s, const double* c, double* c_out, int B, void* stream);
/* 1 (default): phix_surrogate_step runs the fused kernel; 0: the per-layer
 * kernels of phix_surrogate_forward (layers 1 and 4 on CUDA cores).  The two
 * agree to FP32 rounding of the thin layers' sums.  No reference counterpart. */
int phix_surrogate_set_fused(phix_surrogate_t* s, int on);
/* Raw network output o = net(c) as FP32 [B][H][W]. */
int phix_surrogate_forward(phix_surrogate_t* s, const double* c, float* o, int B, void* stream);
/* Gradient of mean((o - (c_next - c)/out_scale)^2) into the internal
 * gradient vector; *loss = the loss.  Synchronous. */
int phix_surrogate_grad(phix_surrogate_t* s, const double* c, const double* c_next, int B, double* loss,
                        void* stream);
/* Adam step (lr) with `grads` (device FP32, NULL = internal vector). */
int phix_surrogate_adam(phix_surrogate_t* s, const float* grads, float lr, void* stream);
/* Device pointer of the internal FP32 gradient vector. */
float* phix_surrogate_grad_ptr(phix_surrogate_t* s);
/* Reads and clears the device error flag of the surrogate's tensor-core
 * kernels: PHIX_ERR_TIMEOUT if one of their bounded mbarrier waits (2 s) gave
 * up since the last check (the kernel then returned without its result),
 * else PHIX_OK.  phix_surrogate_step is asynchronous and does not read the
 * flag; phix_surrogate_grad reads it.  Synchronous on `stream`. */
int phix_surrogate_status(phix_surrogate_t* s, void* stream);
/* Measured multiply-add throughput of the current device: *tflops = 2 x
 * fused multiply-adds per second / 1e12 (best of three launches of a probe
 * that keeps every SM busy with independent FMA chains).  precision PHIX_F64,
 * or PHIX_F32 with packed != 0 for the two-lane f32x2 instruction.  The
 * denominator of the arithmetic-pipe roofline of the stencil kernels.
 * Synchronous.  No reference counterpart. */
int phix_measure_fma_peak(int precision, int packed, double* tflops);
/* Self-test of those bounded waits: one thread waits for an mbarrier of count
 * 1 with a wall-clock limit of limit_s (0 < limit_s <= 2), arriving on it
 * first when `arrive` is non-zero.  Returns PHIX_OK when the wait completed and
 * PHIX_ERR_TIMEOUT when it gave up (no arrival), the kernel having returned
 * and the context still usable.  No reference counterpart. */
int phix_wait_selftest(int arrive, double limit_s, void* stream);
/* Copy the physical plane of a 2-D FP64 stored field to / from a compact
 * [H][W] array. */
int phix_plane_gather(const double* stored, double* plane, int H, int W, int ghost, void* stream);
int phix_plane_scatter(const double* plane, double* stored, int H, int W, int ghost, void* stream);

/* ---- diagnostics (FP64 accumulation) ----------------------------------- */

/* out[0] = sum_phys u * dV (mass), out[1] = free energy
 *   sum_phys [ f(u) + kappa/2 |grad u|^2 ] * dV
 * with the physics' bulk energy density and central gradients on BC-mapped
 * neighbours (develop/Spinodal Decomposition/computeFreeEnergy.py:76-98).
 * fields: 1 (AC, CH) or 2 (CHAC) FP64 stored device arrays.  Synchronous.
 * Returns PHIX_ERR_NONFINITE if any physical value is NaN/Inf. */
int phix_reduce_mass_energy(const double* const* fields, int phys, const double* prm, const phix_grid_t* g,
                            double* out, void* stream);
/* Same diagnostics on the stepper's own current state (FP32 or FP64). */
int phix_stepper_diagnostics(phix_stepper_t* h, double* out);

/* Allocation-free variant of phix_reduce_mass_energy, for callers that cannot
 * allocate device memory (hosts whose device memory is owned by another
 * runtime or allocator, real-time loops that forbid allocation after
 * start-up).  It calls no cudaMalloc, cudaFree or allocating library routine:
 * its scratch is one triple per physical row (n[1]*n[2] rows) in a
 * file-scope device array sized for PHIX_NOALLOC_MAX_ROWS rows (about
 * 1.5 MiB, held on every GPU that loads the library until exit); larger grids
 * return PHIX_ERR_ARG.  The first call on a device looks up that array's
 * device address (cudaGetSymbolAddress) and keeps it for the life of the
 * device's context (do not call it on a device after cudaDeviceReset there).
 * All calls share the one array: calls that overlap on the GPU race and must
 * be serialised.  Synchronous (a device-to-host copy and a wait on `stream`),
 * so not for a stream under capture, nor for stream = NULL while a
 * global-mode capture is active; same outputs and status codes as
 * phix_reduce_mass_energy.  No counterpart in the reference (which has no
 * runtime diagnostics). */
#define PHIX_NOALLOC_MAX_ROWS 65536
int phix_reduce_mass_energy_noalloc(const double* const* fields, int phys, const double* prm, const phix_grid_t* g,
                                    double* out, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* PHIX_B200_H */
