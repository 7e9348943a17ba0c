/*
 * spider_b200.h -- C ABI of the B200 (sm_100a) implementation of SPIDER's
 * Fourier gridding back-projection (BP 3F, BP 32F, BP 3F P, BP 3F M), its
 * trilinear projector (PJ 3Q) and conjugate-gradient reconstruction (BP CG).
 *
 * These entry points are what SPIDER's operation subroutines would bind
 * through ISO_C_BINDING in place of their compute loops; each comment names
 * the reference subroutine (file:line, paths inside the SPIDER source tree)
 * whose computation it replaces.  The Fortran side keeps its prompts, file
 * I/O and RESULTS output; it passes arrays and receives arrays.
 *
 * Conventions
 *  - Every function returns an int status: 0 = success, otherwise an
 *    IRTFLG-style code (46 = allocation failure, 101 = invalid argument,
 *    102 = missing data / radius too large, 200+ = CUDA or cuFFT error);
 *    spi_last_error() returns the message of the last failure on the
 *    calling host thread.
 *  - Arrays are Fortran column-major, i.e. C row-major with the dimensions
 *    reversed: an image is float[nx*nx] with x fastest, a volume
 *    float[nz*ny*nx] with x fastest.
 *  - Angles are triples (psi, theta, phi) in degrees per image: registers
 *    1-3 of SPIDER's angle document, the order BUILDM1 reads them
 *    (bp3f.f:1287).  Symmetries use the same triple order (builds.f:52).
 *  - `half` masks hold one byte per image: nonzero routes the image to the
 *    first sample volume (BP 32F RANDLIST .TRUE., bp32f.f:802-913).
 *  - Buffers are caller-owned.  `on_device` flags say whether a pointer is a
 *    device (cudaMalloc'd, same device as the context) or host pointer.
 *  - A context is bound to one device and one CUDA stream and must be used
 *    from one host thread at a time.  Calls are synchronous unless the name
 *    ends in _async.  `stream` arguments are cudaStream_t values (NULL = the
 *    context's own stream).
 */
#ifndef SPIDER_B200_H
#define SPIDER_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct spi_ctx spi_ctx;

/* Library version (major*10000 + minor*100 + patch). */
int spi_version(void);

/* Message of the last failed call on this host thread ("" if none). */
const char* spi_last_error(void);

/* The generalised Kaiser-Bessel interpolation table of FILLBESSIL
 * (fillbessi0.f:88-125) for padded size n2 = 2*nx: tab = float[5000],
 * fltb receives FLTB.  Host-only, needs no device. */
int spi_kb_table(int n2, float* tab, float* fltb);

/* Create / destroy a context on CUDA device `device`. */
int spi_ctx_create(int device, spi_ctx** out);
int spi_ctx_destroy(spi_ctx* ctx);

/* Number of kernels this library has launched through `ctx` so far. */
long long spi_ctx_launch_count(const spi_ctx* ctx);

/* Device memory the context currently holds, in bytes. */
long long spi_ctx_device_bytes(const spi_ctx* ctx);

/* The CUDA stream (cudaStream_t) the context launches on. */
void* spi_ctx_stream(const spi_ctx* ctx);

/* Per-phase device timing (CUDA events on the context stream).  When on,
 * every phase of the back-projection is bracketed by events and its device
 * milliseconds accumulated; spi_ctx_timing copies SPI_NPHASE totals and
 * resets them.  Phases: 0 stage (PADD2), 1 2D FFT, 2 insert (ONELINE),
 * 3 SYMPLANE0, 4 NRMW2, 5 3D FFT, 6 WINDKB2A, 7 host-to-device copies
 * (only when they are not overlapped), 8 folds of the compensated
 * accumulation.  The events cost the overlap of host-image uploads with the
 * compute (measured: uploads then run serially), so leave timing off
 * outside diagnostics. */
#define SPI_NPHASE 9
int spi_ctx_set_timing(spi_ctx* ctx, int on);
int spi_ctx_timing(spi_ctx* ctx, double* ms_out, long long* count_out);

/* ------------------------------------------------------------------ *
 * Fourier gridding back-projection, streaming form.
 * Replaces BP3FQ's per-image loop (bp3f.f:298-515) and BP32FQ's
 * (bp32f.f:433-939): PADD2 + FMRS_2 + phase + ONELINE per image, then
 * SYMPLANE0 + NRMW2 + FMRS_3 + WINDKB2A per volume.
 * ------------------------------------------------------------------ */

/* Allocate and zero `ngrids` (1 = BP 3F, 2 = BP 32F) Fourier grids for box
 * size nx (8 <= nx <= 512) and set the symmetry list (sym_angles may
 * be NULL when nsym <= 1).  Replaces the grid setup of BP3F (bp3f.f:160-178,
 * 386-394) and BP32F (bp32f.f:163-179, 490-500). */
int spi_bp_open(spi_ctx* ctx, int nx, int ngrids, const float* sym_angles, int nsym);

/* Use caller-owned device memory for the grids of the next spi_bp_open
 * (g1 may be NULL for one grid; NULL, NULL returns to library-owned grids).
 * Each grid is spi_bp_grid_bytes(nx) bytes of float4 {Re X, Im X, W, 0}
 * voxels, [2nx][2nx][nx+1] with i fastest.  Lets a multi-GPU caller sum the
 * per-rank grids with a collective before spi_bp_finish, the step the
 * reference performs with MPI_ALLREDUCE (bp3f.f:1171-1187,
 * bp32f.f:764-774). */
int spi_bp_attach_grids(spi_ctx* ctx, void* g0, void* g1);
int spi_bp_grid_bytes(int nx, long long* bytes);

/* Spectrum storage for subsequent inserts: 0 = FP32 (default), 1 = BF16. */
int spi_bp_set_spectrum_precision(spi_ctx* ctx, int bf16);

/* Grid accumulation of the next spi_bp_open (no counterpart in the
 * reference, whose X += BTQ*W, oneline.f:107-110, is a plain REAL sum).
 * compensated = 1 (default; environment SPI_BP_ACCUM=0 changes the default):
 * the taps of each run of `fold_every` images (0 = the default, 4,096 or
 * SPI_BP_FOLD; a fold follows the insertion launch -- one per FFT sub-batch
 * -- in which the count is reached) are summed with FP32 atomics into a
 * partial grid, which is then folded into the grid by an error-free two-sum
 * whose rounding errors
 * are kept in a compensation grid; the compensation is added in once before
 * SYMPLANE0.  The error of the sums then grows with the images per fold, not
 * with all images.  Costs two more grid-sized buffers and one pass over
 * them per fold.  compensated = 0: every tap is added straight into the
 * grid.  Fails with 101 while a reconstruction is open. */
int spi_bp_set_accumulation(spi_ctx* ctx, int compensated, int fold_every);

/* Insert the images of several classes in one call (no counterpart in the
 * reference, which reconstructs one volume per run; the per-image work is
 * BP32FQ's loop, bp32f.f:802-913).  ctxs[k] is an open reconstruction
 * (spi_bp_open with class k's box size; at most 16 classes and 8 distinct
 * box sizes, one spectrum precision); imgs[k] (nimg[k] images of that box,
 * host or device per imgs_on_device), angles[k] and half[k] (half may be
 * NULL, or hold NULL entries) as for spi_bp_insert.  Each round stages the
 * next FFT sub-batch of every class and inserts all of them with ONE kernel
 * launch whose rows carry their class's box size, table, spectra and grids.
 * All work runs on ctxs[0]'s stream; the call returns when it is done. */
int spi_bp_insert_multi(spi_ctx* const* ctxs, int nclass, const float* const* imgs, const int* nimg,
                        const float* const* angles, const uint8_t* const* half, int imgs_on_device);

/* Complete the grids of the open reconstruction: fold pending partial sums
 * and add the compensation in, so that caller-owned grids hold the full sums
 * (call before summing them across processes).  Synchronises the stream. */
int spi_bp_flush(spi_ctx* ctx);

/* Autotune the insertion launch of the open reconstruction (no counterpart
 * in the reference, whose insertion is a fixed OpenMP loop): times the
 * kernel variants and launch shapes on one sub-batch of synthetic slices,
 * keeps the fastest and zeroes the grids again.  Call it right after
 * spi_bp_open (and spi_bp_set_spectrum_precision); it fails with 101 once
 * images have been inserted.  The choice is cached per (device, nx, number of
 * grids, spectrum precision, symmetry count) for the process; force = 1
 * measures again. */
int spi_bp_autotune(spi_ctx* ctx, int force);

/* The insertion launch in use: kernel (0 tile, 1 direct, 2 five x-tap lanes,
 * 3 four lanes over the nonzero window), threads per CTA, CTAs per SM, and
 * the autotuner's time of one sample launch in ms (0 when not tuned). */
int spi_bp_get_launch(const spi_ctx* ctx, int* kernel, int* threads, int* blocks_per_sm, float* tuned_ms);

/* Insert `nimg` images (float[nimg*nx*nx]) with their angles
 * (float[nimg*3], host) and optional half mask (uint8[nimg], host; NULL
 * routes every image to grid 0).  Replaces the body of the BP3FQ image loop
 * (bp3f.f:403-493) and of BP32FQ's (bp32f.f:809-913).  Images may be host or
 * device memory (`imgs_on_device`); the call returns when the images are in
 * the grids. */
int spi_bp_insert(spi_ctx* ctx, const float* imgs, int nimg, const float* angles,
                  const uint8_t* half, int imgs_on_device);

/* RB 3F / RB 32F insertion: as spi_bp_insert, after rotating and shifting
 * every image with RTSQ (rtsq.f:56-140, quadratic interpolation) by its
 * angle-document registers 6-8: inplane = float[nimg*3] (in-plane angle in
 * degrees, x shift, y shift), host memory.  Replaces the CALLRTSQ branch of
 * the BP3FQ / BP32FQ image loop (bp3f.f:406-425, bp32f.f:816-848). */
int spi_bp_insert_rb(spi_ctx* ctx, const float* imgs, int nimg, const float* angles,
                     const float* inplane, const uint8_t* half, int imgs_on_device);

/* Finish the open grids: SYMPLANE0 (bp32f.f:1051-1088), NRMW2
 * (bp3f.f:1347-1371), inverse FFT (fmrs_3.f:54-59) and WINDKB2A
 * (bp32f.f:945-1045).  With one grid, vol_all receives the BP 3F volume.
 * With two, vol_all receives XE+XO (ADDADA, bp32f.f:345-351), vol_1 the
 * first and vol_2 the second sample volume; any of them may be NULL.
 * Volumes are float[nx*nx*nx]. */
int spi_bp_finish(spi_ctx* ctx, float* vol_all, float* vol_1, float* vol_2, int out_on_device);

/* Copy grid `g` after SYMPLANE0 in BP 3F P's file layout: x_out =
 * float[2nx*2nx*2(nx+1)] (interleaved complex X(0:NX,2NX,2NX)), w_out =
 * float[2nx*2nx*(nx+1)] (W).  Replaces BP3F's HALT branch
 * (bp3f.f:191-248).  Host pointers. */
int spi_bp_partial_out(spi_ctx* ctx, int g, float* x_out, float* w_out);

/* Add a partial X,W pair (layout as spi_bp_partial_out) into grid `g`.
 * With spi_bp_finish this is BP 3F M (BP3F_MERGE, bp3f.f:531-739).
 * Partials are already plane-0 symmetrised, so finishing after merges
 * skips SYMPLANE0 for inputs added this way. */
int spi_bp_partial_add(spi_ctx* ctx, int g, const float* x_in, const float* w_in);

/* Release the grids and chunk buffers of the open reconstruction. */
int spi_bp_close(spi_ctx* ctx);

/* One-shot BP 3F on host arrays (BP3F(.FALSE.,.FALSE.), bp3f.f:79). */
int spi_bp3f(spi_ctx* ctx, const float* imgs, int nx, int nang, const float* angles,
             const float* sym_angles, int nsym, float* vol_out);

/* One-shot BP 32F on host arrays (BP32F(.FALSE.), bp32f.f:57). */
int spi_bp32f(spi_ctx* ctx, const float* imgs, int nx, int nang, const float* angles,
              const float* sym_angles, int nsym, const uint8_t* half,
              float* vol_all, float* vol_1, float* vol_2);

/* ------------------------------------------------------------------ *
 * PJ 3Q: trilinear projection of a volume (PJ3Q_N, pj3q_n.f:41 ->
 * WRITPRO_N, writpro_n.f:60 -> WPRO_N, wpro_n.f:44-150).
 * vol = float[nz*ny*nx]; proj_out = float[nang*ny*nx]; ri = object radius
 * (the reference's default is min(nx,ny,nz)/2 - 2, pj3q_n.f:82).
 * ------------------------------------------------------------------ */
int spi_pj3q(spi_ctx* ctx, const float* vol, int nx, int ny, int nz, float ri,
             const float* angles, int nang, float* proj_out, int on_device);

/* PJ 3F: PJ 3Q with FBS interpolation (PJ3Q_N(.TRUE.), vtil2.f:222-228;
 * writpro_n.f:154-205 -> FBS3_PREP fbs3.f:294-407 -> WPRO_FBS wpro_fbs.f):
 * the voxel runs of PJ 3Q, each sample the tricubic FBS3 interpolant (FFT
 * derivatives, wrapped indices) instead of the trilinear one.  Same
 * arguments as spi_pj3q; cubic volumes only (nx = ny = nz <= 1024); FP32
 * tables and arithmetic (the reference's REAL), FP64 transforms. */
int spi_pj3f(spi_ctx* ctx, const float* vol, int nx, int ny, int nz, float ri,
             const float* angles, int nang, float* proj_out, int on_device);

/* PJ 3Q that allocates nothing -- no counterpart in the reference; an
 * addition for callers that must not allocate device memory: applications
 * whose device memory belongs to a fixed arena or caching allocator, and
 * latency-critical pipelines that cannot take cudaMalloc/cudaFree's implicit
 * synchronisation.  Same operator as spi_pj3q: its rotation matrices are
 * built on the device with the host's FP64 operation order (they differ only
 * where the device's and host's cos/sin differ in a last bit that also moves
 * the single-precision rounding), and its sums differ in the order of the
 * FP32 atomic additions.  vol (float[nz*ny*nx]), angles (float[3*nang]: psi, theta,
 * phi) and proj_out (float[nang*ny*nx]) are device pointers on the current
 * device; work is queued on `stream` (cudaStream_t, NULL = legacy stream) and
 * the call returns without waiting for it.  Its scratch (voxel runs and
 * rotation matrices) is one file-scope __device__ array of 1,114,112 bytes,
 * which every GPU that loads the library holds until exit; hence the limits
 * ny*nz <= 65536 and nang <= 16384 per call (larger requests return 101).
 * Each call looks up that array's device address, which allocates nothing.
 * Under lazy module loading (CUDA_MODULE_LOADING=LAZY, the CUDA default) the
 * first call on a device may be what loads the library's device code, and
 * with it the array: that load is the driver's one implicit allocation, so
 * make the first call before any stream capture and before the caller's
 * memory budget is fixed (or set CUDA_MODULE_LOADING=EAGER, which loads it
 * with the context).  Every call shares the array and overwrites
 * it, so calls that overlap on the GPU (different streams, or different host
 * threads on the same device) race; serialise them. */
int spi_pj3q_noalloc(const float* vol, int nx, int ny, int nz, float ri, const float* angles,
                     int nang, float* proj_out, void* stream);

/* Exact adjoint of spi_pj3q: scatters projections back into a volume with
 * the transposed trilinear weights (vol_out is overwritten). */
int spi_pj3q_adjoint(spi_ctx* ctx, const float* projs, int nx, int ny, int nz, float ri,
                     const float* angles, int nang, float* vol_out, int on_device);

/* PJ 3Q plan (no counterpart in the reference, whose PJ 3Q is one call):
 * the voxel runs (PREPCUB, prepcub.f:54-109) and rotation matrices for one
 * volume shape, radius and angle list (host float[nang*3]), uploaded once.
 * spi_pj3q_plan_forward / _adjoint then only launch kernels on `stream`
 * (a cudaStream_t; NULL = the default stream) with device buffers: they
 * allocate nothing and do not synchronise, so they can be captured in a
 * CUDA graph.  The forward equals spi_pj3q, the adjoint spi_pj3q_adjoint;
 * both overwrite their output.  Besides the runs and matrices a plan holds
 * two buffers: the packed volume of the forward projection (32 bytes per
 * voxel up to 3M voxels, 16 above; refreshed by every forward call) and the
 * adjoint's quad accumulator (16 bytes per voxel), each while it takes at
 * most 8 GB (environment SPI_PJ_QUADMAX, in MiB, lowers that cap), so forward
 * calls of one plan must not overlap on the GPU, nor adjoint calls (a forward
 * and an adjoint may).  A plan keeps a pointer to its context for launch
 * counting and must be destroyed before it. */
typedef struct spi_pj3q_plan spi_pj3q_plan;
int spi_pj3q_plan_create(spi_ctx* ctx, int nx, int ny, int nz, float ri, const float* angles, int nang,
                         spi_pj3q_plan** out);
int spi_pj3q_plan_forward(const spi_pj3q_plan* plan, const float* vol, float* proj_out, void* stream);
int spi_pj3q_plan_adjoint(const spi_pj3q_plan* plan, const float* projs, float* vol_out, void* stream);
int spi_pj3q_plan_destroy(spi_pj3q_plan* plan);

/* ------------------------------------------------------------------ *
 * FourierSlice: the central-slice operator pair on ONELINE's geometry
 * (no counterpart in the reference, which has the insertion, ONELINE
 * oneline.f:38-200, but no extraction with the same kernel).
 *   forward E: grid -> slices, the exact adjoint of the insertion;
 *   adjoint E^T: slices -> grid, ONELINE's X += BTQ*W without the weight
 *   grid (same voxels, table weights, Hermitian flips and reflected points).
 * A grid is float2 [2nx][2nx][nx+1] (complex, i fastest: Fortran
 * X(0:NX,N,N)); slices are float2 [nang][2nx][nx+1] in the layout and sign of
 * the staged spectra (spi_fslice_stage: PADD2, phase, 2D R2C; ONELINE's BI is
 * their conjugate).  All pointers are device pointers; `stream` is a
 * cudaStream_t (NULL = legacy stream).  forward, adjoint and normal allocate
 * nothing and do not synchronise, so they can be captured in a CUDA graph.
 * ------------------------------------------------------------------ */
typedef struct spi_fslice_plan spi_fslice_plan;

/* Slice geometry of nang angle triples (host float[3*nang], psi, theta, phi)
 * for box nx (8..512): CANG per slice (cang.f:44-81) and the FILLBESSIL table
 * (fillbessi0.f:88-125), uploaded once. */
int spi_fslice_plan_create(spi_ctx* ctx, int nx, const float* angles, int nang, spi_fslice_plan** plan);
/* Slices of nang device images float[nang*nx*nx]: PADD2 + ASTA_D + phase
 * (bp3f.f:1307-1343, asta.f:61-92, bp3f.f:453-458) and the 2D transform.
 * Its batch buffer and FFT plans are made on the first call. */
int spi_fslice_stage(spi_fslice_plan* plan, const float* imgs, float* slices, void* stream);
/* slices = E grid (overwritten; pixels without taps are zero). */
int spi_fslice_forward(const spi_fslice_plan* plan, const float* grid, float* slices, void* stream);
/* grid = E^T slices (overwritten). */
int spi_fslice_adjoint(const spi_fslice_plan* plan, const float* slices, float* grid, void* stream);
/* grid_out = E^T E grid_in + lam * grid_in in one pass over the taps
 * (grid_out must not alias grid_in). */
int spi_fslice_normal(const spi_fslice_plan* plan, const float* grid_in, float lam, float* grid_out, void* stream);
/* The same normal operator on FP64 grids (double2 [2nx][2nx][nx+1]): same taps
 * and FP32 table weights, FP64 pixel sums and FP64 atomic scatter.  For CG:
 * late directions p have ||E^T E p|| << ||E^T E|| ||p||, where FP32 sums lose
 * that many digits. */
int spi_fslice_normal64(const spi_fslice_plan* plan, const double* grid_in, double lam, double* grid_out,
                        void* stream);
/* slices = E grid on FP64 arrays (FP64 sums of the same taps; an exact
 * reference for gradient checks of the FP32 extraction). */
int spi_fslice_forward64(const spi_fslice_plan* plan, const double* grid, double* slices, void* stream);
/* grid = E^T slices into an FP64 grid (FP64 scatter; the CG's right-hand side). */
int spi_fslice_adjoint64(const spi_fslice_plan* plan, const float* slices, double* grid, void* stream);
/* Real-space volume float[nx^3] of a grid of spectrum coefficients: the grid
 * models V(k) = sum_v X_v K(k - v), so the volume is the inverse transform of
 * X (plane 0 replaced by its Hermitian part, phase (-1)^(i+j+k), SPIDER's
 * inverse sign, 1/n^3) multiplied by |WKB| (WINDKB2A's table,
 * bp32f.f:964-1005) inside radius nx/2 and zero outside.  Its buffers and
 * FFT plan are made on the first call. */
int spi_fslice_volume(spi_fslice_plan* plan, const float* grid, float* vol_out, void* stream);
int spi_fslice_plan_destroy(spi_fslice_plan* plan);

/* ------------------------------------------------------------------ *
 * BP CG, linear interpolation (BPCG, bpcg.f:70 -> BPCG_2 bpcg.f:425,
 * HIANG hiang.f:40, BPCG_3_LIN bpcg.f:818).  projs = float[nang*n*n];
 * vol_out = float[n*n*n]; log_out (may be NULL) = float[3*maxit] receiving
 * (iteration, DIFFERENCE, CHISQ) as the RESULTS lines (bpcg.f:1213-1216);
 * niter_out receives the iterations run.  mode = 1, 2 or 3 (order of the
 * regulariser); lambda = LAMBDA.  Returns 102 for 'RADIUS TOO LARGE'.
 * ------------------------------------------------------------------ */
int spi_bpcg(spi_ctx* ctx, const float* projs, int n, int nang, const float* angles,
             float ri, float errm, float chim, int maxit, int mode, float lambda,
             float* vol_out, float* log_out, int* niter_out);

/* BP CG across several processes, one GPU each: the reference's MPI form
 * (bpcg.f:522-672, 855-1080).  This rank holds images [first, first+count)
 * of the nang angles (projs = float[count*n*n]; angles = all nang triples);
 * HIANG runs on every rank over all angles and each rank applies the normal
 * operator to its SETPART block of the merged list.  `allreduce` is called
 * with the same sequence on every rank and must sum the device array `data`
 * (count values, FP64 when fp64 = 1, else FP32) over the ranks in place,
 * ordered on `stream` (a cudaStream_t: the library's stream; the sum must be
 * there when work queued on it after the call runs) and return 0: once for
 * CB and once for the three ASTASQ sums, then once per iteration for BCKE
 * (the n^3 all-reduce per iteration); the rest of the iteration is
 * replicated, so every rank returns the same volume and log.  With world = 1
 * and no callback this is spi_bpcg on images [first, first+count).  Sharded
 * runs launch each iteration op by op (no CUDA graph). */
typedef int (*spi_allreduce_fn)(void* data, long long count, int fp64, void* stream, void* user);
int spi_bpcg_shard(spi_ctx* ctx, const float* projs, int first, int count, int n, int nang,
                   const float* angles, float ri, float errm, float chim, int maxit, int mode,
                   float lambda, int rank, int world, spi_allreduce_fn allreduce, void* user,
                   float* vol_out, float* log_out, int* niter_out);

/* Storage and accumulation type of the BP CG vectors and projections:
 * mode = 1 keeps CB, BCKP, BCKE, BCKN and the projections in FP64 (the
 * reference keeps them in REAL; its FP32 CG drifts from the exact iteration
 * by more than 1e-2 at small LAMBDA); mode = 0 uses FP32 as the reference
 * does.  Modes 2 and 3 keep the vectors in FP64, accumulate each projection
 * (PRJCQ_N) in fixed point in shared memory with integer atomics and hand it
 * to BCKPJ_LIN as the PROJT four-term table, made per chunk of images:
 * mode = 2 (default) with a 47-bit grid (~1e-11 of max|x|) and FP32 tables;
 * mode = 4 the same with FP64 tables; mode = 3 with a 31-bit grid and FP32
 * tables (fastest, ~1e-7 per projection, not for ill-conditioned problems).
 * Images beyond one CTA's shared memory (n*n*8 bytes for modes 2/4, n*n*4
 * for mode 3) are split into row bands, up to 8.  Scalars (DELSQ, AKDEN, P,
 * Q) and dot products are FP64 in all modes. */
int spi_ctx_set_cg_precision(spi_ctx* ctx, int mode);

/* Interpolation of BP CG's operators, the 'L' / 'F' answer of BP CG
 * (bpcg.f:177-180): fbs = 0 (default) PRJCQ_N / BCKPJ_LIN, linear;
 * fbs = 1 BPCG_3_FBS (bpcg.f:1760-1822): the projector PRJCQ_FBS3
 * (prjcq.f:97-167) samples the tricubic FBS3 interpolant of the direction
 * along every line of the full cube, the back-projector BCKPJ_FBS
 * (bckpj.f:123-164) the bicubic FBS2 interpolant of each projection; both
 * interpolants come from FFT derivatives (FBS2_PREP fbs2.f:182-247,
 * FBS3_PREP fbs3.f:294-407), computed in FP64.  With FBS the radius limit is
 * RI + MODE <= N/2 (linear: RI + MODE + 1) and N is limited to 512.
 * Precision (spi_ctx_set_cg_precision): modes 1 and 4 are FP64 throughout,
 * modes 2 and 3 keep FP64 vectors and arithmetic with FP32 interpolation
 * tables (half the gathered bytes), mode 0 is FP32. */
int spi_ctx_set_cg_interpolation(spi_ctx* ctx, int fbs);

/* In-plane rotation of spi_bp_insert_rb (RB 3F / RB 32F), SPIDER's FBS mode
 * (`MD` with `FBS ON`, setmode.f:399-409, read by bp3f.f:412-424):
 * fbs = 0 (default) RTSQ (rtsq.f:56-140, quadratic QUADRI); fbs = 1 RTSF
 * (rtsf.f:109-205, SCLI = 1): FBS2_PREP of each image (FFT derivatives,
 * FP64 transforms) and bicubic FBS2 with wrapped indices at every rotated
 * and shifted source position. */
int spi_ctx_set_rb_interpolation(spi_ctx* ctx, int fbs);

/* One application of the BP CG operators on device arrays, for the
 * differentiable wrapper and adjointness checks.  spi_cg_project: PRJCQ_N
 * (prjcq.f:48-82) of vol into projs (overwritten).  spi_cg_backproject:
 * BCKPJ_LIN (bckpj.f:59-94) of projs summed into vol (overwritten). */
int spi_cg_project(spi_ctx* ctx, const float* vol, int n, float ri, const float* angles,
                   int nang, float* projs, int on_device);
int spi_cg_backproject(spi_ctx* ctx, const float* projs, int n, float ri, const float* angles,
                       int nang, float* vol, int on_device);

#ifdef __cplusplus
}
#endif
#endif /* SPIDER_B200_H */
