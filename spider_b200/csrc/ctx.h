// Context object behind the opaque spi_ctx handle.
#pragma once

#include "common.h"
#include "../../include/spider_b200.h"

struct spi_ctx {
  int device = 0;
  int sm_count = 148;
  cudaStream_t stream = nullptr;      // library stream: every call is ordered on it
  cudaStream_t stream2 = nullptr;     // staging stream of the insertion pipeline
  long long launches = 0;

  // ---- Fourier gridding back-projection state ----
  int nx = 0, n = 0, ngrids = 0, nsym = 1;
  std::vector<float> sym_dm;          // 9 * nsym (column-major 3x3 each)
  bool pending_sym0[2] = {false, false};
  bool merged = false;
  bool inserted = false;              // images went into the open grids
  float tuned_ms = 0.0f;              // autotuner: time of the chosen launch on its sample
  int bf16 = 0;
  int insert_mode = 3;                // 0 = tile-privatised, 1 = direct per-tap atomics, 2 = five x-tap lanes,
                                      // 3 = four lanes over the nonzero tap window
  int slice_order = 1;                // 1 = order slices of a chunk by plane normal
  int line_order = 1;                 // x4 insertion order: 0 rows, 2 columns, 1 per slice (SliceDesc::cols)
  int insert_seg_map = 0;             // 1 = warps take 32-pixel row segments, 0 = whole rows
  int insert_threads = 256;           // threads per insert block
  int insert_blocks_per_sm = 0;       // 0 = as many as fit
  int pipeline = 1;                   // 1 = host-image uploads on stream2 under the compute
  int first_piece = 1;                // 1 = a one-chunk host-image call's first FFT sub-batch is one upload piece
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  std::vector<cudaEvent_t> ev_ready, ev_done;  // per FFT sub-batch slot
  int cg_fp64 = 2;                    // BP CG precision: 0 FP32, 1 FP64, 2-4 FP64 vectors + fixed-point projections
  int cg_interp = 0;                  // BP CG interpolation: 0 linear, 1 FBS
  int rb_fbs = 0;                     // RB 3F / RB 32F rotate with RTSF (FBS) instead of RTSQ
  cufftHandle rtsf_plan[2] = {0, 0};  // RTSF: batched 2D D2Z / Z2D of FBS2_PREP
  int rtsf_n = 0, rtsf_k = 0;         // image size and batch of those plans
  spi::DevBuf rtsf_buf;               // RTSF scratch: FP64 FFT arrays + FBS2 tables
  int chunk = 0;                      // images per persistent insert launch
  int sub = 0;                        // images per batched 2D FFT (and per insert launch)
  int sort_group = 0;                 // images per slice-ordering group (groups stay inside FFT sub-batches)
  int upload_images = 0;              // host images per upload piece (0 = ~64 MB)
  int col512 = 4;                     // columns per CTA of the n = 512 column FFT (4 or 8)
  spi::KBTab kb;
  spi::DevBuf grid[2];                // float4 {re, im, w, 0} [n][n][nx+1]
  int accum = 1;                      // 1 = compensated: insert into part[], two-sum fold into grid + comp
  int fold_every = 0;                 // images between folds (compensated accumulation)
  long long unfolded = 0;             // images inserted into part[] since the last fold
  bool comp_dirty = false;            // comp[] may hold nonzero compensation terms
  spi::DevBuf part[2];                // float4 partial sums of the images since the last fold
  spi::DevBuf comp[2];                // float4 low-order compensation of grid[] (two-sum error terms)
  float4* gptr[2] = {nullptr, nullptr};      // grids in use (owned or attached)
  float4* ext_grid[2] = {nullptr, nullptr};  // caller-owned grids (spi_bp_attach_grids)
  int wkb_nx = 0;                     // nx the cached |WKB| table belongs to
  long wkb_m = 0;                     // shell voxel count M of WINDKB2A
  spi::DevBuf kbtab;                  // float[5000]
  spi::DevBuf imgs;                   // float [chunk][nx][nx]
  spi::DevBuf imgs2;                  // float [chunk][nx][nx] (RTSQ output)
  spi::DevBuf rtsq_prm;               // RtsqParm [chunk]
  spi::DevBuf padded;                 // float [sub][n][n]
  spi::DevBuf spectra;                // float2 or bf16x2 [chunk][n][nx+1]
  spi::DevBuf spec_tmp;               // float2 [sub][n][nx+1] (BF16 mode FFT output)
  spi::DevBuf slices;                 // SliceDesc [chunk * nsym]
  spi::DevBuf workctr;                // u64 row counter of the running insert launch
  spi::DevBuf mc_params;              // multi-class insertion: class table + tables of the launch
  spi::HostBuf mc_host;               // multi-class insertion: pinned descriptors, class tables, tables
  spi::DevBuf cplx;                   // float2 [n][n][nx+1] (inverse FFT input)
  spi::DevBuf real3;                  // float [n][n][n]
  spi::DevBuf wkb;                    // float[(nx/2)^2 + 1]
  spi::DevBuf acc;                    // double[8] reduction scratch
  spi::DevBuf volbuf;                 // float [nx^3] (finish output staging)
  spi::DevBuf symtmp;                 // float [nx^3] + symmetry matrices (SYMVOL input)
  spi::HostBuf hslices;
  cufftHandle plan2d = 0;
  int plan2d_n = 0, plan2d_batch = 0;
  int fft_own = 0;                    // 1 = the library's own two-pass R2C (power-of-two n), 0 = cuFFT
  spi::DevBuf fft_tw;                 // float2 W_n^t, t < n/2 (FP64-computed twiddles of the own R2C)
  cufftHandle plan3d = 0;
  int plan3d_n = 0;

  // ---- PJ 3Q / BP CG scratch ----
  spi::DevBuf pj_vol, pj_out, pj_runs, pj_dm;
  spi::DevBuf pj_fbs;                 // PJ 3F: FBS3_PREP scratch + the FBS3 table
  cufftHandle pjf_plan[2] = {0, 0};   // PJ 3F: FBS3_PREP's 3D D2Z and 7-batch Z2D
  int pjf_n = 0;                      // cube size of those plans
  spi::DevBuf pj_v4;                  // PJ 3Q: the volume as float4 quads of x/y neighbours
  spi::DevBuf pj_rows;                // PJ 3Q forward: runs in (y, |z|) order, then the row tasks
  spi::DevBuf cg_buf[8];
  spi::DevBuf cg_fbs[4];              // FBS: 3D scratch + table, 2D chunk scratch, segments, DM(1..9)
  spi::HostBuf hbuf;

  // per-phase event timing
  bool timing = false;
  struct PhaseEv { cudaEvent_t a, b; int phase; cudaStream_t s; };
  std::vector<PhaseEv> ev_pending;
  std::vector<cudaEvent_t> ev_pool;
  double phase_ms[SPI_NPHASE] = {0};
  long long phase_n[SPI_NPHASE] = {0};
  int phase_begin(int phase, cudaStream_t s = nullptr);   // returns slot or -1; s = nullptr: stream
  void phase_end(int slot);
  void phase_collect();         // synchronises on recorded events

  long long device_bytes() const;
  int count(int k = 1) { launches += k; return 0; }
};

namespace spi {
// Release every cuFFT plan and device buffer of the reconstruction state.
void bp_release(spi_ctx* c);
void pj_release(spi_ctx* c);
void cg_release(spi_ctx* c);
void rtsf_release(spi_ctx* c);

// PJ 3Q / PJ 3F voxel runs (PREPCUB, prepcub.f:54-109) and rotations
struct PjRun {
  int i1, i2;     // first/last x (1-based) of the run
  int x, y, z;    // centred coordinates of the first voxel
};
struct PjDM {
  float d[9];
};
// byte offset of the row tasks in pj_rows, after nruns runs (16-byte aligned)
inline size_t pj_tasks_offset(int nruns) { return ((size_t)nruns * sizeof(PjRun) + 15) & ~size_t(15); }
// Validates the arguments, builds the runs of the sphere of radius ri and
// the DM of every angle (psi, theta, phi) and uploads them to pj_runs / pj_dm
// on the context stream.
// Also uploads to pj_rows the runs in (y, |z|) order (z_order: (y, z))
// followed by the row tasks of the warp forward projection (int4 {first run,
// runs, x1, x2}: up to 32 runs of one row y and the union of their x
// ranges); *ntasks_out gets their number.
int pj_common(spi_ctx* c, int nx, int ny, int nz, float ri, const float* angles, int nang, int* nruns_out,
              int* ntasks_out = nullptr, bool z_order = false);
// RTSF (rtsf.f:109-205, SCLI = 1) of nimg device images; prm[b] = {COS(THETA),
// SIN(THETA), MODULO(SHX, NX), MODULO(SHY, NX)}; runs on the context stream.
int rtsf_images(spi_ctx* c, const float* src, float* dst, int nx, int nimg, const float4* prm);
int check_kernel(const char* what);
// PADD2 + ASTA_D + phase shift of nimg device images (box nx) into padded
// [nimg][2nx][2nx] float on stream s (the staging of the back-projection)
int stage_images(const spi_ctx* c, cudaStream_t s, const float* imgs, int nx, int nimg, float* padded);
}  // namespace spi
