/*
 * msbg_gpu.h — C ABI of the B200 sparse block-grid PDE solver.
 *
 * Drop-in GPU path for MSBG entry points (reference = AkirA-fx/MSBG-Flip):
 *   - MultiresSparseGrid::applyChannelPdeFast<float>(..., -(PDE_MEAN_CURVATURE +
 *     OPT_8_COLOR_SCHEME), ...)                          src/msbg4.cpp:59-957
 *   - MultiresSparseGrid::preparePressureSolveFLIP / solvePressureFLIP and
 *     their pieces                                      src/msbg3.cpp:3041-3271
 *   - the FLIP transfers either side of the solve (particleToGrid,
 *     applyGravity, the pressure-gradient update, gridToParticle) on
 *     single-level grids, and gridToParticle through interpVec3MSBG on
 *     mixed-resolution grids                            src/flip_sim.cpp
 *
 * The host keeps owning the MSBG block pool; this library owns device pools and
 * moves data only on explicit upload/download calls.  Every function returns an
 * msbg_status; codes mirror the reference's MI_* codes (src/globdef.h:128-150).
 * No function calls exit(); a failed call leaves a message for
 * msbg_gpu_last_error().  One context = one host thread + one CUDA stream.
 *
 * Grid conventions (identical to the reference, src/sbg.h:1746-1822):
 *   block id  bid = bx + by*nbx + bz*nbx*nby          (nbx = sx / bsx0, ...)
 *   voxel id  vid = vx + vy*bsx + vz*bsx*bsx          (bsx = bsx0 >> level)
 *   block colour (8-colour scheme) = (bx&1) + 2*(by&1) + 4*(bz&1)
 *                                                       src/msbg.h:642-646
 */
#ifndef MSBG_GPU_H
#define MSBG_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes: same values as MI_OK .. MI_EINTERNAL (src/globdef.h:128-150). */
typedef enum {
  MSBG_OK = 0,
  MSBG_ERROR = 1,
  MSBG_ENOMEM = 2,
  MSBG_ENOTIMPL = 4,
  MSBG_EINVARG = 5,
  MSBG_EMATH = 15,
  MSBG_EINTERNAL = 20,
  MSBG_ENODEV = 25, /* MI_ENOTAVAIL: no usable CUDA device */
  MSBG_ETIMEOUT = 30
} msbg_status;

/* Per-block kind of a channel, as the reference's block map holds it
 * (src/sbg.h:1906-2049): NULL entry, value block, const empty, const full. */
enum {
  MSBG_BLOCK_NULL = 0,
  MSBG_BLOCK_VALUE = 1,
  MSBG_BLOCK_EMPTY = 2,
  MSBG_BLOCK_FULL = 3
};

/* Storage type of a channel's values.  MSBG_U16 is the reference's 16-bit
 * render density (RenderDensity = uint16_t under RSURF_16_BIT,
 * src/msbgcell.h:67-68, src/msbg.h:369-376): q in [0, 65535] stands for
 * q / 65535 (src/sbg.h:225-232). */
enum { MSBG_F32 = 0, MSBG_F16 = 1, MSBG_BF16 = 2, MSBG_F64 = 3, MSBG_U16 = 4 };

typedef struct msbg_gpu_ctx msbg_gpu_ctx;

/* Grid topology: the block raster and the resolution level of every block at
 * multigrid level 0 (the refinement map handed to
 * MultiresSparseGrid::setRefinementMap, src/msbg.cpp:1428).  For a
 * single-level grid pass blockLevel = NULL (all blocks at level 0). */
typedef struct {
  int sx, sy, sz;        /* finest-level resolution (multiples of bsx0) */
  int bsx0;              /* base block size: 8, 16 or 32 */
  int nLevels;           /* resolution levels (1..4) */
  const int* blockLevel; /* [nbx*nby*nbz] level per block, or NULL */
  /* Pressure boundary of the six domain faces (-x, +x, -y, +y, -z, +z), as
   * setDomainBoundarySpec_ gives them (src/msbg.cpp:2462, flip_sim.cpp:1621).
   * Outside the grid p = 0, behind a face coupling of
   *   MSBG_DBC_SOLID: 0 (a wall; the callback is not asked);
   *   MSBG_DBC_OPEN:  on a lower face (-x, -y, -z) the coefficient the
   *                   callback returns for the cell's own lower face, on an
   *                   upper face 1, the reference's open-face weight
   *                   (constFaceCoeffAirBlock, src/msbg3.cpp:733-740).
   * NULL: the reference's own FLIP operator, whose diagonal
   * (computeDiagonalFLIP_, src/msbg3.cpp:2714-2722) ignores the spec: lower
   * faces as OPEN, upper faces 0. */
  const int* domainBc;
} msbg_topo_desc;

enum { MSBG_DBC_OPEN = 0, MSBG_DBC_SOLID = 1 }; /* DBC_OPEN, DBC_SOLID (src/msbg.h:191-192) */

/* ---- context ------------------------------------------------------------ */

/* Replaces nothing in the reference (its state lives in MultiresSparseGrid);
 * creates the device context (device memory, stream) on CUDA device `device`. */
int msbg_gpu_init(int device, msbg_gpu_ctx** out);
int msbg_gpu_destroy(msbg_gpu_ctx* ctx);
const char* msbg_gpu_last_error(const msbg_gpu_ctx* ctx);
/* Waits for all work issued on the context's stream. */
int msbg_gpu_sync(msbg_gpu_ctx* ctx);
/* The context's CUDA stream (cudaStream_t as void*), for callers that order
 * their own work or timing events after the library's. */
int msbg_gpu_stream(msbg_gpu_ctx* ctx, void** stream);

/* Mirrors MultiresSparseGrid::create + setRefinementMap for the device side
 * (src/msbg.cpp:131, 1428): stores the block raster; drops all channels. */
int msbg_gpu_sync_topology(msbg_gpu_ctx* ctx, const msbg_topo_desc* desc);

/* ---- channels ------------------------------------------------------------ */

/* Uploads one FP32 channel of resolution level `level` (all blocks of the
 * raster are of size bsx0>>level).  Replaces the host-side reads of
 * SparseGrid<float>::getBlockDataPtr (src/sbg.h:913-979).
 *   kind[nBlocks]      MSBG_BLOCK_* per block id
 *   blockPtrs[nBlocks] host pointer of each value block (others ignored), as
 *                      returned by getBlockDataPtr(bid); may be NULL when
 *                      `packed` is given instead
 *   packed             all value blocks' voxels back to back in ascending bid
 *                      order (alternative to blockPtrs; one copy)
 *   emptyVal/fullVal   values of const empty / full blocks (setEmptyValue /
 *                      setFullValue, src/sbg.h)                           */
int msbg_gpu_upload_channel(msbg_gpu_ctx* ctx, int chan, int level,
                            const int8_t* kind, const float* const* blockPtrs,
                            const float* packed, float emptyVal, float fullVal);

/* Copies a channel's value blocks back to the host (same layouts as upload). */
int msbg_gpu_download_channel(msbg_gpu_ctx* ctx, int chan, float* const* blockPtrs,
                              float* packed);

/* The same for a 16-bit render-density channel (SparseGrid<uint16_t> of
 * getUint16Channel, src/msbg.h:3085): raw values, const blocks hold the raw
 * emptyVal / fullVal.  msbg_gpu_pde_mcf runs on either kind of channel. */
int msbg_gpu_upload_channel_u16(msbg_gpu_ctx* ctx, int chan, int level, const int8_t* kind,
                                const uint16_t* const* blockPtrs, const uint16_t* packed,
                                uint16_t emptyVal, uint16_t fullVal);
int msbg_gpu_download_channel_u16(msbg_gpu_ctx* ctx, int chan, uint16_t* const* blockPtrs,
                                  uint16_t* packed);

/* Number of value blocks of a channel (size of the packed layout / bsx^3). */
int msbg_gpu_channel_num_value_blocks(msbg_gpu_ctx* ctx, int chan, int64_t* out);

/* Device pointer to the packed value blocks of a channel (for callers that
 * keep data resident and launch on the context stream). */
int msbg_gpu_channel_device_ptr(msbg_gpu_ctx* ctx, int chan, void** out);

/* ---- mean-curvature flow -------------------------------------------------- */

/* Replaces MultiresSparseGrid::applyChannelPdeFast<float>(chan, CH_NULL, CH_NULL,
 * &blockList, -(PDE_MEAN_CURVATURE+OPT_8_COLOR_SCHEME), clamp01, 0,0,0,
 * numIter, 1.0f, dt)                        src/msbg4.cpp:59-957, msbg.h:2176
 * and, on a 16-bit channel, applyChannelPdeFast<uint16_t> (the demo's call,
 * src/msbg_demo.cpp:716-727): values widened on load, the result stored as
 * round(phi * 65535) (src/msbg4.cpp:829-839).
 * In-place 8-colour block Gauss-Seidel (Jacobi inside a block) of the
 * 19-point mean-curvature stencil, halo BC_NEUMANN.  numIter is rounded up
 * to an even count as the reference does (src/msbg4.cpp:150-152).  Only
 * blocks of `blockList` are updated; every value block is read as halo.
 * Asynchronous on the context stream. */
int msbg_gpu_pde_mcf(msbg_gpu_ctx* ctx, int chan, const int* blockList, int n,
                     int numIter, float dt, int clamp01);

/* Same smoother on caller-owned device memory, launched on `stream`
 * (cudaStream_t as void*; NULL = the legacy default stream): pool = value blocks [nSlots][bsx^3] FP32,
 * slotOf[nBlocks] = slot or -1 NULL / -2 empty / -3 full; colourList holds
 * the updated blocks' ids grouped by colour with colourStart[9] offsets
 * (device arrays).  For callers that keep the grid resident on the GPU.
 * pool must be 8-byte aligned (MSBG_EINVARG otherwise).
 * A listed block whose slotOf entry is negative is skipped on the device,
 * and the next msbg_gpu_sync returns MSBG_EINVARG for it. */
int msbg_gpu_pde_mcf_device(msbg_gpu_ctx* ctx, float* pool, const int* slotOf,
                            const int* colourList, const int* colourStartHost,
                            int nbx, int nby, int nbz, int bsx, float emptyVal,
                            float fullVal, int numIter, float dt, int clamp01,
                            void* stream);

/* Same smoother for callers that cannot let this library allocate device
 * memory.  No counterpart in the reference (its smoother runs on host memory).
 * Who needs it: simulation codes that reserve all device memory up front with
 * their own pool allocator, where a cudaMalloc from a library fails or
 * fragments that pool, and host threads that must not block in the CUDA
 * allocator's device-wide synchronisation during a time step.
 *   pool, slotOf   caller-owned device arrays, as for msbg_gpu_pde_mcf_device
 *   blockList, n   host array of the block ids to update (value blocks only)
 *   stream         cudaStream_t as void* (NULL = legacy default stream)
 *   timedOut       NULL: return right after the launches; non-NULL: wait for
 *                  the stream and report whether a bounded wait gave up; a
 *                  listed block whose slotOf entry is negative is skipped on
 *                  the device and then makes the call return MSBG_EINVARG
 * No context, no cudaMalloc/cudaFree: the colour-grouped block list and the
 * error flag live in a fixed device array of 2*MSBG_MCF_NOALLOC_MAX_BLOCKS+16
 * ints (2 MB) that every device using this library keeps until the process
 * exits.  n > MSBG_MCF_NOALLOC_MAX_BLOCKS is rejected with MSBG_EINVARG.
 * The first call on a device looks up that array's device address, and with
 * CUDA's default lazy module loading it is also the call that places the
 * array and the kernels' code on the device.  Make that first call (n = 0 is
 * enough) before reserving the device's memory with your own pool and before
 * any stream capture, or run with CUDA_MODULE_LOADING=EAGER.  All calls on a device share
 * the array (each call resets what must start at zero), so calls whose work
 * overlaps on the GPU race: serialise them on one stream. */
#define MSBG_MCF_NOALLOC_MAX_BLOCKS 262144
int msbg_gpu_pde_mcf_noalloc(float* pool, const int* slotOf, const int* blockList, int n,
                             int nbx, int nby, int nbz, int bsx, float emptyVal, float fullVal,
                             int numIter, float dt, int clamp01, void* stream, int* timedOut);

/* ---- FLIP pressure solve (MGPCG) ----------------------------------------- */

/* Same callback contract as the reference's FlipPressureCallbacks
 * (src/msbg.h:829-835; flip_sim.cpp:313-338 is its caller): cell type
 * (0 liquid, CELL_SOLID 1, CELL_FIXED 2, CELL_VOID 0x1000), face coefficient
 * of the LOWER face of cell (x,y,z) in direction dir, RHS per unit volume.
 * Coordinates are fine-voxel coordinates.  The callbacks are called from
 * several host threads at once and must be thread-safe. */
typedef struct {
  uint16_t (*sampleCellType)(void* user, int x, int y, int z);
  float (*sampleFaceCoeff)(void* user, int dir, int x, int y, int z);
  float (*sampleRhs)(void* user, int x, int y, int z);
  void* user;
} msbg_pressure_callbacks;

/* Solver parameters.  The first five fields are the reference's
 * FlipPressureSolveParams (src/msbg.h:837-844); the rest select the GPU
 * variants.  msbg_gpu_solve_params_default() fills the defaults. */
typedef struct {
  int nPre, nPost, nCoarse, maxIter;
  float tol;        /* stop when |r| <= tol*|b| */
  int innerIter;    /* red-black sweeps inside a tile per smoother visit
                       (default 3: fastest at V(2,2) on the 1024^3 workload) */
  int storage;      /* MSBG_F32, MSBG_F16 or MSBG_BF16: storage of the MG
                       level-0 vectors (coarser levels, the operator and all
                       arithmetic stay FP32; dots FP64) */
  int maxRefine;    /* 0: plain MGPCG stopping on the recursive residual (as the
                       reference); >0: stop on the true FP64 residual, with the
                       solution kept in FP64.  FP32 vectors: one MGPCG whose x
                       is accumulated in FP64, the true residual replacing the
                       recursive one whenever that dropped 10x and when it
                       converges (at most maxRefine checks at convergence); 16-bit
                       vectors: up to maxRefine outer steps of
                       FP64 iterative refinement around the 16-bit MGPCG
                       (always on for them; 0 = 30). */
  int useGraph;     /* capture one PCG iteration in a CUDA graph */
  float coarseScale; /* coarse-grid correction factor (default 1.8; 1 = plain) */
  int learned;      /* bit 0: the network attached by msbg_gpu_pressure_set_cnn
                       predicts the initial guess (scaled by the
                       energy-optimal factor); bit 1: the network attached
                       by msbg_gpu_pressure_set_correction_cnn corrects every
                       V-cycle, under flexible CG (FP32 vectors only).  Any
                       bit forces the FP64 path (maxRefine 0 = 30); a learned
                       solve that ends unconverged is redone by plain MGPCG. */
} msbg_gpu_solve_params;

typedef struct {
  int iterations;        /* PCG iterations (summed over refinement steps) */
  int refinements;       /* FP64 true-residual replacements (FP32 vectors) or
                            outer refinement steps (16-bit vectors) */
  int status;            /* 0 converged, 1 maxIter, 2 breakdown, 3 non-finite */
  double relResidual;    /* true |b - A x| / |b| of the delivered iterate: FP32
                            operator and iterate for maxRefine = 0, FP64 for
                            the refined solve */
  double solveSeconds;   /* device time of the solve */
  int64_t fineCells;     /* cells of MG level 0 (liquid) */
  int nMgLevels;
  int64_t kernelLaunches; /* kernels launched inside the timed solve */
  double initialRelResidual; /* |b - A x0| / |b| of the starting iterate
                                (1 without a learned guess) */
  int learnedFallback;       /* 1: the learned solve stopped unconverged and
                                plain MGPCG solved again from zero (iterations,
                                refinements, time and launches count both) */
} msbg_gpu_solve_info;

void msbg_gpu_solve_params_default(msbg_gpu_solve_params* p);

/* Replaces MultiresSparseGrid::preparePressureSolveFLIP(cb)
 * (src/msbg3.cpp:3041-3095): samples the callbacks on the block grid given by
 * topo (refinement map = topo->blockLevel), builds the finite-volume operator
 * of MG level 0 and the multigrid hierarchy, and uploads it. */
int msbg_gpu_pressure_prepare(msbg_gpu_ctx* ctx, const msbg_topo_desc* topo,
                              const msbg_pressure_callbacks* cb);

/* Replaces MultiresSparseGrid::solvePressureFLIP(params) (src/msbg3.cpp:3098-3271):
 * MGPCG with a V-cycle preconditioner, FP64 inner products. */
int msbg_gpu_pressure_solve(msbg_gpu_ctx* ctx, const msbg_gpu_solve_params* p,
                            msbg_gpu_solve_info* info);

/* Pressure of MG level 0 in the reference's block layout: for every block in
 * ascending bid order, (bsx0>>level)^3 values, vid = x + y*bs + z*bs*bs. */
int msbg_gpu_pressure_download(msbg_gpu_ctx* ctx, float* packed, int64_t n);
/* Same layout in FP64: the refined solution (available after a solve with
 * maxRefine > 0; the FP32 download then holds it rounded to FP32). */
int msbg_gpu_pressure_download64(msbg_gpu_ctx* ctx, double* packed, int64_t n);
/* Same layout, the right-hand side b (volume-integrated) of MG level 0. */
int msbg_gpu_pressure_download_rhs(msbg_gpu_ctx* ctx, float* packed, int64_t n);
/* Number of values in that layout. */
int msbg_gpu_pressure_packed_size(msbg_gpu_ctx* ctx, int64_t* n);

/* Sizes and costs of the prepared problem (no counterpart in the reference;
 * the reference logs similar figures through TRC, src/msbg3.cpp:2340-2348). */
typedef struct {
  int nMgLevels;
  int coarseCells;          /* unknowns of the dense FP64 coarsest solve */
  int64_t cells[32];        /* stored cells per MG level (tiles holding liquid) */
  int64_t fluid[32];        /* liquid cells per MG level */
  int64_t tiles[32];
  int64_t h2dBytes;         /* bytes uploaded by msbg_gpu_pressure_prepare */
  int64_t deviceBytesUsed;  /* device memory in use after prepare */
  double prepareSeconds;    /* wall time of msbg_gpu_pressure_prepare */
  double buildSeconds;      /* of which host sampling + hierarchy build */
} msbg_gpu_pressure_stats_t;

int msbg_gpu_pressure_stats(msbg_gpu_ctx* ctx, msbg_gpu_pressure_stats_t* out);

/* Times `reps` calls of one solver part on the context stream with CUDA
 * events: what = 0 one pre-smoothing sweep of MG level 0 (innerIter sweeps
 * inside each tile), 1 the level-0 matrix-vector product with its dot
 * product, 2 one V-cycle (2 pre, 2 post sweeps), 3 the smoothing sweep
 * through the one-CTA-per-tile kernel.  what | (storage << 4) times the
 * same part with level-0 vectors of that storage type (MSBG_F16/MSBG_BF16).
 * *algBytesPerCall is the algorithmic DRAM traffic of one call (per level-0
 * cell: 16 B of operator plus 3 vector values per smoothing sweep, 16 B plus
 * 2 vector values per matvec; summed over the MG levels for a V-cycle). */
int msbg_gpu_pressure_profile(msbg_gpu_ctx* ctx, int what, int reps, int innerIter,
                              double* msPerCall, double* algBytesPerCall);

/* ---- bulk-array prepare and solver components ---------------------------- */

/* Bulk-array form of msbg_gpu_pressure_prepare: the per-cell data that
 * preparePressureSolveFLIPLevel0_ samples through the callbacks
 * (src/msbg3.cpp:2472-2584) handed over as arrays in the packed block layout
 * of MG level 0 (blocks in bid order, each (bsx0>>level)^3 cells at its
 * refinement level, vid = x + y*bs + z*bs*bs):
 *   flags[]  CELL_* bits per cell (CH_CELL_FLAGS)
 *   faceX/Y/Z[] coefficient of the cell's LOWER face in x/y/z (CH_FACE_AREA)
 *   rhs[]    right-hand side per unit volume (CH_DIVERGENCE; may be NULL = 0)
 * A cell's upper face is its +1 neighbour's lower face; faces on the domain
 * boundary outside the arrays have coefficient 0 (the reference's
 * getValueGen_ reads 0 there, src/msbg3.cpp:2700-2708). */
int msbg_gpu_pressure_prepare_arrays(msbg_gpu_ctx* ctx, const msbg_topo_desc* topo,
                                     const uint16_t* flags, const float* faceX,
                                     const float* faceY, const float* faceZ, const float* rhs);

/* The component entry points below run one piece of the prepared solver on
 * vectors in the packed block layout of MG level levelMg: every base block b
 * at level max(map[b], levelMg) (src/msbg.cpp:1650), (bsx0>>level)^3 values,
 * blocks in bid order.  Levels 0 .. nLevels-1 have this layout.  Inputs are
 * host arrays of exactly msbg_gpu_pressure_level_size values; values of
 * blocks that hold no liquid are ignored on input and 0 on output.  Each call
 * waits for its result.  Vectors must be 0 on cells that are not liquid, as
 * the solver keeps them (the reference's CHECK_NONFLUID_ZERO invariant,
 * src/msbgcell.h:89-92). */
int msbg_gpu_pressure_level_size(msbg_gpu_ctx* ctx, int levelMg, int64_t* n);

/* a_ii per cell (0 off liquid) of MG level levelMg.  The reference's
 * CH_DIAGONAL holds D = 1/(sum of the 6 face weights) (computeDiagonalFLIP_,
 * src/msbg3.cpp:2586-2779); away from level interfaces a_ii = h / D. */
int msbg_gpu_pressure_diagonal(msbg_gpu_ctx* ctx, int levelMg, float* diag, int64_t n);

/* y = A x on MG level levelMg.  Replaces multiplyLaplacianMatrixOpt(0,
 * levelMg, chX, CH_NULL, 0, chY, ...) (src/msbg3.cpp:1757-1912, cell kernel
 * 1282-1321: Y = F0/D - sum W F with F = x h), which equals A x wherever the
 * two operators coincide (same-level faces). */
int msbg_gpu_matvec(msbg_gpu_ctx* ctx, int levelMg, const float* x, float* y, int64_t n);

/* r = b - A x on MG level levelMg (0 off liquid).  Replaces
 * multiplyLaplacianMatrixOpt(OPT_CALC_RESIDUAL, levelMg, chX, chB, ...). */
int msbg_gpu_residual(msbg_gpu_ctx* ctx, int levelMg, const float* x, const float* b, float* r,
                      int64_t n);

/* coarse = R fine from MG level levelMgCoarse-1 to levelMgCoarse: the sum over
 * the liquid children of each coarse cell, through the solve's fused
 * residual-and-restriction kernels (with x = 0).  Replaces
 * downsampleChannel<float,float>(levelMgCoarse, src, dst,
 * OPT_SIMPLE_AVERAGE|OPT_ALL_CELLS) (src/msbg4.cpp:1512-1914), whose
 * coarsened blocks hold the 1/8 average (src/msbg4.cpp:1562-1566): for a
 * vector that is 0 off liquid the sum is 8x the average.  Blocks that are not
 * coarsened at that step are copied, as the reference aliases them
 * (src/msbg4.cpp:1648-1650). */
int msbg_gpu_restrict(msbg_gpu_ctx* ctx, int levelMgCoarse, const float* fine, int64_t nFine,
                      float* coarse, int64_t nCoarse);

/* fine += scale * P coarse on the liquid cells of MG level levelMgFine
 * (constant interpolation from the parent).  Replaces
 * prolongateChannel<float>(levelMgFine, chSrc, chDst, 0, alpha)
 * (src/msbg4.cpp:1920-2030, alpha = MG_CONST_PROLONGATION_ALPHA = 1). */
int msbg_gpu_prolongate(msbg_gpu_ctx* ctx, int levelMgFine, const float* coarse, int64_t nCoarse,
                        float* fine, int64_t nFine, float scale);

/* nIter smoothing sweeps of A x = b on MG level levelMg, x updated in place.
 * Replaces relax(0, reverse, levelMg, chX, chB, chTmp, nIter, 0)
 * (src/msbg3.cpp:2245-2369).
 *   mode 0: the solve's smoother: tiles red-black by (level, colour), inside
 *           each tile innerIter red-black Gauss-Seidel sweeps (reverse = the
 *           adjoint order of the post-smoother);
 *   mode 1: the reference's smoother: blocks red-black by (bx+by+bz)&1, in
 *           each block innerIter damped sweeps over 8-cell x groups (Jacobi
 *           inside a group, Gauss-Seidel across groups, directions
 *           alternating, last sweep Jacobi; src/msbg3.cpp:1109-1506,
 *           2171-2240) with damping omega (the reference's _mgSmOmega,
 *           src/msbg3.cpp:3088-3093; innerIter = _mgSmBlockIter = 5).  It needs
 *           one tile per block (16^3 base blocks) and follows the reference
 *           term by term across same-level faces. */
int msbg_gpu_relax(msbg_gpu_ctx* ctx, int levelMg, float* x, const float* b, int64_t n, int nIter,
                   int reverse, int innerIter, int mode, float omega);

/* z = V r on MG level 0 from z = 0: the solve's V-cycle (nPre / nPost
 * smoothing sweeps of innerIter tile sweeps, fused residual and restriction,
 * Galerkin coarse levels, FP64 direct coarsest solve, coarse correction
 * scaled by coarseScale).  Replaces vCycle(0, chZ, chR, chTmp, ...)
 * (src/msbg3.cpp:2412-2465).  The coarse levels differ: the reference's
 * restrictPressureMetaFLIP_ reads the fine flags at the coarse block level
 * (src/msbg3.cpp:2891) and leaves its coarse levels without liquid, so its
 * V-cycle reduces to the pre- and post-smoothing of level 0. */
int msbg_gpu_vcycle(msbg_gpu_ctx* ctx, const float* r, float* z, int64_t n, int nPre, int nPost,
                    int innerIter, float coarseScale);

/* ---- FLIP transfers around the pressure solve -------------------------
 * On the context's single-level grid (msbg_gpu_sync_topology with every block
 * at level 0, the reference's flip_sim grids), with device-resident grid
 * channels in the block layout (blocks in bid order, bsx^3 voxels, vid =
 * x + y*bsx + z*bsx^2).  The vector channels hold per voxel the MAC values
 * (u, v, w) of its lower x, y and z faces. */

/* FlipParticle (src/flip_sim.h:48): position and velocity in voxel units,
 * phase 0 liquid / 1 air; 28 bytes, the reference's layout. */
typedef struct {
  float pos[3], vel[3];
  int phase;
} msbg_flip_particle;

/* The FlipConfig fields the transfers read (src/flip_sim.h:29-45). */
typedef struct {
  float rhoL, rhoG, massEps, betaMin, alphaPhi;
  int particlesPerVoxel;
} msbg_flip_params;

enum { MSBG_FLIP_VEL = 0, MSBG_FLIP_VEL_OLD = 1, MSBG_FLIP_BETA = 2, MSBG_FLIP_MASS = 3 };

/* Replaces FlipSimulation::particleToGrid (src/flip_sim.cpp:579-831): the
 * particles' cell mass and trilinear face weights, the face velocities
 * normalised by their weights (0 where the weight is <= massEps), the face
 * coefficients beta = max(1/rho, betaMin) of the two-phase density with the
 * interface clamp.  activeBlocks / nActive (either may be NULL) receive the
 * ids of the blocks holding a cell with mass > massEps, ascending. */
int msbg_gpu_flip_p2g(msbg_gpu_ctx* ctx, const msbg_flip_particle* particles, int64_t np,
                      const msbg_flip_params* params, int* activeBlocks, int64_t* nActive);
/* Replaces FlipSimulation::applyGravity (src/flip_sim.cpp:832-857): the
 * velocity is kept as MSBG_FLIP_VEL_OLD, gravity*dt is added to the v faces
 * next to liquid, and the reference's wall faces are set to 0. */
int msbg_gpu_flip_gravity(msbg_gpu_ctx* ctx, float gravity, float dt, float massEps);
/* Replaces the pressure-gradient update of FlipSimulation::pressureProjection
 * (src/flip_sim.cpp:1316-1349): u -= dt * beta * (p_b - p_a) on every face
 * with liquid on a side (p = 0 in a cell without), 0 on faces without liquid
 * and on the lower domain faces.  pressure: host array in the block layout
 * (msbg_gpu_pressure_download of a grid whose blocks are all at level 0). */
int msbg_gpu_flip_pressure_gradient(msbg_gpu_ctx* ctx, const float* pressure, float dt,
                                    float massEps);
/* Replaces FlipSimulation::gridToParticle (src/flip_sim.cpp:1526-1545) with
 * the level-0 branch of interpVec3MSBG (src/flip_sim.cpp:1354-1395):
 * vel = (1 - alpha) pic + alpha (vel + pic - old), pic and old trilinear in
 * MSBG_FLIP_VEL and MSBG_FLIP_VEL_OLD.  Updates the particles in place. */
int msbg_gpu_flip_g2p(msbg_gpu_ctx* ctx, msbg_flip_particle* particles, int64_t np,
                      float flipAlpha);
/* The same two transfers on particles that stay in device memory (a
 * cudaMalloc'd array the caller owns), ordered on the context's stream. */
int msbg_gpu_flip_p2g_device(msbg_gpu_ctx* ctx, const msbg_flip_particle* particles, int64_t np,
                             const msbg_flip_params* params, int* activeBlocks, int64_t* nActive);
int msbg_gpu_flip_g2p_device(msbg_gpu_ctx* ctx, msbg_flip_particle* particles, int64_t np,
                             float flipAlpha);
/* Copies a channel out (get = 1) or in (get = 0); n = 3 * voxels for the
 * vector channels, voxels for MSBG_FLIP_MASS. */
int msbg_gpu_flip_channel(msbg_gpu_ctx* ctx, int which, float* data, int64_t n, int get);

/* ---- G2P on mixed-resolution grids --------------------------------------
 * On the context's topology (msbg_gpu_sync_topology; blocks whose 26
 * neighbours differ from them by at most one level, as the reference
 * asserts), with channels in the packed layout of the pressure channels: for
 * every block in ascending bid, its (bsx0>>level)^3 voxels at its own level
 * (vid = x + y*bs + z*bs^2).  A voxel of a level's grid that lies in a block
 * of another level reads 0, as a NULL block of that level's sparse grid. */

/* Builds the fine/coarse distance channel CH_DIST_FINECOARSE of every level
 * as setRefinementMap does (src/msbg.cpp:1700-1723, 1887-1960, 1994-2029) and,
 * where dist / kind are not NULL, copies it out: dist (n = packed voxels)
 * holds the distances (uint16, voxels of the block's level times 1024) of the
 * blocks with a coarser neighbour, 0 elsewhere; kind[l*nBlocks + b] (nk =
 * nLevels * nBlocks) is block b's kind in the channel of level l: 0 empty,
 * 1 value block, 2 full block of value 6*1024 (dTransRes is 6,
 * src/msbg.cpp:201).  msbg_gpu_flip_g2p_mr builds it by itself. */
int msbg_gpu_flip_mr_dist(msbg_gpu_ctx* ctx, uint16_t* dist, int64_t n, int8_t* kind,
                          int64_t nk);
/* Copies the mixed-resolution velocity channel MSBG_FLIP_VEL or
 * MSBG_FLIP_VEL_OLD out (get = 1) or in (get = 0): per voxel the lower-face
 * MAC values (u, v, w) at the voxel's level, n = 3 * packed voxels.  These
 * are the reference's getVecChannel(CH_VEC3_4 / CH_VEC3_2, level, 0) of every
 * level, merged block by block. */
int msbg_gpu_flip_mr_channel(msbg_gpu_ctx* ctx, int which, float* data, int64_t n, int get);
/* Replaces FlipSimulation::gridToParticle (src/flip_sim.cpp:1526-1545) on a
 * grid with several levels: vel = (1 - alpha) pic + alpha (vel + pic - old),
 * pic and old from interpVec3MSBG / interpCompMSBG (src/flip_sim.cpp:
 * 1354-1525): in a level-0 block the trilinear MAC interpolation of the
 * level-0 channel; in a block of level L > 0 that of the level-L channel at
 * the position scaled by 2^-L, blended with the level-0 interpolation by
 * MtLinstep(1.01 sqrt3, 0.99 (dTransRes + 2) / sqrt3, d), d the level-L
 * distance channel interpolated there / 1024.  Updates the particles in
 * place; the _device form takes particles in device memory (a cudaMalloc'd
 * array the caller owns), ordered on the context's stream. */
int msbg_gpu_flip_g2p_mr(msbg_gpu_ctx* ctx, msbg_flip_particle* particles, int64_t np,
                         float flipAlpha);
int msbg_gpu_flip_g2p_mr_device(msbg_gpu_ctx* ctx, msbg_flip_particle* particles, int64_t np,
                                float flipAlpha);

/* Replaces MultiresSparseGrid::downsampleVelocity(levelMg, chSrc, chDst)
 * (src/msbg4.cpp:2035-2270): the velocity of MG level levelMg - 1 restricted
 * to MG level levelMg (1 <= levelMg < nLevels, the sparse MG levels).  At MG
 * level m a block sits at level max(its level, m) (getBlockLevel,
 * src/msbg.h:3574-3590); src (nSrc = 3 * packed voxels of MG level m-1) and
 * dst (nDst = 3 * those of MG level m) use the packed layout at those levels,
 * 3 floats per voxel; flags are the CellFlags of MG level m, packed (the
 * reference's CH_CELL_FLAGS after preparePressureSolveFLIP).  A block already
 * at level >= m is copied (0 in CELL_SOLID or CELL_VOID cells); a coarsened
 * block takes the 4x4x4 (1,3,3,1)^3/512 filter of the finer cells, 0 in
 * CELL_SOLID cells.  Host arrays; the copies are inside the call. */
int msbg_gpu_flip_downsample_velocity(msbg_gpu_ctx* ctx, int levelMg, const uint16_t* flags,
                                      const float* src, int64_t nSrc, float* dst, int64_t nDst);

/* ---- particle splatting -------------------------------------------------- */

/* The splat parameters of the reference's demo (src/msbg_demo.cpp:235-236,
 * rParticle 2, nbDist 2): particles reach rScan = rParticle + nbDist voxels;
 * rScan + 1 must not exceed the base block size. */
typedef struct {
  float rParticle, nbDist;
  int flags; /* MSBG_SPLAT_RAW: leave the quantised squared distances */
} msbg_splat_params;

enum { MSBG_SPLAT_RAW = 1 };

/* Replaces the particle splatting of the reference's demo (msbg_test_sparse,
 * src/msbg_demo.cpp:339-684) on the context's level-0 block raster:
 *   pos[3n]  particle positions in voxel units (x, y, z); particles outside
 *            [1e-4, s - 1e-4] on an axis, or not finite, are dropped
 *            (isInDomainRange + inRange, src/msbg_demo.cpp:358-360)
 *   kind     NULL: every block within rScan of a kept particle becomes a
 *            value block, the others const empty blocks (the demo's marking
 *            and refinement map, src/msbg_demo.cpp:366-500); else the caller's
 *            MSBG_BLOCK_* per block
 *   kindOut  optional [nBlocks]: the kinds used
 * Creates 16-bit channel `chan` (msbg_gpu_upload_channel_u16 layout, const
 * empty 0, full 65535): every value voxel at 65535, lowered by each particle
 * to round(d^2 / rScan^2 * 65535) over the voxels of its scan box within
 * rScan (a particle whose scan meets a block without values stops there, as
 * the reference's goto does), then finalised to
 * round((1 - linstep(-rParticle, rParticle + nbDist, d - rParticle)) * 65535)
 * for d^2 < 0.999 rScan^2, else 0 (src/msbg_demo.cpp:661-675).  The channel
 * is the smoother's input: msbg_gpu_pde_mcf runs on it directly.  Returns
 * when the channel is complete. */
int msbg_gpu_splat_particles(msbg_gpu_ctx* ctx, int chan, const float* pos, int64_t n,
                             const msbg_splat_params* params, const int8_t* kind,
                             int8_t* kindOut);
/* The same with `pos` in device memory (read on the context's stream). */
int msbg_gpu_splat_particles_device(msbg_gpu_ctx* ctx, int chan, const float* pos, int64_t n,
                                    const msbg_splat_params* params, const int8_t* kind,
                                    int8_t* kindOut);

/* Diagnostics without a GPU (no counterpart in the reference): builds the
 * multigrid hierarchy as msbg_gpu_pressure_prepare does, then on the host
 *   yPacked = A xPacked on MG level 0 (block layout; both may be NULL),
 *   fluidPerLevel[m] = liquid cells of MG level m (m < 32),
 *   galerkinErr[m] = max|P^T A_m P x - A_{m+1} x| / max|P^T A_m P x| for a
 *                    random x (m < 32; NULL to skip). */
int msbg_gpu_pressure_host_check(const msbg_topo_desc* topo, const msbg_pressure_callbacks* cb,
                                 const float* xPacked, double* yPacked, int* nMgLevels,
                                 int64_t* fluidPerLevel, double* galerkinErr);

#ifdef __cplusplus
}
#endif

#endif /* MSBG_GPU_H */
