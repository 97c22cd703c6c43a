// Component entry points of the pressure solver: one call each for the
// operator, the residual, the grid transfers, the smoother and the V-cycle of
// a prepared hierarchy, on vectors in the reference's packed block layout of
// one MG level.  They replace single calls of the reference's solver pieces
// (src/msbg3.cpp, src/msbg4.cpp; line ranges at each entry point) so that a
// caller, or a test, can compare them one call at a time.
//
// Each call uploads its inputs, scatters them into the tile layout of the
// level, runs the same kernels the solve launches (k_apply_pipe16 /
// k_matvec_dot, k_residual_restrict / k_apply_pipe16<RESIDUAL>, k_prolong,
// k_smooth_pipe16 / k_smooth, the V-cycle) on temporary vectors, gathers the
// result back into the block layout and waits for it.  The solver's own
// vectors are not touched, except the coarse-level scratch of the V-cycle.
//
// Also here: the reference-compatible block smoother (mode 1 of
// msbg_gpu_relax) and the bulk-array form of msbg_gpu_pressure_prepare.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "pressure_solver.cuh"

namespace msbg {
namespace ps {
namespace {

// ---------------------------------------------------------------------------
// block layout of one MG level
// ---------------------------------------------------------------------------
// MG level m < nLevels holds every base block b at resolution level
// max(map[b], m) (src/msbg.cpp:1650), (bsx0 >> level)^3 cells per block in
// the order vid = x + y*bs + z*bs*bs (src/sbg.h:1818-1822), blocks in bid
// order.  A tile is a cube of cells at one level: part of a block (32^3
// blocks hold 8 tiles) or, on a uniform level, several blocks.
struct TileDesc {
  int64_t off;  // first cell in the level's tile layout
  int level, ts, ox, oy, oz, pad;
};

template <bool TO_PACKED>
__global__ void __launch_bounds__(256) k_block_layout(const TileDesc* __restrict__ td,
                                                      const int64_t* __restrict__ boff, int nbx,
                                                      int nby, int bsx0, float* __restrict__ tv,
                                                      float* __restrict__ packed) {
  const TileDesc T = td[blockIdx.x];
  const int bs = bsx0 >> T.level;
  const int n = T.ts * T.ts * T.ts;
  for (int e = threadIdx.x; e < n; e += blockDim.x) {
    const int X = T.ox + e % T.ts, Y = T.oy + (e / T.ts) % T.ts, Z = T.oz + e / (T.ts * T.ts);
    const int64_t b = (X / bs) + (int64_t)nbx * ((Y / bs) + (int64_t)nby * (Z / bs));
    const int64_t p = boff[b] + (X % bs) + (int64_t)bs * ((Y % bs) + (int64_t)bs * (Z % bs));
    if (TO_PACKED)
      packed[p] = tv[T.off + e];
    else
      tv[T.off + e] = packed[p];
  }
}

// r = b - q on liquid cells (a_ii > 0), 0 elsewhere.
__global__ void k_b_minus(const float* __restrict__ b, const float* __restrict__ q,
                          const float* __restrict__ diag, float* __restrict__ r, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    r[i] = diag[i] > 0.f ? b[i] - q[i] : 0.f;
}

// ---------------------------------------------------------------------------
// the reference's block smoother
// ---------------------------------------------------------------------------
// One call of processBlockLaplacian<LAPL_RELAX> per block (src/msbg3.cpp:
// 564-1044 gather, 1109-1506 update; RELAX_BLOCK_GAUSS_SEIDEL,
// src/msbgcell.h:97), on the tile = block of the level:
//   * the block and its six face slabs are copied into a halo buffer as
//     F = x*h (ghosts frozen for the call; cells of 8-lane groups that hold
//     no liquid read 0);
//   * nIter block-local sweeps over the SW-cell groups of x rows in the
//     order (z, y, x-group), forward or backward: backward when
//     (reverse != 0) == (iteration odd) (src/msbg3.cpp:1148-1161);
//   * in a group, every lane reads the buffer before any lane writes, so the
//     update is Jacobi inside a group and Gauss-Seidel across groups:
//       S = fma(F6, W6, ... fma(F1, W1, 0)) over x-, x+, y-, y+, z-, z+,
//       Y = D != 0 ? omega (B + S) D + (1 - omega) F0 : F0;
//   * iterations 0..nIter-2 write Y into the buffer, the last one writes
//     Y / h to x (so the last sweep is Jacobi with respect to the buffer).
// The group order is a dependence order: group (g, y, z) reads updated values
// only from (g-1, y, z), (g, y-1, z) and (g, y, z-1), and old values only
// from their successors, so the CTA runs the sweep as wavefronts
// t = g + y + z (forward; mirrored backward), one group of SW lanes per
// (g, z) slot.  W are the face weights (couplings / h), D = 1 / (a_ii / h) the
// reference's inverse face sum (src/msbg3.cpp:2686-2731; equal where the
// operators coincide).  Interface faces (level jumps) enter as F = the
// operator's interface sum with W = 1: only same-level faces follow the
// reference term by term.
template <int BS, int SW>
__global__ void __launch_bounds__(BS* BS) k_relax_block_ref(LevelView L, int tileBase,
                                                            float* __restrict__ x,
                                                            const float* __restrict__ b, float h,
                                                            float omega, int nIter, int reverse) {
  constexpr int H = BS + 2, H2 = H * H, N = BS * BS * BS, NG = BS / SW, NT = BS * BS;
  __shared__ float F[H * H * H];
  __shared__ float Dg[N];
  __shared__ float gw[6][BS * BS];  // weights of the ghost faces
  __shared__ unsigned char groupLiquid[N / SW];
  const int ti = tileBase + blockIdx.x;
  const int64_t off = L.tileOff[ti];
  const int tid = threadIdx.x;
  const float hr = 1.0f / h;
  for (int e = tid; e < N / SW; e += NT) {
    bool any = false;
    for (int k = 0; k < SW; k++) any |= L.diag[off + e * SW + k] > 0.f;
    groupLiquid[e] = any;
  }
  for (int e = tid; e < H * H * H; e += NT) F[e] = 0.f;
  __syncthreads();
  for (int e = tid; e < N; e += NT) {
    const int vx = e % BS, vy = (e / BS) % BS, vz = e / (BS * BS);
    const float a = L.diag[off + e];
    Dg[e] = a > 0.f ? 1.0f / (a * hr) : 0.f;
    F[(vx + 1) + H * (vy + 1) + H2 * (vz + 1)] = groupLiquid[e / SW] ? x[off + e] * h : 0.f;
  }
  // face slabs: plane index (a, b) on the face's tangential axes
  for (int f = 0; f < 6; f++) {
    const int dir = f >> 1, side = f & 1;
    const int* Fd = L.face + ((size_t)ti * 6 + f) * FACE_INTS;
    const int kind = Fd[F_KIND];
    const float* cd = dir == 0 ? L.cx : dir == 1 ? L.cy : L.cz;
    for (int q = tid; q < BS * BS; q += NT) {
      const int a = q % BS, bb = q / BS;
      const int p = side ? BS : -1;  // position along dir in block cells
      int c3[3];
      c3[dir] = p;
      c3[dir == 0 ? 1 : 0] = a;
      c3[dir == 2 ? 1 : 2] = bb;
      const int hidx = (c3[0] + 1) + H * (c3[1] + 1) + H2 * (c3[2] + 1);
      float Fv = 0.f, Wv = 0.f;
      if (kind == FACE_SAME) {
        const int64_t no = L.tileOff[Fd[F_T0]];
        Fv = x[no + plane_idx(BS, dir, side ? 0 : BS - 1, a, bb)] * h;
        Wv = side ? cd[no + plane_idx(BS, dir, 0, a, bb)] * hr
                  : cd[off + plane_idx(BS, dir, 0, a, bb)] * hr;
      } else if (kind == FACE_COARSER || kind == FACE_FINER) {
        Fv = ghost_sum<float, float>(L, x, ti, BS, dir, side, a, bb);
        Wv = 1.f;
      } else if (!side) {
        Wv = cd[off + plane_idx(BS, dir, 0, a, bb)] * hr;  // own lower face, ghost F = 0
      }
      F[hidx] = Fv;
      gw[f][q] = Wv;
    }
  }
  __syncthreads();
  const int lane = tid % SW, slot = tid / SW;
  const int sg = slot % NG, sz = slot / NG;  // group column and z of this thread's slot
  const float om1 = 1.0f - omega;
  for (int it = 0; it < nIter; it++) {
    const bool back = (reverse != 0) == ((it & 1) != 0);
    const bool last = it == nIter - 1;
    for (int t = 0; t < NG + 2 * BS - 2; t++) {
      // group of this slot at wavefront t, mirrored for a backward sweep
      int g = sg, vz = sz, vy = t - sg - sz;
      const bool active = vy >= 0 && vy < BS;
      if (back) {
        g = NG - 1 - g;
        vy = BS - 1 - vy;
        vz = BS - 1 - vz;
      }
      float Y = 0.f;
      int c = 0, e = 0;
      bool write = false;
      if (active) {
        const int vx = g * SW + lane;
        e = vx + BS * (vy + BS * vz);
        write = groupLiquid[e / SW] != 0;
        if (write) {
          c = (vx + 1) + H * (vy + 1) + H2 * (vz + 1);
          const float F0 = F[c];
          const float W1 = L.cx[off + e] * hr;
          const float W2 = vx < BS - 1 ? L.cx[off + e + 1] * hr : gw[1][vy + BS * vz];
          const float W3 = L.cy[off + e] * hr;
          const float W4 = vy < BS - 1 ? L.cy[off + e + BS] * hr : gw[3][vx + BS * vz];
          const float W5 = L.cz[off + e] * hr;
          const float W6 = vz < BS - 1 ? L.cz[off + e + BS * BS] * hr : gw[5][vx + BS * vy];
          // lower ghost faces: W from the face slab (interface faces W = 1)
          const float W1g = vx == 0 ? gw[0][vy + BS * vz] : W1;
          const float W3g = vy == 0 ? gw[2][vx + BS * vz] : W3;
          const float W5g = vz == 0 ? gw[4][vx + BS * vy] : W5;
          float S = 0.f;
          S = __fmaf_rn(F[c - 1], W1g, S);
          S = __fmaf_rn(F[c + 1], W2, S);
          S = __fmaf_rn(F[c - H], W3g, S);
          S = __fmaf_rn(F[c + H], W4, S);
          S = __fmaf_rn(F[c - H2], W5g, S);
          S = __fmaf_rn(F[c + H2], W6, S);
          const float D = Dg[e];
          const float B = b[off + e];
          Y = D != 0.f ? __fadd_rn(__fmul_rn(__fmul_rn(omega, __fadd_rn(B, S)), D),
                                   __fmul_rn(om1, F0))
                       : F0;
        }
      }
      __syncthreads();  // every lane of every group has read the buffer
      if (write) {
        if (!last)
          F[c] = Y;
        else
          x[off + e] = Y * hr;
      }
      __syncthreads();
    }
  }
}

// ---------------------------------------------------------------------------
// per-call helper: the level's block layout on the device and temporaries
// ---------------------------------------------------------------------------
struct Part {
  msbg_gpu_ctx* ctx;
  Solver& S;
  int m;
  cudaStream_t st;
  int64_t count = 0;          // packed values of the level
  DeviceBuffer td, boff, packed;

  Part(msbg_gpu_ctx* c, Solver& s, int level) : ctx(c), S(s), m(level), st(c->stream) {}

  int init() {
    const Level& L = S.H.levels[m];
    const int64_t nb = (int64_t)S.nbx * S.nby * S.nbz;
    std::vector<int64_t> bo(nb);
    count = 0;
    for (int64_t b = 0; b < nb; b++) {
      const int bs = S.bsx0 >> std::max(S.blockLevel[b], m);
      bo[b] = count;
      count += (int64_t)bs * bs * bs;
    }
    std::vector<TileDesc> t(L.tiles.size());
    for (size_t i = 0; i < t.size(); i++) {
      const Tile& T = L.tiles[i];
      t[i] = TileDesc{T.off, T.level, T.ts, T.ox, T.oy, T.oz, 0};
    }
    MSBG_CUDA_TRY(ctx, boff.ensure(sizeof(int64_t) * std::max<int64_t>(nb, 1)));
    MSBG_CUDA_TRY(ctx, td.ensure(sizeof(TileDesc) * std::max<size_t>(t.size(), 1)));
    MSBG_CUDA_TRY(ctx, packed.ensure(sizeof(float) * std::max<int64_t>(count, 1)));
    MSBG_CUDA_TRY(ctx, cudaMemcpyAsync(boff.p, bo.data(), sizeof(int64_t) * nb,
                                       cudaMemcpyHostToDevice, st));
    if (!t.empty())
      MSBG_CUDA_TRY(ctx, cudaMemcpyAsync(td.p, t.data(), sizeof(TileDesc) * t.size(),
                                         cudaMemcpyHostToDevice, st));
    MSBG_CUDA_TRY(ctx, cudaStreamSynchronize(st));  // host vectors are temporaries
    return MSBG_OK;
  }
  int64_t cells() const { return S.H.levels[m].nCells; }
  // host packed -> tile layout (cells outside the tiles are dropped)
  int unpack(const float* host, DeviceBuffer& dst) {
    MSBG_CUDA_TRY(ctx, dst.ensure(sizeof(float) * std::max<int64_t>(cells(), 4)));
    MSBG_CUDA_TRY(ctx, cudaMemsetAsync(dst.p, 0, sizeof(float) * std::max<int64_t>(cells(), 4), st));
    MSBG_CUDA_TRY(ctx, copy_h2d(packed.p, host, sizeof(float) * count, st));
    const unsigned nt = (unsigned)S.H.levels[m].tiles.size();
    if (nt)
      k_block_layout<false><<<nt, 256, 0, st>>>(td.as<TileDesc>(), boff.as<int64_t>(), S.nbx,
                                                S.nby, S.bsx0, dst.as<float>(), packed.as<float>());
    MSBG_CUDA_TRY(ctx, cudaGetLastError());
    return MSBG_OK;
  }
  // tile layout -> host packed (cells of blocks without tiles read 0)
  int pack(const DeviceBuffer& src, float* host) {
    MSBG_CUDA_TRY(ctx, cudaMemsetAsync(packed.p, 0, sizeof(float) * count, st));
    const unsigned nt = (unsigned)S.H.levels[m].tiles.size();
    if (nt)
      k_block_layout<true><<<nt, 256, 0, st>>>(td.as<TileDesc>(), boff.as<int64_t>(), S.nbx,
                                               S.nby, S.bsx0, src.as<float>(), packed.as<float>());
    MSBG_CUDA_TRY(ctx, cudaGetLastError());
    MSBG_CUDA_TRY(ctx, copy_d2h(host, packed.p, sizeof(float) * count, st));
    return MSBG_OK;
  }
};

// Solver of a context, its MG level m checked against the block layout.
int part_level(msbg_gpu_ctx* ctx, int m, Solver** out) {
  if (!ctx) return MSBG_EINVARG;
  Solver* S = find_solver(ctx);
  if (!S) return set_error(ctx, MSBG_EINVARG, "no prepared pressure problem");
  if (m < 0 || m >= (int)S->H.levels.size() - 1 || m >= S->H.nLevels)
    return set_error(ctx, MSBG_EINVARG,
                     "MG level %d has no block layout (levels 0..%d of %d resolution levels)", m,
                     std::min((int)S->H.levels.size() - 2, S->H.nLevels - 1), S->H.nLevels);
  cudaSetDevice(ctx->device);
  set_kernel_attrs<float>();
  *out = S;
  return MSBG_OK;
}

int check_count(msbg_gpu_ctx* ctx, const Part& P, int64_t n, const char* what) {
  if (n != P.count)
    return set_error(ctx, MSBG_EINVARG, "%s: %lld values given, MG level %d holds %lld", what,
                     (long long)n, P.m, (long long)P.count);
  return MSBG_OK;
}

// Wait for the stream and report a kernel whose bounded wait gave up.
int finish(msbg_gpu_ctx* ctx) {
  return msbg_gpu_sync(ctx);
}

// q = A_m x over all tiles of level m (the solve's operator kernels).
void launch_matvec(Solver& S, int m, const float* x, float* q, cudaStream_t st, int* err) {
  const Level& L = S.H.levels[m];
  for (const auto& P : L.passes) {
    if (!P.count) continue;
    if (P.ts == 16) {
      const int grid = std::min(P.count, S.numSMs);
      k_apply_pipe16<APPLY_MATVEC, float, float, pipe::NT_APPLY>
          <<<grid, pipe::NT_APPLY, pipe::SMEM, st>>>(S.views[m], P.start, P.count, x, nullptr, q,
                                                     nullptr, nullptr, nullptr, err, nullptr);
    } else {
      const int* lst = S.dev[m]->passTiles.as<int>() + P.start;
      TS_DISPATCH(P.ts, (k_matvec_dot<T, float><<<P.count, T * T, 0, st>>>(S.views[m], lst, x, q,
                                                                            nullptr)));
    }
  }
}

// Reference-compatible smoother: nIter calls of relaxBlockList, each the two
// block-parity passes (src/msbg3.cpp:2171-2240, 2245-2369).
int relax_reference(msbg_gpu_ctx* ctx, Solver& S, int m, float* x, const float* b, int nIter,
                    int reverse, int blockIter, float omega) {
  const Level& L = S.H.levels[m];
  for (const Tile& t : L.tiles)
    if (t.ts != (S.bsx0 >> t.level))
      return set_error(ctx, MSBG_ENOTIMPL,
                       "reference-compatible smoother: MG level %d has %d^3 tiles in %d^3 blocks "
                       "(needs one tile per block, e.g. 16^3 base blocks)",
                       m, t.ts, S.bsx0 >> t.level);
  cudaStream_t st = ctx->stream;
  for (int it = 0; it < nIter; it++)
    for (int k = 0; k < 2; k++) {
      // pass k relaxes the blocks of parity (reverse ? k : 1 - k)
      const int parity = reverse ? k : 1 - k;
      for (const auto& P : L.passes) {
        if (!P.count || P.colour != parity) continue;
        const float h = (float)(1 << P.level);
        switch (P.ts) {
          case 16:
            k_relax_block_ref<16, 8><<<P.count, 256, 0, st>>>(S.views[m], P.start, x, b, h, omega,
                                                              blockIter, reverse);
            break;
          case 8:
            k_relax_block_ref<8, 8><<<P.count, 64, 0, st>>>(S.views[m], P.start, x, b, h, omega,
                                                            blockIter, reverse);
            break;
          case 4:
            k_relax_block_ref<4, 4><<<P.count, 16, 0, st>>>(S.views[m], P.start, x, b, h, omega,
                                                            blockIter, reverse);
            break;
          case 2:
            k_relax_block_ref<2, 2><<<P.count, 4, 0, st>>>(S.views[m], P.start, x, b, h, omega,
                                                           blockIter, reverse);
            break;
          default:
            return set_error(ctx, MSBG_ENOTIMPL, "block size %d", P.ts);
        }
      }
    }
  MSBG_CUDA_TRY(ctx, cudaGetLastError());
  return MSBG_OK;
}

// ---------------------------------------------------------------------------
// bulk-array prepare: callbacks that read the caller's arrays
// ---------------------------------------------------------------------------
}  // namespace
}  // namespace ps
}  // namespace msbg

using namespace msbg;
using namespace msbg::ps;

extern "C" int msbg_gpu_pressure_level_size(msbg_gpu_ctx* ctx, int levelMg, int64_t* n) {
  if (!n) return MSBG_EINVARG;
  Solver* S = nullptr;
  int rc = part_level(ctx, levelMg, &S);
  if (rc) return rc;
  int64_t c = 0;
  for (int l : S->blockLevel) {
    const int bs = S->bsx0 >> std::max(l, levelMg);
    c += (int64_t)bs * bs * bs;
  }
  *n = c;
  return MSBG_OK;
}

extern "C" int msbg_gpu_pressure_diagonal(msbg_gpu_ctx* ctx, int levelMg, float* diag, int64_t n) {
  if (!diag) return MSBG_EINVARG;
  Solver* S = nullptr;
  int rc = part_level(ctx, levelMg, &S);
  if (rc) return rc;
  Part P(ctx, *S, levelMg);
  if ((rc = P.init()) || (rc = check_count(ctx, P, n, "diagonal"))) return rc;
  return P.pack(S->dev[levelMg]->diag, diag);
}

extern "C" int msbg_gpu_matvec(msbg_gpu_ctx* ctx, int levelMg, const float* x, float* y,
                               int64_t n) {
  if (!x || !y) return MSBG_EINVARG;
  Solver* S = nullptr;
  int rc = part_level(ctx, levelMg, &S);
  if (rc) return rc;
  Part P(ctx, *S, levelMg);
  if ((rc = P.init()) || (rc = check_count(ctx, P, n, "matvec"))) return rc;
  DeviceBuffer dx, dy;
  if ((rc = P.unpack(x, dx))) return rc;
  MSBG_CUDA_TRY(ctx, dy.ensure(dx.bytes));
  MSBG_CUDA_TRY(ctx, cudaMemsetAsync(dy.p, 0, dx.bytes, ctx->stream));
  launch_matvec(*S, levelMg, dx.as<float>(), dy.as<float>(), ctx->stream, ctx->errBuf.as<int>());
  MSBG_CUDA_TRY(ctx, cudaGetLastError());
  if ((rc = P.pack(dy, y))) return rc;
  return finish(ctx);
}

extern "C" int msbg_gpu_residual(msbg_gpu_ctx* ctx, int levelMg, const float* x, const float* b,
                                 float* r, int64_t n) {
  if (!x || !b || !r) return MSBG_EINVARG;
  Solver* S = nullptr;
  int rc = part_level(ctx, levelMg, &S);
  if (rc) return rc;
  Part P(ctx, *S, levelMg);
  if ((rc = P.init()) || (rc = check_count(ctx, P, n, "residual"))) return rc;
  DeviceBuffer dx, db, dq;
  if ((rc = P.unpack(x, dx)) || (rc = P.unpack(b, db))) return rc;
  MSBG_CUDA_TRY(ctx, dq.ensure(dx.bytes));
  MSBG_CUDA_TRY(ctx, cudaMemsetAsync(dq.p, 0, dx.bytes, ctx->stream));
  launch_matvec(*S, levelMg, dx.as<float>(), dq.as<float>(), ctx->stream, ctx->errBuf.as<int>());
  k_b_minus<<<2 * S->numSMs, 256, 0, ctx->stream>>>(db.as<float>(), dq.as<float>(),
                                                    S->dev[levelMg]->diag.as<float>(),
                                                    dq.as<float>(), P.cells());
  MSBG_CUDA_TRY(ctx, cudaGetLastError());
  if ((rc = P.pack(dq, r))) return rc;
  return finish(ctx);
}

extern "C" int msbg_gpu_restrict(msbg_gpu_ctx* ctx, int levelMgCoarse, const float* fine,
                                 int64_t nFine, float* coarse, int64_t nCoarse) {
  if (!fine || !coarse) return MSBG_EINVARG;
  Solver* S = nullptr;
  int rc = part_level(ctx, levelMgCoarse - 1, &S);
  if (rc) return rc;
  if (levelMgCoarse >= S->H.nLevels)
    return set_error(ctx, MSBG_EINVARG, "coarse MG level %d has no block layout", levelMgCoarse);
  const int mf = levelMgCoarse - 1;
  Part PF(ctx, *S, mf), PC(ctx, *S, levelMgCoarse);
  if ((rc = PF.init()) || (rc = PC.init()) || (rc = check_count(ctx, PF, nFine, "restrict")) ||
      (rc = check_count(ctx, PC, nCoarse, "restrict")))
    return rc;
  // The solve restricts fused with the residual: r = b - A x, then the sum
  // over the liquid children.  With x = 0 the kernels restrict b itself.
  DeviceBuffer dx, db, dc;
  if ((rc = PF.unpack(fine, db))) return rc;
  MSBG_CUDA_TRY(ctx, dx.ensure(db.bytes));
  MSBG_CUDA_TRY(ctx, cudaMemsetAsync(dx.p, 0, db.bytes, ctx->stream));
  const size_t cb = sizeof(float) * std::max<int64_t>(PC.cells(), 4);
  MSBG_CUDA_TRY(ctx, dc.ensure(cb));
  MSBG_CUDA_TRY(ctx, cudaMemsetAsync(dc.p, 0, cb, ctx->stream));
  const Level& L = S->H.levels[mf];
  const int64_t* coff = S->dev[levelMgCoarse]->tileOff.as<int64_t>();
  cudaStream_t st = ctx->stream;
  int* err = ctx->errBuf.as<int>();
  for (const auto& Pp : L.passes) {
    if (!Pp.count) continue;
    if (Pp.ts == 16) {
      const int grid = std::min(Pp.count, S->numSMs);
      k_apply_pipe16<APPLY_RESIDUAL, float, float, pipe::NT_APPLY>
          <<<grid, pipe::NT_APPLY, pipe::SMEM, st>>>(S->views[mf], Pp.start, Pp.count,
                                                     dx.as<float>(), db.as<float>(), nullptr,
                                                     dc.as<float>(), coff, nullptr, err, nullptr);
    } else {
      const int* lst = S->dev[mf]->passTiles.as<int>() + Pp.start;
      TS_DISPATCH(Pp.ts, (k_residual_restrict<T, float, float><<<Pp.count, T * T, 0, st>>>(
                             S->views[mf], lst, dx.as<float>(), db.as<float>(), dc.as<float>(),
                             coff)));
    }
  }
  MSBG_CUDA_TRY(ctx, cudaGetLastError());
  if ((rc = PC.pack(dc, coarse))) return rc;
  return finish(ctx);
}

extern "C" int msbg_gpu_prolongate(msbg_gpu_ctx* ctx, int levelMgFine, const float* coarse,
                                   int64_t nCoarse, float* fine, int64_t nFine, float scale) {
  if (!fine || !coarse) return MSBG_EINVARG;
  Solver* S = nullptr;
  int rc = part_level(ctx, levelMgFine, &S);
  if (rc) return rc;
  if (levelMgFine + 1 >= S->H.nLevels)
    return set_error(ctx, MSBG_EINVARG, "coarse MG level %d has no block layout", levelMgFine + 1);
  const int mc = levelMgFine + 1;
  Part PF(ctx, *S, levelMgFine), PC(ctx, *S, mc);
  if ((rc = PF.init()) || (rc = PC.init()) || (rc = check_count(ctx, PF, nFine, "prolongate")) ||
      (rc = check_count(ctx, PC, nCoarse, "prolongate")))
    return rc;
  DeviceBuffer dfine, dc;
  if ((rc = PF.unpack(fine, dfine)) || (rc = PC.unpack(coarse, dc))) return rc;
  const Level& L = S->H.levels[levelMgFine];
  const int64_t* coff = S->dev[mc]->tileOff.as<int64_t>();
  cudaStream_t st = ctx->stream;
  for (const auto& g : L.groups) {
    const int* lst = S->dev[levelMgFine]->groupTiles.as<int>() + g.start;
    TS_DISPATCH(g.ts, (k_prolong<T, float, float><<<g.count, T * T, 0, st>>>(
                          S->views[levelMgFine], lst, dfine.as<float>(), dc.as<float>(), coff,
                          scale, nullptr)));
  }
  MSBG_CUDA_TRY(ctx, cudaGetLastError());
  if ((rc = PF.pack(dfine, fine))) return rc;
  return finish(ctx);
}

extern "C" int msbg_gpu_relax(msbg_gpu_ctx* ctx, int levelMg, float* x, const float* b, int64_t n,
                              int nIter, int reverse, int innerIter, int mode, float omega) {
  if (!x || !b || nIter < 0 || innerIter < 1 || (mode != 0 && mode != 1)) return MSBG_EINVARG;
  Solver* S = nullptr;
  int rc = part_level(ctx, levelMg, &S);
  if (rc) return rc;
  Part P(ctx, *S, levelMg);
  if ((rc = P.init()) || (rc = check_count(ctx, P, n, "relax"))) return rc;
  DeviceBuffer dx, db;
  if ((rc = P.unpack(x, dx)) || (rc = P.unpack(b, db))) return rc;
  if (mode == 0) {
    Runner<float> R{*S, ctx->stream, 0, 0, innerIter};
    R.err = ctx->errBuf.as<int>();
    R.numSMs = S->numSMs;
    for (int it = 0; it < nIter; it++) R.smooth(levelMg, dx.as<float>(), db.as<float>(), reverse != 0);
  } else {
    rc = relax_reference(ctx, *S, levelMg, dx.as<float>(), db.as<float>(), nIter, reverse,
                         innerIter, omega);
    if (rc) return rc;
  }
  MSBG_CUDA_TRY(ctx, cudaGetLastError());
  if ((rc = P.pack(dx, x))) return rc;
  return finish(ctx);
}

extern "C" int msbg_gpu_vcycle(msbg_gpu_ctx* ctx, const float* r, float* z, int64_t n, int nPre,
                               int nPost, int innerIter, float coarseScale) {
  if (!r || !z || nPre < 0 || nPost < 0 || innerIter < 1) return MSBG_EINVARG;
  Solver* S = nullptr;
  int rc = part_level(ctx, 0, &S);
  if (rc) return rc;
  Part P(ctx, *S, 0);
  if ((rc = P.init()) || (rc = check_count(ctx, P, n, "vcycle"))) return rc;
  DeviceBuffer dx, db;
  if ((rc = P.unpack(r, db))) return rc;
  MSBG_CUDA_TRY(ctx, dx.ensure(db.bytes));
  Runner<float> R{*S, ctx->stream, nPre, nPost, innerIter};
  R.coarseScale = coarseScale;
  R.err = ctx->errBuf.as<int>();
  R.numSMs = S->numSMs;
  R.vcycle<float>(0, dx.as<float>(), db.as<float>());
  MSBG_CUDA_TRY(ctx, cudaGetLastError());
  if ((rc = P.pack(dx, z))) return rc;
  return finish(ctx);
}

extern "C" int msbg_gpu_pressure_prepare_arrays(msbg_gpu_ctx* ctx, const msbg_topo_desc* topo,
                                                const uint16_t* flags, const float* faceX,
                                                const float* faceY, const float* faceZ,
                                                const float* rhs) {
  if (!ctx || !topo || !flags || !faceX || !faceY || !faceZ) return MSBG_EINVARG;
  if (!(topo->bsx0 == 8 || topo->bsx0 == 16 || topo->bsx0 == 32) || topo->sx <= 0 ||
      topo->sy <= 0 || topo->sz <= 0 || topo->sx % topo->bsx0 || topo->sy % topo->bsx0 ||
      topo->sz % topo->bsx0 || topo->nLevels < 1 || topo->nLevels > 4)
    return msbg_gpu_sync_topology(ctx, topo);  // reports the invalid field
  const int64_t nb =
      (int64_t)(topo->sx / topo->bsx0) * (topo->sy / topo->bsx0) * (topo->sz / topo->bsx0);
  for (int64_t b = 0; topo->blockLevel && b < nb; b++) {
    const int l = topo->blockLevel[b];
    if (l < 0 || l >= topo->nLevels)
      return set_error(ctx, MSBG_EINVARG, "blockLevel[%lld]=%d out of range", (long long)b, l);
  }
  ArrayInput A{flags, {faceX, faceY, faceZ}, rhs};
  return pressure_prepare(ctx, topo, nullptr, &A);
}
