// MGPCG pressure solve on the GPU: tile kernels, V-cycle, PCG driver, C ABI.
//
// Replaces MultiresSparseGrid::preparePressureSolveFLIP + solvePressureFLIP
// (src/msbg3.cpp:3041-3271).  Structure of one PCG iteration as in the
// reference (src/msbg3.cpp:3149-3236): q = A d, alpha = rho/(d.q),
// x += alpha d, r -= alpha q, z = V(r), beta = (r.z)/rho, d = z + beta d;
// stop when |r|^2 <= tol^2 |b|^2 or on breakdown.  Inner products and norms
// are FP64 (two-stage deterministic reductions with warp shuffles).  The
// V-cycle (src/msbg3.cpp:2412-2465) is pre-smooth, residual, restriction,
// recursion, prolongation, post-smooth; the smoother is a tile-wise
// red-black Gauss-Seidel with the tiles themselves visited in red-black
// order per resolution level (the reference visits blocks red-black too,
// src/msbg3.cpp:2185-2219); the post-smoother is the exact adjoint of the
// pre-smoother so the preconditioner is symmetric.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <string>
#include <type_traits>
#include <vector>

#include "common.cuh"
#include "pressure.h"
#include "pressure_kernels.cuh"

namespace msbg {
namespace ps {

// ---------------------------------------------------------------------------
// reductions
// ---------------------------------------------------------------------------
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

// Sum over the CTA; result valid in thread 0.
__device__ double block_sum(double v) {
  __shared__ double ws[32];
  v = warp_sum(v);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) ws[w] = v;
  __syncthreads();
  const int nw = (blockDim.x + 31) >> 5;
  v = (threadIdx.x < nw) ? ws[threadIdx.x] : 0.0;
  if (w == 0) v = warp_sum(v);
  __syncthreads();
  return v;
}

struct Scalars {
  double bb, rho, rhoNew, dq, rr, alpha, beta;
  int status;  // 0 ok, 2 breakdown, 3 non-finite
  int pad;
};

enum { FIN_BB = 0, FIN_DQ_ALPHA = 1, FIN_RR = 2, FIN_RHO = 3, FIN_RHONEW_BETA = 4 };

// Deterministic second stage: fixed-order sum of the CTA partials, then the
// scalar step of PCG that depends on it.
__global__ void __launch_bounds__(1024) k_finalize(const double* __restrict__ partial, int n,
                                                   Scalars* s, int what) {
  double v = 0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) v += partial[i];
  v = block_sum(v);
  if (threadIdx.x != 0) return;
  switch (what) {
    case FIN_BB: s->bb = v; break;
    case FIN_RHO: s->rho = v; break;
    case FIN_RR: s->rr = v; if (!isfinite(v)) s->status = 3; break;
    case FIN_DQ_ALPHA:
      s->dq = v;
      if (!isfinite(v) || !isfinite(s->rho)) s->status = 3;
      else if (!(v > 1e-300) || !(s->rho > 1e-300)) s->status = 2;
      else s->alpha = s->rho / v;
      break;
    case FIN_RHONEW_BETA:
      s->rhoNew = v;
      if (!isfinite(v)) s->status = 3;
      else if (!(v > 1e-300)) s->status = 2;
      else {
        s->beta = v / s->rho;
        s->rho = v;
      }
      break;
  }
}

// ---------------------------------------------------------------------------
// level-0 vector kernels (grid-stride, fixed grid for deterministic partials)
// ---------------------------------------------------------------------------
constexpr int VEC_GRID = 148 * 4, VEC_BLOCK = 512;

__global__ void __launch_bounds__(VEC_BLOCK) k_dot(const float* __restrict__ a,
                                                   const float* __restrict__ b, int64_t n,
                                                   double* __restrict__ partial) {
  double acc = 0;
  const int64_t n4 = n >> 2;
  const float4* a4 = reinterpret_cast<const float4*>(a);
  const float4* b4 = reinterpret_cast<const float4*>(b);
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n4;
       i += (int64_t)gridDim.x * blockDim.x) {
    float4 u = a4[i], v = b4[i];
    acc += (double)u.x * v.x + (double)u.y * v.y + (double)u.z * v.z + (double)u.w * v.w;
  }
  acc = block_sum(acc);
  if (threadIdx.x == 0) partial[blockIdx.x] = acc;
}

// x += alpha d; r -= alpha q; partial |r|^2.  Skipped (norm only) after a breakdown.
__global__ void __launch_bounds__(VEC_BLOCK) k_axpy_norm(float* __restrict__ x,
                                                         float* __restrict__ r,
                                                         const float* __restrict__ d,
                                                         const float* __restrict__ q, int64_t n,
                                                         const Scalars* __restrict__ s,
                                                         double* __restrict__ partial) {
  const bool ok = s->status == 0;
  const float alpha = (float)s->alpha;
  double acc = 0;
  const int64_t n4 = n >> 2;
  float4* x4 = reinterpret_cast<float4*>(x);
  float4* r4 = reinterpret_cast<float4*>(r);
  const float4* d4 = reinterpret_cast<const float4*>(d);
  const float4* q4 = reinterpret_cast<const float4*>(q);
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n4;
       i += (int64_t)gridDim.x * blockDim.x) {
    float4 rv = r4[i];
    if (ok) {
      float4 xv = x4[i], dv = d4[i], qv = q4[i];
      xv.x = fmaf(alpha, dv.x, xv.x); xv.y = fmaf(alpha, dv.y, xv.y);
      xv.z = fmaf(alpha, dv.z, xv.z); xv.w = fmaf(alpha, dv.w, xv.w);
      rv.x = fmaf(-alpha, qv.x, rv.x); rv.y = fmaf(-alpha, qv.y, rv.y);
      rv.z = fmaf(-alpha, qv.z, rv.z); rv.w = fmaf(-alpha, qv.w, rv.w);
      x4[i] = xv;
      r4[i] = rv;
    }
    acc += (double)rv.x * rv.x + (double)rv.y * rv.y + (double)rv.z * rv.z + (double)rv.w * rv.w;
  }
  acc = block_sum(acc);
  if (threadIdx.x == 0) partial[blockIdx.x] = acc;
}

// d = z + beta d
__global__ void __launch_bounds__(VEC_BLOCK) k_update_d(float* __restrict__ d,
                                                        const float* __restrict__ z, int64_t n,
                                                        const Scalars* __restrict__ s) {
  if (s->status) return;
  const float beta = (float)s->beta;
  const int64_t n4 = n >> 2;
  float4* d4 = reinterpret_cast<float4*>(d);
  const float4* z4 = reinterpret_cast<const float4*>(z);
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n4;
       i += (int64_t)gridDim.x * blockDim.x) {
    float4 dv = d4[i], zv = z4[i];
    dv.x = fmaf(beta, dv.x, zv.x); dv.y = fmaf(beta, dv.y, zv.y);
    dv.z = fmaf(beta, dv.z, zv.z); dv.w = fmaf(beta, dv.w, zv.w);
    d4[i] = dv;
  }
}

// ---------------------------------------------------------------------------
// tile kernels
// ---------------------------------------------------------------------------

// In-tile neighbour sum S of cell (i,j,k) from a shared-memory tile, ghosts
// from gs.  cxv etc. point at the tile's couplings (shared or global).
template <int TS>
__device__ __forceinline__ float nbr_sum(const float* xs, const float* cxv, const float* cyv,
                                         const float* czv, const float (*gs)[TS * TS], int i,
                                         int j, int k) {
  const int e = tidx(TS, i, j, k);
  float S = 0.f;
  S += (i > 0) ? cxv[e] * xs[e - 1] : gs[0][j + TS * k];
  S += (i < TS - 1) ? cxv[e + 1] * xs[e + 1] : gs[1][j + TS * k];
  S += (j > 0) ? cyv[e] * xs[e - TS] : gs[2][i + TS * k];
  S += (j < TS - 1) ? cyv[e + TS] * xs[e + TS] : gs[3][i + TS * k];
  S += (k > 0) ? czv[e] * xs[e - TS * TS] : gs[4][i + TS * j];
  S += (k < TS - 1) ? czv[e + TS * TS] * xs[e + TS * TS] : gs[5][i + TS * j];
  return S;
}

// q = A d on the listed tiles, partial d.q per CTA.
template <int TS>
__global__ void __launch_bounds__(TS* TS) k_matvec_dot(LevelView L, const int* __restrict__ tiles,
                                                       const float* __restrict__ d,
                                                       float* __restrict__ q,
                                                       double* __restrict__ partial) {
  constexpr int N = TS * TS * TS, NT = TS * TS;
  __shared__ float xs[N];
  __shared__ float gs[6][NT];
  const int ti = tiles[blockIdx.x];
  const int64_t off = L.tileOff[ti];
  const int t = threadIdx.x, i = t % TS, j = t / TS;
  for (int e = t; e < N; e += NT) xs[e] = d[off + e];
#pragma unroll
  for (int f = 0; f < 6; f++) gs[f][t] = ghost_sum(L, d, ti, TS, f >> 1, f & 1, i, j);
  __syncthreads();
  double acc = 0;
  const float* cxv = L.cx + off;
  const float* cyv = L.cy + off;
  const float* czv = L.cz + off;
#pragma unroll 4
  for (int k = 0; k < TS; k++) {
    const int e = tidx(TS, i, j, k);
    const float dg = L.diag[off + e];
    float y = 0.f;
    if (dg > 0.f) y = dg * xs[e] - nbr_sum<TS>(xs, cxv, cyv, czv, gs, i, j, k);
    q[off + e] = y;
    acc += (double)xs[e] * (double)y;
  }
  acc = block_sum(acc);
  if (t == 0 && partial) partial[blockIdx.x] = acc;
}

// r = b - A x on the listed tiles, restricted (sum over the liquid children,
// P^T) into the coarse right-hand side bc.
template <int TS>
__global__ void __launch_bounds__(TS* TS) k_residual_restrict(LevelView L,
                                                              const int* __restrict__ tiles,
                                                              const float* __restrict__ x,
                                                              const float* __restrict__ b,
                                                              float* __restrict__ bc,
                                                              const int64_t* __restrict__ coarseOff) {
  constexpr int N = TS * TS * TS, NT = TS * TS;
  __shared__ float xs[N];
  __shared__ float rs[N];
  __shared__ float gs[6][NT];
  const int ti = tiles[blockIdx.x];
  const int64_t off = L.tileOff[ti];
  const int t = threadIdx.x, i = t % TS, j = t / TS;
  for (int e = t; e < N; e += NT) xs[e] = x[off + e];
#pragma unroll
  for (int f = 0; f < 6; f++) gs[f][t] = ghost_sum(L, x, ti, TS, f >> 1, f & 1, i, j);
  __syncthreads();
  const float* cxv = L.cx + off;
  const float* cyv = L.cy + off;
  const float* czv = L.cz + off;
#pragma unroll 4
  for (int k = 0; k < TS; k++) {
    const int e = tidx(TS, i, j, k);
    const float dg = L.diag[off + e];
    float r = 0.f;
    if (dg > 0.f) r = b[off + e] - (dg * xs[e] - nbr_sum<TS>(xs, cxv, cyv, czv, gs, i, j, k));
    rs[e] = r;
  }
  __syncthreads();
  const int* tc = L.toCoarse + (size_t)ti * 6;
  const int ct = tc[0], ox = tc[1], oy = tc[2], oz = tc[3], agg = tc[4], cts = tc[5];
  if (ct < 0) return;
  float* dst = bc + coarseOff[ct];
  if (agg) {
    constexpr int H = TS / 2;
    for (int c = t; c < H * H * H; c += NT) {
      const int ci = c % H, cj = (c / H) % H, ck = c / (H * H);
      const int e = tidx(TS, 2 * ci, 2 * cj, 2 * ck);
      const float s = rs[e] + rs[e + 1] + rs[e + TS] + rs[e + TS + 1] + rs[e + TS * TS] +
                      rs[e + TS * TS + 1] + rs[e + TS * TS + TS] + rs[e + TS * TS + TS + 1];
      dst[tidx(cts, ox + ci, oy + cj, oz + ck)] = s;
    }
  } else {
    for (int e = t; e < N; e += NT) {
      const int ii = e % TS, jj = (e / TS) % TS, kk = e / (TS * TS);
      dst[tidx(cts, ox + ii, oy + jj, oz + kk)] = rs[e];
    }
  }
}

// x += P xc (liquid cells only).
template <int TS>
__global__ void __launch_bounds__(TS* TS) k_prolong(LevelView L, const int* __restrict__ tiles,
                                                    float* __restrict__ x,
                                                    const float* __restrict__ xc,
                                                    const int64_t* __restrict__ coarseOff,
                                                    float scale) {
  constexpr int N = TS * TS * TS, NT = TS * TS;
  const int ti = tiles[blockIdx.x];
  const int64_t off = L.tileOff[ti];
  const int* tc = L.toCoarse + (size_t)ti * 6;
  const int ct = tc[0], ox = tc[1], oy = tc[2], oz = tc[3], agg = tc[4], cts = tc[5];
  if (ct < 0) return;
  const float* src = xc + coarseOff[ct];
  for (int e = threadIdx.x; e < N; e += NT) {
    if (!(L.diag[off + e] > 0.f)) continue;
    const int i = e % TS, j = (e / TS) % TS, k = e / (TS * TS);
    const int sh = agg ? 1 : 0;
    x[off + e] += scale * src[tidx(cts, ox + (i >> sh), oy + (j >> sh), oz + (k >> sh))];
  }
}

// Red-black Gauss-Seidel inside each listed tile, `inner` iterations, ghosts
// frozen at their values when the tile is loaded.  reverse=0: red then black;
// reverse=1: black then red (the adjoint order).  Optional partial b.x.
template <int TS>
__global__ void __launch_bounds__(TS* TS) k_smooth(LevelView L, const int* __restrict__ tiles,
                                                   float* __restrict__ x,
                                                   const float* __restrict__ b, int inner,
                                                   int reverse, double* __restrict__ partial) {
  constexpr int N = TS * TS * TS, NT = TS * TS;
  extern __shared__ __align__(128) float sm[];
  float* xs = sm;
  float* cxs = sm + N;
  float* cys = sm + 2 * N;
  float* czs = sm + 3 * N;
  float(*gs)[NT] = reinterpret_cast<float(*)[NT]>(sm + 4 * N);
  const int ti = tiles[blockIdx.x];
  const int64_t off = L.tileOff[ti];
  const int t = threadIdx.x, i = t % TS, j = t / TS;
  for (int e = t; e < N; e += NT) {
    xs[e] = x[off + e];
    cxs[e] = L.cx[off + e];
    cys[e] = L.cy[off + e];
    czs[e] = L.cz[off + e];
  }
  float bb[TS], inv[TS];
#pragma unroll
  for (int k = 0; k < TS; k++) {
    const int e = tidx(TS, i, j, k);
    const float dg = L.diag[off + e];
    inv[k] = dg > 0.f ? 1.0f / dg : 0.f;
    bb[k] = b[off + e];
  }
#pragma unroll
  for (int f = 0; f < 6; f++) gs[f][t] = ghost_sum(L, x, ti, TS, f >> 1, f & 1, i, j);
  __syncthreads();
  for (int it = 0; it < inner; it++) {
#pragma unroll
    for (int h = 0; h < 2; h++) {
      const int colour = reverse ? 1 - h : h;
#pragma unroll
      for (int k = 0; k < TS; k++) {
        if (((i + j + k) & 1) != colour || inv[k] == 0.f) continue;
        const float S = nbr_sum<TS>(xs, cxs, cys, czs, gs, i, j, k);
        xs[tidx(TS, i, j, k)] = (bb[k] + S) * inv[k];
      }
      __syncthreads();
    }
  }
  double acc = 0;
  for (int e = t; e < N; e += NT) {
    x[off + e] = xs[e];
    if (partial) acc += (double)xs[e] * (double)b[off + e];
  }
  if (partial) {
    acc = block_sum(acc);
    if (t == 0) partial[blockIdx.x] = acc;
  }
}

#include "smooth_pipe.cuh"
#include "refine.cuh"

// Coarsest level: x = A^-1 b with the dense FP64 inverse (symmetric).
__global__ void __launch_bounds__(512) k_coarse_solve(const double* __restrict__ Ainv, int n,
                                                      const int64_t* __restrict__ cells,
                                                      const float* __restrict__ b,
                                                      float* __restrict__ x) {
  __shared__ double bs[512];
  const int t = threadIdx.x;
  if (t < n) bs[t] = b[cells[t]];
  __syncthreads();
  if (t >= n) return;
  double s = 0;
  for (int j = 0; j < n; j++) s += Ainv[(size_t)j * n + t] * bs[j];
  x[cells[t]] = (float)s;
}

template <int TS>
size_t smooth_smem() {
  return sizeof(float) * (4 * TS * TS * TS + 6 * TS * TS);
}

// ---------------------------------------------------------------------------
// solver state
// ---------------------------------------------------------------------------
struct Solver {
  Hierarchy H;
  int64_t h2dBytes = 0;
  int numSMs = 148;
  double prepareSeconds = 0, buildSeconds = 0;
  std::vector<std::unique_ptr<LevelDev>> dev;
  std::vector<LevelView> views;
  DeviceBuffer dCoarseInv, dCoarseCells;
  DeviceBuffer rhs0, d0, q0, z0, r0, partial, scal;
  DeviceBuffer x64, rin;  // FP64 solution and inner right-hand side of the refinement
  int maxPartial = 0;
  Scalars* hScal = nullptr;  // pinned
  int bsx0 = 0, nbx = 0, nby = 0, nbz = 0;
  std::vector<int> blockLevel;
};

template <int TS>
void set_smooth_attr() {
  static bool done = false;
  if (!done) {
    cudaFuncSetAttribute(k_smooth<TS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)smooth_smem<TS>());
    done = true;
  }
}

#define TS_DISPATCH(ts, CALL)        \
  switch (ts) {                      \
    case 16: { constexpr int T = 16; CALL; } break; \
    case 8: { constexpr int T = 8; CALL; } break;   \
    case 4: { constexpr int T = 4; CALL; } break;   \
    case 2: { constexpr int T = 2; CALL; } break;   \
    case 1: break;                   \
    default: break;                  \
  }

struct Runner {
  Solver& S;
  cudaStream_t st;
  int nPre, nPost, inner;
  float coarseScale = 1.0f;
  int* err = nullptr;     // device flag set by kernels whose bounded wait gave up
  int numSMs = 148;
  bool usePipe = true;
  int64_t launches = 0;  // kernels launched through this runner

  const int* passList(int m) { return S.dev[m]->passTiles.as<int>(); }
  const int* groupList(int m) { return S.dev[m]->groupTiles.as<int>(); }

  // One smoothing sweep of MG level m: the (level, colour) passes in order
  // (pre) or in reverse order with the adjoint colour order inside (post).
  void smooth(int m, float* x, const float* b, bool post) {
    const Level& L = S.H.levels[m];
    const int np = (int)L.passes.size();
    for (int pi = 0; pi < np; pi++) {
      const Level::Pass& P = L.passes[post ? np - 1 - pi : pi];
      if (!P.count) continue;
      const int* lst = passList(m) + P.start;
      if (P.ts == 16 && usePipe) {
        const int grid = std::min(P.count, numSMs);
        // passes are contiguous tile-id ranges (register_tiles sorts by pass)
        k_smooth_pipe16<<<grid, pipe::NT, pipe::SMEM, st>>>(S.views[m], P.start, P.count, x,
                                                            b, inner, post ? 1 : 0, err);
      } else {
        TS_DISPATCH(P.ts, (k_smooth<T><<<P.count, T * T, smooth_smem<T>(), st>>>(
                               S.views[m], lst, x, b, inner, post ? 1 : 0, nullptr)));
      }
      launches++;
    }
  }

  void vcycle(int m, float* x, const float* b) {
    const int last = (int)S.H.levels.size() - 1;
    const Level& L = S.H.levels[m];
    cudaMemsetAsync(x, 0, sizeof(float) * L.nCells, st);
    if (m == last) {
      k_coarse_solve<<<1, 512, 0, st>>>(S.dCoarseInv.as<double>(), S.H.nCoarse,
                                        S.dCoarseCells.as<int64_t>(), b, x);
      launches++;
      return;
    }
    for (int s = 0; s < nPre; s++) smooth(m, x, b, false);
    LevelDev& C = *S.dev[m + 1];
    residual_restrict(m, x, b);
    vcycle(m + 1, C.x.as<float>(), C.b.as<float>());
    for (const auto& g : L.groups) {
      const int* lst = groupList(m) + g.start;
      TS_DISPATCH(g.ts, (k_prolong<T><<<g.count, T * T, 0, st>>>(S.views[m], lst, x,
                                                                  C.x.as<float>(),
                                                                  C.tileOff.as<int64_t>(),
                                                                  coarseScale)));
      launches++;
    }
    for (int s = 0; s < nPost; s++) smooth(m, x, b, true);
  }

  // q = A d with partial d.q (level 0); returns the number of partials.
  // Passes are contiguous tile ranges of one tile size; 16^3 passes go
  // through the pipelined kernel, the others through the per-tile kernel.
  int matvec_dot(const float* d, float* q, double* partial) {
    const Level& L = S.H.levels[0];
    int off = 0;
    for (const auto& P : L.passes) {
      if (!P.count) continue;
      if (P.ts == 16 && usePipe) {
        const int grid = std::min(P.count, numSMs);
        k_apply_pipe16<APPLY_MATVEC><<<grid, pipe::NT, pipe::SMEM, st>>>(
            S.views[0], P.start, P.count, d, nullptr, q, nullptr, nullptr, partial + off, err);
        off += grid;
      } else {
        const int* lst = passList(0) + P.start;
        TS_DISPATCH(P.ts, (k_matvec_dot<T><<<P.count, T * T, 0, st>>>(S.views[0], lst, d, q,
                                                                       partial + off)));
        off += P.count;
      }
      launches++;
    }
    return off;
  }

  // r = b - A x on MG level m, restricted into the right-hand side of m+1.
  void residual_restrict(int m, const float* x, const float* b) {
    const Level& L = S.H.levels[m];
    LevelDev& C = *S.dev[m + 1];
    for (const auto& P : L.passes) {
      if (!P.count) continue;
      if (P.ts == 16 && usePipe) {
        const int grid = std::min(P.count, numSMs);
        k_apply_pipe16<APPLY_RESIDUAL><<<grid, pipe::NT, pipe::SMEM, st>>>(
            S.views[m], P.start, P.count, x, b, nullptr, C.b.as<float>(),
            C.tileOff.as<int64_t>(), nullptr, err);
      } else {
        const int* lst = passList(m) + P.start;
        TS_DISPATCH(P.ts, (k_residual_restrict<T><<<P.count, T * T, 0, st>>>(
                              S.views[m], lst, x, b, C.b.as<float>(), C.tileOff.as<int64_t>())));
      }
      launches++;
    }
  }
};

}  // namespace ps
}  // namespace msbg

using namespace msbg;
using namespace msbg::ps;

namespace {

std::map<msbg_gpu_ctx*, std::unique_ptr<Solver>>& solvers() {
  static std::map<msbg_gpu_ctx*, std::unique_ptr<Solver>> m;
  return m;
}

std::unique_ptr<Solver>& solver_of(msbg_gpu_ctx* ctx) { return solvers()[ctx]; }

template <typename T>
cudaError_t upload(DeviceBuffer& buf, const std::vector<T>& v, cudaStream_t st) {
  cudaError_t e = buf.ensure(sizeof(T) * std::max<size_t>(v.size(), 1));
  if (e != cudaSuccess) return e;
  if (v.empty()) return cudaSuccess;
  return cudaMemcpyAsync(buf.p, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice, st);
}

}  // namespace

namespace msbg {
void pressure_release(msbg_gpu_ctx* ctx) {
  auto it = solvers().find(ctx);
  if (it == solvers().end()) return;
  if (it->second && it->second->hScal) cudaFreeHost(it->second->hScal);
  solvers().erase(it);
}
}  // namespace msbg

extern "C" void msbg_gpu_solve_params_default(msbg_gpu_solve_params* p) {
  if (!p) return;
  p->nPre = 2;
  p->nPost = 2;
  p->nCoarse = 24;
  p->maxIter = 500;
  p->tol = 1e-6f;
  p->innerIter = 2;
  p->storage = MSBG_F32;
  p->maxRefine = 0;  // plain MGPCG on the recursive residual, as the reference
  p->useGraph = 1;
  // Piecewise-constant transfers with Galerkin coarse operators under-correct
  // smooth errors; scaling the coarse correction by 1.8 restores
  // size-independent convergence (10-13 PCG iterations from 256^3 to 1024^3).
  p->coarseScale = 1.8f;
}

extern "C" int msbg_gpu_pressure_prepare(msbg_gpu_ctx* ctx, const msbg_topo_desc* topo,
                                         const msbg_pressure_callbacks* cb) {
  if (!ctx || !topo || !cb || !cb->sampleCellType || !cb->sampleFaceCoeff || !cb->sampleRhs)
    return MSBG_EINVARG;
  int rc = msbg_gpu_sync_topology(ctx, topo);
  if (rc) return rc;
  cudaSetDevice(ctx->device);
  auto& sp = solver_of(ctx);
  sp.reset(new Solver());
  Solver& S = *sp;
  std::string err;
  auto tp0 = std::chrono::steady_clock::now();
  rc = build_hierarchy(S.H, topo->sx, topo->sy, topo->sz, topo->bsx0, topo->nLevels,
                       topo->blockLevel, cb, 512, &err);
  S.buildSeconds =
      std::chrono::duration<double>(std::chrono::steady_clock::now() - tp0).count();
  if (rc) {
    sp.reset();
    return set_error(ctx, rc, "pressure prepare: %s", err.c_str());
  }
  for (size_t m = 0; m + 1 < S.H.levels.size(); m++)
    for (const Tile& t : S.H.levels[m].tiles)
      if (t.ts < 2 || t.ts > TS_MAX) {
        sp.reset();
        return set_error(ctx, MSBG_EINVARG, "grid dimensions give %d-cell tiles at MG level %d",
                         t.ts, (int)m);
      }
  set_smooth_attr<16>();
  cudaFuncSetAttribute(k_apply_pipe16<APPLY_MATVEC>,
                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)pipe::SMEM);
  cudaFuncSetAttribute(k_apply_pipe16<APPLY_RESIDUAL>,
                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)pipe::SMEM);
  cudaFuncSetAttribute(k_smooth_pipe16, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)pipe::SMEM);
  cudaDeviceGetAttribute(&S.numSMs, cudaDevAttrMultiProcessorCount, ctx->device);
  set_smooth_attr<8>();
  set_smooth_attr<4>();
  set_smooth_attr<2>();
  S.bsx0 = topo->bsx0;
  S.nbx = ctx->nbx;
  S.nby = ctx->nby;
  S.nbz = ctx->nbz;
  S.blockLevel = ctx->blockLevel;
  cudaStream_t st = ctx->stream;
  int maxPartial = VEC_GRID;
  for (size_t m = 0; m < S.H.levels.size(); m++) {
    const Level& L = S.H.levels[m];
    auto D = std::make_unique<LevelDev>();
    std::vector<int64_t> toff(L.tiles.size());
    for (size_t i = 0; i < L.tiles.size(); i++) toff[i] = L.tiles[i].off;
    MSBG_CUDA_TRY(ctx, upload(D->tileOff, toff, st));
    MSBG_CUDA_TRY(ctx, upload(D->face, L.face, st));
    MSBG_CUDA_TRY(ctx, upload(D->ifOff, L.ifOff, st));
    MSBG_CUDA_TRY(ctx, upload(D->toCoarse, L.toCoarse, st));
    MSBG_CUDA_TRY(ctx, upload(D->passTiles, L.passTiles, st));
    MSBG_CUDA_TRY(ctx, upload(D->groupTiles, L.groupTiles, st));
    MSBG_CUDA_TRY(ctx, upload(D->diag, L.diag, st));
    {
      std::vector<float> inv(L.diag.size());
      for (size_t c = 0; c < inv.size(); c++)
        inv[c] = L.diag[c] > 0.f ? (float)(1.0 / (double)L.diag[c]) : 0.f;
      MSBG_CUDA_TRY(ctx, upload(D->invdiag, inv, st));
      MSBG_CUDA_TRY(ctx, upload(D->tileRec, build_tile_records(L), st));
      // the hot-path kernels address passes as contiguous tile-id ranges
      for (size_t i = 0; i < L.passTiles.size(); i++)
        if (L.passTiles[i] != (int)i)
          return set_error(ctx, MSBG_EINTERNAL, "pass tiles are not contiguous");
      MSBG_CUDA_TRY(ctx, cudaStreamSynchronize(st));  // host vectors above are temporaries
    }
    MSBG_CUDA_TRY(ctx, upload(D->cx, L.cx, st));
    MSBG_CUDA_TRY(ctx, upload(D->cy, L.cy, st));
    MSBG_CUDA_TRY(ctx, upload(D->cz, L.cz, st));
    MSBG_CUDA_TRY(ctx, upload(D->ifc, L.ifc, st));
    const size_t nb = sizeof(float) * std::max<int64_t>(L.nCells, 4);
    MSBG_CUDA_TRY(ctx, D->x.ensure(nb));
    MSBG_CUDA_TRY(ctx, D->b.ensure(nb));
    maxPartial = std::max(maxPartial, (int)L.tiles.size());
    LevelView v;
    v.tileOff = D->tileOff.as<int64_t>();
    v.face = D->face.as<int>();
    v.ifOff = D->ifOff.as<int64_t>();
    v.toCoarse = D->toCoarse.as<int>();
    v.diag = D->diag.as<float>();
    v.invdiag = D->invdiag.as<float>();
    v.tileRec = D->tileRec.p;
    v.cx = D->cx.as<float>();
    v.cy = D->cy.as<float>();
    v.cz = D->cz.as<float>();
    v.ifc = D->ifc.as<float>();
    S.views.push_back(v);
    S.dev.push_back(std::move(D));
  }
  const Level& L0 = S.H.levels[0];
  const size_t n0 = sizeof(float) * L0.nCells;
  MSBG_CUDA_TRY(ctx, upload(S.rhs0, L0.rhs, st));
  MSBG_CUDA_TRY(ctx, S.d0.ensure(n0));
  MSBG_CUDA_TRY(ctx, S.q0.ensure(n0));
  MSBG_CUDA_TRY(ctx, S.z0.ensure(n0));
  MSBG_CUDA_TRY(ctx, S.r0.ensure(n0));
  MSBG_CUDA_TRY(ctx, S.partial.ensure(sizeof(double) * maxPartial));
  S.maxPartial = maxPartial;
  MSBG_CUDA_TRY(ctx, S.scal.ensure(sizeof(Scalars)));
  MSBG_CUDA_TRY(ctx, upload(S.dCoarseInv, S.H.coarseInv, st));
  MSBG_CUDA_TRY(ctx, upload(S.dCoarseCells, S.H.coarseCells, st));
  MSBG_CUDA_TRY(ctx, cudaMallocHost(&S.hScal, sizeof(Scalars)));
  MSBG_CUDA_TRY(ctx, cudaStreamSynchronize(st));
  for (const auto& D : S.dev)
    S.h2dBytes += (int64_t)(D->tileOff.bytes + D->face.bytes + D->ifOff.bytes +
                            D->toCoarse.bytes + D->passTiles.bytes + D->groupTiles.bytes +
                            D->diag.bytes + D->cx.bytes + D->cy.bytes + D->cz.bytes +
                            D->ifc.bytes);
  S.h2dBytes += (int64_t)(S.rhs0.bytes + S.dCoarseInv.bytes + S.dCoarseCells.bytes);
  S.prepareSeconds =
      std::chrono::duration<double>(std::chrono::steady_clock::now() - tp0).count();
  return MSBG_OK;
}

namespace {

struct PcgResult {
  int iters = 0;
  int status = 1;  // 0 converged, 1 maxIter, 2 breakdown, 3 non-finite
  double bb = 0;
};

// MGPCG on MG level 0 for A e = bin from e = 0 (e in the level-0 x vector),
// stopping at |r| <= tolRel |bin| (recursive residual, as the reference).
// One iteration is one CUDA graph launch; the graph is captured on the first
// call and reused (all buffers are fixed).
int run_pcg(msbg_gpu_ctx* ctx, Solver& S, Runner& R, const float* bin, double tolRel, int maxIter,
            bool useGraph, cudaGraphExec_t& exec, int64_t& perIter, PcgResult& out) {
  cudaStream_t st = R.st;
  const int64_t n = S.H.levels[0].nCells;
  float* x = S.dev[0]->x.as<float>();
  float* r = S.r0.as<float>();
  float* d = S.d0.as<float>();
  float* q = S.q0.as<float>();
  float* z = S.z0.as<float>();
  double* part = S.partial.as<double>();
  Scalars* sc = S.scal.as<Scalars>();
  // r = b, x = 0, bb = b.b, z = V(r), rho = r.z, d = z
  cudaMemsetAsync(sc, 0, sizeof(Scalars), st);
  cudaMemsetAsync(x, 0, sizeof(float) * n, st);
  cudaMemcpyAsync(r, bin, sizeof(float) * n, cudaMemcpyDeviceToDevice, st);
  k_dot<<<VEC_GRID, VEC_BLOCK, 0, st>>>(bin, bin, n, part);
  k_finalize<<<1, 1024, 0, st>>>(part, VEC_GRID, sc, FIN_BB);
  R.vcycle(0, z, r);
  k_dot<<<VEC_GRID, VEC_BLOCK, 0, st>>>(r, z, n, part);
  k_finalize<<<1, 1024, 0, st>>>(part, VEC_GRID, sc, FIN_RHO);
  cudaMemcpyAsync(d, z, sizeof(float) * n, cudaMemcpyDeviceToDevice, st);
  cudaMemcpyAsync(S.hScal, sc, sizeof(Scalars), cudaMemcpyDeviceToHost, st);
  R.launches += 4;
  MSBG_CUDA_TRY(ctx, cudaStreamSynchronize(st));
  out = PcgResult();
  out.bb = S.hScal->bb;
  if (!(out.bb > 1e-300)) {
    out.status = 0;
    return MSBG_OK;
  }
  auto iteration = [&]() {
    R.launches += 6;  // finalize x3, axpy_norm, dot, update_d
    int nt = R.matvec_dot(d, q, part);
    k_finalize<<<1, 1024, 0, st>>>(part, nt, sc, FIN_DQ_ALPHA);
    k_axpy_norm<<<VEC_GRID, VEC_BLOCK, 0, st>>>(x, r, d, q, n, sc, part);
    k_finalize<<<1, 1024, 0, st>>>(part, VEC_GRID, sc, FIN_RR);
    R.vcycle(0, z, r);
    k_dot<<<VEC_GRID, VEC_BLOCK, 0, st>>>(r, z, n, part);
    k_finalize<<<1, 1024, 0, st>>>(part, VEC_GRID, sc, FIN_RHONEW_BETA);
    k_update_d<<<VEC_GRID, VEC_BLOCK, 0, st>>>(d, z, n, sc);
    cudaMemcpyAsync(S.hScal, sc, sizeof(Scalars), cudaMemcpyDeviceToHost, st);
  };
  if (useGraph && !exec) {
    const int64_t before = R.launches;
    cudaGraph_t g;
    MSBG_CUDA_TRY(ctx, cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    iteration();
    MSBG_CUDA_TRY(ctx, cudaStreamEndCapture(st, &g));
    perIter = R.launches - before;
    R.launches = before;
    MSBG_CUDA_TRY(ctx, cudaGraphInstantiate(&exec, g, 0));
    cudaGraphDestroy(g);
  }
  const double tol2 = tolRel * tolRel;
  for (int it = 0; it < maxIter; it++) {
    if (exec) {
      MSBG_CUDA_TRY(ctx, cudaGraphLaunch(exec, st));
      R.launches += perIter;
    } else {
      iteration();
    }
    MSBG_CUDA_TRY(ctx, cudaStreamSynchronize(st));
    out.iters = it + 1;
    const Scalars hs = *S.hScal;
    if (hs.status) {
      // a breakdown found before the update leaves x, r unchanged
      out.status = hs.status;
      break;
    }
    if (hs.rr <= tol2 * out.bb) {
      out.status = 0;
      break;
    }
  }
  return MSBG_OK;
}

// r32 = b - A x64 (FP64) on level 0; returns |r|^2 in *rr.
int residual64(msbg_gpu_ctx* ctx, Solver& S, Runner& R, const float* b, float* r32,
               double* rr) {
  cudaStream_t st = R.st;
  const Level& L = S.H.levels[0];
  double* part = S.partial.as<double>();
  int off = 0;
  for (const auto& g : L.groups) {
    const int* lst = S.dev[0]->groupTiles.as<int>() + g.start;
    TS_DISPATCH(g.ts, (k_residual64<T><<<g.count, T * T, 0, st>>>(
                          S.views[0], lst, S.x64.as<double>(), b, r32, part + off)));
    off += g.count;
    R.launches++;
  }
  Scalars* sc = S.scal.as<Scalars>();
  k_finalize<<<1, 1024, 0, st>>>(part, off, sc, FIN_RR);
  cudaMemcpyAsync(S.hScal, sc, sizeof(Scalars), cudaMemcpyDeviceToHost, st);
  R.launches++;
  MSBG_CUDA_TRY(ctx, cudaStreamSynchronize(st));
  *rr = S.hScal->rr;
  return MSBG_OK;
}

}  // namespace

extern "C" int msbg_gpu_pressure_solve(msbg_gpu_ctx* ctx, const msbg_gpu_solve_params* p,
                                       msbg_gpu_solve_info* info) {
  if (!ctx || !p) return MSBG_EINVARG;
  auto& sp = solver_of(ctx);
  if (!sp) return set_error(ctx, MSBG_EINVARG, "msbg_gpu_pressure_prepare not called");
  if (p->nPre < 0 || p->nPost < 0 || p->maxIter < 0 || p->innerIter < 1 || !(p->tol >= 0) ||
      p->maxRefine < 0)
    return set_error(ctx, MSBG_EINVARG, "invalid solve parameters");
  if (p->storage != MSBG_F32)
    return set_error(ctx, MSBG_ENOTIMPL, "storage type %d not available", p->storage);
  cudaSetDevice(ctx->device);
  Solver& S = *sp;
  cudaStream_t st = ctx->stream;
  Runner R{S, st, p->nPre, p->nPost, p->innerIter};
  R.coarseScale = p->coarseScale > 0 ? p->coarseScale : 1.0f;
  R.err = ctx->errBuf.as<int>();
  R.numSMs = S.numSMs;
  const Level& L0 = S.H.levels[0];
  const int64_t n = L0.nCells;
  float* x = S.dev[0]->x.as<float>();
  const float* b = S.rhs0.as<float>();
  if (p->maxRefine > 0) {
    MSBG_CUDA_TRY(ctx, S.x64.ensure(sizeof(double) * n));
    MSBG_CUDA_TRY(ctx, S.rin.ensure(sizeof(float) * n));
  }
  cudaGraphExec_t exec = nullptr;
  int64_t perIter = 0;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, st);
  int iters = 0, status = 1, refinements = 0;
  double relres = 0;
  int rc = MSBG_OK;
  if (p->maxRefine == 0) {
    PcgResult pr;
    rc = run_pcg(ctx, S, R, b, p->tol, p->maxIter, p->useGraph, exec, perIter, pr);
    iters = pr.iters;
    status = pr.status;
    cudaEventRecord(e1, st);
    if (rc == MSBG_OK) {
      // true residual of the FP32 iterate, FP32 operator, FP64 norm
      float* q = S.q0.as<float>();
      float* z = S.z0.as<float>();
      float* d = S.d0.as<float>();
      double* part = S.partial.as<double>();
      Scalars* sc = S.scal.as<Scalars>();
      R.matvec_dot(x, q, part);
      cudaMemcpyAsync(z, b, sizeof(float) * n, cudaMemcpyDeviceToDevice, st);
      Scalars one{};
      one.alpha = 1.0;
      cudaMemcpyAsync(sc, &one, sizeof(Scalars), cudaMemcpyHostToDevice, st);
      k_axpy_norm<<<VEC_GRID, VEC_BLOCK, 0, st>>>(d, z, q, q, n, sc, part);  // z = b - q
      k_finalize<<<1, 1024, 0, st>>>(part, VEC_GRID, sc, FIN_RR);
      cudaMemcpyAsync(S.hScal, sc, sizeof(Scalars), cudaMemcpyDeviceToHost, st);
      cudaStreamSynchronize(st);
      relres = pr.bb > 0 ? std::sqrt(S.hScal->rr / pr.bb) : 0.0;
    }
  } else {
    // FP64 iterative refinement around the FP32 MGPCG
    double* x64 = S.x64.as<double>();
    float* rin = S.rin.as<float>();
    cudaMemsetAsync(x64, 0, sizeof(double) * n, st);
    double bb = 0, rr = 0;
    for (int outer = 0;; outer++) {
      rc = residual64(ctx, S, R, b, rin, &rr);
      if (rc) break;
      if (outer == 0) bb = rr;
      relres = bb > 0 ? std::sqrt(rr / bb) : 0.0;
      if (!(bb > 1e-300) || relres <= p->tol) {
        status = 0;
        break;
      }
      if (!std::isfinite(rr)) {
        status = 3;
        break;
      }
      if (outer >= p->maxRefine || iters >= p->maxIter) {
        status = 1;
        break;
      }
      // inner tolerance: what is still missing, not below the FP32 floor
      const double need = p->tol / std::max(relres, 1e-300);
      const double tolIn = std::min(0.5, std::max(need * 0.5, 1e-5));
      PcgResult pr;
      rc = run_pcg(ctx, S, R, rin, tolIn, p->maxIter - iters, p->useGraph, exec, perIter, pr);
      if (rc) break;
      iters += pr.iters;
      refinements++;
      if (pr.status >= 2) {
        status = pr.status;
        break;
      }
      k_add64<<<VEC_GRID, VEC_BLOCK, 0, st>>>(x64, x, n);
      R.launches++;
    }
    k_narrow<<<VEC_GRID, VEC_BLOCK, 0, st>>>(x, x64, n);
    cudaEventRecord(e1, st);
  }
  if (exec) cudaGraphExecDestroy(exec);
  MSBG_CUDA_TRY(ctx, cudaStreamSynchronize(st));
  float ms = 0;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc) return rc;
  if (info) {
    info->iterations = iters;
    info->refinements = refinements;
    info->status = status;
    info->relResidual = relres;
    info->solveSeconds = ms * 1e-3;
    info->fineCells = L0.nFluid;
    info->nMgLevels = (int)S.H.levels.size();
    info->kernelLaunches = R.launches;
  }
  return MSBG_OK;
}

extern "C" int msbg_gpu_pressure_stats(msbg_gpu_ctx* ctx, msbg_gpu_pressure_stats_t* out) {
  if (!ctx || !out) return MSBG_EINVARG;
  auto& sp = solver_of(ctx);
  if (!sp) return set_error(ctx, MSBG_EINVARG, "msbg_gpu_pressure_prepare not called");
  Solver& S = *sp;
  std::memset(out, 0, sizeof(*out));
  out->nMgLevels = (int)S.H.levels.size();
  for (size_t m = 0; m < S.H.levels.size() && m < 32; m++) {
    out->cells[m] = S.H.levels[m].nCells;
    out->fluid[m] = S.H.levels[m].nFluid;
    out->tiles[m] = (int64_t)S.H.levels[m].tiles.size();
  }
  out->h2dBytes = S.h2dBytes;
  out->prepareSeconds = S.prepareSeconds;
  out->buildSeconds = S.buildSeconds;
  size_t fr = 0, tot = 0;
  cudaMemGetInfo(&fr, &tot);
  out->deviceBytesUsed = (int64_t)(tot - fr);
  out->coarseCells = S.H.nCoarse;
  return MSBG_OK;
}

extern "C" int msbg_gpu_pressure_profile(msbg_gpu_ctx* ctx, int what, int reps, int innerIter,
                                         double* msPerCall, double* algBytesPerCall) {
  if (!ctx || reps <= 0 || innerIter < 1) return MSBG_EINVARG;
  auto& sp = solver_of(ctx);
  if (!sp) return set_error(ctx, MSBG_EINVARG, "msbg_gpu_pressure_prepare not called");
  cudaSetDevice(ctx->device);
  Solver& S = *sp;
  cudaStream_t st = ctx->stream;
  Runner R{S, st, 2, 2, innerIter};
  R.err = ctx->errBuf.as<int>();
  R.numSMs = S.numSMs;
  const Level& L0 = S.H.levels[0];
  LevelDev& D0 = *S.dev[0];
  float* x = D0.x.as<float>();
  double* part = S.partial.as<double>();
  const float* b = S.rhs0.as<float>();
  // algorithmic bytes per cell: smoother reads x,b,diag,cx,cy,cz and writes x
  const double smoothB = 28.0, mvB = 24.0, resB = 28.0 + 0.5, prolB = 12.5;
  auto vcycle_bytes = [&]() {
    double s = 0;
    for (size_t m = 0; m + 1 < S.H.levels.size(); m++) {
      const double n = (double)S.H.levels[m].nCells;
      s += n * (4.0 /*zero x*/ + (R.nPre + R.nPost) * smoothB + resB + prolB);
    }
    return s;
  };
  double bytes = 0;
  auto body = [&]() {
    switch (what) {
      case 0: R.smooth(0, x, b, false); break;
      case 3: R.usePipe = false; R.smooth(0, x, b, false); R.usePipe = true; break;
      case 1: R.matvec_dot(x, S.q0.as<float>(), part); break;
      case 2: R.vcycle(0, S.z0.as<float>(), b); break;
      default: break;
    }
  };
  switch (what) {
    case 0:
    case 3: bytes = smoothB * L0.nCells; break;
    case 1: bytes = mvB * L0.nCells; break;
    case 2: bytes = vcycle_bytes(); break;
    default: return set_error(ctx, MSBG_EINVARG, "profile target %d", what);
  }
  MSBG_CUDA_TRY(ctx, cudaMemsetAsync(x, 0, sizeof(float) * L0.nCells, st));
  body();  // warm-up
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, st);
  for (int i = 0; i < reps; i++) body();
  cudaEventRecord(e1, st);
  MSBG_CUDA_TRY(ctx, cudaEventSynchronize(e1));
  float ms = 0;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (msPerCall) *msPerCall = ms / reps;
  if (algBytesPerCall) *algBytesPerCall = bytes;
  return MSBG_OK;
}

namespace {

// Copy a level-0 vector (tile layout) into the reference's packed block layout.
int to_packed(msbg_gpu_ctx* ctx, Solver& S, const float* dvec, float* packed, int64_t n) {
  const Level& L = S.H.levels[0];
  std::vector<float> h(L.nCells);
  MSBG_CUDA_TRY(ctx, cudaMemcpy(h.data(), dvec, sizeof(float) * L.nCells, cudaMemcpyDeviceToHost));
  // block offsets in the packed layout
  const int64_t nb = (int64_t)S.nbx * S.nby * S.nbz;
  std::vector<int64_t> boff(nb + 1, 0);
  for (int64_t b = 0; b < nb; b++) {
    const int bs = S.bsx0 >> S.blockLevel[b];
    boff[b + 1] = boff[b] + (int64_t)bs * bs * bs;
  }
  if (n < boff[nb]) return set_error(ctx, MSBG_EINVARG, "packed buffer too small (%lld < %lld)",
                                     (long long)n, (long long)boff[nb]);
  std::memset(packed, 0, sizeof(float) * boff[nb]);
  for (const Tile& t : L.tiles) {
    for (int k = 0; k < t.ts; k++)
      for (int j = 0; j < t.ts; j++)
        for (int i = 0; i < t.ts; i++) {
          const int X = t.ox + i, Y = t.oy + j, Z = t.oz + k;
          const int bs = S.bsx0 >> t.level;
          const int64_t b = (X / bs) + (int64_t)S.nbx * ((Y / bs) + (int64_t)S.nby * (Z / bs));
          const int vx = X % bs, vy = Y % bs, vz = Z % bs;
          packed[boff[b] + vx + (int64_t)bs * (vy + (int64_t)bs * vz)] =
              h[t.off + i + (int64_t)t.ts * (j + (int64_t)t.ts * k)];
        }
  }
  return MSBG_OK;
}

}  // namespace

extern "C" int msbg_gpu_pressure_packed_size(msbg_gpu_ctx* ctx, int64_t* n) {
  if (!ctx || !n) return MSBG_EINVARG;
  auto& sp = solver_of(ctx);
  if (!sp) return set_error(ctx, MSBG_EINVARG, "msbg_gpu_pressure_prepare not called");
  int64_t s = 0;
  for (int l : sp->blockLevel) {
    const int bs = sp->bsx0 >> l;
    s += (int64_t)bs * bs * bs;
  }
  *n = s;
  return MSBG_OK;
}

extern "C" int msbg_gpu_pressure_download(msbg_gpu_ctx* ctx, float* packed, int64_t n) {
  if (!ctx || !packed) return MSBG_EINVARG;
  auto& sp = solver_of(ctx);
  if (!sp) return set_error(ctx, MSBG_EINVARG, "msbg_gpu_pressure_prepare not called");
  cudaSetDevice(ctx->device);
  MSBG_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  return to_packed(ctx, *sp, sp->dev[0]->x.as<float>(), packed, n);
}

extern "C" int msbg_gpu_pressure_download64(msbg_gpu_ctx* ctx, double* packed, int64_t n) {
  if (!ctx || !packed) return MSBG_EINVARG;
  auto& sp = solver_of(ctx);
  if (!sp) return set_error(ctx, MSBG_EINVARG, "msbg_gpu_pressure_prepare not called");
  Solver& S = *sp;
  if (!S.x64.p) return set_error(ctx, MSBG_EINVARG, "no FP64 solution (solve with maxRefine > 0)");
  cudaSetDevice(ctx->device);
  MSBG_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  const Level& L = S.H.levels[0];
  std::vector<double> h(L.nCells);
  MSBG_CUDA_TRY(ctx, cudaMemcpy(h.data(), S.x64.p, sizeof(double) * L.nCells,
                                cudaMemcpyDeviceToHost));
  const int64_t nb = (int64_t)S.nbx * S.nby * S.nbz;
  std::vector<int64_t> boff(nb + 1, 0);
  for (int64_t b = 0; b < nb; b++) {
    const int bs = S.bsx0 >> S.blockLevel[b];
    boff[b + 1] = boff[b] + (int64_t)bs * bs * bs;
  }
  if (n < boff[nb]) return set_error(ctx, MSBG_EINVARG, "packed buffer too small");
  std::memset(packed, 0, sizeof(double) * boff[nb]);
  for (const Tile& t : L.tiles)
    for (int k = 0; k < t.ts; k++)
      for (int j = 0; j < t.ts; j++)
        for (int i = 0; i < t.ts; i++) {
          const int X = t.ox + i, Y = t.oy + j, Z = t.oz + k;
          const int bs = S.bsx0 >> t.level;
          const int64_t b = (X / bs) + (int64_t)S.nbx * ((Y / bs) + (int64_t)S.nby * (Z / bs));
          packed[boff[b] + (X % bs) + (int64_t)bs * ((Y % bs) + (int64_t)bs * (Z % bs))] =
              h[t.off + i + (int64_t)t.ts * (j + (int64_t)t.ts * k)];
        }
  return MSBG_OK;
}

extern "C" int msbg_gpu_pressure_download_rhs(msbg_gpu_ctx* ctx, float* packed, int64_t n) {
  if (!ctx || !packed) return MSBG_EINVARG;
  auto& sp = solver_of(ctx);
  if (!sp) return set_error(ctx, MSBG_EINVARG, "msbg_gpu_pressure_prepare not called");
  cudaSetDevice(ctx->device);
  MSBG_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  return to_packed(ctx, *sp, sp->rhs0.as<float>(), packed, n);
}
