// Device construction of the pressure hierarchy for the bulk prepare
// (msbg_gpu_pressure_prepare_arrays): the per-cell work of pressure_host.cpp
// on the GPU.  The host keeps the per-tile topology (tile lists, face
// descriptors, interface-plane offsets, the couplings of the upper tile faces,
// which read neighbour blocks); these kernels fill the per-cell arrays:
//   k_build_l0     MG level 0 from the caller's arrays, tile by tile, in the
//                  finite-volume form of sample_level0 (same expressions, same
//                  order, so the results are those of the host build);
//   k_coarse_fluid liquid flags of candidate coarse cells (any liquid child);
//   k_galerkin     exact Galerkin coarsening A_c = P^T A P over the liquid
//                  children, the generic path of galerkin();
//   k_invdiag      1 / a_ii.
#include <cuda_runtime.h>

#include <cstdint>

#include "build_gpu.h"

namespace msbg {
namespace ps {
namespace {

constexpr uint16_t NONFLUID = 0x1 | 0x2 | 0x1000;  // CELL_SOLID | CELL_FIXED | CELL_VOID

__device__ __forceinline__ void axes(int dir, int& a, int& b) {
  a = dir == 0 ? 1 : 0;
  b = dir == 2 ? 1 : 2;
}

__device__ __forceinline__ int tile_at_d(const LevelMapD& M, int l, int X, int Y, int Z) {
  if (l < 0 || l >= MAXRL) return -1;
  const int n = M.tmapN[l];
  if (!n || X < 0 || Y < 0 || Z < 0) return -1;
  const int sh = M.tsSh[l];
  const int tx = X >> sh, ty = Y >> sh, tz = Z >> sh;
  if (tx >= n || ty >= n || tz >= n) return -1;
  return M.tmap[M.tmapOff[l] + tx + (int64_t)n * (ty + (int64_t)n * tz)];
}

__device__ __forceinline__ bool inside_d(const GridD& g, const int f[3]) {
  return f[0] >= 0 && f[1] >= 0 && f[2] >= 0 && f[0] < g.sx && f[1] < g.sy && f[2] < g.sz;
}

__device__ __forceinline__ int level_at_d(const GridD& g, int m, const int f[3]) {
  const int b = (f[0] >> g.sh0) + g.nb1x * ((f[1] >> g.sh0) + g.nb1y * (f[2] >> g.sh0));
  return max(g.blockLevel[b], m);
}

// cell index of level-l cell (X, Y, Z) of a level, or -1
__device__ __forceinline__ int64_t cell_at_d(const LevelMapD& M, int l, int X, int Y, int Z) {
  const int t = tile_at_d(M, l, X, Y, Z);
  if (t < 0) return -1;
  const TileD ft = M.tiles[t];
  return ft.off + (X - ft.ox) + (int64_t)ft.ts * ((Y - ft.oy) + (int64_t)ft.ts * (Z - ft.oz));
}

// ---------------------------------------------------------------------------
// MG level 0: one CTA per tile of the chunk
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_build_l0(L0Args A) {
  const int ti = A.tile0 + blockIdx.x;
  const TileD t = A.tiles[ti];
  const int ts = t.ts, l = t.level, n3 = ts * ts * ts;
  const double h = (double)(1 << l);
  const int64_t r0 = t.off - A.cell0;  // first cell of the tile in the chunk's raw arrays
  const double* planes = A.planes + (size_t)blockIdx.x * 3 * TS_MAX * TS_MAX;
  const float* F[3] = {A.fx, A.fy, A.fz};
  float* CD[3] = {A.cx, A.cy, A.cz};
  int info[6];
  int64_t io[6];
#pragma unroll
  for (int f = 0; f < 6; f++) {
    info[f] = A.faceInfo[ti * 6 + f];
    io[f] = A.ifOff[(size_t)ti * 6 + f];
  }
  unsigned long long fluidCount = 0;
  for (int e = threadIdx.x; e < n3; e += blockDim.x) {
    const int i = e % ts, j = (e / ts) % ts, k = e / (ts * ts);
    const int loc[3] = {i, j, k};
    const int stride[3] = {1, ts, ts * ts};
    const int64_t r = r0 + e, c = t.off + e;
    double diag = 0;
#pragma unroll
    for (int dir = 0; dir < 3; dir++) {
      int ax, bx;
      axes(dir, ax, bx);
      const int pa = loc[ax] + ts * loc[bx];  // index in the face planes
      const double beta = (double)F[dir][r];
      // lower face
      double lo;
      float cd = 0.f;
      if (loc[dir] > 0) {
        lo = h * beta;
        cd = (float)lo;
      } else {
        const int inf = info[2 * dir];
        if (inf < 0) {  // the domain boundary: no coupling through a wall
          lo = A.dbc[2 * dir] == MSBG_DBC_SOLID ? 0.0 : h * beta;
          cd = (float)lo;
        } else if (inf == l) {
          lo = h * beta;
          cd = (float)lo;
        } else if (inf == l + 1) {  // coarser neighbour: (2/3) h beta, on our side
          lo = (2.0 / 3.0) * h * beta;
          if (io[2 * dir] >= 0) A.ifc[io[2 * dir] + pa] = (float)lo;
        } else {  // finer neighbours: four (2/3) (h/2) beta through our own face
          const double hf = (double)(1 << (l - 1));
          lo = 0;
          for (int q = 0; q < 4; q++) lo += (2.0 / 3.0) * hf * beta;
        }
      }
      CD[dir][c] = cd;
      // upper face: the next cell's lower face, or the host's plane
      double up;
      if (loc[dir] < ts - 1) {
        up = h * (double)F[dir][r + stride[dir]];
      } else {
        const int inf = info[2 * dir + 1];
        if (inf < 0) {
          up = A.dbc[2 * dir + 1] == MSBG_DBC_OPEN ? h : 0.0;
        } else {
          up = planes[dir * TS_MAX * TS_MAX + pa];
          if (inf == l + 1 && io[2 * dir + 1] >= 0) A.ifc[io[2 * dir + 1] + pa] = (float)up;
        }
      }
      diag += lo;
      diag += up;
    }
    const uint16_t ct = A.flags[r];
    bool fl = !(ct & NONFLUID);
    uint8_t cty = fl ? CT_LIQUID : (ct & 0x1) ? CT_SOLID : CT_AIR;
    float dg = 0.f, rh = 0.f;
    if (fl) {
      dg = (float)diag;
      const double rv = A.rhs ? (double)A.rhs[r] : 0.0;
      rh = (float)(rv * h * h * h);
      // a cell coupled to nothing: consistent (b = 0) is dropped, otherwise
      // the lowest such cell is reported; a non-finite coefficient too
      if (!isfinite(dg)) {
        atomicMin(A.bad, (unsigned long long)(c * 2));
      } else if (!(dg > 0.f)) {
        if (rh != 0.f) {
          atomicMin(A.bad, (unsigned long long)(c * 2 + 1));
        } else {
          fl = false;
          cty = CT_SOLID;
        }
      }
    }
    A.diag[c] = dg;
    A.rhs0[c] = rh;
    A.ctype[c] = cty;
    A.fluid[c] = fl ? 1 : 0;
    fluidCount += fl ? 1 : 0;
  }
  // CTA sum of the liquid cells
  for (int o = 16; o > 0; o >>= 1) fluidCount += __shfl_down_sync(0xffffffffu, fluidCount, o);
  if ((threadIdx.x & 31) == 0 && fluidCount) atomicAdd(A.nFluid, fluidCount);
}

// ---------------------------------------------------------------------------
// Coarse level m from fine level m-1
// ---------------------------------------------------------------------------
// Liquid flags of the candidate coarse tiles: a cell is liquid if one of its
// children (aggregated) or the same cell (not coarsened here) is.
__global__ void __launch_bounds__(256) k_coarse_fluid(CoarseArgs A) {
  const TileD t = A.cand[blockIdx.x];
  const int ts = t.ts, n3 = ts * ts * ts;
  const int64_t o = A.candOff[blockIdx.x];
  int any = 0;
  for (int e = threadIdx.x; e < n3; e += blockDim.x) {
    const int P[3] = {t.ox + e % ts, t.oy + (e / ts) % ts, t.oz + e / (ts * ts)};
    const int fv[3] = {P[0] << t.level, P[1] << t.level, P[2] << t.level};
    bool f = false;
    if (level_at_d(A.g, A.F.m, fv) == t.level - 1) {
      for (int ch = 0; ch < 8 && !f; ch++) {
        const int64_t fc = cell_at_d(A.F, t.level - 1, 2 * P[0] + (ch & 1),
                                     2 * P[1] + ((ch >> 1) & 1), 2 * P[2] + (ch >> 2));
        f = fc >= 0 && A.fineFluid[fc];
      }
    } else {
      const int64_t fc = cell_at_d(A.F, t.level, P[0], P[1], P[2]);
      f = fc >= 0 && A.fineFluid[fc];
    }
    A.candFluid[o + e] = f ? 1 : 0;
    any |= f ? 1 : 0;
  }
  any = __syncthreads_or(any);
  if (threadIdx.x == 0) A.candAny[blockIdx.x] = any;
}

// The kept candidates' flags into the level's layout, and their count.
__global__ void __launch_bounds__(256) k_place_fluid(const TileD* __restrict__ tiles,
                                                     const int64_t* __restrict__ srcOff,
                                                     const uint8_t* __restrict__ candFluid,
                                                     uint8_t* __restrict__ fluid,
                                                     unsigned long long* __restrict__ nFluid) {
  const TileD t = tiles[blockIdx.x];
  const int n3 = t.ts * t.ts * t.ts;
  const int64_t so = srcOff[blockIdx.x];
  unsigned long long cnt = 0;
  for (int e = threadIdx.x; e < n3; e += blockDim.x) {
    const uint8_t f = candFluid[so + e];
    fluid[t.off + e] = f;
    cnt += f;
  }
  for (int o = 16; o > 0; o >>= 1) cnt += __shfl_down_sync(0xffffffffu, cnt, o);
  if ((threadIdx.x & 31) == 0 && cnt) atomicAdd(nFluid, cnt);
}

// Coupling of fine liquid cell p (level l) across face (dir, side) when the
// neighbour is liquid too, 0 otherwise (pressure_host.cpp fine_pair).
__device__ double fine_pair_d(const GalerkinArgs& A, int l, const int p[3], int dir, int side) {
  const int64_t c0 = cell_at_d(A.F, l, p[0], p[1], p[2]);
  if (c0 < 0 || !A.fineFluid[c0]) return 0;
  int fv[3] = {p[0] << l, p[1] << l, p[2] << l};
  fv[dir] = side ? (p[dir] + 1) << l : (p[dir] << l) - 1;
  if (!inside_d(A.g, fv)) return 0;
  const int l2 = level_at_d(A.g, A.F.m, fv);
  int ax, bx;
  axes(dir, ax, bx);
  if (l2 == l) {
    int q[3] = {p[0], p[1], p[2]};
    q[dir] += side ? 1 : -1;
    const int64_t c1 = cell_at_d(A.F, l, q[0], q[1], q[2]);
    if (c1 < 0 || !A.fineFluid[c1]) return 0;
    const float* cd = dir == 0 ? A.Fcx : dir == 1 ? A.Fcy : A.Fcz;
    return side ? cd[c1] : cd[c0];
  }
  if (l2 == l + 1) {
    const int64_t c1 = cell_at_d(A.F, l + 1, fv[0] >> (l + 1), fv[1] >> (l + 1), fv[2] >> (l + 1));
    if (c1 < 0 || !A.fineFluid[c1]) return 0;
    const int t = tile_at_d(A.F, l, p[0], p[1], p[2]);
    const TileD ft = A.F.tiles[t];
    const int64_t io = A.FifOff[(size_t)t * 6 + dir * 2 + side];
    const int loc[3] = {p[0] - ft.ox, p[1] - ft.oy, p[2] - ft.oz};
    return io >= 0 ? A.Fifc[io + loc[ax] + (int64_t)ft.ts * loc[bx]] : 0.0;
  }
  // finer neighbours: the four fine cells facing us
  double s = 0;
  for (int u = 0; u < 2; u++)
    for (int v = 0; v < 2; v++) {
      int f[3];
      f[dir] = side ? (p[dir] + 1) * 2 : p[dir] * 2 - 1;
      f[ax] = p[ax] * 2 + u;
      f[bx] = p[bx] * 2 + v;
      const int64_t c1 = cell_at_d(A.F, l - 1, f[0], f[1], f[2]);
      if (c1 < 0 || !A.fineFluid[c1]) continue;
      const int t = tile_at_d(A.F, l - 1, f[0], f[1], f[2]);
      const TileD ft = A.F.tiles[t];
      const int64_t io = A.FifOff[(size_t)t * 6 + dir * 2 + (1 - side)];
      const int loc[3] = {f[0] - ft.ox, f[1] - ft.oy, f[2] - ft.oz};
      if (io >= 0) s += A.Fifc[io + loc[ax] + (int64_t)ft.ts * loc[bx]];
    }
  return s;
}

__device__ __forceinline__ bool aggregated_d(const GalerkinArgs& A, int lc, const int P[3]) {
  const int fv[3] = {P[0] << lc, P[1] << lc, P[2] << lc};
  return level_at_d(A.g, A.F.m, fv) == lc - 1;
}

// Coupling of coarse cell P across (dir, side): the sum of the fine liquid
// pairs across that coarse face (pressure_host.cpp coarse_face).
__device__ double coarse_face_d(const GalerkinArgs& A, int lc, const int P[3], int dir, int side) {
  if (!aggregated_d(A, lc, P)) return fine_pair_d(A, lc, P, dir, side);
  int ax, bx;
  axes(dir, ax, bx);
  double s = 0;
  for (int u = 0; u < 2; u++)
    for (int v = 0; v < 2; v++) {
      int f[3];
      f[dir] = P[dir] * 2 + side;
      f[ax] = P[ax] * 2 + u;
      f[bx] = P[bx] * 2 + v;
      s += fine_pair_d(A, lc - 1, f, dir, side);
    }
  return s;
}

// One CTA per coarse tile; the arrays of the coarse level are zeroed before.
__global__ void __launch_bounds__(256) k_galerkin(GalerkinArgs A) {
  const int ti = blockIdx.x;
  const TileD t = A.Gtiles[ti];
  const int lc = t.level, ts = t.ts, n3 = ts * ts * ts;
  float* CD[3] = {A.Gcx, A.Gcy, A.Gcz};
  for (int e = threadIdx.x; e < n3; e += blockDim.x) {
    const int loc[3] = {e % ts, (e / ts) % ts, e / (ts * ts)};
    const int P[3] = {t.ox + loc[0], t.oy + loc[1], t.oz + loc[2]};
    const int64_t c = t.off + e;
    if (!A.coarseFluid[c]) continue;
    double d = 0;
    if (aggregated_d(A, lc, P)) {
      for (int ch = 0; ch < 8; ch++) {
        const int f[3] = {P[0] * 2 + (ch & 1), P[1] * 2 + ((ch >> 1) & 1), P[2] * 2 + (ch >> 2)};
        const int64_t fc = cell_at_d(A.F, lc - 1, f[0], f[1], f[2]);
        if (fc < 0 || !A.fineFluid[fc]) continue;
        d += A.Fdiag[fc];
        // pairs inside the aggregate: each once, from its upper child
        for (int dir = 0; dir < 3; dir++)
          if ((ch >> dir) & 1) d -= 2.0 * fine_pair_d(A, lc - 1, f, dir, 0);
      }
    } else {
      d = A.Fdiag[cell_at_d(A.F, lc, P[0], P[1], P[2])];
    }
    A.Gdiag[c] = (float)d;
    for (int dir = 0; dir < 3; dir++)
      for (int side = 0; side < 2; side++) {
        int fv[3] = {P[0] << lc, P[1] << lc, P[2] << lc};
        fv[dir] = side ? (P[dir] + 1) << lc : (P[dir] << lc) - 1;
        if (!inside_d(A.g, fv)) continue;
        const int l2 = level_at_d(A.g, A.Gm, fv);
        if (l2 == lc && side == 0) {
          CD[dir][c] = (float)coarse_face_d(A, lc, P, dir, side);
        } else if (l2 == lc + 1) {
          const bool onFace = side ? loc[dir] == ts - 1 : loc[dir] == 0;
          const int64_t io = A.GifOff[(size_t)ti * 6 + dir * 2 + side];
          if (onFace && io >= 0) {
            int ax, bx;
            axes(dir, ax, bx);
            A.Gifc[io + loc[ax] + (int64_t)ts * loc[bx]] = (float)coarse_face_d(A, lc, P, dir, side);
          }
        }
      }
  }
}

__global__ void k_invdiag(const float* __restrict__ diag, float* __restrict__ inv, int64_t n) {
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n;
       c += (int64_t)gridDim.x * blockDim.x)
    inv[c] = diag[c] > 0.f ? (float)(1.0 / (double)diag[c]) : 0.f;
}

}  // namespace

cudaError_t launch_build_l0(const L0Args& a, int nTiles, cudaStream_t st) {
  if (nTiles <= 0) return cudaSuccess;
  k_build_l0<<<nTiles, 256, 0, st>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_coarse_fluid(const CoarseArgs& a, int nCand, cudaStream_t st) {
  if (nCand <= 0) return cudaSuccess;
  k_coarse_fluid<<<nCand, 256, 0, st>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_place_fluid(const TileD* tiles, const int64_t* srcOff, const uint8_t* candFluid,
                               uint8_t* fluid, unsigned long long* nFluid, int nTiles,
                               cudaStream_t st) {
  if (nTiles <= 0) return cudaSuccess;
  k_place_fluid<<<nTiles, 256, 0, st>>>(tiles, srcOff, candFluid, fluid, nFluid);
  return cudaGetLastError();
}

cudaError_t launch_galerkin(const GalerkinArgs& a, int nTiles, cudaStream_t st) {
  if (nTiles <= 0) return cudaSuccess;
  k_galerkin<<<nTiles, 256, 0, st>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_invdiag(const float* diag, float* inv, int64_t n, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  const int grid = (int)std::min<int64_t>((n + 255) / 256, 148 * 16);
  k_invdiag<<<grid, 256, 0, st>>>(diag, inv, n);
  return cudaGetLastError();
}

}  // namespace ps
}  // namespace msbg
