// G2P on mixed-resolution grids: the MAC velocity interpolation of
// interpVec3MSBG / interpCompMSBG (src/flip_sim.cpp:1354-1525) inside
// gridToParticle (src/flip_sim.cpp:1526-1545), and the fine/coarse distance
// channel it blends with (CH_DIST_FINECOARSE, built by setRefinementMap,
// src/msbg.cpp:1700-1723, 1887-1960, 1994-2029):
//   msbg_gpu_flip_mr_dist        the distance channel, built on the GPU
//   msbg_gpu_flip_mr_channel     the velocity channels in/out
//   msbg_gpu_flip_g2p_mr(_device) the particle update
//   msbg_gpu_flip_downsample_velocity  downsampleVelocity (src/msbg4.cpp:2035),
//                                the velocity restricted to the next MG level
//
// Layout (the packed layout of the pressure channels): for every block in
// ascending bid, its (bsx0 >> level)^3 voxels at its own level, vid = x +
// y*bs + z*bs^2.  A voxel of a level's grid inside a block of another level
// has no data there and reads 0, as a NULL block of that level's sparse grid
// does in the reference.  Vector channels hold the lower-face MAC values (u,
// v, w) per voxel.
//
// Per particle and component, one sample geometry serves both channels (vel
// and velOld) and the distance lookup; the arithmetic is the reference's, in
// its order, with no contraction into FMAs, and MtLinstep in double
// (src/mtool.c:200-208).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <map>
#include <memory>
#include <vector>

#include "common.cuh"

namespace msbg {
namespace {

// The reference's transition width: MultiresSparseGrid::create fixes
// _dTransRes at 6 whatever it is passed (src/msbg.cpp:198-201, 290).
constexpr int kDTransRes = 6;

struct MrState {
  int sx = 0, sy = 0, sz = 0, bsx0 = 0, nLevels = 0;
  std::vector<int> levels;
  int64_t n = 0;  // packed voxels
  bool distBuilt = false;
  DeviceBuffer level, off, fc, kind, dist, vel, velOld, parts;
  DeviceBuffer dsOffA, dsOffB, dsFlags, dsSrc, dsDst;  // downsampleVelocity
};

std::map<msbg_gpu_ctx*, std::unique_ptr<MrState>>& states() {
  static std::map<msbg_gpu_ctx*, std::unique_ptr<MrState>> m;
  return m;
}

struct MrGrid {
  int sx, sy, sz, sh0, nbx, nby, nbz, nl;
  const int8_t* __restrict__ level;
  const int64_t* __restrict__ off;
  const int8_t* __restrict__ kind;  // [nl][nb]: 0 empty, 1 value, 2 full
  const uint16_t* __restrict__ dist;
  // packed index of voxel (x, y, z) of level lv, or -1 (outside the level's
  // grid, or in a block of another level)
  __device__ __forceinline__ int64_t idx(int lv, int x, int y, int z) const {
    if (x < 0 || y < 0 || z < 0 || x >= (sx >> lv) || y >= (sy >> lv) || z >= (sz >> lv))
      return -1;
    const int sh = sh0 - lv, m = (1 << sh) - 1;
    const int64_t b = (x >> sh) + (int64_t)nbx * ((y >> sh) + (int64_t)nby * (z >> sh));
    if (level[b] != lv) return -1;
    return off[b] + (x & m) + ((int64_t)(y & m) << sh) + ((int64_t)(z & m) << (2 * sh));
  }
};

// BLK_FINE_COARSE per block: a block of a coarser level among its 26
// neighbours (src/msbg.cpp:1700-1723).
__global__ void k_mr_fine_coarse(const int8_t* __restrict__ level, int nbx, int nby, int nbz,
                                 int8_t* __restrict__ fc) {
  const int64_t nb = (int64_t)nbx * nby * nbz;
  for (int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; b < nb;
       b += (int64_t)gridDim.x * blockDim.x) {
    const int bx = (int)(b % nbx), by = (int)((b / nbx) % nby), bz = (int)(b / ((int64_t)nbx * nby));
    const int lv = level[b];
    int8_t f = 0;
    for (int d = 0; d < 27; d++) {
      const int x = bx + d % 3 - 1, y = by + (d / 3) % 3 - 1, z = bz + d / 9 - 1;
      if (d == 13 || x < 0 || y < 0 || z < 0 || x >= nbx || y >= nby || z >= nbz) continue;
      if (level[x + (int64_t)nbx * (y + (int64_t)nby * z)] > lv) f = 1;
    }
    fc[b] = f;
  }
}

// Block kinds of the distance channel of every level: value blocks are the
// BLK_FINE_COARSE blocks of that level; a block of level l or l-1 with a
// BLK_FINE_COARSE neighbour of level l is a full block of value
// dTransRes*1024 in the channel of level l (src/msbg.cpp:1994-2029).
__global__ void k_mr_kind(const int8_t* __restrict__ level, const int8_t* __restrict__ fc,
                          int nbx, int nby, int nbz, int nl, int8_t* __restrict__ kind) {
  const int64_t nb = (int64_t)nbx * nby * nbz;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nb * nl;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int l = (int)(i / nb);
    const int64_t b = i - (int64_t)l * nb;
    const int lv = level[b];
    int8_t k = 0;
    if (lv == l && fc[b]) {
      k = 1;
    } else if (lv == l || lv == l - 1) {
      const int bx = (int)(b % nbx), by = (int)((b / nbx) % nby),
                bz = (int)(b / ((int64_t)nbx * nby));
      for (int d = 0; d < 27; d++) {
        const int x = bx + d % 3 - 1, y = by + (d / 3) % 3 - 1, z = bz + d / 9 - 1;
        if (d == 13 || x < 0 || y < 0 || z < 0 || x >= nbx || y >= nby || z >= nbz) continue;
        const int64_t b2 = x + (int64_t)nbx * (y + (int64_t)nby * z);
        if (level[b2] == l && fc[b2]) k = 2;
      }
    }
    kind[i] = k;
  }
}

// The distance values: one CTA per block (grid-stride over blocks).  A
// BLK_FINE_COARSE block stores per voxel of its level the distance from the
// voxel centre to the nearest coarser neighbour's box (src/msbg.h:3936-3948),
// capped at dTransRes, as (uint16)(dist*1024); every other block stores 0.
// The squared distances are sums of squares of half-integers, exact in FP32,
// and __fsqrt_rn rounds as the host's sqrtf does.
__global__ void __launch_bounds__(256) k_mr_dist(MrGrid g, const int8_t* __restrict__ fc,
                                                 uint16_t* __restrict__ dist) {
  __shared__ int act[26][3];
  __shared__ int nAct;
  const int64_t nb = (int64_t)g.nbx * g.nby * g.nbz;
  for (int64_t b = blockIdx.x; b < nb; b += gridDim.x) {
    const int lv = g.level[b], sh = g.sh0 - lv, bs = 1 << sh;
    const int bx = (int)(b % g.nbx), by = (int)((b / g.nbx) % g.nby),
              bz = (int)(b / ((int64_t)g.nbx * g.nby));
    __syncthreads();  // the previous block's readers are done with act
    if (threadIdx.x == 0) {
      int n = 0;
      if (fc[b])
        for (int d = 0; d < 27; d++) {
          const int x = bx + d % 3 - 1, y = by + (d / 3) % 3 - 1, z = bz + d / 9 - 1;
          if (d == 13 || x < 0 || y < 0 || z < 0 || x >= g.nbx || y >= g.nby || z >= g.nbz)
            continue;
          if (g.level[x + (int64_t)g.nbx * (y + (int64_t)g.nby * z)] <= lv) continue;
          act[n][0] = x;
          act[n][1] = y;
          act[n][2] = z;
          n++;
        }
      nAct = n;
    }
    __syncthreads();
    const int na = nAct, nv = bs * bs * bs;
    uint16_t* out = dist + g.off[b];
    for (int v = threadIdx.x; v < nv; v += blockDim.x) {
      if (!na) {
        out[v] = 0;
        continue;
      }
      const float p[3] = {(float)(bx * bs + (v & (bs - 1))) + 0.5f,
                          (float)(by * bs + ((v >> sh) & (bs - 1))) + 0.5f,
                          (float)(bz * bs + (v >> (2 * sh))) + 0.5f};
      float d2 = 1e20f;
      for (int i = 0; i < na; i++) {
        float s = 0.f;
#pragma unroll
        for (int c = 0; c < 3; c++) {
          const float lo = (float)(act[i][c] * bs), hi = (float)((act[i][c] + 1) * bs);
          float e = fmaxf(__fsub_rn(lo, p[c]), 0.f);
          e = fmaxf(e, __fsub_rn(p[c], hi));
          s = __fadd_rn(s, __fmul_rn(e, e));
        }
        d2 = fminf(d2, s);
      }
      float d = __fsqrt_rn(d2);
      if (d > (float)kDTransRes) d = (float)kDTransRes;
      out[v] = (uint16_t)__fmul_rn(d, 1024.f);
    }
  }
}

// SparseGrid<uint16_t>::interpolateToFloat<IP_LINEAR> with OPT_IPBC_NEUMAN
// (src/sbg.h:1386, 2936-2941, 3111-3420) on the distance channel of level
// lv: cell-centred, the 2x2x2 window clamped to the grid, value blocks read
// their data, full blocks dTransRes*1024, the others 0; p1*t + p0*(1-t)
// along x, then y, then z.
__device__ __forceinline__ float dist_interp(const MrGrid& g, int lv, float px, float py,
                                             float pz) {
  const float x = __fsub_rn(px, 0.5f), y = __fsub_rn(py, 0.5f), z = __fsub_rn(pz, 0.5f);
  const int ix = (int)floorf(x), iy = (int)floorf(y), iz = (int)floorf(z);
  const float u = __fsub_rn(x, (float)ix), v = __fsub_rn(y, (float)iy),
              w = __fsub_rn(z, (float)iz);
  const int nx = g.sx >> lv, ny = g.sy >> lv, nz = g.sz >> lv, sh = g.sh0 - lv;
  const int64_t nb = (int64_t)g.nbx * g.nby * g.nbz;
  const float full = (float)(kDTransRes * 1024);
  float bz2[2];
#pragma unroll
  for (int k = 0; k < 2; k++) {
    const int zz = min(max(iz + k, 0), nz - 1);
    float by2[2];
#pragma unroll
    for (int j = 0; j < 2; j++) {
      const int yy = min(max(iy + j, 0), ny - 1);
      float bx2[2];
#pragma unroll
      for (int i = 0; i < 2; i++) {
        const int xx = min(max(ix + i, 0), nx - 1);
        const int64_t b = (xx >> sh) + (int64_t)g.nbx * ((yy >> sh) + (int64_t)g.nby * (zz >> sh));
        const int kd = g.kind[(int64_t)lv * nb + b];
        bx2[i] = kd == 1 ? (float)g.dist[g.idx(lv, xx, yy, zz)] : kd == 2 ? full : 0.f;
      }
      by2[j] = __fadd_rn(__fmul_rn(bx2[1], u), __fmul_rn(bx2[0], __fsub_rn(1.0f, u)));
    }
    bz2[k] = __fadd_rn(__fmul_rn(by2[1], v), __fmul_rn(by2[0], __fsub_rn(1.0f, v)));
  }
  return __fadd_rn(__fmul_rn(bz2[1], w), __fmul_rn(bz2[0], __fsub_rn(1.0f, w)));
}

__device__ __constant__ float kMrOff[3][3] = {{0.f, 0.5f, 0.5f}, {0.5f, 0.f, 0.5f},
                                              {0.5f, 0.5f, 0.f}};

// Trilinear sums of component d in both channels at level lv, from the
// sample origin (ix0, iy0, iz0) and fractions (fx, fy, fz).
__device__ __forceinline__ void trilinear2(const MrGrid& g, int lv, const float* __restrict__ a,
                                           const float* __restrict__ b, int d, int ix0, int iy0,
                                           int iz0, float fx, float fy, float fz, float& sa,
                                           float& sb) {
  sa = 0.f;
  sb = 0.f;
#pragma unroll
  for (int c = 0; c < 8; c++) {
    const int dx = c & 1, dy = (c >> 1) & 1, dz = c >> 2;
    const int64_t i = g.idx(lv, ix0 + dx, iy0 + dy, iz0 + dz);
    const float va = i < 0 ? 0.f : a[3 * i + d], vb = i < 0 ? 0.f : b[3 * i + d];
    const float w = __fmul_rn(__fmul_rn(dx ? fx : __fsub_rn(1.f, fx), dy ? fy : __fsub_rn(1.f, fy)),
                              dz ? fz : __fsub_rn(1.f, fz));
    sa = __fadd_rn(sa, __fmul_rn(w, va));
    sb = __fadd_rn(sb, __fmul_rn(w, vb));
  }
}

// gridToParticle with interpCompMSBG per component (interpVec3MSBG yields the
// same per component: its shared path, taken when the three staggered
// samples share a block, computes exactly interpCompMSBG's expressions).
// la, lb: MtLinstep's bounds as the reference forms them in float.
__global__ void k_g2p_mr(msbg_flip_particle* __restrict__ p, int64_t np, MrGrid g,
                         const float* __restrict__ vel, const float* __restrict__ velOld,
                         float alpha, double la, double lb) {
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < np;
       k += (int64_t)gridDim.x * blockDim.x) {
    msbg_flip_particle q = p[k];
    const bool finite = isfinite(q.pos[0]) && isfinite(q.pos[1]) && isfinite(q.pos[2]);
#pragma unroll
    for (int d = 0; d < 3; d++) {
      float pic = 0.f, old = 0.f;  // no cell for a particle without a finite position
      if (finite) {
        const float gx = __fsub_rn(q.pos[0], kMrOff[d][0]), gy = __fsub_rn(q.pos[1], kMrOff[d][1]),
                    gz = __fsub_rn(q.pos[2], kMrOff[d][2]);
        const int ix0 = (int)floorf(gx), iy0 = (int)floorf(gy), iz0 = (int)floorf(gz);
        const float fx = __fsub_rn(gx, (float)ix0), fy = __fsub_rn(gy, (float)iy0),
                    fz = __fsub_rn(gz, (float)iz0);
        const int cx = min(max(ix0, 0), g.sx - 1), cy = min(max(iy0, 0), g.sy - 1),
                  cz = min(max(iz0, 0), g.sz - 1);
        const int lv = g.level[(cx >> g.sh0) +
                               (int64_t)g.nbx * ((cy >> g.sh0) + (int64_t)g.nby * (cz >> g.sh0))];
        float fa, fb;
        trilinear2(g, 0, vel, velOld, d, ix0, iy0, iz0, fx, fy, fz, fa, fb);
        if (lv == 0) {
          pic = fa;
          old = fb;
        } else {
          const float scale = 1.f / (float)(1 << lv);  // a power of two: exact
          const float cgx = __fmul_rn(gx, scale), cgy = __fmul_rn(gy, scale),
                      cgz = __fmul_rn(gz, scale);
          const int cix0 = (int)floorf(cgx), ciy0 = (int)floorf(cgy), ciz0 = (int)floorf(cgz);
          const float cfx = __fsub_rn(cgx, (float)cix0), cfy = __fsub_rn(cgy, (float)ciy0),
                      cfz = __fsub_rn(cgz, (float)ciz0);
          float ca, cb;
          trilinear2(g, lv, vel, velOld, d, cix0, ciy0, ciz0, cfx, cfy, cfz, ca, cb);
          const float dist = __fmul_rn(dist_interp(g, lv, cgx, cgy, cgz), 1.0f / 1024.0f);
          const double x = (double)dist;
          const float af = x < la ? 0.f : x >= lb ? 1.f : (float)((x - la) / (lb - la));
          const float bf = __fsub_rn(1.f, af);
          pic = __fadd_rn(__fmul_rn(af, fa), __fmul_rn(bf, ca));
          old = __fadd_rn(__fmul_rn(af, fb), __fmul_rn(bf, cb));
        }
      }
      q.vel[d] = __fadd_rn(__fmul_rn(__fsub_rn(1.f, alpha), pic),
                           __fmul_rn(alpha, __fadd_rn(q.vel[d], __fsub_rn(pic, old))));
    }
    p[k].vel[0] = q.vel[0];
    p[k].vel[1] = q.vel[1];
    p[k].vel[2] = q.vel[2];
  }
}

// downsampleVelocity (src/msbg4.cpp:2035-2270), MG level m-1 -> m, one CTA
// per block (grid-stride), its threads over the block's voxels.  Block b sits
// at level max(level0[b], m - 1) at MG level m-1 (offA) and max(level0[b], m)
// at MG level m (offB).  A block already at level >= m is copied (0 in SOLID
// or VOID cells); a block coarsened at this MG level takes per non-SOLID cell
// the 4x4x4 (1,3,3,1)^3/512 sum over the level-(m-1) cells 2x-1 .. 2x+2
// clamped to that level's grid, each from the level-(m-1) block where it is
// one at MG level m-1, else the level-m value at (x2/2, y2/2, z2/2), summed in
// the reference's order k, j, i without contraction.
__global__ void __launch_bounds__(256)
    k_downsample_velocity(int sx, int sy, int sz, int sh0, int nbx, int nby, int nbz, int m,
                          const int8_t* __restrict__ level0, const int64_t* __restrict__ offA,
                          const int64_t* __restrict__ offB, const uint16_t* __restrict__ flags,
                          const float* __restrict__ src, float* __restrict__ dst) {
  const int64_t nb = (int64_t)nbx * nby * nbz;
  const int fs = m - 1, nsx = sx >> fs, nsy = sy >> fs, nsz = sz >> fs, shA = sh0 - fs;
  for (int64_t b = blockIdx.x; b < nb; b += gridDim.x) {
    const int l0 = level0[b], lv = max(l0, m), sh = sh0 - lv, bs = 1 << sh;
    const int bx = (int)(b % nbx), by = (int)((b / nbx) % nby), bz = (int)(b / ((int64_t)nbx * nby));
    const int nv = bs * bs * bs;
    for (int v = threadIdx.x; v < nv; v += blockDim.x) {
      const uint16_t fl = flags[offB[b] + v];
      float* out = dst + 3 * (offB[b] + v);
      if (l0 >= m) {
        const float* in = src + 3 * (offA[b] + v);
        const bool zero = (fl & (0x1 | 0x1000)) != 0;  // CELL_SOLID | CELL_VOID
        out[0] = zero ? 0.f : in[0];
        out[1] = zero ? 0.f : in[1];
        out[2] = zero ? 0.f : in[2];
        continue;
      }
      float v0 = 0.f, v1 = 0.f, v2 = 0.f;
      if (!(fl & 0x1)) {
        const int x = bx * bs + (v & (bs - 1)), y = by * bs + ((v >> sh) & (bs - 1)),
                  z = bz * bs + (v >> (2 * sh));
        for (int k = 0; k < 4; k++) {
          const int z2 = min(max(2 * z - 1 + k, 0), nsz - 1);
          for (int j = 0; j < 4; j++) {
            const int y2 = min(max(2 * y - 1 + j, 0), nsy - 1);
#pragma unroll
            for (int i = 0; i < 4; i++) {
              const int x2 = min(max(2 * x - 1 + i, 0), nsx - 1);
              const int64_t b2 = (x2 >> shA) + (int64_t)nbx * ((y2 >> shA) + (int64_t)nby * (z2 >> shA));
              const int l2 = max((int)level0[b2], fs);  // its level at MG level m-1
              int64_t q = -1;
              if (l2 == fs) {
                const int mk = (1 << shA) - 1;
                q = offA[b2] + (x2 & mk) + ((int64_t)(y2 & mk) << shA) +
                    ((int64_t)(z2 & mk) << (2 * shA));
              } else if (l2 == fs + 1) {
                const int s2 = shA - 1, mk = (1 << s2) - 1;
                q = offA[b2] + ((x2 >> 1) & mk) + ((int64_t)((y2 >> 1) & mk) << s2) +
                    ((int64_t)((z2 >> 1) & mk) << (2 * s2));
              }
              const float w = (float)((i == 0 || i == 3 ? 1 : 3) * (j == 0 || j == 3 ? 1 : 3) *
                                      (k == 0 || k == 3 ? 1 : 3)) * (1.0f / 512.0f);
              const float f0 = q < 0 ? 0.f : src[3 * q], f1 = q < 0 ? 0.f : src[3 * q + 1],
                          f2 = q < 0 ? 0.f : src[3 * q + 2];
              v0 = __fadd_rn(v0, __fmul_rn(f0, w));
              v1 = __fadd_rn(v1, __fmul_rn(f1, w));
              v2 = __fadd_rn(v2, __fmul_rn(f2, w));
            }
          }
        }
      }
      out[0] = v0;
      out[1] = v1;
      out[2] = v2;
    }
  }
}

int grid_blocks(int64_t n) { return (int)std::min<int64_t>((n + 255) / 256, 148 * 32); }

// The state of a context for its current topology (rebuilt when it changed).
// The reference asserts that 26-neighbour blocks differ by at most one level
// (src/msbg.cpp:1718-1719); such a map is rejected here.
int mr_state(msbg_gpu_ctx* ctx, MrState** out, MrGrid& g) {
  if (!ctx->bsx0 || ctx->nLevels < 1)
    return set_error(ctx, MSBG_EINVARG, "msbg_gpu_sync_topology not called");
  auto& sp = states()[ctx];
  if (!sp || sp->sx != ctx->sx || sp->sy != ctx->sy || sp->sz != ctx->sz ||
      sp->bsx0 != ctx->bsx0 || sp->nLevels != ctx->nLevels || sp->levels != ctx->blockLevel) {
    const int64_t nb = ctx->nb();
    for (int64_t b = 0; b < nb; b++) {
      const int bx = (int)(b % ctx->nbx), by = (int)((b / ctx->nbx) % ctx->nby),
                bz = (int)(b / ((int64_t)ctx->nbx * ctx->nby));
      for (int d = 0; d < 27; d++) {
        const int x = bx + d % 3 - 1, y = by + (d / 3) % 3 - 1, z = bz + d / 9 - 1;
        if (x < 0 || y < 0 || z < 0 || x >= ctx->nbx || y >= ctx->nby || z >= ctx->nbz) continue;
        const int l2 = ctx->blockLevel[x + (int64_t)ctx->nbx * (y + (int64_t)ctx->nby * z)];
        if (std::abs(l2 - ctx->blockLevel[b]) > 1)
          return set_error(ctx, MSBG_EINVARG,
                           "blocks %lld and a neighbour differ by more than one level",
                           (long long)b);
      }
    }
    std::unique_ptr<MrState> s(new MrState());
    s->sx = ctx->sx;
    s->sy = ctx->sy;
    s->sz = ctx->sz;
    s->bsx0 = ctx->bsx0;
    s->nLevels = ctx->nLevels;
    s->levels = ctx->blockLevel;
    std::vector<int8_t> lv8(nb);
    std::vector<int64_t> off(nb);
    int64_t o = 0;
    for (int64_t b = 0; b < nb; b++) {
      lv8[b] = (int8_t)ctx->blockLevel[b];
      off[b] = o;
      const int64_t bs = ctx->bsx0 >> ctx->blockLevel[b];
      o += bs * bs * bs;
    }
    s->n = o;
    cudaStream_t st = ctx->stream;
    MSBG_CUDA_TRY(ctx, s->level.ensure(nb));
    MSBG_CUDA_TRY(ctx, s->off.ensure(8 * nb));
    MSBG_CUDA_TRY(ctx, s->fc.ensure(nb));
    MSBG_CUDA_TRY(ctx, s->kind.ensure((size_t)nb * ctx->nLevels));
    MSBG_CUDA_TRY(ctx, s->dist.ensure(2 * (size_t)o));
    MSBG_CUDA_TRY(ctx, s->vel.ensure(12 * (size_t)o));
    MSBG_CUDA_TRY(ctx, s->velOld.ensure(12 * (size_t)o));
    MSBG_CUDA_TRY(ctx, cudaMemcpyAsync(s->level.p, lv8.data(), nb, cudaMemcpyHostToDevice, st));
    MSBG_CUDA_TRY(ctx, cudaMemcpyAsync(s->off.p, off.data(), 8 * nb, cudaMemcpyHostToDevice, st));
    MSBG_CUDA_TRY(ctx, cudaMemsetAsync(s->vel.p, 0, s->vel.bytes, st));
    MSBG_CUDA_TRY(ctx, cudaMemsetAsync(s->velOld.p, 0, s->velOld.bytes, st));
    // the host vectors are read by the copies above before they go out of scope
    MSBG_CUDA_TRY(ctx, cudaStreamSynchronize(st));
    sp = std::move(s);
  }
  MrState& S = *sp;
  int sh = 0;
  while ((1 << sh) < ctx->bsx0) sh++;
  g = MrGrid{S.sx, S.sy, S.sz, sh, ctx->nbx, ctx->nby, ctx->nbz, S.nLevels,
             S.level.as<int8_t>(), S.off.as<int64_t>(), S.kind.as<int8_t>(),
             S.dist.as<uint16_t>()};
  *out = sp.get();
  return MSBG_OK;
}

int mr_build_dist(msbg_gpu_ctx* ctx, MrState* S, const MrGrid& g) {
  if (S->distBuilt) return MSBG_OK;
  const int64_t nb = ctx->nb();
  cudaStream_t st = ctx->stream;
  k_mr_fine_coarse<<<grid_blocks(nb), 256, 0, st>>>(S->level.as<int8_t>(), ctx->nbx, ctx->nby,
                                                     ctx->nbz, S->fc.as<int8_t>());
  k_mr_kind<<<grid_blocks(nb * S->nLevels), 256, 0, st>>>(S->level.as<int8_t>(),
                                                           S->fc.as<int8_t>(), ctx->nbx, ctx->nby,
                                                           ctx->nbz, S->nLevels,
                                                           S->kind.as<int8_t>());
  k_mr_dist<<<(int)std::min<int64_t>(nb, 148 * 16), 256, 0, st>>>(g, S->fc.as<int8_t>(),
                                                                   S->dist.as<uint16_t>());
  MSBG_CUDA_TRY(ctx, cudaGetLastError());
  S->distBuilt = true;
  return MSBG_OK;
}

}  // namespace

void flip_mr_release(msbg_gpu_ctx* ctx) { states().erase(ctx); }

}  // namespace msbg

using namespace msbg;

extern "C" int msbg_gpu_flip_mr_dist(msbg_gpu_ctx* ctx, uint16_t* dist, int64_t n, int8_t* kind,
                                     int64_t nk) {
  if (!ctx) return MSBG_EINVARG;
  cudaSetDevice(ctx->device);
  MrState* S = nullptr;
  MrGrid g;
  int rc = mr_state(ctx, &S, g);
  if (rc) return rc;
  if (dist && n != S->n)
    return set_error(ctx, MSBG_EINVARG, "distance channel holds %lld voxels, not %lld",
                     (long long)S->n, (long long)n);
  if (kind && nk != ctx->nb() * S->nLevels)
    return set_error(ctx, MSBG_EINVARG, "block kinds: %lld entries, not %lld",
                     (long long)(ctx->nb() * S->nLevels), (long long)nk);
  rc = mr_build_dist(ctx, S, g);
  if (rc) return rc;
  if (dist)
    MSBG_CUDA_TRY(ctx, cudaMemcpyAsync(dist, S->dist.p, 2 * (size_t)n, cudaMemcpyDeviceToHost,
                                       ctx->stream));
  if (kind)
    MSBG_CUDA_TRY(ctx, cudaMemcpyAsync(kind, S->kind.p, (size_t)nk, cudaMemcpyDeviceToHost,
                                       ctx->stream));
  return msbg_gpu_sync(ctx);
}

extern "C" int msbg_gpu_flip_mr_channel(msbg_gpu_ctx* ctx, int which, float* data, int64_t n,
                                        int get) {
  if (!ctx || !data) return MSBG_EINVARG;
  cudaSetDevice(ctx->device);
  MrState* S = nullptr;
  MrGrid g;
  int rc = mr_state(ctx, &S, g);
  if (rc) return rc;
  DeviceBuffer* b = which == MSBG_FLIP_VEL ? &S->vel : which == MSBG_FLIP_VEL_OLD ? &S->velOld
                                                                                  : nullptr;
  if (!b) return set_error(ctx, MSBG_EINVARG, "mixed-resolution channel %d unknown", which);
  if (n != 3 * S->n)
    return set_error(ctx, MSBG_EINVARG, "mixed-resolution channel holds %lld floats, not %lld",
                     (long long)(3 * S->n), (long long)n);
  MSBG_CUDA_TRY(ctx, cudaMemcpyAsync(get ? (void*)data : b->p, get ? b->p : (const void*)data,
                                     sizeof(float) * n,
                                     get ? cudaMemcpyDeviceToHost : cudaMemcpyHostToDevice,
                                     ctx->stream));
  return msbg_gpu_sync(ctx);
}

namespace {
int flip_g2p_mr(msbg_gpu_ctx* ctx, msbg_flip_particle* particles, int64_t np, float flipAlpha,
                bool onDevice) {
  if (!ctx || (!particles && np) || np < 0) return MSBG_EINVARG;
  cudaSetDevice(ctx->device);
  MrState* S = nullptr;
  MrGrid g;
  int rc = mr_state(ctx, &S, g);
  if (rc) return rc;
  rc = mr_build_dist(ctx, S, g);
  if (rc) return rc;
  if (!np) return msbg_gpu_sync(ctx);
  cudaStream_t st = ctx->stream;
  msbg_flip_particle* dp = particles;
  if (!onDevice) {
    MSBG_CUDA_TRY(ctx, S->parts.ensure(sizeof(msbg_flip_particle) * (size_t)np));
    MSBG_CUDA_TRY(ctx, cudaMemcpyAsync(S->parts.p, particles, sizeof(msbg_flip_particle) * np,
                                       cudaMemcpyHostToDevice, st));
    dp = S->parts.as<msbg_flip_particle>();
  }
  // MtLinstep's bounds as interpCompMSBG forms them, in float
  // (src/flip_sim.cpp:1514-1521): stenWidth 2, MT_SQRT3F
  const float sqrt3 = 1.73205080756887f;
  const float la = (1.0f * sqrt3) * 1.01f, lb = (0.99f * ((float)kDTransRes + 2.f)) / sqrt3;
  k_g2p_mr<<<grid_blocks(np), 256, 0, st>>>(dp, np, g, S->vel.as<float>(), S->velOld.as<float>(),
                                            flipAlpha, (double)la, (double)lb);
  MSBG_CUDA_TRY(ctx, cudaGetLastError());
  if (!onDevice)
    MSBG_CUDA_TRY(ctx, cudaMemcpyAsync(particles, dp, sizeof(msbg_flip_particle) * np,
                                       cudaMemcpyDeviceToHost, st));
  return msbg_gpu_sync(ctx);
}
}  // namespace

extern "C" int msbg_gpu_flip_g2p_mr(msbg_gpu_ctx* ctx, msbg_flip_particle* particles, int64_t np,
                                    float flipAlpha) {
  return flip_g2p_mr(ctx, particles, np, flipAlpha, false);
}

extern "C" int msbg_gpu_flip_g2p_mr_device(msbg_gpu_ctx* ctx, msbg_flip_particle* particles,
                                           int64_t np, float flipAlpha) {
  return flip_g2p_mr(ctx, particles, np, flipAlpha, true);
}

extern "C" int msbg_gpu_flip_downsample_velocity(msbg_gpu_ctx* ctx, int levelMg,
                                                 const uint16_t* flags, const float* src,
                                                 int64_t nSrc, float* dst, int64_t nDst) {
  if (!ctx || !flags || !src || !dst) return MSBG_EINVARG;
  cudaSetDevice(ctx->device);
  MrState* S = nullptr;
  MrGrid g;
  int rc = mr_state(ctx, &S, g);
  if (rc) return rc;
  if (levelMg < 1 || levelMg >= ctx->nLevels)
    return set_error(ctx, MSBG_EINVARG, "levelMg=%d: the sparse MG levels are 1..%d", levelMg,
                     ctx->nLevels - 1);
  const int64_t nb = ctx->nb();
  std::vector<int64_t> offA(nb), offB(nb);
  int64_t nA = 0, nB = 0;
  for (int64_t b = 0; b < nb; b++) {
    const int l0 = ctx->blockLevel[b];
    const int64_t bsA = ctx->bsx0 >> std::max(l0, levelMg - 1), bsB = ctx->bsx0 >> std::max(l0, levelMg);
    offA[b] = nA;
    offB[b] = nB;
    nA += bsA * bsA * bsA;
    nB += bsB * bsB * bsB;
  }
  if (nSrc != 3 * nA || nDst != 3 * nB)
    return set_error(ctx, MSBG_EINVARG,
                     "MG levels %d / %d hold %lld / %lld floats, not %lld / %lld", levelMg - 1,
                     levelMg, (long long)(3 * nA), (long long)(3 * nB), (long long)nSrc,
                     (long long)nDst);
  cudaStream_t st = ctx->stream;
  MSBG_CUDA_TRY(ctx, S->dsOffA.ensure(8 * nb));
  MSBG_CUDA_TRY(ctx, S->dsOffB.ensure(8 * nb));
  MSBG_CUDA_TRY(ctx, S->dsFlags.ensure(2 * (size_t)nB));
  MSBG_CUDA_TRY(ctx, S->dsSrc.ensure(12 * (size_t)nA));
  MSBG_CUDA_TRY(ctx, S->dsDst.ensure(12 * (size_t)nB));
  MSBG_CUDA_TRY(ctx, cudaMemcpyAsync(S->dsOffA.p, offA.data(), 8 * nb, cudaMemcpyHostToDevice, st));
  MSBG_CUDA_TRY(ctx, cudaMemcpyAsync(S->dsOffB.p, offB.data(), 8 * nb, cudaMemcpyHostToDevice, st));
  MSBG_CUDA_TRY(ctx, cudaMemcpyAsync(S->dsFlags.p, flags, 2 * nB, cudaMemcpyHostToDevice, st));
  MSBG_CUDA_TRY(ctx, cudaMemcpyAsync(S->dsSrc.p, src, 12 * nA, cudaMemcpyHostToDevice, st));
  k_downsample_velocity<<<(int)std::min<int64_t>(nb, 148 * 16), 256, 0, st>>>(
      ctx->sx, ctx->sy, ctx->sz, g.sh0, ctx->nbx, ctx->nby, ctx->nbz, levelMg,
      S->level.as<int8_t>(), S->dsOffA.as<int64_t>(), S->dsOffB.as<int64_t>(),
      S->dsFlags.as<uint16_t>(), S->dsSrc.as<float>(), S->dsDst.as<float>());
  MSBG_CUDA_TRY(ctx, cudaGetLastError());
  MSBG_CUDA_TRY(ctx, cudaMemcpyAsync(dst, S->dsDst.p, 12 * nB, cudaMemcpyDeviceToHost, st));
  // the offset vectors are read by the copies above before they go out of scope
  return msbg_gpu_sync(ctx);
}
