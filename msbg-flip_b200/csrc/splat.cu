// Particle splatting into a 16-bit render-density channel: the producer of
// the smoother's input in the reference's demo (msbg_test_sparse,
// src/msbg_demo.cpp:339-684):
//   - particles outside the domain bounds (src/sbg.cpp:287-316) or whose
//     truncated cell leaves the grid are dropped (src/msbg_demo.cpp:358-360);
//   - every block within rScan = rParticle + nbDist of a particle is marked
//     active (src/msbg_demo.cpp:366-379) and becomes a value block at 65535,
//     the others const empty blocks at 0 (src/msbg_demo.cpp:472-500);
//   - each particle lowers every voxel of its scan box within rScan to the
//     quantised squared distance round(d^2 / rScan^2 * 65535)
//     (src/msbg_demo.cpp:553-636); the first voxel inside rScan that lies in a
//     block without values ends the particle's scan (its goto loop_exit);
//   - the minimum is finalised to the render density
//     1 - linstep(-rParticle, rParticle + nbDist, sqrt(d^2) - rParticle)
//     (src/msbg_demo.cpp:661-675).
// The reference splats block colour by colour so that no two threads write
// one block; here each value block is one CTA that gathers the particles of
// its 27-block neighbourhood (binned by their own block with a counting sort)
// and takes the minimum in shared memory, so every voxel is written once, by
// one CTA, with the finalised value.  The minimum does not depend on the
// order, so the result equals the reference's bit for bit.
//
// Arithmetic: the squared distance as the reference's build computes it
// (dz*dz + dy*dy contracted to fma(dy, dy, dz*dz), "+ dx*dx" to
// fma(dx, dx, .)); everything else in source order with explicit rounding
// intrinsics, so no further contraction happens.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdint>
#include <map>
#include <memory>
#include <vector>

#include "common.cuh"

namespace msbg {
namespace {

struct SplatState {
  DeviceBuffer pos;     // [3n] host particles copied in
  DeviceBuffer pblk;    // [n] own block of a kept particle, -1 otherwise
  DeviceBuffer rank;    // [n] position in its block's bin
  DeviceBuffer active;  // [nBlocks] bytes: marked blocks
  DeviceBuffer cnt;     // [nValue + 1] particles per value block, then bin starts
  DeviceBuffer start;   // [nValue + 1] int64 bin starts
  DeviceBuffer scanTmp; // partial sums of the scan
  DeviceBuffer sorted;  // [kept] float4 (x, y, z, abort index as int bits)
  DeviceBuffer vbid;    // [nValue] block id of each value slot
};

std::map<msbg_gpu_ctx*, std::unique_ptr<SplatState>>& states() {
  static std::map<msbg_gpu_ctx*, std::unique_ptr<SplatState>> m;
  return m;
}

struct SplatGeom {
  int s[3];   // grid size
  int nb[3];  // blocks per axis
  int sh;     // log2(bsx)
  float lo[3], hi[3];  // domain bounds of a particle position
  float rScan, rScanBsx, toBlock, distSqMax, distSqMaxInv, rParticle, nbDist;
};

__device__ __forceinline__ int64_t geom_bid(const SplatGeom& g, int bx, int by, int bz) {
  return bx + (int64_t)g.nb[0] * (by + (int64_t)g.nb[1] * bz);
}

// the demo's particle test: a finite position within the domain bounds whose
// truncated cell lies in the grid
__device__ __forceinline__ bool splat_keep(const SplatGeom& g, float x, float y, float z,
                                           int c[3]) {
  const float p[3] = {x, y, z};
#pragma unroll
  for (int k = 0; k < 3; k++) {
    if (!isfinite(p[k]) || p[k] < g.lo[k] || p[k] > g.hi[k]) return false;
    c[k] = (int)p[k];
    if (c[k] < 0 || c[k] > g.s[k] - 1) return false;
  }
  return true;
}

// the particle's scan box [i1, i2] (src/msbg_demo.cpp:563-566)
__device__ __forceinline__ void scan_box(const SplatGeom& g, const float p[3], int i1[3],
                                         int i2[3]) {
#pragma unroll
  for (int k = 0; k < 3; k++) {
    const int a = (int)ceilf(__fsub_rn(__fsub_rn(p[k], g.rScan), 0.5f));
    const int e = (int)floorf(__fsub_rn(__fadd_rn(p[k], g.rScan), 0.5f));
    i1[k] = max(a, 0);
    i2[k] = min(e, g.s[k] - 1);
  }
}

__device__ __forceinline__ float splat_dist_sq(float dx, float dy, float dz) {
  return __fmaf_rn(dx, dx, __fmaf_rn(dy, dy, __fmul_rn(dz, dz)));
}

__device__ __forceinline__ uint32_t splat_quantise(const SplatGeom& g, float distSq) {
  return (uint32_t)(int)roundf(__fmul_rn(__fmul_rn(distSq, g.distSqMaxInv), 65535.0f));
}

__device__ __forceinline__ uint16_t splat_finalise(const SplatGeom& g, uint32_t q) {
  float distSq = __fmul_rn((float)q, 1.f / 65535.f);
  if (!(distSq < 0.999f)) return 0;
  distSq = __fmul_rn(distSq, g.distSqMax);
  const float dist = __fsub_rn(__fsqrt_rn(distSq), g.rParticle);
  const float a = -g.rParticle, b = __fadd_rn(g.rParticle, g.nbDist);
  const float t = dist < a ? 0.f : dist >= b ? 1.f : __fdiv_rn(__fsub_rn(dist, a), __fsub_rn(b, a));
  return (uint16_t)(int)roundf(__fmul_rn(__fsub_rn(1.0f, t), 65535.0f));
}

// Keeps or drops each particle; its own block into pblk; with `active` the
// blocks within rScan are marked.
__global__ void k_splat_classify(const float* __restrict__ pos, int64_t n, SplatGeom g,
                                 int* __restrict__ pblk, uint8_t* __restrict__ active) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const float p[3] = {pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]};
    int c[3];
    if (!splat_keep(g, p[0], p[1], p[2], c)) {
      pblk[i] = -1;
      continue;
    }
    pblk[i] = (int)geom_bid(g, c[0] >> g.sh, c[1] >> g.sh, c[2] >> g.sh);
    if (!active) continue;
    int b1[3], b2[3];
#pragma unroll
    for (int k = 0; k < 3; k++) {
      const float bp = __fmul_rn(p[k], g.toBlock);
      b1[k] = max((int)__fsub_rn(bp, g.rScanBsx), 0);
      b2[k] = min((int)__fadd_rn(bp, g.rScanBsx), g.nb[k] - 1);
    }
    for (int bz = b1[2]; bz <= b2[2]; bz++)
      for (int by = b1[1]; by <= b2[1]; by++)
        for (int bx = b1[0]; bx <= b2[0]; bx++) active[geom_bid(g, bx, by, bz)] = 1;
  }
}

// Particles of value blocks: their rank in the block's bin.
__global__ void k_splat_count(const int* __restrict__ pblk, int64_t n,
                              const int* __restrict__ slot, int* __restrict__ cnt,
                              int* __restrict__ rank) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int b = pblk[i];
    const int s = b >= 0 ? slot[b] : -1;
    rank[i] = s >= 0 ? atomicAdd(&cnt[s], 1) : -1;
  }
}

// Exclusive scan of int counts into int64 starts, in tiles of 1024 x 4.
constexpr int SCAN_T = 1024, SCAN_PER = 4, SCAN_TILE = SCAN_T * SCAN_PER;

__device__ __forceinline__ int64_t block_excl_scan(int64_t v, int64_t* sh, int64_t& total) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int64_t x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int64_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) sh[w] = x;
  __syncthreads();
  if (w == 0) {
    int64_t s = lane < (int)(blockDim.x >> 5) ? sh[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int64_t y = __shfl_up_sync(0xffffffffu, s, o);
      if (lane >= o) s += y;
    }
    sh[lane] = s;
  }
  __syncthreads();
  total = sh[(blockDim.x >> 5) - 1];
  const int64_t before = w > 0 ? sh[w - 1] : 0;
  __syncthreads();
  return before + x - v;
}

template <typename In>
__global__ void __launch_bounds__(SCAN_T) k_scan_tiles(const In* __restrict__ in, int64_t m,
                                                       int64_t* __restrict__ out,
                                                       int64_t* __restrict__ tileSum) {
  __shared__ int64_t sh[32];
  const int64_t base = (int64_t)blockIdx.x * SCAN_TILE + (int64_t)threadIdx.x * SCAN_PER;
  int64_t v[SCAN_PER], sum = 0;
#pragma unroll
  for (int j = 0; j < SCAN_PER; j++) {
    v[j] = base + j < m ? (int64_t)in[base + j] : 0;
    sum += v[j];
  }
  int64_t total;
  int64_t run = block_excl_scan(sum, sh, total);
#pragma unroll
  for (int j = 0; j < SCAN_PER; j++) {
    if (base + j < m) out[base + j] = run;
    run += v[j];
  }
  if (threadIdx.x == 0 && tileSum) tileSum[blockIdx.x] = total;
}

__global__ void k_scan_add(int64_t* __restrict__ out, int64_t m,
                           const int64_t* __restrict__ tileOff) {
  const int64_t i = (int64_t)blockIdx.x * SCAN_TILE + threadIdx.x;
  const int64_t off = tileOff[blockIdx.x];
#pragma unroll
  for (int j = 0; j < SCAN_PER; j++) {
    const int64_t k = i + (int64_t)j * SCAN_T;
    if (k < m) out[k] += off;
  }
}

// The bins: float4 (x, y, z, abort) at start[slot] + rank.  abort is the
// index in the particle's scan box (z, then y, then x) of its first voxel
// within rScan that lies in a block without values, INT_MAX when there is
// none; voxels from that index on are not splatted.
__global__ void k_splat_scatter(const float* __restrict__ pos, int64_t n, SplatGeom g,
                                const int* __restrict__ pblk, const int* __restrict__ rank,
                                const int* __restrict__ slot, const int64_t* __restrict__ start,
                                float4* __restrict__ sorted) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int r = rank[i];
    if (r < 0) continue;
    const float p[3] = {pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]};
    int i1[3], i2[3];
    scan_box(g, p, i1, i2);
    bool allValue = true;
    for (int bz = i1[2] >> g.sh; bz <= i2[2] >> g.sh; bz++)
      for (int by = i1[1] >> g.sh; by <= i2[1] >> g.sh; by++)
        for (int bx = i1[0] >> g.sh; bx <= i2[0] >> g.sh; bx++)
          allValue &= slot[geom_bid(g, bx, by, bz)] >= 0;
    int abortIdx = INT_MAX;
    if (!allValue) {
      const float p0[3] = {__fsub_rn(p[0], 0.5f), __fsub_rn(p[1], 0.5f), __fsub_rn(p[2], 0.5f)};
      const int nx = i2[0] - i1[0] + 1, ny = i2[1] - i1[1] + 1;
      for (int iz = i1[2]; iz <= i2[2] && abortIdx == INT_MAX; iz++) {
        const float dz = __fsub_rn((float)iz, p0[2]);
        for (int iy = i1[1]; iy <= i2[1] && abortIdx == INT_MAX; iy++) {
          const float dy = __fsub_rn((float)iy, p0[1]);
          for (int ix = i1[0]; ix <= i2[0]; ix++) {
            const float dx = __fsub_rn((float)ix, p0[0]);
            if (splat_dist_sq(dx, dy, dz) > g.distSqMax) continue;
            if (slot[geom_bid(g, ix >> g.sh, iy >> g.sh, iz >> g.sh)] < 0) {
              abortIdx = ((iz - i1[2]) * ny + (iy - i1[1])) * nx + (ix - i1[0]);
              break;
            }
          }
        }
      }
    }
    sorted[start[slot[pblk[i]]] + r] =
        make_float4(p[0], p[1], p[2], __int_as_float(abortIdx));
  }
}

// One CTA per value block: the minimum squared distance of the particles
// binned in its 27-block neighbourhood, in shared memory, then quantised and
// finalised (or left raw) into the channel's pool.  The quantisation
// round(d^2 / rScan^2 * 65535) is monotonic in d^2, so quantising the minimum
// equals the reference's minimum of quantised values; the tile holds the
// FP32 bits of d^2 (non-negative floats order like their bit patterns), +inf
// where no particle reaches.
template <int BSX>
__global__ void __launch_bounds__(256, 4) k_splat_blocks(SplatGeom g, const int* __restrict__ slot,
                                                      const int* __restrict__ vbid,
                                                      const int64_t* __restrict__ start,
                                                      const float4* __restrict__ sorted,
                                                      uint16_t* __restrict__ pool, int raw) {
  constexpr int NV = BSX * BSX * BSX;
  extern __shared__ uint32_t tile[];
  const int s = blockIdx.x;
  const int bid = vbid[s];
  const int bx = bid % g.nb[0], by = (bid / g.nb[0]) % g.nb[1],
            bz = bid / (g.nb[0] * g.nb[1]);
  const int B0[3] = {bx * BSX, by * BSX, bz * BSX};
  constexpr uint32_t FAR = 0x7f800000u;  // +inf
  for (int v = threadIdx.x; v < NV; v += blockDim.x) tile[v] = FAR;
  __syncthreads();

  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nWarps = blockDim.x >> 5;
  for (int d = 0; d < 27; d++) {
    const int nx = bx + d % 3 - 1, ny = by + (d / 3) % 3 - 1, nz = bz + d / 9 - 1;
    if (nx < 0 || ny < 0 || nz < 0 || nx >= g.nb[0] || ny >= g.nb[1] || nz >= g.nb[2])
      continue;
    const int ns = slot[geom_bid(g, nx, ny, nz)];
    if (ns < 0) continue;
    const int64_t s0 = start[ns], s1 = start[ns + 1];
    for (int64_t base = s0 + (int64_t)warp * 32; base < s1; base += (int64_t)nWarps * 32) {
      const int64_t j = base + lane;
      float4 P = make_float4(0.f, 0.f, 0.f, 0.f);
      bool hit = false;
      if (j < s1) {
        P = sorted[j];
        const float p[3] = {P.x, P.y, P.z};
        int i1[3], i2[3];
        scan_box(g, p, i1, i2);
        hit = true;
#pragma unroll
        for (int k = 0; k < 3; k++)
          hit &= max(i1[k], B0[k]) <= min(i2[k], B0[k] + BSX - 1);
      }
      unsigned m = __ballot_sync(0xffffffffu, hit);
      while (m) {
        const int k = __ffs(m) - 1;
        m &= m - 1;
        const float p[3] = {__shfl_sync(0xffffffffu, P.x, k), __shfl_sync(0xffffffffu, P.y, k),
                            __shfl_sync(0xffffffffu, P.z, k)};
        const int abortIdx = __float_as_int(__shfl_sync(0xffffffffu, P.w, k));
        int i1[3], i2[3], c1[3], c2[3];
        scan_box(g, p, i1, i2);
#pragma unroll
        for (int q = 0; q < 3; q++) {
          c1[q] = max(i1[q], B0[q]);
          c2[q] = min(i2[q], B0[q] + BSX - 1);
        }
        const float p0[3] = {__fsub_rn(p[0], 0.5f), __fsub_rn(p[1], 0.5f),
                             __fsub_rn(p[2], 0.5f)};
        const int wx = c2[0] - c1[0] + 1, wy = c2[1] - c1[1] + 1;
        const int fx = i2[0] - i1[0] + 1, fy = i2[1] - i1[1] + 1;
        // lanes over the (x, y) columns of the clipped box, each marching the
        // z range that can lie within rScan (a bound one voxel wider than
        // the sphere's chord; the exact test decides inside it)
        for (int t = lane; t < wx * wy; t += 32) {
          const int ly = t / wx, ix = c1[0] + (t - ly * wx), iy = c1[1] + ly;
          const float dx = __fsub_rn((float)ix, p0[0]), dy = __fsub_rn((float)iy, p0[1]);
          const float zr2 = g.distSqMax - (dx * dx + dy * dy);
          if (zr2 < -0.5f) continue;
          const float h = sqrtf(fmaxf(zr2, 0.f)) + 1.f;
          const int z1 = max(c1[2], (int)ceilf(p0[2] - h)), z2 = min(c2[2], (int)floorf(p0[2] + h));
          uint32_t* col = tile + (ix - B0[0]) + BSX * (iy - B0[1]);
          for (int iz = z1; iz <= z2; iz++) {
            const float dz = __fsub_rn((float)iz, p0[2]);
            const float distSq = splat_dist_sq(dx, dy, dz);
            if (distSq > g.distSqMax) continue;
            if (abortIdx != INT_MAX &&
                ((iz - i1[2]) * fy + (iy - i1[1])) * fx + (ix - i1[0]) >= abortIdx)
              continue;
            uint32_t* cell = col + BSX * BSX * (iz - B0[2]);
            const uint32_t bits = __float_as_uint(distSq);
            if (bits < *cell) atomicMin(cell, bits);
          }
        }
      }
    }
  }
  __syncthreads();
  uint32_t* out = reinterpret_cast<uint32_t*>(pool + (int64_t)s * NV);
  for (int v = threadIdx.x; v < NV / 2; v += blockDim.x) {
    const uint32_t ta = tile[2 * v], tb = tile[2 * v + 1];
    const uint32_t a = ta == FAR ? 65535u : splat_quantise(g, __uint_as_float(ta));
    const uint32_t b = tb == FAR ? 65535u : splat_quantise(g, __uint_as_float(tb));
    const uint32_t lo = raw ? a : splat_finalise(g, a), hi = raw ? b : splat_finalise(g, b);
    out[v] = lo | (hi << 16);
  }
}

int grid_for(int64_t n) { return (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 148 * 32)); }

template <int BSX>
cudaError_t launch_blocks(const SplatGeom& g, const int* slot, const int* vbid,
                          const int64_t* start, const float4* sorted, uint16_t* pool,
                          int64_t nValue, int raw, cudaStream_t st) {
  const size_t smem = sizeof(uint32_t) * BSX * BSX * BSX;
  cudaError_t e = cudaFuncSetAttribute(k_splat_blocks<BSX>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  k_splat_blocks<BSX><<<(unsigned)nValue, 256, smem, st>>>(g, slot, vbid, start, sorted, pool,
                                                           raw);
  return cudaGetLastError();
}

// Exclusive scan of m int counts into out[0..m] (out[m] = total).
int scan_counts(msbg_gpu_ctx* ctx, SplatState& S, const int* cnt, int64_t m, int64_t* out) {
  cudaStream_t st = ctx->stream;
  // levels of tile sums: m -> ceil(m / TILE) -> ... -> 1
  std::vector<int64_t> sizes{m + 1};
  while (sizes.back() > SCAN_TILE) sizes.push_back((sizes.back() + SCAN_TILE - 1) / SCAN_TILE);
  size_t tmp = 0;
  for (size_t l = 1; l < sizes.size(); l++) tmp += 2 * (size_t)sizes[l];
  MSBG_CUDA_TRY(ctx, S.scanTmp.ensure(sizeof(int64_t) * (tmp + 2)));
  // level 0 reads the int counts (cnt[m] is 0, so out[m] is the total)
  std::vector<int64_t*> lvl(sizes.size()), sums(sizes.size());
  lvl[0] = out;
  int64_t* t = S.scanTmp.as<int64_t>();
  for (size_t l = 1; l < sizes.size(); l++) {
    sums[l - 1] = t;  // tile sums of level l-1 = input of level l
    lvl[l] = t + sizes[l];
    t += 2 * sizes[l];
  }
  const int64_t tiles0 = (sizes[0] + SCAN_TILE - 1) / SCAN_TILE;
  k_scan_tiles<int><<<(unsigned)tiles0, SCAN_T, 0, st>>>(cnt, sizes[0], lvl[0],
                                                          sizes.size() > 1 ? sums[0] : nullptr);
  for (size_t l = 1; l < sizes.size(); l++) {
    const int64_t tiles = (sizes[l] + SCAN_TILE - 1) / SCAN_TILE;
    k_scan_tiles<int64_t><<<(unsigned)tiles, SCAN_T, 0, st>>>(
        sums[l - 1], sizes[l], lvl[l], l + 1 < sizes.size() ? sums[l] : nullptr);
  }
  for (size_t l = sizes.size() - 1; l >= 1; l--) {
    const int64_t tiles = (sizes[l - 1] + SCAN_TILE - 1) / SCAN_TILE;
    k_scan_add<<<(unsigned)tiles, SCAN_T, 0, st>>>(lvl[l - 1], sizes[l - 1], lvl[l]);
  }
  MSBG_CUDA_TRY(ctx, cudaGetLastError());
  return MSBG_OK;
}

int splat_run(msbg_gpu_ctx* ctx, int chan, const float* pos, int64_t n,
              const msbg_splat_params* prm, const int8_t* kind, int8_t* kindOut,
              bool onDevice) {
  if (!ctx || !prm || n < 0 || (n > 0 && !pos)) return MSBG_EINVARG;
  if (ctx->nbx <= 0) return set_error(ctx, MSBG_EINVARG, "splat: no topology");
  const int bsx = ctx->bsx0;
  const float rP = prm->rParticle, nbD = prm->nbDist;
  if (!(rP > 0.f) || !(nbD >= 0.f) || !std::isfinite(rP + nbD))
    return set_error(ctx, MSBG_EINVARG, "splat: rParticle %g, nbDist %g", rP, nbD);
  if (!(rP + nbD + 1.f <= (float)bsx))
    return set_error(ctx, MSBG_ENOTIMPL,
                     "splat: rParticle + nbDist + 1 = %g exceeds the block size %d (a particle "
                     "would reach past the neighbouring blocks)",
                     rP + nbD + 1.f, bsx);
  if (bsx != 8 && bsx != 16 && bsx != 32)
    return set_error(ctx, MSBG_ENOTIMPL, "splat: block size %d", bsx);
  if (n > INT_MAX) return set_error(ctx, MSBG_ENOTIMPL, "splat: %lld particles", (long long)n);
  cudaSetDevice(ctx->device);
  cudaStream_t st = ctx->stream;
  auto& sp = states()[ctx];
  if (!sp) sp = std::make_unique<SplatState>();
  SplatState& S = *sp;
  const int64_t nb = ctx->nb();

  SplatGeom g;
  g.s[0] = ctx->sx;
  g.s[1] = ctx->sy;
  g.s[2] = ctx->sz;
  g.nb[0] = ctx->nbx;
  g.nb[1] = ctx->nby;
  g.nb[2] = ctx->nbz;
  g.sh = bsx == 8 ? 3 : bsx == 16 ? 4 : 5;
  for (int k = 0; k < 3; k++) {  // src/sbg.cpp:287-303: the first try of beps 1e-4
    g.lo[k] = 0.0f + 1e-4f;
    g.hi[k] = (float)g.s[k] - 1e-4f;
  }
  g.rParticle = rP;
  g.nbDist = nbD;
  g.rScan = rP + nbD;
  g.rScanBsx = g.rScan / (float)bsx;
  g.toBlock = 1.0f / (float)bsx;
  g.distSqMax = g.rScan * g.rScan;
  g.distSqMaxInv = 1.0f / g.distSqMax;

  const float* dpos = pos;
  if (!onDevice && n > 0) {
    MSBG_CUDA_TRY(ctx, S.pos.ensure(sizeof(float) * 3 * (size_t)n));
    MSBG_CUDA_TRY(ctx, cudaMemcpyAsync(S.pos.p, pos, sizeof(float) * 3 * (size_t)n,
                                       cudaMemcpyHostToDevice, st));
    dpos = S.pos.as<float>();
  }
  MSBG_CUDA_TRY(ctx, S.pblk.ensure(sizeof(int) * (size_t)std::max<int64_t>(n, 1)));
  MSBG_CUDA_TRY(ctx, S.rank.ensure(sizeof(int) * (size_t)std::max<int64_t>(n, 1)));

  // the block kinds: marked blocks, or the caller's
  std::vector<int8_t> kindHost((size_t)nb);
  if (!kind) {
    MSBG_CUDA_TRY(ctx, S.active.ensure((size_t)nb));
    MSBG_CUDA_TRY(ctx, cudaMemsetAsync(S.active.p, 0, (size_t)nb, st));
  }
  if (n > 0)
    k_splat_classify<<<grid_for(n), 256, 0, st>>>(dpos, n, g, S.pblk.as<int>(),
                                                  kind ? nullptr : S.active.as<uint8_t>());
  MSBG_CUDA_TRY(ctx, cudaGetLastError());
  if (!kind) {
    std::vector<uint8_t> act((size_t)nb);
    MSBG_CUDA_TRY(ctx, cudaMemcpyAsync(act.data(), S.active.p, (size_t)nb,
                                       cudaMemcpyDeviceToHost, st));
    MSBG_CUDA_TRY(ctx, cudaStreamSynchronize(st));
    for (int64_t b = 0; b < nb; b++) kindHost[b] = act[b] ? MSBG_BLOCK_VALUE : MSBG_BLOCK_EMPTY;
  } else {
    for (int64_t b = 0; b < nb; b++) {
      if (kind[b] < MSBG_BLOCK_NULL || kind[b] > MSBG_BLOCK_FULL)
        return set_error(ctx, MSBG_EINVARG, "splat: kind[%lld]=%d", (long long)b, kind[b]);
      kindHost[b] = kind[b];
    }
  }
  if (kindOut) std::copy(kindHost.begin(), kindHost.end(), kindOut);

  // the channel: value blocks at level 0, const blocks at 0 (empty) / 65535
  auto ch = std::make_unique<Channel>();
  {
    auto old = ctx->channels.find(chan);
    if (old != ctx->channels.end()) {  // its allocations are reused; it is gone
      MSBG_CUDA_TRY(ctx, cudaStreamSynchronize(st));
      ch->reuse(*old->second);
      ctx->channels.erase(old);
    }
  }
  ch->level = 0;
  ch->bsx = bsx;
  ch->dtype = MSBG_U16;
  ch->emptyQ = 0;
  ch->fullQ = 65535;
  ch->kindHost = kindHost;
  ch->slotHost.resize((size_t)nb);
  std::vector<int> vb;
  for (int64_t b = 0; b < nb; b++) {
    switch (kindHost[b]) {
      case MSBG_BLOCK_VALUE:
        ch->slotHost[b] = (int)vb.size();
        vb.push_back((int)b);
        break;
      case MSBG_BLOCK_EMPTY: ch->slotHost[b] = SLOT_EMPTY; break;
      case MSBG_BLOCK_FULL: ch->slotHost[b] = SLOT_FULL; break;
      default: ch->slotHost[b] = SLOT_NULL; break;
    }
  }
  const int64_t nValue = (int64_t)vb.size();
  ch->nValue = nValue;
  const size_t nv = (size_t)bsx * bsx * bsx;
  MSBG_CUDA_TRY(ctx, ch->pool.ensure(sizeof(uint16_t) * nv * (size_t)std::max<int64_t>(nValue, 1)));
  MSBG_CUDA_TRY(ctx, ch->slot.ensure(sizeof(int) * (size_t)nb));
  MSBG_CUDA_TRY(ctx, cudaMemcpyAsync(ch->slot.p, ch->slotHost.data(), sizeof(int) * nb,
                                     cudaMemcpyHostToDevice, st));
  if (nValue > 0) {
    MSBG_CUDA_TRY(ctx, S.vbid.ensure(sizeof(int) * (size_t)nValue));
    MSBG_CUDA_TRY(ctx, cudaMemcpyAsync(S.vbid.p, vb.data(), sizeof(int) * nValue,
                                       cudaMemcpyHostToDevice, st));
    // bins of the particles by their own value block
    MSBG_CUDA_TRY(ctx, S.cnt.ensure(sizeof(int) * (size_t)(nValue + 1)));
    MSBG_CUDA_TRY(ctx, S.start.ensure(sizeof(int64_t) * (size_t)(nValue + 1)));
    MSBG_CUDA_TRY(ctx, cudaMemsetAsync(S.cnt.p, 0, sizeof(int) * (size_t)(nValue + 1), st));
    if (n > 0)
      k_splat_count<<<grid_for(n), 256, 0, st>>>(S.pblk.as<int>(), n, ch->slot.as<int>(),
                                                 S.cnt.as<int>(), S.rank.as<int>());
    MSBG_CUDA_TRY(ctx, cudaGetLastError());
    int rc = scan_counts(ctx, S, S.cnt.as<int>(), nValue, S.start.as<int64_t>());
    if (rc) return rc;
    MSBG_CUDA_TRY(ctx, S.sorted.ensure(sizeof(float4) * (size_t)std::max<int64_t>(n, 1)));
    if (n > 0)
      k_splat_scatter<<<grid_for(n), 256, 0, st>>>(dpos, n, g, S.pblk.as<int>(),
                                                   S.rank.as<int>(), ch->slot.as<int>(),
                                                   S.start.as<int64_t>(), S.sorted.as<float4>());
    MSBG_CUDA_TRY(ctx, cudaGetLastError());
    const int raw = (prm->flags & MSBG_SPLAT_RAW) ? 1 : 0;
    cudaError_t e;
    switch (bsx) {
      case 8:
        e = launch_blocks<8>(g, ch->slot.as<int>(), S.vbid.as<int>(), S.start.as<int64_t>(),
                             S.sorted.as<float4>(), ch->pool.as<uint16_t>(), nValue, raw, st);
        break;
      case 16:
        e = launch_blocks<16>(g, ch->slot.as<int>(), S.vbid.as<int>(), S.start.as<int64_t>(),
                              S.sorted.as<float4>(), ch->pool.as<uint16_t>(), nValue, raw, st);
        break;
      default:
        e = launch_blocks<32>(g, ch->slot.as<int>(), S.vbid.as<int>(), S.start.as<int64_t>(),
                              S.sorted.as<float4>(), ch->pool.as<uint16_t>(), nValue, raw, st);
        break;
    }
    MSBG_CUDA_TRY(ctx, e);
  }
  ctx->channels[chan] = std::move(ch);
  return msbg_gpu_sync(ctx);
}

}  // namespace

void splat_release(msbg_gpu_ctx* ctx) { states().erase(ctx); }

}  // namespace msbg

using namespace msbg;

extern "C" int msbg_gpu_splat_particles(msbg_gpu_ctx* ctx, int chan, const float* pos,
                                        int64_t n, const msbg_splat_params* prm,
                                        const int8_t* kind, int8_t* kindOut) {
  return splat_run(ctx, chan, pos, n, prm, kind, kindOut, false);
}

extern "C" int msbg_gpu_splat_particles_device(msbg_gpu_ctx* ctx, int chan, const float* pos,
                                               int64_t n, const msbg_splat_params* prm,
                                               const int8_t* kind, int8_t* kindOut) {
  return splat_run(ctx, chan, pos, n, prm, kind, kindOut, true);
}
