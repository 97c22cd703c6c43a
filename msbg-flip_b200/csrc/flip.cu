// FLIP transfers around the pressure solve, on the context's single-level
// grid (every block at level 0, all blocks present), device-resident grid
// channels in the block layout (blocks in bid order, bsx^3 voxels, vid =
// x + y*bsx + z*bsx^2; vector channels hold the lower-face u, v, w of each
// voxel):
//   msbg_gpu_flip_p2g              FlipSimulation::particleToGrid
//                                  (src/flip_sim.cpp:579-831)
//   msbg_gpu_flip_gravity          applyGravity (src/flip_sim.cpp:832-857)
//   msbg_gpu_flip_pressure_gradient the pressure-gradient update of
//                                  pressureProjection (src/flip_sim.cpp:1316-1349)
//   msbg_gpu_flip_g2p              gridToParticle with the level-0 branch of
//                                  interpVec3MSBG (src/flip_sim.cpp:1354-1395, 1526-1545)
// The scatter of P2G accumulates with float atomics (a sum whose order varies
// from run to run, as the reference's thread-local merge does); every other
// step is one thread per voxel face or per particle, with the reference's
// expressions in its order and no contraction into FMAs.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <map>
#include <memory>
#include <vector>

#include "common.cuh"

namespace msbg {
namespace {

struct FlipState {
  int sx = 0, sy = 0, sz = 0, bsx = 0;
  int64_t n = 0;
  DeviceBuffer vel, velOld, beta, mass, liq, acc, active, parts;
};

std::map<msbg_gpu_ctx*, std::unique_ptr<FlipState>>& states() {
  static std::map<msbg_gpu_ctx*, std::unique_ptr<FlipState>> m;
  return m;
}

struct GridF {
  int sx, sy, sz, sh, nbx, nby;
  // voxel index in the block layout, or -1 outside the grid
  __device__ __forceinline__ int64_t idx(int x, int y, int z) const {
    if (x < 0 || y < 0 || z < 0 || x >= sx || y >= sy || z >= sz) return -1;
    const int m = (1 << sh) - 1;
    const int64_t bid = (x >> sh) + (int64_t)nbx * ((y >> sh) + (int64_t)nby * (z >> sh));
    return (bid << (3 * sh)) + (x & m) + ((int64_t)(y & m) << sh) + ((int64_t)(z & m) << (2 * sh));
  }
  // voxel coordinates of block-layout index i
  __device__ __forceinline__ void coords(int64_t i, int& x, int& y, int& z) const {
    const int m = (1 << sh) - 1;
    const int64_t bid = i >> (3 * sh);
    const int v = (int)(i & ((1 << (3 * sh)) - 1));
    x = (int)(bid % nbx) * (1 << sh) + (v & m);
    y = (int)((bid / nbx) % nby) * (1 << sh) + ((v >> sh) & m);
    z = (int)(bid / ((int64_t)nbx * nby)) * (1 << sh) + (v >> (2 * sh));
  }
};

__device__ __constant__ float kOff[3][3] = {{0.f, 0.5f, 0.5f}, {0.5f, 0.f, 0.5f},
                                            {0.5f, 0.5f, 0.f}};

// The particles' cell mass and trilinear face weights (particleToGrid's
// scatter loop).  acc: [vx vy vz wu wv ww ru rv rw][n].
__global__ void k_p2g_scatter(const msbg_flip_particle* __restrict__ p, int64_t np, GridF g,
                              int64_t n, float rhoL, float rhoG, float* __restrict__ acc,
                              float* __restrict__ mass, int* __restrict__ liq) {
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < np;
       k += (int64_t)gridDim.x * blockDim.x) {
    const msbg_flip_particle q = p[k];
    // a particle without a finite position reaches no cell
    if (!isfinite(q.pos[0]) || !isfinite(q.pos[1]) || !isfinite(q.pos[2])) continue;
    const float mp = q.phase == 0 ? rhoL : rhoG;
    const int64_t ci = g.idx((int)floorf(q.pos[0]), (int)floorf(q.pos[1]), (int)floorf(q.pos[2]));
    if (ci >= 0) {
      atomicAdd(&mass[ci], 1.f);
      if (q.phase == 0) atomicAdd(&liq[ci], 1);
    }
#pragma unroll
    for (int d = 0; d < 3; d++) {
      const float gx = __fsub_rn(q.pos[0], kOff[d][0]), gy = __fsub_rn(q.pos[1], kOff[d][1]),
                  gz = __fsub_rn(q.pos[2], kOff[d][2]);
      const int ix0 = (int)floorf(gx), iy0 = (int)floorf(gy), iz0 = (int)floorf(gz);
      const float fx = __fsub_rn(gx, (float)ix0), fy = __fsub_rn(gy, (float)iy0),
                  fz = __fsub_rn(gz, (float)iz0);
#pragma unroll
      for (int c = 0; c < 8; c++) {
        const int dx = c & 1, dy = (c >> 1) & 1, dz = c >> 2;
        const float w = __fmul_rn(__fmul_rn(dx ? fx : __fsub_rn(1.f, fx), dy ? fy : __fsub_rn(1.f, fy)),
                                  dz ? fz : __fsub_rn(1.f, fz));
        const int64_t i = g.idx(ix0 + dx, iy0 + dy, iz0 + dz);
        if (i < 0) continue;
        atomicAdd(&acc[(size_t)d * n + i], __fmul_rn(q.vel[d], w));
        atomicAdd(&acc[(size_t)(3 + d) * n + i], w);
        atomicAdd(&acc[(size_t)(6 + d) * n + i], __fmul_rn(mp, w));
      }
    }
  }
}

struct P2GConst {
  float massEps, rhoL, rhoG, betaMin, rtMin, phiDen;
};

// Phase of a cell for the interface clamp: -1 empty or outside, 0 liquid
// (more than half of its particles liquid), 1 air.
__device__ __forceinline__ int cell_phase(const GridF& g, const float* mass, const int* liq,
                                          float eps, int x, int y, int z) {
  const int64_t j = g.idx(x, y, z);
  if (j < 0 || !(mass[j] > eps)) return -1;
  return liq[j] * 2 > (int)__fadd_rn(mass[j], 0.5f) ? 0 : 1;
}

// Face velocities normalised by their weights; beta = max(1/rho, betaMin)
// from the two-phase density, clamped where both cells of a face agree; the
// blocks holding mass.
__global__ void k_p2g_finish(GridF g, int64_t n, P2GConst c, const float* __restrict__ acc,
                             const float* __restrict__ mass, const int* __restrict__ liq,
                             float* __restrict__ vel, float* __restrict__ beta,
                             int* __restrict__ active) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    int x, y, z;
    g.coords(i, x, y, z);
#pragma unroll
    for (int d = 0; d < 3; d++) {
      const float w = acc[(size_t)(3 + d) * n + i];
      vel[3 * i + d] = w > c.massEps ? __fdiv_rn(acc[(size_t)d * n + i], w) : 0.f;
    }
    if (mass[i] > c.massEps) active[i >> (3 * g.sh)] = 1;
#pragma unroll
    for (int d = 0; d < 3; d++) {
      const float rt = acc[(size_t)(6 + d) * n + i];
      float phi = 0.f;
      if (!(rt < c.rtMin)) phi = fminf(__fsqrt_rn(__fdiv_rn(fmaxf(__fsub_rn(rt, c.rtMin), 0.f), c.phiDen)), 1.f);
      const int pa = cell_phase(g, mass, liq, c.massEps, x - (d == 0), y - (d == 1), z - (d == 2));
      const int pb = cell_phase(g, mass, liq, c.massEps, x, y, z);
      if (pa == 0 && pb == 0)
        phi = 1.f;
      else if (pa == 1 && pb == 1)
        phi = 0.f;
      const float rho = __fadd_rn(c.rhoG, __fmul_rn(phi, __fsub_rn(c.rhoL, c.rhoG)));
      beta[3 * i + d] = fmaxf(__fdiv_rn(1.f, rho), c.betaMin);
    }
  }
}

// vel_old = vel; gravity on the v faces next to liquid; the reference's wall
// faces set to 0 (x at 0 and sx-1, y at 0, z at 0 and sz-1).
__global__ void k_gravity(GridF g, int64_t n, float* __restrict__ vel,
                          float* __restrict__ velOld, const float* __restrict__ mass, float gdt,
                          float eps) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    int x, y, z;
    g.coords(i, x, y, z);
    float v[3] = {vel[3 * i], vel[3 * i + 1], vel[3 * i + 2]};
    velOld[3 * i] = v[0];
    velOld[3 * i + 1] = v[1];
    velOld[3 * i + 2] = v[2];
    const int64_t lo = g.idx(x, y - 1, z);
    if ((lo >= 0 && mass[lo] > eps) || mass[i] > eps) v[1] = __fadd_rn(v[1], gdt);
    if (x == 0 || x == g.sx - 1) v[0] = 0.f;
    if (y == 0) v[1] = 0.f;
    if (z == 0 || z == g.sz - 1) v[2] = 0.f;
    vel[3 * i] = v[0];
    vel[3 * i + 1] = v[1];
    vel[3 * i + 2] = v[2];
  }
}

// u -= dt beta (p_b - p_a) on each lower face, pressure 0 in a cell without
// liquid; faces between two cells without liquid and the lower domain faces 0.
__global__ void k_gradient(GridF g, int64_t n, float* __restrict__ vel,
                           const float* __restrict__ mass, const float* __restrict__ beta,
                           const float* __restrict__ pres, float dt, float eps) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    int x, y, z;
    g.coords(i, x, y, z);
    const int p[3] = {x, y, z};
    const bool fb = mass[i] > eps;
#pragma unroll
    for (int d = 0; d < 3; d++) {
      if (p[d] == 0) {
        vel[3 * i + d] = 0.f;
        continue;
      }
      const int64_t j = g.idx(x - (d == 0), y - (d == 1), z - (d == 2));
      const bool fa = mass[j] > eps;
      if (!fa && !fb) {
        vel[3 * i + d] = 0.f;
        continue;
      }
      const float pa = fa ? pres[j] : 0.f, pb = fb ? pres[i] : 0.f;
      const float v =
          __fsub_rn(vel[3 * i + d], __fmul_rn(__fmul_rn(dt, beta[3 * i + d]), __fsub_rn(pb, pa)));
      vel[3 * i + d] = isfinite(v) ? v : 0.f;
    }
  }
}

__device__ __forceinline__ float interp_comp(const GridF& g, const float* __restrict__ v,
                                             const float pos[3], int d) {
  if (!isfinite(pos[0]) || !isfinite(pos[1]) || !isfinite(pos[2])) return 0.f;  // no cell
  const float gx = __fsub_rn(pos[0], kOff[d][0]), gy = __fsub_rn(pos[1], kOff[d][1]),
              gz = __fsub_rn(pos[2], kOff[d][2]);
  const int ix0 = (int)floorf(gx), iy0 = (int)floorf(gy), iz0 = (int)floorf(gz);
  const float fx = __fsub_rn(gx, (float)ix0), fy = __fsub_rn(gy, (float)iy0),
              fz = __fsub_rn(gz, (float)iz0);
  float sum = 0.f;
#pragma unroll
  for (int c = 0; c < 8; c++) {
    const int dx = c & 1, dy = (c >> 1) & 1, dz = c >> 2;
    const int64_t i = g.idx(ix0 + dx, iy0 + dy, iz0 + dz);
    const float val = i < 0 ? 0.f : v[3 * i + d];
    const float w = __fmul_rn(__fmul_rn(dx ? fx : __fsub_rn(1.f, fx), dy ? fy : __fsub_rn(1.f, fy)),
                              dz ? fz : __fsub_rn(1.f, fz));
    sum = __fadd_rn(sum, __fmul_rn(w, val));
  }
  return sum;
}

__global__ void k_g2p(msbg_flip_particle* __restrict__ p, int64_t np, GridF g,
                      const float* __restrict__ vel, const float* __restrict__ velOld,
                      float alpha) {
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < np;
       k += (int64_t)gridDim.x * blockDim.x) {
    msbg_flip_particle q = p[k];
#pragma unroll
    for (int d = 0; d < 3; d++) {
      const float pic = interp_comp(g, vel, q.pos, d), old = interp_comp(g, velOld, q.pos, d);
      q.vel[d] = __fadd_rn(__fmul_rn(__fsub_rn(1.f, alpha), pic),
                           __fmul_rn(alpha, __fadd_rn(q.vel[d], __fsub_rn(pic, old))));
    }
    p[k].vel[0] = q.vel[0];
    p[k].vel[1] = q.vel[1];
    p[k].vel[2] = q.vel[2];
  }
}

int grid_of(msbg_gpu_ctx* ctx, GridF& g) {
  if (!ctx->bsx0 || ctx->nLevels < 1)
    return set_error(ctx, MSBG_EINVARG, "msbg_gpu_sync_topology not called");
  for (int l : ctx->blockLevel)
    if (l != 0) return set_error(ctx, MSBG_ENOTIMPL, "the FLIP transfers need every block at level 0");
  int sh = 0;
  while ((1 << sh) < ctx->bsx0) sh++;
  g = GridF{ctx->sx, ctx->sy, ctx->sz, sh, ctx->nbx, ctx->nby};
  return MSBG_OK;
}

// The grid channels of a context for its current topology (reallocated when
// the topology changed).
int state_of(msbg_gpu_ctx* ctx, FlipState** out, GridF& g) {
  int rc = grid_of(ctx, g);
  if (rc) return rc;
  auto& sp = states()[ctx];
  if (!sp || sp->sx != ctx->sx || sp->sy != ctx->sy || sp->sz != ctx->sz || sp->bsx != ctx->bsx0) {
    sp.reset(new FlipState());
    FlipState& S = *sp;
    S.sx = ctx->sx;
    S.sy = ctx->sy;
    S.sz = ctx->sz;
    S.bsx = ctx->bsx0;
    S.n = (int64_t)S.sx * S.sy * S.sz;
    const size_t n = (size_t)S.n;
    MSBG_CUDA_TRY(ctx, S.vel.ensure(12 * n));
    MSBG_CUDA_TRY(ctx, S.velOld.ensure(12 * n));
    MSBG_CUDA_TRY(ctx, S.beta.ensure(12 * n));
    MSBG_CUDA_TRY(ctx, S.mass.ensure(4 * n));
    MSBG_CUDA_TRY(ctx, S.liq.ensure(4 * n));
    MSBG_CUDA_TRY(ctx, S.active.ensure(4 * (size_t)ctx->nb()));
    for (DeviceBuffer* b : {&S.vel, &S.velOld, &S.beta, &S.mass})
      MSBG_CUDA_TRY(ctx, cudaMemsetAsync(b->p, 0, b->bytes, ctx->stream));
  }
  *out = sp.get();
  return MSBG_OK;
}

int grid_blocks(int64_t n) { return (int)std::min<int64_t>((n + 255) / 256, 148 * 32); }

}  // namespace

void flip_release(msbg_gpu_ctx* ctx) { states().erase(ctx); }

}  // namespace msbg

using namespace msbg;

namespace {

int flip_p2g(msbg_gpu_ctx* ctx, const msbg_flip_particle* particles, int64_t np,
             const msbg_flip_params* prm, int* activeBlocks, int64_t* nActive, bool onDevice) {
  if (!ctx || (!particles && np) || np < 0 || !prm) return MSBG_EINVARG;
  if (!(prm->rhoL > 0.f) || !(prm->rhoG > 0.f) || prm->particlesPerVoxel <= 0 ||
      !(prm->alphaPhi > 0.f))
    return set_error(ctx, MSBG_EINVARG, "FLIP parameters: densities, alphaPhi and particles "
                                        "per voxel must be positive");
  cudaSetDevice(ctx->device);
  FlipState* S = nullptr;
  GridF g;
  int rc = state_of(ctx, &S, g);
  if (rc) return rc;
  cudaStream_t st = ctx->stream;
  const int64_t n = S->n;
  MSBG_CUDA_TRY(ctx, S->acc.ensure(sizeof(float) * 9 * (size_t)n));
  MSBG_CUDA_TRY(ctx, cudaMemsetAsync(S->acc.p, 0, S->acc.bytes, st));
  MSBG_CUDA_TRY(ctx, cudaMemsetAsync(S->mass.p, 0, 4 * (size_t)n, st));
  MSBG_CUDA_TRY(ctx, cudaMemsetAsync(S->liq.p, 0, 4 * (size_t)n, st));
  MSBG_CUDA_TRY(ctx, cudaMemsetAsync(S->active.p, 0, S->active.bytes, st));
  const msbg_flip_particle* dp = particles;
  if (np && !onDevice) {
    MSBG_CUDA_TRY(ctx, S->parts.ensure(sizeof(msbg_flip_particle) * (size_t)np));
    MSBG_CUDA_TRY(ctx, cudaMemcpyAsync(S->parts.p, particles, sizeof(msbg_flip_particle) * np,
                                       cudaMemcpyHostToDevice, st));
    dp = S->parts.as<msbg_flip_particle>();
  }
  if (np)
    k_p2g_scatter<<<grid_blocks(np), 256, 0, st>>>(dp, np, g, n, prm->rhoL, prm->rhoG,
                                                   S->acc.as<float>(), S->mass.as<float>(),
                                                   S->liq.as<int>());
  P2GConst c;
  c.massEps = prm->massEps;
  c.rhoL = prm->rhoL;
  c.rhoG = prm->rhoG;
  c.betaMin = prm->betaMin;
  const float rt0 = (float)prm->particlesPerVoxel;
  c.rtMin = logf(prm->rhoL / prm->rhoG) * prm->rhoG * rt0;
  c.phiDen = prm->alphaPhi * rt0 * prm->rhoL;
  k_p2g_finish<<<grid_blocks(n), 256, 0, st>>>(g, n, c, S->acc.as<float>(), S->mass.as<float>(),
                                               S->liq.as<int>(), S->vel.as<float>(),
                                               S->beta.as<float>(), S->active.as<int>());
  MSBG_CUDA_TRY(ctx, cudaGetLastError());
  if (activeBlocks || nActive) {
    std::vector<int> flags((size_t)ctx->nb());
    MSBG_CUDA_TRY(ctx, cudaMemcpyAsync(flags.data(), S->active.p, 4 * flags.size(),
                                       cudaMemcpyDeviceToHost, st));
    MSBG_CUDA_TRY(ctx, cudaStreamSynchronize(st));
    int64_t k = 0;
    for (size_t b = 0; b < flags.size(); b++)
      if (flags[b]) {
        if (activeBlocks) activeBlocks[k] = (int)b;
        k++;
      }
    if (nActive) *nActive = k;
  }
  return msbg_gpu_sync(ctx);
}

int flip_g2p(msbg_gpu_ctx* ctx, msbg_flip_particle* particles, int64_t np, float flipAlpha,
             bool onDevice) {
  if (!ctx || (!particles && np) || np < 0) return MSBG_EINVARG;
  cudaSetDevice(ctx->device);
  FlipState* S = nullptr;
  GridF g;
  int rc = state_of(ctx, &S, g);
  if (rc) return rc;
  if (!np) return MSBG_OK;
  cudaStream_t st = ctx->stream;
  msbg_flip_particle* dp = particles;
  if (!onDevice) {
    MSBG_CUDA_TRY(ctx, S->parts.ensure(sizeof(msbg_flip_particle) * (size_t)np));
    MSBG_CUDA_TRY(ctx, cudaMemcpyAsync(S->parts.p, particles, sizeof(msbg_flip_particle) * np,
                                       cudaMemcpyHostToDevice, st));
    dp = S->parts.as<msbg_flip_particle>();
  }
  k_g2p<<<grid_blocks(np), 256, 0, st>>>(dp, np, g, S->vel.as<float>(), S->velOld.as<float>(),
                                         flipAlpha);
  MSBG_CUDA_TRY(ctx, cudaGetLastError());
  if (!onDevice)
    MSBG_CUDA_TRY(ctx, cudaMemcpyAsync(particles, dp, sizeof(msbg_flip_particle) * np,
                                       cudaMemcpyDeviceToHost, st));
  return msbg_gpu_sync(ctx);
}

}  // namespace

extern "C" int msbg_gpu_flip_p2g(msbg_gpu_ctx* ctx, const msbg_flip_particle* particles,
                                 int64_t np, const msbg_flip_params* prm, int* activeBlocks,
                                 int64_t* nActive) {
  return flip_p2g(ctx, particles, np, prm, activeBlocks, nActive, false);
}

extern "C" int msbg_gpu_flip_p2g_device(msbg_gpu_ctx* ctx, const msbg_flip_particle* particles,
                                        int64_t np, const msbg_flip_params* prm,
                                        int* activeBlocks, int64_t* nActive) {
  return flip_p2g(ctx, particles, np, prm, activeBlocks, nActive, true);
}

extern "C" int msbg_gpu_flip_gravity(msbg_gpu_ctx* ctx, float gravity, float dt, float massEps) {
  if (!ctx) return MSBG_EINVARG;
  cudaSetDevice(ctx->device);
  FlipState* S = nullptr;
  GridF g;
  int rc = state_of(ctx, &S, g);
  if (rc) return rc;
  k_gravity<<<grid_blocks(S->n), 256, 0, ctx->stream>>>(g, S->n, S->vel.as<float>(),
                                                         S->velOld.as<float>(),
                                                         S->mass.as<float>(), gravity * dt,
                                                         massEps);
  MSBG_CUDA_TRY(ctx, cudaGetLastError());
  return msbg_gpu_sync(ctx);
}

extern "C" int msbg_gpu_flip_pressure_gradient(msbg_gpu_ctx* ctx, const float* pressure,
                                               float dt, float massEps) {
  if (!ctx || !pressure) return MSBG_EINVARG;
  cudaSetDevice(ctx->device);
  FlipState* S = nullptr;
  GridF g;
  int rc = state_of(ctx, &S, g);
  if (rc) return rc;
  cudaStream_t st = ctx->stream;
  MSBG_CUDA_TRY(ctx, S->acc.ensure(sizeof(float) * (size_t)S->n));
  MSBG_CUDA_TRY(ctx, cudaMemcpyAsync(S->acc.p, pressure, sizeof(float) * S->n,
                                     cudaMemcpyHostToDevice, st));
  k_gradient<<<grid_blocks(S->n), 256, 0, st>>>(g, S->n, S->vel.as<float>(), S->mass.as<float>(),
                                                S->beta.as<float>(), S->acc.as<float>(), dt,
                                                massEps);
  MSBG_CUDA_TRY(ctx, cudaGetLastError());
  return msbg_gpu_sync(ctx);
}

extern "C" int msbg_gpu_flip_g2p(msbg_gpu_ctx* ctx, msbg_flip_particle* particles, int64_t np,
                                 float flipAlpha) {
  return flip_g2p(ctx, particles, np, flipAlpha, false);
}

extern "C" int msbg_gpu_flip_g2p_device(msbg_gpu_ctx* ctx, msbg_flip_particle* particles,
                                        int64_t np, float flipAlpha) {
  return flip_g2p(ctx, particles, np, flipAlpha, true);
}

namespace {
DeviceBuffer* flip_channel(FlipState* S, int which, int& comps) {
  comps = which == MSBG_FLIP_MASS ? 1 : 3;
  switch (which) {
    case MSBG_FLIP_VEL: return &S->vel;
    case MSBG_FLIP_VEL_OLD: return &S->velOld;
    case MSBG_FLIP_BETA: return &S->beta;
    case MSBG_FLIP_MASS: return &S->mass;
    default: return nullptr;
  }
}
}  // namespace

extern "C" int msbg_gpu_flip_channel(msbg_gpu_ctx* ctx, int which, float* data, int64_t n,
                                     int get) {
  if (!ctx || !data) return MSBG_EINVARG;
  cudaSetDevice(ctx->device);
  FlipState* S = nullptr;
  GridF g;
  int rc = state_of(ctx, &S, g);
  if (rc) return rc;
  int comps = 0;
  DeviceBuffer* b = flip_channel(S, which, comps);
  if (!b) return set_error(ctx, MSBG_EINVARG, "FLIP channel %d unknown", which);
  if (n != comps * S->n)
    return set_error(ctx, MSBG_EINVARG, "FLIP channel %d holds %lld floats, not %lld", which,
                     (long long)(comps * S->n), (long long)n);
  MSBG_CUDA_TRY(ctx, cudaMemcpyAsync(get ? (void*)data : b->p, get ? b->p : (const void*)data,
                                     sizeof(float) * n,
                                     get ? cudaMemcpyDeviceToHost : cudaMemcpyHostToDevice,
                                     ctx->stream));
  return msbg_gpu_sync(ctx);
}
