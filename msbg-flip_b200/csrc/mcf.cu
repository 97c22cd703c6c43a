// 8-colour in-place mean-curvature flow on a sparse block grid (sm_100a).
//
// Restates the GPU way what MultiresSparseGrid::applyChannelPdeFast<float>
// does for laplTyp PDE_MEAN_CURVATURE with OPT_8_COLOR_SCHEME
// (src/msbg4.cpp:348-851): per iteration, 8 colour passes; in a pass every
// block of that colour copies itself plus a 1-voxel halo (26 neighbours,
// src/halo.cpp:266-479, BC_NEUMANN src/halo.h:280-287) into on-chip memory,
// applies the 19-point curvature stencil (src/msbg4.cpp:559-637) and writes
// the result in place.  Same-colour blocks are never 26-neighbours, so one
// CTA per block and one launch per colour reproduces the reference's
// parallel pass exactly.
//
// CTA layout: one block per CTA, BSX*BSX threads, thread (x,y) owns a z
// column and keeps a 3-plane register window of the 5-point cross, so each
// voxel costs 9 shared-memory reads instead of 19.  The block and its
// 26-neighbour shell arrive in the padded (BSX+2)^3 tile by asynchronous
// 4-byte copies (cp.async), every thread's copies in flight at once; with no
// staging buffer a 16^3 block needs 23 KB and 8 CTAs fill an SM.  The
// kernel has no waits that could time out.  A listed block whose slot is not
// a value block (NULL, const, or a caller's slot map that disagrees with the
// list) is skipped and reported through errFlag (MCF_ERR_NOT_VALUE).
#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>

#include "common.cuh"

namespace msbg {
namespace {

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// 4-byte asynchronous global -> shared copy (no register round trip); the
// thread's copies complete at cp_async_wait_all.
__device__ __forceinline__ void cp_async4(float* dst, const float* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(smem_u32(dst)), "l"(src)
               : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.wait_all;" ::: "memory");
}

template <int BSX>
struct McfTile {
  static constexpr int H = BSX + 2;
  static constexpr int NV = BSX * BSX * BSX;
  static constexpr int NT = BSX * BSX;
  static constexpr int NHALO = 2 * H * H + 2 * H * (H - 2) + 2 * (H - 2) * (H - 2);
  // dynamic smem: the padded H^3 tile (23 KB for 16^3 blocks, so 8 CTAs of
  // 256 threads fit an SM)
  static constexpr size_t SMEM = sizeof(float) * H * H * H;
};

// Decode the i-th voxel of the 1-voxel shell around the block into padded
// tile coordinates (hx,hy,hz) in [0,H).
template <int H>
__device__ __forceinline__ void shell_coord(int i, int& hx, int& hy, int& hz) {
  constexpr int A = H * H, B = H * (H - 2), C = (H - 2) * (H - 2);
  if (i < 2 * A) {
    hz = (i >= A) ? H - 1 : 0;
    int r = i - ((i >= A) ? A : 0);
    hy = r / H;
    hx = r - hy * H;
  } else if (i < 2 * A + 2 * B) {
    int j = i - 2 * A;
    hy = (j >= B) ? H - 1 : 0;
    int r = j - ((j >= B) ? B : 0);
    hz = 1 + r / H;
    hx = r - (hz - 1) * H;
  } else {
    int k = i - 2 * A - 2 * B;
    hx = (k >= C) ? H - 1 : 0;
    int r = k - ((k >= C) ? C : 0);
    hz = 1 + r / (H - 2);
    hy = 1 + (r - (hz - 1) * (H - 2));
  }
}

template <int BSX>
__global__ void __launch_bounds__(BSX* BSX)
    mcf_colour_kernel(float* __restrict__ pool, const int* __restrict__ slotOf,
                      const int* __restrict__ list, int nbx, int nby, int nbz,
                      float emptyVal, float fullVal, float dt, int clamp01,
                      int* __restrict__ errFlag) {
  using T = McfTile<BSX>;
  constexpr int H = T::H, H2 = H * H, NV = T::NV, NT = T::NT;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  float* tile = reinterpret_cast<float*>(smem_raw);
  __shared__ int nbSlot[27];

  const int tid = threadIdx.x;
  const int bid = list[blockIdx.x];
  const int bx = bid % nbx, by = (bid / nbx) % nby, bz = bid / (nbx * nby);
  const int slot0 = slotOf[bid];
  if (slot0 < 0) {  // uniform per CTA, before any barrier or copy
    if (tid == 0) atomicOr(errFlag, MCF_ERR_NOT_VALUE);
    return;
  }
  const float* own = pool + (size_t)slot0 * NV;

  if (tid < 27) {
    int dx = tid % 3 - 1, dy = (tid / 3) % 3 - 1, dz = tid / 9 - 1;
    int x = bx + dx, y = by + dy, z = bz + dz;
    int s = SLOT_OUT;
    if (x >= 0 && y >= 0 && z >= 0 && x < nbx && y < nby && z < nbz)
      s = slotOf[x + nbx * (y + nby * z)];
    nbSlot[tid] = s;
  }
  __syncthreads();
  // The interior: one asynchronous 4-byte copy per voxel straight into the
  // padded tile (consecutive threads, consecutive voxels).
  for (int e = tid; e < NV; e += NT) {
    const int x = e % BSX, y = (e / BSX) % BSX, z = e / (BSX * BSX);
    cp_async4(tile + (x + 1) + H * (y + 1) + H2 * (z + 1), own + e);
  }

  // Gather the 26 neighbour pieces straight into the padded tile: voxels of
  // stored blocks by asynchronous copies (all of a thread's copies in flight
  // at once), constant blocks by plain stores.
  for (int i = tid; i < T::NHALO; i += NT) {
    int hx, hy, hz;
    shell_coord<H>(i, hx, hy, hz);
    int x = hx - 1, y = hy - 1, z = hz - 1;
    int dx = x < 0 ? -1 : (x >= BSX ? 1 : 0);
    int dy = y < 0 ? -1 : (y >= BSX ? 1 : 0);
    int dz = z < 0 ? -1 : (z >= BSX ? 1 : 0);
    int s = nbSlot[(dz + 1) * 9 + (dy + 1) * 3 + (dx + 1)];
    float* d = tile + hx + H * hy + H2 * hz;
    if (s >= 0) {
      cp_async4(d, pool + (size_t)s * NV + ((x & (BSX - 1)) + BSX * ((y & (BSX - 1)) + BSX * (z & (BSX - 1)))));
    } else if (s == SLOT_EMPTY) {
      *d = emptyVal;
    } else if (s == SLOT_FULL) {
      *d = fullVal;
    } else {  // NULL block or outside the domain: Neumann, own value clamped
      int cx = min(max(x, 0), BSX - 1), cy = min(max(y, 0), BSX - 1), cz = min(max(z, 0), BSX - 1);
      cp_async4(d, own + (cx + BSX * (cy + BSX * cz)));
    }
  }
  cp_async_wait_all();

  __syncthreads();  // every thread's copies have landed (waited above)

  // Column sweep with a 3-plane register window of the 5-point cross.
  const int x = tid % BSX, y = tid / BSX;
  const float* col = tile + (x + 1) + H * (y + 1);
  float* out = pool + (size_t)slot0 * NV + x + BSX * y;
  float cm = col[0], xmm = col[-1], xpm = col[1], ymm = col[-H], ypm = col[H];            // z-1
  float c0 = col[H2], xm0 = col[H2 - 1], xp0 = col[H2 + 1], ym0 = col[H2 - H], yp0 = col[H2 + H];  // z
#pragma unroll
  for (int z = 0; z < BSX; z++) {
    const float* p1 = col + H2 * (z + 2);
    float cp = p1[0], xmp = p1[-1], xpp = p1[1], ymp = p1[-H], ypp = p1[H];  // z+1
    const float* p0 = col + H2 * (z + 1);
    float fpp = p0[1 + H], fpm = p0[1 - H], fmp = p0[-1 + H], fmm = p0[-1 - H];

    float f0 = c0, f1 = xm0, f2 = xp0, f3 = ym0, f4 = yp0, f5 = cm, f6 = cp;
    float fx = 0.5f * (f2 - f1), fy = 0.5f * (f4 - f3), fz = 0.5f * (f6 - f5);
    float fxx = f1 + f2 - 2.f * f0, fyy = f3 + f4 - 2.f * f0, fzz = f5 + f6 - 2.f * f0;
    float fy_right = (fpp - fpm) * 0.5f, fy_left = (fmp - fmm) * 0.5f;
    float fz_right = (xpp - xpm) * 0.5f, fz_left = (xmp - xmm) * 0.5f;
    float fz_up = (ypp - ypm) * 0.5f, fz_down = (ymp - ymm) * 0.5f;
    float fyx = (fy_right - fy_left) * 0.5f;
    float fzx = (fz_right - fz_left) * 0.5f;
    float fzy = (fz_up - fz_down) * 0.5f;
    float fx2 = fx * fx, fy2 = fy * fy, fz2 = fz * fz;
    float H_ = (fy2 + fz2) * fxx + (fx2 + fz2) * fyy + (fx2 + fy2) * fzz -
               2.0f * (fx * fy * fyx + fx * fz * fzx + fy * fz * fzy);
    float g = fx2 + fy2 + fz2;
    H_ = g > 1e-7f ? __fdividef(H_, g) : 0.0f;
    float D = fminf(fmaxf(dt * H_, -0.1f), 0.1f);
    float phi = f0 + D;
    if (clamp01) phi = fminf(fmaxf(phi, 0.0f), 1.0f);
    out[BSX * BSX * z] = phi;

    cm = c0; xmm = xm0; xpm = xp0; ymm = ym0; ypm = yp0;
    c0 = cp; xm0 = xmp; xp0 = xpp; ym0 = ymp; yp0 = ypp;
  }
}

template <int BSX>
cudaError_t launch_mcf_t(float* pool, const int* slotOf, const int* colourList,
                         const int* colourStart, int nbx, int nby, int nbz,
                         float emptyVal, float fullVal, int nIter, float dt,
                         int clamp01, int* errFlag, cudaStream_t stream) {
  using T = McfTile<BSX>;
  // The shared-memory limit is an attribute of the kernel on each device:
  // set it once per device (bit per device; a race only repeats the call).
  static std::atomic<uint64_t> attrSet{0};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  const uint64_t bit = dev < 64 ? (uint64_t)1 << dev : 0;
  if (!bit || !(attrSet.load(std::memory_order_acquire) & bit)) {
    e = cudaFuncSetAttribute(mcf_colour_kernel<BSX>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)T::SMEM);
    if (e != cudaSuccess) return e;
    attrSet.fetch_or(bit, std::memory_order_acq_rel);
  }
  for (int it = 0; it < nIter; it++)
    for (int c = 0; c < 8; c++) {
      int n = colourStart[c + 1] - colourStart[c];
      if (n <= 0) continue;
      mcf_colour_kernel<BSX><<<n, T::NT, T::SMEM, stream>>>(
          pool, slotOf, colourList + colourStart[c], nbx, nby, nbz, emptyVal, fullVal, dt,
          clamp01, errFlag);
    }
  return cudaGetLastError();
}

}  // namespace

cudaError_t launch_mcf(float* pool, const int* slotOf, const int* colourList,
                       const int* colourStart, int nbx, int nby, int nbz, int bsx,
                       float emptyVal, float fullVal, int nIter, float dt, int clamp01,
                       int* errFlag, cudaStream_t stream) {
  switch (bsx) {
    case 8:
      return launch_mcf_t<8>(pool, slotOf, colourList, colourStart, nbx, nby, nbz, emptyVal,
                             fullVal, nIter, dt, clamp01, errFlag, stream);
    case 16:
      return launch_mcf_t<16>(pool, slotOf, colourList, colourStart, nbx, nby, nbz, emptyVal,
                              fullVal, nIter, dt, clamp01, errFlag, stream);
    case 32:
      return launch_mcf_t<32>(pool, slotOf, colourList, colourStart, nbx, nby, nbz, emptyVal,
                              fullVal, nIter, dt, clamp01, errFlag, stream);
    default:
      return cudaErrorInvalidValue;
  }
}

}  // namespace msbg
