// 8-colour in-place mean-curvature flow on a sparse block grid (sm_100a).
//
// Restates the GPU way what MultiresSparseGrid::applyChannelPdeFast<float>
// does for laplTyp PDE_MEAN_CURVATURE with OPT_8_COLOR_SCHEME
// (src/msbg4.cpp:348-851): per iteration, 8 colour passes; in a pass every
// block of that colour copies itself plus a 1-voxel halo (src/halo.cpp:266-479,
// BC_NEUMANN src/halo.h:280-287) into on-chip memory, applies the 19-point
// curvature stencil (src/msbg4.cpp:559-637) and writes the result in place.
// Same-colour blocks are never 26-neighbours, so one CTA per block and one
// launch per colour reproduces the reference's parallel pass exactly.
//
// The stencil is issue-bound (about 60 FP32 operations and 9 shared-memory
// reads per voxel against 8 bytes of HBM traffic), so the kernel works on
// pairs of x-adjacent voxels with the packed FP32 instructions of sm_100
// (add/sub/mul/fma.rn.f32x2): one instruction updates both voxels of a pair,
// and a pair arrives from shared memory in one 8-byte load.
//   * CTA layout: BSX*BSX threads per block; thread (i, y, h) owns the x pair
//     (2i, 2i+1) of row y and marches up one half h of z with a three-plane
//     register window of the 5-point cross.
//   * The padded tile holds x in [-2, BSX+1] (row pitch BSX+4, so every pair
//     starts on an 8-byte boundary) and y, z in [-1, BSX].  The x-1 and x+1
//     pairs are rebuilt in registers from three aligned pairs.
//   * The block and its 1-voxel shell (faces and edges; the 19-point stencil
//     reads no corner) arrive by asynchronous copies straight into the tile:
//     for FP32 16^3 blocks of a context channel the block is one tensor box
//     (cp.async.bulk.tensor, mcf_colour_kernel_tma), otherwise 8-byte copies
//     for x pairs; 4-byte copies for the x faces.
//   * The curvature is evaluated with the central differences left unscaled:
//     with d = f(+1) - f(-1) (= 2 f_x) and s = the mixed second difference
//     (= 4 f_xy) the reference's H = [...] / |grad f|^2 becomes
//     (N1 - N2/2) / G, G = |d|^2, with the threshold |grad f|^2 > 1e-7 read as
//     G > 4e-7: every rescaling is by a power of two and so exact.
// Channels are FP32 or the reference's 16-bit render density (RSURF_16_BIT,
// src/msbgcell.h:67-68): q in [0, 65535] read as q * (1/65535) and stored as
// round(phi * 65535) (src/sbg.h:225-232, 360-368; src/msbg4.cpp:829-839).
// 16-bit blocks arrive through ordinary loads and are widened into the
// FP32 tile.
// A listed block whose slot is not a value block (NULL, const, or a caller's
// slot map that disagrees with the list) is skipped and reported through
// errFlag (MCF_ERR_NOT_VALUE).  The kernel has no waits that could time out.
#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <atomic>
#include <cstdint>
#include <type_traits>

#include "common.cuh"

namespace msbg {
namespace {

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Asynchronous global -> shared copies (no register round trip); a thread's
// copies complete at cp_async_wait_all.
__device__ __forceinline__ void cp_async4(float* dst, const float* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(smem_u32(dst)), "l"(src)
               : "memory");
}
__device__ __forceinline__ void cp_async8(float* dst, const float* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_u32(dst)), "l"(src)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;" ::: "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait_group() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// A pair of FP32 values in one 64-bit register and the packed arithmetic.
typedef unsigned long long f2;
__device__ __forceinline__ f2 pk(float lo, float hi) {
  f2 r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
  return r;
}
__device__ __forceinline__ void upk(f2 v, float& lo, float& hi) {
  asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
}
__device__ __forceinline__ f2 add2(f2 a, f2 b) {
  f2 r;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}
__device__ __forceinline__ f2 sub2(f2 a, f2 b) {
  f2 r;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}
__device__ __forceinline__ f2 mul2(f2 a, f2 b) {
  f2 r;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}
__device__ __forceinline__ f2 fma2(f2 a, f2 b, f2 c) {
  f2 r;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(a), "l"(b), "l"(c));
  return r;
}
__device__ __forceinline__ f2 ld2(const float* p) {
  return *reinterpret_cast<const f2*>(p);
}
// (hi of a, lo of b): the pair shifted by one voxel
__device__ __forceinline__ f2 mid2(f2 a, f2 b) {
  float a0, a1, b0, b1;
  upk(a, a0, a1);
  upk(b, b0, b1);
  return pk(a1, b0);
}

// The padded tile: x in [-XOFF, BSX + XOFF) (row pitch BSX + 2 XOFF, so every
// x pair starts on an 8-byte boundary), y and z in [-1, BSX].  XOFF = 2 for
// the copies issued by threads; XOFF = 4 when the block arrives as one tensor
// box, whose x origin must sit on a 16-byte boundary (x = -4).
template <int BSX, int XOFF = 2>
struct McfTile {
  static constexpr int RP = BSX + 2 * XOFF;  // row pitch
  static constexpr int PP = RP * (BSX + 2);  // plane pitch: y + 1 in [0, BSX + 2)
  static constexpr int NV = BSX * BSX * BSX;
  static constexpr int NT = BSX * BSX;       // one thread per x pair of a row and z half
  static constexpr int HP = BSX / 2;         // pairs per row
  static constexpr size_t SMEM = sizeof(float) * PP * (BSX + 2);
  __host__ __device__ static constexpr int at(int x, int y, int z) {
    return (x + XOFF) + RP * (y + 1) + PP * (z + 1);
  }
};

// Where halo voxel (x, y, z) (block coordinates, some outside [0, BSX)) comes
// from: a neighbour value block, a const block, or the own block clamped to
// its boundary (BC_NEUMANN for NULL neighbours and the domain boundary).
template <int BSX, typename T>
__device__ __forceinline__ const T* halo_src(const T* pool, const int* nbSlot, const T* own,
                                             int x, int y, int z, int& constKind) {
  constexpr int M = BSX - 1;
  const int dx = x < 0 ? -1 : (x > M ? 1 : 0);
  const int dy = y < 0 ? -1 : (y > M ? 1 : 0);
  const int dz = z < 0 ? -1 : (z > M ? 1 : 0);
  const int s = nbSlot[(dz + 1) * 9 + (dy + 1) * 3 + (dx + 1)];
  constKind = 0;
  if (s >= 0)
    return pool + (size_t)s * (BSX * BSX * BSX) + ((x & M) + BSX * ((y & M) + BSX * (z & M)));
  if (s == SLOT_EMPTY || s == SLOT_FULL) {
    constKind = s == SLOT_EMPTY ? 1 : 2;
    return nullptr;
  }
  const int cx = min(max(x, 0), M), cy = min(max(y, 0), M), cz = min(max(z, 0), M);
  return own + (cx + BSX * (cy + BSX * cz));
}

constexpr float U16_SCALE = 1.0f / 65535.0f;  // RENDER_DENS_TO_FLOAT_UI16

// Issue the copies of one block and its shell into a tile (FP32: asynchronous
// copies, completed by the caller's cp.async wait; 16-bit: loads widened into
// the tile on the spot).  nbSlot: the slots of the 27 blocks around it.
// The x faces of a block's neighbours: with a face cache xf (per slot the
// planes x = 0 and x = BSX-1 as [2][z][y], kept current by the kernel), one
// contiguous 4-byte value per halo voxel; without it, a 4-byte value out of
// a 64-byte row of the neighbour block.
template <int BSX, typename T>
__device__ __forceinline__ const T* xface_src(const T* pool, const T* xf, const int* nbSlot,
                                              int x, int y, int z, int& constKind) {
  if (!xf) {
    const T* own = pool + (size_t)nbSlot[13] * (BSX * BSX * BSX);
    return halo_src<BSX, T>(pool, nbSlot, own, x, y, z, constKind);
  }
  constexpr int M = BSX - 1, F = BSX * BSX;
  const int dx = x < 0 ? -1 : 1;
  const int dy = y < 0 ? -1 : (y > M ? 1 : 0);
  const int dz = z < 0 ? -1 : (z > M ? 1 : 0);
  const int s = nbSlot[(dz + 1) * 9 + (dy + 1) * 3 + (dx + 1)];
  constKind = 0;
  if (s >= 0)  // the neighbour's plane that faces us: x = BSX-1 for dx < 0
    return xf + ((size_t)s * 2 + (dx < 0 ? 1 : 0)) * F + (z & M) * BSX + (y & M);
  if (s == SLOT_EMPTY || s == SLOT_FULL) {
    constKind = s == SLOT_EMPTY ? 1 : 2;
    return nullptr;
  }
  // NULL neighbour or outside the domain: our own boundary plane, clamped
  const int cy = min(max(y, 0), M), cz = min(max(z, 0), M);
  return xf + ((size_t)nbSlot[13] * 2 + (dx < 0 ? 0 : 1)) * F + cz * BSX + cy;
}

template <int BSX, typename T>
__device__ __forceinline__ void mcf_fill(float* tile, const T* __restrict__ pool,
                                         const T* __restrict__ xf, const int* nbSlot,
                                         float emptyVal, float fullVal, int tid) {
  using Tl = McfTile<BSX>;
  constexpr int NV = Tl::NV, NT = Tl::NT, HP = Tl::HP;
  constexpr bool F32 = std::is_same<T, float>::value;
  const T* own = pool + (size_t)nbSlot[13] * NV;
  // interior: one x pair per copy (8-byte asynchronous copies for FP32; for
  // 16-bit values one 4-byte load, widened into the tile)
#pragma unroll 8
  for (int p = tid; p < NV / 2; p += NT) {
    const int e = 2 * p;
    const int x = e % BSX, y = (e / BSX) % BSX, z = e / (BSX * BSX);
    float* d = tile + Tl::at(x, y, z);
    if constexpr (F32) {
      cp_async8(d, own + e);
    } else {
      const uint32_t v = *reinterpret_cast<const uint32_t*>(own + e);
      *reinterpret_cast<float2*>(d) =
          make_float2((float)(v & 0xffffu) * U16_SCALE, (float)(v >> 16) * U16_SCALE);
    }
  }
  // shell voxels with x inside the block (z faces, y faces, x-direction
  // edges): the ring of (y, z) around the block, one x pair each
  constexpr int RING = 4 * BSX + 4;
  for (int q = tid; q < RING * HP; q += NT) {
    const int r = q / HP, x = 2 * (q % HP);
    int y, z;
    if (r < 2 * (BSX + 2)) {  // z = -1 and z = BSX, y in [-1, BSX]
      z = r < BSX + 2 ? -1 : BSX;
      y = (r % (BSX + 2)) - 1;
    } else {  // y = -1 and y = BSX, z in [0, BSX)
      const int r2 = r - 2 * (BSX + 2);
      y = r2 < BSX ? -1 : BSX;
      z = r2 % BSX;
    }
    int ck;
    const T* src = halo_src<BSX, T>(pool, nbSlot, own, x, y, z, ck);
    float* d = tile + Tl::at(x, y, z);
    if (src) {
      if constexpr (F32) {
        cp_async8(d, src);
      } else {
        const uint32_t v = *reinterpret_cast<const uint32_t*>(src);
        d[0] = (float)(v & 0xffffu) * U16_SCALE;
        d[1] = (float)(v >> 16) * U16_SCALE;
      }
    } else {
      const float v = ck == 1 ? emptyVal : fullVal;
      d[0] = v;
      d[1] = v;
    }
  }
  // shell voxels with x = -1 or x = BSX (x faces, y- and z-direction edges):
  // (y, z) in [-1, BSX]^2 without the four corners, one voxel each
  constexpr int SIDE = (BSX + 2) * (BSX + 2);
  for (int q = tid; q < 2 * SIDE; q += NT) {
    const int side = q / SIDE, r = q % SIDE;
    const int y = r % (BSX + 2) - 1, z = r / (BSX + 2) - 1;
    if ((y < 0 || y >= BSX) && (z < 0 || z >= BSX)) continue;  // corner: not read
    const int x = side ? BSX : -1;
    int ck;
    const T* src = xface_src<BSX, T>(pool, xf, nbSlot, x, y, z, ck);
    float* d = tile + Tl::at(x, y, z);
    if (src) {
      if constexpr (F32)
        cp_async4(d, src);
      else
        *d = (float)(*src) * U16_SCALE;
    } else {
      *d = ck == 1 ? emptyVal : fullVal;
    }
  }
}

// The 19-point update of one block from its tile, stored in place.
template <int BSX, typename T, int XOFF = 2>
__device__ __forceinline__ void mcf_compute(const float* tile, T* __restrict__ block,
                                            T* __restrict__ xfOwn, float dt, int clamp01,
                                            int tid) {
  using Tl = McfTile<BSX, XOFF>;
  constexpr int RP = Tl::RP, PP = Tl::PP, HP = Tl::HP;
  // Column march of the x pair (x0, x0 + 1) of row y over one half of z.
  constexpr int ZN = BSX / 2;
  const int x0 = 2 * (tid % HP), y = (tid / HP) % BSX, zb = ZN * (tid / (HP * BSX));
  const float* col = tile + Tl::at(x0, y, zb - 1);  // plane zb - 1
  T* out = block + x0 + BSX * y + BSX * BSX * zb;
  const f2 m2 = pk(-2.f, -2.f), mh = pk(-0.5f, -0.5f);
  // window: centre, x-1, x+1 pairs of row y; centre pairs of rows y-1, y+1
  f2 Cm, XMm, XPm, YMm, YPm;  // plane z-1
  f2 C0, XM0, XP0, YM0, YP0;  // plane z
  {
    const float* p = col;
    const f2 a = ld2(p - 2), b = ld2(p), c = ld2(p + 2);
    Cm = b; XMm = mid2(a, b); XPm = mid2(b, c);
    YMm = ld2(p - RP); YPm = ld2(p + RP);
    p += PP;
    const f2 a1 = ld2(p - 2), b1 = ld2(p), c1 = ld2(p + 2);
    C0 = b1; XM0 = mid2(a1, b1); XP0 = mid2(b1, c1);
    YM0 = ld2(p - RP); YP0 = ld2(p + RP);
  }
#pragma unroll 4
  for (int z = 0; z < ZN; z++) {
    const float* p0 = col + PP * (z + 1);  // plane zb + z
    const float* p1 = p0 + PP;             // plane z+1
    const f2 a = ld2(p1 - 2), b = ld2(p1), c = ld2(p1 + 2);
    const f2 Cp = b, XMp = mid2(a, b), XPp = mid2(b, c);
    const f2 YMp = ld2(p1 - RP), YPp = ld2(p1 + RP);
    // x-1 and x+1 pairs of rows y-1 and y+1 in plane z (the xy diagonals)
    const f2 XMYM = mid2(ld2(p0 - RP - 2), YM0), XPYM = mid2(YM0, ld2(p0 - RP + 2));
    const f2 XMYP = mid2(ld2(p0 + RP - 2), YP0), XPYP = mid2(YP0, ld2(p0 + RP + 2));

    const f2 dx = sub2(XP0, XM0), dy = sub2(YP0, YM0), dz = sub2(Cp, Cm);  // 2 f_x ...
    const f2 fxx = fma2(m2, C0, add2(XM0, XP0));
    const f2 fyy = fma2(m2, C0, add2(YM0, YP0));
    const f2 fzz = fma2(m2, C0, add2(Cm, Cp));
    const f2 sxy = sub2(sub2(XPYP, XPYM), sub2(XMYP, XMYM));  // 4 f_xy
    const f2 sxz = sub2(sub2(XPp, XPm), sub2(XMp, XMm));      // 4 f_xz
    const f2 syz = sub2(sub2(YPp, YPm), sub2(YMp, YMm));      // 4 f_yz
    const f2 dx2 = mul2(dx, dx), dy2 = mul2(dy, dy), dz2 = mul2(dz, dz);
    f2 n1 = mul2(add2(dy2, dz2), fxx);
    n1 = fma2(add2(dx2, dz2), fyy, n1);
    n1 = fma2(add2(dx2, dy2), fzz, n1);
    f2 n2 = mul2(mul2(dx, dy), sxy);
    n2 = fma2(mul2(dx, dz), sxz, n2);
    n2 = fma2(mul2(dy, dz), syz, n2);
    const f2 num = fma2(mh, n2, n1);
    const f2 G = add2(add2(dx2, dy2), dz2);
    float nl, nh, gl, gh, fl, fh;
    upk(num, nl, nh);
    upk(G, gl, gh);
    upk(C0, fl, fh);
    constexpr float GMIN = 4.0f * 1e-7f;  // |grad f|^2 > 1e-7 with d = 2 grad f
    const float hl = gl > GMIN ? __fdividef(nl, gl) : 0.0f;
    const float hh = gh > GMIN ? __fdividef(nh, gh) : 0.0f;
    float pl = fl + fminf(fmaxf(dt * hl, -0.1f), 0.1f);
    float ph = fh + fminf(fmaxf(dt * hh, -0.1f), 0.1f);
    if (clamp01) {
      pl = fminf(fmaxf(pl, 0.0f), 1.0f);
      ph = fminf(fmaxf(ph, 0.0f), 1.0f);
    }
    T vl, vh;
    if constexpr (std::is_same<T, float>::value) {
      vl = pl;
      vh = ph;
      *reinterpret_cast<float2*>(out + BSX * BSX * z) = make_float2(pl, ph);
    } else {  // round to nearest (even), as round_to_int under the default MXCSR
      const uint32_t ql = (uint32_t)min(max(__float2int_rn(pl * 65535.0f), 0), 65535);
      const uint32_t qh = (uint32_t)min(max(__float2int_rn(ph * 65535.0f), 0), 65535);
      vl = (T)ql;
      vh = (T)qh;
      *reinterpret_cast<uint32_t*>(out + BSX * BSX * z) = ql | (qh << 16);
    }
    if (xfOwn) {  // keep the face cache of this block current
      if (x0 == 0) xfOwn[(zb + z) * BSX + y] = vl;
      if (x0 + 1 == BSX - 1) xfOwn[BSX * BSX + (zb + z) * BSX + y] = vh;
    }

    Cm = C0; XMm = XM0; XPm = XP0; YMm = YM0; YPm = YP0;
    C0 = Cp; XM0 = XMp; XP0 = XPp; YM0 = YMp; YP0 = YPp;
  }
}

// Tile stages per CTA: two (the next block's copies in flight while this one
// is computed) where two tiles fit next to the other CTAs of an SM, one for
// 32^3 blocks (a 166 KB tile).
template <int BSX>
__host__ __device__ constexpr int mcf_stages() { return BSX <= 16 ? 2 : 1; }
// CTAs per SM the launch plans for (persistent grid = SMs x this), chosen so
// that the column march keeps its window in registers without spilling: for
// 16^3 blocks three CTAs of 256 threads (85 registers per thread; measured 6 %
// faster than four CTAs at 64 registers with spills), for 8^3 blocks twelve
// of 64.
template <int BSX>
__host__ __device__ constexpr int mcf_ctas_per_sm() { return BSX == 8 ? 12 : BSX == 16 ? 3 : 1; }

// One colour pass: the CTAs walk the pass's block list with a stride of
// gridDim.x; with two stages the copies of block k + gridDim.x are issued
// before block k is computed.
template <int BSX, typename T>
__global__ void __launch_bounds__(BSX* BSX, mcf_ctas_per_sm<BSX>())
    mcf_colour_kernel(T* __restrict__ pool, T* __restrict__ xf, const int* __restrict__ slotOf,
                      const int* __restrict__ list, int n, int nbx, int nby, int nbz,
                      float emptyVal, float fullVal, float dt, int clamp01,
                      int* __restrict__ errFlag) {
  using Tl = McfTile<BSX>;
  constexpr int ST = mcf_stages<BSX>();
  constexpr int TILE = Tl::PP * (BSX + 2);
  extern __shared__ __align__(128) unsigned char smem_raw[];
  float* tiles = reinterpret_cast<float*>(smem_raw);
  __shared__ int nbSlot[2][27];
  const int tid = threadIdx.x;
  const int G = gridDim.x;
  int k = blockIdx.x;
  if (k >= n) return;
  // the slots of the 27 blocks around list[kk] into nbSlot[s]
  auto neighbours = [&](int kk, int s) {
    if (tid < 27) {
      const int bid = list[kk];
      const int bx = bid % nbx, by = (bid / nbx) % nby, bz = bid / (nbx * nby);
      const int dx = tid % 3 - 1, dy = (tid / 3) % 3 - 1, dz = tid / 9 - 1;
      const int x = bx + dx, y = by + dy, z = bz + dz;
      int sl = SLOT_OUT;
      if (x >= 0 && y >= 0 && z >= 0 && x < nbx && y < nby && z < nbz)
        sl = slotOf[x + nbx * (y + nby * z)];
      nbSlot[s][tid] = sl;
    }
  };
  // a listed block whose own slot is not a value block is skipped (uniform
  // per CTA: every thread reads the same shared slot)
  auto fill = [&](int s) {
    if (nbSlot[s][13] >= 0)
      mcf_fill<BSX, T>(tiles + s * TILE, pool, xf, nbSlot[s], emptyVal, fullVal, tid);
    cp_async_commit();
  };
  neighbours(k, 0);
  __syncthreads();
  fill(0);
  for (int it = 0; k < n; it++, k += G) {
    const int s = ST == 2 ? (it & 1) : 0;
    const int kn = k + G;
    if (ST == 2) {
      if (kn < n) neighbours(kn, s ^ 1);
      __syncthreads();  // nbSlot[s^1] written; stage s^1 is free since the last pass
      if (kn < n) fill(s ^ 1);
      else cp_async_commit();
      cp_async_wait_group<1>();  // block k's copies have landed (the newest may fly)
    } else {
      cp_async_wait_group<0>();
    }
    __syncthreads();
    const int slot0 = nbSlot[s][13];
    if (slot0 < 0) {
      if (tid == 0) atomicOr(errFlag, MCF_ERR_NOT_VALUE);
    } else {
      mcf_compute<BSX, T>(tiles + s * TILE, pool + (size_t)slot0 * Tl::NV,
                          xf ? xf + (size_t)slot0 * 2 * BSX * BSX : nullptr, dt, clamp01, tid);
    }
    __syncthreads();  // stage s may be refilled
    if (ST == 1 && kn < n) {
      neighbours(kn, 0);
      __syncthreads();
      fill(0);
    }
  }
}

// ---------------------------------------------------------------------------
// FP32 16^3 blocks of a context pool: the block arrives as one tensor box
// ---------------------------------------------------------------------------
// The pool is a 4-D tensor (x, y, z, slot) of 16^3 FP32 blocks.  One box of
// 24 x 18 x 16 voxels at (-4, -1, 0, slot) lands as planes 1..16 of the padded
// tile (XOFF = 4: row pitch 24, plane pitch 432), x and y outside the block
// filled with zeros by the copy.  What the stencil reads there - the x faces,
// the y faces and the four edges along z - is loaded into registers while the
// previous block is computed and stored once the box has landed; the z = -1
// and z = 16 planes (faces and the edges in them) arrive by 8- and 4-byte
// asynchronous copies, which no box overlaps.  One mbarrier per tile stage
// counts the box's bytes; its waits are bounded.
namespace tma {

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}
__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}
// Bounded wait on the given phase parity; false if the copy never landed.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  uint32_t done = 0;
  for (int i = 0; i < (1 << 24); i++) {
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}
// One box of the 4-D tensor map into shared memory (no multicast).
__device__ __forceinline__ void box_g2s(void* dst, const CUtensorMap* map, int x, int y, int z,
                                        int w, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(w), "r"(smem_u32(bar))
      : "memory");
}

constexpr int BS = 16, XO = 4;
using Tl = McfTile<BS, XO>;
constexpr int TILE = Tl::PP * (BS + 2);                      // floats per stage
constexpr uint32_t BOX_BYTES = sizeof(float) * Tl::RP * (BS + 2) * BS;
// the box lands at plane 1 of a stage: the stages start where that plane is
// 128-byte aligned (TILE floats keep the second stage aligned too)
static_assert((TILE * 4) % 128 == 0 && (Tl::PP * 4) % 16 == 0, "stage alignment");
constexpr size_t SMEM = 2 * sizeof(float) * TILE + 128;

// Register-staged halo of one block: thread t holds one y-face pair, two
// x-face values and (t < 64) one edge along z.
struct Halo {
  float y0, y1, x0, x1, e;
};

__device__ __forceinline__ float const_val(int ck, float emptyVal, float fullVal) {
  return ck == 1 ? emptyVal : fullVal;
}

__device__ __forceinline__ void halo_load(Halo& h, const float* __restrict__ pool,
                                          const float* __restrict__ xf, const int* nbSlot,
                                          float emptyVal, float fullVal, int tid) {
  const float* own = pool + (size_t)nbSlot[13] * Tl::NV;
  {  // y faces: y = -1 / 16, z in [0, 16), one x pair
    const int side = tid >> 7, r = tid & 127, z = r >> 3, x = 2 * (r & 7);
    int ck;
    const float* src = halo_src<BS, float>(pool, nbSlot, own, x, side ? BS : -1, z, ck);
    if (src) {
      const float2 v = *reinterpret_cast<const float2*>(src);
      h.y0 = v.x;
      h.y1 = v.y;
    } else {
      h.y0 = h.y1 = const_val(ck, emptyVal, fullVal);
    }
  }
#pragma unroll
  for (int q = 0; q < 2; q++) {  // x faces: x = -1 / 16, (y, z) in [0, 16)^2
    const int g = tid + 256 * q, side = g >> 8, y = g & 15, z = (g >> 4) & 15;
    int ck;
    const float* src = xface_src<BS, float>(pool, xf, nbSlot, side ? BS : -1, y, z, ck);
    const float v = src ? *src : const_val(ck, emptyVal, fullVal);
    if (q == 0) h.x0 = v; else h.x1 = v;
  }
  if (tid < 64) {  // edges along z: (x, y) in {-1, 16}^2
    const int c = tid >> 4, z = tid & 15;
    const int x = (c & 1) ? BS : -1, y = (c & 2) ? BS : -1;
    int ck;
    const float* src = halo_src<BS, float>(pool, nbSlot, own, x, y, z, ck);
    h.e = src ? *src : const_val(ck, emptyVal, fullVal);
  }
}

__device__ __forceinline__ void halo_store(const Halo& h, float* tile, int tid) {
  {
    const int side = tid >> 7, r = tid & 127, z = r >> 3, x = 2 * (r & 7);
    float* d = tile + Tl::at(x, side ? BS : -1, z);
    *reinterpret_cast<float2*>(d) = make_float2(h.y0, h.y1);
  }
#pragma unroll
  for (int q = 0; q < 2; q++) {
    const int g = tid + 256 * q, side = g >> 8, y = g & 15, z = (g >> 4) & 15;
    tile[Tl::at(side ? BS : -1, y, z)] = q == 0 ? h.x0 : h.x1;
  }
  if (tid < 64) {
    const int c = tid >> 4, z = tid & 15;
    tile[Tl::at((c & 1) ? BS : -1, (c & 2) ? BS : -1, z)] = h.e;
  }
}

// The z = -1 and z = 16 planes: faces (x pairs, y in [-1, 16]) and the edges
// along y (x = -1 / 16, y in [0, 16)), by asynchronous copies.
__device__ __forceinline__ void zplanes_fill(float* tile, const float* __restrict__ pool,
                                             const float* __restrict__ xf, const int* nbSlot,
                                             float emptyVal, float fullVal, int tid) {
  const float* own = pool + (size_t)nbSlot[13] * Tl::NV;
  constexpr int ROWS = BS + 2, PAIRS = 2 * ROWS * (BS / 2);  // 288
  for (int q = tid; q < PAIRS; q += Tl::NT) {
    const int side = q / (ROWS * (BS / 2)), r = q % (ROWS * (BS / 2));
    const int y = r / (BS / 2) - 1, x = 2 * (r % (BS / 2)), z = side ? BS : -1;
    int ck;
    const float* src = halo_src<BS, float>(pool, nbSlot, own, x, y, z, ck);
    float* d = tile + Tl::at(x, y, z);
    if (src) {
      cp_async8(d, src);
    } else {
      const float v = const_val(ck, emptyVal, fullVal);
      d[0] = v;
      d[1] = v;
    }
  }
  if (tid < 64) {
    const int side = tid >> 5, xs = (tid >> 4) & 1, y = tid & 15;
    const int z = side ? BS : -1, x = xs ? BS : -1;
    int ck;
    const float* src = xface_src<BS, float>(pool, xf, nbSlot, x, y, z, ck);
    float* d = tile + Tl::at(x, y, z);
    if (src)
      cp_async4(d, src);
    else
      *d = const_val(ck, emptyVal, fullVal);
  }
}

}  // namespace tma

__global__ void __launch_bounds__(256, 3)
    mcf_colour_kernel_tma(const __grid_constant__ CUtensorMap map, float* __restrict__ pool,
                          float* __restrict__ xf, const int* __restrict__ slotOf,
                          const int* __restrict__ list, int n, int nbx, int nby, int nbz,
                          float emptyVal, float fullVal, float dt, int clamp01,
                          int* __restrict__ errFlag) {
  using namespace tma;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  const uint32_t pad = (128u - ((smem_u32(smem_raw) + Tl::PP * 4u) & 127u)) & 127u;
  float* tiles = reinterpret_cast<float*>(smem_raw + pad);
  __shared__ int nbSlot[2][27];
  __shared__ __align__(8) uint64_t bar[2];
  const int tid = threadIdx.x;
  const int G = gridDim.x;
  int k = blockIdx.x;
  if (k >= n) return;
  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    fence_mbar_init();
  }
  auto neighbours = [&](int kk, int s) {
    if (tid < 27) {
      const int bid = list[kk];
      const int bx = bid % nbx, by = (bid / nbx) % nby, bz = bid / (nbx * nby);
      const int dx = tid % 3 - 1, dy = (tid / 3) % 3 - 1, dz = tid / 9 - 1;
      const int x = bx + dx, y = by + dy, z = bz + dz;
      int sl = SLOT_OUT;
      if (x >= 0 && y >= 0 && z >= 0 && x < nbx && y < nby && z < nbz)
        sl = slotOf[x + nbx * (y + nby * z)];
      nbSlot[s][tid] = sl;
    }
  };
  Halo h{0.f, 0.f, 0.f, 0.f, 0.f};
  // per stage (bit s): a box is in flight / the parity of its next phase
  // (uniform: every thread reads the same shared slot)
  uint32_t issued = 0u, phase = 0u;
  // block kk into stage s: the box (one thread), the z planes, the halo loads
  auto issue = [&](int s) {
    const int slot = nbSlot[s][13];
    if (slot < 0) {
      issued &= ~(1u << s);
      cp_async_commit();
      return;
    }
    issued |= 1u << s;
    float* tile = tiles + s * TILE;
    if (tid == 0) {
      fence_proxy_async();  // the stage was last written by ordinary stores
      mbar_expect_tx(&bar[s], BOX_BYTES);
      box_g2s(tile + Tl::PP, &map, -XO, -1, 0, slot, &bar[s]);
    }
    zplanes_fill(tile, pool, xf, nbSlot[s], emptyVal, fullVal, tid);
    cp_async_commit();
    halo_load(h, pool, xf, nbSlot[s], emptyVal, fullVal, tid);
  };
  __syncthreads();  // barriers initialised
  neighbours(k, 0);
  __syncthreads();
  issue(0);
  for (int it = 0; k < n; it++, k += G) {
    const int s = it & 1;
    const int kn = k + G;
    // the block's box has landed: its register halo into the tile
    if ((issued >> s) & 1u) {
      const uint32_t par = (phase >> s) & 1u;
      const bool ok = __syncthreads_and(mbar_wait(&bar[s], par));
      if (!ok) {
        if (tid == 0) atomicOr(errFlag, ERR_WAIT_TIMEOUT);
        mbar_wait(&bar[s], par);  // bounded: the box in flight
        cp_async_wait_group<0>();
        return;
      }
      phase ^= 1u << s;
      halo_store(h, tiles + s * TILE, tid);
    }
    cp_async_wait_group<0>();
    if (kn < n) neighbours(kn, s ^ 1);
    __syncthreads();  // stage s complete, nbSlot[s ^ 1] written
    if (kn < n) issue(s ^ 1);
    const int slot0 = nbSlot[s][13];
    if (slot0 < 0) {
      if (tid == 0) atomicOr(errFlag, MCF_ERR_NOT_VALUE);
    } else {
      mcf_compute<BS, float, XO>(tiles + s * TILE, pool + (size_t)slot0 * Tl::NV,
                                 xf + (size_t)slot0 * 2 * BS * BS, dt, clamp01, tid);
    }
    __syncthreads();  // stage s may be refilled
  }
}

// Fills the face cache: the planes x = 0 and x = BSX-1 of every value block
// (slots 0..nSlots-1), as [slot][2][z][y].
template <int BSX, typename T>
__global__ void __launch_bounds__(256) k_mcf_xfaces(const T* __restrict__ pool, int64_t nSlots,
                                                    T* __restrict__ xf) {
  constexpr int F = BSX * BSX;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nSlots * 2 * F;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t sl = i / (2 * F);
    const int r = (int)(i % (2 * F)), side = r / F, y = r % BSX, z = (r % F) / BSX;
    xf[i] = pool[sl * (BSX * BSX * BSX) + (side ? BSX - 1 : 0) + BSX * (y + BSX * z)];
  }
}

// The tensor map of an FP32 16^3 pool of nSlots blocks (see
// mcf_colour_kernel_tma); false if the driver's encoder is not available or
// refuses the pool, and the copies issued by threads are used instead.
bool mcf_tensor_map(CUtensorMap* map, float* pool, int64_t nSlots) {
  static std::atomic<PFN_cuTensorMapEncodeTiled_v12000> encode{nullptr};
  PFN_cuTensorMapEncodeTiled_v12000 fn = encode.load(std::memory_order_acquire);
  if (!fn) {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) !=
            cudaSuccess ||
        q != cudaDriverEntryPointSuccess || !f)
      return false;
    fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(f);
    encode.store(fn, std::memory_order_release);
  }
  if ((reinterpret_cast<uintptr_t>(pool) & 15) != 0 || nSlots <= 0) return false;
  constexpr int B = tma::BS;
  const cuuint64_t dim[4] = {B, B, B, (cuuint64_t)nSlots};
  const cuuint64_t stride[3] = {sizeof(float) * B, sizeof(float) * B * B,
                                sizeof(float) * B * B * B};
  const cuuint32_t box[4] = {(cuuint32_t)tma::Tl::RP, B + 2, B, 1};
  const cuuint32_t estride[4] = {1, 1, 1, 1};
  return fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, pool, dim, stride, box, estride,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
            CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <int BSX, typename T>
cudaError_t launch_mcf_t(T* pool, T* xf, int64_t nSlots, const int* slotOf,
                         const int* colourList, const int* colourStart, int nbx, int nby,
                         int nbz, float emptyVal, float fullVal, int nIter, float dt,
                         int clamp01, int* errFlag, cudaStream_t stream) {
  using Tl = McfTile<BSX>;
  // The shared-memory limit is an attribute of the kernel on each device:
  // set it once per device (bit per device; a race only repeats the call).
  static std::atomic<uint64_t> attrSet{0};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  const uint64_t bit = dev < 64 ? (uint64_t)1 << dev : 0;
  if (!bit || !(attrSet.load(std::memory_order_acquire) & bit)) {
    e = cudaFuncSetAttribute(mcf_colour_kernel<BSX, T>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)(Tl::SMEM * mcf_stages<BSX>()));
    if (e != cudaSuccess) return e;
    attrSet.fetch_or(bit, std::memory_order_acq_rel);
  }
  static int numSMs[64] = {0};
  if (dev < 64 && !numSMs[dev]) {
    int v = 0;
    e = cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
    numSMs[dev] = v;
  }
  const int maxGrid = (dev < 64 ? numSMs[dev] : 148) * mcf_ctas_per_sm<BSX>();
  if (xf && nSlots > 0 && nIter > 0)
    k_mcf_xfaces<BSX, T><<<(dev < 64 ? numSMs[dev] : 148) * 4, 256, 0, stream>>>(pool, nSlots,
                                                                               xf);
  // FP32 16^3 blocks of a context pool: the block arrives as one tensor box
  if constexpr (BSX == 16 && std::is_same<T, float>::value) {
    CUtensorMap map;
    if (xf && nSlots > 0 && mcf_tensor_map(&map, pool, nSlots)) {
      static std::atomic<uint64_t> tmaAttr{0};
      if (!bit || !(tmaAttr.load(std::memory_order_acquire) & bit)) {
        e = cudaFuncSetAttribute(mcf_colour_kernel_tma, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)tma::SMEM);
        if (e != cudaSuccess) return e;
        tmaAttr.fetch_or(bit, std::memory_order_acq_rel);
      }
      for (int it = 0; it < nIter; it++)
        for (int c = 0; c < 8; c++) {
          const int n = colourStart[c + 1] - colourStart[c];
          if (n <= 0) continue;
          mcf_colour_kernel_tma<<<std::min(n, maxGrid), tma::Tl::NT, tma::SMEM, stream>>>(
              map, pool, xf, slotOf, colourList + colourStart[c], n, nbx, nby, nbz, emptyVal,
              fullVal, dt, clamp01, errFlag);
        }
      return cudaGetLastError();
    }
  }
  for (int it = 0; it < nIter; it++)
    for (int c = 0; c < 8; c++) {
      int n = colourStart[c + 1] - colourStart[c];
      if (n <= 0) continue;
      const int grid = mcf_stages<BSX>() == 2 ? std::min(n, maxGrid) : n;
      mcf_colour_kernel<BSX, T><<<grid, Tl::NT, Tl::SMEM * mcf_stages<BSX>(), stream>>>(
          pool, xf, slotOf, colourList + colourStart[c], n, nbx, nby, nbz, emptyVal, fullVal, dt,
          clamp01, errFlag);
    }
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_mcf_typed(T* pool, T* xf, int64_t nSlots, const int* slotOf,
                             const int* colourList, const int* colourStart, int nbx, int nby,
                             int nbz, int bsx, float emptyVal, float fullVal, int nIter, float dt,
                             int clamp01, int* errFlag, cudaStream_t stream) {
  switch (bsx) {
    case 8:
      return launch_mcf_t<8, T>(pool, xf, nSlots, slotOf, colourList, colourStart, nbx, nby, nbz,
                                emptyVal, fullVal, nIter, dt, clamp01, errFlag, stream);
    case 16:
      return launch_mcf_t<16, T>(pool, xf, nSlots, slotOf, colourList, colourStart, nbx, nby,
                                 nbz, emptyVal, fullVal, nIter, dt, clamp01, errFlag, stream);
    case 32:
      return launch_mcf_t<32, T>(pool, xf, nSlots, slotOf, colourList, colourStart, nbx, nby,
                                 nbz, emptyVal, fullVal, nIter, dt, clamp01, errFlag, stream);
    default:
      return cudaErrorInvalidValue;
  }
}

}  // namespace

cudaError_t launch_mcf(float* pool, const int* slotOf, const int* colourList,
                       const int* colourStart, int nbx, int nby, int nbz, int bsx,
                       float emptyVal, float fullVal, int nIter, float dt, int clamp01,
                       int* errFlag, cudaStream_t stream, void* xfaces, int64_t nSlots) {
  return launch_mcf_typed<float>(pool, static_cast<float*>(xfaces), nSlots, slotOf, colourList,
                                 colourStart, nbx, nby, nbz, bsx, emptyVal, fullVal, nIter, dt,
                                 clamp01, errFlag, stream);
}

cudaError_t launch_mcf_u16(uint16_t* pool, const int* slotOf, const int* colourList,
                           const int* colourStart, int nbx, int nby, int nbz, int bsx,
                           uint16_t emptyVal, uint16_t fullVal, int nIter, float dt, int clamp01,
                           int* errFlag, cudaStream_t stream, void* xfaces, int64_t nSlots) {
  // const blocks read like stored values: q * (1/65535)
  return launch_mcf_typed<uint16_t>(pool, static_cast<uint16_t*>(xfaces), nSlots, slotOf,
                                    colourList, colourStart, nbx, nby, nbz, bsx,
                                    (float)emptyVal * U16_SCALE, (float)fullVal * U16_SCALE, nIter,
                                    dt, clamp01, errFlag, stream);
}

}  // namespace msbg
