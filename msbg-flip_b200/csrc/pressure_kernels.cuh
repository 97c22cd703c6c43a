// Device kernels of the MGPCG pressure solver (tile-based, sm_100a).
//
// Data of one MG level: tiles of TS^3 cells stored back to back (cell index
// i + TS*(j + TS*k) inside a tile); operator diag (a_ii), cx/cy/cz (coupling
// to the same-level -x/-y/-z neighbour), ifc (interface couplings on the finer
// side of a level jump, one per fine boundary cell).  One CTA per tile, thread
// (i,j) owns the z column of the tile.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "pressure.h"

namespace msbg {
namespace ps {

struct LevelView {
  const int64_t* tileOff;
  const int* face;
  const int64_t* ifOff;
  const int* toCoarse;
  const float* diag;
  const float* invdiag;  // 1/a_ii (0 for cells that are not liquid)
  const void* tileRec;   // per-tile records of the pipelined smoother
  const float* cx;
  const float* cy;
  const float* cz;
  const float* ifc;
  // the x = 0 plane of cx of every 16^3 tile, packed: 256 floats at tile
  // offset / 16 (the coupling across a tile's upper x face, read as one
  // contiguous run instead of 256 values 64 bytes apart); nullptr if absent
  const float* cxf = nullptr;
};

// Packed x faces of a level vector on 16^3 tiles: the x = 0 plane at
// tile offset / 8 and the x = 15 plane 256 further, each face cell (y, z) at
// y + 16 z.  Kernels that write such a vector also write its faces, so the
// x-face halo of a neighbour is read in full 128-byte lines.
__host__ __device__ __forceinline__ int64_t xface_slot(int64_t off, int side, int y, int z) {
  return (off >> 3) + (side ? 256 : 0) + y + 16 * z;
}
__host__ __device__ __forceinline__ int64_t xface_len(int64_t nCells) { return nCells / 8 + 512; }
// the same rounded up to whole groups of 4 (the vector kernels' unit)
__host__ __device__ __forceinline__ int64_t xface_words(int64_t nCells) {
  return (xface_len(nCells) + 3) & ~(int64_t)3;
}

__host__ __device__ __forceinline__ int tidx(int ts, int i, int j, int k) { return i + ts * (j + ts * k); }

// Cell of a tile addressed by its face plane: position along dir = p, face
// coordinates (a,b).
__host__ __device__ __forceinline__ int plane_idx(int ts, int dir, int p, int a, int b) {
  return dir == 0 ? tidx(ts, p, a, b) : dir == 1 ? tidx(ts, a, p, b) : tidx(ts, a, b, p);
}

// Sum over the neighbours across face (dir, side) of face cell (a,b) of tile
// ti: coupling * x(neighbour), accumulated in AT.  x = vector of this level.
template <typename XT, typename AT = float>
__host__ __device__ __forceinline__ AT ghost_sum(const LevelView& L, const XT* __restrict__ x,
                                                 int ti, int ts, int dir, int side, int a,
                                                 int b) {
  const int* F = L.face + ((size_t)ti * 6 + dir * 2 + side) * FACE_INTS;
  const int kind = F[F_KIND];
  if (kind == FACE_NONE) return AT(0);
  const float* cd = dir == 0 ? L.cx : dir == 1 ? L.cy : L.cz;
  if (kind == FACE_SAME) {
    const int nb = F[F_T0];
    const int64_t no = L.tileOff[nb];
    const int pn = side ? 0 : ts - 1;
    const AT xn = (AT)x[no + plane_idx(ts, dir, pn, a, b)];
    const AT c = side ? (AT)cd[no + plane_idx(ts, dir, 0, a, b)]
                      : (AT)cd[L.tileOff[ti] + plane_idx(ts, dir, 0, a, b)];
    return c * xn;
  }
  if (kind == FACE_COARSER) {
    const int nb = F[F_T0], nts = F[F_NTS];
    const int64_t no = L.tileOff[nb];
    const int pn = side ? 0 : nts - 1;
    const AT xn = (AT)x[no + plane_idx(nts, dir, pn, F[F_OA] + (a >> 1), F[F_OB] + (b >> 1))];
    const AT c = (AT)L.ifc[L.ifOff[(size_t)ti * 6 + dir * 2 + side] + a + ts * b];
    return c * xn;
  }
  // FACE_FINER
  const int cov = F[F_COV], nts = F[F_NTS];
  const int per = ts / cov;
  const int nb = F[F_T0 + (a / cov) + per * (b / cov)];
  if (nb < 0) return AT(0);
  const int64_t no = L.tileOff[nb];
  const int64_t io = L.ifOff[(size_t)nb * 6 + dir * 2 + (1 - side)];
  if (io < 0) return AT(0);
  const int pn = side ? 0 : nts - 1;
  const int fa0 = 2 * (a % cov), fb0 = 2 * (b % cov);
  AT s = AT(0);
#pragma unroll
  for (int v = 0; v < 2; v++)
#pragma unroll
    for (int u = 0; u < 2; u++) {
      const int fa = fa0 + u, fb = fb0 + v;
      s += (AT)L.ifc[io + fa + nts * fb] * (AT)x[no + plane_idx(nts, dir, pn, fa, fb)];
    }
  return s;
}

}  // namespace ps
}  // namespace msbg
