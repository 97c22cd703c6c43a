// Device construction of the pressure hierarchy from the bulk prepare's
// per-cell arrays (build_gpu.cu): argument blocks and launches.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "pressure.h"

namespace msbg {
namespace ps {

// A tile as the kernels see it (Tile, with the offset last).
struct TileD {
  int level, ts, ox, oy, oz, pad;
  int64_t off;
};

// Tile lookup of one MG level: per resolution level l a raster of tile ids
// (tmapN[l]^3 entries at tmapOff[l], -1 = none) with tiles of 2^tsSh[l] cells.
constexpr int MAXRL = 16;
struct LevelMapD {
  const TileD* tiles;
  const int* tmap;
  int64_t tmapOff[MAXRL];
  int tmapN[MAXRL];
  int tsSh[MAXRL];
  int m;  // the MG level
};

// The block raster (refinement map of MG level 0).
struct GridD {
  int sx, sy, sz, sh0, nb1x, nb1y;
  const int* blockLevel;
};

// MG level 0, one chunk of consecutive tiles [tile0, tile0 + nTiles): the raw
// arrays hold the chunk's cells in the level's cell order (cell c at c - cell0),
// planes[tile - tile0][dir][TS_MAX^2] the couplings (FP64, as the host sums
// them) of the upper tile faces that read neighbour blocks.
// faceInfo[tile][face]: -1 outside the domain, else the resolution level of
// the region behind the face.
struct L0Args {
  const TileD* tiles;
  const int* faceInfo;
  const int64_t* ifOff;
  int tile0;
  int64_t cell0;
  const uint16_t* flags;
  const float *fx, *fy, *fz, *rhs;
  const double* planes;
  int dbc[6];  // MSBG_DBC_OPEN / MSBG_DBC_SOLID / DBC_REFERENCE
  float *diag, *cx, *cy, *cz, *rhs0, *ifc;
  uint8_t *ctype, *fluid;
  unsigned long long* bad;     // lowest (cell * 2 + isolated) with an unsolvable equation
  unsigned long long* nFluid;  // liquid cells
};

// Candidate coarse tiles (candidates that overlap a fine tile), their cell
// offsets in candFluid, and the fine level.
struct CoarseArgs {
  const TileD* cand;
  const int64_t* candOff;
  LevelMapD F;
  GridD g;
  const uint8_t* fineFluid;
  uint8_t* candFluid;
  int* candAny;
};

struct GalerkinArgs {
  LevelMapD F;
  GridD g;
  const uint8_t* fineFluid;
  const float *Fdiag, *Fcx, *Fcy, *Fcz, *Fifc;
  const int64_t* FifOff;
  const TileD* Gtiles;
  const int64_t* GifOff;
  const uint8_t* coarseFluid;
  int Gm;
  float *Gdiag, *Gcx, *Gcy, *Gcz, *Gifc;
};

cudaError_t launch_build_l0(const L0Args& a, int nTiles, cudaStream_t st);
cudaError_t launch_coarse_fluid(const CoarseArgs& a, int nCand, cudaStream_t st);
cudaError_t launch_place_fluid(const TileD* tiles, const int64_t* srcOff, const uint8_t* candFluid,
                               uint8_t* fluid, unsigned long long* nFluid, int nTiles,
                               cudaStream_t st);
cudaError_t launch_galerkin(const GalerkinArgs& a, int nTiles, cudaStream_t st);
cudaError_t launch_invdiag(const float* diag, float* inv, int64_t n, cudaStream_t st);

}  // namespace ps
}  // namespace msbg
