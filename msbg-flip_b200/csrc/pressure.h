// Pressure solver internals: multigrid hierarchy of tiles on the MSBG block
// grid (host description + device mirrors).  See pressure_host.cpp for the
// construction and pressure.cu for the kernels and the MGPCG driver.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <map>
#include <memory>
#include <utility>
#include <string>
#include <vector>

#include "common.cuh"
#include "msbg_gpu.h"

namespace msbg {
namespace ps {

constexpr int TS_MAX = 16;  // tile edge in cells (a 32^3 block is 8 tiles)

// Allocator whose resize() leaves new elements uninitialised: the per-cell
// arrays of the hierarchy (hundreds of MB at 1024^3) are then first touched,
// zeroed and filled by the threads that own their tiles, instead of by one
// thread's serial zero-fill.
template <typename T>
struct NoInitAlloc : std::allocator<T> {
  using value_type = T;
  template <typename U>
  struct rebind {
    using other = NoInitAlloc<U>;
  };
  NoInitAlloc() = default;
  template <typename U>
  NoInitAlloc(const NoInitAlloc<U>&) noexcept {}
  template <typename U>
  void construct(U* p) noexcept {
    ::new (static_cast<void*>(p)) U;
  }
  template <typename U, typename... A>
  void construct(U* p, A&&... a) {
    ::new (static_cast<void*>(p)) U(std::forward<A>(a)...);
  }
};
template <typename T>
using HostArray = std::vector<T, NoInitAlloc<T>>;

// Face neighbour kinds of a tile face.
enum : int {
  FACE_NONE = 0,    // domain boundary, or a region whose tile holds no liquid
  FACE_SAME = 1,    // same-level tile
  FACE_COARSER = 2, // one level coarser tile (our face is part of its face)
  FACE_FINER = 3    // one level finer tiles (1..4 of them cover our face)
};

// Per face: kind, t[4] neighbour tile ids, oa/ob offsets (FACE_COARSER: our
// first face cell in neighbour cells; FACE_FINER: unused), cov (FACE_FINER:
// our cells covered per fine tile along a/b), nts (neighbour tile size).
constexpr int FACE_INTS = 9;
enum { F_KIND = 0, F_T0 = 1, F_OA = 5, F_OB = 6, F_COV = 7, F_NTS = 8 };

// Face order: -x,+x,-y,+y,-z,+z (face = 2*dir + side).  Tangential axes of a
// face plane: dir 0 -> (y,z), dir 1 -> (x,z), dir 2 -> (x,y); plane index
// a + ts*b.

// Cell types kept for the learned network's mask channels (MG level 0).
enum : uint8_t { CT_AIR = 0, CT_LIQUID = 1, CT_SOLID = 2 };

struct Tile {
  int level;       // resolution level: cell edge = 2^level fine voxels
  int ts;          // cells per edge
  int ox, oy, oz;  // origin in level cells
  int64_t off;     // first cell in the level pools
};

struct Level {
  int m = 0;                       // multigrid level
  std::vector<Tile> tiles;
  std::vector<int> face;           // [nTiles*6*FACE_INTS]
  std::vector<int64_t> ifOff;      // [nTiles*6] offset of the interface plane or -1
  int64_t nCells = 0, nIf = 0;
  // operator: a_ii, lower-face couplings to same-level neighbours, interface
  // couplings (stored on the finer side, one per fine boundary cell)
  HostArray<float> diag, cx, cy, cz, ifc, rhs;
  HostArray<uint8_t> ctype;        // MG level 0 only: CT_* per cell
  // tile maps per resolution level: dense raster of tile ids (-1 = none)
  std::vector<std::vector<int>> tmap = std::vector<std::vector<int>>(32);
  std::vector<int> tmapN = std::vector<int>(32, 0);  // tiles per edge (0 = level absent)
  std::vector<int> tsOf = std::vector<int>(32, 0);   // tile edge per level
  // restriction map to level m+1: per tile coarse tile, offset, aggregated?
  std::vector<int> toCoarse;       // [nTiles*6]: coarse tile, ox, oy, oz, aggregated, coarse ts
  // smoothing passes: tile ids grouped by (level, colour), and per tile size
  struct Pass {
    int level, colour, ts;
    int start, count;              // into passTiles
  };
  std::vector<Pass> passes;
  std::vector<int> passTiles;
  // all tiles grouped by tile size (for matvec/residual/restrict/prolong)
  struct Group {
    int ts, start, count;
  };
  std::vector<Group> groups;
  std::vector<int> groupTiles;
  int64_t nFluid = 0;
};

// Device mirror of one level.
struct LevelDev {
  DeviceBuffer tileOff, face, ifOff, toCoarse, passTiles, groupTiles;
  DeviceBuffer diag, invdiag, cx, cy, cz, ifc;
  DeviceBuffer tileRec;            // 256-byte per-tile records (smooth_pipe.cuh)
  DeviceBuffer x, b, r;            // FP32 work vectors of this level
  DeviceBuffer ctype;              // level 0: CT_* per cell
  DeviceBuffer fluid;              // liquid flag per cell (device build only)
  // packed x = 0 plane of cx per 16^3 tile, and the packed x faces of the
  // V-cycle's x on this level (pressure_kernels.cuh: xface_slot)
  DeviceBuffer cxf, xf;
};

// Domain faces without a caller spec follow the reference's FLIP operator:
// the lower faces (-x, -y, -z) couple to p = 0 outside with the coefficient
// the callback returns for the cell's own lower face, the upper faces have no
// coupling, because computeDiagonalFLIP_ reads the face channel past the
// grid as its empty value 0 (src/msbg3.cpp:2714-2722, sbg.h:880-894).
constexpr int DBC_REFERENCE = -1;

struct Hierarchy {
  int res = 0, bsx0 = 0, nLevels = 0, nb1x = 0, nb1y = 0, nb1z = 0;
  int sx = 0, sy = 0, sz = 0;
  std::vector<int> blockLevel;     // refinement map (MG level 0)
  // per domain face (2*dir + side): MSBG_DBC_OPEN, MSBG_DBC_SOLID, or
  // DBC_REFERENCE when the caller gave no spec
  int domainBc[6] = {DBC_REFERENCE, DBC_REFERENCE, DBC_REFERENCE,
                     DBC_REFERENCE, DBC_REFERENCE, DBC_REFERENCE};
  std::vector<Level> levels;
  // coarsest-level dense inverse (FP64), fluid cell indices
  int nCoarse = 0;
  std::vector<double> coarseInv;
  std::vector<int64_t> coarseCells;
  int64_t deviceBuildH2D = 0;      // bytes a device build copied to the GPU
};

// Per-cell arrays of MG level 0 in the packed block layout (for every block
// in bid order, (bsx0 >> level)^3 cells, vid = x + y*bs + z*bs*bs): cell
// flags, lower-face coefficient per direction, right-hand side (may be NULL).
// A level-l cell reads the entry of the cell holding its lowest fine voxel,
// as the callbacks would be asked.
struct ArrayInput {
  const uint16_t* flags;
  const float* face[3];
  const float* rhs;
};

// Construction of the hierarchy from the arrays with the per-cell work on the
// GPU (pressure_host.cpp, build_gpu.cu): H receives the topology of every
// level (tiles, faces, restriction maps, passes) and the coarsest inverse;
// dev[m] the operator of level m (diag, invdiag, cx, cy, cz, ifc, ifOff;
// level 0 also ctype), rhs0 the right-hand side of level 0.
int build_hierarchy_device(Hierarchy& H, std::vector<std::unique_ptr<LevelDev>>& dev,
                           DeviceBuffer& rhs0, int sx, int sy, int sz, int bsx0, int nLevels,
                           const int* blockLevel, const int* domainBc, const ArrayInput& arr,
                           int maxCoarseCells, cudaStream_t st, std::string* err);

// Host construction (pressure_host.cpp) from the callbacks cb, or from the
// arrays arr when arr is given (cb is then not used).
int build_hierarchy(Hierarchy& H, int sx, int sy, int sz, int bsx0, int nLevels,
                    const int* blockLevel, const int* domainBc,
                    const msbg_pressure_callbacks* cb, int maxCoarseCells, std::string* err,
                    const ArrayInput* arr = nullptr);

}  // namespace ps
}  // namespace msbg
