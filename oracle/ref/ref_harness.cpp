// Reference harness (test infrastructure; never part of the GPU product).
//
// Drives the unmodified reference MSBG CPU solver through its own public API so
// that tests can pin the oracle against it and bench.py can time it as the CPU
// baseline.  Every entry point takes plain arrays, builds a MultiresSparseGrid
// exactly the way the reference's own callers do (msbg_demo.cpp:283-502 for
// the smoother), runs the reference routine and copies the result back.
//
// Block kinds in the `kind` arrays: 0 = no block (NULL in the block map),
// 1 = value block (data supplied), 2 = const "empty" block, 3 = const "full"
// block (sbg.h:2037-2049).
#include <chrono>
#include <cstdint>
#include <cstring>
#include <vector>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <functional>
#include <iostream>
#include <limits>
#include <map>
#include <memory>
#include <mutex>
#include <sstream>
#include <string>
#include <type_traits>
#include <thread>
#include <omp.h>
#include "tbb/tbb.h"
#include <vectorclass/vectorclass.h>
// Test-only access to the solver internals the harness drives.
#define private public
#define protected public
#include "common_headers.h"
#include "msbg.h"
#include "thread.h"

int nMaxThreads = -1;  // defined by the reference's main.cpp:29 in the demo

// The reference's image writers are not compiled (they need libpng/libjpeg);
// the smoother and solver never call them.
extern "C" int BmpWritePNG(FILE*, void*, void*, int, int, int) { return 1; }
extern "C" int BmpSaveBitmapJPG(void*, char*, int, int) { return 1; }
// MultiresSparseGrid::interpolate<1> is declared but never instantiated in
// the reference sources; only its slice visualiser refers to it.  A no-op
// definition under its mangled name lets the library load eagerly.
extern "C" void _ZN4MSBG18MultiresSparseGrid11interpolateILi1EEEviPfjRN11BasicVector10Vector3DimIfEEb() {}

using namespace MSBG;
using namespace SBG;

static bool g_inited = false;

extern "C" int ref_init(int nThreads) {
  LogLevel = 0;
  if (!g_inited) {
    ThrInit();
    g_inited = true;
  }
  int a = 0, b = 0;
  ThrGetMaxNumberOfThreads(&a, &b);
  nMaxThreads = std::max(a, b);
  if (nThreads > 0) {
    omp_set_num_threads(nThreads);
    nMaxThreads = nThreads;
  }
  return nMaxThreads;
}

// A single-level grid with one channel filled from the packed values, the
// way the reference's demo builds its render-density grid
// (src/msbg_demo.cpp:283-502): kind[nBlocks], values packed for kind==1 blocks
// in ascending bid order.  T = float uses CH_FLOAT_1, T = uint16_t the
// render-density channel CH_UINT16_1 (RenderDensity under RSURF_16_BIT,
// src/msbgcell.h:67-68).
namespace {

template <typename T> SparseGrid<T>* mcf_channel(MultiresSparseGrid* m, int chan);
template <> SparseGrid<float>* mcf_channel<float>(MultiresSparseGrid* m, int chan) {
  return m->getFloatChannel(chan, 0);
}
template <> SparseGrid<uint16_t>* mcf_channel<uint16_t>(MultiresSparseGrid* m, int chan) {
  return m->getUint16Channel(chan, 0);
}
template <typename T> constexpr int mcf_chan() {
  return std::is_same<T, float>::value ? CH_FLOAT_1 : CH_UINT16_1;
}

template <typename T>
MultiresSparseGrid* mcf_grid_create(int sx, int sy, int sz, int bsx, const int8_t* kind,
                                    T emptyVal, T fullVal, const T* values) {
  MultiresSparseGrid* msbg = MultiresSparseGrid::create(
      "REF", sx, sy, sz, bsx, -1, 0, -1, MSBG::OPT_SINGLE_LEVEL | MSBG::OPT_SINGLE_CHANNEL_FLOAT);
  if (!msbg) return nullptr;
  const int nb = msbg->nBlocks();
  {
    std::vector<int> levels(nb, 0);
    msbg->regularizeRefinementMap(levels.data());
    msbg->setRefinementMap(levels.data(), NULL, -1, NULL, false);
  }
  SparseGrid<T>* sg = mcf_channel<T>(msbg, mcf_chan<T>());
  if (!sg) {
    MultiresSparseGrid::destroy(msbg);
    return nullptr;
  }
  sg->reset();
  sg->prepareDataAccess();
  sg->setEmptyValue(emptyVal);
  sg->setFullValue(fullVal);
  const int nv = sg->nVoxelsInBlock();
  size_t off = 0;
  for (int bid = 0; bid < nb; bid++) {
    switch (kind[bid]) {
      case 1: {
        T* d = sg->getBlockDataPtr(bid, 1, 0);
        std::memcpy(d, values + off, sizeof(T) * nv);
        off += nv;
        break;
      }
      case 2: sg->setEmptyBlock(bid); break;
      case 3: sg->setFullBlock(bid); break;
      default: break;
    }
  }
  return msbg;
}

template <typename T>
void mcf_grid_read(MultiresSparseGrid* msbg, const int8_t* kind, T* values) {
  SparseGrid<T>* sg = mcf_channel<T>(msbg, mcf_chan<T>());
  const int nv = sg->nVoxelsInBlock();
  size_t off = 0;
  for (int bid = 0; bid < msbg->nBlocks(); bid++) {
    if (kind[bid] != 1) continue;
    std::memcpy(values + off, sg->getBlockDataPtr(bid), sizeof(T) * nv);
    off += nv;
  }
}

template <typename T>
int mcf_run(int sx, int sy, int sz, int bsx, const int8_t* kind, T emptyVal, T fullVal,
            T* values, const int* update, int nUpdate, int numIter, float dt, int clamp01,
            double* seconds) {
  MultiresSparseGrid* msbg = mcf_grid_create<T>(sx, sy, sz, bsx, kind, emptyVal, fullVal, values);
  if (!msbg) return 1;
  std::vector<int> blockList(update, update + nUpdate);
  auto t0 = std::chrono::steady_clock::now();
  msbg->applyChannelPdeFast<T>(mcf_chan<T>(), CH_NULL, CH_NULL, &blockList,
                               -(PDE_MEAN_CURVATURE + OPT_8_COLOR_SCHEME), clamp01, 0, 0, 0,
                               numIter, 1.0f, dt);
  auto t1 = std::chrono::steady_clock::now();
  if (seconds) *seconds = std::chrono::duration<double>(t1 - t0).count();
  mcf_grid_read<T>(msbg, kind, values);
  MultiresSparseGrid::destroy(msbg);
  return 0;
}

}  // namespace

// Mean-curvature flow, 8-colour in-place scheme, FP32 channel.
// Mirrors msbg_demo.cpp:716-727 (applyChannelPdeFast with
// -(PDE_MEAN_CURVATURE+OPT_8_COLOR_SCHEME)) on a single-level grid.
//   update[nUpdate] = block ids handed to the smoother as its block list.
extern "C" int ref_mcf(int sx, int sy, int sz, int bsx, const int8_t* kind,
                       float emptyVal, float fullVal, float* values,
                       const int* update, int nUpdate, int numIter, float dt,
                       int clamp01, double* seconds) {
  return mcf_run<float>(sx, sy, sz, bsx, kind, emptyVal, fullVal, values, update, nUpdate,
                        numIter, dt, clamp01, seconds);
}

// Mean-curvature flow on the quantised render-density channel the reference
// is built with, as msbg_demo.cpp:297-298 and 716-727 run it: values stored
// as round(phi * 65535) and read as q * (1/65535) (src/sbg.h:225-232,
// 360-368).  Values and the const blocks' emptyVal / fullVal are raw 16-bit
// integers.
extern "C" int ref_mcf_u16(int sx, int sy, int sz, int bsx, const int8_t* kind, uint16_t emptyVal,
                           uint16_t fullVal, uint16_t* values, const int* update, int nUpdate,
                           int numIter, float dt, int clamp01, double* seconds) {
  return mcf_run<uint16_t>(sx, sy, sz, bsx, kind, emptyVal, fullVal, values, update, nUpdate,
                           numIter, dt, clamp01, seconds);
}

// The same grids for a caller that runs its own code on them (the
// integration adapter): create, read the channel back, destroy.
extern "C" void* ref_grid_create_f32(int sx, int sy, int sz, int bsx, const int8_t* kind,
                                     float emptyVal, float fullVal, const float* values) {
  return mcf_grid_create<float>(sx, sy, sz, bsx, kind, emptyVal, fullVal, values);
}
extern "C" void* ref_grid_create_u16(int sx, int sy, int sz, int bsx, const int8_t* kind,
                                     uint16_t emptyVal, uint16_t fullVal, const uint16_t* values) {
  return mcf_grid_create<uint16_t>(sx, sy, sz, bsx, kind, emptyVal, fullVal, values);
}
extern "C" void ref_grid_read_f32(void* m, const int8_t* kind, float* values) {
  mcf_grid_read<float>((MultiresSparseGrid*)m, kind, values);
}
extern "C" void ref_grid_read_u16(void* m, const int8_t* kind, uint16_t* values) {
  mcf_grid_read<uint16_t>((MultiresSparseGrid*)m, kind, values);
}
extern "C" void ref_grid_destroy(void* m) {
  MultiresSparseGrid* g = (MultiresSparseGrid*)m;
  MultiresSparseGrid::destroy(g);
}

// ---------------------------------------------------------------------------
// FLIP pressure solver (src/msbg3.cpp:2467-3271) driven from arrays.
//
// The callbacks are the caller's (the same seeded scene the GPU path samples);
// the reference calls them with unscaled coordinates for coarse blocks
// (src/msbg3.cpp:2494-2503), exactly as it does in its own FLIP driver.
// Channel data move in a packed layout: for every block id in ascending order,
// the block's (bsx0>>level)^3 values at its level for the given MG level.
// ---------------------------------------------------------------------------
namespace {

typedef CellFlags (*PsCellTypeFn)(void*, int, int, int);
typedef float (*PsFaceFn)(void*, int, int, int, int);
typedef float (*PsRhsFn)(void*, int, int, int);

struct PsHandle {
  MultiresSparseGrid* msbg;
};

// Channel ids understood by ref_ps_get/set: the reference's channel ids, plus
//   -1,-2,-3 = face coefficients dir 0,1,2 (CH_FACE_AREA), -10 = cell flags.
SparseGrid<float>* ps_float_grid(MultiresSparseGrid* m, int ch, int level, int levelMg) {
  if (ch <= -1 && ch >= -3) return m->getFaceAreaChannel(-ch - 1, level, levelMg);
  if (ch == CH_DIAGONAL) return m->getPSFloatChannel(CH_DIAGONAL, level, levelMg);
  return m->getFloatChannel(ch, level, levelMg);
}

}  // namespace

extern "C" void* ref_ps_create(int sx, int sy, int sz, int bsx0, int nLevels,
                               const int* blockLevel, const int* domBc, PsCellTypeFn cellType,
                               PsFaceFn face, PsRhsFn rhs, void* user, double* prepSeconds) {
  MultiresSparseGrid* m = MultiresSparseGrid::create("PS", sx, sy, sz, bsx0, -1, 0, -1, 0,
                                                     NULL, NULL, nLevels);
  if (!m) return nullptr;
  const int nb = m->nBlocks();
  std::vector<int> levels(blockLevel, blockLevel + nb);
  m->setRefinementMap(levels.data(), NULL, -1, NULL, false, true);
  m->setDomainBoundarySpec_(domBc[0], domBc[1], domBc[2], domBc[3], domBc[4], domBc[5]);
  auto* h = new PsHandle{m};
  FlipPressureCallbacks cb;
  cb.sampleCellType = cellType;
  cb.sampleFaceCoeff = face;
  cb.sampleRhs = rhs;
  cb.user = user;
  auto t0 = std::chrono::steady_clock::now();
  m->preparePressureSolveFLIP(cb);
  auto t1 = std::chrono::steady_clock::now();
  if (prepSeconds) *prepSeconds = std::chrono::duration<double>(t1 - t0).count();
  return h;
}

extern "C" void ref_ps_destroy(void* hp) {
  auto* h = (PsHandle*)hp;
  MultiresSparseGrid::destroy(h->msbg);
  delete h;
}

// The prepared grid itself, for a caller that runs its own code on it.
extern "C" void* ref_ps_grid(void* hp) { return ((PsHandle*)hp)->msbg; }

extern "C" float ref_ps_omega(void* hp) { return ((PsHandle*)hp)->msbg->_mgSmOmega; }
extern "C" int ref_ps_num_levels(void* hp) { return ((PsHandle*)hp)->msbg->getNumLevels(); }

// Block level and flags per block at MG level levelMg.
extern "C" int ref_ps_block_info(void* hp, int levelMg, int* level, int* flags) {
  auto* m = ((PsHandle*)hp)->msbg;
  for (int b = 0; b < m->nBlocks(); b++) {
    BlockInfo* bi = m->getBlockInfo(b, levelMg);
    level[b] = bi ? bi->level : -1;
    flags[b] = bi ? bi->flags : 0;
  }
  return 0;
}

// Packed size (number of values) of a channel at MG level levelMg.
extern "C" long long ref_ps_packed_size(void* hp, int levelMg) {
  auto* m = ((PsHandle*)hp)->msbg;
  long long n = 0;
  const int bsx0 = m->sg0()->bsx();
  for (int b = 0; b < m->nBlocks(); b++) {
    int l = m->getBlockInfo(b, levelMg)->level;
    int bs = bsx0 >> l;
    n += (long long)bs * bs * bs;
  }
  return n;
}

// Copy a channel out (get=1) or in (get=0).  Missing blocks read as 0 and
// are skipped on write (written with allocation when alloc != 0).
extern "C" int ref_ps_channel(void* hp, int ch, int levelMg, float* data, int get, int alloc) {
  auto* m = ((PsHandle*)hp)->msbg;
  const int bsx0 = m->sg0()->bsx();
  size_t off = 0;
  for (int b = 0; b < m->nBlocks(); b++) {
    int l = m->getBlockInfo(b, levelMg)->level;
    int bs = bsx0 >> l, nv = bs * bs * bs;
    if (ch == -10) {
      SparseGrid<CellFlags>* sg = m->getFlagsChannel(CH_CELL_FLAGS, l, levelMg);
      CellFlags* d = sg ? sg->getBlockDataPtr(b) : nullptr;
      for (int i = 0; i < nv; i++) {
        if (get) data[off + i] = d ? (float)d[i] : -1.f;
      }
    } else {
      SparseGrid<float>* sg = ps_float_grid(m, ch, l, levelMg);
      float* d = sg ? sg->getBlockDataPtr(b, (!get && alloc) ? 1 : 0, 0) : nullptr;
      if (get) {
        for (int i = 0; i < nv; i++) data[off + i] = d ? d[i] : 0.f;
      } else if (d) {
        std::memcpy(d, data + off, sizeof(float) * nv);
      }
    }
    off += nv;
  }
  return 0;
}

// q = A x (residual=0) or r = b - A x (residual=1) on MG level levelMg
// (src/msbg3.cpp:1757-1912).
extern "C" int ref_ps_multiply(void* hp, int levelMg, int chX, int chB, int chDst,
                               int residual) {
  auto* m = ((PsHandle*)hp)->msbg;
  m->multiplyLaplacianMatrixOpt(residual ? OPT_CALC_RESIDUAL : 0, levelMg, chX,
                                residual ? chB : CH_NULL, 0.0f, chDst, nullptr, nullptr);
  return 0;
}

// nIter block red-black sweeps of the smoother on MG level levelMg
// (src/msbg3.cpp:2245-2369).
extern "C" int ref_ps_relax(void* hp, int levelMg, int chX, int chB, int chTmp, int nIter,
                            int reverse) {
  auto* m = ((PsHandle*)hp)->msbg;
  m->relax(0, reverse, levelMg, chX, chB, chTmp, nIter, 0);
  return 0;
}

extern "C" int ref_ps_downsample(void* hp, int levelMgCoarse, int chSrc, int chDst) {
  auto* m = ((PsHandle*)hp)->msbg;
  m->downsampleChannel<float, float>(levelMgCoarse, chSrc, chDst,
                                     OPT_SIMPLE_AVERAGE | OPT_ALL_CELLS);
  return 0;
}

extern "C" int ref_ps_prolongate(void* hp, int levelMgFine, int chSrc, int chDst) {
  auto* m = ((PsHandle*)hp)->msbg;
  m->prolongateChannel<float>(levelMgFine, chSrc, chDst, 0, MG_CONST_PROLONGATION_ALPHA);
  return 0;
}

extern "C" int ref_ps_vcycle(void* hp, int chX, int chB, int chR, int chTmp, int nPre,
                             int nPost, int nCoarse) {
  auto* m = ((PsHandle*)hp)->msbg;
  m->vCycle(0, chX, chB, chR, chTmp, nPre, nPost, nCoarse);
  return 0;
}

extern "C" int ref_ps_solve(void* hp, int nPre, int nPost, int nCoarse, int maxIter, float tol,
                            float* relRes, double* seconds) {
  auto* m = ((PsHandle*)hp)->msbg;
  FlipPressureSolveParams p;
  p.nPre = nPre;
  p.nPost = nPost;
  p.nCoarse = nCoarse;
  p.maxIter = maxIter;
  p.tol = tol;
  auto t0 = std::chrono::steady_clock::now();
  int it = m->solvePressureFLIP(p, relRes);
  auto t1 = std::chrono::steady_clock::now();
  if (seconds) *seconds = std::chrono::duration<double>(t1 - t0).count();
  return it;
}

// ---------------------------------------------------------------------------
// Mixed-resolution grids for the velocity interpolation of G2P.
//
// A MultiresSparseGrid with the given block levels, set up by the
// reference's own setRefinementMap (src/msbg.cpp:1428), which flags the blocks
// with a coarser neighbour (BLK_FINE_COARSE, src/msbg.cpp:1700-1723) and fills
// their fine/coarse distance channel (CH_DIST_FINECOARSE,
// src/msbg.cpp:1887-1960).  Channel data move in the packed layout: for every
// block id in ascending order, the block's (bsx0>>level)^3 values at its level.
// ---------------------------------------------------------------------------
extern "C" void* ref_mr_create(int sx, int sy, int sz, int bsx0, int nLevels,
                               const int* blockLevel) {
  MultiresSparseGrid* m = MultiresSparseGrid::create("MR", sx, sy, sz, bsx0, -1, 0, -1, 0,
                                                     NULL, NULL, nLevels);
  if (!m) return nullptr;
  std::vector<int> levels(blockLevel, blockLevel + m->nBlocks());
  m->setRefinementMap(levels.data(), NULL, -1, NULL, false, true);
  return m;
}

extern "C" void ref_mr_destroy(void* mp) {
  MultiresSparseGrid* m = (MultiresSparseGrid*)mp;
  MultiresSparseGrid::destroy(m);
}

extern "C" int ref_mr_dtransres(void* m) { return ((MultiresSparseGrid*)m)->dTransRes(); }

// Block levels and flags (BLK_*) at MG level 0, as the grid holds them.
extern "C" void ref_mr_block_info(void* mp, int* level, int* flags) {
  auto* m = (MultiresSparseGrid*)mp;
  for (int b = 0; b < m->nBlocks(); b++) {
    level[b] = m->getBlockInfo(b, 0)->level;
    flags[b] = m->getBlockInfo(b, 0)->flags;
  }
}

// The distance channel of every level: kind[l*nBlocks + b] is block b's kind
// in the channel of level l (0 = no block or empty, 1 = value block, 2 = full
// block of value dTransRes*1024, src/msbg.cpp:1994-2029); value blocks (only
// ever at their own level, src/msbg.cpp:1887-1960) land in `out` in the packed
// layout, every other packed voxel reads 0, the channel's empty value
// (src/sbg.cpp:348).  Returns the packed size, or -1 for a value block at a
// level other than its own.
extern "C" long long ref_mr_dist(void* mp, uint16_t* out, int8_t* kind) {
  auto* m = (MultiresSparseGrid*)mp;
  const int bsx0 = m->sg0()->bsx(), nb = m->nBlocks(), nl = m->getNumLevels();
  for (int l = 0; l < nl; l++) {
    SparseGrid<uint16_t>* sg = m->getDistFineCoarseChannel(l);
    for (int b = 0; b < nb; b++) {
      int k = 0;
      if (sg && sg->isValueBlock(b)) k = 1;
      else if (sg && sg->isFullBlock(b)) k = 2;
      kind[(size_t)l * nb + b] = (int8_t)k;
      if (k == 1 && m->getBlockInfo(b, 0)->level != l) return -1;
    }
  }
  long long off = 0;
  for (int b = 0; b < nb; b++) {
    const int l = m->getBlockInfo(b, 0)->level;
    const int bs = bsx0 >> l, nv = bs * bs * bs;
    SparseGrid<uint16_t>* sg = m->getDistFineCoarseChannel(l);
    const uint16_t* d = (sg && sg->isValueBlock(b)) ? sg->getBlockDataPtr(b) : nullptr;
    for (int i = 0; i < nv; i++) out[off + i] = d ? d[i] : 0;
    off += nv;
  }
  return off;
}

// The reference's own linear interpolation of the distance channel of level
// `level` with Neumann borders, at n positions in that level's voxel units:
// the call interpVec3MSBG makes (src/flip_sim.cpp:1430-1432), without the
// division by 1024.
extern "C" void ref_mr_dist_interp(void* mp, int level, const float* pos, long long n,
                                   float* out) {
  auto* m = (MultiresSparseGrid*)mp;
  SparseGrid<uint16_t>* sg = m->getDistFineCoarseChannel(level);
  for (long long i = 0; i < n; i++) {
    float p[3] = {pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]};
    out[i] = sg ? sg->interpolateToFloat<IP_LINEAR>(p, OPT_IPBC_NEUMAN) : 0.f;
  }
}

namespace {
// The reference allocates a sparse grid's block map on first data access
// (SparseGrid::prepareDataAccess, src/sbg.cpp:702-720; its FLIP driver does
// it per channel); the vector channels of every (level, MG level) pair.
void ps_prepare_vec(MultiresSparseGrid* m, int ch) {
  for (int l = 0; l < m->getNumLevels(); l++)
    for (int lMg = 0; lMg <= l; lMg++) {
      SparseGrid<Vec3Float>* sg = m->getVecChannel(ch, l, lMg);
      if (sg && !sg->hasData()) sg->prepareDataAccess();
    }
}
}  // namespace

// Vector channel ch (CH_VEC3_*) of MG level levelMg in the packed layout, 3
// floats per voxel; -1 where the reference has no such channel at a block's
// level.  Missing blocks read 0 and are skipped on write (written with
// allocation when alloc != 0).
extern "C" int ref_ps_vec_channel(void* hp, int ch, int levelMg, float* data, int get,
                                  int alloc) {
  auto* m = ((PsHandle*)hp)->msbg;
  ps_prepare_vec(m, ch);
  const int bsx0 = m->sg0()->bsx();
  size_t off = 0;
  for (int b = 0; b < m->nBlocks(); b++) {
    const int l = m->getBlockInfo(b, levelMg)->level;
    const int bs = bsx0 >> l, nv = bs * bs * bs;
    SparseGrid<Vec3Float>* sg = m->getVecChannel(ch, l, levelMg);
    if (!sg) return -1;
    Vec3Float* d = sg->getBlockDataPtr(b, (!get && alloc) ? 1 : 0, 0);
    for (int i = 0; i < nv; i++) {
      if (get) {
        data[3 * (off + i)] = d ? d[i].x : 0.f;
        data[3 * (off + i) + 1] = d ? d[i].y : 0.f;
        data[3 * (off + i) + 2] = d ? d[i].z : 0.f;
      } else if (d) {
        d[i] = Vec3Float(data[3 * (off + i)], data[3 * (off + i) + 1], data[3 * (off + i) + 2]);
      }
    }
    off += nv;
  }
  return 0;
}

// downsampleVelocity(levelMg, chSrc, chDst) (src/msbg4.cpp:2035-2270): the
// velocity of MG level levelMg - 1 restricted to MG level levelMg.
extern "C" int ref_ps_downsample_velocity(void* hp, int levelMg, int chSrc, int chDst) {
  auto* m = ((PsHandle*)hp)->msbg;
  if (levelMg < 1 || levelMg >= m->getNumLevels()) return -1;
  ps_prepare_vec(m, chSrc);
  ps_prepare_vec(m, chDst);
  m->downsampleVelocity(levelMg, chSrc, chDst);
  return 0;
}

// Fills vector channel ch (CH_VEC3_*) of a grid made by ref_mr_create from the
// packed layout (3 floats per voxel, each block at its own level), as the
// reference's FLIP driver holds its velocity: getVecChannel(ch, level, 0) of
// every level, block maps prepared first (SparseGrid::prepareDataAccess,
// src/sbg.cpp:702-720).
extern "C" int ref_mr_set_vec(void* mp, int ch, const float* data) {
  auto* m = (MultiresSparseGrid*)mp;
  const int bsx0 = m->sg0()->bsx();
  for (int l = 0; l < m->getNumLevels(); l++) {
    SparseGrid<Vec3Float>* sg = m->getVecChannel(ch, l, 0);
    if (!sg) return -1;
    if (!sg->hasData()) sg->prepareDataAccess();
  }
  size_t off = 0;
  for (int b = 0; b < m->nBlocks(); b++) {
    const int l = m->getBlockInfo(b, 0)->level;
    const int bs = bsx0 >> l, nv = bs * bs * bs;
    Vec3Float* d = m->getVecChannel(ch, l, 0)->getBlockDataPtr(b, 1, 0);
    if (!d) return -1;
    for (int i = 0; i < nv; i++)
      d[i] = Vec3Float(data[3 * (off + i)], data[3 * (off + i) + 1], data[3 * (off + i) + 2]);
    off += nv;
  }
  return 0;
}
