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

// Mean-curvature flow, 8-colour in-place scheme, FP32 channel.
// Mirrors msbg_demo.cpp:716-727 (applyChannelPdeFast with
// -(PDE_MEAN_CURVATURE+OPT_8_COLOR_SCHEME)) on a single-level grid.
//   kind[nBlocks], values packed for kind==1 blocks in ascending bid order.
//   update[nUpdate] = block ids handed to the smoother as its block list.
extern "C" int ref_mcf(int sx, int sy, int sz, int bsx, const int8_t* kind,
                       float emptyVal, float fullVal, float* values,
                       const int* update, int nUpdate, int numIter, float dt,
                       int clamp01, double* seconds) {
  MultiresSparseGrid* msbg = MultiresSparseGrid::create(
      "REF", sx, sy, sz, bsx, -1, 0, -1,
      MSBG::OPT_SINGLE_LEVEL | MSBG::OPT_SINGLE_CHANNEL_FLOAT);
  if (!msbg) return 1;
  const int nb = msbg->nBlocks();
  {
    std::vector<int> levels(nb, 0);
    msbg->regularizeRefinementMap(levels.data());
    msbg->setRefinementMap(levels.data(), NULL, -1, NULL, false);
  }
  const int chan = CH_FLOAT_1;
  SparseGrid<float>* sg = msbg->getFloatChannel(chan, 0);
  sg->reset();
  sg->prepareDataAccess();
  sg->setEmptyValue(emptyVal);
  sg->setFullValue(fullVal);
  const int nv = sg->nVoxelsInBlock();
  size_t off = 0;
  for (int bid = 0; bid < nb; bid++) {
    switch (kind[bid]) {
      case 1: {
        float* d = sg->getBlockDataPtr(bid, 1, 0);
        std::memcpy(d, values + off, sizeof(float) * nv);
        off += nv;
        break;
      }
      case 2: sg->setEmptyBlock(bid); break;
      case 3: sg->setFullBlock(bid); break;
      default: break;
    }
  }
  std::vector<int> blockList(update, update + nUpdate);
  auto t0 = std::chrono::steady_clock::now();
  msbg->applyChannelPdeFast<float>(chan, CH_NULL, CH_NULL, &blockList,
                                   -(PDE_MEAN_CURVATURE + OPT_8_COLOR_SCHEME),
                                   clamp01, 0, 0, 0, numIter, 1.0f, dt);
  auto t1 = std::chrono::steady_clock::now();
  if (seconds) *seconds = std::chrono::duration<double>(t1 - t0).count();
  off = 0;
  for (int bid = 0; bid < nb; bid++) {
    if (kind[bid] != 1) continue;
    const float* d = sg->getBlockDataPtr(bid);
    std::memcpy(values + off, d, sizeof(float) * nv);
    off += nv;
  }
  MultiresSparseGrid::destroy(msbg);
  return 0;
}
