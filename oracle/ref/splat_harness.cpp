// Particle-splatting capture harness (test infrastructure; never part of the
// GPU product).
//
// The reference's particle splatting lives inside its demo driver
// msbg_test_sparse (src/msbg_demo.cpp:228-767), which has no entry point for
// the splat alone.  This translation unit compiles that file as it stands
// (included from the reference tree, not copied) and observes three points of
// its run without changing what it computes:
//   - FREEMEM(particlesPerBlock) (src/msbg_demo.cpp:643): the per-block
//     particle lists are still alive; their particles' positions are copied;
//   - FREEMEM(particles) (src/msbg_demo.cpp:644): the splat loop has finished;
//     the channel holds the quantised minimum squared distances, copied;
//   - the call of applyChannelPdeFast<uint16_t> (src/msbg_demo.cpp:716): the
//     distance finalisation has finished; the channel and the active block
//     list are copied, and the run is left with longjmp (the smoothing and the
//     rendering that follow are not needed; the grid is not freed).
// The FREEMEM macro is redefined to call the observer first; its freeing
// behaviour is the reference's (src/mm.h:207-214).  The applyChannelPdeFast
// specialisation defined here takes the place of the reference's own
// instantiation for calls from this library (linked with -Bsymbolic-functions).
#include <chrono>
#include <csetjmp>
#include <cstdint>
#include <cstring>
#include <sstream>
#include <vector>

#include "tbb/tbb.h"
#include "common_headers.h"
#include "msbg.h"
#include "render.h"

namespace {

struct SplatCapture {
  int bsx = 0;
  int64_t nBlocks = 0;
  std::vector<float> pos;          // [n][3] the splatted particles
  std::vector<int> rawBlocks;      // value blocks at the end of the splat loop
  std::vector<uint16_t> raw;       // their voxels (quantised squared distances)
  std::vector<int> finalBlocks;    // the active block list after finalisation
  std::vector<uint16_t> finalVals; // their voxels (render density)
  bool done = false;
  // seconds from the call: the refinement map set (after the particle
  // positions, active-block marking and block lists), the splat loop ended,
  // the finalisation ended
  std::chrono::steady_clock::time_point t0;
  double tMarked = 0, tSplat = 0, tFinal = 0;
};

double since(const std::chrono::steady_clock::time_point& t0) {
  return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

SplatCapture* g_cap = nullptr;
std::jmp_buf g_jmp;

void copy_value_blocks(SBG::SparseGrid<uint16_t>* sg, std::vector<int>& ids,
                       std::vector<uint16_t>& vals) {
  ids.clear();
  vals.clear();
  const int nv = sg->nVoxelsInBlock();
  for (int bid = 0; bid < sg->nBlocks(); bid++) {
    if (!sg->isValueBlock(bid)) continue;
    const uint16_t* d = sg->getBlockDataPtr(bid);
    ids.push_back(bid);
    vals.insert(vals.end(), d, d + nv);
  }
}

void splat_free_observer(const char* name, const void* ptr, SBG::SparseGrid<uint16_t>* sg0);

}  // namespace

#undef FREEMEM
#define FREEMEM(objptr_)                                  \
  {                                                       \
    splat_free_observer(#objptr_, (const void*)(objptr_), sg0); \
    if (objptr_) {                                        \
      MM_free(objptr_);                                   \
      objptr_ = NULL;                                     \
    }                                                     \
  }

namespace MSBG {
template <>
void MultiresSparseGrid::applyChannelPdeFast<uint16_t>(
    int chPhi, int chTmp, int chTmp2, std::vector<int>* blockList, int laplTyp,
    int doConstrZeroOne, float densThr, float densThrTol1, float densThrTol2, int numIter,
    float gridSpacing, float timeStep, float velMagThr, MultiresSparseGrid* msgVel, float lambda,
    float lambdaSDF, float taubin, float redist, float anisDiffAlpha, int veldep_on,
    float* veldep_fit, int visOpt);
}

#include "msbg_demo.cpp"

namespace {

void splat_free_observer(const char* name, const void* ptr, SBG::SparseGrid<uint16_t>* sg0) {
  if (!g_cap || !ptr) return;
  if (std::strcmp(name, "blockActive") == 0 && !g_cap->done) {
    g_cap->tMarked = since(g_cap->t0);
  } else if (std::strcmp(name, "particlesPerBlock") == 0 && !g_cap->done) {
    g_cap->tSplat = since(g_cap->t0);
    // walk every block's list while the particles are alive
    const ParticleIdx* lists = static_cast<const ParticleIdx*>(ptr);
    g_cap->pos.clear();
    for (int bid = 0; bid < sg0->nBlocks(); bid++)
      for (ParticleIdx ixp = lists[bid]; ixp; ixp = particles[ixp].idxNext) {
        const Particle& p = particles[ixp];
        g_cap->pos.push_back(p.pos.x);
        g_cap->pos.push_back(p.pos.y);
        g_cap->pos.push_back(p.pos.z);
      }
  } else if (std::strcmp(name, "particles") == 0 && !g_cap->done) {
    copy_value_blocks(sg0, g_cap->rawBlocks, g_cap->raw);
  }
}

}  // namespace

namespace MSBG {
template <>
void MultiresSparseGrid::applyChannelPdeFast<uint16_t>(
    int chPhi, int, int, std::vector<int>* blockList, int, int, float, float, float, int, float,
    float, float, MultiresSparseGrid*, float, float, float, float, float, int, float*, int) {
  if (!g_cap) return;
  g_cap->tFinal = since(g_cap->t0);
  SBG::SparseGrid<uint16_t>* sg = getUint16Channel(chPhi, 0);
  std::vector<int> ids;
  copy_value_blocks(sg, ids, g_cap->finalVals);
  g_cap->finalBlocks.assign(blockList->begin(), blockList->end());
  std::sort(g_cap->finalBlocks.begin(), g_cap->finalBlocks.end());
  g_cap->bsx = sg->bsx();
  g_cap->nBlocks = sg->nBlocks();
  g_cap->done = true;
  std::longjmp(g_jmp, 1);
}
}  // namespace MSBG

namespace {
SplatCapture g_last;
}

// Runs msbg_test_sparse(testCase, plyPath, bsx0, sx, sy, sz) up to the
// smoothing call.  Returns 0 when the capture is complete; the sizes of the
// captured arrays are then available from ref_splat_sizes and the arrays
// from ref_splat_copy.
extern "C" int ref_splat_demo(int testCase, const char* plyPath, int bsx0, int sx, int sy,
                              int sz) {
  g_last = SplatCapture();
  g_last.t0 = std::chrono::steady_clock::now();
  g_cap = &g_last;
  if (setjmp(g_jmp) == 0) msbg_test_sparse(testCase, plyPath, bsx0, sx, sy, sz);
  g_cap = nullptr;
  return g_last.done ? 0 : 1;
}

// sizes[0] particles, [1] value blocks at the end of the splat, [2] active
// blocks after finalisation, [3] bsx, [4] blocks of the raster
extern "C" void ref_splat_sizes(int64_t* sizes) {
  sizes[0] = (int64_t)g_last.pos.size() / 3;
  sizes[1] = (int64_t)g_last.rawBlocks.size();
  sizes[2] = (int64_t)g_last.finalBlocks.size();
  sizes[3] = g_last.bsx;
  sizes[4] = g_last.nBlocks;
}

extern "C" void ref_splat_copy(float* pos, int* rawBlocks, uint16_t* raw, int* finalBlocks,
                               uint16_t* finalVals) {
  std::memcpy(pos, g_last.pos.data(), sizeof(float) * g_last.pos.size());
  std::memcpy(rawBlocks, g_last.rawBlocks.data(), sizeof(int) * g_last.rawBlocks.size());
  std::memcpy(raw, g_last.raw.data(), sizeof(uint16_t) * g_last.raw.size());
  std::memcpy(finalBlocks, g_last.finalBlocks.data(), sizeof(int) * g_last.finalBlocks.size());
  std::memcpy(finalVals, g_last.finalVals.data(), sizeof(uint16_t) * g_last.finalVals.size());
}

// times[0..2]: seconds from the call to the end of the marking phase, of the
// splat loop (block allocation and initialisation included), of the
// finalisation
extern "C" void ref_splat_times(double* times) {
  times[0] = g_last.tMarked;
  times[1] = g_last.tSplat;
  times[2] = g_last.tFinal;
}

// The demo's particle test (src/msbg_demo.cpp:358-360) on a grid created as
// the demo creates it: out[i] = isInDomainRange(p) && inRange(trunc(p)).
extern "C" int ref_splat_in_domain(int sx, int sy, int sz, int bsx0, const float* pts, int64_t n,
                                   int* out) {
  MSBG::MultiresSparseGrid* msbg = MSBG::MultiresSparseGrid::create(
      "TEST", sx, sy, sz, bsx0, -1, 0, -1,
      MSBG::OPT_SINGLE_LEVEL | MSBG::OPT_SINGLE_CHANNEL_FLOAT);
  if (!msbg) return 1;
  SBG::SparseGrid<uint16_t>* sg0 = msbg->getUint16Channel(MSBG::CH_UINT16_1, 0);
  for (int64_t i = 0; i < n; i++) {
    const Vec4f pos(pts[3 * i], pts[3 * i + 1], pts[3 * i + 2], 0.f);
    int keep = msbg->isInDomainRange(pos);
    if (keep) keep = sg0->inRange(truncate_to_int(pos));
    out[i] = keep ? 1 : 0;
  }
  MSBG::MultiresSparseGrid::destroy(msbg);
  return 0;
}
