// Integration adapter (test infrastructure; never part of the GPU product).
//
// Compiles the code blocks of INTEGRATION.md exactly as they stand (copied
// into oracle/_ref/integration_*.inc by oracle/ref/extract_snippets.py)
// against the reference's own headers, and runs them on real
// MultiresSparseGrid objects built by the reference harness
// (oracle/ref/ref_harness.cpp), so the tests can compare the drop-in's
// results with the reference routines the snippets replace.  Each function
// declares the variables its snippet expects from the reference call site
// (src/msbg_demo.cpp:716-727, src/flip_sim.cpp:1289-1304, 1526-1545).
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>

#include <omp.h>
#include "tbb/tbb.h"
#include <vectorclass/vectorclass.h>
#include "common_headers.h"
#include "msbg.h"

using namespace MSBG;
using namespace SBG;

#include "integration_header.inc"

extern "C" void* ref_grid_create_f32(int sx, int sy, int sz, int bsx, const int8_t* kind,
                                     float emptyVal, float fullVal, const float* values);
extern "C" void* ref_grid_create_u16(int sx, int sy, int sz, int bsx, const int8_t* kind,
                                     uint16_t emptyVal, uint16_t fullVal, const uint16_t* values);
extern "C" void ref_grid_read_f32(void* m, const int8_t* kind, float* values);
extern "C" void ref_grid_read_u16(void* m, const int8_t* kind, uint16_t* values);
extern "C" void ref_grid_destroy(void* m);
extern "C" void* ref_ps_grid(void* hp);

namespace {

// INTEGRATION.md "mcf_u16": the demo's render-density smoothing.
int run_mcf_u16(MultiresSparseGrid* msbg, int chan, std::vector<int>& activeBlocks, int nIterPde,
                float dt) {
#include "integration_mcf_u16.inc"
  return rc;
}

// INTEGRATION.md "mcf_f32": the same on an FP32 channel.
int run_mcf_f32(MultiresSparseGrid* msbg, int chan, std::vector<int>& activeBlocks, int nIter,
                float dt, int doConstrZeroOne) {
#include "integration_mcf_f32.inc"
  return rc;
}

// INTEGRATION.md "pressure": the FLIP pressure solve into CH_PRESSURE.
int run_pressure(MultiresSparseGrid* msbg, const FlipPressureCallbacks& cb,
                 const FlipPressureSolveParams& sp, msbg_gpu_solve_info* out) {
#include "integration_pressure.inc"
  *out = info;
  return rc;
}

// INTEGRATION.md "splat": the demo's splat and smoothing from particle
// positions into the render-density channel; the active blocks out.
int run_splat(MultiresSparseGrid* msbg, int chan, const std::vector<float>& pos, int nIterPde,
              float dt, std::vector<int>& activeOut) {
#include "integration_splat.inc"
  activeOut = activeBlocks;
  return rc;
}

// The FlipConfig field the G2P snippet reads (src/flip_sim.h:29-45).
struct G2pConfig {
  float flipAlpha;
};

// INTEGRATION.md "g2p_mr": gridToParticle on a mixed-resolution grid.
int run_g2p_mr(MultiresSparseGrid* msbg, msbg_flip_particle* P, int64_t np,
               const G2pConfig& cfg_) {
#include "integration_g2p_mr.inc"
  return rc;
}

}  // namespace

// The G2P snippet on a grid made by ref_mr_create whose CH_VEC3_4 / CH_VEC3_2
// channels were filled with ref_mr_set_vec; the particles are updated in place.
extern "C" int integ_g2p_mr(void* mrGrid, msbg_flip_particle* particles, int64_t np,
                            float flipAlpha) {
  G2pConfig cfg = {flipAlpha};
  return run_g2p_mr((MultiresSparseGrid*)mrGrid, particles, np, cfg);
}

// The demo's call on a single-level render-density grid: kind / values as in
// ref_mcf_u16; values are overwritten with the result.  Returns the snippet's
// status (MSBG_OK = 0).
extern "C" int integ_mcf_u16(int sx, int sy, int sz, int bsx, const int8_t* kind,
                             uint16_t emptyVal, uint16_t fullVal, uint16_t* values,
                             const int* update, int nUpdate, int nIterPde, float dt) {
  void* m = ref_grid_create_u16(sx, sy, sz, bsx, kind, emptyVal, fullVal, values);
  if (!m) return -1;
  std::vector<int> activeBlocks(update, update + nUpdate);
  const int rc = run_mcf_u16((MultiresSparseGrid*)m, CH_UINT16_1, activeBlocks, nIterPde, dt);
  ref_grid_read_u16(m, kind, values);
  ref_grid_destroy(m);
  return rc;
}

extern "C" int integ_mcf_f32(int sx, int sy, int sz, int bsx, const int8_t* kind, float emptyVal,
                             float fullVal, float* values, const int* update, int nUpdate,
                             int nIter, float dt, int clamp01) {
  void* m = ref_grid_create_f32(sx, sy, sz, bsx, kind, emptyVal, fullVal, values);
  if (!m) return -1;
  std::vector<int> activeBlocks(update, update + nUpdate);
  const int rc =
      run_mcf_f32((MultiresSparseGrid*)m, CH_FLOAT_1, activeBlocks, nIter, dt, clamp01);
  ref_grid_read_f32(m, kind, values);
  ref_grid_destroy(m);
  return rc;
}

// The pressure snippet on a grid the reference harness prepared
// (ref_ps_create); the solution lands in its CH_PRESSURE channel.
extern "C" int integ_pressure(void* refHandle, CellFlags (*cellType)(void*, int, int, int),
                              float (*face)(void*, int, int, int, int),
                              float (*rhs)(void*, int, int, int), void* user, float tol,
                              int maxIter, int* status, int* iterations, double* relRes) {
  FlipPressureCallbacks cb;
  cb.sampleCellType = cellType;
  cb.sampleFaceCoeff = face;
  cb.sampleRhs = rhs;
  cb.user = user;
  FlipPressureSolveParams sp;
  sp.tol = tol;
  sp.maxIter = maxIter;
  msbg_gpu_solve_info info = {};
  const int rc = run_pressure((MultiresSparseGrid*)ref_ps_grid(refHandle), cb, sp, &info);
  if (status) *status = info.status;
  if (iterations) *iterations = info.iterations;
  if (relRes) *relRes = info.relResidual;
  return rc;
}

// The splat snippet on a single-level grid of sx*sy*sz voxels in bsx^3 blocks
// with no blocks yet: active[nBlocks] receives 1 for the blocks it made value
// blocks, values their voxels after the smoothing (packed in bid order, room
// for every block).  Returns the snippet's status.
extern "C" int integ_splat(int sx, int sy, int sz, int bsx, const float* pos, int64_t n,
                           int nIterPde, float dt, int8_t* active, uint16_t* values) {
  const int nb = (sx / bsx) * (sy / bsx) * (sz / bsx);
  std::vector<int8_t> none(nb, 0);
  void* m = ref_grid_create_u16(sx, sy, sz, bsx, none.data(), 0, 65535, nullptr);
  if (!m) return -1;
  std::vector<float> p(pos, pos + 3 * n);
  std::vector<int> act;
  const int rc = run_splat((MultiresSparseGrid*)m, CH_UINT16_1, p, nIterPde, dt, act);
  std::memset(active, 0, nb);
  for (int b : act) active[b] = 1;
  ref_grid_read_u16(m, active, values);
  ref_grid_destroy(m);
  return rc;
}
