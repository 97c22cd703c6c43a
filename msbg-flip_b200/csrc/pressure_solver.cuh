// Solver state and kernel launcher of the MGPCG pressure solve, shared by
// the solve (pressure.cu) and the component entry points (pressure_parts.cu).
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "common.cuh"
#include "pressure.h"
#include "pressure_kernels.cuh"
#include "vec_types.cuh"
#include "cnn.cuh"

namespace msbg {
namespace ps {

#include "tile_kernels.cuh"
#include "smooth_pipe.cuh"
#include "refine.cuh"
#include "cnn_features.cuh"

// ---------------------------------------------------------------------------
// solver state
// ---------------------------------------------------------------------------
struct Solver {
  Hierarchy H;
  int64_t h2dBytes = 0;
  int numSMs = 148;
  double prepareSeconds = 0, buildSeconds = 0;
  std::vector<std::unique_ptr<LevelDev>> dev;
  std::vector<LevelView> views;
  DeviceBuffer dCoarseInv, dCoarseCells;
  DeviceBuffer rhs0, d0, q0, z0, r0, partial, scal;
  DeviceBuffer x64, rin;  // FP64 solution and inner right-hand side of the refinement
  DeviceBuffer rinv;      // the inner right-hand side scaled and stored in 16 bits
  DeviceBuffer tq;        // A z of the learned two-stage preconditioner
  int maxPartial = 0;
  Scalars* hScal = nullptr;  // pinned
  int bsx0 = 0, nbx = 0, nby = 0, nbz = 0;
  std::vector<int> blockLevel;
  // learned networks (not owned: initial guess, per-V-cycle correction) and
  // the level-0 16^3 tiles they run on
  msbg_cnn* net = nullptr;
  msbg_cnn* netCorr = nullptr;
  int nCnnTiles = 0;
  float levelNorm = 0.f;
  DeviceBuffer cnnTiles, cnnLevel;          // [nCnnTiles] tile id, resolution level
  DeviceBuffer cFeat, cScale, cOff, cX0, cS1, cS2, guess, cIdx;
  std::vector<int> cnnTilesHost, cnnLevelHost;
  int cnnChunk = 0;
  bool haveX64 = false;  // x64 holds the solution of the last refined solve
  DeviceBuffer packTiles, packBuf;  // device-side packing into the block layout
  DeviceBuffer df;                  // packed x faces of the PCG direction d0
};

// Dynamic shared-memory limits of the kernels a level-0 vector type needs
// (coarse levels always run in FP32).  The limit is an attribute of the
// kernel on the current device, and every translation unit that includes
// this header has its own copies of the kernels: each entry point sets it on
// its own copies, on the context's device (a few host calls, no GPU work).
template <typename VT>
void set_kernel_attrs() {
  const int pipeSmem = (int)pipe::SMEM;
  cudaFuncSetAttribute(k_smooth<16, VT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)smooth_smem<16>());
  cudaFuncSetAttribute(k_smooth<8, VT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)smooth_smem<8>());
  cudaFuncSetAttribute(k_smooth_pipe16<VT, pipe::NT_SMOOTH>,
                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)pipe::SMEM_SMOOTH);
  cudaFuncSetAttribute(k_apply_pipe16<APPLY_MATVEC, VT, VT, pipe::NT_APPLY>,
                       cudaFuncAttributeMaxDynamicSharedMemorySize, pipeSmem);
  cudaFuncSetAttribute(k_apply_pipe16<APPLY_RESIDUAL, VT, float, pipe::NT_APPLY>,
                       cudaFuncAttributeMaxDynamicSharedMemorySize, pipeSmem);
}

// MSBG_PRESSURE_FACES=0 turns the packed x faces off (the halo then reads
// the neighbours' strided x planes); the results are the same bits.
inline bool packed_faces_enabled() {
  const char* e = std::getenv("MSBG_PRESSURE_FACES");
  return !(e && std::strcmp(e, "0") == 0);
}

#define TS_DISPATCH(ts, CALL)        \
  switch (ts) {                      \
    case 16: { constexpr int T = 16; CALL; } break; \
    case 8: { constexpr int T = 8; CALL; } break;   \
    case 4: { constexpr int T = 4; CALL; } break;   \
    case 2: { constexpr int T = 2; CALL; } break;   \
    case 1: break;                   \
    default: break;                  \
  }

// Launches the V-cycle and operator kernels.  VT is the storage type of the
// level-0 vectors; the coarser levels hold FP32 vectors (they carry 1/8 of
// the cells and the restricted right-hand sides grow by up to 8x per level).
template <typename VT>
struct Runner {
  Solver& S;
  cudaStream_t st;
  int nPre, nPost, inner;
  float coarseScale = 1.0f;
  int* err = nullptr;     // device flag set by kernels whose bounded wait gave up
  int numSMs = 148;
  bool usePipe = true;
  // the V-cycle keeps packed x faces of its x on every level that has them
  // (LevelDev::xf); callers that smooth a vector outside a V-cycle pass none
  bool useFaces = packed_faces_enabled();
  int64_t launches = 0;  // kernels launched through this runner

  template <typename V>
  V* faces(int m) {
    LevelDev& D = *S.dev[m];
    return useFaces && usePipe && D.xf.p && S.views[m].cxf ? D.xf.template as<V>() : nullptr;
  }

  const int* passList(int m) { return S.dev[m]->passTiles.template as<int>(); }
  const int* groupList(int m) { return S.dev[m]->groupTiles.template as<int>(); }

  // One smoothing sweep of MG level m: the (level, colour) passes in order
  // (pre) or in reverse order with the adjoint colour order inside (post).
  template <typename V>
  void smooth(int m, V* x, const V* b, bool post, V* xf = nullptr) {
    const Level& L = S.H.levels[m];
    const int np = (int)L.passes.size();
    for (int pi = 0; pi < np; pi++) {
      const Level::Pass& P = L.passes[post ? np - 1 - pi : pi];
      if (!P.count) continue;
      const int* lst = passList(m) + P.start;
      if (P.ts == 16 && usePipe) {
        const int grid = std::min(P.count, numSMs);
        // passes are contiguous tile-id ranges (register_tiles sorts by pass)
        k_smooth_pipe16<V, pipe::NT_SMOOTH><<<grid, pipe::NT_SMOOTH, pipe::SMEM_SMOOTH, st>>>(
            S.views[m], P.start, P.count, x, b, inner, post ? 1 : 0, err, xf);
      } else {
        TS_DISPATCH(P.ts, (k_smooth<T, V><<<P.count, T * T, smooth_smem<T>(), st>>>(
                               S.views[m], lst, x, b, inner, post ? 1 : 0)));
      }
      launches++;
    }
  }

  template <typename V>
  void vcycle(int m, V* x, const V* b) {
    const int last = (int)S.H.levels.size() - 1;
    const Level& L = S.H.levels[m];
    cudaMemsetAsync(x, 0, sizeof(V) * L.nCells, st);
    V* xf = m == last ? nullptr : faces<V>(m);
    if (xf) cudaMemsetAsync(xf, 0, sizeof(V) * xface_len(L.nCells), st);
    if (m == last) {
      k_coarse_solve<V><<<1, 512, 0, st>>>(S.dCoarseInv.template as<double>(), S.H.nCoarse,
                                           S.dCoarseCells.template as<int64_t>(), b, x);
      launches++;
      return;
    }
    for (int s = 0; s < nPre; s++) smooth(m, x, b, false, xf);
    LevelDev& C = *S.dev[m + 1];
    residual_restrict(m, x, b, xf);
    float* xc = C.x.template as<float>();
    vcycle<float>(m + 1, xc, C.b.template as<float>());
    for (const auto& g : L.groups) {
      const int* lst = groupList(m) + g.start;
      TS_DISPATCH(g.ts, (k_prolong<T, V, float><<<g.count, T * T, 0, st>>>(
                            S.views[m], lst, x, xc, C.tileOff.template as<int64_t>(),
                            coarseScale, xf)));
      launches++;
    }
    for (int s = 0; s < nPost; s++) smooth(m, x, b, true, xf);
  }

  // q = A d with partial d.q (level 0); returns the number of partials.
  // Passes are contiguous tile ranges of one tile size; 16^3 passes go
  // through the pipelined kernel, the others through the per-tile kernel.
  // df: packed x faces of d (nullptr: strided halo reads).
  int matvec_dot(const VT* d, VT* q, double* partial, const VT* df = nullptr) {
    const Level& L = S.H.levels[0];
    int off = 0;
    for (const auto& P : L.passes) {
      if (!P.count) continue;
      if (P.ts == 16 && usePipe) {
        const int grid = std::min(P.count, numSMs);
        k_apply_pipe16<APPLY_MATVEC, VT, VT, pipe::NT_APPLY><<<grid, pipe::NT_APPLY, pipe::SMEM, st>>>(
            S.views[0], P.start, P.count, d, nullptr, q, nullptr, nullptr, partial + off, err,
            S.views[0].cxf ? df : nullptr);
        off += grid;
      } else {
        const int* lst = passList(0) + P.start;
        TS_DISPATCH(P.ts, (k_matvec_dot<T, VT><<<P.count, T * T, 0, st>>>(S.views[0], lst, d, q,
                                                                           partial + off)));
        off += P.count;
      }
      launches++;
    }
    return off;
  }

  // r = b - A x on MG level m, restricted into the (FP32) right-hand side of m+1.
  template <typename V>
  void residual_restrict(int m, const V* x, const V* b, const V* xf = nullptr) {
    const Level& L = S.H.levels[m];
    LevelDev& C = *S.dev[m + 1];
    float* bc = C.b.template as<float>();
    const int64_t* coff = C.tileOff.template as<int64_t>();
    for (const auto& P : L.passes) {
      if (!P.count) continue;
      if (P.ts == 16 && usePipe) {
        const int grid = std::min(P.count, numSMs);
        k_apply_pipe16<APPLY_RESIDUAL, V, float, pipe::NT_APPLY><<<grid, pipe::NT_APPLY, pipe::SMEM, st>>>(
            S.views[m], P.start, P.count, x, b, nullptr, bc, coff, nullptr, err, xf);
      } else {
        const int* lst = passList(m) + P.start;
        TS_DISPATCH(P.ts, (k_residual_restrict<T, V, float><<<P.count, T * T, 0, st>>>(
                              S.views[m], lst, x, b, bc, coff)));
      }
      launches++;
    }
  }
};

// The prepared solver of a context (nullptr before msbg_gpu_pressure_prepare).
Solver* find_solver(msbg_gpu_ctx* ctx);

// msbg_gpu_pressure_prepare from the callbacks cb, or from the per-cell arrays
// arr (msbg_gpu_pressure_prepare_arrays) when arr is given (pressure.cu).
int pressure_prepare(msbg_gpu_ctx* ctx, const msbg_topo_desc* topo,
                     const msbg_pressure_callbacks* cb, const ArrayInput* arr);

// True when p points into page-locked host memory (pressure.cu).
bool host_pinned(const void* p);

// Host <-> device copies through pinned staging buffers (pressure.cu); a
// page-locked host side is copied directly.
cudaError_t copy_h2d(void* dst, const void* src, size_t bytes, cudaStream_t st);
cudaError_t copy_d2h(void* dst, const void* src, size_t bytes, cudaStream_t st);

}  // namespace ps
}  // namespace msbg
