// MGPCG pressure solve on the GPU: tile kernels, V-cycle, PCG driver, C ABI.
//
// Replaces MultiresSparseGrid::preparePressureSolveFLIP + solvePressureFLIP
// (src/msbg3.cpp:3041-3271).  Structure of one PCG iteration as in the
// reference (src/msbg3.cpp:3149-3236): q = A d, alpha = rho/(d.q),
// x += alpha d, r -= alpha q, z = V(r), beta = (r.z)/rho, d = z + beta d;
// stop when |r|^2 <= tol^2 |b|^2 or on breakdown.  Inner products and norms
// are FP64 (two-stage deterministic reductions with warp shuffles).  The
// V-cycle (src/msbg3.cpp:2412-2465) is pre-smooth, residual, restriction,
// recursion, prolongation, post-smooth; the smoother is a tile-wise
// red-black Gauss-Seidel with the tiles themselves visited in red-black
// order per resolution level (the reference visits blocks red-black too,
// src/msbg3.cpp:2185-2219); the post-smoother is the exact adjoint of the
// pre-smoother so the preconditioner is symmetric.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <string>
#include <type_traits>
#include <vector>

#include "pressure_solver.cuh"

using namespace msbg;
using namespace msbg::ps;

namespace {

std::map<msbg_gpu_ctx*, std::unique_ptr<Solver>>& solvers() {
  static std::map<msbg_gpu_ctx*, std::unique_ptr<Solver>> m;
  return m;
}

std::unique_ptr<Solver>& solver_of(msbg_gpu_ctx* ctx) { return solvers()[ctx]; }

template <typename V>
cudaError_t upload(DeviceBuffer& buf, const V& v, cudaStream_t st) {
  using T = typename V::value_type;
  cudaError_t e = buf.ensure(sizeof(T) * std::max<size_t>(v.size(), 1));
  if (e != cudaSuccess) return e;
  if (v.empty()) return cudaSuccess;
  return copy_h2d(buf.p, v.data(), sizeof(T) * v.size(), st);
}

}  // namespace

namespace msbg {
namespace ps {

Solver* find_solver(msbg_gpu_ctx* ctx) {
  auto it = solvers().find(ctx);
  return it == solvers().end() ? nullptr : it->second.get();
}

// Host -> device copies of the prepared arrays.  Large arrays go through two
// pinned 64 MB staging buffers of the calling thread: a parallel memcpy fills
// one while the DMA of the other runs (a pageable copy is staged by the
// driver on one thread at a few GB/s).
struct PinnedStaging {
  static constexpr size_t CH = 64u << 20;
  void* buf[2] = {nullptr, nullptr};
  cudaEvent_t ev[2] = {nullptr, nullptr};
  int device = -1;
  bool used[2] = {false, false};
  ~PinnedStaging() {
    for (int i = 0; i < 2; i++) {
      if (ev[i]) cudaEventDestroy(ev[i]);
      if (buf[i]) cudaFreeHost(buf[i]);
    }
  }
  bool ready(int dev) {
    if (device == dev) return true;
    if (device >= 0) return false;  // one device per host thread
    for (int i = 0; i < 2; i++)
      if (cudaMallocHost(&buf[i], CH) != cudaSuccess ||
          cudaEventCreateWithFlags(&ev[i], cudaEventDisableTiming) != cudaSuccess)
        return false;
    device = dev;
    return true;
  }
};

PinnedStaging& staging() {
  thread_local PinnedStaging stg;
  return stg;
}

// True when p points into page-locked host memory (cudaMallocHost,
// cudaHostRegister, a pinned torch tensor): the DMA then reads or writes it
// directly, with no staging copy.
bool host_pinned(const void* p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();  // pageable memory may report an error on older drivers
    return false;
  }
  return a.type == cudaMemoryTypeHost;
}

cudaError_t copy_h2d(void* dst, const void* src, size_t bytes, cudaStream_t st) {
  PinnedStaging& stg = staging();
  int dev = 0;
  cudaGetDevice(&dev);
  if (bytes < (8u << 20) || host_pinned(src) || !stg.ready(dev))
    return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, st);
  for (size_t o = 0, c = 0; o < bytes; o += PinnedStaging::CH, c++) {
    const int k = (int)(c & 1);
    const size_t len = std::min(PinnedStaging::CH, bytes - o);
    if (stg.used[k]) {
      cudaError_t e = cudaEventSynchronize(stg.ev[k]);
      if (e != cudaSuccess) return e;
    }
    const char* s = static_cast<const char*>(src) + o;
    char* d = static_cast<char*>(stg.buf[k]);
    const int64_t parts = 16;
#pragma omp parallel for schedule(static)
    for (int64_t q = 0; q < parts; q++) {
      const size_t a = len * q / parts, b = len * (q + 1) / parts;
      std::memcpy(d + a, s + a, b - a);
    }
    cudaError_t e = cudaMemcpyAsync(static_cast<char*>(dst) + o, d, len, cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return e;
    e = cudaEventRecord(stg.ev[k], st);
    if (e != cudaSuccess) return e;
    stg.used[k] = true;
  }
  return cudaSuccess;
}

// Device -> host into pageable memory, through the same staging buffers: the
// DMA of chunk c+1 runs while chunk c is copied out in parallel.  Returns
// after the last byte has landed.
cudaError_t copy_d2h(void* dst, const void* src, size_t bytes, cudaStream_t st) {
  PinnedStaging& stg = staging();
  int dev = 0;
  cudaGetDevice(&dev);
  if (bytes < (8u << 20) || host_pinned(dst) || !stg.ready(dev)) {
    cudaError_t e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, st);
    return e != cudaSuccess ? e : cudaStreamSynchronize(st);
  }
  const size_t CH = PinnedStaging::CH;
  const size_t nch = (bytes + CH - 1) / CH;
  auto issue = [&](size_t c) {
    const int k = (int)(c & 1);
    const size_t o = c * CH, len = std::min(CH, bytes - o);
    cudaError_t e = cudaMemcpyAsync(stg.buf[k], static_cast<const char*>(src) + o, len,
                                    cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaEventRecord(stg.ev[k], st);
    stg.used[k] = true;
    return e;
  };
  cudaError_t e = issue(0);
  for (size_t c = 0; c < nch && e == cudaSuccess; c++) {
    const int k = (int)(c & 1);
    const size_t o = c * CH, len = std::min(CH, bytes - o);
    e = cudaEventSynchronize(stg.ev[k]);
    if (e != cudaSuccess) break;
    if (c + 1 < nch) {
      // the other buffer was copied out in the previous round
      e = issue(c + 1);
      if (e != cudaSuccess) break;
    }
    const char* s = static_cast<const char*>(stg.buf[k]);
    char* d = static_cast<char*>(dst) + o;
    const int64_t parts = 16;
#pragma omp parallel for schedule(static)
    for (int64_t q = 0; q < parts; q++) {
      const size_t a = len * q / parts, b = len * (q + 1) / parts;
      std::memcpy(d + a, s + a, b - a);
    }
  }
  return e;
}

}  // namespace ps
}  // namespace msbg

namespace msbg {
void pressure_release(msbg_gpu_ctx* ctx) {
  auto it = solvers().find(ctx);
  if (it == solvers().end()) return;
  if (it->second && it->second->hScal) cudaFreeHost(it->second->hScal);
  solvers().erase(it);
}
}  // namespace msbg

extern "C" void msbg_gpu_solve_params_default(msbg_gpu_solve_params* p) {
  if (!p) return;
  p->nPre = 2;
  p->nPost = 2;
  p->nCoarse = 24;
  p->maxIter = 500;
  p->tol = 1e-6f;
  p->innerIter = 3;
  p->storage = MSBG_F32;
  p->maxRefine = 0;  // plain MGPCG on the recursive residual, as the reference
  p->useGraph = 1;
  // Piecewise-constant transfers with Galerkin coarse operators under-correct
  // smooth errors; scaling the coarse correction by 1.8 restores
  // size-independent convergence (10-13 PCG iterations from 256^3 to 1024^3).
  p->coarseScale = 1.8f;
  p->learned = 0;
}

extern "C" int msbg_gpu_pressure_prepare(msbg_gpu_ctx* ctx, const msbg_topo_desc* topo,
                                         const msbg_pressure_callbacks* cb) {
  if (!ctx || !topo || !cb || !cb->sampleCellType || !cb->sampleFaceCoeff || !cb->sampleRhs)
    return MSBG_EINVARG;
  return msbg::ps::pressure_prepare(ctx, topo, cb, nullptr);
}

int msbg::ps::pressure_prepare(msbg_gpu_ctx* ctx, const msbg_topo_desc* topo,
                               const msbg_pressure_callbacks* cb, const ArrayInput* arr) {
  int rc = msbg_gpu_sync_topology(ctx, topo);
  if (rc) return rc;
  cudaSetDevice(ctx->device);
  auto& sp = solver_of(ctx);
  sp.reset(new Solver());
  Solver& S = *sp;
  std::string err;
  auto tp0 = std::chrono::steady_clock::now();
  // per-cell arrays: the per-cell work of the build runs on the GPU (set
  // MSBG_PRESSURE_BUILD=host to build them on the host as the callbacks are)
  const char* bsel = getenv("MSBG_PRESSURE_BUILD");
  const bool onDeviceReq = arr && !(bsel && std::strcmp(bsel, "host") == 0);
  std::vector<std::unique_ptr<LevelDev>> built;
  bool onDevice = onDeviceReq;
  if (onDevice) {
    rc = build_hierarchy_device(S.H, built, S.rhs0, topo->sx, topo->sy, topo->sz, topo->bsx0,
                                topo->nLevels, topo->blockLevel, topo->domainBc, *arr, 512,
                                ctx->stream, &err);
    if (rc == MSBG_ENOTIMPL) {  // no staging for this device on this thread: host build
      onDevice = false;
      built.clear();
      err.clear();
    }
  }
  if (!onDevice)
    rc = build_hierarchy(S.H, topo->sx, topo->sy, topo->sz, topo->bsx0, topo->nLevels,
                         topo->blockLevel, topo->domainBc, cb, 512, &err, arr);
  S.buildSeconds =
      std::chrono::duration<double>(std::chrono::steady_clock::now() - tp0).count();
  if (rc) {
    sp.reset();
    return set_error(ctx, rc, "pressure prepare: %s", err.c_str());
  }
  for (size_t m = 0; m + 1 < S.H.levels.size(); m++)
    for (const Tile& t : S.H.levels[m].tiles)
      if (t.ts < 2 || t.ts > TS_MAX) {
        sp.reset();
        return set_error(ctx, MSBG_EINVARG, "grid dimensions give %d-cell tiles at MG level %d",
                         t.ts, (int)m);
      }
  set_kernel_attrs<float>();
  set_kernel_attrs<__half>();
  set_kernel_attrs<__nv_bfloat16>();
  cudaDeviceGetAttribute(&S.numSMs, cudaDevAttrMultiProcessorCount, ctx->device);
  S.bsx0 = topo->bsx0;
  S.nbx = ctx->nbx;
  S.nby = ctx->nby;
  S.nbz = ctx->nbz;
  S.blockLevel = ctx->blockLevel;
  cudaStream_t st = ctx->stream;
  int maxPartial = VEC_GRID;
  for (size_t m = 0; m < S.H.levels.size(); m++) {
    const Level& L = S.H.levels[m];
    // the operator of a device build is in place already
    auto D = onDevice ? std::move(built[m]) : std::make_unique<LevelDev>();
    std::vector<int64_t> toff(L.tiles.size());
    for (size_t i = 0; i < L.tiles.size(); i++) toff[i] = L.tiles[i].off;
    MSBG_CUDA_TRY(ctx, upload(D->tileOff, toff, st));
    MSBG_CUDA_TRY(ctx, upload(D->face, L.face, st));
    if (!onDevice) MSBG_CUDA_TRY(ctx, upload(D->ifOff, L.ifOff, st));
    MSBG_CUDA_TRY(ctx, upload(D->toCoarse, L.toCoarse, st));
    MSBG_CUDA_TRY(ctx, upload(D->passTiles, L.passTiles, st));
    MSBG_CUDA_TRY(ctx, upload(D->groupTiles, L.groupTiles, st));
    if (!onDevice) {
      MSBG_CUDA_TRY(ctx, upload(D->diag, L.diag, st));
      if (m == 0) MSBG_CUDA_TRY(ctx, upload(D->ctype, L.ctype, st));
    }
    {
      if (!onDevice) {
        HostArray<float> inv;
        inv.resize(L.diag.size());
        const int64_t nInv = (int64_t)inv.size();
#pragma omp parallel for schedule(static)
        for (int64_t c = 0; c < nInv; c++)
          inv[c] = L.diag[c] > 0.f ? (float)(1.0 / (double)L.diag[c]) : 0.f;
        MSBG_CUDA_TRY(ctx, upload(D->invdiag, inv, st));
        MSBG_CUDA_TRY(ctx, cudaStreamSynchronize(st));  // inv is a temporary
      }
      MSBG_CUDA_TRY(ctx, upload(D->tileRec, build_tile_records(L), st));
      // the hot-path kernels address passes as contiguous tile-id ranges
      for (size_t i = 0; i < L.passTiles.size(); i++)
        if (L.passTiles[i] != (int)i)
          return set_error(ctx, MSBG_EINTERNAL, "pass tiles are not contiguous");
      MSBG_CUDA_TRY(ctx, cudaStreamSynchronize(st));  // host vectors above are temporaries
    }
    if (!onDevice) {
      MSBG_CUDA_TRY(ctx, upload(D->cx, L.cx, st));
      MSBG_CUDA_TRY(ctx, upload(D->cy, L.cy, st));
      MSBG_CUDA_TRY(ctx, upload(D->cz, L.cz, st));
      MSBG_CUDA_TRY(ctx, upload(D->ifc, L.ifc, st));
    }
    const size_t nb = sizeof(float) * std::max<int64_t>(L.nCells, 4);
    MSBG_CUDA_TRY(ctx, D->x.ensure(nb));
    MSBG_CUDA_TRY(ctx, D->b.ensure(nb));
    // Coarse cells whose finer tiles do not exist are never written by the
    // restriction; they must read as 0 (not as recycled device memory).
    MSBG_CUDA_TRY(ctx, cudaMemsetAsync(D->x.p, 0, nb, st));
    MSBG_CUDA_TRY(ctx, cudaMemsetAsync(D->b.p, 0, nb, st));
    maxPartial = std::max(maxPartial, (int)L.tiles.size());
    // packed x faces on levels with 16^3 passes: the x = 0 plane of cx,
    // gathered once, and room for the faces of the V-cycle's x
    bool has16 = false;
    for (const auto& P : L.passes) has16 |= P.ts == 16 && P.count > 0;
    if (has16 && m + 1 < S.H.levels.size()) {
      const size_t nf = (size_t)xface_words(L.nCells);
      MSBG_CUDA_TRY(ctx, D->cxf.ensure(sizeof(float) * (nf / 2 + 256)));
      MSBG_CUDA_TRY(ctx, D->xf.ensure(sizeof(float) * nf));
      MSBG_CUDA_TRY(ctx, cudaMemsetAsync(D->xf.p, 0, sizeof(float) * nf, st));
      for (const auto& P : L.passes)
        if (P.ts == 16 && P.count > 0)
          k_pack_cx_plane<16><<<P.count, 256, 0, st>>>(D->tileOff.as<int64_t>(), P.start,
                                                   D->cx.as<float>(), D->cxf.as<float>());
      MSBG_CUDA_TRY(ctx, cudaGetLastError());
    }
    LevelView v;
    v.tileOff = D->tileOff.as<int64_t>();
    v.face = D->face.as<int>();
    v.ifOff = D->ifOff.as<int64_t>();
    v.toCoarse = D->toCoarse.as<int>();
    v.diag = D->diag.as<float>();
    v.invdiag = D->invdiag.as<float>();
    v.tileRec = D->tileRec.p;
    v.cx = D->cx.as<float>();
    v.cy = D->cy.as<float>();
    v.cz = D->cz.as<float>();
    v.ifc = D->ifc.as<float>();
    v.cxf = D->cxf.p ? D->cxf.as<float>() : nullptr;
    S.views.push_back(v);
    if (m == 0) {
      // tiles the learned network runs on: the 16^3 tiles of level 0
      std::vector<int> ids, lv;
      int maxLv = 0;
      for (size_t i = 0; i < L.tiles.size(); i++) {
        maxLv = std::max(maxLv, L.tiles[i].level);
        if (L.tiles[i].ts == cnn::TS) {
          ids.push_back((int)i);
          lv.push_back(L.tiles[i].level);
        }
      }
      S.nCnnTiles = (int)ids.size();
      S.cnnTilesHost = ids;
      S.cnnLevelHost = lv;
      S.levelNorm = 1.0f / (float)std::max(1, topo->nLevels - 1);
      MSBG_CUDA_TRY(ctx, upload(S.cnnTiles, ids, st));
      MSBG_CUDA_TRY(ctx, upload(S.cnnLevel, lv, st));
      MSBG_CUDA_TRY(ctx, cudaStreamSynchronize(st));  // host vectors are temporaries
    }
    S.dev.push_back(std::move(D));
  }
  const Level& L0 = S.H.levels[0];
  const size_t n0 = sizeof(float) * L0.nCells;
  if (!onDevice) MSBG_CUDA_TRY(ctx, upload(S.rhs0, L0.rhs, st));
  MSBG_CUDA_TRY(ctx, S.d0.ensure(n0));
  MSBG_CUDA_TRY(ctx, S.q0.ensure(n0));
  MSBG_CUDA_TRY(ctx, S.z0.ensure(n0));
  MSBG_CUDA_TRY(ctx, S.r0.ensure(n0));
  MSBG_CUDA_TRY(ctx, S.partial.ensure(sizeof(double) * maxPartial));
  S.maxPartial = maxPartial;
  MSBG_CUDA_TRY(ctx, S.scal.ensure(sizeof(Scalars)));
  MSBG_CUDA_TRY(ctx, upload(S.dCoarseInv, S.H.coarseInv, st));
  MSBG_CUDA_TRY(ctx, upload(S.dCoarseCells, S.H.coarseCells, st));
  MSBG_CUDA_TRY(ctx, cudaMallocHost(&S.hScal, sizeof(Scalars)));
  MSBG_CUDA_TRY(ctx, cudaStreamSynchronize(st));
  for (const auto& D : S.dev)
    S.h2dBytes += (int64_t)(D->tileOff.bytes + D->face.bytes + D->ifOff.bytes +
                            D->toCoarse.bytes + D->passTiles.bytes + D->groupTiles.bytes +
                            (onDevice ? 0
                                      : D->diag.bytes + D->cx.bytes + D->cy.bytes +
                                            D->cz.bytes + D->ifc.bytes));
  S.h2dBytes += (int64_t)(S.dCoarseInv.bytes + S.dCoarseCells.bytes) +
                (onDevice ? S.H.deviceBuildH2D : (int64_t)S.rhs0.bytes);
  S.prepareSeconds =
      std::chrono::duration<double>(std::chrono::steady_clock::now() - tp0).count();
  return MSBG_OK;
}

namespace {

struct PcgResult {
  int iters = 0;
  int status = 1;  // 0 converged, 1 maxIter, 2 breakdown, 3 non-finite
  double bb = 0;
};

// MGPCG on MG level 0 for A e = bin from e = 0 (e in the level-0 x vector),
// stopping at |r| <= tolRel |bin| (recursive residual, as the reference).
// One iteration is one CUDA graph launch; the graph is captured on the first
// call and reused (all buffers are fixed).
template <typename VT>
int run_pcg(msbg_gpu_ctx* ctx, Solver& S, Runner<VT>& R, const VT* bin, double tolRel,
            int maxIter, bool useGraph, cudaGraphExec_t& exec, int64_t& perIter,
            PcgResult& out) {
  cudaStream_t st = R.st;
  const int64_t n = S.H.levels[0].nCells;
  VT* x = S.dev[0]->x.as<VT>();
  VT* r = S.r0.as<VT>();
  VT* d = S.d0.as<VT>();
  VT* q = S.q0.as<VT>();
  VT* z = S.z0.as<VT>();
  double* part = S.partial.as<double>();
  Scalars* sc = S.scal.as<Scalars>();
  // r = b, x = 0, bb = b.b, z = V(r), rho = r.z, d = z
  cudaMemsetAsync(sc, 0, sizeof(Scalars), st);
  cudaMemsetAsync(x, 0, sizeof(VT) * n, st);
  cudaMemcpyAsync(r, bin, sizeof(VT) * n, cudaMemcpyDeviceToDevice, st);
  k_dot<<<VEC_GRID, VEC_BLOCK, 0, st>>>(bin, bin, n, part);
  k_finalize<<<1, 1024, 0, st>>>(part, VEC_GRID, sc, FIN_BB);
  // packed x faces of the direction d, kept by the same updates as d from
  // the faces of z that the V-cycle leaves (d = z, then d = z + beta d)
  VT* zf = R.template faces<VT>(0);
  const int64_t nf = xface_words(n);
  if (zf) MSBG_CUDA_TRY(ctx, S.df.ensure(sizeof(float) * nf));
  VT* df = zf ? S.df.as<VT>() : nullptr;
  R.vcycle(0, z, r);
  k_dot<<<VEC_GRID, VEC_BLOCK, 0, st>>>(r, z, n, part);
  k_finalize<<<1, 1024, 0, st>>>(part, VEC_GRID, sc, FIN_RHO);
  cudaMemcpyAsync(d, z, sizeof(VT) * n, cudaMemcpyDeviceToDevice, st);
  if (df) cudaMemcpyAsync(df, zf, sizeof(VT) * nf, cudaMemcpyDeviceToDevice, st);
  cudaMemcpyAsync(S.hScal, sc, sizeof(Scalars), cudaMemcpyDeviceToHost, st);
  R.launches += 4;
  MSBG_CUDA_TRY(ctx, cudaStreamSynchronize(st));
  out = PcgResult();
  out.bb = S.hScal->bb;
  if (!std::isfinite(out.bb) || !std::isfinite(S.hScal->rho)) {
    out.status = 3;
    return MSBG_OK;
  }
  if (!(out.bb > 1e-300)) {
    out.status = 0;
    return MSBG_OK;
  }
  auto iteration = [&]() {
    R.launches += 6;  // finalize x3, axpy_norm, dot, update_d
    int nt = R.matvec_dot(d, q, part, df);
    k_finalize<<<1, 1024, 0, st>>>(part, nt, sc, FIN_DQ_ALPHA);
    k_axpy_norm<<<VEC_GRID, VEC_BLOCK, 0, st>>>(x, r, d, q, n, sc, part);
    k_finalize<<<1, 1024, 0, st>>>(part, VEC_GRID, sc, FIN_RR);
    R.vcycle(0, z, r);
    k_dot<<<VEC_GRID, VEC_BLOCK, 0, st>>>(r, z, n, part);
    k_finalize<<<1, 1024, 0, st>>>(part, VEC_GRID, sc, FIN_RHONEW_BETA);
    k_update_d<<<VEC_GRID, VEC_BLOCK, 0, st>>>(d, z, n, sc);
    if (df) {
      k_update_d<<<VEC_GRID, VEC_BLOCK, 0, st>>>(df, zf, nf, sc);
      R.launches++;
    }
    cudaMemcpyAsync(S.hScal, sc, sizeof(Scalars), cudaMemcpyDeviceToHost, st);
  };
  if (useGraph && !exec) {
    const int64_t before = R.launches;
    cudaGraph_t g;
    MSBG_CUDA_TRY(ctx, cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    iteration();
    MSBG_CUDA_TRY(ctx, cudaStreamEndCapture(st, &g));
    perIter = R.launches - before;
    R.launches = before;
    MSBG_CUDA_TRY(ctx, cudaGraphInstantiate(&exec, g, 0));
    cudaGraphDestroy(g);
  }
  const double tol2 = tolRel * tolRel;
  for (int it = 0; it < maxIter; it++) {
    if (exec) {
      MSBG_CUDA_TRY(ctx, cudaGraphLaunch(exec, st));
      R.launches += perIter;
    } else {
      iteration();
    }
    MSBG_CUDA_TRY(ctx, cudaStreamSynchronize(st));
    out.iters = it + 1;
    const Scalars hs = *S.hScal;
    if (hs.status) {
      // a breakdown found before the update leaves x, r unchanged
      out.status = hs.status;
      break;
    }
    if (hs.rr <= tol2 * out.bb) {
      out.status = 0;
      break;
    }
  }
  return MSBG_OK;
}

// r32 = b - A x64 (FP64) on level 0; returns |r|^2 in *rr.
template <typename VT>
int residual64(msbg_gpu_ctx* ctx, Solver& S, Runner<VT>& R, const float* b, float* r32,
               double* rr) {
  cudaStream_t st = R.st;
  const Level& L = S.H.levels[0];
  double* part = S.partial.as<double>();
  int off = 0;
  for (const auto& g : L.groups) {
    const int* lst = S.dev[0]->groupTiles.as<int>() + g.start;
    TS_DISPATCH(g.ts, (k_residual64<T><<<g.count, T * T * res64_split<T>(), 0, st>>>(
                          S.views[0], lst, S.x64.as<double>(), b, r32, part + off)));
    off += g.count;
    R.launches++;
  }
  Scalars* sc = S.scal.as<Scalars>();
  k_finalize<<<1, 1024, 0, st>>>(part, off, sc, FIN_RR);
  cudaMemcpyAsync(S.hScal, sc, sizeof(Scalars), cudaMemcpyDeviceToHost, st);
  R.launches++;
  MSBG_CUDA_TRY(ctx, cudaStreamSynchronize(st));
  *rr = S.hScal->rr;
  return MSBG_OK;
}

// max |v| over the n level-0 values of v.
template <typename VT, typename V>
int absmax(msbg_gpu_ctx* ctx, Solver& S, Runner<VT>& R, const V* v, int64_t n, double* m) {
  cudaStream_t st = R.st;
  Scalars* sc = S.scal.as<Scalars>();
  k_absmax<<<VEC_GRID, VEC_BLOCK, 0, st>>>(v, n, S.partial.as<double>());
  k_finalize_max<<<1, 32, 0, st>>>(S.partial.as<double>(), VEC_GRID, sc);
  cudaMemcpyAsync(S.hScal, sc, sizeof(Scalars), cudaMemcpyDeviceToHost, st);
  R.launches += 2;
  MSBG_CUDA_TRY(ctx, cudaStreamSynchronize(st));
  *m = S.hScal->amax;
  return MSBG_OK;
}

struct SolveOut {
  int iters = 0, status = 1, refinements = 0;
  double relres = 0;
  double initialRelres = 1;  // |b - A x0| / |b| of the starting iterate
};

// Plain MGPCG on the FP32 right-hand side, stopping on the recursive
// residual (the reference's criterion); relres is the true FP32 residual.
int solve_plain(msbg_gpu_ctx* ctx, Solver& S, Runner<float>& R, const msbg_gpu_solve_params* p,
                cudaGraphExec_t& exec, int64_t& perIter, cudaEvent_t e1, SolveOut& o) {
  cudaStream_t st = R.st;
  const int64_t n = S.H.levels[0].nCells;
  float* x = S.dev[0]->x.as<float>();
  const float* b = S.rhs0.as<float>();
  PcgResult pr;
  int rc = run_pcg(ctx, S, R, b, p->tol, p->maxIter, p->useGraph, exec, perIter, pr);
  o.iters = pr.iters;
  o.status = pr.status;
  cudaEventRecord(e1, st);
  if (rc) return rc;
  // true residual of the FP32 iterate, FP32 operator, FP64 norm
  float* q = S.q0.as<float>();
  float* z = S.z0.as<float>();
  float* d = S.d0.as<float>();
  double* part = S.partial.as<double>();
  Scalars* sc = S.scal.as<Scalars>();
  R.matvec_dot(x, q, part);
  cudaMemcpyAsync(z, b, sizeof(float) * n, cudaMemcpyDeviceToDevice, st);
  Scalars one{};
  one.alpha = 1.0;
  cudaMemcpyAsync(sc, &one, sizeof(Scalars), cudaMemcpyHostToDevice, st);
  k_axpy_norm<<<VEC_GRID, VEC_BLOCK, 0, st>>>(d, z, q, q, n, sc, part);  // z = b - q
  k_finalize<<<1, 1024, 0, st>>>(part, VEC_GRID, sc, FIN_RR);
  cudaMemcpyAsync(S.hScal, sc, sizeof(Scalars), cudaMemcpyDeviceToHost, st);
  MSBG_CUDA_TRY(ctx, cudaStreamSynchronize(st));
  o.relres = pr.bb > 0 ? std::sqrt(S.hScal->rr / pr.bb) : 0.0;
  return MSBG_OK;
}

// Learned prediction from a level-0 FP32 vector `val` (right-hand side or
// residual) into out (all level-0 cells; cells of tiles the network does not
// cover stay 0), in chunks of up to 4096 tiles.
int learned_predict(msbg_gpu_ctx* ctx, Solver& S, msbg_cnn* net, cudaStream_t st, const float* val,
                    float* out, int64_t& launches, bool inGraph = false) {
  const int64_t n = S.H.levels[0].nCells;
  MSBG_CUDA_TRY(ctx, cudaMemsetAsync(out, 0, sizeof(float) * n, st));
  if (!S.nCnnTiles) return MSBG_OK;
  const int CH = std::min(4096, S.nCnnTiles);
  if (S.cnnChunk < CH) {
    MSBG_CUDA_TRY(ctx, S.cFeat.ensure(sizeof(float) * CH * cnn::NFEAT * cnn::NPAD));
    MSBG_CUDA_TRY(ctx, S.cScale.ensure(sizeof(float) * CH));
    MSBG_CUDA_TRY(ctx, S.cOff.ensure(sizeof(int64_t) * CH));
    for (DeviceBuffer* b : {&S.cX0, &S.cS1, &S.cS2}) {
      MSBG_CUDA_TRY(ctx, b->ensure(cnn::ACT_BYTES * CH));
      MSBG_CUDA_TRY(ctx, cudaMemsetAsync(b->p, 0, cnn::ACT_BYTES * CH, st));  // zero halos
    }
    S.cnnChunk = CH;
  }
  for (int c0 = 0; c0 < S.nCnnTiles; c0 += CH) {
    const int cnt = std::min(CH, S.nCnnTiles - c0);
    k_cnn_features<<<cnt, FEAT_THREADS, 0, st>>>(
        S.views[0], S.dev[0]->ctype.as<uint8_t>(), S.cnnTiles.as<int>() + c0,
        S.cnnLevel.as<int>() + c0, S.levelNorm, val, nullptr, S.cFeat.as<float>(),
        S.cScale.as<float>(), S.cOff.as<int64_t>(), nullptr, nullptr);
    if (cnn::forward(net, S.cFeat.as<float>(), out, S.cOff.as<int64_t>(), S.cScale.as<float>(),
                     cnt, st, S.cX0.as<uint4>(), S.cS1.as<uint4>(), S.cS2.as<uint4>()))
      return set_error(ctx, MSBG_ERROR, "learned network launch failed");
    launches += 6;
  }
  if (inGraph) return MSBG_OK;  // no host sync inside a capture; checked after the solve
  MSBG_CUDA_TRY(ctx, cudaGetLastError());
  const int e = cnn::take_error(net, st);
  if (e) return set_error(ctx, e, "learned network: a tensor-core wait gave up");
  return MSBG_OK;
}

// x64 = omega g: the guess g the network predicts from b, scaled by the
// energy-optimal omega = (g.b)/(g.Ag), so that |x* - x64|_A <= |x*|_A
// whatever the network returns.  Leaves r32 = b - A g.
template <typename VT>
int learned_start(msbg_gpu_ctx* ctx, Solver& S, Runner<VT>& R, const float* b, float* r32) {
  cudaStream_t st = R.st;
  const int64_t n = S.H.levels[0].nCells;
  float* g = S.guess.as<float>();
  double* part = S.partial.as<double>();
  Scalars* sc = S.scal.as<Scalars>();
  int rc = learned_predict(ctx, S, S.net, st, b, g, R.launches);
  if (rc) return rc;
  k_mask<<<VEC_GRID, VEC_BLOCK, 0, st>>>(g, S.views[0].diag, n);
  k_set64_masked<<<VEC_GRID, VEC_BLOCK, 0, st>>>(S.x64.as<double>(), g, S.views[0].diag, n);
  double rr = 0;
  rc = residual64(ctx, S, R, b, r32, &rr);
  if (rc) return rc;
  k_dot<<<VEC_GRID, VEC_BLOCK, 0, st>>>(g, b, n, part);
  k_finalize<<<1, 1024, 0, st>>>(part, VEC_GRID, sc, FIN_CR);
  k_dot<<<VEC_GRID, VEC_BLOCK, 0, st>>>(g, (const float*)r32, n, part);
  k_finalize<<<1, 1024, 0, st>>>(part, VEC_GRID, sc, FIN_OMEGA_GUESS);
  k_scale64<<<VEC_GRID, VEC_BLOCK, 0, st>>>(S.x64.as<double>(), sc, n);
  R.launches += 7;
  return MSBG_OK;
}

// Inner relative tolerance floor per storage type: a few unit roundoffs of
// the stored vectors (FP32 2^-24, FP16 2^-11, BF16 2^-8).
template <typename VT> constexpr double inner_floor() { return 1e-5; }
template <> constexpr double inner_floor<__half>() { return 2e-3; }
template <> constexpr double inner_floor<__nv_bfloat16>() { return 1.5e-2; }

// FP64 iterative refinement: x64 += s^-1 MGPCG_VT(s (b - A x64)).  For
// 16-bit vectors the inner right-hand side is scaled by a power of two s that
// keeps the inner solution inside the FP16 range: the first step aims at
// max|s r| = 2^-4, later steps at max|e| = 2^10 through the measured gain
// max|e| / max|s r| of the previous inner solve (the gain moves by up to
// about 20x between steps, the FP16 range leaves 64x).  An inner solve whose
// residual or solution is non-finite (an FP16 overflow) is repeated with s
// reduced by 2^8, at most twice.  Inner solves of 16-bit vectors stop at 40
// iterations or at a breakdown: their recursive residual stagnates near the
// rounding level, and the outer step then recomputes the true residual in
// FP64 and continues from the iterate reached.
template <typename VT>
int solve_refined(msbg_gpu_ctx* ctx, Solver& S, Runner<VT>& R, const msbg_gpu_solve_params* p,
                  int maxRefine, cudaGraphExec_t& exec, int64_t& perIter, SolveOut& o) {
  cudaStream_t st = R.st;
  const int64_t n = S.H.levels[0].nCells;
  constexpr bool WIDE = std::is_same<VT, float>::value;
  constexpr int INNER_MAX_16 = 40;
  double* x64 = S.x64.as<double>();
  float* rin = S.rin.as<float>();
  VT* rinV = WIDE ? reinterpret_cast<VT*>(rin) : S.rinv.as<VT>();
  VT* e = S.dev[0]->x.as<VT>();
  const float* b = S.rhs0.as<float>();
  int rc = MSBG_OK;
  if (p->learned & 1) {
    // initial guess predicted by the network from the right-hand side
    rc = learned_start(ctx, S, R, b, rin);
    if (rc) return rc;
  } else {
    cudaMemsetAsync(x64, 0, sizeof(double) * n, st);
  }
  double bb = 0, rr = 0, gain = 0;
  for (int outer = 0;; outer++) {
    rc = residual64(ctx, S, R, b, rin, &rr);
    if (rc) return rc;
    if (outer == 0) {
      // |b|^2 (the guess, when there is one, is not part of the reference norm)
      bb = rr;
      if (p->learned & 1) {
        double* part = S.partial.as<double>();
        Scalars* sc = S.scal.as<Scalars>();
        k_dot<<<VEC_GRID, VEC_BLOCK, 0, st>>>(b, b, n, part);
        k_finalize<<<1, 1024, 0, st>>>(part, VEC_GRID, sc, FIN_BB);
        cudaMemcpyAsync(S.hScal, sc, sizeof(Scalars), cudaMemcpyDeviceToHost, st);
        R.launches += 2;
        MSBG_CUDA_TRY(ctx, cudaStreamSynchronize(st));
        bb = S.hScal->bb;
        o.initialRelres = bb > 0 ? std::sqrt(rr / bb) : 0.0;
      }
    }
    o.relres = bb > 0 ? std::sqrt(rr / bb) : 0.0;
    // a non-finite right-hand side or residual is reported before any
    // convergence test (NaN compares false with every tolerance)
    if (!std::isfinite(rr) || !std::isfinite(bb)) {
      o.status = 3;
      break;
    }
    if (!(bb > 1e-300) || o.relres <= p->tol) {
      o.status = 0;
      break;
    }
    if (outer >= maxRefine || o.iters >= p->maxIter) {
      o.status = 1;
      break;
    }
    // inner tolerance: what is still missing, not below the storage floor
    const double need = p->tol / std::max(o.relres, 1e-300);
    const double tolIn = std::min(0.5, std::max(need * 0.5, inner_floor<VT>()));
    double scale = 1.0, rmax = 0, emax = 0;
    if (!WIDE) {
      rc = absmax(ctx, S, R, rin, n, &rmax);
      if (rc) return rc;
      if (!(rmax > 0) || !std::isfinite(rmax)) {
        o.status = std::isfinite(rmax) ? 0 : 3;
        break;
      }
      const double target = gain > 0 ? std::ldexp(1.0, 10) / gain : std::ldexp(1.0, -4);
      scale = std::ldexp(1.0, (int)std::floor(std::log2(target / rmax)));
    }
    PcgResult pr;
    const int budget = p->maxIter - o.iters;
    for (int attempt = 0;; attempt++) {
      if (!WIDE) {
        k_convert<<<VEC_GRID, VEC_BLOCK, 0, st>>>(rinV, rin, n, (float)scale);
        R.launches++;
      }
      rc = run_pcg(ctx, S, R, (const VT*)rinV, tolIn,
                   WIDE ? budget : std::min(budget, INNER_MAX_16), p->useGraph, exec, perIter,
                   pr);
      if (rc) return rc;
      o.iters += pr.iters;
      if (WIDE) break;
      rc = absmax(ctx, S, R, e, n, &emax);
      if (rc) return rc;
      const bool overflow = pr.status == 3 || !std::isfinite(emax);
      if (!overflow || attempt == 2) {
        if (overflow) pr.status = 3;
        break;
      }
      scale = std::ldexp(scale, -8);
    }
    o.refinements++;
    if (pr.status == 3 || (pr.status == 2 && WIDE)) {
      o.status = pr.status;
      break;
    }
    if (!WIDE) gain = emax > 0 ? emax / (rmax * scale) : 0.0;
    k_add64<<<VEC_GRID, VEC_BLOCK, 0, st>>>(x64, e, n, 1.0 / scale);
    R.launches++;
  }
  k_narrow<<<VEC_GRID, VEC_BLOCK, 0, st>>>(S.dev[0]->x.as<float>(), x64, n);
  R.launches++;
  return MSBG_OK;
}

// FP32 vectors with the solution accumulated in FP64 and reliable residual
// replacement: one MGPCG run (no restarts) whose x is kept in FP64
// (x64 += alpha d) while r, d, q, z stay FP32.  Whenever the recursive
// residual has dropped by 10x since the last replacement, and when it reaches
// tol, the true residual b - A x64 is recomputed in FP64 and replaces r; the
// iteration continues with its search directions (Sleijpen & van der Vorst,
// "Reliable updated residuals in hybrid Bi-CG methods", Computing 56, 1996).
// Replacing often keeps the swapped-in residual close to the recursive one
// (an FP32 product A d on smooth directions loses accuracy in proportion to
// the condition number, so the two drift apart).  Convergence is judged on
// the true residual only.  An iteration is two CUDA graphs around
// the host's convergence check: [q = A d, alpha, x/r update, |r|^2] and
// [z = V r, rho, beta, d update].
int solve_reliable(msbg_gpu_ctx* ctx, Solver& S, Runner<float>& R, const msbg_gpu_solve_params* p,
                   int maxChecks, SolveOut& o) {
  cudaStream_t st = R.st;
  const int64_t n = S.H.levels[0].nCells;
  double* x64 = S.x64.as<double>();
  float* r = S.r0.as<float>();
  float* d = S.d0.as<float>();
  float* q = S.q0.as<float>();
  float* z = S.z0.as<float>();
  double* part = S.partial.as<double>();
  Scalars* sc = S.scal.as<Scalars>();
  const float* b = S.rhs0.as<float>();
  int rc = MSBG_OK;
  if (p->learned & 1) {
    rc = learned_start(ctx, S, R, b, r);
    if (rc) return rc;
  } else {
    cudaMemsetAsync(x64, 0, sizeof(double) * n, st);
  }
  // r = b - A x64, |b|^2
  double rr = 0;
  rc = residual64(ctx, S, R, b, r, &rr);
  if (rc) return rc;
  cudaMemsetAsync(sc, 0, sizeof(Scalars), st);
  k_dot<<<VEC_GRID, VEC_BLOCK, 0, st>>>(b, b, n, part);
  k_finalize<<<1, 1024, 0, st>>>(part, VEC_GRID, sc, FIN_BB);
  // learned & 2: the preconditioner is the V-cycle followed by the
  // correction network's estimate c of the error the V-cycle leaves,
  // z = V r + omega c, c = N(r'), r' = r - A V r, omega = (c.r')/(c.Ac) (the
  // energy-optimal multiple, 0 for a useless c).  It is not linear, so the
  // iteration is flexible CG (Notay 2000, FCG(1)): alpha = (d.r)/(d.q),
  // beta = -(z.q)/(d.q).
  const bool corr = (p->learned & 2) != 0;
  float* tq = corr ? S.tq.as<float>() : nullptr;
  float* rt = corr ? S.rin.as<float>() : nullptr;
  float* ec = corr ? S.guess.as<float>() : nullptr;
  auto precond = [&](bool inGraph) -> int {
    R.vcycle(0, z, (const float*)r);
    if (!corr) return MSBG_OK;
    R.matvec_dot(z, tq, part);
    k_sub<<<VEC_GRID, VEC_BLOCK, 0, st>>>(rt, r, tq, n);
    int e = learned_predict(ctx, S, S.netCorr, st, rt, ec, R.launches, inGraph);
    if (e) return e;
    k_mask<<<VEC_GRID, VEC_BLOCK, 0, st>>>(ec, S.views[0].diag, n);
    const int nt = R.matvec_dot((const float*)ec, tq, part);
    k_finalize<<<1, 1024, 0, st>>>(part, nt, sc, FIN_CC);
    k_dot<<<VEC_GRID, VEC_BLOCK, 0, st>>>((const float*)ec, (const float*)rt, n, part);
    k_finalize<<<1, 1024, 0, st>>>(part, VEC_GRID, sc, FIN_OMEGA_CORR);
    k_add_omega<<<VEC_GRID, VEC_BLOCK, 0, st>>>(z, ec, sc, n);
    R.launches += 6;
    return MSBG_OK;
  };
  // packed x faces of d, kept from the V-cycle's faces of z (not with the
  // correction, which changes z after the V-cycle)
  float* zf = corr ? nullptr : R.template faces<float>(0);
  const int64_t nf = xface_words(n);
  if (zf) MSBG_CUDA_TRY(ctx, S.df.ensure(sizeof(float) * nf));
  float* df = zf ? S.df.as<float>() : nullptr;
  // z = B r, rho = r.z, d = z
  rc = precond(false);
  if (rc) return rc;
  k_dot<<<VEC_GRID, VEC_BLOCK, 0, st>>>(r, z, n, part);
  k_finalize<<<1, 1024, 0, st>>>(part, VEC_GRID, sc, FIN_RHO);
  cudaMemcpyAsync(d, z, sizeof(float) * n, cudaMemcpyDeviceToDevice, st);
  if (df) cudaMemcpyAsync(df, zf, sizeof(float) * nf, cudaMemcpyDeviceToDevice, st);
  cudaMemcpyAsync(S.hScal, sc, sizeof(Scalars), cudaMemcpyDeviceToHost, st);
  R.launches += 4;
  MSBG_CUDA_TRY(ctx, cudaStreamSynchronize(st));
  const double bb = S.hScal->bb;
  o.initialRelres = bb > 0 ? std::sqrt(rr / bb) : 0.0;
  o.relres = o.initialRelres;
  if (!std::isfinite(rr) || !std::isfinite(bb) || !std::isfinite(S.hScal->rho)) {
    o.status = 3;  // before the convergence test: NaN compares false with any tolerance
    return MSBG_OK;
  }
  if (!(bb > 1e-300) || o.relres <= p->tol) {
    o.status = 0;
    return MSBG_OK;
  }
  auto part1 = [&]() {
    R.launches += 3;
    const int nt = R.matvec_dot(d, q, part, df);
    k_finalize<<<1, 1024, 0, st>>>(part, nt, sc, corr ? FIN_FCG_DQ_ALPHA : FIN_DQ_ALPHA);
    k_axpy64_norm<<<VEC_GRID, VEC_BLOCK, 0, st>>>(x64, r, d, q, n, sc, part);
    k_finalize<<<1, 1024, 0, st>>>(part, VEC_GRID, sc, FIN_RR);
    cudaMemcpyAsync(S.hScal, sc, sizeof(Scalars), cudaMemcpyDeviceToHost, st);
  };
  int precondRc = MSBG_OK;
  auto part2 = [&]() {
    R.launches += 3;
    const int e = precond(true);
    if (e) precondRc = e;
    if (!corr) {
      k_dot<<<VEC_GRID, VEC_BLOCK, 0, st>>>(r, z, n, part);
      k_finalize<<<1, 1024, 0, st>>>(part, VEC_GRID, sc, FIN_RHONEW_BETA);
      k_update_d<<<VEC_GRID, VEC_BLOCK, 0, st>>>(d, z, n, sc);
      if (df) {
        k_update_d<<<VEC_GRID, VEC_BLOCK, 0, st>>>(df, zf, nf, sc);
        R.launches++;
      }
    } else {
      // beta = -(z.q)/(d.q); d = z + beta d; rho = d.r for the next alpha
      k_dot<<<VEC_GRID, VEC_BLOCK, 0, st>>>(z, q, n, part);
      k_finalize<<<1, 1024, 0, st>>>(part, VEC_GRID, sc, FIN_FCG_BETA);
      k_update_d<<<VEC_GRID, VEC_BLOCK, 0, st>>>(d, z, n, sc);
      k_dot<<<VEC_GRID, VEC_BLOCK, 0, st>>>(d, r, n, part);
      k_finalize<<<1, 1024, 0, st>>>(part, VEC_GRID, sc, FIN_RHO);
      R.launches += 3;
    }
  };
  cudaGraphExec_t g1 = nullptr, g2 = nullptr;
  int64_t per1 = 0, per2 = 0;
  auto capture = [&](auto&& body, cudaGraphExec_t& ex, int64_t& per) -> int {
    const int64_t before = R.launches;
    cudaGraph_t g;
    MSBG_CUDA_TRY(ctx, cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    body();
    MSBG_CUDA_TRY(ctx, cudaStreamEndCapture(st, &g));
    per = R.launches - before;
    R.launches = before;
    const cudaError_t e = cudaGraphInstantiate(&ex, g, 0);
    cudaGraphDestroy(g);
    MSBG_CUDA_TRY(ctx, e);
    return MSBG_OK;
  };
  if (p->useGraph) {
    rc = capture(part1, g1, per1);
    if (!rc) rc = capture(part2, g2, per2);
  }
  auto run = [&](cudaGraphExec_t ex, int64_t per, auto&& body) -> int {
    if (ex) {
      MSBG_CUDA_TRY(ctx, cudaGraphLaunch(ex, st));
      R.launches += per;
    } else {
      body();
    }
    return MSBG_OK;
  };
  const double tol2 = (double)p->tol * p->tol;
  constexpr double DELTA2 = 1e-2;  // replace when |r| dropped by 10x
  double rrRef = rr;               // true |r|^2 at the last replacement
  int checks = 0;                  // true-residual checks at recursive convergence
  o.status = 1;
  for (int it = 0; !rc && it < p->maxIter; it++) {
    rc = run(g1, per1, part1);
    if (rc) break;
    rc = [&]() -> int {
      MSBG_CUDA_TRY(ctx, cudaStreamSynchronize(st));
      return MSBG_OK;
    }();
    if (rc) break;
    o.iters = it + 1;
    const Scalars hs = *S.hScal;
    if (hs.status) {
      o.status = hs.status;
      break;
    }
    if (hs.rr <= tol2 * bb || hs.rr <= DELTA2 * rrRef) {
      // replace the recursive residual by the true FP64 one (and judge it)
      if (hs.rr <= tol2 * bb) checks++;
      rc = residual64(ctx, S, R, b, r, &rr);
      if (rc) break;
      o.refinements++;
      o.relres = std::sqrt(rr / bb);
      if (!std::isfinite(rr)) {
        o.status = 3;
        break;
      }
      if (rr <= tol2 * bb) {
        o.status = 0;
        break;
      }
      if (checks >= maxChecks) break;  // status 1
      rrRef = rr;
      // r now holds the true residual; continue with the directions
    }
    rc = run(g2, per2, part2);
  }
  if (!rc && o.status == 1 && o.iters > 0) {
    // the true residual of the delivered iterate
    rc = residual64(ctx, S, R, b, r, &rr);
    if (!rc) o.relres = std::sqrt(rr / bb);
  }
  if (g1) cudaGraphExecDestroy(g1);
  if (g2) cudaGraphExecDestroy(g2);
  if (!rc && precondRc) rc = precondRc;
  if (!rc && corr) {
    const int e = cnn::take_error(S.netCorr, st);
    if (e) rc = set_error(ctx, e, "learned network: a tensor-core wait gave up");
  }
  if (rc) return rc;
  k_narrow<<<VEC_GRID, VEC_BLOCK, 0, st>>>(S.dev[0]->x.as<float>(), x64, n);
  R.launches++;
  return MSBG_OK;
}

template <typename VT>
int solve_typed(msbg_gpu_ctx* ctx, Solver& S, const msbg_gpu_solve_params* p, cudaEvent_t e0,
                cudaEvent_t e1, SolveOut& o, int64_t* launches) {
  cudaStream_t st = ctx->stream;
  Runner<VT> R{S, st, p->nPre, p->nPost, p->innerIter};
  R.coarseScale = p->coarseScale > 0 ? p->coarseScale : 1.0f;
  R.err = ctx->errBuf.as<int>();
  R.numSMs = S.numSMs;
  const int64_t n = S.H.levels[0].nCells;
  constexpr bool WIDE = std::is_same<VT, float>::value;
  // 16-bit vectors and the learned guess always run under the FP64 refinement
  const int maxRefine = p->maxRefine > 0 ? p->maxRefine : (WIDE && !p->learned ? 0 : 30);
  S.haveX64 = false;
  if (maxRefine > 0) {
    MSBG_CUDA_TRY(ctx, S.x64.ensure(sizeof(double) * n));
    MSBG_CUDA_TRY(ctx, S.rin.ensure(sizeof(float) * n));
    if (!WIDE) MSBG_CUDA_TRY(ctx, S.rinv.ensure(sizeof(VT) * n));
    if (p->learned) MSBG_CUDA_TRY(ctx, S.guess.ensure(sizeof(float) * n));
    if (p->learned & 2) MSBG_CUDA_TRY(ctx, S.tq.ensure(sizeof(float) * n));
  }
  cudaGraphExec_t exec = nullptr;
  int64_t perIter = 0;
  cudaEventRecord(e0, st);
  int rc = MSBG_OK;
  if constexpr (WIDE) {
    if (maxRefine == 0) rc = solve_plain(ctx, S, R, p, exec, perIter, e1, o);
  }
  if (maxRefine > 0) {
    if constexpr (WIDE)
      rc = solve_reliable(ctx, S, R, p, maxRefine, o);  // FP32: FP64 x, reliable updates
    else
      rc = solve_refined(ctx, S, R, p, maxRefine, exec, perIter, o);
    cudaEventRecord(e1, st);
    S.haveX64 = rc == MSBG_OK;
  }
  if (exec) cudaGraphExecDestroy(exec);
  *launches = R.launches;
  return rc;
}

}  // namespace

extern "C" int msbg_gpu_pressure_solve(msbg_gpu_ctx* ctx, const msbg_gpu_solve_params* p,
                                       msbg_gpu_solve_info* info) {
  if (!ctx || !p) return MSBG_EINVARG;
  auto& sp = solver_of(ctx);
  if (!sp) return set_error(ctx, MSBG_EINVARG, "msbg_gpu_pressure_prepare not called");
  if (p->nPre < 0 || p->nPost < 0 || p->maxIter < 0 || p->innerIter < 1 || !(p->tol >= 0) ||
      p->maxRefine < 0)
    return set_error(ctx, MSBG_EINVARG, "invalid solve parameters");
  if (p->storage != MSBG_F32 && p->storage != MSBG_F16 && p->storage != MSBG_BF16)
    return set_error(ctx, MSBG_ENOTIMPL, "storage type %d not available", p->storage);
  if (p->learned < 0 || p->learned > 3)
    return set_error(ctx, MSBG_EINVARG, "learned = %d (bit 0 guess, bit 1 correction)", p->learned);
  if ((p->learned & 2) && p->storage != MSBG_F32)
    return set_error(ctx, MSBG_ENOTIMPL, "the learned correction runs with FP32 vectors");
  if ((p->learned & 1) && !ctx->cnn)
    return set_error(ctx, MSBG_EINVARG, "learned guess without a network (msbg_gpu_pressure_set_cnn)");
  if ((p->learned & 2) && !ctx->cnnCorr)
    return set_error(ctx, MSBG_EINVARG,
                     "learned correction without a network (msbg_gpu_pressure_set_correction_cnn)");
  cudaSetDevice(ctx->device);
  Solver& S = *sp;
  S.net = ctx->cnn;
  S.netCorr = ctx->cnnCorr;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  auto run = [&](const msbg_gpu_solve_params* q, SolveOut& o, int64_t* launches, float* ms) -> int {
    int rc;
    switch (q->storage) {
      case MSBG_F16: rc = solve_typed<__half>(ctx, S, q, e0, e1, o, launches); break;
      case MSBG_BF16: rc = solve_typed<__nv_bfloat16>(ctx, S, q, e0, e1, o, launches); break;
      default: rc = solve_typed<float>(ctx, S, q, e0, e1, o, launches); break;
    }
    const cudaError_t se = cudaStreamSynchronize(ctx->stream);
    *ms = 0;
    if (rc == MSBG_OK && se == cudaSuccess) cudaEventElapsedTime(ms, e0, e1);
    if (rc) return rc;
    MSBG_CUDA_TRY(ctx, se);
    return MSBG_OK;
  };
  SolveOut o;
  int64_t launches = 0;
  float ms = 0;
  int rc = run(p, o, &launches, &ms);
  int fellBack = 0;
  if (rc == MSBG_OK && p->learned && o.status != 0) {
    // plain MGPCG is the fallback of the learned solve: the same storage and
    // FP64 refinement from a zero guess; the time and work of both count
    msbg_gpu_solve_params q = *p;
    q.learned = 0;
    if (q.storage == MSBG_F32 && q.maxRefine == 0) q.maxRefine = 30;
    SolveOut o2;
    int64_t l2 = 0;
    float ms2 = 0;
    rc = run(&q, o2, &l2, &ms2);
    o2.iters += o.iters;
    o2.refinements += o.refinements;
    o2.initialRelres = o.initialRelres;
    o = o2;
    launches += l2;
    ms += ms2;
    fellBack = 1;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc) return rc;
  // a pipelined kernel that gave up a bounded wait has set the context's
  // error flag and left its tile unsmoothed: the solution is not delivered
  rc = msbg_gpu_sync(ctx);
  if (rc) return rc;
  if (info) {
    const Level& L0 = S.H.levels[0];
    info->iterations = o.iters;
    info->refinements = o.refinements;
    info->status = o.status;
    info->relResidual = o.relres;
    info->solveSeconds = ms * 1e-3;
    info->fineCells = L0.nFluid;
    info->nMgLevels = (int)S.H.levels.size();
    info->kernelLaunches = launches;
    info->initialRelResidual = o.initialRelres;
    info->learnedFallback = fellBack;
  }
  return MSBG_OK;
}

extern "C" int msbg_gpu_pressure_set_cnn(msbg_gpu_ctx* ctx, msbg_cnn* net) {
  if (!ctx) return MSBG_EINVARG;
  ctx->cnn = net;
  return MSBG_OK;
}

extern "C" int msbg_gpu_pressure_set_correction_cnn(msbg_gpu_ctx* ctx, msbg_cnn* net) {
  if (!ctx) return MSBG_EINVARG;
  ctx->cnnCorr = net;
  return MSBG_OK;
}

namespace {
// np training tiles spread evenly over the network's tile list, uploaded to
// S.cIdx as [tile ids | levels].
int select_pair_tiles(msbg_gpu_ctx* ctx, Solver& S, int np, cudaStream_t st) {
  std::vector<int> sel(2 * (size_t)np);
  for (int i = 0; i < np; i++) {
    const int k = (int)((int64_t)i * S.nCnnTiles / np);
    sel[i] = S.cnnTilesHost[k];
    sel[np + i] = S.cnnLevelHost[k];
  }
  MSBG_CUDA_TRY(ctx, upload(S.cIdx, sel, st));
  return MSBG_OK;
}
}  // namespace

extern "C" int msbg_gpu_pressure_training_pairs(msbg_gpu_ctx* ctx, float* feat, float* target,
                                                float* mask, int maxPairs, int* nPairs) {
  if (!ctx || !feat || !target || !mask || maxPairs <= 0 || !nPairs) return MSBG_EINVARG;
  auto& sp = solver_of(ctx);
  if (!sp) return set_error(ctx, MSBG_EINVARG, "msbg_gpu_pressure_prepare not called");
  Solver& S = *sp;
  if (!S.haveX64)
    return set_error(ctx, MSBG_EINVARG, "training pairs need a refined solve (maxRefine > 0) first");
  cudaSetDevice(ctx->device);
  cudaStream_t st = ctx->stream;
  const int np = std::min(maxPairs, S.nCnnTiles);
  *nPairs = np;
  if (np == 0) return MSBG_OK;
  int rc = select_pair_tiles(ctx, S, np, st);
  if (rc) return rc;
  DeviceBuffer scale, off;
  MSBG_CUDA_TRY(ctx, scale.ensure(sizeof(float) * np));
  MSBG_CUDA_TRY(ctx, off.ensure(sizeof(int64_t) * np));
  k_cnn_features<<<np, FEAT_THREADS, 0, st>>>(
      S.views[0], S.dev[0]->ctype.as<uint8_t>(), S.cIdx.as<int>(), S.cIdx.as<int>() + np,
      S.levelNorm, S.rhs0.as<float>(), S.x64.as<double>(), feat, scale.as<float>(),
      off.as<int64_t>(), target, mask);
  MSBG_CUDA_TRY(ctx, cudaGetLastError());
  MSBG_CUDA_TRY(ctx, cudaStreamSynchronize(st));
  return MSBG_OK;
}

// Training pairs of the correction network: the state a PCG iteration hands
// to the correction stage.  After pcgIters iterations of plain MGPCG (FP32
// vectors, FP64 iterate x_k) from zero, y = x_k + V(b - A x_k); the input is
// the residual r' = b - A y and the target the error x* - y, x* being the
// refined solution of the last solve (which is restored afterwards).
extern "C" int msbg_gpu_pressure_correction_pairs(msbg_gpu_ctx* ctx,
                                                  const msbg_gpu_solve_params* p, int pcgIters,
                                                  float* feat, float* target, float* mask,
                                                  int maxPairs, int* nPairs) {
  if (!ctx || !p || !feat || !target || !mask || maxPairs <= 0 || !nPairs || pcgIters < 0)
    return MSBG_EINVARG;
  auto& sp = solver_of(ctx);
  if (!sp) return set_error(ctx, MSBG_EINVARG, "msbg_gpu_pressure_prepare not called");
  Solver& S = *sp;
  if (!S.haveX64)
    return set_error(ctx, MSBG_EINVARG, "training pairs need a refined solve (maxRefine > 0) first");
  if (p->nPre < 0 || p->nPost < 0 || p->innerIter < 1)
    return set_error(ctx, MSBG_EINVARG, "invalid V-cycle parameters");
  cudaSetDevice(ctx->device);
  cudaStream_t st = ctx->stream;
  const int np = std::min(maxPairs, S.nCnnTiles);
  *nPairs = np;
  if (np == 0) return MSBG_OK;
  const int64_t n = S.H.levels[0].nCells;
  double* x64 = S.x64.as<double>();
  DeviceBuffer xs, err, scale, off;
  MSBG_CUDA_TRY(ctx, xs.ensure(sizeof(double) * n));
  MSBG_CUDA_TRY(ctx, err.ensure(sizeof(double) * n));
  MSBG_CUDA_TRY(ctx, scale.ensure(sizeof(float) * np));
  MSBG_CUDA_TRY(ctx, off.ensure(sizeof(int64_t) * np));
  MSBG_CUDA_TRY(ctx, cudaMemcpyAsync(xs.p, x64, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
  auto body = [&]() -> int {
    int rc = MSBG_OK;
    if (pcgIters > 0) {
      msbg_gpu_solve_params q = *p;
      q.storage = MSBG_F32;
      q.learned = 0;
      q.tol = 0;
      q.maxIter = pcgIters;
      q.maxRefine = 1 << 20;
      cudaEvent_t e0, e1;
      cudaEventCreate(&e0);
      cudaEventCreate(&e1);
      SolveOut o;
      int64_t launches = 0;
      rc = solve_typed<float>(ctx, S, &q, e0, e1, o, &launches);
      cudaStreamSynchronize(st);
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
      if (rc) return rc;
    } else {
      MSBG_CUDA_TRY(ctx, cudaMemsetAsync(x64, 0, sizeof(double) * n, st));
    }
    Runner<float> R{S, st, p->nPre, p->nPost, p->innerIter};
    R.coarseScale = p->coarseScale > 0 ? p->coarseScale : 1.0f;
    R.err = ctx->errBuf.as<int>();
    R.numSMs = S.numSMs;
    const float* b = S.rhs0.as<float>();
    float* r = S.r0.as<float>();
    float* z = S.z0.as<float>();
    double rr = 0;
    rc = residual64(ctx, S, R, b, r, &rr);
    if (rc) return rc;
    R.vcycle(0, z, (const float*)r);
    k_add64<float><<<VEC_GRID, VEC_BLOCK, 0, st>>>(x64, z, n, 1.0);
    rc = residual64(ctx, S, R, b, r, &rr);
    if (rc) return rc;
    k_sub64<<<VEC_GRID, VEC_BLOCK, 0, st>>>(err.as<double>(), xs.as<double>(), x64, n);
    rc = select_pair_tiles(ctx, S, np, st);
    if (rc) return rc;
    k_cnn_features<<<np, FEAT_THREADS, 0, st>>>(
        S.views[0], S.dev[0]->ctype.as<uint8_t>(), S.cIdx.as<int>(), S.cIdx.as<int>() + np,
        S.levelNorm, r, err.as<double>(), feat, scale.as<float>(), off.as<int64_t>(), target, mask);
    MSBG_CUDA_TRY(ctx, cudaGetLastError());
    return MSBG_OK;
  };
  const int rc = body();
  // restore the refined solution (after a failure in between too)
  cudaError_t e = cudaMemcpyAsync(x64, xs.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, st);
  if (e == cudaSuccess) {
    k_narrow<<<VEC_GRID, VEC_BLOCK, 0, st>>>(S.dev[0]->x.as<float>(), x64, n);
    e = cudaGetLastError();
  }
  const cudaError_t es = cudaStreamSynchronize(st);
  S.haveX64 = e == cudaSuccess && es == cudaSuccess;
  if (rc) return rc;
  MSBG_CUDA_TRY(ctx, e);
  MSBG_CUDA_TRY(ctx, es);
  return MSBG_OK;
}

extern "C" int msbg_gpu_pressure_stats(msbg_gpu_ctx* ctx, msbg_gpu_pressure_stats_t* out) {
  if (!ctx || !out) return MSBG_EINVARG;
  auto& sp = solver_of(ctx);
  if (!sp) return set_error(ctx, MSBG_EINVARG, "msbg_gpu_pressure_prepare not called");
  Solver& S = *sp;
  std::memset(out, 0, sizeof(*out));
  out->nMgLevels = (int)S.H.levels.size();
  for (size_t m = 0; m < S.H.levels.size() && m < 32; m++) {
    out->cells[m] = S.H.levels[m].nCells;
    out->fluid[m] = S.H.levels[m].nFluid;
    out->tiles[m] = (int64_t)S.H.levels[m].tiles.size();
  }
  out->h2dBytes = S.h2dBytes;
  out->prepareSeconds = S.prepareSeconds;
  out->buildSeconds = S.buildSeconds;
  size_t fr = 0, tot = 0;
  cudaMemGetInfo(&fr, &tot);
  out->deviceBytesUsed = (int64_t)(tot - fr);
  out->coarseCells = S.H.nCoarse;
  return MSBG_OK;
}

namespace {

template <typename VT>
int profile_typed(msbg_gpu_ctx* ctx, Solver& S, int what, int reps, int innerIter,
                  double* msPerCall, double* algBytesPerCall) {
  cudaStream_t st = ctx->stream;
  Runner<VT> R{S, st, 2, 2, innerIter};
  R.err = ctx->errBuf.as<int>();
  R.numSMs = S.numSMs;
  const Level& L0 = S.H.levels[0];
  LevelDev& D0 = *S.dev[0];
  VT* x = D0.x.as<VT>();
  double* part = S.partial.as<double>();
  // a VT copy of the right-hand side (FP32 storage reads it in place)
  VT* b = std::is_same<VT, float>::value ? (VT*)S.rhs0.as<float>() : S.r0.as<VT>();
  if (!std::is_same<VT, float>::value)
    k_convert<<<VEC_GRID, VEC_BLOCK, 0, st>>>(b, S.rhs0.as<float>(), L0.nCells, 1.0f);
  // algorithmic bytes per cell: the smoother reads x, b, 1/a_ii, cx, cy, cz
  // and writes x; the matvec reads d, a_ii, cx, cy, cz and writes q
  const double v = sizeof(VT);
  const double smooth0 = 16.0 + 3 * v, smoothC = 28.0, mvB = 16.0 + 2 * v;
  // the sweep keeps the packed x faces of x, as inside a V-cycle
  VT* xf0 = R.template faces<VT>(0);
  auto vcycle_bytes = [&]() {
    double s = 0;
    for (size_t m = 0; m + 1 < S.H.levels.size(); m++) {
      const double n = (double)S.H.levels[m].nCells;
      const double vs = m == 0 ? v : 4.0;
      const double sm = m == 0 ? smooth0 : smoothC;
      // zero x, sweeps, residual (x, b, operator, 1/8 restricted write),
      // prolongation (a_ii mask, x read + write, 1/8 coarse read)
      s += n * (vs + (R.nPre + R.nPost) * sm + (16.0 + 2 * vs + 0.5) + (4.0 + 2 * vs + 0.5));
    }
    return s;
  };
  double bytes = 0;
  auto body = [&]() {
    switch (what) {
      case 0: R.smooth(0, x, (const VT*)b, false, xf0); break;
      case 3: R.usePipe = false; R.smooth(0, x, (const VT*)b, false); R.usePipe = true; break;
      case 1: R.matvec_dot(x, S.q0.as<VT>(), part); break;
      case 2: R.vcycle(0, S.z0.as<VT>(), (const VT*)b); break;
      default: break;
    }
  };
  switch (what) {
    case 0:
    case 3: bytes = smooth0 * L0.nCells; break;
    case 1: bytes = mvB * L0.nCells; break;
    case 2: bytes = vcycle_bytes(); break;
    default: return set_error(ctx, MSBG_EINVARG, "profile target %d", what);
  }
  MSBG_CUDA_TRY(ctx, cudaMemsetAsync(x, 0, sizeof(VT) * L0.nCells, st));
  if (xf0) MSBG_CUDA_TRY(ctx, cudaMemsetAsync(xf0, 0, sizeof(VT) * xface_len(L0.nCells), st));
  body();  // warm-up
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, st);
  for (int i = 0; i < reps; i++) body();
  cudaEventRecord(e1, st);
  const cudaError_t se = cudaEventSynchronize(e1);
  float ms = 0;
  if (se == cudaSuccess) cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  MSBG_CUDA_TRY(ctx, se);
  if (msPerCall) *msPerCall = ms / reps;
  if (algBytesPerCall) *algBytesPerCall = bytes;
  return MSBG_OK;
}

}  // namespace

extern "C" int msbg_gpu_pressure_profile(msbg_gpu_ctx* ctx, int what, int reps, int innerIter,
                                         double* msPerCall, double* algBytesPerCall) {
  if (!ctx || reps <= 0 || innerIter < 1) return MSBG_EINVARG;
  auto& sp = solver_of(ctx);
  if (!sp) return set_error(ctx, MSBG_EINVARG, "msbg_gpu_pressure_prepare not called");
  cudaSetDevice(ctx->device);
  Solver& S = *sp;
  const int target = what & 15, storage = what >> 4;
  switch (storage) {
    case MSBG_F32: return profile_typed<float>(ctx, S, target, reps, innerIter, msPerCall,
                                               algBytesPerCall);
    case MSBG_F16: return profile_typed<__half>(ctx, S, target, reps, innerIter, msPerCall,
                                                algBytesPerCall);
    case MSBG_BF16: return profile_typed<__nv_bfloat16>(ctx, S, target, reps, innerIter,
                                                        msPerCall, algBytesPerCall);
    default: return set_error(ctx, MSBG_ENOTIMPL, "storage type %d not available", storage);
  }
}

namespace {

// Copy a level-0 vector (tile layout) into the reference's packed block layout.
// The reference's block layout (packed): per block in bid order,
// (bsx0 >> level)^3 values, vid = x + y*bs + z*bs*bs.  A tile lies inside one
// block, so its cell (i, j, k) lands at base + i + bs*(j + bs*k).
struct PackTile {
  int64_t base;  // packed index of the tile's first cell
  int bs, ts;
};

template <typename T>
__global__ void __launch_bounds__(256) k_to_packed(const T* __restrict__ v,
                                                   const int64_t* __restrict__ tileOff,
                                                   const PackTile* __restrict__ pt,
                                                   T* __restrict__ out) {
  const PackTile P = pt[blockIdx.x];
  const int64_t off = tileOff[blockIdx.x];
  const int n = P.ts * P.ts * P.ts;
  for (int e = threadIdx.x; e < n; e += blockDim.x) {
    const int i = e % P.ts, j = (e / P.ts) % P.ts, k = e / (P.ts * P.ts);
    out[P.base + i + (int64_t)P.bs * (j + (int64_t)P.bs * k)] = v[off + e];
  }
}

int64_t packed_count(const Solver& S) {
  int64_t s = 0;
  for (int l : S.blockLevel) {
    const int bs = S.bsx0 >> l;
    s += (int64_t)bs * bs * bs;
  }
  return s;
}

// Packs level-0 vector dvec on the device and copies it into `packed`.
template <typename T>
int to_packed(msbg_gpu_ctx* ctx, Solver& S, const T* dvec, T* packed, int64_t n) {
  const Level& L = S.H.levels[0];
  const int64_t need = packed_count(S);
  if (n < need)
    return set_error(ctx, MSBG_EINVARG, "packed buffer too small (%lld < %lld)", (long long)n,
                     (long long)need);
  cudaStream_t st = ctx->stream;
  if (!S.packTiles.p) {
    const int64_t nb = (int64_t)S.nbx * S.nby * S.nbz;
    std::vector<int64_t> boff(nb + 1, 0);
    for (int64_t bb = 0; bb < nb; bb++) {
      const int bs = S.bsx0 >> S.blockLevel[bb];
      boff[bb + 1] = boff[bb] + (int64_t)bs * bs * bs;
    }
    std::vector<PackTile> pt(L.tiles.size());
    for (size_t ti = 0; ti < L.tiles.size(); ti++) {
      const Tile& t = L.tiles[ti];
      const int bs = S.bsx0 >> t.level;
      const int64_t blk = (t.ox / bs) + (int64_t)S.nbx * ((t.oy / bs) + (int64_t)S.nby * (t.oz / bs));
      pt[ti].base = boff[blk] + (t.ox % bs) + (int64_t)bs * ((t.oy % bs) + (int64_t)bs * (t.oz % bs));
      pt[ti].bs = bs;
      pt[ti].ts = t.ts;
    }
    MSBG_CUDA_TRY(ctx, upload(S.packTiles, pt, st));
    MSBG_CUDA_TRY(ctx, cudaStreamSynchronize(st));
  }
  MSBG_CUDA_TRY(ctx, S.packBuf.ensure(sizeof(T) * need));
  MSBG_CUDA_TRY(ctx, cudaMemsetAsync(S.packBuf.p, 0, sizeof(T) * need, st));
  if (!L.tiles.empty())
    k_to_packed<T><<<(unsigned)L.tiles.size(), 256, 0, st>>>(
        dvec, S.dev[0]->tileOff.as<int64_t>(), S.packTiles.as<PackTile>(), S.packBuf.as<T>());
  MSBG_CUDA_TRY(ctx, cudaGetLastError());
  MSBG_CUDA_TRY(ctx, copy_d2h(packed, S.packBuf.p, sizeof(T) * need, st));
  return MSBG_OK;
}

}  // namespace

extern "C" int msbg_gpu_pressure_packed_size(msbg_gpu_ctx* ctx, int64_t* n) {
  if (!ctx || !n) return MSBG_EINVARG;
  auto& sp = solver_of(ctx);
  if (!sp) return set_error(ctx, MSBG_EINVARG, "msbg_gpu_pressure_prepare not called");
  *n = packed_count(*sp);
  return MSBG_OK;
}

extern "C" int msbg_gpu_pressure_download(msbg_gpu_ctx* ctx, float* packed, int64_t n) {
  if (!ctx || !packed) return MSBG_EINVARG;
  auto& sp = solver_of(ctx);
  if (!sp) return set_error(ctx, MSBG_EINVARG, "msbg_gpu_pressure_prepare not called");
  cudaSetDevice(ctx->device);
  MSBG_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  return to_packed(ctx, *sp, sp->dev[0]->x.as<float>(), packed, n);
}

extern "C" int msbg_gpu_pressure_learned_guess(msbg_gpu_ctx* ctx, float* packed, int64_t n) {
  if (!ctx || !packed) return MSBG_EINVARG;
  auto& sp = solver_of(ctx);
  if (!sp) return set_error(ctx, MSBG_EINVARG, "msbg_gpu_pressure_prepare not called");
  if (!ctx->cnn) return set_error(ctx, MSBG_EINVARG, "no network (msbg_gpu_pressure_set_cnn)");
  cudaSetDevice(ctx->device);
  Solver& S = *sp;
  S.net = ctx->cnn;
  cudaStream_t st = ctx->stream;
  const int64_t nc = S.H.levels[0].nCells;
  MSBG_CUDA_TRY(ctx, S.guess.ensure(sizeof(float) * nc));
  int64_t launches = 0;
  int rc = learned_predict(ctx, S, S.net, st, S.rhs0.as<float>(), S.guess.as<float>(), launches);
  if (rc) return rc;
  DeviceBuffer tmp;
  MSBG_CUDA_TRY(ctx, tmp.ensure(sizeof(double) * nc));
  k_set64_masked<<<VEC_GRID, VEC_BLOCK, 0, st>>>(tmp.as<double>(), S.guess.as<float>(),
                                                 S.views[0].diag, nc);
  k_narrow<<<VEC_GRID, VEC_BLOCK, 0, st>>>(S.guess.as<float>(), tmp.as<double>(), nc);
  MSBG_CUDA_TRY(ctx, cudaStreamSynchronize(st));
  return to_packed(ctx, S, S.guess.as<float>(), packed, n);
}

extern "C" int msbg_gpu_pressure_download64(msbg_gpu_ctx* ctx, double* packed, int64_t n) {
  if (!ctx || !packed) return MSBG_EINVARG;
  auto& sp = solver_of(ctx);
  if (!sp) return set_error(ctx, MSBG_EINVARG, "msbg_gpu_pressure_prepare not called");
  Solver& S = *sp;
  if (!S.x64.p) return set_error(ctx, MSBG_EINVARG, "no FP64 solution (solve with maxRefine > 0)");
  cudaSetDevice(ctx->device);
  MSBG_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  return to_packed(ctx, S, S.x64.as<double>(), packed, n);
}

extern "C" int msbg_gpu_pressure_download_rhs(msbg_gpu_ctx* ctx, float* packed, int64_t n) {
  if (!ctx || !packed) return MSBG_EINVARG;
  auto& sp = solver_of(ctx);
  if (!sp) return set_error(ctx, MSBG_EINVARG, "msbg_gpu_pressure_prepare not called");
  cudaSetDevice(ctx->device);
  MSBG_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  return to_packed(ctx, *sp, sp->rhs0.as<float>(), packed, n);
}
