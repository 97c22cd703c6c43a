// Shared definitions of the B200 sparse block-grid solver library.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "msbg_gpu.h"

namespace msbg {

// Neighbour / block-map codes stored in slot tables (slot >= 0 = value block).
enum : int {
  SLOT_NULL = -1,   // no block in the map: BC_NEUMANN clamp to own block
  SLOT_EMPTY = -2,  // const empty block
  SLOT_FULL = -3,   // const full block
  SLOT_OUT = -4     // outside the domain: BC_NEUMANN clamp to own block
};

// Bits of the device error flag that kernels set (msbg_gpu_sync reads it).
enum : int {
  ERR_WAIT_TIMEOUT = 1,   // a bounded wait gave up
  MCF_ERR_NOT_VALUE = 2   // a listed block is not a value block; it was skipped
};

struct DeviceBuffer {
  void* p = nullptr;
  size_t bytes = 0;
  DeviceBuffer() = default;
  DeviceBuffer(const DeviceBuffer&) = delete;
  DeviceBuffer& operator=(const DeviceBuffer&) = delete;
  ~DeviceBuffer() { release(); }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
  }
  cudaError_t ensure(size_t n) {
    if (n <= bytes && p) return cudaSuccess;
    release();
    cudaError_t e = cudaMalloc(&p, n ? n : 16);
    if (e == cudaSuccess) bytes = n;
    return e;
  }
  template <typename T>
  T* as() const { return reinterpret_cast<T*>(p); }
  // takes over o's allocation (o is left empty)
  void adopt(DeviceBuffer& o) {
    if (&o == this) return;
    release();
    p = o.p;
    bytes = o.bytes;
    o.p = nullptr;
    o.bytes = 0;
  }
};

// One uploaded channel at one resolution level: FP32 or 16-bit render
// density (dtype MSBG_F32 / MSBG_U16).
struct Channel {
  int level = 0;
  int bsx = 0;
  int dtype = MSBG_F32;
  uint16_t emptyQ = 0, fullQ = 0;  // const values of a 16-bit channel (raw)
  int64_t nValue = 0;
  float emptyVal = 0.f, fullVal = 0.f;
  std::vector<int> slotHost;   // [nb] slot or SLOT_* code
  std::vector<int8_t> kindHost;
  DeviceBuffer pool;           // [nValue][bsx^3] float or uint16_t
  DeviceBuffer xfaces;         // [nValue][2][bsx^2]: the x = 0 and x = bsx-1 planes
  DeviceBuffer slot;           // [nb] int
  // a channel that replaces an earlier one of the same id keeps its device
  // allocations (no cudaMalloc / cudaFree per upload when the sizes fit)
  void reuse(Channel& old) {
    pool.adopt(old.pool);
    xfaces.adopt(old.xfaces);
    slot.adopt(old.slot);
  }
};

}  // namespace msbg

struct msbg_cnn;

struct msbg_gpu_ctx {
  int device = 0;
  msbg_cnn* cnn = nullptr;      // learned initial guess of the pressure solves (not owned)
  msbg_cnn* cnnCorr = nullptr;  // learned per-V-cycle correction (not owned)
  cudaStream_t stream = nullptr;
  int sx = 0, sy = 0, sz = 0, bsx0 = 0, nLevels = 1;
  int nbx = 0, nby = 0, nbz = 0;
  std::vector<int> blockLevel;
  std::map<int, std::unique_ptr<msbg::Channel>> channels;
  std::string lastError;
  // scratch for block lists (grouped by colour)
  msbg::DeviceBuffer listBuf;
  msbg::DeviceBuffer errBuf;  // int: set by kernels whose bounded wait gave up
  std::vector<int> listHost;
  void* pinned = nullptr;
  size_t pinnedBytes = 0;
  int64_t nb() const { return (int64_t)nbx * nby * nbz; }
};

namespace msbg {

int set_error(msbg_gpu_ctx* ctx, int code, const char* fmt, ...);

#define MSBG_CUDA_TRY(ctx, expr)                                                   \
  do {                                                                             \
    cudaError_t _e = (expr);                                                       \
    if (_e != cudaSuccess)                                                         \
      return ::msbg::set_error((ctx), _e == cudaErrorMemoryAllocation ? MSBG_ENOMEM \
                                                                      : MSBG_ERROR, \
                               "%s: %s (%s:%d)", #expr, cudaGetErrorString(_e),   \
                               __FILE__, __LINE__);                                \
  } while (0)

// Releases the pressure solver state of a context (pressure.cu).
void pressure_release(msbg_gpu_ctx* ctx);
// Releases the FLIP transfer channels of a context (flip.cu).
void flip_release(msbg_gpu_ctx* ctx);
// Releases the particle-splatting buffers of a context (splat.cu).
void splat_release(msbg_gpu_ctx* ctx);
// Releases the mixed-resolution G2P state of a context (flip_mr.cu).
void flip_mr_release(msbg_gpu_ctx* ctx);

// Launches of the 8-colour mean-curvature-flow passes (mcf.cu).  xfaces:
// optional face cache of nSlots value blocks (2 * bsx^2 values each, the
// pool's element type), refilled at the start of the call and kept current by
// the passes; NULL reads the neighbours' x faces from the pool.
cudaError_t launch_mcf(float* pool, const int* slotOf, const int* colourList,
                       const int* colourStart, int nbx, int nby, int nbz, int bsx,
                       float emptyVal, float fullVal, int nIter, float dt, int clamp01,
                       int* errFlag, cudaStream_t stream, void* xfaces = nullptr,
                       int64_t nSlots = 0);
// The same passes on a 16-bit render-density pool (const values raw).
cudaError_t launch_mcf_u16(uint16_t* pool, const int* slotOf, const int* colourList,
                           const int* colourStart, int nbx, int nby, int nbz, int bsx,
                           uint16_t emptyVal, uint16_t fullVal, int nIter, float dt, int clamp01,
                           int* errFlag, cudaStream_t stream, void* xfaces = nullptr,
                           int64_t nSlots = 0);

}  // namespace msbg
