// C-ABI entry points: context, topology, channels, mean-curvature flow.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdarg>
#include <cstring>
#include <new>

#include "common.cuh"
#include "msbg_gpu.h"

namespace msbg {

int set_error(msbg_gpu_ctx* ctx, int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  if (ctx) ctx->lastError = buf;
  return code;
}

namespace {

bool pow2(int v) { return v > 0 && (v & (v - 1)) == 0; }

// Device scalar through which kernels report a bounded wait that gave up.
int* err_flag(msbg_gpu_ctx* ctx) { return ctx->errBuf.as<int>(); }

}  // namespace
}  // namespace msbg

using namespace msbg;

extern "C" int msbg_gpu_init(int device, msbg_gpu_ctx** out) {
  if (!out) return MSBG_EINVARG;
  *out = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n <= 0) return MSBG_ENODEV;
  if (device < 0 || device >= n) return MSBG_EINVARG;
  msbg_gpu_ctx* ctx = new (std::nothrow) msbg_gpu_ctx();
  if (!ctx) return MSBG_ENOMEM;
  ctx->device = device;
  if (cudaSetDevice(device) != cudaSuccess ||
      cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess ||
      ctx->errBuf.ensure(sizeof(int)) != cudaSuccess ||
      cudaMemset(ctx->errBuf.p, 0, sizeof(int)) != cudaSuccess) {
    delete ctx;
    return MSBG_ERROR;
  }
  *out = ctx;
  return MSBG_OK;
}

extern "C" int msbg_gpu_destroy(msbg_gpu_ctx* ctx) {
  if (!ctx) return MSBG_EINVARG;
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  pressure_release(ctx);
  flip_release(ctx);
  splat_release(ctx);
  flip_mr_release(ctx);
  ctx->channels.clear();
  ctx->listBuf.release();
  ctx->errBuf.release();
  if (ctx->pinned) cudaFreeHost(ctx->pinned);
  cudaStreamDestroy(ctx->stream);
  delete ctx;
  return MSBG_OK;
}

extern "C" const char* msbg_gpu_last_error(const msbg_gpu_ctx* ctx) {
  return ctx ? ctx->lastError.c_str() : "null context";
}

extern "C" int msbg_gpu_sync(msbg_gpu_ctx* ctx) {
  if (!ctx) return MSBG_EINVARG;
  MSBG_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  int* f = err_flag(ctx);
  if (f) {
    int h = 0;
    MSBG_CUDA_TRY(ctx, cudaMemcpy(&h, f, sizeof(int), cudaMemcpyDeviceToHost));
    if (h) {
      cudaMemset(f, 0, sizeof(int));
      if (h & MCF_ERR_NOT_VALUE)
        return set_error(ctx, MSBG_EINVARG,
                         "a listed block is not a value block of the pool (skipped)");
      return set_error(ctx, MSBG_ETIMEOUT, "a kernel gave up a bounded wait");
    }
  }
  return MSBG_OK;
}

extern "C" int msbg_gpu_stream(msbg_gpu_ctx* ctx, void** stream) {
  if (!ctx || !stream) return MSBG_EINVARG;
  *stream = ctx->stream;
  return MSBG_OK;
}

extern "C" int msbg_gpu_sync_topology(msbg_gpu_ctx* ctx, const msbg_topo_desc* d) {
  if (!ctx || !d) return MSBG_EINVARG;
  if (!(d->bsx0 == 8 || d->bsx0 == 16 || d->bsx0 == 32))
    return set_error(ctx, MSBG_EINVARG, "bsx0=%d: supported 8, 16, 32", d->bsx0);
  if (d->sx <= 0 || d->sy <= 0 || d->sz <= 0 || d->sx % d->bsx0 || d->sy % d->bsx0 ||
      d->sz % d->bsx0)
    return set_error(ctx, MSBG_EINVARG, "grid %dx%dx%d not a multiple of bsx0=%d", d->sx,
                     d->sy, d->sz, d->bsx0);
  if (d->nLevels < 1 || d->nLevels > 4 || (d->bsx0 >> (d->nLevels - 1)) < 2)
    return set_error(ctx, MSBG_EINVARG, "nLevels=%d invalid for bsx0=%d", d->nLevels, d->bsx0);
  ctx->sx = d->sx;
  ctx->sy = d->sy;
  ctx->sz = d->sz;
  ctx->bsx0 = d->bsx0;
  ctx->nLevels = d->nLevels;
  ctx->nbx = d->sx / d->bsx0;
  ctx->nby = d->sy / d->bsx0;
  ctx->nbz = d->sz / d->bsx0;
  const int64_t nb = ctx->nb();
  ctx->blockLevel.assign(nb, 0);
  if (d->blockLevel) {
    for (int64_t i = 0; i < nb; i++) {
      int l = d->blockLevel[i];
      if (l < 0 || l >= d->nLevels)
        return set_error(ctx, MSBG_EINVARG, "blockLevel[%lld]=%d out of range", (long long)i, l);
      ctx->blockLevel[i] = l;
    }
  }
  ctx->channels.clear();
  return MSBG_OK;
}

namespace {

// Upload of one channel of element type T (float, or uint16_t for the 16-bit
// render density): block kinds -> slot map, value blocks -> device pool.
template <typename T>
int upload_channel_t(msbg_gpu_ctx* ctx, int chan, int level, const int8_t* kind,
                     const T* const* blockPtrs, const T* packed, int dtype, float emptyVal,
                     float fullVal, uint16_t emptyQ, uint16_t fullQ) {
  if (!ctx || !kind || (!blockPtrs && !packed)) return MSBG_EINVARG;
  if (ctx->nbx <= 0) return set_error(ctx, MSBG_EINVARG, "no topology");
  if (level < 0 || level >= ctx->nLevels)
    return set_error(ctx, MSBG_EINVARG, "level %d out of range", level);
  cudaSetDevice(ctx->device);
  const int64_t nb = ctx->nb();
  auto ch = std::make_unique<Channel>();
  ch->level = level;
  ch->bsx = ctx->bsx0 >> level;
  ch->dtype = dtype;
  ch->emptyVal = emptyVal;
  ch->fullVal = fullVal;
  ch->emptyQ = emptyQ;
  ch->fullQ = fullQ;
  ch->kindHost.assign(kind, kind + nb);
  ch->slotHost.resize(nb);
  int64_t s = 0;
  for (int64_t b = 0; b < nb; b++) {
    switch (kind[b]) {
      case MSBG_BLOCK_VALUE: ch->slotHost[b] = (int)s++; break;
      case MSBG_BLOCK_EMPTY: ch->slotHost[b] = SLOT_EMPTY; break;
      case MSBG_BLOCK_FULL: ch->slotHost[b] = SLOT_FULL; break;
      case MSBG_BLOCK_NULL: ch->slotHost[b] = SLOT_NULL; break;
      default: return set_error(ctx, MSBG_EINVARG, "kind[%lld]=%d", (long long)b, kind[b]);
    }
  }
  ch->nValue = s;
  {
    // an earlier channel of this id hands over its allocations (the stream
    // may still read them: it finishes first); it is gone from here on, so a
    // failure below leaves no channel behind
    auto old = ctx->channels.find(chan);
    if (old != ctx->channels.end()) {
      MSBG_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
      ch->reuse(*old->second);
      ctx->channels.erase(old);
    }
  }
  const size_t nv = (size_t)ch->bsx * ch->bsx * ch->bsx;
  const size_t bytes = sizeof(T) * nv * (size_t)s;
  MSBG_CUDA_TRY(ctx, ch->pool.ensure(bytes));
  MSBG_CUDA_TRY(ctx, ch->slot.ensure(sizeof(int) * nb));
  MSBG_CUDA_TRY(ctx, cudaMemcpyAsync(ch->slot.p, ch->slotHost.data(), sizeof(int) * nb,
                                     cudaMemcpyHostToDevice, ctx->stream));
  if (packed) {
    MSBG_CUDA_TRY(ctx, cudaMemcpyAsync(ch->pool.p, packed, bytes, cudaMemcpyHostToDevice,
                                       ctx->stream));
  } else {
    // Gather the scattered host blocks into one pinned staging buffer, then
    // one transfer (MSBG blocks live in separate pool allocations).
    if (ctx->pinnedBytes < bytes) {
      MSBG_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
      if (ctx->pinned) cudaFreeHost(ctx->pinned);
      ctx->pinned = nullptr;
      ctx->pinnedBytes = 0;
      MSBG_CUDA_TRY(ctx, cudaMallocHost(&ctx->pinned, bytes));
      ctx->pinnedBytes = bytes;
    } else {
      MSBG_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    }
    T* stage = static_cast<T*>(ctx->pinned);
    for (int64_t b = 0; b < nb; b++) {
      if (kind[b] != MSBG_BLOCK_VALUE) continue;
      if (!blockPtrs[b])
        return set_error(ctx, MSBG_EINVARG, "value block %lld has no pointer", (long long)b);
      std::memcpy(stage + (size_t)ch->slotHost[b] * nv, blockPtrs[b], sizeof(T) * nv);
    }
    MSBG_CUDA_TRY(ctx, cudaMemcpyAsync(ch->pool.p, stage, bytes, cudaMemcpyHostToDevice,
                                       ctx->stream));
  }
  ctx->channels[chan] = std::move(ch);
  return MSBG_OK;
}

template <typename T>
int download_channel_t(msbg_gpu_ctx* ctx, int chan, int dtype, T* const* blockPtrs, T* packed) {
  if (!ctx || (!blockPtrs && !packed)) return MSBG_EINVARG;
  auto it = ctx->channels.find(chan);
  if (it == ctx->channels.end()) return set_error(ctx, MSBG_EINVARG, "channel %d not uploaded", chan);
  Channel& ch = *it->second;
  if (ch.dtype != dtype)
    return set_error(ctx, MSBG_EINVARG, "channel %d holds another value type", chan);
  cudaSetDevice(ctx->device);
  const size_t nv = (size_t)ch.bsx * ch.bsx * ch.bsx;
  const size_t bytes = sizeof(T) * nv * (size_t)ch.nValue;
  if (packed) {
    MSBG_CUDA_TRY(ctx, cudaMemcpyAsync(packed, ch.pool.p, bytes, cudaMemcpyDeviceToHost,
                                       ctx->stream));
    MSBG_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    return MSBG_OK;
  }
  if (ctx->pinnedBytes < bytes) {
    MSBG_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    if (ctx->pinned) cudaFreeHost(ctx->pinned);
    ctx->pinned = nullptr;
    ctx->pinnedBytes = 0;
    MSBG_CUDA_TRY(ctx, cudaMallocHost(&ctx->pinned, bytes));
    ctx->pinnedBytes = bytes;
  }
  MSBG_CUDA_TRY(ctx, cudaMemcpyAsync(ctx->pinned, ch.pool.p, bytes, cudaMemcpyDeviceToHost,
                                     ctx->stream));
  MSBG_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  const T* stage = static_cast<const T*>(ctx->pinned);
  for (size_t b = 0; b < ch.slotHost.size(); b++) {
    if (ch.slotHost[b] < 0 || !blockPtrs[b]) continue;
    std::memcpy(blockPtrs[b], stage + (size_t)ch.slotHost[b] * nv, sizeof(T) * nv);
  }
  return MSBG_OK;
}

}  // namespace

extern "C" int msbg_gpu_upload_channel(msbg_gpu_ctx* ctx, int chan, int level,
                                       const int8_t* kind, const float* const* blockPtrs,
                                       const float* packed, float emptyVal, float fullVal) {
  return upload_channel_t<float>(ctx, chan, level, kind, blockPtrs, packed, MSBG_F32, emptyVal,
                                 fullVal, 0, 0);
}

extern "C" int msbg_gpu_upload_channel_u16(msbg_gpu_ctx* ctx, int chan, int level,
                                           const int8_t* kind, const uint16_t* const* blockPtrs,
                                           const uint16_t* packed, uint16_t emptyVal,
                                           uint16_t fullVal) {
  return upload_channel_t<uint16_t>(ctx, chan, level, kind, blockPtrs, packed, MSBG_U16, 0.f, 0.f,
                                    emptyVal, fullVal);
}

extern "C" int msbg_gpu_download_channel(msbg_gpu_ctx* ctx, int chan, float* const* blockPtrs,
                                         float* packed) {
  return download_channel_t<float>(ctx, chan, MSBG_F32, blockPtrs, packed);
}

extern "C" int msbg_gpu_download_channel_u16(msbg_gpu_ctx* ctx, int chan,
                                             uint16_t* const* blockPtrs, uint16_t* packed) {
  return download_channel_t<uint16_t>(ctx, chan, MSBG_U16, blockPtrs, packed);
}

extern "C" int msbg_gpu_channel_num_value_blocks(msbg_gpu_ctx* ctx, int chan, int64_t* out) {
  if (!ctx || !out) return MSBG_EINVARG;
  auto it = ctx->channels.find(chan);
  if (it == ctx->channels.end()) return set_error(ctx, MSBG_EINVARG, "channel %d not uploaded", chan);
  *out = it->second->nValue;
  return MSBG_OK;
}

extern "C" int msbg_gpu_channel_device_ptr(msbg_gpu_ctx* ctx, int chan, void** out) {
  if (!ctx || !out) return MSBG_EINVARG;
  auto it = ctx->channels.find(chan);
  if (it == ctx->channels.end()) return set_error(ctx, MSBG_EINVARG, "channel %d not uploaded", chan);
  *out = it->second->pool.p;
  return MSBG_OK;
}

extern "C" int msbg_gpu_pde_mcf(msbg_gpu_ctx* ctx, int chan, const int* blockList, int n,
                                int numIter, float dt, int clamp01) {
  if (!ctx || (n > 0 && !blockList) || n < 0 || numIter < 0) return MSBG_EINVARG;
  auto it = ctx->channels.find(chan);
  if (it == ctx->channels.end()) return set_error(ctx, MSBG_EINVARG, "channel %d not uploaded", chan);
  Channel& ch = *it->second;
  if (ch.level != 0)
    return set_error(ctx, MSBG_EINVARG, "smoother runs on level-0 blocks (src/msbg4.cpp:470)");
  cudaSetDevice(ctx->device);
  // Group the list by colour (src/msbg.h:642-646); the reference skips
  // blocks of other colours in each of its 8 passes (src/msbg4.cpp:456-462).
  int start[9] = {0};
  std::vector<int> lst(n);
  {
    int cnt[8] = {0};
    for (int i = 0; i < n; i++) {
      int b = blockList[i];
      if (b < 0 || b >= ctx->nb() || ch.slotHost[b] < 0)
        return set_error(ctx, MSBG_EINVARG, "blockList[%d]=%d is not a value block", i, b);
      int bx = b % ctx->nbx, by = (b / ctx->nbx) % ctx->nby, bz = b / (ctx->nbx * ctx->nby);
      cnt[(bx & 1) + 2 * (by & 1) + 4 * (bz & 1)]++;
    }
    for (int c = 0; c < 8; c++) start[c + 1] = start[c] + cnt[c];
    int pos[8];
    for (int c = 0; c < 8; c++) pos[c] = start[c];
    for (int i = 0; i < n; i++) {
      int b = blockList[i];
      int bx = b % ctx->nbx, by = (b / ctx->nbx) % ctx->nby, bz = b / (ctx->nbx * ctx->nby);
      lst[pos[(bx & 1) + 2 * (by & 1) + 4 * (bz & 1)]++] = b;
    }
  }
  // The grouped list on the device is reused when a call repeats the last
  // list (the usual time-step loop): no host synchronisation then.  A new
  // list waits for the work that may still read the old one.
  if (lst != ctx->listHost || !ctx->listBuf.p) {
    MSBG_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));  // listBuf may be in use
    MSBG_CUDA_TRY(ctx, ctx->listBuf.ensure(sizeof(int) * std::max(n, 1)));
    ctx->listHost = lst;
    MSBG_CUDA_TRY(ctx, cudaMemcpyAsync(ctx->listBuf.p, ctx->listHost.data(), sizeof(int) * n,
                                       cudaMemcpyHostToDevice, ctx->stream));
  }
  const int nIter = numIter + (numIter & 1);  // src/msbg4.cpp:150-152
  int* ef = err_flag(ctx);
  if (!ef) return set_error(ctx, MSBG_ENOMEM, "error flag allocation failed");
  // the face cache: each block's two x planes, contiguous, so the x halo of a
  // neighbour is read in full sectors instead of one 4-byte value per row
  const size_t esz = ch.dtype == MSBG_U16 ? 2 : 4;
  MSBG_CUDA_TRY(ctx, ch.xfaces.ensure(esz * 2 * ch.bsx * ch.bsx * (size_t)std::max<int64_t>(
                                                                      ch.nValue, 1)));
  if (ch.dtype == MSBG_U16)
    MSBG_CUDA_TRY(ctx, launch_mcf_u16(ch.pool.as<uint16_t>(), ch.slot.as<int>(),
                                      ctx->listBuf.as<int>(), start, ctx->nbx, ctx->nby, ctx->nbz,
                                      ch.bsx, ch.emptyQ, ch.fullQ, nIter, dt, clamp01, ef,
                                      ctx->stream, ch.xfaces.p, ch.nValue));
  else
    MSBG_CUDA_TRY(ctx, launch_mcf(ch.pool.as<float>(), ch.slot.as<int>(), ctx->listBuf.as<int>(),
                                  start, ctx->nbx, ctx->nby, ctx->nbz, ch.bsx, ch.emptyVal,
                                  ch.fullVal, nIter, dt, clamp01, ef, ctx->stream, ch.xfaces.p,
                                  ch.nValue));
  return MSBG_OK;
}

extern "C" int msbg_gpu_pde_mcf_device(msbg_gpu_ctx* ctx, float* pool, const int* slotOf,
                                       const int* colourList, const int* colourStartHost,
                                       int nbx, int nby, int nbz, int bsx, float emptyVal,
                                       float fullVal, int numIter, float dt, int clamp01,
                                       void* stream) {
  if (!ctx || !pool || !slotOf || !colourList || !colourStartHost || numIter < 0)
    return MSBG_EINVARG;
  if (!(bsx == 8 || bsx == 16 || bsx == 32)) return set_error(ctx, MSBG_EINVARG, "bsx=%d", bsx);
  if (!pow2(bsx)) return MSBG_EINVARG;
  if (reinterpret_cast<uintptr_t>(pool) % 8)
    return set_error(ctx, MSBG_EINVARG, "pool must be 8-byte aligned (voxel pairs are copied whole)");
  const int nIter = numIter + (numIter & 1);
  int* ef = err_flag(ctx);
  if (!ef) return set_error(ctx, MSBG_ENOMEM, "error flag allocation failed");
  MSBG_CUDA_TRY(ctx, launch_mcf(pool, slotOf, colourList, colourStartHost, nbx, nby, nbz, bsx,
                                emptyVal, fullVal, nIter, dt, clamp01, ef,
                                (cudaStream_t)stream));
  return MSBG_OK;
}
