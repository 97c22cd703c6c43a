// The learned 3D CNN on the tensor cores: implicit-GEMM convolution with
// tcgen05 (BF16 operands in shared memory, FP32 accumulators in tensor
// memory), weight gradients, loss, Adam and the C ABI of include/msbg_cnn.h.
// No counterpart in the reference.
//
// Convolution as an implicit GEMM.  One CTA holds a tile's input (16^3 cells
// plus a 1-cell halo, 16 channels) in shared memory as two channel halves,
// each a [z][y][x] array of 18^3 cells x 16 bytes (8 bf16 channels).  An
// M = 128 block of output cells is 8 consecutive x by the 16 y rows of one z
// plane; its A operand for kernel tap (kz, ky, kx) is the same array read
// from a start address shifted by the tap: 8 rows (x) of 16 bytes form a
// core matrix, the 16 y rows are core-matrix groups 18 cells apart (SBO) and
// the two channel halves are the two K halves (LBO).  So every tap is one
// tcgen05.mma of M = 128, N = 16, K = 16 straight from the activations, with
// no im2col copy; 27 taps accumulate in tensor memory.  While the epilogue
// of plane z reads its accumulators, the MMAs of plane z+1 run into the
// other half of a 64-column tensor-memory allocation.
//
// Backward: the data gradient of a "same" convolution is a "same"
// convolution of the output gradient with the flipped, transposed kernel, so
// it runs through the same kernel (weight image `bwd`) with the ReLU mask of
// the layer input applied in the epilogue.  The weight gradient, a
// 432 x 16 result reduced over all cells, runs on FP32 CUDA cores with
// per-CTA partials reduced in a fixed order (deterministic).
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include "cnn.cuh"
#include "cnn_tc.cuh"
#include "common.cuh"
#include "msbg_cnn.h"

namespace msbg {
namespace cnn {

// ---------------------------------------------------------------------------
// weight images
// ---------------------------------------------------------------------------
// Image element (tap, n, k) of the B operand (N x K, K-major, no swizzle):
// tap*256 + (k>>3)*128 + n*8 + (k&7).  Forward: n = cout, k = cin, W[n][k][tap].
// Backward-data: n = cin, k = cout, W[k][n][26 - tap].  Unused rows/columns
// (cin = 4 of layer 1, cout = 1 of layer 4) are zero.
__global__ void k_pack(const float* __restrict__ w, __nv_bfloat16* __restrict__ fwd,
                       __nv_bfloat16* __restrict__ bwd) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= NLAYER * WIMG) return;
  const int l = i / WIMG, e = i % WIMG;
  const int tap = e / 256, r = e % 256, kh = r / 128, n = (r % 128) / 8, k = kh * 8 + (r % 8);
  const int cin = layer_cin(l), cout = layer_cout(l);
  const float* W = w + layer_off(l);
  float f = 0.f, b = 0.f;
  if (n < cout && k < cin) f = W[((size_t)n * cin + k) * 27 + tap];
  if (n < cin && k < cout) b = W[((size_t)k * cin + n) * 27 + (26 - tap)];
  fwd[i] = __float2bfloat16_rn(f);
  bwd[i] = __float2bfloat16_rn(b);
}

// ---------------------------------------------------------------------------
// layout conversion
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t pack_bf2(float a, float b) {
  __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
  return *reinterpret_cast<uint32_t*>(&h);
}

// feat [n][4][NPAD] FP32 planes -> padded bf16 layout (half 0: the 4
// features and 4 zero channels; half 1: zeros).  One thread per padded cell.
__global__ void k_feat_pack(int n, const float* __restrict__ feat, uint4* __restrict__ x) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= (int64_t)n * NPAD) return;
  const int64_t t = i / NPAD;
  const int c = (int)(i % NPAD);
  const float* f = feat + t * NFEAT * NPAD;
  uint4 v;
  v.x = pack_bf2(f[c], f[NPAD + c]);
  v.y = pack_bf2(f[2 * NPAD + c], f[3 * NPAD + c]);
  v.z = 0u;
  v.w = 0u;
  x[(t * 2) * NPAD + c] = v;
  x[(t * 2 + 1) * NPAD + c] = make_uint4(0, 0, 0, 0);
}

// ---------------------------------------------------------------------------
// convolution (tcgen05)
// ---------------------------------------------------------------------------
// One CTA of 256 threads per SM walks its tiles.  A tile's input (padded
// layout) arrives by two bulk copies of one channel half each.  Thread 0
// issues the 54 MMAs of plane z+1 (into the other TMEM column set) before
// everyone drains plane z: warp w reads TMEM lanes 32*(w%4).. of column half
// w/4 (the x half of the plane), applies the epilogue and writes the cells.
// The next tile's copies are issued as soon as the last plane's MMAs are
// done, so they overlap the last epilogue.  A tcgen05.mma of N = 16 costs
// about 45 cycles whatever its operands (measured), so 864 MMAs bound a tile
// to ~20 us per layer.  Every wait is bounded.
template <int EPI>
__global__ void __launch_bounds__(CONV_THREADS, 1) k_conv3_tc(ConvArgs a) {
  extern __shared__ __align__(1024) uint8_t sm[];
  uint8_t* act = sm;
  uint8_t* wts = sm + 2 * HALF_BYTES;
  uint64_t* bar = reinterpret_cast<uint64_t*>(sm + 2 * HALF_BYTES + WIMG * 2);  // [0,1] MMA, [2] input
  uint32_t* tslot = reinterpret_cast<uint32_t*>(bar + 3);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int G = gridDim.x;
  if ((int)blockIdx.x >= a.n) return;

  for (int i = tid; i < WIMG * 2 / 16; i += CONV_THREADS)
    reinterpret_cast<uint4*>(wts)[i] = reinterpret_cast<const uint4*>(a.wimg)[i];
  if (tid == 0) {
    for (int b = 0; b < 3; b++) mbar_init(&bar[b], 1);
    fence_mbar_init();
  }
  if (warp == 0) {
    tmem_alloc(tslot, 64);
    tmem_relinquish();
  }
  fence_proxy_async();  // the weight image (generic writes) -> tensor core
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tbase = *tslot;
  const uint32_t idesc = idesc_bf16_f32(128, 16);
  const uint64_t a0 = smem_desc(smem_addr(act), HALF_BYTES, PD * 16);
  const uint64_t b0 = smem_desc(smem_addr(wts), 256, 128);
  auto load_tile = [&](int t) {
    mbar_expect_tx(&bar[2], 2 * HALF_BYTES);
    bulk_g2s(act, a.in + (size_t)t * 2 * NPAD, HALF_BYTES, &bar[2]);
    bulk_g2s(act + HALF_BYTES, a.in + ((size_t)t * 2 + 1) * NPAD, HALF_BYTES, &bar[2]);
  };
  // Descriptors are built once; the start address field (address / 16) is the
  // low bits: one cell = 16 bytes = +1, and no start reaches 2^14 * 16 bytes.
  auto issue = [&](int z) {
    tc_fence_after();
    const uint32_t cb = tbase + (uint32_t)((z & 1) * 32);
    const uint64_t az = a0 + (uint64_t)(z * PLANE);
#pragma unroll
    for (int tap = 0; tap < 27; tap++)
#pragma unroll
      for (int xh = 0; xh < 2; xh++) {
        const int kz = tap / 9, ky = (tap / 3) % 3, kx = tap % 3;
        mma_bf16(cb + 16 * xh, az + (uint64_t)((kz * PD + ky) * PD + 8 * xh + kx),
                 b0 + (uint64_t)(tap * 32), idesc, tap > 0 ? 1u : 0u);
      }
    mma_commit(&bar[z & 1]);
  };
  if (tid == 0) load_tile(blockIdx.x);
  const int xh = warp >> 2, quarter = warp & 3;
  const int r = 32 * quarter + lane;
  const int x = 8 * xh + (r & 7), y = r >> 3;
  bool ok = true;
  for (int j = 0, t = blockIdx.x; t < a.n && ok; j++, t += G) {
    if (!__syncthreads_and(mbar_wait(&bar[2], (uint32_t)(j & 1)))) {
      ok = false;
      break;
    }
    if (tid == 0) issue(0);
    const float s = (EPI == EPI_OUT0 && a.outScale) ? a.outScale[t] : 1.f;
    const int64_t base = (EPI == EPI_OUT0) ? (a.outOff ? a.outOff[t] : (int64_t)t * NCELL) : 0;
    for (int z = 0; z < TS; z++) {
      if (tid == 0 && z + 1 < TS) issue(z + 1);
      if (!__syncthreads_and(mbar_wait(&bar[z & 1], (uint32_t)((z >> 1) & 1)))) {
        ok = false;
        break;
      }
      // the tile's MMAs are all done: its input buffer takes the next tile
      if (z == TS - 1 && tid == 0 && t + G < a.n) load_tile(t + G);
      tc_fence_after();
      float v[16];
      tmem_ld16(tbase + ((uint32_t)(32 * quarter) << 16) + (uint32_t)((z & 1) * 32 + 16 * xh), v);
      const int cell = x + TS * (y + TS * z);
      if (EPI == EPI_OUT0) {
        a.out0[base + cell] = v[0] * s;
      } else {
        const size_t pc = (size_t)pad_index(cell);
        const size_t o0 = ((size_t)t * 2) * NPAD + pc, o1 = o0 + NPAD;
        if (EPI == EPI_MASK) {
          uint4 m2[2] = {a.mask[o0], a.mask[o1]};
          const __nv_bfloat16* mb = reinterpret_cast<const __nv_bfloat16*>(m2);
#pragma unroll
          for (int c = 0; c < 16; c++)
            if (!(__bfloat162float(mb[c]) > 0.f)) v[c] = 0.f;
        } else {
#pragma unroll
          for (int c = 0; c < 16; c++) v[c] = fmaxf(v[c], 0.f);
        }
        uint4 q0, q1;
        q0.x = pack_bf2(v[0], v[1]);
        q0.y = pack_bf2(v[2], v[3]);
        q0.z = pack_bf2(v[4], v[5]);
        q0.w = pack_bf2(v[6], v[7]);
        q1.x = pack_bf2(v[8], v[9]);
        q1.y = pack_bf2(v[10], v[11]);
        q1.z = pack_bf2(v[12], v[13]);
        q1.w = pack_bf2(v[14], v[15]);
        a.out[o0] = q0;
        a.out[o1] = q1;
      }
      tc_fence_before();
      __syncthreads();
    }
  }
  if (!ok && tid == 0) {
    // a wait gave up: flag it, give the work in flight one more bounded wait
    atomicExch(a.err, 1);
    mbar_wait(&bar[0], 0);
    mbar_wait(&bar[1], 0);
    mbar_wait(&bar[2], 0);
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0) tmem_dealloc(tbase, 64);
}

// ---------------------------------------------------------------------------
// weight gradient (FP32 CUDA cores)
// ---------------------------------------------------------------------------
// partial[blockIdx][co][ci][tap] = sum over this CTA's tiles and their cells o
// of dz[o][co] * X[o + tap][ci], X the layer input on the padded box and dz
// the output gradient (both in the padded bf16 layout, as the forward pass
// reads them).  Thread (co, ci) = (tid >> 4, tid & 15).
constexpr int WG_SLAB = 4;  // output planes per shared-memory slab
constexpr size_t WG_SMEM = (size_t)(WG_SLAB + 2) * PLANE * 32 + (size_t)WG_SLAB * TS * TS * 32;

__global__ void __launch_bounds__(256) k_wgrad(int n, const uint4* __restrict__ X,
                                               const uint4* __restrict__ dz,
                                               float* __restrict__ partial) {
  extern __shared__ __align__(16) uint8_t smw[];
  __nv_bfloat16* Xs = reinterpret_cast<__nv_bfloat16*>(smw);  // [(WG_SLAB+2)*PLANE][16]
  __nv_bfloat16* Ds = reinterpret_cast<__nv_bfloat16*>(smw + (size_t)(WG_SLAB + 2) * PLANE * 32);
  const int tid = threadIdx.x, co = tid >> 4, ci = tid & 15;
  float acc[27];
#pragma unroll
  for (int k = 0; k < 27; k++) acc[k] = 0.f;
  for (int t = blockIdx.x; t < n; t += gridDim.x) {
    const uint4* Xt = X + (size_t)t * 2 * NPAD;
    const uint4* Dt = dz + (size_t)t * 2 * NPAD;
    for (int z0 = 0; z0 < TS; z0 += WG_SLAB) {
      __syncthreads();
      for (int c = tid; c < (WG_SLAB + 2) * PLANE; c += 256) {
        const int pc = z0 * PLANE + c;
        reinterpret_cast<uint4*>(Xs)[2 * c] = Xt[pc];
        reinterpret_cast<uint4*>(Xs)[2 * c + 1] = Xt[NPAD + pc];
      }
      for (int c = tid; c < WG_SLAB * TS * TS; c += 256) {
        const int pc = pad_index(z0 * TS * TS + c);
        reinterpret_cast<uint4*>(Ds)[2 * c] = Dt[pc];
        reinterpret_cast<uint4*>(Ds)[2 * c + 1] = Dt[NPAD + pc];
      }
      __syncthreads();
#pragma unroll 1
      for (int o = 0; o < WG_SLAB * TS * TS; o++) {
        const float d = __bfloat162float(Ds[o * NC + co]);
        if (d == 0.f) continue;
        const int ox = o % TS, oy = (o / TS) % TS, oz = o / (TS * TS);
        const int base = ox + PD * (oy + PD * oz);
#pragma unroll
        for (int k = 0; k < 27; k++) {
          const int kz = k / 9, ky = (k / 3) % 3, kx = k % 3;
          acc[k] = fmaf(d, __bfloat162float(Xs[(base + kx + PD * (ky + PD * kz)) * NC + ci]), acc[k]);
        }
      }
    }
  }
  float* p = partial + (size_t)blockIdx.x * NC * NC * 27 + ((size_t)co * NC + ci) * 27;
#pragma unroll
  for (int k = 0; k < 27; k++) p[k] = acc[k];
}

// grad[layer weights] = sum over the CTA partials, fixed order, FP64.
__global__ void k_wgrad_reduce(const float* __restrict__ partial, int nPart, int cin, int cout,
                               float* __restrict__ g) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= cout * cin * 27) return;
  const int co = i / (cin * 27), ci = (i / 27) % cin, k = i % 27;
  double s = 0;
  for (int p = 0; p < nPart; p++) s += partial[(size_t)p * NC * NC * 27 + ((size_t)co * NC + ci) * 27 + k];
  g[i] = (float)s;
}

// ---------------------------------------------------------------------------
// loss, Adam
// ---------------------------------------------------------------------------
// loss = sum m (y - t)^2 / count; dy = 2 m (y - t) / count into channel 0 of
// a padded-layout bf16 gradient (all other values stay 0).  Per-CTA partial.
constexpr int LOSS_GRID = 148 * 2;
__global__ void __launch_bounds__(512) k_loss(int64_t nc, const float* __restrict__ y,
                                              const float* __restrict__ tgt,
                                              const float* __restrict__ m, float invCount,
                                              __nv_bfloat16* __restrict__ dy,
                                              double* __restrict__ partial) {
  // dy: padded layout, channel 0 of half 0 at the interior cells
  __shared__ double ws[16];
  double acc = 0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nc;
       i += (int64_t)gridDim.x * blockDim.x) {
    const float d = m[i] > 0.f ? y[i] - tgt[i] : 0.f;
    acc += (double)d * d;
    if (dy) {
      const int64_t t = i / NCELL;
      dy[((size_t)t * 2 * NPAD + pad_index((int)(i % NCELL))) * 8] =
          __float2bfloat16_rn(2.f * d * invCount);
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) s += ws[w];
    partial[blockIdx.x] = s * invCount;
  }
}

__global__ void k_adam(float* __restrict__ w, float* __restrict__ m, float* __restrict__ v,
                       const float* __restrict__ g, int n, float lr, float b1, float b2,
                       float eps, float c1, float c2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.f - b1) * gi;
  const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

// Gather of training / inference samples lives in cnn_features.cu.

}  // namespace cnn
}  // namespace msbg

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
using namespace msbg;
using namespace msbg::cnn;

struct msbg_cnn {
  int device = 0;
  cudaStream_t stream = nullptr;
  std::string lastError;
  DeviceBuffer w, m, v, g;       // FP32 [NPARAM]
  DeviceBuffer imgF, imgB;       // bf16 [NLAYER][WIMG]
  DeviceBuffer err;              // int
  int step = 0;
  int numSMs = 148;
  // training scratch for `cap` tiles
  int cap = 0;
  DeviceBuffer x0, a1, a2, a3, y, dy, dz3, dz2, dz1, part, lossPart;  // padded layout
};

namespace {

int cnn_error(msbg_cnn* n, int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  if (n) n->lastError = buf;
  return code;
}

#define CNN_TRY(net, expr)                                                                 \
  do {                                                                                     \
    cudaError_t _e = (expr);                                                               \
    if (_e != cudaSuccess)                                                                 \
      return cnn_error((net), _e == cudaErrorMemoryAllocation ? MSBG_ENOMEM : MSBG_ERROR, \
                       "%s: %s (%s:%d)", #expr, cudaGetErrorString(_e), __FILE__, __LINE__); \
  } while (0)

void set_attrs() {
  static bool done = false;
  if (done) return;
  cudaFuncSetAttribute(k_conv3_tc<EPI_RELU>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)CONV_SMEM);
  cudaFuncSetAttribute(k_conv3_tc<EPI_MASK>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)CONV_SMEM);
  cudaFuncSetAttribute(k_conv3_tc<EPI_OUT0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)CONV_SMEM);
  cudaFuncSetAttribute(k_wgrad, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)WG_SMEM);
  done = true;
}

template <int EPI>
void conv(msbg_cnn* net, int layer, bool backward, int n, const uint4* in, uint4* out,
          const uint4* mask, float* out0, const int64_t* outOff, const float* outScale,
          cudaStream_t st) {
  ConvArgs a;
  a.n = n;
  a.in = in;
  a.wimg = (backward ? net->imgB : net->imgF).as<__nv_bfloat16>() + (size_t)layer * WIMG;
  a.out = out;
  a.mask = mask;
  a.out0 = out0;
  a.outOff = outOff;
  a.outScale = outScale;
  a.err = net->err.as<int>();
  const int grid = std::min(n, net->numSMs);
  k_conv3_tc<EPI><<<grid, CONV_THREADS, CONV_SMEM, st>>>(a);
}

void feat_pack(int n, const float* feat, uint4* x0, cudaStream_t st) {
  const int64_t cnt = (int64_t)n * NPAD;
  k_feat_pack<<<(unsigned)((cnt + 255) / 256), 256, 0, st>>>(n, feat, x0);
}

int ensure_cap(msbg_cnn* net, int n) {
  if (n <= net->cap) return MSBG_OK;
  const size_t act = (size_t)n * ACT_BYTES;
  DeviceBuffer* bufs[] = {&net->x0, &net->a1, &net->a2, &net->a3,
                          &net->dz3, &net->dz2, &net->dz1, &net->dy};
  for (DeviceBuffer* b : bufs) {
    CNN_TRY(net, b->ensure(act));
    CNN_TRY(net, cudaMemsetAsync(b->p, 0, act, net->stream));  // zero halos
  }
  CNN_TRY(net, net->y.ensure((size_t)n * NCELL * sizeof(float)));
  CNN_TRY(net, net->part.ensure((size_t)net->numSMs * NC * NC * 27 * sizeof(float)));
  CNN_TRY(net, net->lossPart.ensure(LOSS_GRID * sizeof(double)));
  net->cap = n;
  return MSBG_OK;
}

int pack(msbg_cnn* net) {
  k_pack<<<(NLAYER * WIMG + 255) / 256, 256, 0, net->stream>>>(
      net->w.as<float>(), net->imgF.as<__nv_bfloat16>(), net->imgB.as<__nv_bfloat16>());
  CNN_TRY(net, cudaGetLastError());
  return MSBG_OK;
}

int check_err(msbg_cnn* net) {
  int e = 0;
  CNN_TRY(net, cudaMemcpyAsync(&e, net->err.p, sizeof(int), cudaMemcpyDeviceToHost, net->stream));
  CNN_TRY(net, cudaStreamSynchronize(net->stream));
  if (e) {
    cudaMemsetAsync(net->err.p, 0, sizeof(int), net->stream);
    return cnn_error(net, MSBG_ETIMEOUT, "a tensor-core wait gave up");
  }
  return MSBG_OK;
}

}  // namespace

namespace msbg {
namespace cnn {
// Forward pass into out0 (see msbg_cnn_forward); used by the pressure solver.
int forward(msbg_cnn* net, const float* feat, float* out0, const int64_t* outOff,
            const float* outScale, int n, cudaStream_t st, uint4* x0, uint4* s1, uint4* s2) {
  if (n <= 0) return MSBG_OK;
  feat_pack(n, feat, x0, st);
  conv<EPI_RELU>(net, 0, false, n, x0, s1, nullptr, nullptr, nullptr, nullptr, st);
  conv<EPI_RELU>(net, 1, false, n, s1, s2, nullptr, nullptr, nullptr, nullptr, st);
  conv<EPI_RELU>(net, 2, false, n, s2, s1, nullptr, nullptr, nullptr, nullptr, st);
  conv<EPI_OUT0>(net, 3, false, n, s1, nullptr, nullptr, out0, outOff, outScale, st);
  return cudaGetLastError() == cudaSuccess ? MSBG_OK : MSBG_ERROR;
}

int take_error(msbg_cnn* net, cudaStream_t st) {
  int e = 0;
  if (cudaMemcpyAsync(&e, net->err.p, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return MSBG_ERROR;
  if (e) cudaMemsetAsync(net->err.p, 0, sizeof(int), st);
  return e ? MSBG_ETIMEOUT : MSBG_OK;
}
}  // namespace cnn
}  // namespace msbg

extern "C" int msbg_cnn_create(int device, msbg_cnn** out) {
  if (!out) return MSBG_EINVARG;
  *out = nullptr;
  int nd = 0;
  if (cudaGetDeviceCount(&nd) != cudaSuccess || device < 0 || device >= nd) return MSBG_ENODEV;
  cudaSetDevice(device);
  auto* net = new msbg_cnn();
  net->device = device;
  cudaDeviceGetAttribute(&net->numSMs, cudaDevAttrMultiProcessorCount, device);
  set_attrs();
  if (cudaStreamCreateWithFlags(&net->stream, cudaStreamNonBlocking) != cudaSuccess ||
      net->w.ensure(NPARAM * sizeof(float)) != cudaSuccess ||
      net->m.ensure(NPARAM * sizeof(float)) != cudaSuccess ||
      net->v.ensure(NPARAM * sizeof(float)) != cudaSuccess ||
      net->g.ensure(NPARAM * sizeof(float)) != cudaSuccess ||
      net->imgF.ensure(NLAYER * WIMG * 2) != cudaSuccess ||
      net->imgB.ensure(NLAYER * WIMG * 2) != cudaSuccess ||
      net->err.ensure(sizeof(int)) != cudaSuccess) {
    if (net->stream) cudaStreamDestroy(net->stream);
    delete net;
    return MSBG_ENOMEM;
  }
  cudaMemsetAsync(net->err.p, 0, sizeof(int), net->stream);
  cudaMemsetAsync(net->m.p, 0, NPARAM * sizeof(float), net->stream);
  cudaMemsetAsync(net->v.p, 0, NPARAM * sizeof(float), net->stream);
  // He-uniform initial weights from a fixed seed
  std::vector<float> w(NPARAM);
  std::mt19937_64 rng(12345);
  for (int l = 0; l < NLAYER; l++) {
    const float b = std::sqrt(6.0f / (27.0f * layer_cin(l)));
    std::uniform_real_distribution<float> U(-b, b);
    for (int i = 0; i < layer_cout(l) * layer_cin(l) * 27; i++) w[layer_off(l) + i] = U(rng);
  }
  cudaMemcpyAsync(net->w.p, w.data(), NPARAM * sizeof(float), cudaMemcpyHostToDevice, net->stream);
  if (pack(net) != MSBG_OK || cudaStreamSynchronize(net->stream) != cudaSuccess) {
    cudaStreamDestroy(net->stream);
    delete net;
    return MSBG_ERROR;
  }
  *out = net;
  return MSBG_OK;
}

extern "C" int msbg_cnn_destroy(msbg_cnn* net) {
  if (!net) return MSBG_EINVARG;
  cudaSetDevice(net->device);
  cudaStreamSynchronize(net->stream);
  cudaStreamDestroy(net->stream);
  delete net;
  return MSBG_OK;
}

extern "C" const char* msbg_cnn_last_error(msbg_cnn* net) {
  return net ? net->lastError.c_str() : "null network";
}

extern "C" int msbg_cnn_num_params(void) { return NPARAM; }

extern "C" int msbg_cnn_set_weights(msbg_cnn* net, const float* w, int64_t n) {
  if (!net || !w || n != NPARAM) return cnn_error(net, MSBG_EINVARG, "expected %d weights", NPARAM);
  cudaSetDevice(net->device);
  CNN_TRY(net, cudaMemcpyAsync(net->w.p, w, NPARAM * sizeof(float), cudaMemcpyHostToDevice, net->stream));
  CNN_TRY(net, cudaMemsetAsync(net->m.p, 0, NPARAM * sizeof(float), net->stream));
  CNN_TRY(net, cudaMemsetAsync(net->v.p, 0, NPARAM * sizeof(float), net->stream));
  net->step = 0;
  int rc = pack(net);
  if (rc) return rc;
  CNN_TRY(net, cudaStreamSynchronize(net->stream));
  return MSBG_OK;
}

extern "C" int msbg_cnn_get_weights(msbg_cnn* net, float* w, int64_t n) {
  if (!net || !w || n != NPARAM) return cnn_error(net, MSBG_EINVARG, "expected %d weights", NPARAM);
  cudaSetDevice(net->device);
  CNN_TRY(net, cudaMemcpyAsync(w, net->w.p, NPARAM * sizeof(float), cudaMemcpyDeviceToHost, net->stream));
  CNN_TRY(net, cudaStreamSynchronize(net->stream));
  return MSBG_OK;
}

extern "C" int msbg_cnn_forward(msbg_cnn* net, const float* feat, float* out, int n) {
  if (!net || n < 0 || (n > 0 && (!feat || !out))) return cnn_error(net, MSBG_EINVARG, "bad arguments");
  if (n == 0) return MSBG_OK;
  cudaSetDevice(net->device);
  int rc = ensure_cap(net, n);
  if (rc) return rc;
  rc = forward(net, feat, out, nullptr, nullptr, n, net->stream, net->x0.as<uint4>(),
               net->a1.as<uint4>(), net->a2.as<uint4>());
  if (rc) return cnn_error(net, rc, "forward launch failed: %s", cudaGetErrorString(cudaGetLastError()));
  return check_err(net);
}

// Loss and gradient of a batch (device inputs); the gradient stays on the
// device (and is copied to gradHost when given).
extern "C" int msbg_cnn_loss_grad(msbg_cnn* net, const float* feat, const float* target,
                                  const float* mask, int n, double count, double* loss,
                                  float* gradHost) {
  if (!net || n <= 0 || !feat || !target || !mask || !(count > 0))
    return cnn_error(net, MSBG_EINVARG, "bad arguments");
  cudaSetDevice(net->device);
  int rc = ensure_cap(net, n);
  if (rc) return rc;
  cudaStream_t st = net->stream;
  uint4* x0 = net->x0.as<uint4>();
  uint4* a1 = net->a1.as<uint4>();
  uint4* a2 = net->a2.as<uint4>();
  uint4* a3 = net->a3.as<uint4>();
  uint4* dy = net->dy.as<uint4>();
  uint4* dz3 = net->dz3.as<uint4>();
  uint4* dz2 = net->dz2.as<uint4>();
  uint4* dz1 = net->dz1.as<uint4>();
  float* y = net->y.as<float>();
  // forward, keeping the activations
  feat_pack(n, feat, x0, st);
  conv<EPI_RELU>(net, 0, false, n, x0, a1, nullptr, nullptr, nullptr, nullptr, st);
  conv<EPI_RELU>(net, 1, false, n, a1, a2, nullptr, nullptr, nullptr, nullptr, st);
  conv<EPI_RELU>(net, 2, false, n, a2, a3, nullptr, nullptr, nullptr, nullptr, st);
  conv<EPI_OUT0>(net, 3, false, n, a3, nullptr, nullptr, y, nullptr, nullptr, st);
  // loss and dL/dy
  k_loss<<<LOSS_GRID, 512, 0, st>>>((int64_t)n * NCELL, y, target, mask, (float)(1.0 / count),
                                    reinterpret_cast<__nv_bfloat16*>(dy), net->lossPart.as<double>());
  // backward-data through layers 4, 3, 2 (ReLU masks of their inputs)
  conv<EPI_MASK>(net, 3, true, n, dy, dz3, a3, nullptr, nullptr, nullptr, st);
  conv<EPI_MASK>(net, 2, true, n, dz3, dz2, a2, nullptr, nullptr, nullptr, st);
  conv<EPI_MASK>(net, 1, true, n, dz2, dz1, a1, nullptr, nullptr, nullptr, st);
  // weight gradients
  const int grid = std::min(n, net->numSMs);
  float* part = net->part.as<float>();
  float* g = net->g.as<float>();
  const uint4* dzs[NLAYER] = {dz1, dz2, dz3, dy};
  const uint4* ins[NLAYER] = {x0, a1, a2, a3};
  for (int l = 0; l < NLAYER; l++) {
    k_wgrad<<<grid, 256, WG_SMEM, st>>>(n, ins[l], dzs[l], part);
    const int cnt = layer_cout(l) * layer_cin(l) * 27;
    k_wgrad_reduce<<<(cnt + 255) / 256, 256, 0, st>>>(part, grid, layer_cin(l), layer_cout(l),
                                                      g + layer_off(l));
  }
  CNN_TRY(net, cudaGetLastError());
  std::vector<double> lp(LOSS_GRID);
  CNN_TRY(net, cudaMemcpyAsync(lp.data(), net->lossPart.p, LOSS_GRID * sizeof(double),
                               cudaMemcpyDeviceToHost, st));
  if (gradHost)
    CNN_TRY(net, cudaMemcpyAsync(gradHost, g, NPARAM * sizeof(float), cudaMemcpyDeviceToHost, st));
  rc = check_err(net);
  if (rc) return rc;
  if (loss) {
    double s = 0;
    for (double v : lp) s += v;
    *loss = s;
  }
  return MSBG_OK;
}

extern "C" int msbg_cnn_adam_step(msbg_cnn* net, float lr, float beta1, float beta2, float eps) {
  if (!net || !(lr > 0)) return cnn_error(net, MSBG_EINVARG, "bad arguments");
  cudaSetDevice(net->device);
  net->step++;
  const float c1 = 1.f - std::pow(beta1, (float)net->step);
  const float c2 = 1.f - std::pow(beta2, (float)net->step);
  k_adam<<<(NPARAM + 255) / 256, 256, 0, net->stream>>>(net->w.as<float>(), net->m.as<float>(),
                                                       net->v.as<float>(), net->g.as<float>(),
                                                       NPARAM, lr, beta1, beta2, eps, c1, c2);
  int rc = pack(net);
  if (rc) return rc;
  CNN_TRY(net, cudaStreamSynchronize(net->stream));
  return MSBG_OK;
}
