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
// convolution (tcgen05)
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t pack_bf2(float a, float b) {
  __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
  return *reinterpret_cast<uint32_t*>(&h);
}

template <int IN, int EPI>
__global__ void __launch_bounds__(CONV_THREADS, 1) k_conv3_tc(ConvArgs a) {
  extern __shared__ __align__(1024) uint8_t sm[];
  uint8_t* act = sm;
  uint8_t* wts = sm + 2 * HALF_BYTES;
  uint64_t* bar = reinterpret_cast<uint64_t*>(sm + 2 * HALF_BYTES + WIMG * 2);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(bar + 2);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if ((int)blockIdx.x >= a.n) return;

  for (int i = tid; i < WIMG * 2 / 16; i += CONV_THREADS)
    reinterpret_cast<uint4*>(wts)[i] = reinterpret_cast<const uint4*>(a.wimg)[i];
  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    fence_mbar_init();
  }
  if (warp == 0) {
    tmem_alloc(tslot, 64);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tbase = *tslot;
  const uint32_t idesc = idesc_bf16_f32(128, 16);
  const uint32_t actA = smem_addr(act), wA = smem_addr(wts);
  // one plane = 2 M blocks (x halves) x 27 taps, into columns (z&1)*32 + 16*xh
  auto issue = [&](int z) {
    tc_fence_after();
    const uint32_t cb = tbase + (uint32_t)((z & 1) * 32);
#pragma unroll 1
    for (int xh = 0; xh < 2; xh++)
#pragma unroll 1
      for (int tap = 0; tap < 27; tap++) {
        const int kz = tap / 9, ky = (tap / 3) % 3, kx = tap % 3;
        const uint32_t aa = actA + (uint32_t)((((z + kz) * PD + ky) * PD + 8 * xh + kx) * 16);
        mma_bf16(cb + 16 * xh, smem_desc(aa, HALF_BYTES, PD * 16),
                 smem_desc(wA + tap * 512, 256, 128), idesc, tap > 0 ? 1u : 0u);
      }
    mma_commit(&bar[z & 1]);
  };
  bool ok = true;
  for (int t = blockIdx.x; t < a.n && ok; t += gridDim.x) {
    // ---- the tile's input -> shared memory (bf16, two channel halves) ----
    if (IN == IN_FEAT) {
      const float* f = a.feat + (size_t)t * NFEAT * NPAD;
      for (int c = tid; c < NPAD; c += CONV_THREADS) {
        uint4 v;
        v.x = pack_bf2(f[c], f[NPAD + c]);
        v.y = pack_bf2(f[2 * NPAD + c], f[3 * NPAD + c]);
        v.z = 0u;
        v.w = 0u;
        *reinterpret_cast<uint4*>(act + (size_t)c * 16) = v;
        *reinterpret_cast<uint4*>(act + HALF_BYTES + (size_t)c * 16) = make_uint4(0, 0, 0, 0);
      }
    } else {
      const uint4* src = reinterpret_cast<const uint4*>(a.in + (size_t)t * NCELL * NC);
      for (int c = tid; c < NPAD; c += CONV_THREADS) {
        const int px = c % PD, py = (c / PD) % PD, pz = c / (PD * PD);
        uint4 lo = make_uint4(0, 0, 0, 0), hi = lo;
        if (px >= 1 && px <= TS && py >= 1 && py <= TS && pz >= 1 && pz <= TS) {
          const int cell = (px - 1) + TS * ((py - 1) + TS * (pz - 1));
          lo = src[2 * cell];
          hi = src[2 * cell + 1];
        }
        *reinterpret_cast<uint4*>(act + (size_t)c * 16) = lo;
        *reinterpret_cast<uint4*>(act + HALF_BYTES + (size_t)c * 16) = hi;
      }
    }
    fence_proxy_async();
    tc_fence_before();
    __syncthreads();
    if (tid == 0) issue(0);
    for (int z = 0; z < TS; z++) {
      if (tid == 0 && z + 1 < TS) issue(z + 1);
      if (!__syncthreads_and(mbar_wait(&bar[z & 1], (uint32_t)((z >> 1) & 1)))) {
        ok = false;
        break;
      }
      tc_fence_after();
      float v[16];
      const int xh = warp >> 2, quarter = warp & 3;
      tmem_ld16(tbase + ((uint32_t)(32 * quarter) << 16) + (uint32_t)((z & 1) * 32 + 16 * xh), v);
      const int r = 32 * quarter + lane;
      const int x = 8 * xh + (r & 7), y = r >> 3;
      const int cell = x + TS * (y + TS * z);
      if (EPI == EPI_OUT0) {
        const float s = a.outScale ? a.outScale[t] : 1.f;
        const int64_t base = a.outOff ? a.outOff[t] : (int64_t)t * NCELL;
        a.out0[base + cell] = v[0] * s;
      } else {
        if (EPI == EPI_MASK) {
          const uint4* mp = reinterpret_cast<const uint4*>(a.mask + ((size_t)t * NCELL + cell) * NC);
          uint4 m2[2] = {mp[0], mp[1]};
          const __nv_bfloat16* mb = reinterpret_cast<const __nv_bfloat16*>(m2);
#pragma unroll
          for (int c = 0; c < 16; c++)
            if (!(__bfloat162float(mb[c]) > 0.f)) v[c] = 0.f;
        } else {
#pragma unroll
          for (int c = 0; c < 16; c++) v[c] = fmaxf(v[c], 0.f);
        }
        uint4 o0, o1;
        o0.x = pack_bf2(v[0], v[1]);
        o0.y = pack_bf2(v[2], v[3]);
        o0.z = pack_bf2(v[4], v[5]);
        o0.w = pack_bf2(v[6], v[7]);
        o1.x = pack_bf2(v[8], v[9]);
        o1.y = pack_bf2(v[10], v[11]);
        o1.z = pack_bf2(v[12], v[13]);
        o1.w = pack_bf2(v[14], v[15]);
        uint4* op = reinterpret_cast<uint4*>(a.out + ((size_t)t * NCELL + cell) * NC);
        op[0] = o0;
        op[1] = o1;
      }
      tc_fence_before();
      __syncthreads();
    }
  }
  if (!ok) {
    // a wait gave up: flag it, give the MMAs in flight one more bounded wait
    if (tid == 0) {
      atomicExch(a.err, 1);
      mbar_wait(&bar[0], 0);
      mbar_wait(&bar[1], 0);
    }
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
// of dz[o][co] * X[o + tap][ci], X the layer input on the padded box (bf16,
// as the forward pass reads it).  Thread (co, ci) = (tid >> 4, tid & 15).
constexpr int WG_SLAB = 4;  // output planes per shared-memory slab
constexpr size_t WG_SMEM = (size_t)(WG_SLAB + 2) * PD * PD * NC * 2 + (size_t)WG_SLAB * TS * TS * NC * 2;

template <int IN>
__global__ void __launch_bounds__(256) k_wgrad(int n, const float* __restrict__ feat,
                                               const __nv_bfloat16* __restrict__ in,
                                               const __nv_bfloat16* __restrict__ dz,
                                               float* __restrict__ partial) {
  extern __shared__ __align__(16) uint8_t smw[];
  __nv_bfloat16* X = reinterpret_cast<__nv_bfloat16*>(smw);  // [(WG_SLAB+2)*PD*PD][16]
  __nv_bfloat16* D =
      reinterpret_cast<__nv_bfloat16*>(smw + (size_t)(WG_SLAB + 2) * PD * PD * NC * 2);  // [WG_SLAB*256][16]
  const int tid = threadIdx.x, co = tid >> 4, ci = tid & 15;
  float acc[27];
#pragma unroll
  for (int k = 0; k < 27; k++) acc[k] = 0.f;
  for (int t = blockIdx.x; t < n; t += gridDim.x) {
    for (int z0 = 0; z0 < TS; z0 += WG_SLAB) {
      __syncthreads();
      // padded planes z0 .. z0+WG_SLAB+1
      for (int c = tid; c < (WG_SLAB + 2) * PD * PD; c += 256) {
        const int px = c % PD, py = (c / PD) % PD, pz = z0 + c / (PD * PD);
        uint4 lo = make_uint4(0, 0, 0, 0), hi = lo;
        if (IN == IN_FEAT) {
          const float* f = feat + (size_t)t * NFEAT * NPAD;
          const int pc = px + PD * (py + PD * pz);
          lo.x = pack_bf2(f[pc], f[NPAD + pc]);
          lo.y = pack_bf2(f[2 * NPAD + pc], f[3 * NPAD + pc]);
        } else if (px >= 1 && px <= TS && py >= 1 && py <= TS && pz >= 1 && pz <= TS) {
          const uint4* s = reinterpret_cast<const uint4*>(in + ((size_t)t * NCELL +
                                                               (px - 1) + TS * ((py - 1) + TS * (pz - 1))) * NC);
          lo = s[0];
          hi = s[1];
        }
        reinterpret_cast<uint4*>(X)[2 * c] = lo;
        reinterpret_cast<uint4*>(X)[2 * c + 1] = hi;
      }
      for (int c = tid; c < WG_SLAB * TS * TS; c += 256) {
        const uint4* s = reinterpret_cast<const uint4*>(dz + ((size_t)t * NCELL + (size_t)z0 * TS * TS + c) * NC);
        reinterpret_cast<uint4*>(D)[2 * c] = s[0];
        reinterpret_cast<uint4*>(D)[2 * c + 1] = s[1];
      }
      __syncthreads();
#pragma unroll 1
      for (int o = 0; o < WG_SLAB * TS * TS; o++) {
        const float d = __bfloat162float(D[o * NC + co]);
        if (d == 0.f) continue;
        const int ox = o % TS, oy = (o / TS) % TS, oz = o / (TS * TS);
        const int base = ox + PD * (oy + PD * oz);
#pragma unroll
        for (int k = 0; k < 27; k++) {
          const int kz = k / 9, ky = (k / 3) % 3, kx = k % 3;
          acc[k] = fmaf(d, __bfloat162float(X[(base + kx + PD * (ky + PD * kz)) * NC + ci]), acc[k]);
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
// a [n][NCELL][16] bf16 gradient (channels 1..15 stay 0).  Per-CTA partial.
constexpr int LOSS_GRID = 148 * 2;
__global__ void __launch_bounds__(512) k_loss(int64_t nc, const float* __restrict__ y,
                                              const float* __restrict__ tgt,
                                              const float* __restrict__ m, float invCount,
                                              __nv_bfloat16* __restrict__ dy,
                                              double* __restrict__ partial) {
  __shared__ double ws[16];
  double acc = 0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nc;
       i += (int64_t)gridDim.x * blockDim.x) {
    const float d = m[i] > 0.f ? y[i] - tgt[i] : 0.f;
    acc += (double)d * d;
    if (dy) dy[i * NC] = __float2bfloat16_rn(2.f * d * invCount);
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
  DeviceBuffer a1, a2, a3, y, dy, dz3, dz2, dz1, part, lossPart;
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
  cudaFuncSetAttribute(k_conv3_tc<IN_FEAT, EPI_RELU>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)CONV_SMEM);
  cudaFuncSetAttribute(k_conv3_tc<IN_ACT, EPI_RELU>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)CONV_SMEM);
  cudaFuncSetAttribute(k_conv3_tc<IN_ACT, EPI_MASK>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)CONV_SMEM);
  cudaFuncSetAttribute(k_conv3_tc<IN_ACT, EPI_OUT0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)CONV_SMEM);
  cudaFuncSetAttribute(k_wgrad<IN_FEAT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)WG_SMEM);
  cudaFuncSetAttribute(k_wgrad<IN_ACT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)WG_SMEM);
  done = true;
}

template <int IN, int EPI>
void conv(msbg_cnn* net, int layer, bool backward, int n, const float* feat,
          const __nv_bfloat16* in, __nv_bfloat16* out, const __nv_bfloat16* mask, float* out0,
          const int64_t* outOff, const float* outScale, cudaStream_t st) {
  ConvArgs a;
  a.n = n;
  a.feat = feat;
  a.in = in;
  a.wimg = (backward ? net->imgB : net->imgF).as<__nv_bfloat16>() + (size_t)layer * WIMG;
  a.out = out;
  a.mask = mask;
  a.out0 = out0;
  a.outOff = outOff;
  a.outScale = outScale;
  a.err = net->err.as<int>();
  const int grid = std::min(n, net->numSMs);
  k_conv3_tc<IN, EPI><<<grid, CONV_THREADS, CONV_SMEM, st>>>(a);
}

int ensure_cap(msbg_cnn* net, int n) {
  if (n <= net->cap) return MSBG_OK;
  const size_t act = (size_t)n * NCELL * NC * sizeof(__nv_bfloat16);
  CNN_TRY(net, net->a1.ensure(act));
  CNN_TRY(net, net->a2.ensure(act));
  CNN_TRY(net, net->a3.ensure(act));
  CNN_TRY(net, net->dz3.ensure(act));
  CNN_TRY(net, net->dz2.ensure(act));
  CNN_TRY(net, net->dz1.ensure(act));
  CNN_TRY(net, net->dy.ensure(act));
  CNN_TRY(net, cudaMemsetAsync(net->dy.p, 0, act, net->stream));
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
            const float* outScale, int n, cudaStream_t st, __nv_bfloat16* s1, __nv_bfloat16* s2) {
  if (n <= 0) return MSBG_OK;
  conv<IN_FEAT, EPI_RELU>(net, 0, false, n, feat, nullptr, s1, nullptr, nullptr, nullptr, nullptr, st);
  conv<IN_ACT, EPI_RELU>(net, 1, false, n, nullptr, s1, s2, nullptr, nullptr, nullptr, nullptr, st);
  conv<IN_ACT, EPI_RELU>(net, 2, false, n, nullptr, s2, s1, nullptr, nullptr, nullptr, nullptr, st);
  conv<IN_ACT, EPI_OUT0>(net, 3, false, n, nullptr, s1, nullptr, nullptr, out0, outOff, outScale, st);
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
  rc = forward(net, feat, out, nullptr, nullptr, n, net->stream, net->a1.as<__nv_bfloat16>(),
               net->a2.as<__nv_bfloat16>());
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
  auto* a1 = net->a1.as<__nv_bfloat16>();
  auto* a2 = net->a2.as<__nv_bfloat16>();
  auto* a3 = net->a3.as<__nv_bfloat16>();
  auto* dy = net->dy.as<__nv_bfloat16>();
  auto* dz3 = net->dz3.as<__nv_bfloat16>();
  auto* dz2 = net->dz2.as<__nv_bfloat16>();
  auto* dz1 = net->dz1.as<__nv_bfloat16>();
  float* y = net->y.as<float>();
  // forward, keeping the activations
  conv<IN_FEAT, EPI_RELU>(net, 0, false, n, feat, nullptr, a1, nullptr, nullptr, nullptr, nullptr, st);
  conv<IN_ACT, EPI_RELU>(net, 1, false, n, nullptr, a1, a2, nullptr, nullptr, nullptr, nullptr, st);
  conv<IN_ACT, EPI_RELU>(net, 2, false, n, nullptr, a2, a3, nullptr, nullptr, nullptr, nullptr, st);
  conv<IN_ACT, EPI_OUT0>(net, 3, false, n, nullptr, a3, nullptr, nullptr, y, nullptr, nullptr, st);
  // loss and dL/dy
  k_loss<<<LOSS_GRID, 512, 0, st>>>((int64_t)n * NCELL, y, target, mask, (float)(1.0 / count), dy,
                                    net->lossPart.as<double>());
  // backward-data through layers 4, 3, 2 (ReLU masks of their inputs)
  conv<IN_ACT, EPI_MASK>(net, 3, true, n, nullptr, dy, dz3, a3, nullptr, nullptr, nullptr, st);
  conv<IN_ACT, EPI_MASK>(net, 2, true, n, nullptr, dz3, dz2, a2, nullptr, nullptr, nullptr, st);
  conv<IN_ACT, EPI_MASK>(net, 1, true, n, nullptr, dz2, dz1, a1, nullptr, nullptr, nullptr, st);
  // weight gradients
  const int grid = std::min(n, net->numSMs);
  float* part = net->part.as<float>();
  float* g = net->g.as<float>();
  const __nv_bfloat16* dzs[NLAYER] = {dz1, dz2, dz3, dy};
  const __nv_bfloat16* ins[NLAYER] = {nullptr, a1, a2, a3};
  for (int l = 0; l < NLAYER; l++) {
    if (l == 0)
      k_wgrad<IN_FEAT><<<grid, 256, WG_SMEM, st>>>(n, feat, nullptr, dzs[l], part);
    else
      k_wgrad<IN_ACT><<<grid, 256, WG_SMEM, st>>>(n, nullptr, ins[l], dzs[l], part);
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
