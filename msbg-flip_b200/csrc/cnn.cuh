// The learned 3D CNN of the pressure solver: shapes, weight layout and the
// device kernels (forward / backward-data convolution on the tensor cores,
// weight gradients, loss, Adam).  No counterpart in the reference.
//
// Network (per 16^3 tile with a 1-cell halo, 18^3 inputs):
//   conv1 4->16, 3^3, valid on the 18^3 box (-> 16^3), ReLU
//   conv2 16->16, 3^3, zero padding, ReLU
//   conv3 16->16, 3^3, zero padding, ReLU
//   conv4 16->1,  3^3, zero padding
// No biases: the network is positively homogeneous in its value channel
// scale, which the per-tile normalisation relies on.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "msbg_cnn.h"

namespace msbg {
namespace cnn {

constexpr int TS = 16;                  // tile edge
constexpr int PD = 18;                  // padded edge
constexpr int NPAD = PD * PD * PD;      // 5832 padded cells
constexpr int NCELL = TS * TS * TS;     // 4096 cells
constexpr int NC = 16;                  // channels of the hidden layers
constexpr int NFEAT = 4;                // input channels
constexpr int NLAYER = 4;
constexpr uint32_t HALF_BYTES = NPAD * 16;  // one channel half (8 x bf16) of the padded box
constexpr int WIMG = 27 * 256;              // bf16 elements of one layer's weight image

// Master weights, FP32, PyTorch Conv3d order per layer: [cout][cin][kz][ky][kx].
__host__ __device__ constexpr int layer_cin(int l) { return l == 0 ? NFEAT : NC; }
__host__ __device__ constexpr int layer_cout(int l) { return l == NLAYER - 1 ? 1 : NC; }
__host__ __device__ constexpr int layer_off(int l) {
  return l == 0 ? 0 : l == 1 ? 27 * NFEAT * NC : l == 2 ? 27 * NFEAT * NC + 27 * NC * NC
                                                        : 27 * NFEAT * NC + 2 * 27 * NC * NC;
}
constexpr int NPARAM = 27 * NFEAT * NC + 2 * 27 * NC * NC + 27 * NC;  // 15984

// Activation tensors in global memory use the shared-memory layout of the
// convolution: per tile two channel halves, each NPAD padded cells x 16 bytes
// (8 bf16 channels), z slowest; halo cells are zero except in the first
// layer's input.  One padded z plane of one half is PLANE_BYTES contiguous.
constexpr int PLANE = PD * PD;
constexpr uint32_t PLANE_BYTES = PLANE * 16;        // 5184
constexpr size_t ACT_BYTES = 2 * (size_t)HALF_BYTES;  // per tile
__host__ __device__ constexpr int pad_index(int cell) {
  return (cell % TS + 1) + PD * ((cell / TS) % TS + 1 + PD * (cell / (TS * TS) + 1));
}

enum { EPI_RELU = 0, EPI_MASK = 1, EPI_OUT0 = 2 };

struct ConvArgs {
  int n;                              // tiles
  const uint4* in;                    // [n][2][NPAD] 16-byte cells (padded layout)
  const __nv_bfloat16* wimg;          // [27][2][16][8] bf16 image of the layer
  uint4* out;                         // EPI_RELU / EPI_MASK: padded layout, interior written
  const uint4* mask;                  // EPI_MASK: padded layout; out = acc where mask > 0
  float* out0;                        // EPI_OUT0: channel 0
  const int64_t* outOff;              // EPI_OUT0: per-tile first cell in out0 (null: t*NCELL)
  const float* outScale;              // EPI_OUT0: per-tile factor (null: 1)
  int* err;                           // set when a bounded wait gives up
};

// 8 warps: warp w drains TMEM lanes 32*(w%4) of column half w/4.
constexpr int CONV_THREADS = 256;
constexpr size_t CONV_SMEM = 2 * (size_t)HALF_BYTES + WIMG * 2 + 256;

// Inference of n tiles on stream st: out0[outOff[t] + cell] = outScale[t] *
// net(feat[t]) (cnn.cu).  x0, s1, s2: scratch of n * ACT_BYTES each; s1 and
// s2 must have zero halos (zeroed once when allocated).
int forward(msbg_cnn* net, const float* feat, float* out0, const int64_t* outOff,
            const float* outScale, int n, cudaStream_t st, uint4* x0, uint4* s1, uint4* s2);
// Status of the network's bounded waits since the last call (0 = none gave up); clears it.
int take_error(msbg_cnn* net, cudaStream_t st);

}  // namespace cnn
}  // namespace msbg
