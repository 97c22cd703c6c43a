// Inputs of the learned network gathered from MG level 0 of the pressure
// solver (included inside namespace msbg::ps of pressure.cu).
//
// Sample s = 16^3 tile tiles[s] of level 0 with a 1-cell halo:
//   channel 0  value / vmax      (value = right-hand side or residual; vmax =
//                                 max |value| over the tile's cells)
//   channel 1  solid mask
//   channel 2  air mask (Dirichlet p = 0 cells)
//   channel 3  resolution level / max(1, levels - 1)
// Halo cells across a face with a same-level neighbour tile take the
// neighbour's boundary values and types; other halo cells are 0.
// outScale[s] = vmax / mean(a_ii over the tile's liquid cells) turns the
// network output into pressure; outOff[s] = first cell of the tile.
// With `solution`, also the training target solution * mean(a_ii) / vmax and
// the liquid mask of the tile's cells.

constexpr int FEAT_THREADS = 256;

static __global__ void __launch_bounds__(FEAT_THREADS) k_cnn_features(
    LevelView L, const uint8_t* __restrict__ ctype, const int* __restrict__ tiles,
    const int* __restrict__ tileLevel, float levelNorm, const float* __restrict__ val,
    const double* __restrict__ solution, float* __restrict__ feat, float* __restrict__ outScale,
    int64_t* __restrict__ outOff, float* __restrict__ target, float* __restrict__ mask) {
  constexpr int TSZ = cnn::TS, PDZ = cnn::PD, NP = cnn::NPAD, NCL = cnn::NCELL;
  __shared__ float smax[FEAT_THREADS / 32];
  __shared__ double sdiag[FEAT_THREADS / 32];
  __shared__ int sliq[FEAT_THREADS / 32];
  const int s = blockIdx.x, tid = threadIdx.x;
  const int ti = tiles[s];
  const int64_t off = L.tileOff[ti];
  float m = 0.f;
  double dsum = 0;
  int nl = 0;
  for (int c = tid; c < NCL; c += FEAT_THREADS) {
    m = fmaxf(m, fabsf(val[off + c]));
    const float dg = L.diag[off + c];
    if (dg > 0.f) {
      dsum += dg;
      nl++;
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    m = fmaxf(m, __shfl_down_sync(0xffffffffu, m, o));
    dsum += __shfl_down_sync(0xffffffffu, dsum, o);
    nl += __shfl_down_sync(0xffffffffu, nl, o);
  }
  if ((tid & 31) == 0) {
    smax[tid >> 5] = m;
    sdiag[tid >> 5] = dsum;
    sliq[tid >> 5] = nl;
  }
  __syncthreads();
  float vmax = 0.f;
  double dtot = 0;
  int ltot = 0;
  for (int w = 0; w < FEAT_THREADS / 32; w++) {
    vmax = fmaxf(vmax, smax[w]);
    dtot += sdiag[w];
    ltot += sliq[w];
  }
  const float dbar = ltot > 0 ? (float)(dtot / ltot) : 1.f;
  const float inv = vmax > 0.f ? 1.f / vmax : 0.f;
  if (tid == 0) {
    outScale[s] = vmax / dbar;
    outOff[s] = off;
  }
  const float lv = (float)tileLevel[s] * levelNorm;
  float* F = feat + (size_t)s * cnn::NFEAT * NP;
  for (int p = tid; p < NP; p += FEAT_THREADS) {
    const int px = p % PDZ, py = (p / PDZ) % PDZ, pz = p / (PDZ * PDZ);
    const int q[3] = {px - 1, py - 1, pz - 1};
    int outAxis = -1, nOut = 0;
#pragma unroll
    for (int a = 0; a < 3; a++)
      if (q[a] < 0 || q[a] >= TSZ) {
        outAxis = a;
        nOut++;
      }
    float v = 0.f, solid = 0.f, air = 0.f;
    if (nOut == 0) {
      const int64_t c = off + q[0] + TSZ * (q[1] + TSZ * q[2]);
      v = val[c] * inv;
      solid = ctype[c] == CT_SOLID ? 1.f : 0.f;
      air = ctype[c] == CT_AIR ? 1.f : 0.f;
    } else if (nOut == 1) {
      const int side = q[outAxis] >= TSZ ? 1 : 0;
      const int* Fc = L.face + ((size_t)ti * 6 + outAxis * 2 + side) * FACE_INTS;
      if (Fc[F_KIND] == FACE_SAME) {
        int r[3] = {q[0], q[1], q[2]};
        r[outAxis] = side ? 0 : TSZ - 1;
        const int64_t c = L.tileOff[Fc[F_T0]] + r[0] + TSZ * (r[1] + TSZ * r[2]);
        v = val[c] * inv;
        solid = ctype[c] == CT_SOLID ? 1.f : 0.f;
        air = ctype[c] == CT_AIR ? 1.f : 0.f;
      }
    }
    F[p] = v;
    F[NP + p] = solid;
    F[2 * NP + p] = air;
    F[3 * NP + p] = lv;
  }
  if (solution) {
    const float g = vmax > 0.f ? dbar / vmax : 0.f;
    for (int c = tid; c < NCL; c += FEAT_THREADS) {
      const bool liq = L.diag[off + c] > 0.f;
      target[(size_t)s * NCL + c] = liq ? (float)(solution[off + c] * g) : 0.f;
      mask[(size_t)s * NCL + c] = liq ? 1.f : 0.f;
    }
  }
}

// x64[i] = guess[i] on liquid cells, 0 elsewhere.
static __global__ void __launch_bounds__(512) k_set64_masked(double* __restrict__ x,
                                                      const float* __restrict__ g,
                                                      const float* __restrict__ diag, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    x[i] = diag[i] > 0.f ? (double)g[i] : 0.0;
}
