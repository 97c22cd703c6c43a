// FP64 outer iterative refinement of the pressure solve (included inside
// namespace msbg::ps of pressure.cu after the reduction helpers).
//
// The solution is accumulated in FP64; each outer step recomputes
// r = b - A x in FP64 (FP32 operator entries widened exactly, FP64 sums),
// hands r to the inner MGPCG as its right-hand side and adds the inner
// correction to x in FP64.  This is what lets the true residual reach 1e-6
// where an FP32 iterate cannot represent it.

// r32 = b - A x64 on MG level 0 (one CTA per tile; thread (i,j,h) owns the
// h-th part of the z column (i,j): 16^3 tiles in two halves, so a CTA has
// 512 threads and more loads in flight), per-CTA partial |r|^2 in FP64.
template <int TS>
__host__ __device__ constexpr int res64_split() { return TS == 16 ? 2 : 1; }
template <int TS>
__global__ void __launch_bounds__(TS* TS* res64_split<TS>())
    k_residual64(LevelView L, const int* __restrict__ tiles, const double* __restrict__ x,
                 const float* __restrict__ b, float* __restrict__ r,
                 double* __restrict__ partial) {
  constexpr int N = TS * TS * TS, NF = TS * TS, SPLIT = res64_split<TS>(), NT = NF * SPLIT;
  constexpr int ZC = TS / SPLIT;  // cells of a thread's z column part
  __shared__ double xs[N];
  __shared__ double gs[6][NF];
  const int ti = tiles[blockIdx.x];
  const int64_t off = L.tileOff[ti];
  const int t = threadIdx.x, i = t % TS, j = (t / TS) % TS, h = t / NF;
  for (int e = t; e < N; e += NT) xs[e] = x[off + e];
  for (int q = t; q < 6 * NF; q += NT) {
    const int f = q / NF, c = q % NF;
    gs[f][c] = ghost_sum<double, double>(L, x, ti, TS, f >> 1, f & 1, c % TS, c / TS);
  }
  __syncthreads();
  const float* cx = L.cx + off;
  const float* cy = L.cy + off;
  const float* cz = L.cz + off;
  double acc = 0;
  for (int k = h * ZC; k < (h + 1) * ZC; k++) {
    const int e = tidx(TS, i, j, k);
    const double dg = L.diag[off + e];
    double rv = 0;
    if (dg > 0) {
      double S = 0;
      S += (i > 0) ? (double)cx[e] * xs[e - 1] : gs[0][j + TS * k];
      S += (i < TS - 1) ? (double)cx[e + 1] * xs[e + 1] : gs[1][j + TS * k];
      S += (j > 0) ? (double)cy[e] * xs[e - TS] : gs[2][i + TS * k];
      S += (j < TS - 1) ? (double)cy[e + TS] * xs[e + TS] : gs[3][i + TS * k];
      S += (k > 0) ? (double)cz[e] * xs[e - TS * TS] : gs[4][i + TS * j];
      S += (k < TS - 1) ? (double)cz[e + TS * TS] * xs[e + TS * TS] : gs[5][i + TS * j];
      rv = (double)b[off + e] - (dg * xs[e] - S);
    }
    r[off + e] = (float)rv;
    acc += rv * rv;
  }
  acc = block_sum(acc);
  if (t == 0) partial[blockIdx.x] = acc;
}

// x64 += e * unscale (all cells; e is 0 off the liquid)
template <typename VT>
__global__ void __launch_bounds__(512) k_add64(double* __restrict__ x, const VT* __restrict__ e,
                                               int64_t n, double unscale) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    x[i] += (double)to_f(e[i]) * unscale;
}

// x32 = (float) x64
static __global__ void __launch_bounds__(512) k_narrow(float* __restrict__ y, const double* __restrict__ x,
                                                int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    y[i] = (float)x[i];
}

// Per-CTA partial max |v| (grid-stride over groups of 4).
template <typename VT>
__global__ void __launch_bounds__(VEC_BLOCK) k_absmax(const VT* __restrict__ v, int64_t n,
                                                      double* __restrict__ partial) {
  __shared__ float ws[32];
  float m = 0.f;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < (n >> 2);
       i += (int64_t)gridDim.x * blockDim.x) {
    const F4 u = load4(v + 4 * i);
    m = fmaxf(m, fmaxf(fmaxf(fabsf(u.x), fabsf(u.y)), fmaxf(fabsf(u.z), fabsf(u.w))));
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_down_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); w++) m = fmaxf(m, ws[w]);
    partial[blockIdx.x] = m;
  }
}

// Max of the partials into s->amax.
static __global__ void __launch_bounds__(32) k_finalize_max(const double* __restrict__ partial, int n,
                                                     Scalars* s) {
  if (threadIdx.x != 0) return;
  double m = 0;
  for (int i = 0; i < n; i++) m = (partial[i] != partial[i] || m != m) ? NAN : fmax(m, partial[i]);
  s->amax = m;
}

// x64 += alpha d (FP64 accumulation of the FP32 direction); r -= alpha q;
// partial |r|^2.  Skipped (norm only) after a breakdown.
static __global__ void __launch_bounds__(VEC_BLOCK) k_axpy64_norm(double* __restrict__ x,
                                                           float* __restrict__ r,
                                                           const float* __restrict__ d,
                                                           const float* __restrict__ q, int64_t n,
                                                           const Scalars* __restrict__ s,
                                                           double* __restrict__ partial) {
  const bool ok = s->status == 0;
  const double alpha = s->alpha;
  const float af = (float)alpha;
  double acc = 0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < (n >> 2);
       i += (int64_t)gridDim.x * blockDim.x) {
    float4 rv = reinterpret_cast<const float4*>(r)[i];
    if (ok) {
      const float4 dv = reinterpret_cast<const float4*>(d)[i];
      const float4 qv = reinterpret_cast<const float4*>(q)[i];
      double2* xp = reinterpret_cast<double2*>(x) + 2 * i;
      double2 x0 = xp[0], x1 = xp[1];
      x0.x += alpha * dv.x; x0.y += alpha * dv.y; x1.x += alpha * dv.z; x1.y += alpha * dv.w;
      xp[0] = x0;
      xp[1] = x1;
      rv.x = fmaf(-af, qv.x, rv.x); rv.y = fmaf(-af, qv.y, rv.y);
      rv.z = fmaf(-af, qv.z, rv.z); rv.w = fmaf(-af, qv.w, rv.w);
      reinterpret_cast<float4*>(r)[i] = rv;
    }
    acc += (double)rv.x * rv.x + (double)rv.y * rv.y + (double)rv.z * rv.z + (double)rv.w * rv.w;
  }
  acc = block_sum(acc);
  if (threadIdx.x == 0) partial[blockIdx.x] = acc;
}

// y = a - b (all cells)
static __global__ void __launch_bounds__(VEC_BLOCK) k_sub(float* __restrict__ y, const float* __restrict__ a,
                                                   const float* __restrict__ b, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < (n >> 2);
       i += (int64_t)gridDim.x * blockDim.x) {
    const float4 u = reinterpret_cast<const float4*>(a)[i], v = reinterpret_cast<const float4*>(b)[i];
    reinterpret_cast<float4*>(y)[i] = make_float4(u.x - v.x, u.y - v.y, u.z - v.z, u.w - v.w);
  }
}

// v = 0 outside the liquid cells
static __global__ void __launch_bounds__(VEC_BLOCK) k_mask(float* __restrict__ v,
                                                    const float* __restrict__ diag, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    if (!(diag[i] > 0.f)) v[i] = 0.f;
}

// z += omega c
static __global__ void __launch_bounds__(VEC_BLOCK) k_add_omega(float* __restrict__ z,
                                                         const float* __restrict__ c,
                                                         const Scalars* __restrict__ s, int64_t n) {
  const float w = (float)s->omega;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    z[i] = fmaf(w, c[i], z[i]);
}

// x *= omega (FP64)
static __global__ void __launch_bounds__(VEC_BLOCK) k_scale64(double* __restrict__ x,
                                                       const Scalars* __restrict__ s, int64_t n) {
  const double w = s->omega;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    x[i] *= w;
}

// e = a - b (FP64)
static __global__ void __launch_bounds__(VEC_BLOCK) k_sub64(double* __restrict__ e,
                                                     const double* __restrict__ a,
                                                     const double* __restrict__ b, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    e[i] = a[i] - b[i];
}
