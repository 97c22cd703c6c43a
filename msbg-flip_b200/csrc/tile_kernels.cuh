// Reductions, PCG vector kernels and per-tile kernels of the pressure solver
// (included inside namespace msbg::ps of pressure.cu).  Vectors are stored
// as VT (float, __half or __nv_bfloat16) and computed in FP32; inner products
// accumulate in FP64.

// ---------------------------------------------------------------------------
// reductions
// ---------------------------------------------------------------------------
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

// Sum over the CTA; result valid in thread 0.
__device__ __forceinline__ double block_sum(double v) {
  __shared__ double ws[32];
  v = warp_sum(v);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) ws[w] = v;
  __syncthreads();
  const int nw = (blockDim.x + 31) >> 5;
  v = (threadIdx.x < nw) ? ws[threadIdx.x] : 0.0;
  if (w == 0) v = warp_sum(v);
  __syncthreads();
  return v;
}

struct Scalars {
  double bb, rho, rhoNew, dq, rr, alpha, beta, amax;
  double cc, cr, omega;  // energy-optimal scaling of a learned vector c
  int status;  // 0 ok, 2 breakdown, 3 non-finite
  int pad;
};

enum {
  FIN_BB = 0,
  FIN_DQ_ALPHA = 1,
  FIN_RR = 2,
  FIN_RHO = 3,
  FIN_RHONEW_BETA = 4,
  FIN_FCG_BETA = 5,      // flexible CG: beta = -(z.q)/(d.q)
  FIN_FCG_DQ_ALPHA = 6,  // flexible CG: alpha = (d.r)/(d.q), d.r of either sign
  FIN_CC = 7,            // c.Ac
  FIN_CR = 8,            // c.r
  FIN_OMEGA_CORR = 9,    // omega = (c.r)/(c.Ac): v = c.r
  FIN_OMEGA_GUESS = 10,  // omega = (g.b)/(g.b - g.r), r = b - A g: v = g.r
};

// Deterministic second stage: fixed-order sum of the CTA partials, then the
// scalar step of PCG that depends on it.
static __global__ void __launch_bounds__(1024) k_finalize(const double* __restrict__ partial, int n,
                                                   Scalars* s, int what) {
  double v = 0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) v += partial[i];
  v = block_sum(v);
  if (threadIdx.x != 0) return;
  switch (what) {
    case FIN_BB: s->bb = v; break;
    case FIN_RHO: s->rho = v; break;
    case FIN_RR:
      s->rr = v;
      if (!isfinite(v)) s->status = 3;
      break;
    case FIN_DQ_ALPHA:
      s->dq = v;
      if (!isfinite(v) || !isfinite(s->rho)) s->status = 3;
      else if (!(v > 1e-300) || !(s->rho > 1e-300)) s->status = 2;
      else s->alpha = s->rho / v;
      break;
    case FIN_RHONEW_BETA:
      s->rhoNew = v;
      if (!isfinite(v)) s->status = 3;
      else if (!(v > 1e-300)) s->status = 2;
      else {
        s->beta = v / s->rho;
        s->rho = v;
      }
      break;
    case FIN_FCG_BETA:  // q = A d of the last step
      if (!isfinite(v)) s->status = 3;
      else s->beta = -v / s->dq;
      break;
    case FIN_CC: s->cc = v; break;
    case FIN_CR: s->cr = v; break;
    // The scaled vector omega*c minimises |e - omega c|_A for A e = r: it
    // never leaves a larger energy error than c = 0 does.  A degenerate c
    // gets omega = 0.
    case FIN_OMEGA_CORR:
      s->omega = (isfinite(v) && isfinite(s->cc) && s->cc > 1e-300) ? v / s->cc : 0.0;
      break;
    case FIN_OMEGA_GUESS: {
      const double gag = s->cr - v;  // g.Ag = g.b - g.(b - Ag)
      s->omega = (isfinite(v) && isfinite(s->cr) && gag > 1e-300) ? s->cr / gag : 0.0;
      break;
    }
    case FIN_FCG_DQ_ALPHA:
      // a non-linear preconditioner need not make d.r positive; the step
      // along d still minimises the energy norm as long as d.q > 0
      s->dq = v;
      if (!isfinite(v) || !isfinite(s->rho)) s->status = 3;
      else if (!(v > 1e-300)) s->status = 2;
      else s->alpha = s->rho / v;
      break;
  }
}

// ---------------------------------------------------------------------------
// level-0 vector kernels (grid-stride over groups of 4, fixed grid so the
// partial sums are deterministic)
// ---------------------------------------------------------------------------
constexpr int VEC_GRID = 148 * 4, VEC_BLOCK = 512;

template <typename VA, typename VB>
__global__ void __launch_bounds__(VEC_BLOCK) k_dot(const VA* __restrict__ a,
                                                   const VB* __restrict__ b, int64_t n,
                                                   double* __restrict__ partial) {
  double acc = 0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < (n >> 2);
       i += (int64_t)gridDim.x * blockDim.x) {
    const F4 u = load4(a + 4 * i), v = load4(b + 4 * i);
    acc += (double)u.x * v.x + (double)u.y * v.y + (double)u.z * v.z + (double)u.w * v.w;
  }
  acc = block_sum(acc);
  if (threadIdx.x == 0) partial[blockIdx.x] = acc;
}

// x += alpha d; r -= alpha q; partial |r|^2.  Skipped (norm only) after a breakdown.
template <typename VT>
__global__ void __launch_bounds__(VEC_BLOCK) k_axpy_norm(VT* __restrict__ x, VT* __restrict__ r,
                                                         const VT* __restrict__ d,
                                                         const VT* __restrict__ q, int64_t n,
                                                         const Scalars* __restrict__ s,
                                                         double* __restrict__ partial) {
  const bool ok = s->status == 0;
  const float alpha = (float)s->alpha;
  double acc = 0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < (n >> 2);
       i += (int64_t)gridDim.x * blockDim.x) {
    F4 rv = load4(r + 4 * i);
    if (ok) {
      F4 xv = load4(x + 4 * i);
      const F4 dv = load4(d + 4 * i), qv = load4(q + 4 * i);
      xv.x = fmaf(alpha, dv.x, xv.x); xv.y = fmaf(alpha, dv.y, xv.y);
      xv.z = fmaf(alpha, dv.z, xv.z); xv.w = fmaf(alpha, dv.w, xv.w);
      rv.x = fmaf(-alpha, qv.x, rv.x); rv.y = fmaf(-alpha, qv.y, rv.y);
      rv.z = fmaf(-alpha, qv.z, rv.z); rv.w = fmaf(-alpha, qv.w, rv.w);
      store4(x + 4 * i, xv);
      store4(r + 4 * i, rv);
      rv = load4(r + 4 * i);  // the norm of what is stored
    }
    acc += (double)rv.x * rv.x + (double)rv.y * rv.y + (double)rv.z * rv.z + (double)rv.w * rv.w;
  }
  acc = block_sum(acc);
  if (threadIdx.x == 0) partial[blockIdx.x] = acc;
}

// d = z + beta d
template <typename VT>
__global__ void __launch_bounds__(VEC_BLOCK) k_update_d(VT* __restrict__ d,
                                                        const VT* __restrict__ z, int64_t n,
                                                        const Scalars* __restrict__ s) {
  if (s->status) return;
  const float beta = (float)s->beta;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < (n >> 2);
       i += (int64_t)gridDim.x * blockDim.x) {
    F4 dv = load4(d + 4 * i);
    const F4 zv = load4(z + 4 * i);
    dv.x = fmaf(beta, dv.x, zv.x); dv.y = fmaf(beta, dv.y, zv.y);
    dv.z = fmaf(beta, dv.z, zv.z); dv.w = fmaf(beta, dv.w, zv.w);
    store4(d + 4 * i, dv);
  }
}

// y = scale * x (type conversion)
template <typename VS, typename VD>
__global__ void __launch_bounds__(VEC_BLOCK) k_convert(VD* __restrict__ y, const VS* __restrict__ x,
                                                       int64_t n, float scale) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < (n >> 2);
       i += (int64_t)gridDim.x * blockDim.x) {
    F4 v = load4(x + 4 * i);
    v.x *= scale; v.y *= scale; v.z *= scale; v.w *= scale;
    store4(y + 4 * i, v);
  }
}

// ---------------------------------------------------------------------------
// per-tile kernels (any tile size TS <= 16; one CTA per tile, thread (i,j)
// owns the z column)
// ---------------------------------------------------------------------------

// In-tile neighbour sum S of cell (i,j,k) from a shared-memory tile, ghosts
// from gs.  cxv etc. point at the tile's couplings (shared or global).
template <int TS>
__device__ __forceinline__ float nbr_sum(const float* xs, const float* cxv, const float* cyv,
                                         const float* czv, const float (*gs)[TS * TS], int i,
                                         int j, int k) {
  const int e = tidx(TS, i, j, k);
  float S = 0.f;
  S += (i > 0) ? cxv[e] * xs[e - 1] : gs[0][j + TS * k];
  S += (i < TS - 1) ? cxv[e + 1] * xs[e + 1] : gs[1][j + TS * k];
  S += (j > 0) ? cyv[e] * xs[e - TS] : gs[2][i + TS * k];
  S += (j < TS - 1) ? cyv[e + TS] * xs[e + TS] : gs[3][i + TS * k];
  S += (k > 0) ? czv[e] * xs[e - TS * TS] : gs[4][i + TS * j];
  S += (k < TS - 1) ? czv[e + TS * TS] * xs[e + TS * TS] : gs[5][i + TS * j];
  return S;
}

// q = A d on the listed tiles, partial d.q per CTA.
template <int TS, typename VT>
__global__ void __launch_bounds__(TS* TS) k_matvec_dot(LevelView L, const int* __restrict__ tiles,
                                                       const VT* __restrict__ d,
                                                       VT* __restrict__ q,
                                                       double* __restrict__ partial) {
  constexpr int N = TS * TS * TS, NT = TS * TS;
  __shared__ float xs[N];
  __shared__ float gs[6][NT];
  const int ti = tiles[blockIdx.x];
  const int64_t off = L.tileOff[ti];
  const int t = threadIdx.x, i = t % TS, j = t / TS;
  for (int e = t; e < N; e += NT) xs[e] = to_f(d[off + e]);
#pragma unroll
  for (int f = 0; f < 6; f++) gs[f][t] = ghost_sum(L, d, ti, TS, f >> 1, f & 1, i, j);
  __syncthreads();
  double acc = 0;
  const float* cxv = L.cx + off;
  const float* cyv = L.cy + off;
  const float* czv = L.cz + off;
#pragma unroll 4
  for (int k = 0; k < TS; k++) {
    const int e = tidx(TS, i, j, k);
    const float dg = L.diag[off + e];
    float y = 0.f;
    if (dg > 0.f) y = dg * xs[e] - nbr_sum<TS>(xs, cxv, cyv, czv, gs, i, j, k);
    q[off + e] = from_f<VT>(y);
    acc += (double)xs[e] * (double)to_f(from_f<VT>(y));
  }
  acc = block_sum(acc);
  if (t == 0 && partial) partial[blockIdx.x] = acc;
}

// r = b - A x on the listed tiles, restricted (sum over the liquid children,
// P^T) into the coarse right-hand side bc (vectors VT, coarse vectors VC).
template <int TS, typename VT, typename VC>
__global__ void __launch_bounds__(TS* TS) k_residual_restrict(LevelView L,
                                                              const int* __restrict__ tiles,
                                                              const VT* __restrict__ x,
                                                              const VT* __restrict__ b,
                                                              VC* __restrict__ bc,
                                                              const int64_t* __restrict__ coarseOff) {
  constexpr int N = TS * TS * TS, NT = TS * TS;
  __shared__ float xs[N];
  __shared__ float rs[N];
  __shared__ float gs[6][NT];
  const int ti = tiles[blockIdx.x];
  const int64_t off = L.tileOff[ti];
  const int t = threadIdx.x, i = t % TS, j = t / TS;
  for (int e = t; e < N; e += NT) xs[e] = to_f(x[off + e]);
#pragma unroll
  for (int f = 0; f < 6; f++) gs[f][t] = ghost_sum(L, x, ti, TS, f >> 1, f & 1, i, j);
  __syncthreads();
  const float* cxv = L.cx + off;
  const float* cyv = L.cy + off;
  const float* czv = L.cz + off;
#pragma unroll 4
  for (int k = 0; k < TS; k++) {
    const int e = tidx(TS, i, j, k);
    const float dg = L.diag[off + e];
    float r = 0.f;
    if (dg > 0.f)
      r = to_f(b[off + e]) - (dg * xs[e] - nbr_sum<TS>(xs, cxv, cyv, czv, gs, i, j, k));
    rs[e] = r;
  }
  __syncthreads();
  const int* tc = L.toCoarse + (size_t)ti * 6;
  const int ct = tc[0], ox = tc[1], oy = tc[2], oz = tc[3], agg = tc[4], cts = tc[5];
  if (ct < 0) return;
  VC* dst = bc + coarseOff[ct];
  if (agg) {
    constexpr int H = TS / 2;
    for (int c = t; c < H * H * H; c += NT) {
      const int ci = c % H, cj = (c / H) % H, ck = c / (H * H);
      const int e = tidx(TS, 2 * ci, 2 * cj, 2 * ck);
      const float s = rs[e] + rs[e + 1] + rs[e + TS] + rs[e + TS + 1] + rs[e + TS * TS] +
                      rs[e + TS * TS + 1] + rs[e + TS * TS + TS] + rs[e + TS * TS + TS + 1];
      dst[tidx(cts, ox + ci, oy + cj, oz + ck)] = from_f<VC>(s);
    }
  } else {
    for (int e = t; e < N; e += NT) {
      const int ii = e % TS, jj = (e / TS) % TS, kk = e / (TS * TS);
      dst[tidx(cts, ox + ii, oy + jj, oz + kk)] = from_f<VC>(rs[e]);
    }
  }
}

// The x = 0 plane of cx of the TS^3 tiles tileBase, tileBase+1, ... (one CTA
// per tile) into the packed layout of LevelView::cxf.
template <int TS = 16>
__global__ void __launch_bounds__(TS* TS) k_pack_cx_plane(const int64_t* __restrict__ tileOff,
                                                          int tileBase,
                                                          const float* __restrict__ cx,
                                                          float* __restrict__ cxf) {
  const int64_t off = tileOff[tileBase + blockIdx.x];
  const int c = threadIdx.x;  // y + TS z
  cxf[(off >> 4) + c] = cx[off + TS * c];
}

// x += scale * P xc (liquid cells only; vectors VT, coarse vectors VC).  On
// 16^3 tiles the packed x faces xf (if given) are written too.
template <int TS, typename VT, typename VC>
__global__ void __launch_bounds__(TS* TS) k_prolong(LevelView L, const int* __restrict__ tiles,
                                                    VT* __restrict__ x,
                                                    const VC* __restrict__ xc,
                                                    const int64_t* __restrict__ coarseOff,
                                                    float scale, VT* __restrict__ xf) {
  constexpr int N = TS * TS * TS, NT = TS * TS;
  const int ti = tiles[blockIdx.x];
  const int64_t off = L.tileOff[ti];
  const int* tc = L.toCoarse + (size_t)ti * 6;
  const int ct = tc[0], ox = tc[1], oy = tc[2], oz = tc[3], agg = tc[4], cts = tc[5];
  if (ct < 0) return;
  const VC* src = xc + coarseOff[ct];
  const int sh = agg ? 1 : 0;
  if constexpr (TS >= 4) {
    // groups of 4 x-consecutive cells: every load of a thread's groups is
    // issued before any is used (non-liquid cells are written back unchanged)
    constexpr int PER = (N / 4 + NT - 1) / NT;
    F4 dv[PER], xv[PER], cv[PER];
#pragma unroll
    for (int p = 0; p < PER; p++) {
      const int e = 4 * (threadIdx.x + NT * p);
      if (e >= N) continue;
      const int i = e % TS, j = (e / TS) % TS, k = e / (TS * TS);
      dv[p] = load4(L.diag + off + e);
      xv[p] = load4(x + off + e);
      const VC* row = src + tidx(cts, 0, oy + (j >> sh), oz + (k >> sh));
      cv[p].x = to_f(row[ox + (i >> sh)]);
      cv[p].y = to_f(row[ox + ((i + 1) >> sh)]);
      cv[p].z = to_f(row[ox + ((i + 2) >> sh)]);
      cv[p].w = to_f(row[ox + ((i + 3) >> sh)]);
    }
#pragma unroll
    for (int p = 0; p < PER; p++) {
      const int e = 4 * (threadIdx.x + NT * p);
      if (e >= N) continue;
      F4 o = xv[p];
      if (dv[p].x > 0.f) o.x = to_f(from_f<VT>(xv[p].x + scale * cv[p].x));
      if (dv[p].y > 0.f) o.y = to_f(from_f<VT>(xv[p].y + scale * cv[p].y));
      if (dv[p].z > 0.f) o.z = to_f(from_f<VT>(xv[p].z + scale * cv[p].z));
      if (dv[p].w > 0.f) o.w = to_f(from_f<VT>(xv[p].w + scale * cv[p].w));
      store4(x + off + e, o);
      if (TS == 16 && xf) {
        const int i = e % TS, j = (e / TS) % TS, k = e / (TS * TS);
        if (i == 0) xf[xface_slot(off, 0, j, k)] = from_f<VT>(o.x);
        if (i == TS - 4) xf[xface_slot(off, 1, j, k)] = from_f<VT>(o.w);
      }
    }
  } else {
    for (int e = threadIdx.x; e < N; e += NT) {
      if (!(L.diag[off + e] > 0.f)) continue;
      const int i = e % TS, j = (e / TS) % TS, k = e / (TS * TS);
      const float c = to_f(src[tidx(cts, ox + (i >> sh), oy + (j >> sh), oz + (k >> sh))]);
      x[off + e] = from_f<VT>(to_f(x[off + e]) + scale * c);
    }
  }
}

// Red-black Gauss-Seidel inside each listed tile, `inner` iterations, ghosts
// frozen at their values when the tile is loaded.  reverse=0: red then black;
// reverse=1: black then red (the adjoint order).
template <int TS, typename VT>
__global__ void __launch_bounds__(TS* TS) k_smooth(LevelView L, const int* __restrict__ tiles,
                                                   VT* __restrict__ x, const VT* __restrict__ b,
                                                   int inner, int reverse) {
  constexpr int N = TS * TS * TS, NT = TS * TS;
  extern __shared__ __align__(128) float sm[];
  float* xs = sm;
  float* cxs = sm + N;
  float* cys = sm + 2 * N;
  float* czs = sm + 3 * N;
  float(*gs)[NT] = reinterpret_cast<float(*)[NT]>(sm + 4 * N);
  const int ti = tiles[blockIdx.x];
  const int64_t off = L.tileOff[ti];
  const int t = threadIdx.x, i = t % TS, j = t / TS;
  for (int e = t; e < N; e += NT) {
    xs[e] = to_f(x[off + e]);
    cxs[e] = L.cx[off + e];
    cys[e] = L.cy[off + e];
    czs[e] = L.cz[off + e];
  }
  float bb[TS], inv[TS];
#pragma unroll
  for (int k = 0; k < TS; k++) {
    const int e = tidx(TS, i, j, k);
    inv[k] = L.invdiag[off + e];
    bb[k] = to_f(b[off + e]);
  }
#pragma unroll
  for (int f = 0; f < 6; f++) gs[f][t] = ghost_sum(L, x, ti, TS, f >> 1, f & 1, i, j);
  __syncthreads();
  for (int it = 0; it < inner; it++) {
#pragma unroll
    for (int h = 0; h < 2; h++) {
      const int colour = reverse ? 1 - h : h;
#pragma unroll
      for (int k = 0; k < TS; k++) {
        if (((i + j + k) & 1) != colour || inv[k] == 0.f) continue;
        const float S = nbr_sum<TS>(xs, cxs, cys, czs, gs, i, j, k);
        xs[tidx(TS, i, j, k)] = (bb[k] + S) * inv[k];
      }
      __syncthreads();
    }
  }
  for (int e = t; e < N; e += NT) x[off + e] = from_f<VT>(xs[e]);
}

template <int TS>
size_t smooth_smem() {
  return sizeof(float) * (4 * TS * TS * TS + 6 * TS * TS);
}

// Coarsest level: x = A^-1 b with the dense FP64 inverse (symmetric).
template <typename VT>
__global__ void __launch_bounds__(512) k_coarse_solve(const double* __restrict__ Ainv, int n,
                                                      const int64_t* __restrict__ cells,
                                                      const VT* __restrict__ b,
                                                      VT* __restrict__ x) {
  __shared__ double bs[512];
  const int t = threadIdx.x;
  if (t < n) bs[t] = to_f(b[cells[t]]);
  __syncthreads();
  if (t >= n) return;
  double s = 0;
  for (int j = 0; j < n; j++) s += Ainv[(size_t)j * n + t] * bs[j];
  x[cells[t]] = from_f<VT>((float)s);
}
