// Persistent, TMA-pipelined red-black tile smoother for 16^3 tiles (the
// level-0 hot path of the pressure V-cycle).  Included inside namespace
// msbg::ps of pressure.cu.
//
// One CTA per SM walks a pass (a contiguous range of tile ids of one level and
// colour) with a stride of gridDim.x.  Per tile:
//   * the six contiguous 16 KB arrays (x, b, 1/a_ii, cx, cy, cz) arrive by bulk
//     asynchronous copies (cp.async.bulk, completion on an mbarrier) into one
//     of two shared-memory stages, issued one tile ahead;
//   * the tile's 256-byte record (its offset and the resolved data of its six
//     faces) arrives the same way two tiles ahead, so no dependent global load
//     sits on the critical path;
//   * the halo values of the next tile are loaded into registers before the
//     current tile is smoothed and summed afterwards;
//   * the smoothed x leaves by one bulk store.
// 512 threads; per colour each thread owns 4 cells whose couplings, 1/a_ii
// and right-hand side (with the constant halo sums folded in) sit in
// registers, laid out so a warp's shared-memory accesses hit 32 banks.
//
// Vectors may be stored in 16 bits (VT = __half / __nv_bfloat16): x and b
// then arrive together in stage slot 1 and x is widened into the FP32
// working slot 0; the smoothed tile is narrowed back into slot 1 for the
// bulk store.  The operator arrays are always FP32.

namespace pipe {

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}
__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}
// Bounded wait on the given phase parity; false if the copies never landed.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  uint32_t done = 0;
  for (int i = 0; i < (1 << 24); i++) {
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes,
                                         uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cta.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void bulk_s2g(void* dst, const void* src, uint32_t bytes) {
  asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(dst),
               "r"(smem_u32(src)), "r"(bytes)
               : "memory");
  asm volatile("cp.async.bulk.commit_group;" ::: "memory");
}
// Wait until the bulk stores issued so far have finished reading shared memory.
__device__ __forceinline__ void bulk_wait_read() {
  asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
}
__device__ __forceinline__ void bulk_wait_all() {
  asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
}

constexpr int TS = 16, N = TS * TS * TS, NT = 512;
constexpr int NT_SMOOTH = 1024;  // threads of the smoother CTA
constexpr int NT_APPLY = 1024;   // threads of the operator-application CTA

// Per-face data of a tile needed to gather its halo.
struct FaceRes {
  int kind, nts, oa, ob, cov, pad;
  int64_t nOff;   // SAME/COARSER: neighbour tile offset
  int64_t ifOwn;  // COARSER: our interface-coupling plane
};
struct __align__(16) TileRec {
  int64_t off;
  int64_t pad;
  FaceRes f[6];
};
static_assert(sizeof(TileRec) == 256, "tile record is one 256-byte bulk copy");

// A zeroed guard band in front of the first stage keeps the neighbour reads
// of boundary cells (whose couplings are zero) inside shared memory.
constexpr int GUARD = TS * TS;
constexpr int ZERO_FLOATS = GUARD + 12 * N + 2 * 6 * TS * TS;
constexpr size_t SMEM = sizeof(float) * ZERO_FLOATS + 3 * sizeof(TileRec) + 3 * sizeof(uint64_t);

// Issue the global loads of one halo cell of a SAME/COARSER face; the own
// lower-face coupling of a SAME face is taken later from shared memory.
template <typename VT>
__device__ __forceinline__ void halo_load(const LevelView& L, const VT* __restrict__ x,
                                          const FaceRes& r, int dir, int side, int a, int b,
                                          float& xv, float& cv) {
  const float* cd = dir == 0 ? L.cx : dir == 1 ? L.cy : L.cz;
  xv = 0.f;
  cv = 0.f;
  if (r.kind == FACE_SAME) {
    xv = to_f(__ldg(x + r.nOff + plane_idx(TS, dir, side ? 0 : TS - 1, a, b)));
    if (side) cv = __ldg(cd + r.nOff + plane_idx(TS, dir, 0, a, b));
  } else if (r.kind == FACE_COARSER) {
    xv = to_f(__ldg(x + r.nOff + plane_idx(r.nts, dir, side ? 0 : r.nts - 1, r.oa + (a >> 1),
                                           r.ob + (b >> 1))));
    cv = __ldg(L.ifc + r.ifOwn + a + TS * b);
  }
}

// Where the x and b vectors of a tile land in a stage: FP32 x straight into
// the working slot 0 and b into slot 1; 16-bit x and b both into slot 1.
template <typename VT>
__device__ __forceinline__ VT* raw_x(float* st) {
  return std::is_same<VT, float>::value ? reinterpret_cast<VT*>(st)
                                        : reinterpret_cast<VT*>(st + N);
}
template <typename VT>
__device__ __forceinline__ VT* raw_b(float* st) {
  return reinterpret_cast<VT*>(st + N) + (std::is_same<VT, float>::value ? 0 : N);
}
// Widen a 16-bit x tile into the FP32 working slot (no-op for FP32).
template <typename VT, int NTH = NT>
__device__ __forceinline__ void widen_x(float* st, int tid) {
  if (std::is_same<VT, float>::value) return;
  const VT* xr = raw_x<VT>(st);
  for (int e = tid; e < N; e += NTH) st[e] = to_f(xr[e]);
}

}  // namespace pipe

// NTH threads: each owns KK cells of each colour (NTH = 512: 4, 1024: 2).
template <typename VT, int NTH>
__global__ void __launch_bounds__(NTH, 1)
    k_smooth_pipe16(LevelView L, int tileBase, int count, VT* __restrict__ x,
                    const VT* __restrict__ b, int inner, int reverse, int* __restrict__ err) {
  using namespace pipe;
  constexpr int KK = N / (2 * NTH);           // cells per colour per thread
  constexpr int KSTRIDE = TS / KK;             // z distance of a thread's cells
  constexpr int NHALO = 6 * TS * TS;           // halo cells of a tile
  constexpr int HQ = (NHALO + NTH - 1) / NTH;  // halo cells per thread
  extern __shared__ __align__(128) float sm[];
  float* stages[2] = {sm + GUARD, sm + GUARD + 6 * N};
  float(*gsb)[6][TS * TS] = reinterpret_cast<float(*)[6][TS * TS]>(sm + GUARD + 12 * N);
  TileRec* recs = reinterpret_cast<TileRec*>(sm + ZERO_FLOATS);
  uint64_t* bar = reinterpret_cast<uint64_t*>(recs + 3);  // [0],[1] stages, [2] prologue
  const TileRec* grec = reinterpret_cast<const TileRec*>(L.tileRec) + tileBase;
  const int tid = threadIdx.x;
  const int G = gridDim.x;
  int t = blockIdx.x;
  if (t >= count) return;
  // every float of shared memory holds 0 or a value of our (finite) arrays
  for (int q = tid; q < ZERO_FLOATS / 4; q += NTH)
    reinterpret_cast<float4*>(sm)[q] = make_float4(0.f, 0.f, 0.f, 0.f);
  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    mbar_init(&bar[2], 1);
    fence_mbar_init();
  }
  __syncthreads();
  auto issue_arrays = [&](const TileRec& r, float* st, uint64_t* br, int tRec, int slot) {
    fence_proxy_async();
    const bool rec = tRec < count;
    mbar_expect_tx(br, 2 * N * sizeof(VT) + 4 * N * sizeof(float) + (rec ? sizeof(TileRec) : 0));
    const int64_t off = r.off;
    bulk_g2s(raw_x<VT>(st), x + off, N * sizeof(VT), br);
    bulk_g2s(raw_b<VT>(st), b + off, N * sizeof(VT), br);
    bulk_g2s(st + 2 * N, L.invdiag + off, N * sizeof(float), br);
    bulk_g2s(st + 3 * N, L.cx + off, N * sizeof(float), br);
    bulk_g2s(st + 4 * N, L.cy + off, N * sizeof(float), br);
    bulk_g2s(st + 5 * N, L.cz + off, N * sizeof(float), br);
    if (rec) bulk_g2s(&recs[slot], grec + tRec, sizeof(TileRec), br);
  };
  float hx[HQ], hc[HQ];
  auto halo_issue = [&](const TileRec& r) {
#pragma unroll
    for (int q = 0; q < HQ; q++) {
      const int g = tid + NTH * q, f = g >> 8, c = g & 255;
      if (NHALO % NTH == 0 || g < NHALO)
        halo_load(L, x, r.f[f], f >> 1, f & 1, c & 15, c >> 4, hx[q], hc[q]);
    }
  };
  auto halo_combine = [&](const TileRec& r, int ti, int u) {
    widen_x<VT, NTH>(stages[u], tid);
    const float* st = stages[u];
#pragma unroll
    for (int q = 0; q < HQ; q++) {
      const int g = tid + NTH * q, f = g >> 8, c = g & 255;
      if (NHALO % NTH != 0 && g >= NHALO) continue;
      const int dir = f >> 1, side = f & 1, a = c & 15, bb = c >> 4;
      const int kind = r.f[f].kind;
      float v = 0.f;
      if (kind == FACE_SAME) {
        const float cown = st[(3 + dir) * N + plane_idx(TS, dir, 0, a, bb)];
        v = (side ? hc[q] : cown) * hx[q];
      } else if (kind == FACE_COARSER) {
        v = hc[q] * hx[q];
      } else if (kind == FACE_FINER) {
        v = ghost_sum(L, x, ti, TS, dir, side, a, bb);
      }
      gsb[u][f][c] = v;
    }
  };
  // prologue: the first tile's record, then its arrays (which bring the
  // second tile's record along: the arrays of tile m carry record m+1)
  if (tid == 0) {
    mbar_expect_tx(&bar[2], sizeof(TileRec));
    bulk_g2s(&recs[0], grec + t, sizeof(TileRec), &bar[2]);
  }
  if (!__syncthreads_and(mbar_wait(&bar[2], 0))) {
    if (tid == 0) atomicExch(err, 1);
    return;
  }
  if (tid == 0) issue_arrays(recs[0], stages[0], &bar[0], t + G, 1);
  halo_issue(recs[0]);
  if (!__syncthreads_and(mbar_wait(&bar[0], 0))) {
    if (tid == 0) {
      atomicExch(err, 1);
      mbar_wait(&bar[0], 0);  // one more bounded wait for the copies in flight
    }
    return;
  }
  halo_combine(recs[0], tileBase + t, 0);
  __syncthreads();
  const int ip = tid & 7, jj = 2 * ((tid >> 5) & 7) + ((tid >> 3) & 1);
  const int kb = ((tid >> 4) & 1) + 2 * (tid >> 8);
  for (int n = 0; t < count; n++, t += G) {
    const int s = n & 1, u = s ^ 1;
    const int tn = t + G;
    const bool hasNext = tn < count;
    const TileRec& rc = recs[n % 3];
    const TileRec& rn = recs[(n + 1) % 3];
    // 1: prefetch the next tile (arrays + the record two ahead), halo loads
    if (hasNext) {
      if (tid == 0) {
        bulk_wait_read();  // the store from stage u (tile n-1) has read it
        issue_arrays(rn, stages[u], &bar[u], tn + G, (n + 2) % 3);
      }
      halo_issue(rn);
    }
    // 2: registers: couplings, 1/a_ii, b with the halo sums folded in
    float* X = stages[s];
    const VT* B = raw_b<VT>(X);
    const float* IV = X + 2 * N;
    const float* CX = X + 3 * N;
    const float* CY = X + 4 * N;
    const float* CZ = X + 5 * N;
    const float(*gs)[TS * TS] = gsb[s];
    float R[2][KK], I[2][KK], Cm[2][KK][3], Cp[2][KK][3];
    // A thread's two cells at (jj, k) are x-neighbours 2ip, 2ip+1 (one per
    // colour): their coefficients come as float2 pairs.  The even cell has
    // colour (jj + k) & 1; runtime selects keep the arrays compile-time indexed.
#pragma unroll
    for (int kk = 0; kk < KK; kk++) {
      const int k = kb + KSTRIDE * kk;
      const int e0 = tidx(TS, 2 * ip, jj, k);
      const float2 iv2 = *reinterpret_cast<const float2*>(IV + e0);
      const float2 cx2 = *reinterpret_cast<const float2*>(CX + e0);
      const float cxn = CX[e0 + 2];  // past the row end only when unused (ii = 15)
      const float2 cy2 = *reinterpret_cast<const float2*>(CY + e0);
      const float2 cyn = *reinterpret_cast<const float2*>(CY + e0 + TS);
      const float2 cz2 = *reinterpret_cast<const float2*>(CZ + e0);
      const float2 czn = *reinterpret_cast<const float2*>(CZ + e0 + TS * TS);
      const float ivv[2] = {iv2.x, iv2.y};
      float rr[2] = {to_f(B[e0]), to_f(B[e0 + 1])};
      float cm[2][3], cp[2][3];
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const int ii = 2 * ip + h;
        const bool fl = ivv[h] > 0.f;
        if (ii == 0) rr[h] += gs[0][jj + TS * k];
        if (ii == TS - 1) rr[h] += gs[1][jj + TS * k];
        if (jj == 0) rr[h] += gs[2][ii + TS * k];
        if (jj == TS - 1) rr[h] += gs[3][ii + TS * k];
        if (k == 0) rr[h] += gs[4][ii + TS * jj];
        if (k == TS - 1) rr[h] += gs[5][ii + TS * jj];
        cm[h][0] = (fl && ii > 0) ? (h ? cx2.y : cx2.x) : 0.f;
        cp[h][0] = (fl && ii < TS - 1) ? (h ? cxn : cx2.y) : 0.f;
        cm[h][1] = (fl && jj > 0) ? (h ? cy2.y : cy2.x) : 0.f;
        cp[h][1] = (fl && jj < TS - 1) ? (h ? cyn.y : cyn.x) : 0.f;
        cm[h][2] = (fl && k > 0) ? (h ? cz2.y : cz2.x) : 0.f;
        cp[h][2] = (fl && k < TS - 1) ? (h ? czn.y : czn.x) : 0.f;
      }
      const bool evenIs0 = ((jj + k) & 1) == 0;  // colour 0 is the even cell
#pragma unroll
      for (int c = 0; c < 2; c++) {
        const bool ev = (c == 0) == evenIs0;
        I[c][kk] = ev ? ivv[0] : ivv[1];
        R[c][kk] = ev ? rr[0] : rr[1];
#pragma unroll
        for (int d = 0; d < 3; d++) {
          Cm[c][kk][d] = ev ? cm[0][d] : cm[1][d];
          Cp[c][kk][d] = ev ? cp[0][d] : cp[1][d];
        }
      }
    }
    // 3: red-black sweeps (colour compile-time so the arrays stay in registers)
    auto half = [&](auto cc) {
      constexpr int c = decltype(cc)::value;
#pragma unroll
      for (int kk = 0; kk < KK; kk++) {
        const int k = kb + KSTRIDE * kk, ii = 2 * ip + ((jj + k + c) & 1);
        const int e = tidx(TS, ii, jj, k);
        // out-of-tile neighbours have zero coupling; their reads stay inside
        // shared memory (guard band / adjacent arrays, all finite)
        float S = R[c][kk];
        S = fmaf(Cm[c][kk][0], X[e - 1], S);
        S = fmaf(Cp[c][kk][0], X[e + 1], S);
        S = fmaf(Cm[c][kk][1], X[e - TS], S);
        S = fmaf(Cp[c][kk][1], X[e + TS], S);
        S = fmaf(Cm[c][kk][2], X[e - TS * TS], S);
        S = fmaf(Cp[c][kk][2], X[e + TS * TS], S);
        X[e] = S * I[c][kk];
      }
      __syncthreads();
    };
    for (int it = 0; it < inner; it++) {
      if (reverse) {
        half(std::integral_constant<int, 1>());
        half(std::integral_constant<int, 0>());
      } else {
        half(std::integral_constant<int, 0>());
        half(std::integral_constant<int, 1>());
      }
    }
    // 4: the tile leaves by one bulk store (narrowed into slot 1 first when
    // the vectors are 16-bit; slot 1's b is no longer read)
    if (!std::is_same<VT, float>::value) {
      VT* xr = raw_x<VT>(X);
      for (int e = tid; e < N; e += NTH) xr[e] = from_f<VT>(X[e]);
      __syncthreads();
    }
    if (tid == 0) {
      fence_proxy_async();
      bulk_s2g(x + rc.off, raw_x<VT>(X), N * sizeof(VT));
    }
    // 5: next tile's arrays landed -> its halo sums
    if (hasNext) {
      if (!__syncthreads_and(mbar_wait(&bar[u], ((n + 1) >> 1) & 1))) {
        if (tid == 0) {
          atomicExch(err, 1);
          bulk_wait_all();
        }
        return;
      }
      halo_combine(rn, tileBase + tn, u);
    }
    __syncthreads();  // stage s, gsb[s] and record slot n%3 are free again
  }
  if (tid == 0) bulk_wait_all();
}

// Host side: the 256-byte tile records of one level (offset + resolved faces).
inline std::vector<pipe::TileRec> build_tile_records(const Level& L) {
  std::vector<pipe::TileRec> recs(L.tiles.size());
  for (size_t ti = 0; ti < L.tiles.size(); ti++) {
    pipe::TileRec& r = recs[ti];
    std::memset(&r, 0, sizeof(r));
    r.off = L.tiles[ti].off;
    for (int f = 0; f < 6; f++) {
      const int* F = &L.face[(ti * 6 + f) * FACE_INTS];
      pipe::FaceRes& fr = r.f[f];
      fr.kind = F[F_KIND];
      fr.nts = F[F_NTS];
      fr.oa = F[F_OA];
      fr.ob = F[F_OB];
      fr.cov = F[F_COV];
      fr.nOff = (fr.kind == FACE_SAME || fr.kind == FACE_COARSER) ? L.tiles[F[F_T0]].off : 0;
      fr.ifOwn = fr.kind == FACE_COARSER ? L.ifOff[ti * 6 + f] : 0;
    }
  }
  return recs;
}

// ---------------------------------------------------------------------------
// Persistent, TMA-pipelined operator application on 16^3 tiles (same
// pipeline as the smoother, read-only on x, no colouring):
//   APPLY_MATVEC:   q = A d, per-CTA partial d.q           (b unused)
//   APPLY_RESIDUAL: r = b - A x, restricted into the coarse right-hand side
//                   (sum over the liquid children, or copy for cells that do
//                   not coarsen) through the tile's coarse map.
// Thread (i, j, half) marches 8 cells of the z column (i, j) with a register
// window; warps read shared memory without bank conflicts.
// ---------------------------------------------------------------------------
enum { APPLY_MATVEC = 0, APPLY_RESIDUAL = 1 };

template <int MODE, typename VT, typename VC, int NTH>
__global__ void __launch_bounds__(NTH, 1)
    k_apply_pipe16(LevelView L, int tileBase, int count, const VT* __restrict__ x,
                   const VT* __restrict__ b, VT* __restrict__ y,
                   VC* __restrict__ bc, const int64_t* __restrict__ coarseOff,
                   double* __restrict__ partial, int* __restrict__ err) {
  using namespace pipe;
  constexpr int ZC = TS / (NTH / (TS * TS));  // cells of a thread's z column
  constexpr int NHALO = 6 * TS * TS;
  constexpr int HQ = (NHALO + NTH - 1) / NTH;
  constexpr int NVEC = MODE == APPLY_RESIDUAL ? 2 : 1;  // x, [b]
  extern __shared__ __align__(128) float sm[];
  float* stages[2] = {sm + GUARD, sm + GUARD + 6 * N};
  float(*gsb)[6][TS * TS] = reinterpret_cast<float(*)[6][TS * TS]>(sm + GUARD + 12 * N);
  TileRec* recs = reinterpret_cast<TileRec*>(sm + ZERO_FLOATS);
  uint64_t* bar = reinterpret_cast<uint64_t*>(recs + 3);
  __shared__ int cmap[2][6];  // coarse tile, ox, oy, oz, aggregated, coarse ts
  const TileRec* grec = reinterpret_cast<const TileRec*>(L.tileRec) + tileBase;
  const int tid = threadIdx.x;
  const int G = gridDim.x;
  int t = blockIdx.x;
  double acc = 0;
  if (t < count) {
    if (tid == 0) {
      mbar_init(&bar[0], 1);
      mbar_init(&bar[1], 1);
      mbar_init(&bar[2], 1);
      fence_mbar_init();
    }
    __syncthreads();
    // stage arrays: 0 x, 1 b (residual), 2 a_ii, 3..5 couplings
    auto issue_arrays = [&](const TileRec& r, float* st, uint64_t* br, int tRec, int slot) {
      fence_proxy_async();
      const bool rec = tRec < count;
      mbar_expect_tx(br, NVEC * N * sizeof(VT) + 4 * N * sizeof(float) +
                             (rec ? sizeof(TileRec) : 0));
      const int64_t off = r.off;
      bulk_g2s(raw_x<VT>(st), x + off, N * sizeof(VT), br);
      if (MODE == APPLY_RESIDUAL) bulk_g2s(raw_b<VT>(st), b + off, N * sizeof(VT), br);
      bulk_g2s(st + 2 * N, L.diag + off, N * sizeof(float), br);
      bulk_g2s(st + 3 * N, L.cx + off, N * sizeof(float), br);
      bulk_g2s(st + 4 * N, L.cy + off, N * sizeof(float), br);
      bulk_g2s(st + 5 * N, L.cz + off, N * sizeof(float), br);
      if (rec) bulk_g2s(&recs[slot], grec + tRec, sizeof(TileRec), br);
    };
    float hx[HQ], hc[HQ];
    auto halo_issue = [&](const TileRec& r, int ti, int u) {
#pragma unroll
      for (int q = 0; q < HQ; q++) {
        const int g = tid + NTH * q, f = g >> 8, c = g & 255;
        if (NHALO % NTH == 0 || g < NHALO)
          halo_load(L, x, r.f[f], f >> 1, f & 1, c & 15, c >> 4, hx[q], hc[q]);
      }
      if (MODE == APPLY_RESIDUAL && tid < 6) cmap[u][tid] = L.toCoarse[(size_t)ti * 6 + tid];
    };
    auto halo_combine = [&](const TileRec& r, int ti, int u) {
      widen_x<VT, NTH>(stages[u], tid);
      const float* st = stages[u];
#pragma unroll
      for (int q = 0; q < HQ; q++) {
        const int g = tid + NTH * q, f = g >> 8, c = g & 255;
        if (NHALO % NTH != 0 && g >= NHALO) continue;
        const int dir = f >> 1, side = f & 1, a = c & 15, bb = c >> 4;
        const int kind = r.f[f].kind;
        float v = 0.f;
        if (kind == FACE_SAME) {
          const float cown = st[(3 + dir) * N + plane_idx(TS, dir, 0, a, bb)];
          v = (side ? hc[q] : cown) * hx[q];
        } else if (kind == FACE_COARSER) {
          v = hc[q] * hx[q];
        } else if (kind == FACE_FINER) {
          v = ghost_sum(L, x, ti, TS, dir, side, a, bb);
        }
        gsb[u][f][c] = v;
      }
    };
    if (tid == 0) {
      mbar_expect_tx(&bar[2], sizeof(TileRec));
      bulk_g2s(&recs[0], grec + t, sizeof(TileRec), &bar[2]);
    }
    bool ok = __syncthreads_and(mbar_wait(&bar[2], 0));
    if (ok) {
      if (tid == 0) issue_arrays(recs[0], stages[0], &bar[0], t + G, 1);
      halo_issue(recs[0], tileBase + t, 0);
      ok = __syncthreads_and(mbar_wait(&bar[0], 0));
      if (!ok && tid == 0) mbar_wait(&bar[0], 0);
    }
    if (!ok) {
      if (tid == 0) atomicExch(err, 1);
      t = count;  // skip the loop, still write this CTA's partial
    } else {
      halo_combine(recs[0], tileBase + t, 0);
      __syncthreads();
    }
    const int i = tid & 15, j = (tid >> 4) & 15, kh = tid >> 8;
    for (int n = 0; t < count; n++, t += G) {
      const int s = n & 1, u = s ^ 1;
      const int tn = t + G;
      const bool hasNext = tn < count;
      const TileRec& rc = recs[n % 3];
      const TileRec& rn = recs[(n + 1) % 3];
      if (hasNext) {
        if (tid == 0) {
          bulk_wait_read();
          issue_arrays(rn, stages[u], &bar[u], tn + G, (n + 2) % 3);
        }
        halo_issue(rn, tileBase + tn, u);
      }
      float* X = stages[s];
      const VT* B = raw_b<VT>(X);
      const float* D = X + 2 * N;
      const float* CX = X + 3 * N;
      const float* CY = X + 4 * N;
      const float* CZ = X + 5 * N;
      const float(*gs)[TS * TS] = gsb[s];
      float* Y = X + 2 * N;  // results overwrite the a_ii array in place (each
                             // thread reads its own a_ii before writing it)
      const int k0 = ZC * kh;
      float xm = k0 > 0 ? X[tidx(TS, i, j, k0 - 1)] : 0.f;
      float xc = X[tidx(TS, i, j, k0)];
      float yv[ZC];
#pragma unroll
      for (int kk = 0; kk < ZC; kk++) {
        const int k = k0 + kk, e = tidx(TS, i, j, k);
        const float xp = k < TS - 1 ? X[e + TS * TS] : 0.f;
        const float dg = D[e];
        float S = 0.f;
        S += i > 0 ? CX[e] * X[e - 1] : gs[0][j + TS * k];
        S += i < TS - 1 ? CX[e + 1] * X[e + 1] : gs[1][j + TS * k];
        S += j > 0 ? CY[e] * X[e - TS] : gs[2][i + TS * k];
        S += j < TS - 1 ? CY[e + TS] * X[e + TS] : gs[3][i + TS * k];
        S += k > 0 ? CZ[e] * xm : gs[4][i + TS * j];
        S += k < TS - 1 ? CZ[e + TS * TS] * xp : gs[5][i + TS * j];
        float v = 0.f;
        if (dg > 0.f) v = dg * xc - S;
        if (MODE == APPLY_RESIDUAL) {
          if (dg > 0.f) v = to_f(B[e]) - v;
        } else {
          v = to_f(from_f<VT>(v));  // the dot product sees the stored q
          acc += (double)xc * (double)v;
        }
        yv[kk] = v;
        xm = xc;
        xc = xp;
      }
      __syncthreads();  // every thread has read its D / neighbours before Y is written
      if (MODE == APPLY_MATVEC) {
        VT* Yv = reinterpret_cast<VT*>(Y);
#pragma unroll
        for (int kk = 0; kk < ZC; kk++) Yv[tidx(TS, i, j, k0 + kk)] = from_f<VT>(yv[kk]);
      } else {
#pragma unroll
        for (int kk = 0; kk < ZC; kk++) Y[tidx(TS, i, j, k0 + kk)] = yv[kk];
      }
      __syncthreads();
      if (MODE == APPLY_MATVEC) {
        if (tid == 0) {
          fence_proxy_async();
          bulk_s2g(y + rc.off, Y, N * sizeof(VT));
        }
      } else {
        const int* tc = cmap[s];
        const int ct = tc[0];
        if (ct >= 0) {
          VC* dst = bc + coarseOff[ct];
          const int ox = tc[1], oy = tc[2], oz = tc[3], cts = tc[5];
          if (tc[4]) {
            constexpr int H = TS / 2;
            for (int c = tid; c < H * H * H; c += NTH) {  // 512 coarse cells
            const int ci = c % H, cj = (c / H) % H, ck = c / (H * H);
            const int e = tidx(TS, 2 * ci, 2 * cj, 2 * ck);
            const float sum = Y[e] + Y[e + 1] + Y[e + TS] + Y[e + TS + 1] + Y[e + TS * TS] +
                              Y[e + TS * TS + 1] + Y[e + TS * TS + TS] +
                              Y[e + TS * TS + TS + 1];
            dst[tidx(cts, ox + ci, oy + cj, oz + ck)] = from_f<VC>(sum);
            }
          } else {
            for (int e = tid; e < N; e += NTH) {
              const int ii = e % TS, jj = (e / TS) % TS, kk = e / (TS * TS);
              dst[tidx(cts, ox + ii, oy + jj, oz + kk)] = from_f<VC>(Y[e]);
            }
          }
        }
      }
      if (hasNext) {
        if (!__syncthreads_and(mbar_wait(&bar[u], ((n + 1) >> 1) & 1))) {
          if (tid == 0) {
            atomicExch(err, 1);
            bulk_wait_all();
          }
          break;
        }
        halo_combine(rn, tileBase + tn, u);
      }
      __syncthreads();
    }
    if (tid == 0) bulk_wait_all();
  }
  if (MODE == APPLY_MATVEC && partial) {
    acc = block_sum(acc);
    if (tid == 0) partial[blockIdx.x] = acc;
  }
}
