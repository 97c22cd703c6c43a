// Persistent, TMA-pipelined red-black tile smoother for 16^3 tiles (the
// level-0 hot path of the pressure V-cycle).  Included inside namespace
// msbg::ps of pressure.cu.
//
// One CTA per SM walks a pass (a contiguous range of tile ids of one level and
// colour) with a stride of gridDim.x.  Per tile:
//   * the six contiguous 16 KB arrays (x, b, 1/a_ii, cx, cy, cz) arrive by bulk
//     asynchronous copies (cp.async.bulk, completion on an mbarrier) into one
//     of two shared-memory stages, issued one tile ahead, each copy by lane 0
//     of its own warp (FP32 x plane by plane into a padded slot);
//   * the tile's 256-byte record (its offset and the resolved data of its six
//     faces) arrives the same way two tiles ahead, so no dependent global load
//     sits on the critical path;
//   * the halo values of the next tile are loaded into registers before the
//     current tile is smoothed and summed afterwards;
//   * the smoothed x leaves from the registers (each thread stores its own
//     cells), so no store has to drain before a stage is refilled.
// 1024 threads, each owning a 2 x 2 block of cells (x pair, z pair) whose
// couplings, 1/a_ii, right-hand side (with the constant halo sums folded in)
// and x values sit in registers.
//
// Vectors may be stored in 16 bits (VT = __half / __nv_bfloat16): x and b
// then arrive together in the b slot and x is widened into the FP32 working
// slot; results are narrowed in registers as they are stored.  The operator
// arrays are always FP32.

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

// Issue the global loads of one halo cell of a SAME/COARSER face (the own
// lower-face coupling of a SAME face is taken later from shared memory).
// The branches only choose the addresses: each value is one load straight
// into its register, raw, so nothing waits for it before it is used (faces
// without these values load a harmless word and ignore it).  With the packed
// x faces xf of x (and L.cxf), an x face reads the neighbour's packed plane.
template <typename VT>
__device__ __forceinline__ void halo_load(const LevelView& L, const VT* __restrict__ x,
                                          const VT* __restrict__ xf, const FaceRes& r, int dir,
                                          int side, int a, int b, VT& xv, float& cv) {
  const float* cd = dir == 0 ? L.cx : dir == 1 ? L.cy : L.cz;
  const VT* px = x;
  const float* pc = cd;
  if (r.kind == FACE_SAME) {
    if (dir == 0 && xf) {
      px = xf + xface_slot(r.nOff, side ? 0 : 1, a, b);
      if (side) pc = L.cxf + (r.nOff >> 4) + a + TS * b;
    } else {
      px = x + r.nOff + plane_idx(TS, dir, side ? 0 : TS - 1, a, b);
      if (side) pc = cd + r.nOff + plane_idx(TS, dir, 0, a, b);
    }
  } else if (r.kind == FACE_COARSER) {
    px = x + r.nOff + plane_idx(r.nts, dir, side ? 0 : r.nts - 1, r.oa + (a >> 1), r.ob + (b >> 1));
    pc = L.ifc + r.ifOwn + a + TS * b;
  }
  xv = __ldg(px);
  cv = __ldg(pc);
}

// Where the x and b vectors of a tile land in a stage of the operator
// kernels: FP32 x straight into the working slot 0 and b into slot 1; 16-bit
// x and b both into slot 1.
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

// Shared-memory layout of the smoother: two stages of [x | b | 1/a_ii | cx |
// cy | cz], x with its z planes XP = 264 floats apart (the 8-float pad per
// plane makes the z-pair thread map below bank-conflict free), behind a
// zeroed guard of one padded plane, then the halo sums of both stages.
constexpr int XP = TS * TS + 8;
constexpr int XS = TS * XP;
constexpr int SGUARD = XP;
constexpr int SSTAGE = XS + 5 * N;
constexpr int SOFF_B = XS, SOFF_IV = XS + N, SOFF_C = XS + 2 * N;  // cx, cy, cz follow
constexpr int SZERO_FLOATS = SGUARD + 2 * SSTAGE + 2 * 6 * TS * TS;
constexpr size_t SMEM_SMOOTH =
    sizeof(float) * SZERO_FLOATS + 3 * sizeof(TileRec) + 3 * sizeof(uint64_t);
static_assert((SGUARD * 4) % 16 == 0 && (SSTAGE * 4) % 16 == 0 && (XP * 4) % 16 == 0,
              "bulk copy destinations stay 16-byte aligned");
static_assert(SMEM_SMOOTH <= 227 * 1024, "smoother stages fit one SM");
__host__ __device__ __forceinline__ int xpad(int e) { return e + 8 * (e >> 8); }

// 16-bit x and b of a tile arrive together in the b slot; FP32 b alone.
template <typename VT>
__device__ __forceinline__ VT* sraw_x(float* st) {
  return reinterpret_cast<VT*>(st + SOFF_B);
}
template <typename VT>
__device__ __forceinline__ VT* sraw_b(float* st) {
  return reinterpret_cast<VT*>(st + SOFF_B) + (std::is_same<VT, float>::value ? 0 : N);
}

}  // namespace pipe

// 1024 threads.  Thread (ip, jj, kp) owns the 2 x 2 cells x = 2ip + {0,1},
// z = 2kp + {0,1} of row jj: per colour one cell of each z plane, and for
// each of them the x- and the z-neighbour of the other colour are the
// thread's own cells, held in registers; 4 of the 6 neighbour values come
// from shared memory.  The arithmetic per update is that of the reference's
// order (x-, x+, y-, y+, z-, z+).
template <typename VT, int NTH>
__global__ void __launch_bounds__(NTH, 1)
    k_smooth_pipe16(LevelView L, int tileBase, int count, VT* __restrict__ x,
                    const VT* __restrict__ b, int inner, int reverse, int* __restrict__ err,
                    VT* __restrict__ xf) {
  using namespace pipe;
  static_assert(NTH == 1024, "the z-pair thread map covers a 16^3 tile with 1024 threads");
  constexpr int NHALO = 6 * TS * TS;           // halo cells of a tile
  constexpr int HQ = (NHALO + NTH - 1) / NTH;  // halo cells per thread
  constexpr bool WIDE = std::is_same<VT, float>::value;
  extern __shared__ __align__(128) float sm[];
  auto stage = [&](int i) { return sm + SGUARD + i * SSTAGE; };
  float(*gsb)[6][TS * TS] = reinterpret_cast<float(*)[6][TS * TS]>(sm + SGUARD + 2 * SSTAGE);
  TileRec* recs = reinterpret_cast<TileRec*>(sm + SZERO_FLOATS);
  uint64_t* bar = reinterpret_cast<uint64_t*>(recs + 3);  // [0],[1] stages, [2] prologue
  const TileRec* grec = reinterpret_cast<const TileRec*>(L.tileRec) + tileBase;
  const int tid = threadIdx.x;
  const int G = gridDim.x;
  int t = blockIdx.x;
  if (t >= count) return;
  // every float of shared memory holds 0, a value of our (finite) arrays or
  // two finite 16-bit values (never a float NaN/Inf pattern)
  for (int q = tid; q < SZERO_FLOATS / 4; q += NTH)
    reinterpret_cast<float4*>(sm)[q] = make_float4(0.f, 0.f, 0.f, 0.f);
  // The copies of a stage are issued in parallel, each by lane 0 of its own
  // warp (a bulk copy holds its issuing thread for ~100 cycles): FP32 x
  // plane by plane (warps 0-15) or 16-bit x whole (warp 0), then b, 1/a_ii,
  // cx, cy, cz, then the record; the stage barrier counts one arrival each.
  constexpr int NXC = WIDE ? TS : 1;
  constexpr int NISS = NXC + 6;
  if (tid == 0) {
    mbar_init(&bar[0], NISS);
    mbar_init(&bar[1], NISS);
    mbar_init(&bar[2], 1);
    fence_mbar_init();
  }
  __syncthreads();
  auto issue_arrays = [&](const TileRec& r, float* st, uint64_t* br, int tRec, int slot) {
    const int w = tid >> 5;
    if ((tid & 31) != 0 || w >= NISS) return;
    fence_proxy_async();
    const int64_t off = r.off;
    if (w == NISS - 1) {  // the record two tiles ahead, if there is one
      const bool rec = tRec < count;
      mbar_expect_tx(br, rec ? sizeof(TileRec) : 0);
      if (rec) bulk_g2s(&recs[slot], grec + tRec, sizeof(TileRec), br);
      return;
    }
    const void* src;
    void* dst;
    uint32_t bytes = N * sizeof(float);
    if (w < NXC) {
      if (WIDE) {
        src = x + off + w * TS * TS;
        dst = st + w * XP;
        bytes = TS * TS * sizeof(VT);
      } else {
        src = x + off;
        dst = sraw_x<VT>(st);
        bytes = N * sizeof(VT);
      }
    } else {
      switch (w - NXC) {
        case 0: src = b + off; dst = sraw_b<VT>(st); bytes = N * sizeof(VT); break;
        case 1: src = L.invdiag + off; dst = st + SOFF_IV; break;
        case 2: src = L.cx + off; dst = st + SOFF_C; break;
        case 3: src = L.cy + off; dst = st + SOFF_C + N; break;
        default: src = L.cz + off; dst = st + SOFF_C + 2 * N; break;
      }
    }
    mbar_expect_tx(br, bytes);
    bulk_g2s(dst, src, bytes, br);
  };
  VT hx[HQ];
  float hc[HQ];
  // packed x faces only with the packed upper-face couplings
  const VT* xfr = L.cxf ? xf : nullptr;
  auto halo_issue = [&](const TileRec& r) {
#pragma unroll
    for (int q = 0; q < HQ; q++) {
      const int g = tid + NTH * q, f = g >> 8, c = g & 255;
      if (NHALO % NTH == 0 || g < NHALO)
        halo_load(L, x, xfr, r.f[f], f >> 1, f & 1, c & 15, c >> 4, hx[q], hc[q]);
    }
  };
  auto halo_combine = [&](const TileRec& r, int ti, int u) {
    float* st = stage(u);
    if (!WIDE) {
      const VT* xr = sraw_x<VT>(st);
      for (int e = tid; e < N; e += NTH) st[xpad(e)] = to_f(xr[e]);
    }
#pragma unroll
    for (int q = 0; q < HQ; q++) {
      const int g = tid + NTH * q, f = g >> 8, c = g & 255;
      if (NHALO % NTH != 0 && g >= NHALO) continue;
      const int dir = f >> 1, side = f & 1, a = c & 15, bb = c >> 4;
      const int kind = r.f[f].kind;
      float v = 0.f;
      if (kind == FACE_SAME) {
        const float cown = st[SOFF_C + dir * N + plane_idx(TS, dir, 0, a, bb)];
        v = (side ? hc[q] : cown) * to_f(hx[q]);
      } else if (kind == FACE_COARSER) {
        v = hc[q] * to_f(hx[q]);
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
  issue_arrays(recs[0], stage(0), &bar[0], t + G, 1);
  halo_issue(recs[0]);
  if (!__syncthreads_and(mbar_wait(&bar[0], 0))) {
    if (tid == 0) atomicExch(err, 1);
    mbar_wait(&bar[0], 0);  // one more bounded wait for the copies in flight
    return;
  }
  halo_combine(recs[0], tileBase + t, 0);
  __syncthreads();
  const int ip = tid & 7;
  const int jj = ((tid >> 3) & 1) + 2 * ((tid >> 5) & 7);
  const int kp = ((tid >> 4) & 1) + 2 * (tid >> 8);
  const int q = jj & 1;
  // colour c, z slot s: the cell x = 2ip + dx(c, s), z = 2kp + s
  auto dxof = [&](int c, int s) { return (c + q + s) & 1; };
  const int eb = 2 * ip + TS * jj + XP * 2 * kp;  // padded index of (2ip, jj, 2kp)
  for (int n = 0; t < count; n++, t += G) {
    const int s = n & 1, u = s ^ 1;
    const int tn = t + G;
    const bool hasNext = tn < count;
    const TileRec& rc = recs[n % 3];
    const TileRec& rn = recs[(n + 1) % 3];
    // 1: prefetch the next tile (arrays + the record two ahead), halo loads
    if (hasNext) {
      issue_arrays(rn, stage(u), &bar[u], tn + G, (n + 2) % 3);
      halo_issue(rn);
    }
    // 2: registers: couplings, 1/a_ii, b with the halo sums folded in, and
    // the thread's own four x values
    float* X = stage(s);
    const VT* B = sraw_b<VT>(X);
    const float* IV = X + SOFF_IV;
    const float* CX = X + SOFF_C;
    const float* CY = CX + N;
    const float* CZ = CY + N;
    const float(*gs)[TS * TS] = gsb[s];
    // Per colour c and z slot sl: 1/a_ii, b + halo sums, x, and the
    // couplings to the x- and z-neighbours read from shared memory (Cxo,
    // Czo) and to y-1, y+1.  The coupling inside the x pair (cx of cell
    // 2ip+1) and inside the z pair (cz of plane 2kp+1) is shared by the two
    // cells it joins.  Couplings across the tile boundary are zero; the
    // reference's extra zeroing for non-liquid cells is implied by their
    // 1/a_ii = 0.
    float R[2][2], I[2][2], xv[2][2], Cxo[2][2], Cym[2][2], Cyp[2][2], Czo[2][2];
    float Cxp[2], Czp[2];  // pair couplings: x per z slot, z per x cell (h)
    const int u0 = 2 * ip + TS * jj + TS * TS * 2 * kp;
    {
      // cz of the planes 2kp, 2kp+1, 2kp+2 (the last read past plane 15
      // only when kp = 7, where it is unused)
      const float2 cz0 = *reinterpret_cast<const float2*>(CZ + u0);
      const float2 cz1 = *reinterpret_cast<const float2*>(CZ + u0 + TS * TS);
      const float2 cz2 = *reinterpret_cast<const float2*>(CZ + u0 + 2 * TS * TS);
      Czp[0] = cz1.x;
      Czp[1] = cz1.y;
#pragma unroll
      for (int sl = 0; sl < 2; sl++) {
        const int k = 2 * kp + sl;
        const int e0 = u0 + TS * TS * sl;
        const float2 iv2 = *reinterpret_cast<const float2*>(IV + e0);
        const float2 cx2 = *reinterpret_cast<const float2*>(CX + e0);
        const float cxn = CX[e0 + 2];  // past the row end only when unused (ip = 7)
        const float2 cy2 = *reinterpret_cast<const float2*>(CY + e0);
        const float2 cyn = *reinterpret_cast<const float2*>(CY + e0 + TS);
        const float2 x2 = *reinterpret_cast<const float2*>(X + eb + XP * sl);
        Cxp[sl] = cx2.y;
        const float ivv[2] = {iv2.x, iv2.y};
        const float xx[2] = {x2.x, x2.y};
        // the x coupling away from the pair: x-1 of cell 0, x+1 of cell 1
        const float cxo[2] = {ip > 0 ? cx2.x : 0.f, ip < 7 ? cxn : 0.f};
        const float cym[2] = {jj > 0 ? cy2.x : 0.f, jj > 0 ? cy2.y : 0.f};
        const float cyp[2] = {jj < TS - 1 ? cyn.x : 0.f, jj < TS - 1 ? cyn.y : 0.f};
        // the z coupling away from the pair: z-1 of plane 2kp, z+1 of 2kp+1
        const float czo[2] = {sl ? (kp < 7 ? cz2.x : 0.f) : (kp > 0 ? cz0.x : 0.f),
                              sl ? (kp < 7 ? cz2.y : 0.f) : (kp > 0 ? cz0.y : 0.f)};
        float rr[2] = {to_f(B[e0]), to_f(B[e0 + 1])};
#pragma unroll
        for (int h = 0; h < 2; h++) {
          const int ii = 2 * ip + h;
          if (ii == 0) rr[h] += gs[0][jj + TS * k];
          if (ii == TS - 1) rr[h] += gs[1][jj + TS * k];
          if (jj == 0) rr[h] += gs[2][ii + TS * k];
          if (jj == TS - 1) rr[h] += gs[3][ii + TS * k];
          if (k == 0) rr[h] += gs[4][ii + TS * jj];
          if (k == TS - 1) rr[h] += gs[5][ii + TS * jj];
        }
#pragma unroll
        for (int c = 0; c < 2; c++) {
          const bool h1 = dxof(c, sl) == 1;
          I[c][sl] = h1 ? ivv[1] : ivv[0];
          R[c][sl] = h1 ? rr[1] : rr[0];
          xv[c][sl] = h1 ? xx[1] : xx[0];
          Cxo[c][sl] = h1 ? cxo[1] : cxo[0];
          Cym[c][sl] = h1 ? cym[1] : cym[0];
          Cyp[c][sl] = h1 ? cyp[1] : cyp[0];
          Czo[c][sl] = h1 ? czo[1] : czo[0];
        }
      }
    }
    // 3: red-black sweeps (colour compile-time so the arrays stay in registers)
    auto half = [&](auto cc) {
      constexpr int c = decltype(cc)::value;
#pragma unroll
      for (int sl = 0; sl < 2; sl++) {
        const int dx = dxof(c, sl);
        const int e = eb + dx + XP * sl;
        // the x-neighbour of the other colour inside the pair is ours; the
        // one beyond is read (out-of-tile reads have zero coupling and stay
        // inside shared memory: guard band, pads, adjacent arrays)
        const float xo = X[dx ? e + 1 : e - 1], xs = xv[1 - c][sl];
        // z: plane 2kp reads z-1 and owns z+1; plane 2kp+1 the reverse
        const float zo = X[sl ? e + XP : e - XP], zs = xv[1 - c][1 - sl];
        const float czs = dx ? Czp[1] : Czp[0];
        // terms in the order x-, x+, y-, y+, z-, z+
        float S = R[c][sl];
        S = fmaf(dx ? Cxp[sl] : Cxo[c][sl], dx ? xs : xo, S);
        S = fmaf(dx ? Cxo[c][sl] : Cxp[sl], dx ? xo : xs, S);
        S = fmaf(Cym[c][sl], X[e - TS], S);
        S = fmaf(Cyp[c][sl], X[e + TS], S);
        if (sl) {
          S = fmaf(czs, zs, S);
          S = fmaf(Czo[c][sl], zo, S);
        } else {
          S = fmaf(Czo[c][sl], zo, S);
          S = fmaf(czs, zs, S);
        }
        xv[c][sl] = S * I[c][sl];
        X[e] = xv[c][sl];
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
    // 4: the tile leaves from the registers: each thread stores its two
    // x pairs (a warp writes four full 64-byte rows)
    {
      VT* xg = x + rc.off + 2 * ip + TS * jj + TS * TS * 2 * kp;
#pragma unroll
      for (int sl = 0; sl < 2; sl++) {
        const bool c1lo = dxof(1, sl) == 0;  // colour 1 holds the even cell
        const float lo = c1lo ? xv[1][sl] : xv[0][sl], hi = c1lo ? xv[0][sl] : xv[1][sl];
        store2(xg + TS * TS * sl, lo, hi);
      }
      // the tile's own x faces, read back from the stage (final after the
      // last half sweep's barrier) so each warp writes whole lines
      if (xf && tid < 2 * TS * TS) {
        const int side = tid >> 8, c = tid & 255;
        xf[xface_slot(rc.off, side, 0, 0) + c] =
            from_f<VT>(X[xpad(side * (TS - 1) + TS * c)]);
      }
    }
    // 5: next tile's arrays landed -> its halo sums
    if (hasNext) {
      if (!__syncthreads_and(mbar_wait(&bar[u], ((n + 1) >> 1) & 1))) {
        if (tid == 0) atomicExch(err, 1);
        mbar_wait(&bar[u], ((n + 1) >> 1) & 1);  // bounded: copies in flight
        return;
      }
      halo_combine(rn, tileBase + tn, u);
    }
    __syncthreads();  // stage s, gsb[s] and record slot n%3 are free again
  }
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
                   double* __restrict__ partial, int* __restrict__ err,
                   const VT* __restrict__ xf) {
  using namespace pipe;
  constexpr int ZC = TS / (NTH / (TS * TS));  // cells of a thread's z column
  constexpr int NHALO = 6 * TS * TS;
  constexpr int HQ = (NHALO + NTH - 1) / NTH;
  constexpr int NVEC = MODE == APPLY_RESIDUAL ? 2 : 1;  // x, [b]
  extern __shared__ __align__(128) float sm[];
  auto stage = [&](int i) { return sm + GUARD + i * 6 * N; };
  float(*gsb)[6][TS * TS] = reinterpret_cast<float(*)[6][TS * TS]>(sm + GUARD + 12 * N);
  TileRec* recs = reinterpret_cast<TileRec*>(sm + ZERO_FLOATS);
  uint64_t* bar = reinterpret_cast<uint64_t*>(recs + 3);
  __shared__ int cmap[2][6];  // coarse tile, ox, oy, oz, aggregated, coarse ts
  const TileRec* grec = reinterpret_cast<const TileRec*>(L.tileRec) + tileBase;
  const int tid = threadIdx.x;
  const int G = gridDim.x;
  int t = blockIdx.x;
  double acc = 0;
  // one issuing thread (lane 0 of its own warp) per copy: x, [b], a_ii,
  // cx, cy, cz, record; the stage barrier counts one arrival each
  constexpr int NISS = NVEC + 5;
  if (t < count) {
    if (tid == 0) {
      mbar_init(&bar[0], NISS);
      mbar_init(&bar[1], NISS);
      mbar_init(&bar[2], 1);
      fence_mbar_init();
    }
    __syncthreads();
    // stage arrays: 0 x, 1 b (residual), 2 a_ii, 3..5 couplings
    auto issue_arrays = [&](const TileRec& r, float* st, uint64_t* br, int tRec, int slot) {
      const int w = tid >> 5;
      if ((tid & 31) != 0 || w >= NISS) return;
      fence_proxy_async();
      const int64_t off = r.off;
      if (w == NISS - 1) {
        const bool rec = tRec < count;
        mbar_expect_tx(br, rec ? sizeof(TileRec) : 0);
        if (rec) bulk_g2s(&recs[slot], grec + tRec, sizeof(TileRec), br);
        return;
      }
      const int a = w < NVEC ? w : w - NVEC + 2;  // array index 0..5
      const void* src;
      void* dst;
      uint32_t bytes = N * sizeof(float);
      switch (a) {
        case 0: src = x + off; dst = raw_x<VT>(st); bytes = N * sizeof(VT); break;
        case 1: src = b + off; dst = raw_b<VT>(st); bytes = N * sizeof(VT); break;
        case 2: src = L.diag + off; dst = st + 2 * N; break;
        case 3: src = L.cx + off; dst = st + 3 * N; break;
        case 4: src = L.cy + off; dst = st + 4 * N; break;
        default: src = L.cz + off; dst = st + 5 * N; break;
      }
      mbar_expect_tx(br, bytes);
      bulk_g2s(dst, src, bytes, br);
    };
    VT hx[HQ];
    float hc[HQ];
    const VT* xfr = L.cxf ? xf : nullptr;
    auto halo_issue = [&](const TileRec& r, int ti, int u) {
#pragma unroll
      for (int q = 0; q < HQ; q++) {
        const int g = tid + NTH * q, f = g >> 8, c = g & 255;
        if (NHALO % NTH == 0 || g < NHALO)
          halo_load(L, x, xfr, r.f[f], f >> 1, f & 1, c & 15, c >> 4, hx[q], hc[q]);
      }
      if (MODE == APPLY_RESIDUAL && tid < 6) cmap[u][tid] = L.toCoarse[(size_t)ti * 6 + tid];
    };
    auto halo_combine = [&](const TileRec& r, int ti, int u) {
      widen_x<VT, NTH>(stage(u), tid);
      const float* st = stage(u);
#pragma unroll
      for (int q = 0; q < HQ; q++) {
        const int g = tid + NTH * q, f = g >> 8, c = g & 255;
        if (NHALO % NTH != 0 && g >= NHALO) continue;
        const int dir = f >> 1, side = f & 1, a = c & 15, bb = c >> 4;
        const int kind = r.f[f].kind;
        float v = 0.f;
        if (kind == FACE_SAME) {
          const float cown = st[(3 + dir) * N + plane_idx(TS, dir, 0, a, bb)];
          v = (side ? hc[q] : cown) * to_f(hx[q]);
        } else if (kind == FACE_COARSER) {
          v = hc[q] * to_f(hx[q]);
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
      issue_arrays(recs[0], stage(0), &bar[0], t + G, 1);
      halo_issue(recs[0], tileBase + t, 0);
      ok = __syncthreads_and(mbar_wait(&bar[0], 0));
      if (!ok) mbar_wait(&bar[0], 0);
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
        issue_arrays(rn, stage(u), &bar[u], tn + G, (n + 2) % 3);
        halo_issue(rn, tileBase + tn, u);
      }
      float* X = stage(s);
      const VT* B = raw_b<VT>(X);
      const float* D = X + 2 * N;
      const float* CX = X + 3 * N;
      const float* CY = X + 4 * N;
      const float* CZ = X + 5 * N;
      const float(*gs)[TS * TS] = gsb[s];
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
      if (MODE == APPLY_MATVEC) {
        // q leaves from the registers (a warp writes two full 64-byte rows)
#pragma unroll
        for (int kk = 0; kk < ZC; kk++) y[rc.off + tidx(TS, i, j, k0 + kk)] = from_f<VT>(yv[kk]);
      } else {
        // the restriction from the registers: a warp holds rows j, j+1 of 16
        // cells, so the x and y partners of a 2 x 2 x 2 group are lanes ^1
        // and ^16, and the z partner the thread's next value; the sum keeps
        // the order x, then y, then z of the group's eight cells
        static_assert(ZC % 2 == 0 && NTH / (TS * TS) * ZC == TS, "z pairs inside a thread");
        const int* tc = cmap[s];
        const int ct = tc[0];
        if (ct >= 0) {
          VC* dst = bc + coarseOff[ct];
          const int ox = tc[1], oy = tc[2], oz = tc[3], cts = tc[5];
          if (tc[4]) {
#pragma unroll
            for (int zz = 0; zz < ZC; zz += 2) {
              const float a000 = yv[zz], a001 = yv[zz + 1];
              const float a100 = __shfl_xor_sync(0xffffffffu, a000, 1);
              const float a101 = __shfl_xor_sync(0xffffffffu, a001, 1);
              const float a010 = __shfl_xor_sync(0xffffffffu, a000, 16);
              const float a011 = __shfl_xor_sync(0xffffffffu, a001, 16);
              const float a110 = __shfl_xor_sync(0xffffffffu, a100, 16);
              const float a111 = __shfl_xor_sync(0xffffffffu, a101, 16);
              if (!(i & 1) && !(j & 1)) {
                const float sum = a000 + a100 + a010 + a110 + a001 + a101 + a011 + a111;
                dst[tidx(cts, ox + (i >> 1), oy + (j >> 1), oz + ((k0 + zz) >> 1))] =
                    from_f<VC>(sum);
              }
            }
          } else {
#pragma unroll
            for (int kk = 0; kk < ZC; kk++)
              dst[tidx(cts, ox + i, oy + j, oz + k0 + kk)] = from_f<VC>(yv[kk]);
          }
        }
      }
      if (hasNext) {
        if (!__syncthreads_and(mbar_wait(&bar[u], ((n + 1) >> 1) & 1))) {
          if (tid == 0) atomicExch(err, 1);
          mbar_wait(&bar[u], ((n + 1) >> 1) & 1);  // bounded: copies in flight
          break;
        }
        halo_combine(rn, tileBase + tn, u);
      }
      __syncthreads();
    }
  }
  if (MODE == APPLY_MATVEC && partial) {
    acc = block_sum(acc);
    if (tid == 0) partial[blockIdx.x] = acc;
  }
}
