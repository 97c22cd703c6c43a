// Host construction of the pressure multigrid hierarchy.
//
// MG level 0 is the reference's discretisation of the FLIP pressure equation
// on the adaptive block grid (src/msbg3.cpp:564-1044 for the ghost couplings,
// src/msbg3.cpp:2586-2779 for the diagonal), in finite-volume form:
//   coupling across a same-level face of cells of edge h   = h * beta
//   coupling across a fine(h)/coarse(2h) interface face    = (2/3) * h * beta
//       (DPMR_GRAD_COEFF_FC, src/msbg.h:82-87; the reference's procNeighMixedRes2
//        builds the same 2/3 weight, src/msbg3.cpp:59-161)
//   a_ii = sum of the couplings of all faces of cell i (neighbours that are
//       air/outside act as p = 0, solid faces have beta = 0)
//   b_i  = rhs * h^3 (volume integral)
// The diagonal differs from the reference only at level interfaces, where the
// reference drops the interface coupling from a_ii and the resulting matrix is
// not an M-matrix (see the design notes); here A is symmetric positive
// definite.  Coarse MG levels are exact Galerkin products A_c = P^T A P with
// piecewise-constant P over the liquid children, the same 2x2x2 aggregation
// the reference's restriction uses (src/msbg4.cpp:1512-1914), on the block
// hierarchy level(b, m) = max(map(b), m) of the reference (src/msbg.cpp:1650).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <numeric>
#include <string>
#include <map>
#include <memory>
#include <tuple>

#include "build_gpu.h"
#include "pressure.h"

namespace msbg {
namespace ps {
namespace {

constexpr uint16_t CELL_NONFLUID = 0x1 | 0x2 | 0x1000;  // SOLID | FIXED | VOID
constexpr uint16_t CELL_SOLID_BIT = 0x1;

int pow2_divisor(int v, int cap) {
  int p = 1;
  while (p < cap && v % (p * 2) == 0) p *= 2;
  return p;
}

struct Ctx {
  Hierarchy& H;
  const msbg_pressure_callbacks* cb = nullptr;
  // per-cell arrays of MG level 0 instead of callbacks (the bulk prepare):
  // first cell of each block, log2(bsx0)
  const ArrayInput* arr = nullptr;
  std::vector<int64_t> boff;
  int sh0 = 0;
  int maxMap = 0;
  explicit Ctx(Hierarchy& h) : H(h) {}

  // packed array cell holding fine voxel (x, y, z), inside the domain
  int64_t cell(int x, int y, int z) const {
    const int64_t b = (x >> sh0) + (int64_t)H.nb1x * ((y >> sh0) + (int64_t)H.nb1y * (z >> sh0));
    const int l = H.blockLevel[b], lsh = sh0 - l, m = (1 << sh0) - 1;
    return boff[b] + ((x & m) >> l) + ((int64_t)((y & m) >> l) << lsh) +
           ((int64_t)((z & m) >> l) << (2 * lsh));
  }
  // packed array cell of the first cell of tile t (a tile lies in one block),
  // and the block's edge in cells of the tile's level
  int64_t tile_cell0(const Tile& t, int& bs) const {
    const int l = t.level;
    const int64_t b = ((t.ox << l) >> sh0) +
                      (int64_t)H.nb1x * (((t.oy << l) >> sh0) + (int64_t)H.nb1y * ((t.oz << l) >> sh0));
    bs = H.bsx0 >> l;
    const int m = bs - 1;
    return boff[b] + (t.ox & m) + (int64_t)bs * ((t.oy & m) + (int64_t)bs * (t.oz & m));
  }
  // The scene at fine voxel (x, y, z): from the callbacks, or from the arrays
  // (outside the domain: solid, no face, no right-hand side).
  uint16_t cell_type(int x, int y, int z) const {
    if (!arr) return cb->sampleCellType(cb->user, x, y, z);
    return inside(x, y, z) ? arr->flags[cell(x, y, z)] : (uint16_t)0x1;
  }
  float face(int dir, int x, int y, int z) const {
    if (!arr) return cb->sampleFaceCoeff(cb->user, dir, x, y, z);
    return inside(x, y, z) ? arr->face[dir][cell(x, y, z)] : 0.f;
  }
  float rhs(int x, int y, int z) const {
    if (!arr) return cb->sampleRhs(cb->user, x, y, z);
    return inside(x, y, z) && arr->rhs ? arr->rhs[cell(x, y, z)] : 0.f;
  }

  // level of the fine-voxel region (fx,fy,fz) at MG level m
  int level_at(int m, int fx, int fy, int fz) const {
    int b = (fx >> sh0) + H.nb1x * ((fy >> sh0) + H.nb1y * (fz >> sh0));
    return std::max(H.blockLevel[b], m);
  }
  bool inside(int fx, int fy, int fz) const {
    return fx >= 0 && fy >= 0 && fz >= 0 && fx < H.sx && fy < H.sy && fz < H.sz;
  }
  bool uniform(int m) const { return m >= maxMap; }
  int ts_of(int m, int l) const {
    if (uniform(m))
      return pow2_divisor(std::gcd(std::gcd(H.sx >> l, H.sy >> l), H.sz >> l), TS_MAX);
    return std::min(TS_MAX, H.bsx0 >> l);
  }
};

inline void face_axes(int dir, int& a, int& b) {
  a = dir == 0 ? 1 : 0;
  b = dir == 2 ? 1 : 2;
}

// Tile lookup at resolution level l of MG level m for level-l cell coords.
inline int tile_at(const Level& L, int l, int X, int Y, int Z) {
  if (l < 0 || l >= 32) return -1;
  const int n = L.tmapN[l];
  if (!n || X < 0 || Y < 0 || Z < 0) return -1;
  const int sh = __builtin_ctz(L.tsOf[l]);  // tile edges are powers of two
  int tx = X >> sh, ty = Y >> sh, tz = Z >> sh;
  if (tx >= n || ty >= n || tz >= n) return -1;
  return L.tmap[l][tx + (size_t)n * (ty + (size_t)n * tz)];
}

// Create the candidate tiles of MG level m (regions whose level equals the
// tile's level); fluid filtering happens later.
void enumerate_tiles(const Ctx& C, int m, Level& L, std::vector<Tile>& cand) {
  const Hierarchy& H = C.H;
  std::vector<int> present;
  for (int l = m; l <= std::max(m, C.maxMap); l++) present.push_back(l);
  for (int l : present) {
    if ((H.sx >> l) << l != H.sx || (H.sy >> l) << l != H.sy || (H.sz >> l) << l != H.sz) continue;
    const int ts = C.ts_of(m, l);
    const int nx = (H.sx >> l) / ts, ny = (H.sy >> l) / ts, nz = (H.sz >> l) / ts;
    if (nx <= 0 || ny <= 0 || nz <= 0) continue;
    L.tsOf[l] = ts;
    L.tmapN[l] = std::max({nx, ny, nz});
    const int n = L.tmapN[l];
    L.tmap[l].assign((size_t)n * n * n, -1);
    for (int tz = 0; tz < nz; tz++)
      for (int ty = 0; ty < ny; ty++)
        for (int tx = 0; tx < nx; tx++) {
          const int fx = (tx * ts) << l, fy = (ty * ts) << l, fz = (tz * ts) << l;
          if (C.level_at(m, fx, fy, fz) != l) continue;
          Tile t;
          t.level = l;
          t.ts = ts;
          t.ox = tx * ts;
          t.oy = ty * ts;
          t.oz = tz * ts;
          t.off = 0;
          cand.push_back(t);
        }
  }
}

void register_tiles(Level& L, std::vector<Tile>& tiles) {
  // order by (level, colour) so each smoothing pass is a contiguous range
  std::stable_sort(tiles.begin(), tiles.end(), [&](const Tile& a, const Tile& b) {
    if (a.level != b.level) return a.level < b.level;
    int ca = ((a.ox / a.ts) + (a.oy / a.ts) + (a.oz / a.ts)) & 1;
    int cb = ((b.ox / b.ts) + (b.oy / b.ts) + (b.oz / b.ts)) & 1;
    return ca < cb;
  });
  int64_t off = 0;
  for (auto& t : tiles) {
    t.off = off;
    off += (int64_t)t.ts * t.ts * t.ts;
  }
  L.tiles = tiles;
  L.nCells = off;
  for (size_t i = 0; i < tiles.size(); i++) {
    const Tile& t = tiles[i];
    const int n = L.tmapN[t.level];
    L.tmap[t.level][(t.ox / t.ts) + (size_t)n * ((t.oy / t.ts) + (size_t)n * (t.oz / t.ts))] = (int)i;
  }
  // passes: (level, colour) ranges; groups: by tile size
  L.passes.clear();
  L.passTiles.resize(tiles.size());
  for (size_t i = 0; i < tiles.size(); i++) L.passTiles[i] = (int)i;
  for (size_t i = 0; i < tiles.size();) {
    const Tile& t = tiles[i];
    int col = ((t.ox / t.ts) + (t.oy / t.ts) + (t.oz / t.ts)) & 1;
    size_t j = i;
    while (j < tiles.size() && tiles[j].level == t.level &&
           (((tiles[j].ox / tiles[j].ts) + (tiles[j].oy / tiles[j].ts) + (tiles[j].oz / tiles[j].ts)) & 1) == col)
      j++;
    L.passes.push_back({t.level, col, t.ts, (int)i, (int)(j - i)});
    i = j;
  }
  L.groups.clear();
  L.groupTiles.clear();
  std::map<int, std::vector<int>> byTs;
  for (size_t i = 0; i < tiles.size(); i++) byTs[tiles[i].ts].push_back((int)i);
  for (auto& kv : byTs) {
    L.groups.push_back({kv.first, (int)L.groupTiles.size(), (int)kv.second.size()});
    L.groupTiles.insert(L.groupTiles.end(), kv.second.begin(), kv.second.end());
  }
}

// Face descriptors and interface-plane offsets.
void build_faces(const Ctx& C, Level& L) {
  const int nT = (int)L.tiles.size();
  L.face.assign((size_t)nT * 6 * FACE_INTS, 0);
  L.ifOff.assign((size_t)nT * 6, -1);
  int64_t nIf = 0;
  for (int ti = 0; ti < nT; ti++) {
    const Tile& t = L.tiles[ti];
    const int l = t.level, ts = t.ts;
    const int o[3] = {t.ox, t.oy, t.oz};
    for (int dir = 0; dir < 3; dir++)
      for (int side = 0; side < 2; side++) {
        int* F = &L.face[((size_t)ti * 6 + dir * 2 + side) * FACE_INTS];
        for (int k = 0; k < 4; k++) F[F_T0 + k] = -1;
        F[F_KIND] = FACE_NONE;
        // first fine voxel just outside the face
        int cell[3] = {o[0], o[1], o[2]};
        cell[dir] = side ? o[dir] + ts : o[dir] - 1;
        int fv[3];
        for (int k = 0; k < 3; k++) fv[k] = cell[k] << l;
        if (side == 0) fv[dir] = (o[dir] << l) - 1;
        if (!C.inside(fv[0], fv[1], fv[2])) continue;
        const int l2 = C.level_at(L.m, fv[0], fv[1], fv[2]);
        int ax, bx;
        face_axes(dir, ax, bx);
        if (l2 == l) {
          int nb = tile_at(L, l, cell[0], cell[1], cell[2]);
          if (nb < 0) continue;
          F[F_KIND] = FACE_SAME;
          F[F_T0] = nb;
          F[F_NTS] = ts;
        } else if (l2 == l + 1) {
          int cc[3];
          for (int k = 0; k < 3; k++) cc[k] = fv[k] >> (l + 1);
          int nb = tile_at(L, l + 1, cc[0], cc[1], cc[2]);
          // interface plane is needed for the coupling even if the coarse
          // side holds no liquid (it is zero then; kept for uniformity)
          L.ifOff[(size_t)ti * 6 + dir * 2 + side] = nIf;
          nIf += (int64_t)ts * ts;
          if (nb < 0) continue;
          const Tile& tn = L.tiles[nb];
          const int no[3] = {tn.ox, tn.oy, tn.oz};
          F[F_KIND] = FACE_COARSER;
          F[F_T0] = nb;
          F[F_OA] = (o[ax] >> 1) - no[ax];
          F[F_OB] = (o[bx] >> 1) - no[bx];
          F[F_NTS] = tn.ts;
        } else if (l2 == l - 1) {
          // fine cells just outside, level l-1 coordinates
          const int tsf = L.tsOf[l - 1];
          const int cov = tsf / 2;  // our cells per fine tile along a/b
          const int per = ts / cov;  // fine tiles per axis (1 or 2)
          int fc[3];
          fc[dir] = side ? (o[dir] + ts) * 2 : o[dir] * 2 - 1;
          bool any = false;
          for (int qb = 0; qb < per; qb++)
            for (int qa = 0; qa < per; qa++) {
              fc[ax] = (o[ax] + qa * cov) * 2;
              fc[bx] = (o[bx] + qb * cov) * 2;
              int nb = tile_at(L, l - 1, fc[0], fc[1], fc[2]);
              F[F_T0 + qa + per * qb] = nb;
              any |= nb >= 0;
            }
          if (!any) continue;
          F[F_KIND] = FACE_FINER;
          F[F_COV] = cov;
          F[F_NTS] = tsf;
        }
      }
  }
  L.nIf = nIf;
}

// Fine-side coupling across a face of a level-l cell (h = 2^l) whose
// neighbour region is coarser: (2/3) h beta, beta sampled on the shared face.
inline double interface_coupling(const Ctx& C, int l, int dir, int side, int X, int Y, int Z) {
  int c[3] = {X, Y, Z};
  if (side) c[dir] += 1;
  const double h = (double)(1 << l);
  return (2.0 / 3.0) * h * C.face(dir, c[0] << l, c[1] << l, c[2] << l);
}

// Coupling of level-l cell p across its upper face in dir when the region
// behind it (inside the domain) is at level l2: sample_level0's face_c for
// side 1 on a tile face.
double upper_coupling(const Ctx& C, int l, int l2, int dir, const int p[3]) {
  const double h = (double)(1 << l);
  if (l2 == l) {
    int q[3] = {p[0], p[1], p[2]};
    q[dir] += 1;
    return h * C.face(dir, q[0] << l, q[1] << l, q[2] << l);
  }
  if (l2 == l + 1) return interface_coupling(C, l, dir, 1, p[0], p[1], p[2]);
  int ax, bx;
  face_axes(dir, ax, bx);
  double c = 0;
  for (int u = 0; u < 2; u++)
    for (int v = 0; v < 2; v++) {
      int f[3];
      f[dir] = (p[dir] + 1) * 2;
      f[ax] = p[ax] * 2 + u;
      f[bx] = p[bx] * 2 + v;
      c += interface_coupling(C, l - 1, dir, 0, f[0], f[1], f[2]);
    }
  return c;
}

// Zeroes tile ti's cells of diag, cx, cy, cz (and rhs) and its interface
// planes: the first touch of that memory, by the thread that fills it.
void zero_tile(Level& L, int ti, bool withRhs) {
  const Tile& t = L.tiles[ti];
  const size_t n3 = (size_t)t.ts * t.ts * t.ts;
  std::fill_n(L.diag.begin() + t.off, n3, 0.f);
  std::fill_n(L.cx.begin() + t.off, n3, 0.f);
  std::fill_n(L.cy.begin() + t.off, n3, 0.f);
  std::fill_n(L.cz.begin() + t.off, n3, 0.f);
  if (withRhs) std::fill_n(L.rhs.begin() + t.off, n3, 0.f);
  for (int f = 0; f < 6; f++) {
    const int64_t io = L.ifOff[(size_t)ti * 6 + f];
    if (io >= 0) std::fill_n(L.ifc.begin() + io, (size_t)t.ts * t.ts, 0.f);
  }
}

// Level 0 operator from the callbacks.
void sample_level0(const Ctx& C, Level& L, std::vector<uint8_t>& fluid) {
  const int nT = (int)L.tiles.size();
  // allocated untouched; each tile zeroes its own cells and interface planes
  L.diag.resize(L.nCells);
  L.cx.resize(L.nCells);
  L.cy.resize(L.nCells);
  L.cz.resize(L.nCells);
  L.rhs.resize(L.nCells);
  L.ifc.resize(L.nIf);
#pragma omp parallel for schedule(dynamic, 1)
  for (int ti = 0; ti < nT; ti++) {
    const Tile& t = L.tiles[ti];
    const int l = t.level, ts = t.ts;
    const double h = (double)(1 << l);
    zero_tile(L, ti, true);
    float* cdir[3] = {&L.cx[t.off], &L.cy[t.off], &L.cz[t.off]};
    // Across a tile face the neighbour region (and whether it is inside the
    // domain) is the same for every cell: a tile face lies within one block
    // face.  Resolve it once per face; interior neighbours are this level.
    int faceLevel[3][2];
    bool faceInside[3][2];
    for (int dir = 0; dir < 3; dir++)
      for (int side = 0; side < 2; side++) {
        int fv[3] = {t.ox << l, t.oy << l, t.oz << l};
        const int pd = side ? (dir == 0 ? t.ox : dir == 1 ? t.oy : t.oz) + ts - 1
                            : (dir == 0 ? t.ox : dir == 1 ? t.oy : t.oz);
        fv[dir] = side ? (pd + 1) << l : (pd << l) - 1;
        faceInside[dir][side] = C.inside(fv[0], fv[1], fv[2]);
        faceLevel[dir][side] = faceInside[dir][side] ? C.level_at(L.m, fv[0], fv[1], fv[2]) : -1;
      }
    // coupling of cell (i,j,k) across face (dir, side); records the interface
    // couplings and, for lower faces to the same level, the face array
    auto face_c = [&](int i, int j, int k, int dir, int side) -> double {
      const int64_t ci = i + (int64_t)ts * (j + (int64_t)ts * k);
      const int X = t.ox + i, Y = t.oy + j, Z = t.oz + k;
      const int p[3] = {X, Y, Z}, loc[3] = {i, j, k};
      const bool onTileFace = side ? loc[dir] == ts - 1 : loc[dir] == 0;
      int q[3] = {p[0], p[1], p[2]};
      if (side) q[dir] += 1;
      double c;
      if (onTileFace && !faceInside[dir][side]) {
        // the domain boundary, p = 0 outside behind the coupling c: a wall
        // has none; an open face has the callback's coefficient on the lower
        // side and the constant 1 of the reference's open-face weights
        // (constFaceCoeffAirBlock, src/msbg3.cpp:733-740) on the upper side;
        // without a spec, the reference's operator (DBC_REFERENCE)
        const int bc = C.H.domainBc[2 * dir + side];
        if (bc == MSBG_DBC_SOLID || (bc == DBC_REFERENCE && side == 1))
          c = 0.0;
        else if (side == 1)
          c = h;
        else
          c = h * C.face(dir, q[0] << l, q[1] << l, q[2] << l);
        if (side == 0) cdir[dir][ci] = (float)c;
        return c;
      }
      const int l2 = onTileFace ? faceLevel[dir][side] : l;
      if (l2 == l) {
        c = h * C.face(dir, q[0] << l, q[1] << l, q[2] << l);
        if (side == 0) cdir[dir][ci] = (float)c;
      } else if (l2 == l + 1) {
        c = interface_coupling(C, l, dir, side, X, Y, Z);
        int64_t io = L.ifOff[(size_t)ti * 6 + dir * 2 + side];
        int ax, bx;
        face_axes(dir, ax, bx);
        if (io >= 0) L.ifc[io + loc[ax] + (int64_t)ts * loc[bx]] = (float)c;
      } else {
        // finer neighbours: 4 fine cells share this face
        int ax, bx;
        face_axes(dir, ax, bx);
        c = 0;
        for (int u = 0; u < 2; u++)
          for (int v = 0; v < 2; v++) {
            int f[3];
            f[dir] = side ? (p[dir] + 1) * 2 : p[dir] * 2 - 1;
            f[ax] = p[ax] * 2 + u;
            f[bx] = p[bx] * 2 + v;
            c += interface_coupling(C, l - 1, dir, 1 - side, f[0], f[1], f[2]);
          }
      }
      return c;
    };
    // pass 1: lower faces (each interior face once); pass 2: upper faces,
    // which inside the tile are the next cell's lower faces
    const size_t n3 = (size_t)ts * ts * ts;
    thread_local std::vector<double> low;  // reused across this thread's tiles
    if (low.size() < 3 * n3) low.resize(3 * n3);
    // with arrays, a lower face inside the tile is the cell's own entry
    int pbs = 0;
    const int64_t pc0 = C.arr ? C.tile_cell0(t, pbs) : 0;
    const float* const* af = C.arr ? C.arr->face : nullptr;
    for (int k = 0; k < ts; k++)
      for (int j = 0; j < ts; j++)
        for (int i = 0; i < ts; i++) {
          const int64_t ci = i + (int64_t)ts * (j + (int64_t)ts * k);
          const int64_t pc = pc0 + i + (int64_t)pbs * (j + (int64_t)pbs * k);
          const int loc[3] = {i, j, k};
          for (int dir = 0; dir < 3; dir++) {
            if (af && loc[dir] > 0) {
              const double c = h * af[dir][pc];
              low[dir * n3 + ci] = c;
              cdir[dir][ci] = (float)c;
            } else {
              low[dir * n3 + ci] = face_c(i, j, k, dir, 0);
            }
          }
        }
    const int64_t stride[3] = {1, ts, (int64_t)ts * ts};
    for (int k = 0; k < ts; k++)
      for (int j = 0; j < ts; j++)
        for (int i = 0; i < ts; i++) {
          const int64_t ci = i + (int64_t)ts * (j + (int64_t)ts * k);
          const int loc[3] = {i, j, k};
          const bool isFluid = !fluid.empty() ? fluid[t.off + ci] : false;
          double diag = 0;
          for (int dir = 0; dir < 3; dir++) {
            diag += low[dir * n3 + ci];
            diag += loc[dir] < ts - 1 ? low[dir * n3 + ci + stride[dir]] : face_c(i, j, k, dir, 1);
          }
          if (isFluid) {
            const int X = t.ox + i, Y = t.oy + j, Z = t.oz + k;
            L.diag[t.off + ci] = (float)diag;
            const double r =
                C.arr ? (C.arr->rhs ? C.arr->rhs[pc0 + i + (int64_t)pbs * (j + (int64_t)pbs * k)]
                                    : 0.f)
                      : C.rhs(X << l, Y << l, Z << l);
            L.rhs[t.off + ci] = (float)(r * h * h * h);
          }
        }
  }
}

// Exact Galerkin coarsening: level m (fine) -> level m+1 (coarse).
// fineFluid/coarseFluid: per-cell liquid flags.
void galerkin(const Ctx& C, const Level& F, const std::vector<uint8_t>& fineFluid, Level& G,
              const std::vector<uint8_t>& coarseFluid) {
  const int nT = (int)G.tiles.size();
  // allocated untouched; each tile zeroes its own cells and interface planes
  G.diag.resize(G.nCells);
  G.cx.resize(G.nCells);
  G.cy.resize(G.nCells);
  G.cz.resize(G.nCells);
  G.ifc.resize(G.nIf);
  // fine cell lookup: (level, cell coords) -> global fine cell index or -1
  auto fine_cell = [&](int l, int X, int Y, int Z) -> int64_t {
    int t = tile_at(F, l, X, Y, Z);
    if (t < 0) return -1;
    const Tile& ft = F.tiles[t];
    return ft.off + (X - ft.ox) + (int64_t)ft.ts * ((Y - ft.oy) + (int64_t)ft.ts * (Z - ft.oz));
  };
  auto fine_fluid = [&](int64_t c) { return c >= 0 && fineFluid[c]; };
  // coupling between fine cell c (level l, coords p) and its neighbour across
  // face (dir, side), if both are liquid; 0 otherwise.
  auto fine_pair = [&](int l, const int p[3], int dir, int side) -> double {
    int64_t c0 = fine_cell(l, p[0], p[1], p[2]);
    if (!fine_fluid(c0)) return 0;
    int fv[3] = {p[0] << l, p[1] << l, p[2] << l};
    fv[dir] = side ? (p[dir] + 1) << l : (p[dir] << l) - 1;
    if (!C.inside(fv[0], fv[1], fv[2])) return 0;
    const int l2 = C.level_at(F.m, fv[0], fv[1], fv[2]);
    if (l2 == l) {
      int q[3] = {p[0], p[1], p[2]};
      q[dir] += side ? 1 : -1;
      int64_t c1 = fine_cell(l, q[0], q[1], q[2]);
      if (!fine_fluid(c1)) return 0;
      const float* cd = dir == 0 ? F.cx.data() : dir == 1 ? F.cy.data() : F.cz.data();
      return side ? cd[c1] : cd[c0];
    }
    if (l2 == l + 1) {
      int cc[3];
      for (int k = 0; k < 3; k++) cc[k] = fv[k] >> (l + 1);
      int64_t c1 = fine_cell(l + 1, cc[0], cc[1], cc[2]);
      if (!fine_fluid(c1)) return 0;
      int t = tile_at(F, l, p[0], p[1], p[2]);
      const Tile& ft = F.tiles[t];
      int64_t io = F.ifOff[(size_t)t * 6 + dir * 2 + side];
      int ax, bx;
      face_axes(dir, ax, bx);
      const int loc[3] = {p[0] - ft.ox, p[1] - ft.oy, p[2] - ft.oz};
      return io >= 0 ? F.ifc[io + loc[ax] + (int64_t)ft.ts * loc[bx]] : 0.0;
    }
    // finer neighbour: sum over the 4 fine cells facing us
    int ax, bx;
    face_axes(dir, ax, bx);
    double s = 0;
    for (int u = 0; u < 2; u++)
      for (int v = 0; v < 2; v++) {
        int f[3];
        f[dir] = side ? (p[dir] + 1) * 2 : p[dir] * 2 - 1;
        f[ax] = p[ax] * 2 + u;
        f[bx] = p[bx] * 2 + v;
        int64_t c1 = fine_cell(l - 1, f[0], f[1], f[2]);
        if (!fine_fluid(c1)) continue;
        int t = tile_at(F, l - 1, f[0], f[1], f[2]);
        const Tile& ft = F.tiles[t];
        int64_t io = F.ifOff[(size_t)t * 6 + dir * 2 + (1 - side)];
        const int loc[3] = {f[0] - ft.ox, f[1] - ft.oy, f[2] - ft.oz};
        if (io >= 0) s += F.ifc[io + loc[ax] + (int64_t)ft.ts * loc[bx]];
      }
    return s;
  };
  // is the coarse cell (level lc, coords P) an aggregate of level lc-1 cells?
  auto aggregated = [&](int lc, const int P[3]) {
    int fv[3] = {P[0] << lc, P[1] << lc, P[2] << lc};
    return C.level_at(F.m, fv[0], fv[1], fv[2]) == lc - 1;
  };
  // coupling between coarse cell P and its neighbour across (dir, side):
  // sum of the fine liquid pairs across that coarse face.
  auto coarse_face = [&](int lc, const int P[3], int dir, int side) -> double {
    if (!aggregated(lc, P)) return fine_pair(lc, P, dir, side);
    int ax, bx;
    face_axes(dir, ax, bx);
    double s = 0;
    for (int u = 0; u < 2; u++)
      for (int v = 0; v < 2; v++) {
        int f[3];
        f[dir] = P[dir] * 2 + side;
        f[ax] = P[ax] * 2 + u;
        f[bx] = P[bx] * 2 + v;
        s += fine_pair(lc - 1, f, dir, side);
      }
    return s;
  };
#pragma omp parallel for schedule(dynamic, 1)
  for (int ti = 0; ti < nT; ti++) {
    const Tile& t = G.tiles[ti];
    const int lc = t.level, ts = t.ts;
    zero_tile(G, ti, false);
    float* cdir[3] = {&G.cx[t.off], &G.cy[t.off], &G.cz[t.off]};
    // Fast path of a tile whose cells all aggregate: its children fill a
    // fine region of (2 ts)^3 cells at level lc-1 covered by whole fine tiles,
    // resolved once.  A tile of a uniform level spans several blocks, which
    // may aggregate or not; such a tile takes the per-cell path.
    bool aggT = true;
    {
      const int ext = t.ts << lc, o[3] = {t.ox << lc, t.oy << lc, t.oz << lc};
      const int step = std::min(ext, C.H.bsx0);
      for (int z = o[2]; z < o[2] + ext && aggT; z += step)
        for (int y = o[1]; y < o[1] + ext && aggT; y += step)
          for (int x = o[0]; x < o[0] + ext && aggT; x += step)
            aggT = C.level_at(F.m, x, y, z) == lc - 1;
    }
    const int tsf = aggT ? F.tsOf[lc - 1] : 0;
    const int nsub = aggT && tsf > 0 ? (2 * ts) / tsf : 0;
    int64_t subOff[64];
    bool fast = aggT && tsf > 0 && nsub * tsf == 2 * ts && nsub * nsub * nsub <= 64;
    for (int sz = 0; fast && sz < nsub; sz++)
      for (int sy = 0; sy < nsub; sy++)
        for (int sx = 0; sx < nsub; sx++) {
          const int ft = tile_at(F, lc - 1, 2 * t.ox + sx * tsf, 2 * t.oy + sy * tsf,
                                 2 * t.oz + sz * tsf);
          subOff[sx + nsub * (sy + nsub * sz)] = ft >= 0 ? F.tiles[ft].off : -1;
        }
    // fine cell of region coords (x, y, z) in [0, 2 ts), or -1
    const int fsh = tsf > 0 ? __builtin_ctz(tsf) : 0, fm = tsf - 1;  // tsf is a power of two
    auto fidx = [&](int x, int y, int z) -> int64_t {
      const int64_t o = subOff[(x >> fsh) + nsub * ((y >> fsh) + nsub * (z >> fsh))];
      if (o < 0) return -1;
      return o + (x & fm) + ((int64_t)(y & fm) << fsh) + ((int64_t)(z & fm) << (2 * fsh));
    };
    const float* fcd[3] = {F.cx.data(), F.cy.data(), F.cz.data()};
    for (int k = 0; k < ts; k++)
      for (int j = 0; j < ts; j++)
        for (int i = 0; i < ts; i++) {
          const int64_t ci = i + (int64_t)ts * (j + (int64_t)ts * k);
          const int P[3] = {t.ox + i, t.oy + j, t.oz + k};
          const int loc[3] = {i, j, k};
          if (!coarseFluid[t.off + ci]) continue;
          if (fast) {
            // children, their diagonal and internal pairs
            int64_t ch[8];
            for (int c = 0; c < 8; c++) {
              const int64_t fc = fidx(2 * i + (c & 1), 2 * j + ((c >> 1) & 1), 2 * k + (c >> 2));
              ch[c] = fine_fluid(fc) ? fc : -1;
            }
            double d = 0;
            for (int c = 0; c < 8; c++) {
              if (ch[c] < 0) continue;
              d += F.diag[ch[c]];
              for (int dir = 0; dir < 3; dir++)
                if ((c >> dir) & 1)
                  if (ch[c ^ (1 << dir)] >= 0) d -= 2.0 * fcd[dir][ch[c]];
            }
            G.diag[t.off + ci] = (float)d;
            // lower faces inside the tile: 4 fine pairs each
            for (int dir = 0; dir < 3; dir++) {
              if (loc[dir] == 0) continue;  // tile face: generic path below
              double cs = 0;
              for (int c = 0; c < 8; c++) {
                if ((c >> dir) & 1 || ch[c] < 0) continue;  // lower children of P
                int f[3] = {2 * i + (c & 1), 2 * j + ((c >> 1) & 1), 2 * k + (c >> 2)};
                f[dir] -= 1;
                if (fine_fluid(fidx(f[0], f[1], f[2]))) cs += fcd[dir][ch[c]];
              }
              cdir[dir][ci] = (float)cs;
            }
            // tile faces (same level, lower side) and level interfaces
            for (int dir = 0; dir < 3; dir++)
              for (int side = 0; side < 2; side++) {
                const bool onFace = side ? loc[dir] == ts - 1 : loc[dir] == 0;
                if (!onFace) continue;
                int fv[3] = {P[0] << lc, P[1] << lc, P[2] << lc};
                fv[dir] = side ? (P[dir] + 1) << lc : (P[dir] << lc) - 1;
                if (!C.inside(fv[0], fv[1], fv[2])) continue;
                const int l2 = C.level_at(G.m, fv[0], fv[1], fv[2]);
                if (l2 == lc && side == 0) {
                  cdir[dir][ci] = (float)coarse_face(lc, P, dir, side);
                } else if (l2 == lc + 1) {
                  int64_t io = G.ifOff[(size_t)ti * 6 + dir * 2 + side];
                  if (io >= 0) {
                    int ax, bx;
                    face_axes(dir, ax, bx);
                    G.ifc[io + loc[ax] + (int64_t)ts * loc[bx]] =
                        (float)coarse_face(lc, P, dir, side);
                  }
                }
              }
            continue;
          }
          // diagonal
          double d = 0;
          if (aggregated(lc, P)) {
            for (int c = 0; c < 8; c++) {
              int f[3] = {P[0] * 2 + (c & 1), P[1] * 2 + ((c >> 1) & 1), P[2] * 2 + (c >> 2)};
              int64_t fc = fine_cell(lc - 1, f[0], f[1], f[2]);
              if (!fine_fluid(fc)) continue;
              d += F.diag[fc];
              // internal pairs: count each once (the upper child of each pair)
              for (int dir = 0; dir < 3; dir++) {
                const int bit = dir == 0 ? (c & 1) : dir == 1 ? ((c >> 1) & 1) : (c >> 2);
                if (bit) d -= 2.0 * fine_pair(lc - 1, f, dir, 0);
              }
            }
          } else {
            int64_t fc = fine_cell(lc, P[0], P[1], P[2]);
            d = F.diag[fc];
          }
          G.diag[t.off + ci] = (float)d;
          // couplings on the lower faces / interface planes
          for (int dir = 0; dir < 3; dir++)
            for (int side = 0; side < 2; side++) {
              int fv[3] = {P[0] << lc, P[1] << lc, P[2] << lc};
              fv[dir] = side ? (P[dir] + 1) << lc : (P[dir] << lc) - 1;
              if (!C.inside(fv[0], fv[1], fv[2])) continue;
              const int l2 = C.level_at(G.m, fv[0], fv[1], fv[2]);
              if (l2 == lc && side == 0) {
                cdir[dir][ci] = (float)coarse_face(lc, P, dir, side);
              } else if (l2 == lc + 1) {
                const bool onFace = side ? loc[dir] == ts - 1 : loc[dir] == 0;
                int64_t io = G.ifOff[(size_t)ti * 6 + dir * 2 + side];
                if (onFace && io >= 0) {
                  int ax, bx;
                  face_axes(dir, ax, bx);
                  G.ifc[io + loc[ax] + (int64_t)ts * loc[bx]] = (float)coarse_face(lc, P, dir, side);
                }
              }
            }
        }
  }
}

// Coarse tile of every fine tile: (coarse tile, offset x,y,z in coarse cells, aggregated).
void build_restriction(const Ctx& C, Level& F, const Level& G) {
  F.toCoarse.assign(F.tiles.size() * 6, -1);
  for (size_t ti = 0; ti < F.tiles.size(); ti++) {
    const Tile& t = F.tiles[ti];
    const int fv[3] = {t.ox << t.level, t.oy << t.level, t.oz << t.level};
    const int lc = C.level_at(G.m, fv[0], fv[1], fv[2]);
    const bool agg = lc == t.level + 1;
    const int sh = agg ? 1 : 0;
    int P[3] = {t.ox >> sh, t.oy >> sh, t.oz >> sh};
    int ct = tile_at(G, lc, P[0], P[1], P[2]);
    int* r = &F.toCoarse[ti * 6];
    r[0] = ct;
    if (ct >= 0) {
      const Tile& g = G.tiles[ct];
      r[1] = P[0] - g.ox;
      r[2] = P[1] - g.oy;
      r[3] = P[2] - g.oz;
    }
    r[4] = agg ? 1 : 0;
    r[5] = ct >= 0 ? G.tiles[ct].ts : 0;
  }
}

// Cholesky of a dense SPD matrix (lower), then its inverse.  Returns false if
// the matrix is not positive definite.
bool dense_spd_inverse(std::vector<double>& A, int n, std::vector<double>& inv) {
  std::vector<double> Lm(A);
  for (int j = 0; j < n; j++) {
    double s = Lm[(size_t)j * n + j];
    for (int k = 0; k < j; k++) s -= Lm[(size_t)j * n + k] * Lm[(size_t)j * n + k];
    if (!(s > 0)) return false;
    const double d = std::sqrt(s);
    Lm[(size_t)j * n + j] = d;
    for (int i = j + 1; i < n; i++) {
      double v = Lm[(size_t)i * n + j];
      for (int k = 0; k < j; k++) v -= Lm[(size_t)i * n + k] * Lm[(size_t)j * n + k];
      Lm[(size_t)i * n + j] = v / d;
    }
  }
  inv.assign((size_t)n * n, 0.0);
  std::vector<double> e(n), y(n);
  for (int c = 0; c < n; c++) {
    std::fill(e.begin(), e.end(), 0.0);
    e[c] = 1;
    for (int i = 0; i < n; i++) {
      double v = e[i];
      for (int k = 0; k < i; k++) v -= Lm[(size_t)i * n + k] * y[k];
      y[i] = v / Lm[(size_t)i * n + i];
    }
    for (int i = n - 1; i >= 0; i--) {
      double v = y[i];
      for (int k = i + 1; k < n; k++) v -= Lm[(size_t)k * n + i] * inv[(size_t)k * n + c];
      inv[(size_t)i * n + c] = v / Lm[(size_t)i * n + i];
    }
  }
  return true;
}

}  // namespace

// Dense FP64 inverse of the coarsest level over its liquid cells (fluid:
// the level's per-cell liquid flags; the level's host arrays hold its operator).
static int coarsest_inverse(Hierarchy& H, const std::vector<uint8_t>& fineFluid,
                            std::string* err) {
  const Level& L = H.levels.back();
  std::vector<int64_t> cells;
  std::vector<int> idx(L.nCells, -1);
  for (int64_t c = 0; c < L.nCells; c++)
    if (fineFluid[c]) {
      idx[c] = (int)cells.size();
      cells.push_back(c);
    }
  const int n = (int)cells.size();
  std::vector<double> A((size_t)n * n, 0.0);
  for (int r = 0; r < n; r++) A[(size_t)r * n + r] = L.diag[cells[r]];
  // off-diagonals: same-level lower faces and interface planes
  for (size_t ti = 0; ti < L.tiles.size(); ti++) {
    const Tile& t = L.tiles[ti];
    const int ts = t.ts;
    for (int k = 0; k < ts; k++)
      for (int j = 0; j < ts; j++)
        for (int i = 0; i < ts; i++) {
          const int64_t c = t.off + i + (int64_t)ts * (j + (int64_t)ts * k);
          if (idx[c] < 0) continue;
          const int P[3] = {t.ox + i, t.oy + j, t.oz + k};
          const float* cd[3] = {L.cx.data(), L.cy.data(), L.cz.data()};
          for (int dir = 0; dir < 3; dir++) {
            int q[3] = {P[0], P[1], P[2]};
            q[dir] -= 1;
            int nt = q[dir] >= 0 ? tile_at(L, t.level, q[0], q[1], q[2]) : -1;
            if (nt < 0) continue;
            const Tile& u = L.tiles[nt];
            int64_t c2 = u.off + (q[0] - u.ox) + (int64_t)u.ts * ((q[1] - u.oy) + (int64_t)u.ts * (q[2] - u.oz));
            if (idx[c2] < 0) continue;
            const double w = cd[dir][c];
            A[(size_t)idx[c] * n + idx[c2]] -= w;
            A[(size_t)idx[c2] * n + idx[c]] -= w;
          }
          // interface couplings (this cell on the finer side)
          for (int dir = 0; dir < 3; dir++)
            for (int side = 0; side < 2; side++) {
              int64_t io = L.ifOff[ti * 6 + dir * 2 + side];
              const int loc[3] = {i, j, k};
              if (io < 0 || (side ? loc[dir] != ts - 1 : loc[dir] != 0)) continue;
              int fv[3] = {P[0] << t.level, P[1] << t.level, P[2] << t.level};
              fv[dir] = side ? (P[dir] + 1) << t.level : (P[dir] << t.level) - 1;
              int cc[3];
              for (int kk = 0; kk < 3; kk++) cc[kk] = fv[kk] >> (t.level + 1);
              int nt = tile_at(L, t.level + 1, cc[0], cc[1], cc[2]);
              if (nt < 0) continue;
              const Tile& u = L.tiles[nt];
              int64_t c2 = u.off + (cc[0] - u.ox) + (int64_t)u.ts * ((cc[1] - u.oy) + (int64_t)u.ts * (cc[2] - u.oz));
              if (idx[c2] < 0) continue;
              int ax, bx;
              face_axes(dir, ax, bx);
              const double w = L.ifc[io + loc[ax] + (int64_t)ts * loc[bx]];
              A[(size_t)idx[c] * n + idx[c2]] -= w;
              A[(size_t)idx[c2] * n + idx[c]] -= w;
            }
        }
  }
  if (!dense_spd_inverse(A, n, H.coarseInv)) {
    if (err) *err = "coarsest operator is not positive definite";
    return MSBG_EMATH;
  }
  H.nCoarse = n;
  H.coarseCells = cells;
    return MSBG_OK;
}

// The grid fields of H and the sampling context of a build (both paths).
static int init_build(Hierarchy& H, Ctx& C, int sx, int sy, int sz, int bsx0, int nLevels,
                      const int* blockLevel, const int* domainBc,
                      const msbg_pressure_callbacks* cb, const ArrayInput* arr,
                      std::string* err) {
  H = Hierarchy();
  if (bsx0 != 8 && bsx0 != 16 && bsx0 != 32) {
    if (err) *err = "bsx0 must be 8, 16 or 32";
    return MSBG_EINVARG;
  }
  if (domainBc)
    for (int f = 0; f < 6; f++) {
      if (domainBc[f] != MSBG_DBC_OPEN && domainBc[f] != MSBG_DBC_SOLID) {
        if (err) *err = "domainBc entries must be MSBG_DBC_OPEN or MSBG_DBC_SOLID";
        return MSBG_EINVARG;
      }
      H.domainBc[f] = domainBc[f];
    }
  H.sx = sx;
  H.sy = sy;
  H.sz = sz;
  H.res = std::max({sx, sy, sz});
  H.bsx0 = bsx0;
  H.nLevels = nLevels;
  H.nb1x = sx / bsx0;
  H.nb1y = sy / bsx0;
  H.nb1z = sz / bsx0;
  const int64_t nb = (int64_t)H.nb1x * H.nb1y * H.nb1z;
  H.blockLevel.assign(nb, 0);
  if (blockLevel) std::copy(blockLevel, blockLevel + nb, H.blockLevel.begin());
  C.cb = cb;
  C.arr = arr;
  C.sh0 = 0;
  while ((1 << C.sh0) < bsx0) C.sh0++;
  if (arr) {
    C.boff.assign(nb, 0);
    int64_t o = 0;
    for (int64_t b = 0; b < nb; b++) {
      C.boff[b] = o;
      const int bs = bsx0 >> H.blockLevel[b];
      o += (int64_t)bs * bs * bs;
    }
  }
  C.maxMap = 0;
  for (int v : H.blockLevel) C.maxMap = std::max(C.maxMap, v);
  return MSBG_OK;
}

int build_hierarchy(Hierarchy& H, int sx, int sy, int sz, int bsx0, int nLevels,
                    const int* blockLevel, const int* domainBc,
                    const msbg_pressure_callbacks* cb, int maxCoarseCells, std::string* err,
                    const ArrayInput* arr) {
  Ctx C(H);
  int rc0 = init_build(H, C, sx, sy, sz, bsx0, nLevels, blockLevel, domainBc, cb, arr, err);
  if (rc0) return rc0;

  // ---- MG level 0 ----
  std::vector<uint8_t> fluid;
  {
    Level L;
    L.m = 0;
    std::vector<Tile> cand;
    enumerate_tiles(C, 0, L, cand);
    // keep tiles that hold liquid
    std::vector<uint8_t> keep(cand.size(), 0);
#pragma omp parallel for schedule(dynamic, 4)
    for (int64_t i = 0; i < (int64_t)cand.size(); i++) {
      const Tile& t = cand[i];
      bool any = false;
      int pbs = 0;
      const int64_t pc0 = arr ? C.tile_cell0(t, pbs) : 0;
      for (int k = 0; k < t.ts && !any; k++)
        for (int j = 0; j < t.ts && !any; j++)
          for (int ii = 0; ii < t.ts; ii++) {
            uint16_t ct = arr ? arr->flags[pc0 + ii + (int64_t)pbs * (j + (int64_t)pbs * k)]
                              : C.cell_type((t.ox + ii) << t.level, (t.oy + j) << t.level,
                                            (t.oz + k) << t.level);
            if (!(ct & CELL_NONFLUID)) {
              any = true;
              break;
            }
          }
      keep[i] = any;
    }
    std::vector<Tile> tiles;
    for (size_t i = 0; i < cand.size(); i++)
      if (keep[i]) tiles.push_back(cand[i]);
    register_tiles(L, tiles);
    build_faces(C, L);
    fluid.assign(L.nCells, 0);
    L.ctype.resize(L.nCells);  // every cell is written below
#pragma omp parallel for schedule(dynamic, 4)
    for (int64_t ti = 0; ti < (int64_t)L.tiles.size(); ti++) {
      const Tile& t = L.tiles[ti];
      int pbs = 0;
      const int64_t pc0 = arr ? C.tile_cell0(t, pbs) : 0;
      for (int k = 0; k < t.ts; k++)
        for (int j = 0; j < t.ts; j++)
          for (int i = 0; i < t.ts; i++) {
            uint16_t ct = arr ? arr->flags[pc0 + i + (int64_t)pbs * (j + (int64_t)pbs * k)]
                              : C.cell_type((t.ox + i) << t.level, (t.oy + j) << t.level,
                                            (t.oz + k) << t.level);
            const int64_t c = t.off + i + (int64_t)t.ts * (j + (int64_t)t.ts * k);
            fluid[c] = !(ct & CELL_NONFLUID);
            L.ctype[c] = fluid[c] ? CT_LIQUID : (ct & CELL_SOLID_BIT) ? CT_SOLID : CT_AIR;
          }
    }
    sample_level0(C, L, fluid);
    // A liquid cell whose faces all have coefficient 0 is coupled to nothing:
    // its equation 0 * p = b holds only for b = 0.  The reference gives such a
    // cell D = 0 and skips it (src/msbg3.cpp:2727, 1284-1285), leaving its
    // equation unmet; here a consistent one (b = 0) is dropped (p = 0) and an
    // unsatisfiable one is an error.  A non-finite coefficient is an error too.
    int64_t badCell = -1;
    bool badIsolated = false;
    for (int64_t c = 0; c < L.nCells && badCell < 0; c++) {
      if (!fluid[c]) continue;
      if (!std::isfinite(L.diag[c])) {
        badCell = c;
      } else if (!(L.diag[c] > 0.f)) {
        if (L.rhs[c] != 0.f) {
          badCell = c;
          badIsolated = true;
        } else {
          fluid[c] = 0;
          L.ctype[c] = CT_SOLID;
        }
      }
    }
    if (badCell >= 0) {
      size_t ti = 0;
      while (ti + 1 < L.tiles.size() && L.tiles[ti + 1].off <= badCell) ti++;
      const Tile& t = L.tiles[ti];
      const int64_t e = badCell - t.off;
      const int X = t.ox + (int)(e % t.ts), Y = t.oy + (int)((e / t.ts) % t.ts),
                Z = t.oz + (int)(e / ((int64_t)t.ts * t.ts));
      if (err) {
        char buf[200];
        snprintf(buf, sizeof(buf),
                 badIsolated ? "liquid cell (%d,%d,%d) of level %d has no face with a nonzero "
                               "coefficient but a nonzero right-hand side"
                             : "non-finite face coefficient at liquid cell (%d,%d,%d) of level %d",
                 X, Y, Z, t.level);
        *err = buf;
      }
      return MSBG_EMATH;
    }
    int64_t nf = 0;
    for (auto f : fluid) nf += f;
    L.nFluid = nf;
    H.levels.push_back(std::move(L));
  }
  if (H.levels[0].nFluid == 0) {
    if (err) *err = "no liquid cells";
    return MSBG_EINVARG;
  }

  // ---- coarser MG levels (Galerkin) ----
  std::vector<uint8_t> fineFluid = fluid;
  for (int m = 1;; m++) {
    Level& F = H.levels.back();
    if (F.nFluid <= maxCoarseCells) break;
    // can we coarsen once more?
    const int lmin = m;  // finest level present at MG level m
    if ((sx >> lmin) << lmin != sx || (sy >> lmin) << lmin != sy || (sz >> lmin) << lmin != sz ||
        (sx >> lmin) < 1 || (sy >> lmin) < 1 || (sz >> lmin) < 1) {
      if (err) *err = "grid cannot be coarsened to the direct-solve size";
      return MSBG_EINVARG;
    }
    Level G;
    G.m = m;
    std::vector<Tile> cand;
    enumerate_tiles(C, m, G, cand);
    // coarse liquid flags: any liquid child (aggregates) or same cell
    auto fine_cell = [&](int l, int X, int Y, int Z) -> int64_t {
      int t = tile_at(F, l, X, Y, Z);
      if (t < 0) return -1;
      const Tile& ft = F.tiles[t];
      return ft.off + (X - ft.ox) + (int64_t)ft.ts * ((Y - ft.oy) + (int64_t)ft.ts * (Z - ft.oz));
    };
    std::vector<std::vector<uint8_t>> candFluid(cand.size());
    std::vector<uint8_t> keep(cand.size(), 0);
    // does any fine tile (level t.level-1 or t.level) overlap coarse tile t?
    // Without one every coarse cell is dry, so the per-cell test is skipped.
    auto any_fine_tile = [&](const Tile& t) {
      for (int lv = std::max(0, t.level - 1); lv <= t.level; lv++) {
        const int fts = F.tsOf[lv];
        if (!fts || !F.tmapN[lv]) continue;
        const int sh = t.level - lv;
        const int o[3] = {t.ox << sh, t.oy << sh, t.oz << sh}, e = t.ts << sh;
        // start on the fine tile grid so every overlapping fine tile is visited
        for (int z = o[2] - o[2] % fts; z < o[2] + e; z += fts)
          for (int y = o[1] - o[1] % fts; y < o[1] + e; y += fts)
            for (int x = o[0] - o[0] % fts; x < o[0] + e; x += fts)
              if (tile_at(F, lv, x, y, z) >= 0) return true;
      }
      return false;
    };
#pragma omp parallel for schedule(dynamic, 4)
    for (int64_t i = 0; i < (int64_t)cand.size(); i++) {
      const Tile& t = cand[i];
      if (!any_fine_tile(t)) continue;  // keep[i] stays 0
      auto& cf = candFluid[i];
      cf.assign((size_t)t.ts * t.ts * t.ts, 0);
      bool any = false;
      for (int k = 0; k < t.ts; k++)
        for (int j = 0; j < t.ts; j++)
          for (int ii = 0; ii < t.ts; ii++) {
            const int P[3] = {t.ox + ii, t.oy + j, t.oz + k};
            const int fv[3] = {P[0] << t.level, P[1] << t.level, P[2] << t.level};
            bool f = false;
            if (C.level_at(F.m, fv[0], fv[1], fv[2]) == t.level - 1) {
              for (int c = 0; c < 8 && !f; c++) {
                int64_t fc = fine_cell(t.level - 1, P[0] * 2 + (c & 1), P[1] * 2 + ((c >> 1) & 1),
                                       P[2] * 2 + (c >> 2));
                f = fc >= 0 && fineFluid[fc];
              }
            } else {
              int64_t fc = fine_cell(t.level, P[0], P[1], P[2]);
              f = fc >= 0 && fineFluid[fc];
            }
            cf[ii + (size_t)t.ts * (j + (size_t)t.ts * k)] = f;
            any |= f;
          }
      keep[i] = any;
    }
    std::vector<Tile> tiles;
    std::vector<int> order;
    for (size_t i = 0; i < cand.size(); i++)
      if (keep[i]) {
        tiles.push_back(cand[i]);
        order.push_back((int)i);
      }
    // register_tiles sorts; recover each tile's fluid flags by origin
    std::map<std::tuple<int, int, int, int>, int> byOrigin;
    for (size_t i = 0; i < tiles.size(); i++)
      byOrigin[{tiles[i].level, tiles[i].ox, tiles[i].oy, tiles[i].oz}] = order[i];
    register_tiles(G, tiles);
    build_faces(C, G);
    std::vector<uint8_t> coarseFluid(G.nCells, 0);
    int64_t nf = 0;
    for (const Tile& t : G.tiles) {
      const auto& cf = candFluid[byOrigin[{t.level, t.ox, t.oy, t.oz}]];
      std::copy(cf.begin(), cf.end(), coarseFluid.begin() + t.off);
      for (auto f : cf) nf += f;
    }
    G.nFluid = nf;
    galerkin(C, F, fineFluid, G, coarseFluid);
    build_restriction(C, F, G);
    H.levels.push_back(std::move(G));
    fineFluid.swap(coarseFluid);
    if (m > 24) {
      if (err) *err = "too many multigrid levels";
      return MSBG_EINTERNAL;
    }
  }

  // ---- coarsest: dense FP64 inverse over the liquid cells ----
  return coarsest_inverse(H, fineFluid, err);
}


// ---------------------------------------------------------------------------
// The bulk prepare with the per-cell work on the GPU (build_gpu.cu)
// ---------------------------------------------------------------------------
namespace {

template <typename T>
cudaError_t upload_vec(DeviceBuffer& b, const std::vector<T>& v, cudaStream_t st) {
  cudaError_t e = b.ensure(sizeof(T) * std::max<size_t>(v.size(), 1));
  if (e != cudaSuccess || v.empty()) return e;
  return cudaMemcpyAsync(b.p, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice, st);
}
template <typename T, typename A>
cudaError_t upload_vec(DeviceBuffer& b, const std::vector<T, A>& v, cudaStream_t st) {
  cudaError_t e = b.ensure(sizeof(T) * std::max<size_t>(v.size(), 1));
  if (e != cudaSuccess || v.empty()) return e;
  return cudaMemcpyAsync(b.p, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice, st);
}

// Device copy of a level's tiles and tile maps.
struct LevelMap {
  DeviceBuffer tiles, tmap;
  LevelMapD view{};
};

int upload_map(const Level& L, LevelMap& M, cudaStream_t st) {
  std::vector<TileD> td(L.tiles.size());
  for (size_t i = 0; i < L.tiles.size(); i++) {
    const Tile& t = L.tiles[i];
    td[i] = TileD{t.level, t.ts, t.ox, t.oy, t.oz, 0, t.off};
  }
  std::vector<int> tm;
  for (int l = 0; l < 32; l++) {
    if (l >= MAXRL) {
      if (L.tmapN[l]) return MSBG_EINTERNAL;
      continue;
    }
    M.view.tmapN[l] = L.tmapN[l];
    M.view.tsSh[l] = L.tsOf[l] ? __builtin_ctz(L.tsOf[l]) : 0;
    M.view.tmapOff[l] = (int64_t)tm.size();
    tm.insert(tm.end(), L.tmap[l].begin(), L.tmap[l].end());
  }
  if (upload_vec(M.tiles, td, st) != cudaSuccess || upload_vec(M.tmap, tm, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)  // td, tm are temporaries
    return MSBG_ENOMEM;
  M.view.tiles = M.tiles.as<TileD>();
  M.view.tmap = M.tmap.as<int>();
  M.view.m = L.m;
  return MSBG_OK;
}

// Pinned staging and device buffers of the level-0 chunks (per host thread,
// kept across prepares): a parallel gather fills one while the other's copy
// and kernel run.
struct BuildStaging {
  static constexpr int64_t CH_CELLS = 4 << 20, CH_TILES = 4096;
  static constexpr size_t BYTES =
      (size_t)CH_CELLS * (2 + 4 * 4) + 6 * 16 + (size_t)CH_TILES * 3 * TS_MAX * TS_MAX * 8;
  void* buf[2] = {nullptr, nullptr};
  cudaEvent_t ev[2] = {nullptr, nullptr};
  DeviceBuffer raw[2];
  bool used[2] = {false, false};
  int device = -1;
  ~BuildStaging() {
    for (int i = 0; i < 2; i++) {
      if (ev[i]) cudaEventDestroy(ev[i]);
      if (buf[i]) cudaFreeHost(buf[i]);
    }
  }
  bool ready(int dev) {
    if (device == dev) return true;
    if (device >= 0) return false;
    // (a partial earlier attempt keeps what it got; nothing is allocated twice)
    for (int i = 0; i < 2; i++)
      if ((!buf[i] && cudaMallocHost(&buf[i], BYTES) != cudaSuccess) ||
          (!ev[i] && cudaEventCreateWithFlags(&ev[i], cudaEventDisableTiming) != cudaSuccess) ||
          raw[i].ensure(BYTES) != cudaSuccess)
        return false;
    device = dev;
    return true;
  }
};

BuildStaging& build_staging() {
  thread_local BuildStaging s;
  return s;
}

size_t align16(size_t v) { return (v + 15) & ~(size_t)15; }

}  // namespace

int build_hierarchy_device(Hierarchy& H, std::vector<std::unique_ptr<LevelDev>>& dev,
                           DeviceBuffer& rhs0, int sx, int sy, int sz, int bsx0, int nLevels,
                           const int* blockLevel, const int* domainBc, const ArrayInput& arr,
                           int maxCoarseCells, cudaStream_t st, std::string* err) {
  Ctx C(H);
  int rc = init_build(H, C, sx, sy, sz, bsx0, nLevels, blockLevel, domainBc, nullptr, &arr, err);
  if (rc) return rc;
  dev.clear();
  auto fail = [&](int code, const char* what) {
    if (err) *err = what;
    return code;
  };
#define DB_TRY(expr)                                                   \
  do {                                                                 \
    if ((expr) != cudaSuccess) return fail(MSBG_ENOMEM, #expr);        \
  } while (0)
  int device = 0;
  DB_TRY(cudaGetDevice(&device));

  // ---- MG level 0: topology on the host ----
  Level L;
  L.m = 0;
  {
    std::vector<Tile> cand;
    enumerate_tiles(C, 0, L, cand);
    std::vector<uint8_t> keep(cand.size(), 0);
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t i = 0; i < (int64_t)cand.size(); i++) {
      const Tile& t = cand[i];
      int pbs = 0;
      const int64_t pc0 = C.tile_cell0(t, pbs);
      bool any = false;
      for (int k = 0; k < t.ts && !any; k++)
        for (int j = 0; j < t.ts && !any; j++) {
          const uint16_t* f = arr.flags + pc0 + (int64_t)pbs * (j + (int64_t)pbs * k);
          for (int ii = 0; ii < t.ts; ii++)
            if (!(f[ii] & CELL_NONFLUID)) {
              any = true;
              break;
            }
        }
      keep[i] = any;
    }
    std::vector<Tile> tiles;
    for (size_t i = 0; i < cand.size(); i++)
      if (keep[i]) tiles.push_back(cand[i]);
    register_tiles(L, tiles);
    build_faces(C, L);
  }
  if (L.tiles.empty()) return fail(MSBG_EINVARG, "no liquid cells");
  const int nT0 = (int)L.tiles.size();
  // the region behind each tile face: -1 outside the domain, else its level
  std::vector<int> faceInfo((size_t)nT0 * 6);
#pragma omp parallel for schedule(static)
  for (int ti = 0; ti < nT0; ti++) {
    const Tile& t = L.tiles[ti];
    const int l = t.level, o[3] = {t.ox, t.oy, t.oz};
    for (int dir = 0; dir < 3; dir++)
      for (int side = 0; side < 2; side++) {
        int fv[3] = {t.ox << l, t.oy << l, t.oz << l};
        const int pd = side ? o[dir] + t.ts - 1 : o[dir];
        fv[dir] = side ? (pd + 1) << l : (pd << l) - 1;
        faceInfo[(size_t)ti * 6 + dir * 2 + side] =
            C.inside(fv[0], fv[1], fv[2]) ? C.level_at(0, fv[0], fv[1], fv[2]) : -1;
      }
  }

  // ---- MG level 0: per-cell arrays on the GPU, chunk by chunk ----
  auto D0 = std::make_unique<LevelDev>();
  auto M0 = std::make_unique<LevelMap>();
  if ((rc = upload_map(L, *M0, st))) return fail(rc, "level-0 tile map");
  const int64_t n0 = L.nCells;
  DeviceBuffer dFace, dScal;
  DB_TRY(D0->diag.ensure(sizeof(float) * n0));
  DB_TRY(D0->cx.ensure(sizeof(float) * n0));
  DB_TRY(D0->cy.ensure(sizeof(float) * n0));
  DB_TRY(D0->cz.ensure(sizeof(float) * n0));
  DB_TRY(D0->ifc.ensure(sizeof(float) * std::max<int64_t>(L.nIf, 1)));
  DB_TRY(D0->ctype.ensure(n0));
  DB_TRY(D0->fluid.ensure(n0));
  DB_TRY(rhs0.ensure(sizeof(float) * n0));
  DB_TRY(upload_vec(D0->ifOff, L.ifOff, st));
  DB_TRY(upload_vec(dFace, faceInfo, st));
  const unsigned long long scal0[2] = {~0ull, 0ull};
  DB_TRY(dScal.ensure(sizeof(scal0)));
  DB_TRY(cudaMemcpyAsync(dScal.p, scal0, sizeof(scal0), cudaMemcpyHostToDevice, st));
  BuildStaging& stg = build_staging();
  // (the staging of a host thread serves one device; the caller then builds
  // on the host)
  if (!stg.ready(device)) return fail(MSBG_ENOTIMPL, "no pinned staging for this device");
  for (int k = 0; k < 2; k++)
    if (stg.used[k]) DB_TRY(cudaEventSynchronize(stg.ev[k]));
  stg.used[0] = stg.used[1] = false;
  L0Args a{};
  a.tiles = M0->view.tiles;
  a.faceInfo = dFace.as<int>();
  a.ifOff = D0->ifOff.as<int64_t>();
  for (int f = 0; f < 6; f++) a.dbc[f] = H.domainBc[f];
  a.diag = D0->diag.as<float>();
  a.cx = D0->cx.as<float>();
  a.cy = D0->cy.as<float>();
  a.cz = D0->cz.as<float>();
  a.rhs0 = rhs0.as<float>();
  a.ifc = D0->ifc.as<float>();
  a.ctype = D0->ctype.as<uint8_t>();
  a.fluid = D0->fluid.as<uint8_t>();
  a.bad = dScal.as<unsigned long long>();
  a.nFluid = a.bad + 1;
  for (int t0 = 0, q = 0; t0 < nT0; q++) {
    // the chunk: consecutive tiles within the staging limits
    int t1 = t0;
    while (t1 < nT0 && t1 - t0 < BuildStaging::CH_TILES &&
           L.tiles[t1].off + (int64_t)L.tiles[t1].ts * L.tiles[t1].ts * L.tiles[t1].ts -
                   L.tiles[t0].off <= BuildStaging::CH_CELLS)
      t1++;
    const int64_t c0 = L.tiles[t0].off;
    const int64_t nc = (t1 < nT0 ? L.tiles[t1].off : n0) - c0;
    const size_t oF = 0, oX = align16(sizeof(uint16_t) * nc), oY = oX + align16(4 * nc),
                 oZ = oY + align16(4 * nc), oR = oZ + align16(4 * nc), oP = oR + align16(4 * nc);
    const size_t bytes = oP + (size_t)(t1 - t0) * 3 * TS_MAX * TS_MAX * 8;
    const int k = q & 1;
    if (stg.used[k]) DB_TRY(cudaEventSynchronize(stg.ev[k]));
    char* hb = static_cast<char*>(stg.buf[k]);
    uint16_t* hf = reinterpret_cast<uint16_t*>(hb + oF);
    float* hx[4] = {reinterpret_cast<float*>(hb + oX), reinterpret_cast<float*>(hb + oY),
                    reinterpret_cast<float*>(hb + oZ), reinterpret_cast<float*>(hb + oR)};
    double* hp = reinterpret_cast<double*>(hb + oP);
    const float* src[4] = {arr.face[0], arr.face[1], arr.face[2], arr.rhs};
#pragma omp parallel for schedule(dynamic, 4)
    for (int ti = t0; ti < t1; ti++) {
      const Tile& t = L.tiles[ti];
      const int ts = t.ts, l = t.level;
      int pbs = 0;
      const int64_t pc0 = C.tile_cell0(t, pbs);
      const int64_t d0 = t.off - c0;
      for (int kk = 0; kk < ts; kk++)
        for (int j = 0; j < ts; j++) {
          const int64_t s0 = pc0 + (int64_t)pbs * (j + (int64_t)pbs * kk);
          const int64_t dd = d0 + (int64_t)ts * (j + (int64_t)ts * kk);
          std::memcpy(hf + dd, arr.flags + s0, sizeof(uint16_t) * ts);
          for (int w = 0; w < 4; w++) {
            if (src[w])
              std::memcpy(hx[w] + dd, src[w] + s0, sizeof(float) * ts);
            else
              std::memset(hx[w] + dd, 0, sizeof(float) * ts);
          }
        }
      // couplings of the upper tile faces inside the domain
      double* pl = hp + (size_t)(ti - t0) * 3 * TS_MAX * TS_MAX;
      for (int dir = 0; dir < 3; dir++) {
        const int l2 = faceInfo[(size_t)ti * 6 + dir * 2 + 1];
        if (l2 < 0) continue;
        int ax, bx;
        face_axes(dir, ax, bx);
        for (int b = 0; b < ts; b++)
          for (int aa = 0; aa < ts; aa++) {
            int p[3] = {t.ox, t.oy, t.oz};
            p[dir] += ts - 1;
            p[ax] += aa;
            p[bx] += b;
            pl[dir * TS_MAX * TS_MAX + aa + ts * b] = upper_coupling(C, l, l2, dir, p);
          }
      }
    }
    char* db = static_cast<char*>(stg.raw[k].p);
    DB_TRY(cudaMemcpyAsync(db, hb, bytes, cudaMemcpyHostToDevice, st));
    H.deviceBuildH2D += (int64_t)bytes;
    a.tile0 = t0;
    a.cell0 = c0;
    a.flags = reinterpret_cast<const uint16_t*>(db + oF);
    a.fx = reinterpret_cast<const float*>(db + oX);
    a.fy = reinterpret_cast<const float*>(db + oY);
    a.fz = reinterpret_cast<const float*>(db + oZ);
    a.rhs = reinterpret_cast<const float*>(db + oR);
    a.planes = reinterpret_cast<const double*>(db + oP);
    DB_TRY(launch_build_l0(a, t1 - t0, st));
    DB_TRY(cudaEventRecord(stg.ev[k], st));
    stg.used[k] = true;
    t0 = t1;
  }
  unsigned long long scal[2];
  DB_TRY(cudaMemcpyAsync(scal, dScal.p, sizeof(scal), cudaMemcpyDeviceToHost, st));
  DB_TRY(cudaStreamSynchronize(st));
  if (scal[0] != ~0ull) {
    const int64_t badCell = (int64_t)(scal[0] >> 1);
    const bool isolated = scal[0] & 1;
    size_t ti = 0;
    while (ti + 1 < L.tiles.size() && L.tiles[ti + 1].off <= badCell) ti++;
    const Tile& t = L.tiles[ti];
    const int64_t e = badCell - t.off;
    const int X = t.ox + (int)(e % t.ts), Y = t.oy + (int)((e / t.ts) % t.ts),
              Z = t.oz + (int)(e / ((int64_t)t.ts * t.ts));
    char buf[200];
    snprintf(buf, sizeof(buf),
             isolated ? "liquid cell (%d,%d,%d) of level %d has no face with a nonzero "
                        "coefficient but a nonzero right-hand side"
                      : "non-finite face coefficient at liquid cell (%d,%d,%d) of level %d",
             X, Y, Z, t.level);
    return fail(MSBG_EMATH, buf);
  }
  L.nFluid = (int64_t)scal[1];
  if (L.nFluid == 0) return fail(MSBG_EINVARG, "no liquid cells");
  H.levels.push_back(std::move(L));
  dev.push_back(std::move(D0));
  std::vector<std::unique_ptr<LevelMap>> maps;
  maps.push_back(std::move(M0));

  // ---- coarser MG levels: Galerkin on the GPU ----
  DeviceBuffer dBL;
  DB_TRY(upload_vec(dBL, H.blockLevel, st));
  const GridD g{sx, sy, sz, C.sh0, H.nb1x, H.nb1y, dBL.as<int>()};
  for (int m = 1;; m++) {
    Level& F = H.levels.back();
    LevelDev& DF = *dev.back();
    if (F.nFluid <= maxCoarseCells) break;
    const int lmin = m;
    if ((sx >> lmin) << lmin != sx || (sy >> lmin) << lmin != sy || (sz >> lmin) << lmin != sz ||
        (sx >> lmin) < 1 || (sy >> lmin) < 1 || (sz >> lmin) < 1)
      return fail(MSBG_EINVARG, "grid cannot be coarsened to the direct-solve size");
    if (m > 24) return fail(MSBG_EINTERNAL, "too many multigrid levels");
    Level G;
    G.m = m;
    std::vector<Tile> cand;
    enumerate_tiles(C, m, G, cand);
    // candidates that overlap a fine tile (the others hold no liquid)
    std::vector<int> ci;
    std::vector<TileD> ctd;
    std::vector<int64_t> coff;
    int64_t ncf = 0;
    for (size_t i = 0; i < cand.size(); i++) {
      const Tile& t = cand[i];
      bool any = false;
      for (int lv = std::max(0, t.level - 1); lv <= t.level && !any; lv++) {
        const int fts = F.tsOf[lv];
        if (!fts || !F.tmapN[lv]) continue;
        const int sh = t.level - lv;
        const int o[3] = {t.ox << sh, t.oy << sh, t.oz << sh}, e = t.ts << sh;
        for (int z = o[2] - o[2] % fts; z < o[2] + e && !any; z += fts)
          for (int y = o[1] - o[1] % fts; y < o[1] + e && !any; y += fts)
            for (int x = o[0] - o[0] % fts; x < o[0] + e && !any; x += fts)
              any = tile_at(F, lv, x, y, z) >= 0;
      }
      if (!any) continue;
      ci.push_back((int)i);
      ctd.push_back(TileD{t.level, t.ts, t.ox, t.oy, t.oz, 0, 0});
      coff.push_back(ncf);
      ncf += (int64_t)t.ts * t.ts * t.ts;
    }
    const int nc = (int)ci.size();
    DeviceBuffer dCand, dCoff, dCandFluid, dCandAny;
    DB_TRY(upload_vec(dCand, ctd, st));
    DB_TRY(upload_vec(dCoff, coff, st));
    DB_TRY(dCandFluid.ensure(std::max<int64_t>(ncf, 1)));
    DB_TRY(dCandAny.ensure(sizeof(int) * std::max(nc, 1)));
    CoarseArgs ca{dCand.as<TileD>(), dCoff.as<int64_t>(), maps.back()->view, g,
                  DF.fluid.as<uint8_t>(), dCandFluid.as<uint8_t>(), dCandAny.as<int>()};
    DB_TRY(launch_coarse_fluid(ca, nc, st));
    std::vector<int> candAny(nc);
    if (nc) DB_TRY(cudaMemcpyAsync(candAny.data(), dCandAny.p, sizeof(int) * nc,
                                   cudaMemcpyDeviceToHost, st));
    DB_TRY(cudaStreamSynchronize(st));
    std::vector<Tile> tiles;
    std::map<std::tuple<int, int, int, int>, int64_t> srcOf;
    for (int k = 0; k < nc; k++)
      if (candAny[k]) {
        const Tile& t = cand[ci[k]];
        tiles.push_back(t);
        srcOf[{t.level, t.ox, t.oy, t.oz}] = coff[k];
      }
    register_tiles(G, tiles);
    build_faces(C, G);
    std::vector<int64_t> srcOff(G.tiles.size());
    for (size_t i = 0; i < G.tiles.size(); i++) {
      const Tile& t = G.tiles[i];
      srcOff[i] = srcOf[{t.level, t.ox, t.oy, t.oz}];
    }
    auto DG = std::make_unique<LevelDev>();
    auto MG = std::make_unique<LevelMap>();
    if ((rc = upload_map(G, *MG, st))) return fail(rc, "coarse tile map");
    const int64_t nG = G.nCells;
    DeviceBuffer dSrc;
    DB_TRY(upload_vec(dSrc, srcOff, st));
    DB_TRY(DG->fluid.ensure(std::max<int64_t>(nG, 1)));
    DB_TRY(cudaMemsetAsync(dScal.p, 0, sizeof(unsigned long long) * 2, st));
    DB_TRY(launch_place_fluid(MG->view.tiles, dSrc.as<int64_t>(), dCandFluid.as<uint8_t>(),
                              DG->fluid.as<uint8_t>(), dScal.as<unsigned long long>() + 1,
                              (int)G.tiles.size(), st));
    for (DeviceBuffer* b : {&DG->diag, &DG->cx, &DG->cy, &DG->cz}) {
      DB_TRY(b->ensure(sizeof(float) * std::max<int64_t>(nG, 1)));
      DB_TRY(cudaMemsetAsync(b->p, 0, sizeof(float) * std::max<int64_t>(nG, 1), st));
    }
    DB_TRY(DG->ifc.ensure(sizeof(float) * std::max<int64_t>(G.nIf, 1)));
    DB_TRY(cudaMemsetAsync(DG->ifc.p, 0, sizeof(float) * std::max<int64_t>(G.nIf, 1), st));
    DB_TRY(upload_vec(DG->ifOff, G.ifOff, st));
    GalerkinArgs ga{};
    ga.F = maps.back()->view;
    ga.g = g;
    ga.fineFluid = DF.fluid.as<uint8_t>();
    ga.Fdiag = DF.diag.as<float>();
    ga.Fcx = DF.cx.as<float>();
    ga.Fcy = DF.cy.as<float>();
    ga.Fcz = DF.cz.as<float>();
    ga.Fifc = DF.ifc.as<float>();
    ga.FifOff = DF.ifOff.as<int64_t>();
    ga.Gtiles = MG->view.tiles;
    ga.GifOff = DG->ifOff.as<int64_t>();
    ga.coarseFluid = DG->fluid.as<uint8_t>();
    ga.Gm = m;
    ga.Gdiag = DG->diag.as<float>();
    ga.Gcx = DG->cx.as<float>();
    ga.Gcy = DG->cy.as<float>();
    ga.Gcz = DG->cz.as<float>();
    ga.Gifc = DG->ifc.as<float>();
    DB_TRY(launch_galerkin(ga, (int)G.tiles.size(), st));
    unsigned long long nf = 0;
    DB_TRY(cudaMemcpyAsync(&nf, dScal.as<unsigned long long>() + 1, sizeof(nf),
                           cudaMemcpyDeviceToHost, st));
    DB_TRY(cudaStreamSynchronize(st));  // the temporaries above are released below
    G.nFluid = (int64_t)nf;
    build_restriction(C, F, G);
    DF.fluid.release();  // the finer level's flags are done with
    H.levels.push_back(std::move(G));
    dev.push_back(std::move(DG));
    maps.push_back(std::move(MG));
  }

  // 1 / a_ii of every level
  for (size_t m = 0; m < dev.size(); m++) {
    LevelDev& D = *dev[m];
    const int64_t n = std::max<int64_t>(H.levels[m].nCells, 1);
    DB_TRY(D.invdiag.ensure(sizeof(float) * n));
    DB_TRY(launch_invdiag(D.diag.as<float>(), D.invdiag.as<float>(), H.levels[m].nCells, st));
  }

  // ---- coarsest: its operator to the host, dense FP64 inverse ----
  Level& Lc = H.levels.back();
  LevelDev& Dc = *dev.back();
  const int64_t nCc = Lc.nCells;
  Lc.diag.resize(nCc);
  Lc.cx.resize(nCc);
  Lc.cy.resize(nCc);
  Lc.cz.resize(nCc);
  Lc.ifc.resize(std::max<int64_t>(Lc.nIf, 0));
  std::vector<uint8_t> fluidC(nCc);
  DB_TRY(cudaMemcpyAsync(Lc.diag.data(), Dc.diag.p, 4 * nCc, cudaMemcpyDeviceToHost, st));
  DB_TRY(cudaMemcpyAsync(Lc.cx.data(), Dc.cx.p, 4 * nCc, cudaMemcpyDeviceToHost, st));
  DB_TRY(cudaMemcpyAsync(Lc.cy.data(), Dc.cy.p, 4 * nCc, cudaMemcpyDeviceToHost, st));
  DB_TRY(cudaMemcpyAsync(Lc.cz.data(), Dc.cz.p, 4 * nCc, cudaMemcpyDeviceToHost, st));
  if (Lc.nIf > 0)
    DB_TRY(cudaMemcpyAsync(Lc.ifc.data(), Dc.ifc.p, 4 * Lc.nIf, cudaMemcpyDeviceToHost, st));
  DB_TRY(cudaMemcpyAsync(fluidC.data(), Dc.fluid.p, nCc, cudaMemcpyDeviceToHost, st));
  DB_TRY(cudaStreamSynchronize(st));
  Dc.fluid.release();
#undef DB_TRY
  return coarsest_inverse(H, fluidC, err);
}

}  // namespace ps
}  // namespace msbg
