/* CPU restatement of the mixed-resolution MAC velocity interpolation of G2P
 * (TEST INFRASTRUCTURE ONLY: the oracle the GPU kernels of csrc/flip_mr.cu
 * are checked against; nothing of the product calls it).
 *
 * Grid: sx*sy*sz voxels in bsx0^3 blocks (nbx*nby*nbz, bid = bx + nbx*(by +
 * nby*bz)), block b at resolution level level[b] (0 = finest).  Channels use
 * the packed layout: for every block in ascending bid, its (bsx0>>level)^3
 * voxels at its own level (vid = x + y*bs + z*bs*bs); off[b] is the first
 * voxel of block b.  Vector channels hold 3 floats per voxel, the MAC values
 * (u, v, w) of the voxel's lower x, y and z faces.
 *
 *   oracle_mr_dist        CH_DIST_FINECOARSE as setRefinementMap builds it
 *                         (src/msbg.cpp:1700-1723 flag rule, 1887-1960 channel)
 *   oracle_mr_dist_interp SparseGrid<uint16_t>::interpolateToFloat<IP_LINEAR>
 *                         with OPT_IPBC_NEUMAN (src/sbg.h:1386, 2936-2941,
 *                         3111-3420)
 *   oracle_mr_g2p         gridToParticle (src/flip_sim.cpp:1526-1545) through
 *                         interpVec3MSBG / interpCompMSBG
 *                         (src/flip_sim.cpp:1354-1525)
 *
 * Float arithmetic in the reference's order, compiled without contraction
 * (-ffp-contract=off); MtLinstep (src/mtool.c:200-208) in double as there.
 *
 * Parity status: oracle_mr_dist and oracle_mr_dist_interp are pinned to the
 * compiled reference (tests/test_oracle_flip_mr.py).  The rest restates
 * src/flip_sim.cpp, which is not compiled here (it includes hypre's headers
 * and calls MultiresSparseGrid::prepareDataAccess, which the reference's
 * msbg.h does not declare): that part is unpinned. */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>

#include "msbg_oracle.h"

int64_t oracle_mr_layout(int nbx, int nby, int nbz, int bsx0, const int* level, int64_t* off) {
  int64_t o = 0;
  for (int64_t b = 0; b < (int64_t)nbx * nby * nbz; b++) {
    const int bs = bsx0 >> level[b];
    off[b] = o;
    o += (int64_t)bs * bs * bs;
  }
  return o;
}

/* Fills CH_DIST_FINECOARSE of every level as setRefinementMap does.
 * Value blocks (src/msbg.cpp:1700-1723, 1887-1960): a block with a coarser
 * block among its 26 neighbours (BLK_FINE_COARSE) holds, per voxel of its own
 * level (at the voxel centre, in that level's units), the distance to the
 * nearest coarser neighbour's box (distToBoxSq, src/msbg.h:3936-3948), capped
 * at dTransRes, stored as (uint16)(dist*1024).  Full blocks
 * (src/msbg.cpp:1994-2029): in the channel of level l, a block of level l or
 * l-1 that is not a value block there and has a BLK_FINE_COARSE neighbour of
 * level l reads dTransRes*1024.  kind[l*nb + b]: 0 empty (reads 0), 1 value,
 * 2 full; dist: the value blocks in the packed layout, 0 elsewhere. */
void oracle_mr_dist(int nbx, int nby, int nbz, int bsx0, const int* level, int nLevels,
                    int dTransRes, uint16_t* dist, int8_t* kind) {
  const int64_t nb = (int64_t)nbx * nby * nbz;
  uint8_t* fc = (uint8_t*)calloc((size_t)nb, 1);
  int64_t off = 0;
  for (int64_t b = 0; b < nb; b++) {
    const int lv = level[b], bs = bsx0 >> lv;
    const int64_t nv = (int64_t)bs * bs * bs;
    const int bx = (int)(b % nbx), by = (int)((b / nbx) % nby), bz = (int)(b / ((int64_t)nbx * nby));
    int nAct = 0, act[26][3];
    for (int dz = -1; dz <= 1; dz++)
      for (int dy = -1; dy <= 1; dy++)
        for (int dx = -1; dx <= 1; dx++) {
          if (!dx && !dy && !dz) continue;
          const int x2 = bx + dx, y2 = by + dy, z2 = bz + dz;
          if (x2 < 0 || y2 < 0 || z2 < 0 || x2 >= nbx || y2 >= nby || z2 >= nbz) continue;
          if (level[x2 + (int64_t)nbx * (y2 + (int64_t)nby * z2)] <= lv) continue;
          act[nAct][0] = x2;
          act[nAct][1] = y2;
          act[nAct][2] = z2;
          nAct++;
        }
    fc[b] = nAct > 0;
    for (int64_t v = 0; v < nv; v++) dist[off + v] = 0;
    if (nAct) {
      int64_t vid = 0;
      for (int z1 = bz * bs; z1 < (bz + 1) * bs; z1++)
        for (int y1 = by * bs; y1 < (by + 1) * bs; y1++)
          for (int x1 = bx * bs; x1 < (bx + 1) * bs; x1++, vid++) {
            const float p[3] = {x1 + 0.5f, y1 + 0.5f, z1 + 0.5f};
            float d2 = 1e20f;
            for (int i = 0; i < nAct; i++) {
              float s = 0.f;
              for (int c = 0; c < 3; c++) {
                const float lo = (float)(act[i][c] * bs), hi = (float)((act[i][c] + 1) * bs);
                float e = lo - p[c];
                if (e < 0.f) e = 0.f;
                if (p[c] - hi > e) e = p[c] - hi;
                s += e * e;
              }
              if (s < d2) d2 = s;
            }
            float d = sqrtf(d2);
            if (d < 0.f || d > (float)dTransRes) d = (float)dTransRes;
            dist[off + vid] = (uint16_t)(d * 1024.f);
          }
    }
    off += nv;
  }
  for (int l = 0; l < nLevels; l++)
    for (int64_t b = 0; b < nb; b++) {
      int8_t k = 0;
      if (level[b] == l && fc[b]) {
        k = 1;
      } else if (level[b] == l || level[b] == l - 1) {
        const int bx = (int)(b % nbx), by = (int)((b / nbx) % nby),
                  bz = (int)(b / ((int64_t)nbx * nby));
        for (int dz = -1; dz <= 1 && !k; dz++)
          for (int dy = -1; dy <= 1 && !k; dy++)
            for (int dx = -1; dx <= 1 && !k; dx++) {
              if (!dx && !dy && !dz) continue;
              const int x2 = bx + dx, y2 = by + dy, z2 = bz + dz;
              if (x2 < 0 || y2 < 0 || z2 < 0 || x2 >= nbx || y2 >= nby || z2 >= nbz) continue;
              const int64_t b2 = x2 + (int64_t)nbx * (y2 + (int64_t)nby * z2);
              if (level[b2] == l && fc[b2]) k = 2;
            }
      }
      kind[(int64_t)l * nb + b] = k;
    }
  free(fc);
}

typedef struct {
  int sx, sy, sz, bsx0, nbx, nby, nbz;
  const int* level;
  const int64_t* off;
} MRGrid;

/* Packed index of voxel (x, y, z) of resolution level lv, or -1 where the
 * level's grid has no data there (outside the grid, or a block of another
 * level: its block data pointer is NULL in that level's channel). */
static int64_t mr_idx(const MRGrid* g, int lv, int x, int y, int z) {
  const int bs = g->bsx0 >> lv;
  if (x < 0 || y < 0 || z < 0 || x >= (g->sx >> lv) || y >= (g->sy >> lv) || z >= (g->sz >> lv))
    return -1;
  const int64_t b = x / bs + (int64_t)g->nbx * (y / bs + (int64_t)g->nby * (z / bs));
  if (g->level[b] != lv) return -1;
  return g->off[b] + x % bs + (int64_t)bs * (y % bs + (int64_t)bs * (z % bs));
}

/* interpolateGen0<float, float, IP_LINEAR> (src/sbg.h:3111-3420) on the
 * distance channel of level lv: cell-centred (p - 0.5), the 2x2x2 window
 * clamped to the grid where it leaves it (OPT_IPBC_NEUMAN); value blocks read
 * their data, full blocks `full`, the others 0; Interpolate1D is p1*t + p0*(1-t) along x,
 * then y, then z. */
static float mr_dist_interp(const MRGrid* g, const uint16_t* dist, const int8_t* kind,
                            int full, int lv, const float p0[3]) {
  const float x = p0[0] - 0.5f, y = p0[1] - 0.5f, z = p0[2] - 0.5f;
  const int ix = (int)floorf(x), iy = (int)floorf(y), iz = (int)floorf(z);
  const float u = x - ix, v = y - iy, w = z - iz;
  const int n[3] = {g->sx >> lv, g->sy >> lv, g->sz >> lv};
  float bz[2];
  for (int k = 0; k < 2; k++) {
    int zz = iz + k;
    if (zz < 0) zz = 0;
    if (zz >= n[2]) zz = n[2] - 1;
    float by[2];
    for (int j = 0; j < 2; j++) {
      int yy = iy + j;
      if (yy < 0) yy = 0;
      if (yy >= n[1]) yy = n[1] - 1;
      float bx[2];
      for (int i = 0; i < 2; i++) {
        int xx = ix + i;
        if (xx < 0) xx = 0;
        if (xx >= n[0]) xx = n[0] - 1;
        const int bs = g->bsx0 >> lv;
        const int64_t b = xx / bs + (int64_t)g->nbx * (yy / bs + (int64_t)g->nby * (zz / bs));
        const int k = kind[(int64_t)lv * g->nbx * g->nby * g->nbz + b];
        bx[i] = k == 1 ? (float)dist[mr_idx(g, lv, xx, yy, zz)] : k == 2 ? (float)full : 0.f;
      }
      by[j] = bx[1] * u + bx[0] * (1.0f - u);
    }
    bz[k] = by[1] * v + by[0] * (1.0f - v);
  }
  return bz[1] * w + bz[0] * (1.0f - w);
}

void oracle_mr_dist_interp(int sx, int sy, int sz, int bsx0, int nbx, int nby, int nbz,
                           const int* level, const int64_t* off, const uint16_t* dist,
                           const int8_t* kind, int dTransRes, int lv, const float* pos,
                           int64_t n, float* out) {
  MRGrid g = {sx, sy, sz, bsx0, nbx, nby, nbz, level, off};
  for (int64_t i = 0; i < n; i++)
    out[i] = mr_dist_interp(&g, dist, kind, dTransRes * 1024, lv, pos + 3 * i);
}

/* MtLinstep (src/mtool.c:200-208) */
static double linstep(double a, double b, double x) {
  if (x < a) return 0;
  if (x >= b) return 1;
  return (x - a) / (b - a);
}

/* interpCompMSBG (src/flip_sim.cpp:1450-1524); interpVec3MSBG
 * (src/flip_sim.cpp:1354-1448) gives, per component, the same value with the
 * level of that component's own sample block, whether it takes its shared
 * path or falls back to this one. */
static float mr_interp_comp(const MRGrid* g, const float* vel, const uint16_t* dist,
                            const int8_t* kind, int dTransRes, const float pos[3],
                            const float off[3], int comp) {
  if (!isfinite(pos[0]) || !isfinite(pos[1]) || !isfinite(pos[2])) return 0.f; /* no cell */
  const float gx = pos[0] - off[0], gy = pos[1] - off[1], gz = pos[2] - off[2];
  const int ix0 = (int)floorf(gx), iy0 = (int)floorf(gy), iz0 = (int)floorf(gz);
  const float fx = gx - ix0, fy = gy - iy0, fz = gz - iz0;
  int cx = ix0 < 0 ? 0 : ix0 >= g->sx ? g->sx - 1 : ix0;
  int cy = iy0 < 0 ? 0 : iy0 >= g->sy ? g->sy - 1 : iy0;
  int cz = iz0 < 0 ? 0 : iz0 >= g->sz ? g->sz - 1 : iz0;
  const int bs0 = g->bsx0;
  const int lv = g->level[cx / bs0 + (int64_t)g->nbx * (cy / bs0 + (int64_t)g->nby * (cz / bs0))];
  /* trilinear in the level-0 channel (getVC: 0 outside the grid and in blocks
   * without level-0 data) */
  float fine = 0.f;
  for (int dz = 0; dz <= 1; dz++)
    for (int dy = 0; dy <= 1; dy++)
      for (int dx = 0; dx <= 1; dx++) {
        const int64_t q = mr_idx(g, 0, ix0 + dx, iy0 + dy, iz0 + dz);
        const float val = q < 0 ? 0.f : vel[3 * q + comp];
        fine += (dx ? fx : 1.f - fx) * (dy ? fy : 1.f - fy) * (dz ? fz : 1.f - fz) * val;
      }
  if (lv == 0) return fine;
  const float scale = 1.f / (float)(1 << lv);
  const float cgx = gx * scale, cgy = gy * scale, cgz = gz * scale;
  const int cix0 = (int)floorf(cgx), ciy0 = (int)floorf(cgy), ciz0 = (int)floorf(cgz);
  const float cfx = cgx - cix0, cfy = cgy - ciy0, cfz = cgz - ciz0;
  float coarse = 0.f;
  for (int dz = 0; dz <= 1; dz++)
    for (int dy = 0; dy <= 1; dy++)
      for (int dx = 0; dx <= 1; dx++) {
        const int64_t q = mr_idx(g, lv, cix0 + dx, ciy0 + dy, ciz0 + dz);
        const float val = q < 0 ? 0.f : vel[3 * q + comp];
        coarse += (dx ? cfx : 1.f - cfx) * (dy ? cfy : 1.f - cfy) * (dz ? cfz : 1.f - cfz) * val;
      }
  const float cpos[3] = {cgx, cgy, cgz};
  const float d = mr_dist_interp(g, dist, kind, dTransRes * 1024, lv, cpos) / 1024.0f;
  const int stenWidth = 2;
  const float a = (stenWidth / 2.f - 0.f) * 1.73205080756887f * 1.01f;
  const float b = 0.99f * ((float)dTransRes + 2.f) / 1.73205080756887f;
  const float alphaFine = (float)linstep(a, b, d);
  return alphaFine * fine + (1.f - alphaFine) * coarse;
}

void oracle_mr_g2p(int sx, int sy, int sz, int bsx0, const int* level, int dTransRes,
                   oracle_flip_particle* p, int64_t np, const float* vel, const float* velOld,
                   const uint16_t* dist, const int8_t* kind, float alpha) {
  const int nbx = sx / bsx0, nby = sy / bsx0, nbz = sz / bsx0;
  int64_t* off = (int64_t*)malloc(sizeof(int64_t) * (size_t)nbx * nby * nbz);
  oracle_mr_layout(nbx, nby, nbz, bsx0, level, off);
  MRGrid g = {sx, sy, sz, bsx0, nbx, nby, nbz, level, off};
  static const float OFF[3][3] = {{0.f, 0.5f, 0.5f}, {0.5f, 0.f, 0.5f}, {0.5f, 0.5f, 0.f}};
  for (int64_t k = 0; k < np; k++) {
    float pic[3], old[3];
    for (int d = 0; d < 3; d++) {
      pic[d] = mr_interp_comp(&g, vel, dist, kind, dTransRes, p[k].pos, OFF[d], d);
      old[d] = mr_interp_comp(&g, velOld, dist, kind, dTransRes, p[k].pos, OFF[d], d);
    }
    for (int d = 0; d < 3; d++)
      p[k].vel[d] = (1.f - alpha) * pic[d] + alpha * (p[k].vel[d] + (pic[d] - old[d]));
  }
  free(off);
}

/* downsampleVelocity (src/msbg4.cpp:2035-2270): the velocity of MG level m-1
 * restricted to MG level m (1 <= m < nLevels, the sparse MG levels).  At MG
 * level m block b sits at level max(level0[b], m) (getBlockLevel,
 * src/msbg.h:3574-3590); src and dst are packed at MG levels m-1 and m, 3
 * floats per voxel; flags (CellFlags) packed at MG level m.
 *   level0[b] >= m: a copy of the block, 0 in SOLID or VOID cells;
 *   level0[b] <  m: per non-SOLID cell (x, y, z) of level m, the 4x4x4 sum of
 *     w_ijk * f over the level-(m-1) cells (2x-1+i, 2y-1+j, 2z-1+k) clamped to
 *     that level's grid, w = (1,3,3,1)^3 / 512 (G3D_GetGausslikeKernel4x4x4,
 *     src/grid.c:30-75), f from the level-(m-1) block where it exists at MG
 *     level m-1, else the level-m value at (x2/2, y2/2, z2/2); SOLID cells 0.
 * Accumulated in float in the order k, j, i. */
void oracle_mr_downsample_velocity(int sx, int sy, int sz, int bsx0, const int* level0, int m,
                                   const uint16_t* flags, const float* src, float* dst) {
  const int nbx = sx / bsx0, nby = sy / bsx0, nbz = sz / bsx0;
  const int64_t nb = (int64_t)nbx * nby * nbz;
  int* lvA = (int*)malloc(sizeof(int) * (size_t)nb); /* levels at MG m-1 */
  int* lvB = (int*)malloc(sizeof(int) * (size_t)nb); /* levels at MG m */
  int64_t* offA = (int64_t*)malloc(sizeof(int64_t) * (size_t)nb);
  int64_t* offB = (int64_t*)malloc(sizeof(int64_t) * (size_t)nb);
  for (int64_t b = 0; b < nb; b++) {
    lvA[b] = level0[b] > m - 1 ? level0[b] : m - 1;
    lvB[b] = level0[b] > m ? level0[b] : m;
  }
  oracle_mr_layout(nbx, nby, nbz, bsx0, lvA, offA);
  oracle_mr_layout(nbx, nby, nbz, bsx0, lvB, offB);
  const float k1[4] = {1.f, 3.f, 3.f, 1.f};
  float krn[64];
  for (int k = 0; k < 4; k++)
    for (int j = 0; j < 4; j++)
      for (int i = 0; i < 4; i++) krn[i + 4 * j + 16 * k] = (float)((double)(k1[i] * k1[j] * k1[k]) / 512.0);
  MRGrid gA = {sx, sy, sz, bsx0, nbx, nby, nbz, lvA, offA};
  const int fs = m - 1; /* the finer source level */
  const int nsx = sx >> fs, nsy = sy >> fs, nsz = sz >> fs;
  for (int64_t b = 0; b < nb; b++) {
    const int lv = lvB[b], bs = bsx0 >> lv;
    const int bx = (int)(b % nbx), by = (int)((b / nbx) % nby), bz = (int)(b / ((int64_t)nbx * nby));
    const int64_t nv = (int64_t)bs * bs * bs;
    for (int64_t v = 0; v < nv; v++) {
      const uint16_t fl = flags[offB[b] + v];
      float* out = dst + 3 * (offB[b] + v);
      if (level0[b] >= m) {
        const float* in = src + 3 * (offA[b] + v);
        const int zero = (fl & (0x1 | 0x1000)) != 0; /* CELL_SOLID | CELL_VOID */
        for (int c = 0; c < 3; c++) out[c] = zero ? 0.f : in[c];
        continue;
      }
      float val[3] = {0.f, 0.f, 0.f};
      if (!(fl & 0x1)) {
        const int x = bx * bs + (int)(v % bs), y = by * bs + (int)((v / bs) % bs),
                  z = bz * bs + (int)(v / ((int64_t)bs * bs));
        for (int k = 0; k < 4; k++) {
          int z2 = 2 * z - 1 + k;
          z2 = z2 < 0 ? 0 : z2 >= nsz ? nsz - 1 : z2;
          for (int j = 0; j < 4; j++) {
            int y2 = 2 * y - 1 + j;
            y2 = y2 < 0 ? 0 : y2 >= nsy ? nsy - 1 : y2;
            for (int i = 0; i < 4; i++) {
              int x2 = 2 * x - 1 + i;
              x2 = x2 < 0 ? 0 : x2 >= nsx ? nsx - 1 : x2;
              int64_t q = mr_idx(&gA, fs, x2, y2, z2);
              if (q < 0) q = mr_idx(&gA, fs + 1, x2 / 2, y2 / 2, z2 / 2);
              const float w = krn[i + 4 * j + 16 * k];
              for (int c = 0; c < 3; c++) val[c] += (q < 0 ? 0.f : src[3 * q + c]) * w;
            }
          }
        }
      }
      for (int c = 0; c < 3; c++) out[c] = val[c];
    }
  }
  free(lvA);
  free(lvB);
  free(offA);
  free(offB);
}
