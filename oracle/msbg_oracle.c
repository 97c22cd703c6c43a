/*
 * msbg_oracle.c — CPU restatement of the reference MSBG solver path.
 *
 * TEST INFRASTRUCTURE ONLY (the checker, never the product; see
 * msbg_oracle.h).  Plain C, FP32 arithmetic in the reference's expression
 * order with contraction disabled (-ffp-contract=off), so it is the
 * un-fused form of the reference's float expressions.
 */
#include "msbg_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* Block colour, src/msbg.h:642-646. */
static inline int colour8(int bx, int by, int bz) {
  return (bx & 1) + ((by & 1) << 1) + ((bz & 1) << 2);
}

/* Fill an (bsx+2)^3 halo copy of block (bx,by,bz), src/halo.cpp:266-479:
 * in-domain voxel whose block is non-NULL -> that block's value (a const
 * block yields its constant); NULL block or outside the domain ->
 * OPT_BC_NEUMANN: own block's value at the coordinates clamped to the own
 * block (src/halo.h:280-287). */
static void fill_halo(int nbx, int nby, int nbz, int bsx, const int8_t* kind,
                      const int64_t* slot, float emptyVal, float fullVal,
                      const float* values, int bx, int by, int bz, float* h) {
  const int hsx = bsx + 2, nv = bsx * bsx * bsx;
  const int sx = nbx * bsx, sy = nby * bsx, sz = nbz * bsx;
  const int64_t bid0 = bx + (int64_t)nbx * (by + (int64_t)nby * bz);
  const float* own = values + slot[bid0] * nv;
  const int x0 = bx * bsx, y0 = by * bsx, z0 = bz * bsx;
  for (int hz = 0; hz < hsx; hz++)
    for (int hy = 0; hy < hsx; hy++)
      for (int hx = 0; hx < hsx; hx++) {
        int x = x0 + hx - 1, y = y0 + hy - 1, z = z0 + hz - 1;
        float v;
        int valid = 0;
        if (x >= 0 && y >= 0 && z >= 0 && x < sx && y < sy && z < sz) {
          int64_t b = x / bsx + (int64_t)nbx * (y / bsx + (int64_t)nby * (z / bsx));
          int vid = (x % bsx) + bsx * ((y % bsx) + bsx * (z % bsx));
          switch (kind[b]) {
            case 1: v = values[slot[b] * nv + vid]; valid = 1; break;
            case 2: v = emptyVal; valid = 1; break;
            case 3: v = fullVal; valid = 1; break;
            default: break;
          }
        }
        if (!valid) {
          int cx = x < x0 ? x0 : (x > x0 + bsx - 1 ? x0 + bsx - 1 : x);
          int cy = y < y0 ? y0 : (y > y0 + bsx - 1 ? y0 + bsx - 1 : y);
          int cz = z < z0 ? z0 : (z > z0 + bsx - 1 ? z0 + bsx - 1 : z);
          v = own[(cx - x0) + bsx * ((cy - y0) + bsx * (cz - z0))];
        }
        h[hx + hsx * (hy + hsx * hz)] = v;
      }
}

/* MCF stencil on one block, src/msbg4.cpp:559-637 (laplTyp 4) followed by
 * the [0,1] clamp (819-825) when requested. */
static void mcf_block(int bsx, const float* h, float* out, float dt, int clamp01) {
  const int hsx = bsx + 2, hsx2 = hsx * hsx;
#define F_(dx, dy, dz) p[(dx) + (dy)*hsx + (dz)*hsx2]
  for (int vz = 0; vz < bsx; vz++)
    for (int vy = 0; vy < bsx; vy++)
      for (int vx = 0; vx < bsx; vx++) {
        const float* p = h + (vx + 1) + hsx * ((vy + 1) + hsx * (vz + 1));
        float f0 = F_(0, 0, 0), f1 = F_(-1, 0, 0), f2 = F_(1, 0, 0), f3 = F_(0, -1, 0),
              f4 = F_(0, 1, 0), f5 = F_(0, 0, -1), f6 = F_(0, 0, 1);
        float fx = 0.5f * (f2 - f1), fy = 0.5f * (f4 - f3), fz = 0.5f * (f6 - f5);
        float fxx = f1 + f2 - 2 * f0, fyy = f3 + f4 - 2 * f0, fzz = f5 + f6 - 2 * f0;
        float fy_right = (F_(1, 1, 0) - F_(1, -1, 0)) * 0.5f;
        float fy_left = (F_(-1, 1, 0) - F_(-1, -1, 0)) * 0.5f;
        float fz_right = (F_(1, 0, 1) - F_(1, 0, -1)) * 0.5f;
        float fz_left = (F_(-1, 0, 1) - F_(-1, 0, -1)) * 0.5f;
        float fz_up = (F_(0, 1, 1) - F_(0, 1, -1)) * 0.5f;
        float fz_down = (F_(0, -1, 1) - F_(0, -1, -1)) * 0.5f;
        float fyx = (fy_right - fy_left) * 0.5f;
        float fzx = (fz_right - fz_left) * 0.5f;
        float fzy = (fz_up - fz_down) * 0.5f;
        float H = (fy * fy + fz * fz) * fxx + (fx * fx + fz * fz) * fyy +
                  (fx * fx + fy * fy) * fzz -
                  2.0f * (fx * fy * fyx + fx * fz * fzx + fy * fz * fzy);
        float g = fx * fx + fy * fy + fz * fz;
        H = g > 1e-7f ? H / g : 0.0f;
        float D = dt * H;
        D = fminf(fmaxf(D, -0.1f), 0.1f);
        float phi = f0 + D;
        if (clamp01) phi = fminf(fmaxf(phi, 0.0f), 1.0f);
        out[vx + bsx * (vy + bsx * vz)] = phi;
      }
#undef F_
}

int oracle_mcf(int nbx, int nby, int nbz, int bsx, const int8_t* kind,
               float emptyVal, float fullVal, float* values, const int* update,
               int nUpdate, int numIter, float dt, int clamp01, int exactIter) {
  if (nbx <= 0 || nby <= 0 || nbz <= 0 || bsx <= 0 || !kind || !values) return 5;
  const int64_t nb = (int64_t)nbx * nby * nbz;
  const int nv = bsx * bsx * bsx, hsx = bsx + 2;
  int64_t* slot = (int64_t*)malloc(sizeof(int64_t) * nb);
  if (!slot) return 2;
  int64_t s = 0;
  for (int64_t b = 0; b < nb; b++) slot[b] = kind[b] == 1 ? s++ : -1;
  for (int i = 0; i < nUpdate; i++)
    if (update[i] < 0 || update[i] >= nb || kind[update[i]] != 1) {
      free(slot);
      return 5;
    }
  int nIter = numIter;
  if (!exactIter && (nIter % 2) == 1) nIter++; /* src/msbg4.cpp:150-152 */
  for (int it = 0; it < nIter; it++) {
    for (int col = 0; col < 8; col++) {
      /* Same-colour blocks are never 26-neighbours, so processing them one
       * after another equals the reference's parallel pass. */
#pragma omp parallel
      {
        float* h = (float*)malloc(sizeof(float) * hsx * hsx * hsx);
#pragma omp for schedule(dynamic, 4)
        for (int i = 0; i < nUpdate; i++) {
          int bid = update[i];
          int bx = bid % nbx, by = (bid / nbx) % nby, bz = bid / (nbx * nby);
          if (colour8(bx, by, bz) != col) continue;
          fill_halo(nbx, nby, nbz, bsx, kind, slot, emptyVal, fullVal, values, bx, by, bz, h);
          mcf_block(bsx, h, values + slot[bid] * nv, dt, clamp01);
        }
        free(h);
      }
    }
  }
  free(slot);
  return 0;
}
