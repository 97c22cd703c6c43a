/* CPU restatement of the reference's particle splatting into a 16-bit
 * render-density channel (TEST INFRASTRUCTURE ONLY: the oracle the GPU
 * kernels of csrc/splat.cu are checked against, and the CPU baseline's
 * port; nothing of the product calls it).
 *
 * Follows msbg_test_sparse in src/msbg_demo.cpp of the reference:
 *   oracle_splat_domain  the particle domain test: isInDomainRange
 *                        (src/msbg.h:2937-2945) with the bounds of
 *                        src/sbg.cpp:287-316 (beps 1e-4: sbg.cpp is compiled
 *                        without PARTICLE_QUANT_POS, which only
 *                        src/msbgcell.h defines), then inRange of the
 *                        truncated position (src/msbg_demo.cpp:358-360)
 *   oracle_splat_mark    active-block marking     src/msbg_demo.cpp:366-379
 *   oracle_splat         allocation of the value blocks at 65535, the
 *                        8-colour lock-free splat and the distance
 *                        finalisation              src/msbg_demo.cpp:465-684
 * The grid is sx*sy*sz voxels in bsx^3 blocks (blocks in bid order, voxel
 * vid = x + y*bsx + z*bsx*bsx); value blocks are packed in ascending bid
 * order.
 *
 * Arithmetic: the squared distance is the one the reference's build computes
 * (-O2 -ffast-math -march=x86-64-v3): dz*dz + dy*dy contracted into
 * fmaf(dy, dy, dz*dz) and "+ dx*dx" into fmaf(dx, dx, .); every other
 * expression in source order without contraction (this file is compiled with
 * -ffp-contract=off).  Parity: pinned against the reference demo itself run
 * through oracle/ref/splat_harness.cpp (fixtures under tests/golden/). */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "msbg_oracle.h"

void oracle_splat_domain(int sx, int sy, int sz, float lo[3], float hi[3]) {
  /* the first try of the loop at src/sbg.cpp:291-303 already satisfies its
   * test for every grid size */
  const float beps = 1e-4f;
  const int s[3] = {sx, sy, sz};
  for (int k = 0; k < 3; k++) {
    lo[k] = 0.0f + beps;
    hi[k] = (float)s[k] - beps;
  }
}

/* 1 when the demo keeps the particle (a finite position inside the domain
 * bounds whose truncated cell lies in the grid); its cell in c[3] */
static int splat_keep(const float* p, const float lo[3], const float hi[3], const int s[3],
                      int c[3]) {
  for (int k = 0; k < 3; k++) {
    if (!isfinite(p[k])) return 0;
    if (p[k] < lo[k] || p[k] > hi[k]) return 0;
  }
  for (int k = 0; k < 3; k++) {
    c[k] = (int)p[k];
    if (c[k] < 0 || c[k] > s[k] - 1) return 0;
  }
  return 1;
}

int oracle_splat_mark(int sx, int sy, int sz, int bsx, const float* pos, int64_t n,
                      float rParticle, float nbDist, int8_t* active) {
  if (bsx <= 0 || sx % bsx || sy % bsx || sz % bsx) return 1;
  const int nb[3] = {sx / bsx, sy / bsx, sz / bsx};
  const int s[3] = {sx, sy, sz};
  float lo[3], hi[3];
  oracle_splat_domain(sx, sy, sz, lo, hi);
  memset(active, 0, (size_t)nb[0] * nb[1] * nb[2]);
  const float rScan = rParticle + nbDist;
  const float toBlock = 1.0f / (float)bsx, rScanBsx = rScan / (float)bsx;
  for (int64_t i = 0; i < n; i++) {
    const float* p = pos + 3 * i;
    int c[3];
    if (!splat_keep(p, lo, hi, s, c)) continue;
    int b1[3], b2[3];
    for (int k = 0; k < 3; k++) {
      const float bp = p[k] * toBlock;
      int a = (int)(bp - rScanBsx), b = (int)(bp + rScanBsx);
      b1[k] = a < 0 ? 0 : a;
      b2[k] = b > nb[k] - 1 ? nb[k] - 1 : b;
    }
    for (int bz = b1[2]; bz <= b2[2]; bz++)
      for (int by = b1[1]; by <= b2[1]; by++)
        for (int bx = b1[0]; bx <= b2[0]; bx++)
          active[bx + (int64_t)nb[0] * (by + (int64_t)nb[1] * bz)] = 1;
  }
  return 0;
}

static uint16_t dens_from_float(float f) { /* renderDensFromFloat_<uint16_t> */
  return (uint16_t)(int)roundf(f * 65535.0f);
}

/* MT_LINSTEPF, src/mtool.h:400-409 */
static float linstep(float a, float b, float x) {
  if (x < a) return 0;
  if (x >= b) return 1;
  return (x - a) / (b - a);
}

uint16_t oracle_splat_finalize_value(uint16_t q, float rParticle, float nbDist) {
  const float rScan = rParticle + nbDist, distSqMax = rScan * rScan;
  float distSq = (float)q * (1.f / 65535.f); /* renderDensToFloat_<uint16_t> */
  if (!(distSq < 0.999f)) return 0;
  distSq *= distSqMax;
  const float dist = sqrtf(distSq) - rParticle;
  const float f = 1.0f - linstep(-rParticle, rParticle + nbDist, dist);
  return dens_from_float(f);
}

int oracle_splat(int sx, int sy, int sz, int bsx, const int8_t* kind, const float* pos,
                 int64_t n, float rParticle, float nbDist, int finalize, uint16_t* out) {
  if (bsx <= 0 || sx % bsx || sy % bsx || sz % bsx) return 1;
  const int nb[3] = {sx / bsx, sy / bsx, sz / bsx};
  const int64_t nBlocks = (int64_t)nb[0] * nb[1] * nb[2];
  const int s[3] = {sx, sy, sz};
  const int64_t nv = (int64_t)bsx * bsx * bsx;
  int64_t* slot = (int64_t*)malloc(sizeof(int64_t) * nBlocks);
  int64_t* head = (int64_t*)malloc(sizeof(int64_t) * nBlocks);
  int64_t* next = (int64_t*)malloc(sizeof(int64_t) * (n > 0 ? n : 1));
  if (!slot || !head || !next) {
    free(slot);
    free(head);
    free(next);
    return 2;
  }
  int64_t nValue = 0;
  for (int64_t b = 0; b < nBlocks; b++) {
    slot[b] = kind[b] == 1 ? nValue++ : -1;
    head[b] = -1;
  }
  for (int64_t i = 0; i < nValue * nv; i++) out[i] = 65535; /* renderDensFromFloat_(1) */

  /* per-block particle lists of the particles' own blocks (pushToListMonotonic) */
  float lo[3], hi[3];
  oracle_splat_domain(sx, sy, sz, lo, hi);
  for (int64_t i = 0; i < n; i++) {
    int c[3];
    if (!splat_keep(pos + 3 * i, lo, hi, s, c)) continue;
    const int64_t b = c[0] / bsx + (int64_t)nb[0] * (c[1] / bsx + (int64_t)nb[1] * (c[2] / bsx));
    next[i] = head[b];
    head[b] = i;
  }

  const float rScan = rParticle + nbDist;
  const float distSqMax = rScan * rScan, distSqMaxInv = 1.0f / distSqMax;
  /* colour = (bx&1) + 2(by&1) + 4(bz&1) (getBlockColor8, src/msbg.h:642-646):
   * blocks of one colour are two apart, so their particles' writes (within
   * rScan + 0.5 < bsx of the own block) never meet */
  for (int col = 0; col < 8; col++) {
#pragma omp parallel for schedule(dynamic, 4)
    for (int64_t b = 0; b < nBlocks; b++) {
      const int bx = (int)(b % nb[0]), by = (int)((b / nb[0]) % nb[1]),
                bz = (int)(b / ((int64_t)nb[0] * nb[1]));
      if (slot[b] < 0 || ((bx & 1) + ((by & 1) << 1) + ((bz & 1) << 2)) != col) continue;
      for (int64_t i = head[b]; i >= 0; i = next[i]) {
        const float* p = pos + 3 * i;
        int i1[3], i2[3];
        float p0[3];
        for (int k = 0; k < 3; k++) {
          const int a = (int)ceilf(p[k] - rScan - 0.5f), e = (int)floorf(p[k] + rScan - 0.5f);
          i1[k] = a < 0 ? 0 : a;
          i2[k] = e > s[k] - 1 ? s[k] - 1 : e;
          p0[k] = p[k] - 0.5f;
        }
        for (int iz = i1[2]; iz <= i2[2]; iz++) {
          const float dz = (float)iz - p0[2];
          for (int iy = i1[1]; iy <= i2[1]; iy++) {
            const float dy = (float)iy - p0[1];
            const float distSqZY = fmaf(dy, dy, dz * dz);
            for (int ix = i1[0]; ix <= i2[0]; ix++) {
              const float dx = (float)ix - p0[0];
              const float distSq = fmaf(dx, dx, distSqZY);
              if (distSq > distSqMax) continue;
              const int64_t vb =
                  ix / bsx + (int64_t)nb[0] * (iy / bsx + (int64_t)nb[1] * (iz / bsx));
              if (slot[vb] < 0) goto loop_exit; /* the demo leaves the particle here */
              {
                uint16_t* d = out + slot[vb] * nv + (ix % bsx) +
                              (int64_t)bsx * ((iy % bsx) + (int64_t)bsx * (iz % bsx));
                const uint16_t q = dens_from_float(distSq * distSqMaxInv);
                if (q < *d) *d = q;
              }
            }
          }
        }
      loop_exit:;
      }
    }
  }
  if (finalize) {
#pragma omp parallel for
    for (int64_t i = 0; i < nValue * nv; i++)
      out[i] = oracle_splat_finalize_value(out[i], rParticle, nbDist);
  }
  free(slot);
  free(head);
  free(next);
  return 0;
}
