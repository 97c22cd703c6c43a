/* CPU restatement of the FLIP transfers around the pressure solve
 * (TEST INFRASTRUCTURE ONLY: the oracle the GPU kernels of csrc/flip.cu are
 * checked against; nothing of the product calls it).
 *
 * Follows FlipSimulation in src/flip_sim.cpp of the reference, on a grid of
 * sx*sy*sz voxels stored in bsx^3 blocks (blocks in bid order, voxel
 * vid = x + y*bsx + z*bsx*bsx), every block present (the single-level grid of
 * the reference's flip_sim):
 *   oracle_flip_p2g       particleToGrid             src/flip_sim.cpp:579-831
 *   oracle_flip_gravity   applyGravity               src/flip_sim.cpp:832-857
 *   oracle_flip_gradient  pressure-gradient update   src/flip_sim.cpp:1316-1349
 *   oracle_flip_g2p       gridToParticle with the level-0 branch of
 *                         interpVec3MSBG              src/flip_sim.cpp:1354-1395, 1526-1545
 * Vector channels hold 3 floats per voxel: the MAC face values (u, v, w) of
 * the voxel's lower x, y and z faces.  Float arithmetic in the reference's
 * order, compiled without contraction (-ffp-contract=off).
 *
 * Parity status: the reference's flip_sim.cpp includes the headers of hypre,
 * an external library absent here, so it is not compiled; this restatement
 * is not pinned to the reference's own output ("parity unpinned"). */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "msbg_oracle.h"

typedef struct {
  int sx, sy, sz, bsx, nbx, nby;
} FGrid;

static int64_t fidx(const FGrid* g, int x, int y, int z) {
  if (x < 0 || y < 0 || z < 0 || x >= g->sx || y >= g->sy || z >= g->sz) return -1;
  const int b = g->bsx;
  const int64_t bid = (x / b) + (int64_t)g->nbx * ((y / b) + (int64_t)g->nby * (z / b));
  return bid * b * b * b + (x % b) + (int64_t)b * ((y % b) + (int64_t)b * (z % b));
}

static void fgrid(FGrid* g, int sx, int sy, int sz, int bsx) {
  g->sx = sx;
  g->sy = sy;
  g->sz = sz;
  g->bsx = bsx;
  g->nbx = sx / bsx;
  g->nby = sy / bsx;
}

/* one staggered component: trilinear weights of the 8 faces around
 * (pos - offset), as the reference's U/V/W loops */
static void scatter_comp(const FGrid* g, const float pos[3], const float off[3], float vel,
                         float mp, float* acc_v, float* acc_w, float* acc_r) {
  const float gx = pos[0] - off[0], gy = pos[1] - off[1], gz = pos[2] - off[2];
  const int ix0 = (int)floorf(gx), iy0 = (int)floorf(gy), iz0 = (int)floorf(gz);
  const float fx = gx - ix0, fy = gy - iy0, fz = gz - iz0;
  for (int dz = 0; dz <= 1; dz++)
    for (int dy = 0; dy <= 1; dy++)
      for (int dx = 0; dx <= 1; dx++) {
        const float w = (dx ? fx : 1.f - fx) * (dy ? fy : 1.f - fy) * (dz ? fz : 1.f - fz);
        const int64_t i = fidx(g, ix0 + dx, iy0 + dy, iz0 + dz);
        if (i < 0) continue;
        acc_v[i] += vel * w;
        acc_w[i] += w;
        acc_r[i] += mp * w;
      }
}

int oracle_flip_p2g(int sx, int sy, int sz, int bsx, const oracle_flip_particle* p, int64_t np,
                    const oracle_flip_params* c, float* vel, float* mass, float* beta,
                    uint8_t* activeBlock) {
  FGrid g;
  fgrid(&g, sx, sy, sz, bsx);
  const int64_t n = (int64_t)sx * sy * sz;
  float* acc = (float*)calloc((size_t)n * 9, sizeof(float)); /* vx vy vz wu wv ww ru rv rw */
  int* liq = (int*)calloc((size_t)n, sizeof(int));
  if (!acc || !liq) {
    free(acc);
    free(liq);
    return 2;
  }
  memset(mass, 0, sizeof(float) * n);
  static const float OFF[3][3] = {{0.f, 0.5f, 0.5f}, {0.5f, 0.f, 0.5f}, {0.5f, 0.5f, 0.f}};
  for (int64_t k = 0; k < np; k++) {
    const oracle_flip_particle* q = &p[k];
    /* a particle without a finite position reaches no cell (the reference's
     * float-to-int conversion of it is undefined) */
    if (!isfinite(q->pos[0]) || !isfinite(q->pos[1]) || !isfinite(q->pos[2])) continue;
    const float mp = q->phase == 0 ? c->rhoL : c->rhoG;
    const int64_t ci =
        fidx(&g, (int)floorf(q->pos[0]), (int)floorf(q->pos[1]), (int)floorf(q->pos[2]));
    if (ci >= 0) {
      mass[ci] += 1.f;
      if (q->phase == 0) liq[ci]++;
    }
    for (int d = 0; d < 3; d++)
      scatter_comp(&g, q->pos, OFF[d], q->vel[d], mp, acc + (size_t)d * n,
                   acc + (size_t)(3 + d) * n, acc + (size_t)(6 + d) * n);
  }
  /* phi of the two-phase density, then beta = max(1/rho, betaMin) */
  const float rt0 = (float)c->particlesPerVoxel;
  const float etaPhi = logf(c->rhoL / c->rhoG);
  const float rtMin = etaPhi * c->rhoG * rt0;
  const float phiDen = c->alphaPhi * rt0 * c->rhoL;
  const int nb = (sx / bsx) * (sy / bsx) * (sz / bsx);
  for (int b = 0; b < nb; b++) activeBlock[b] = 0;
  for (int z = 0; z < sz; z++)
    for (int y = 0; y < sy; y++)
      for (int x = 0; x < sx; x++) {
        const int64_t i = fidx(&g, x, y, z);
        for (int d = 0; d < 3; d++) {
          const float w = acc[(size_t)(3 + d) * n + i];
          vel[3 * i + d] = w > c->massEps ? acc[(size_t)d * n + i] / w : 0.f;
        }
        if (mass[i] > c->massEps) activeBlock[i / ((int64_t)bsx * bsx * bsx)] = 1;
        float phi[3];
        for (int d = 0; d < 3; d++) {
          const float rt = acc[(size_t)(6 + d) * n + i];
          float v = 0.f;
          if (!(rt < rtMin)) {
            v = sqrtf(fmaxf(rt - rtMin, 0.f) / phiDen);
            v = fminf(v, 1.f);
          }
          phi[d] = v;
        }
        /* interface clamp: both cells of a face liquid -> 1, both air -> 0 */
        for (int d = 0; d < 3; d++) {
          int ph[2];
          for (int s = 0; s < 2; s++) {
            const int64_t j = fidx(&g, x - (d == 0 && !s), y - (d == 1 && !s), z - (d == 2 && !s));
            if (j < 0 || !(mass[j] > c->massEps))
              ph[s] = -1;
            else
              ph[s] = liq[j] * 2 > (int)(mass[j] + 0.5f) ? 0 : 1;
          }
          if (ph[0] == 0 && ph[1] == 0)
            phi[d] = 1.f;
          else if (ph[0] == 1 && ph[1] == 1)
            phi[d] = 0.f;
          const float rho = c->rhoG + phi[d] * (c->rhoL - c->rhoG);
          beta[3 * i + d] = fmaxf(1.f / rho, c->betaMin);
        }
      }
  free(acc);
  free(liq);
  return 0;
}

static int fluid(const FGrid* g, const float* mass, int x, int y, int z, float eps) {
  const int64_t i = fidx(g, x, y, z);
  return i >= 0 && mass[i] > eps;
}

void oracle_flip_gravity(int sx, int sy, int sz, int bsx, float* vel, float* velOld,
                         const float* mass, float gravity, float dt, float massEps) {
  FGrid g;
  fgrid(&g, sx, sy, sz, bsx);
  const int64_t n = (int64_t)sx * sy * sz;
  memcpy(velOld, vel, sizeof(float) * 3 * n);
  for (int z = 0; z < sz; z++)
    for (int y = 0; y < sy; y++)
      for (int x = 0; x < sx; x++) {
        const int lo = y > 0 && fluid(&g, mass, x, y - 1, z, massEps);
        const int hi = fluid(&g, mass, x, y, z, massEps);
        if (lo || hi) vel[3 * fidx(&g, x, y, z) + 1] += gravity * dt;
      }
  /* the reference's wall faces (src/flip_sim.cpp:846-853) */
  for (int z = 0; z < sz; z++)
    for (int y = 0; y < sy; y++) {
      vel[3 * fidx(&g, 0, y, z) + 0] = 0.f;
      vel[3 * fidx(&g, sx - 1, y, z) + 0] = 0.f;
    }
  for (int z = 0; z < sz; z++)
    for (int x = 0; x < sx; x++) vel[3 * fidx(&g, x, 0, z) + 1] = 0.f;
  for (int y = 0; y < sy; y++)
    for (int x = 0; x < sx; x++) {
      vel[3 * fidx(&g, x, y, 0) + 2] = 0.f;
      vel[3 * fidx(&g, x, y, sz - 1) + 2] = 0.f;
    }
}

void oracle_flip_gradient(int sx, int sy, int sz, int bsx, float* vel, const float* mass,
                          const float* beta, const float* pressure, float dt, float massEps) {
  FGrid g;
  fgrid(&g, sx, sy, sz, bsx);
  for (int z = 0; z < sz; z++)
    for (int y = 0; y < sy; y++)
      for (int x = 0; x < sx; x++) {
        const int64_t i = fidx(&g, x, y, z);
        const int p[3] = {x, y, z};
        for (int d = 0; d < 3; d++) {
          if (p[d] == 0) {
            vel[3 * i + d] = 0.f;
            continue;
          }
          const int64_t j = fidx(&g, x - (d == 0), y - (d == 1), z - (d == 2));
          const int fa = mass[j] > massEps, fb = mass[i] > massEps;
          if (!fa && !fb) {
            vel[3 * i + d] = 0.f;
            continue;
          }
          const float pa = fa ? pressure[j] : 0.f, pb = fb ? pressure[i] : 0.f;
          const float v = vel[3 * i + d] - dt * beta[3 * i + d] * (pb - pa);
          vel[3 * i + d] = isfinite(v) ? v : 0.f;
        }
      }
}

static float interp_comp(const FGrid* g, const float* vel, const float pos[3], const float off[3],
                         int comp) {
  if (!isfinite(pos[0]) || !isfinite(pos[1]) || !isfinite(pos[2])) return 0.f; /* no cell */
  const float gx = pos[0] - off[0], gy = pos[1] - off[1], gz = pos[2] - off[2];
  const int ix0 = (int)floorf(gx), iy0 = (int)floorf(gy), iz0 = (int)floorf(gz);
  const float fx = gx - ix0, fy = gy - iy0, fz = gz - iz0;
  float sum = 0.f;
  for (int dz = 0; dz <= 1; dz++)
    for (int dy = 0; dy <= 1; dy++)
      for (int dx = 0; dx <= 1; dx++) {
        const int64_t i = fidx(g, ix0 + dx, iy0 + dy, iz0 + dz);
        const float v = i < 0 ? 0.f : vel[3 * i + comp];
        sum += (dx ? fx : 1.f - fx) * (dy ? fy : 1.f - fy) * (dz ? fz : 1.f - fz) * v;
      }
  return sum;
}

void oracle_flip_g2p(int sx, int sy, int sz, int bsx, oracle_flip_particle* p, int64_t np,
                     const float* vel, const float* velOld, float alpha) {
  FGrid g;
  fgrid(&g, sx, sy, sz, bsx);
  static const float OFF[3][3] = {{0.f, 0.5f, 0.5f}, {0.5f, 0.f, 0.5f}, {0.5f, 0.5f, 0.f}};
  for (int64_t k = 0; k < np; k++) {
    float pic[3], old[3];
    for (int d = 0; d < 3; d++) {
      pic[d] = interp_comp(&g, vel, p[k].pos, OFF[d], d);
      old[d] = interp_comp(&g, velOld, p[k].pos, OFF[d], d);
    }
    for (int d = 0; d < 3; d++)
      p[k].vel[d] = (1.f - alpha) * pic[d] + alpha * (p[k].vel[d] + (pic[d] - old[d]));
  }
}
