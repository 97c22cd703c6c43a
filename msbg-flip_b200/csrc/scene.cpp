// Seeded synthetic workloads (host side).  See include/msbg_scene.h.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "msbg_gpu.h"
#include "msbg_scene.h"

namespace {

struct SplitMix64 {
  uint64_t s;
  explicit SplitMix64(uint64_t seed) : s(seed) {}
  uint64_t next() {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  }
  double uniform() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }
};

struct Sphere {
  double cx, cy, cz, r;
};

// Distance bounds of an axis-aligned box [lo,hi]^3 to point c.
inline void box_dist(const double lo[3], const double hi[3], const Sphere& s,
                     double& dmin, double& dmax) {
  const double c[3] = {s.cx, s.cy, s.cz};
  double a = 0, b = 0;
  for (int k = 0; k < 3; k++) {
    double d0 = std::max({lo[k] - c[k], 0.0, c[k] - hi[k]});
    double d1 = std::max(std::fabs(c[k] - lo[k]), std::fabs(c[k] - hi[k]));
    a += d0 * d0;
    b += d1 * d1;
  }
  dmin = std::sqrt(a);
  dmax = std::sqrt(b);
}

}  // namespace

extern "C" int msbg_scene_sphere_sdf(int res, int bsx, int nSpheres, float rmin,
                                     float rmax, float band, int dilate,
                                     uint64_t seed, int8_t* kind, float* values,
                                     int64_t* nValueBlocks) {
  if (res <= 0 || bsx <= 0 || res % bsx || nSpheres <= 0 || !kind || dilate < 0)
    return MSBG_EINVARG;
  SplitMix64 rng(seed);
  std::vector<Sphere> sp(nSpheres);
  for (auto& s : sp) {
    s.cx = rng.uniform() * res;
    s.cy = rng.uniform() * res;
    s.cz = rng.uniform() * res;
    s.r = rmin + rng.uniform() * (rmax - rmin);
  }
  const int nb1 = res / bsx;
  const int64_t nb = (int64_t)nb1 * nb1 * nb1;
  // Pass 1: classify blocks by bounds of phi over the block's voxel centres.
  std::vector<int8_t> band_blk(nb, 0), sign_blk(nb, 0);
#pragma omp parallel for schedule(dynamic, 64)
  for (int64_t bid = 0; bid < nb; bid++) {
    int bx = (int)(bid % nb1), by = (int)((bid / nb1) % nb1), bz = (int)(bid / ((int64_t)nb1 * nb1));
    double lo[3] = {bx * bsx + 0.5, by * bsx + 0.5, bz * bsx + 0.5};
    double hi[3] = {lo[0] + bsx - 1, lo[1] + bsx - 1, lo[2] + bsx - 1};
    double pmin = 1e300, pmax = 1e300;
    for (const auto& s : sp) {
      double dmin, dmax;
      box_dist(lo, hi, s, dmin, dmax);
      pmin = std::min(pmin, dmin - s.r);
      pmax = std::min(pmax, dmax - s.r);
    }
    // phi over the block lies in [pmin, pmax]
    bool maybe = !(pmin > band || pmax < -band);
    int8_t isband = 0;
    if (maybe) {
      // exact check on voxels (with sphere pruning)
      std::vector<const Sphere*> cand;
      for (const auto& s : sp) {
        double dmin, dmax;
        box_dist(lo, hi, s, dmin, dmax);
        if (dmin - s.r <= pmax) cand.push_back(&s);
      }
      for (int vz = 0; vz < bsx && !isband; vz++)
        for (int vy = 0; vy < bsx && !isband; vy++)
          for (int vx = 0; vx < bsx; vx++) {
            double x = lo[0] + vx, y = lo[1] + vy, z = lo[2] + vz, p = 1e300;
            for (const Sphere* s : cand) {
              double dx = x - s->cx, dy = y - s->cy, dz = z - s->cz;
              p = std::min(p, std::sqrt(dx * dx + dy * dy + dz * dz) - s->r);
            }
            float pf = (float)p;
            if (std::fabs(pf) <= band) {
              isband = 1;
              break;
            }
          }
    }
    band_blk[bid] = isband;
    sign_blk[bid] = (pmin + pmax) * 0.5 < 0 ? -1 : 1;
  }
  // Pass 2: dilate and assign kinds.
  int64_t nval = 0;
  for (int64_t bid = 0; bid < nb; bid++) {
    int bx = (int)(bid % nb1), by = (int)((bid / nb1) % nb1), bz = (int)(bid / ((int64_t)nb1 * nb1));
    bool v = false;
    for (int dz = -dilate; dz <= dilate && !v; dz++)
      for (int dy = -dilate; dy <= dilate && !v; dy++)
        for (int dx = -dilate; dx <= dilate; dx++) {
          int x = bx + dx, y = by + dy, z = bz + dz;
          if (x < 0 || y < 0 || z < 0 || x >= nb1 || y >= nb1 || z >= nb1) continue;
          if (band_blk[x + (int64_t)y * nb1 + (int64_t)z * nb1 * nb1]) {
            v = true;
            break;
          }
        }
    kind[bid] = v ? MSBG_BLOCK_VALUE : (sign_blk[bid] > 0 ? MSBG_BLOCK_EMPTY : MSBG_BLOCK_FULL);
    nval += v;
  }
  if (nValueBlocks) *nValueBlocks = nval;
  if (!values) return MSBG_OK;
  // Pass 3: exact values of value blocks.
  std::vector<int64_t> slot(nb, -1);
  {
    int64_t s = 0;
    for (int64_t bid = 0; bid < nb; bid++)
      if (kind[bid] == MSBG_BLOCK_VALUE) slot[bid] = s++;
  }
  const int nv = bsx * bsx * bsx;
#pragma omp parallel for schedule(dynamic, 16)
  for (int64_t bid = 0; bid < nb; bid++) {
    if (slot[bid] < 0) continue;
    int bx = (int)(bid % nb1), by = (int)((bid / nb1) % nb1), bz = (int)(bid / ((int64_t)nb1 * nb1));
    double lo[3] = {bx * bsx + 0.5, by * bsx + 0.5, bz * bsx + 0.5};
    double hi[3] = {lo[0] + bsx - 1, lo[1] + bsx - 1, lo[2] + bsx - 1};
    double pmax = 1e300;
    for (const auto& s : sp) {
      double dmin, dmax;
      box_dist(lo, hi, s, dmin, dmax);
      pmax = std::min(pmax, dmax - s.r);
    }
    std::vector<const Sphere*> cand;
    for (const auto& s : sp) {
      double dmin, dmax;
      box_dist(lo, hi, s, dmin, dmax);
      if (dmin - s.r <= pmax) cand.push_back(&s);
    }
    float* out = values + slot[bid] * nv;
    for (int vz = 0; vz < bsx; vz++)
      for (int vy = 0; vy < bsx; vy++)
        for (int vx = 0; vx < bsx; vx++) {
          double x = lo[0] + vx, y = lo[1] + vy, z = lo[2] + vz, p = 1e300;
          for (const Sphere* s : cand) {
            double dx = x - s->cx, dy = y - s->cy, dz = z - s->cz;
            p = std::min(p, std::sqrt(dx * dx + dy * dy + dz * dz) - s->r);
          }
          out[vx + bsx * (vy + bsx * vz)] = (float)p;
        }
  }
  return MSBG_OK;
}
