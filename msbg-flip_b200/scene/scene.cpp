// Seeded synthetic workloads (host side).  See include/msbg_scene.h.
//
// Built into its own library, libmsbg_scene.so, apart from the solver
// library: the tests, the benchmark and the reference CPU baseline all load
// it to produce identical inputs, and the reference's timed path never loads
// the solver library.
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

// ---------------------------------------------------------------------------
// Free-surface pressure problem (see include/msbg_scene.h).
// ---------------------------------------------------------------------------
struct msbg_pressure_scene {
  int res, bsx0, nLevels;
  float zLiquid, band;
  // free-surface height per (x, y) column at the cell centre, in voxels
  // (a plane z = zLiquid * res, or that plane plus the waves)
  std::vector<double> surf;
  std::vector<Sphere> spheres;
  struct Box { double lo[3], hi[3]; };
  std::vector<Box> boxes;
  struct Mode { int k[3]; double a[3], phi; double coef; };  // div = coef*cos(theta)
  std::vector<Mode> modes;
  std::vector<int> levels;
  // Per mode and axis, exp(i w k_d (x + 0.5)) for every cell index x, and
  // coef * exp(i phi): cos(theta) of a cell is the real part of a product of
  // table entries (the callbacks are sampled once per cell, so this replaces
  // 16 cosines by 16 complex products).
  std::vector<double> etab;  // [axis][res][mode][2]: a cell's entries are contiguous
  std::vector<double> ephi;  // [mode][2]
  // Boxes that can contain a cell centre of each RG^3 region (bit b = box b;
  // built when there are at most 64 boxes, else every box is tested).
  // RG = 8, or res/128 for larger grids (the masks then stay small).
  int RG = 8;
  int nrg = 0;
  std::vector<uint64_t> boxMask;
  // Spheres that can contain a cell centre of each RG^3 region: sphereWords
  // 64-bit words per region (bit s = sphere s).
  int sphereWords = 0;
  std::vector<uint64_t> sphereMask;

  double surface(double x, double y) const {
    const int ix = std::min(std::max((int)std::floor(x), 0), res - 1);
    const int iy = std::min(std::max((int)std::floor(y), 0), res - 1);
    return surf[ix + (size_t)res * iy];
  }
  // signed distance to the liquid (vertical distance to the free surface)
  double liquid_sdf(double x, double y, double z) const {
    double d = z - surface(x, y);
    for (const auto& s : spheres) {
      double dx = x - s.cx, dy = y - s.cy, dz = z - s.cz;
      d = std::min(d, std::sqrt(dx * dx + dy * dy + dz * dz) - s.r);
    }
    return d;
  }
  bool in_box(const Box& b, const double* p) const {
    return p[0] >= b.lo[0] && p[0] < b.hi[0] && p[1] >= b.lo[1] && p[1] < b.hi[1] &&
           p[2] >= b.lo[2] && p[2] < b.hi[2];
  }
  bool solid(int x, int y, int z) const {
    const double p[3] = {x + 0.5, y + 0.5, z + 0.5};
    if (!boxMask.empty()) {
      uint64_t m = boxMask[(x / RG) + (size_t)nrg * ((y / RG) + (size_t)nrg * (z / RG))];
      while (m) {
        const int b = __builtin_ctzll(m);
        m &= m - 1;
        if (in_box(boxes[b], p)) return true;
      }
      return false;
    }
    for (const auto& b : boxes)
      if (in_box(b, p)) return true;
    return false;
  }
  bool inside(int x, int y, int z) const {
    return x >= 0 && y >= 0 && z >= 0 && x < res && y < res && z < res;
  }
  // liquid: below the plane or inside a sphere (the sign of liquid_sdf,
  // tested on squared distances)
  bool in_sphere(const Sphere& s, double x, double y, double z) const {
    double dx = x - s.cx, dy = y - s.cy, dz = z - s.cz;
    return dx * dx + dy * dy + dz * dz < s.r * s.r;
  }
  bool liquid_cell(int ix, int iy, int iz) const {
    const double x = ix + 0.5, y = iy + 0.5, z = iz + 0.5;
    if (z < surf[ix + (size_t)res * iy]) return true;
    if (!sphereMask.empty()) {
      const uint64_t* m0 =
          &sphereMask[((ix / RG) + (size_t)nrg * ((iy / RG) + (size_t)nrg * (iz / RG))) *
                      sphereWords];
      for (int w = 0; w < sphereWords; w++) {
        uint64_t m = m0[w];
        while (m) {
          const int b = __builtin_ctzll(m);
          m &= m - 1;
          if (in_sphere(spheres[64 * w + b], x, y, z)) return true;
        }
      }
      return false;
    }
    for (const auto& s : spheres)
      if (in_sphere(s, x, y, z)) return true;
    return false;
  }
  uint16_t cell_type(int x, int y, int z) const {
    if (!inside(x, y, z) || solid(x, y, z)) return 1;  // CELL_SOLID
    return liquid_cell(x, y, z) ? 0 : 0x1000;           // CELL_VOID
  }
  float face(int dir, int x, int y, int z) const {
    int xm = x - (dir == 0), ym = y - (dir == 1), zm = z - (dir == 2);
    if (!inside(x, y, z) || !inside(xm, ym, zm)) return 0.f;
    if (solid(x, y, z) || solid(xm, ym, zm)) return 0.f;
    return 1.f;
  }
  float rhs(int x, int y, int z) const {
    if (cell_type(x, y, z) != 0) return 0.f;
    double s = 0;
    const int nm = (int)modes.size();
    for (int m = 0; m < nm; m++) {
      const double* ex = &etab[(((size_t)0 * res + x) * nm + m) * 2];
      const double* ey = &etab[(((size_t)1 * res + y) * nm + m) * 2];
      const double* ez = &etab[(((size_t)2 * res + z) * nm + m) * 2];
      const double pr = ex[0] * ey[0] - ex[1] * ey[1], pi = ex[0] * ey[1] + ex[1] * ey[0];
      const double qr = pr * ez[0] - pi * ez[1], qi = pr * ez[1] + pi * ez[0];
      s += qr * ephi[2 * m] - qi * ephi[2 * m + 1];  // Re(coef e^{i phi} q)
    }
    return (float)s;
  }
};

extern "C" msbg_pressure_scene* msbg_scene_pressure_create(int res, int bsx0, int nLevels,
                                                           float zLiquid, int nSpheres,
                                                           float rMin, float rMax, int nCuboids,
                                                           int nModes, int kMax, float band,
                                                           uint64_t seed) {
  return msbg_scene_pressure_create_wavy(res, bsx0, nLevels, zLiquid, 0.f, 0, nSpheres, rMin,
                                         rMax, nCuboids, nModes, kMax, band, seed);
}

extern "C" msbg_pressure_scene* msbg_scene_pressure_create_wavy(
    int res, int bsx0, int nLevels, float zLiquid, float waveAmp, int nWaves, int nSpheres,
    float rMin, float rMax, int nCuboids, int nModes, int kMax, float band, uint64_t seed) {
  if (res <= 0 || bsx0 <= 0 || res % bsx0 || nLevels < 1 || nLevels > 4 || nWaves < 0 ||
      nSpheres < 0 || nSpheres > 4096)
    return nullptr;
  auto* s = new msbg_pressure_scene();
  s->RG = std::max(8, res / 128);
  s->res = res;
  s->bsx0 = bsx0;
  s->nLevels = nLevels;
  s->zLiquid = zLiquid;
  s->band = band;
  SplitMix64 rng(seed);
  for (int i = 0; i < nSpheres; i++) {
    Sphere sp;
    sp.cx = rng.uniform() * res;
    sp.cy = rng.uniform() * res;
    sp.cz = rng.uniform() * res;
    sp.r = (rMin + rng.uniform() * (rMax - rMin)) * res;
    s->spheres.push_back(sp);
  }
  for (int i = 0; i < nCuboids; i++) {
    msbg_pressure_scene::Box b;
    for (int k = 0; k < 3; k++) {
      double side = (0.05 + 0.10 * rng.uniform()) * res;
      double c = rng.uniform() * res;
      b.lo[k] = c - side / 2;
      b.hi[k] = c + side / 2;
    }
    s->boxes.push_back(b);
  }
  if (res % s->RG == 0 && s->boxes.size() <= 64) {
    const int RG = s->RG;
    s->nrg = res / RG;
    s->boxMask.assign((size_t)s->nrg * s->nrg * s->nrg, 0);
    for (size_t bi = 0; bi < s->boxes.size(); bi++) {
      const auto& b = s->boxes[bi];
      int r0[3], r1[3];  // regions whose cell centres can fall inside the box
      for (int k = 0; k < 3; k++) {
        r0[k] = std::max(0, (int)std::floor(b.lo[k] - 0.5) / RG);
        r1[k] = std::min(s->nrg - 1, (int)std::floor(std::max(b.hi[k] - 0.5, 0.0)) / RG);
      }
      for (int z = r0[2]; z <= r1[2]; z++)
        for (int y = r0[1]; y <= r1[1]; y++)
          for (int x = r0[0]; x <= r1[0]; x++)
            s->boxMask[x + (size_t)s->nrg * (y + (size_t)s->nrg * z)] |= 1ull << bi;
    }
  }
  if (res % s->RG == 0 && !s->spheres.empty()) {
    const int RG = s->RG, nrg = res / RG;
    s->nrg = nrg;
    const int W = (int)(s->spheres.size() + 63) / 64;
    s->sphereWords = W;
    s->sphereMask.assign((size_t)nrg * nrg * nrg * W, 0);
    for (size_t si = 0; si < s->spheres.size(); si++) {
      const Sphere& sp = s->spheres[si];
      const double c[3] = {sp.cx, sp.cy, sp.cz};
      int r0[3], r1[3];
      for (int k = 0; k < 3; k++) {
        r0[k] = std::max(0, (int)std::floor((c[k] - sp.r - 1) / RG));
        r1[k] = std::min(nrg - 1, (int)std::floor((c[k] + sp.r + 1) / RG));
      }
      for (int z = r0[2]; z <= r1[2]; z++)
        for (int y = r0[1]; y <= r1[1]; y++)
          for (int x = r0[0]; x <= r1[0]; x++) {
            // distance from the centre to the region's cell-centre box; a
            // unit of slack keeps every sphere a point could be inside
            const int rr[3] = {x, y, z};
            double d2 = 0;
            for (int k = 0; k < 3; k++) {
              const double lo = rr[k] * RG + 0.5, hi = rr[k] * RG + RG - 0.5;
              const double q = std::min(std::max(c[k], lo), hi) - c[k];
              d2 += q * q;
            }
            if (d2 < sp.r * sp.r + 1.0)
              s->sphereMask[(x + (size_t)nrg * (y + (size_t)nrg * z)) * W + si / 64] |=
                  1ull << (si % 64);
          }
    }
  }
  // Box-Muller normals for the amplitudes.
  auto normal = [&]() {
    double u1 = std::max(rng.uniform(), 1e-300), u2 = rng.uniform();
    return std::sqrt(-2.0 * std::log(u1)) * std::cos(2 * M_PI * u2);
  };
  for (int i = 0; i < nModes; i++) {
    msbg_pressure_scene::Mode m;
    do {
      for (int k = 0; k < 3; k++) m.k[k] = (int)(rng.uniform() * (2 * kMax + 1)) - kMax;
    } while (std::max({std::abs(m.k[0]), std::abs(m.k[1]), std::abs(m.k[2])}) < 1);
    for (int k = 0; k < 3; k++) m.a[k] = normal();
    m.phi = rng.uniform() * 2 * M_PI;
    // Discrete MAC divergence of a_d sin(w k.x + phi) sampled on faces:
    // sum_d a_d [sin(theta + pi k_d/res) - sin(theta - pi k_d/res)]
    //   = 2 cos(theta) sum_d a_d sin(pi k_d / res).
    double c = 0;
    for (int k = 0; k < 3; k++) c += m.a[k] * std::sin(M_PI * m.k[k] / res);
    m.coef = 2 * c;
    s->modes.push_back(m);
  }
  const double w = 2.0 * M_PI / res;
  s->etab.resize((size_t)nModes * 3 * res * 2);
  s->ephi.resize((size_t)nModes * 2);
  for (int i = 0; i < nModes; i++) {
    const auto& m = s->modes[i];
    s->ephi[2 * i] = m.coef * std::cos(m.phi);
    s->ephi[2 * i + 1] = m.coef * std::sin(m.phi);
    for (int d = 0; d < 3; d++)
      for (int x = 0; x < res; x++) {
        const double a = w * m.k[d] * (x + 0.5);
        s->etab[(((size_t)d * res + x) * nModes + i) * 2] = std::cos(a);
        s->etab[(((size_t)d * res + x) * nModes + i) * 2 + 1] = std::sin(a);
      }
  }
  // Free surface: the plane z = zLiquid*res plus nWaves sinusoids in x and y
  // (wave numbers 1..3 per axis, random phases) whose amplitudes sum to
  // waveAmp*res.  The waves are drawn last, so scenes without waves keep
  // their sequence of random numbers.
  {
    std::vector<double> wa(nWaves), wp(nWaves);
    std::vector<int> wk(2 * nWaves);
    double asum = 0;
    for (int i = 0; i < nWaves; i++) {
      wk[2 * i] = 1 + (int)(rng.uniform() * 3);
      wk[2 * i + 1] = 1 + (int)(rng.uniform() * 3);
      if (rng.uniform() < 0.5) wk[2 * i] = -wk[2 * i];
      wa[i] = 0.2 + rng.uniform();
      wp[i] = rng.uniform() * 2 * M_PI;
      asum += wa[i];
    }
    s->surf.assign((size_t)res * res, zLiquid * (double)res);
    if (nWaves > 0) {
      const double scale = waveAmp * res / asum;
#pragma omp parallel for schedule(static)
      for (int y = 0; y < res; y++)
        for (int x = 0; x < res; x++) {
          double h = 0;
          for (int i = 0; i < nWaves; i++)
            h += wa[i] * std::sin(w * (wk[2 * i] * (x + 0.5) + wk[2 * i + 1] * (y + 0.5)) + wp[i]);
          s->surf[x + (size_t)res * y] += scale * h;
        }
    }
  }
  // Refinement map.
  const int nb1 = res / bsx0;
  const int64_t nb = (int64_t)nb1 * nb1 * nb1;
  s->levels.assign(nb, nLevels - 1);
  const double halfDiag = bsx0 * std::sqrt(3.0) / 2;
#pragma omp parallel for schedule(static)
  for (int64_t b = 0; b < nb; b++) {
    int bx = (int)(b % nb1), by = (int)((b / nb1) % nb1), bz = (int)(b / ((int64_t)nb1 * nb1));
    double d = std::fabs(s->liquid_sdf((bx + 0.5) * bsx0, (by + 0.5) * bsx0, (bz + 0.5) * bsx0));
    int l = nLevels - 1;
    double w = band;
    for (int k = 0; k < nLevels - 1; k++) {
      if (d <= w + halfDiag) { l = k; break; }
      w += band * (2 << k);
    }
    s->levels[b] = l;
  }
  // 2:1 grading over the 26-neighbourhood (src/msbg.cpp:1202-1423 enforces the same).
  for (bool changed = true; changed;) {
    changed = false;
    std::vector<int> nl = s->levels;
    for (int64_t b = 0; b < nb; b++) {
      int bx = (int)(b % nb1), by = (int)((b / nb1) % nb1), bz = (int)(b / ((int64_t)nb1 * nb1));
      int lm = s->levels[b];
      for (int dz = -1; dz <= 1; dz++)
        for (int dy = -1; dy <= 1; dy++)
          for (int dx = -1; dx <= 1; dx++) {
            int x = bx + dx, y = by + dy, z = bz + dz;
            if (x < 0 || y < 0 || z < 0 || x >= nb1 || y >= nb1 || z >= nb1) continue;
            lm = std::min(lm, s->levels[x + (int64_t)nb1 * (y + (int64_t)nb1 * z)] + 1);
          }
      if (lm < nl[b]) {
        nl[b] = lm;
        changed = true;
      }
    }
    s->levels.swap(nl);
  }
  return s;
}

extern "C" void msbg_scene_pressure_destroy(msbg_pressure_scene* s) { delete s; }

extern "C" int msbg_scene_pressure_block_levels(const msbg_pressure_scene* s, int* levels) {
  if (!s || !levels) return MSBG_EINVARG;
  std::memcpy(levels, s->levels.data(), sizeof(int) * s->levels.size());
  return MSBG_OK;
}

extern "C" uint16_t msbg_scene_cell_type(void* p, int x, int y, int z) {
  return static_cast<msbg_pressure_scene*>(p)->cell_type(x, y, z);
}
extern "C" float msbg_scene_face_coeff(void* p, int dir, int x, int y, int z) {
  return static_cast<msbg_pressure_scene*>(p)->face(dir, x, y, z);
}
extern "C" float msbg_scene_rhs(void* p, int x, int y, int z) {
  return static_cast<msbg_pressure_scene*>(p)->rhs(x, y, z);
}

// The scene sampled into the per-cell arrays of msbg_gpu_pressure_prepare_arrays:
// for every base block in bid order, (bsx0 >> level)^3 cells in the block's
// voxel order, each sampled at the fine voxel of its lowest corner.
extern "C" int msbg_scene_pressure_arrays(const msbg_pressure_scene* s, uint16_t* flags,
                                          float* faceX, float* faceY, float* faceZ,
                                          float* rhs) {
  if (!s || !flags || !faceX || !faceY || !faceZ || !rhs) return MSBG_EINVARG;
  const int bs0 = s->bsx0, nbx = s->res / bs0;
  const int64_t nb = (int64_t)nbx * nbx * nbx;
  std::vector<int64_t> boff(nb + 1, 0);
  for (int64_t b = 0; b < nb; b++) {
    const int bs = bs0 >> s->levels[b];
    boff[b + 1] = boff[b] + (int64_t)bs * bs * bs;
  }
  float* face[3] = {faceX, faceY, faceZ};
#pragma omp parallel for schedule(dynamic, 4)
  for (int64_t b = 0; b < nb; b++) {
    const int l = s->levels[b], bs = bs0 >> l;
    const int ox = (int)(b % nbx) * bs0, oy = (int)((b / nbx) % nbx) * bs0,
              oz = (int)(b / ((int64_t)nbx * nbx)) * bs0;
    int64_t c = boff[b];
    for (int k = 0; k < bs; k++)
      for (int j = 0; j < bs; j++)
        for (int i = 0; i < bs; i++, c++) {
          const int x = ox + (i << l), y = oy + (j << l), z = oz + (k << l);
          flags[c] = s->cell_type(x, y, z);
          for (int d = 0; d < 3; d++) face[d][c] = s->face(d, x, y, z);
          rhs[c] = s->rhs(x, y, z);
        }
  }
  return MSBG_OK;
}
