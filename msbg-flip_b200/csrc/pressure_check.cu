// Host-side consistency check of the pressure hierarchy (no GPU needed).
//
// Builds the hierarchy exactly as msbg_gpu_pressure_prepare does and, on the
// host, (1) applies the MG-level-0 operator through the same face-descriptor
// ghost code the kernels use (ghost_sum), so a test can compare it with an
// independently assembled matrix; (2) measures how far each coarse operator is
// from the Galerkin product P^T A P on a random vector.
#include <cmath>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include "pressure.h"
#include "pressure_kernels.cuh"

namespace msbg {
namespace ps {
namespace {

LevelView host_view(const Level& L, std::vector<int64_t>& toff) {
  toff.resize(L.tiles.size());
  for (size_t i = 0; i < L.tiles.size(); i++) toff[i] = L.tiles[i].off;
  LevelView v;
  v.tileOff = toff.data();
  v.face = L.face.data();
  v.ifOff = L.ifOff.data();
  v.toCoarse = L.toCoarse.data();
  v.diag = L.diag.data();
  v.cx = L.cx.data();
  v.cy = L.cy.data();
  v.cz = L.cz.data();
  v.ifc = L.ifc.data();
  return v;
}

// y = A x on one level, FP64 accumulation of the same terms the kernels use.
void host_apply(const Level& L, const std::vector<float>& x, std::vector<double>& y) {
  std::vector<int64_t> toff;
  LevelView v = host_view(L, toff);
  y.assign(L.nCells, 0.0);
  for (size_t ti = 0; ti < L.tiles.size(); ti++) {
    const Tile& t = L.tiles[ti];
    const int ts = t.ts;
    const float* X = x.data() + t.off;
    for (int k = 0; k < ts; k++)
      for (int j = 0; j < ts; j++)
        for (int i = 0; i < ts; i++) {
          const int e = tidx(ts, i, j, k);
          const double dg = L.diag[t.off + e];
          if (!(dg > 0)) continue;
          double S = 0;
          const float* cx = L.cx.data() + t.off;
          const float* cy = L.cy.data() + t.off;
          const float* cz = L.cz.data() + t.off;
          S += i > 0 ? (double)cx[e] * X[e - 1] : ghost_sum(v, x.data(), (int)ti, ts, 0, 0, j, k);
          S += i < ts - 1 ? (double)cx[e + 1] * X[e + 1] : ghost_sum(v, x.data(), (int)ti, ts, 0, 1, j, k);
          S += j > 0 ? (double)cy[e] * X[e - ts] : ghost_sum(v, x.data(), (int)ti, ts, 1, 0, i, k);
          S += j < ts - 1 ? (double)cy[e + ts] * X[e + ts] : ghost_sum(v, x.data(), (int)ti, ts, 1, 1, i, k);
          S += k > 0 ? (double)cz[e] * X[e - ts * ts] : ghost_sum(v, x.data(), (int)ti, ts, 2, 0, i, j);
          S += k < ts - 1 ? (double)cz[e + ts * ts] * X[e + ts * ts] : ghost_sum(v, x.data(), (int)ti, ts, 2, 1, i, j);
          y[t.off + e] = dg * X[e] - S;
        }
  }
}

// P^T (sum over liquid children) and P (copy to liquid children) between
// levels F (fine) and G (coarse).
void host_restrict(const Level& F, const Level& G, const std::vector<double>& r,
                   std::vector<double>& rc) {
  rc.assign(G.nCells, 0.0);
  for (size_t ti = 0; ti < F.tiles.size(); ti++) {
    const Tile& t = F.tiles[ti];
    const int* tc = &F.toCoarse[ti * 6];
    if (tc[0] < 0) continue;
    const int64_t co = G.tiles[tc[0]].off;
    const int sh = tc[4] ? 1 : 0;
    for (int k = 0; k < t.ts; k++)
      for (int j = 0; j < t.ts; j++)
        for (int i = 0; i < t.ts; i++) {
          const int64_t c = t.off + tidx(t.ts, i, j, k);
          if (!(F.diag[c] > 0)) continue;
          rc[co + tidx(tc[5], tc[1] + (i >> sh), tc[2] + (j >> sh), tc[3] + (k >> sh))] += r[c];
        }
  }
}

void host_prolong(const Level& F, const Level& G, const std::vector<float>& xc,
                  std::vector<float>& x) {
  x.assign(F.nCells, 0.f);
  for (size_t ti = 0; ti < F.tiles.size(); ti++) {
    const Tile& t = F.tiles[ti];
    const int* tc = &F.toCoarse[ti * 6];
    if (tc[0] < 0) continue;
    const int64_t co = G.tiles[tc[0]].off;
    const int sh = tc[4] ? 1 : 0;
    for (int k = 0; k < t.ts; k++)
      for (int j = 0; j < t.ts; j++)
        for (int i = 0; i < t.ts; i++) {
          const int64_t c = t.off + tidx(t.ts, i, j, k);
          if (!(F.diag[c] > 0)) continue;
          x[c] = xc[co + tidx(tc[5], tc[1] + (i >> sh), tc[2] + (j >> sh), tc[3] + (k >> sh))];
        }
  }
}

// level-0 tile layout <-> reference block layout (blocks in bid order)
struct Packing {
  std::vector<int64_t> boff;
  int bsx0, nbx, nby;
  const std::vector<int>* lev;
  int64_t index(int level, int X, int Y, int Z) const {
    const int bs = bsx0 >> level;
    const int64_t b = (X / bs) + (int64_t)nbx * ((Y / bs) + (int64_t)nby * (Z / bs));
    return boff[b] + (X % bs) + (int64_t)bs * ((Y % bs) + (int64_t)bs * (Z % bs));
  }
};

}  // namespace
}  // namespace ps
}  // namespace msbg

using namespace msbg;
using namespace msbg::ps;

static int host_check(const msbg_topo_desc* topo, const msbg_pressure_callbacks* cb,
                      const ArrayInput* arr, const float* xPacked, double* yPacked,
                      int* nMgLevels, int64_t* fluidPerLevel, double* galerkinErr) {
  Hierarchy H;
  std::string err;
  int rc = build_hierarchy(H, topo->sx, topo->sy, topo->sz, topo->bsx0, topo->nLevels,
                           topo->blockLevel, topo->domainBc, cb, 512, &err, arr);
  if (rc) {
    fprintf(stderr, "msbg_gpu_pressure_host_check: %s\n", err.c_str());
    return rc;
  }
  const int nL = (int)H.levels.size();
  if (nMgLevels) *nMgLevels = nL;
  if (fluidPerLevel)
    for (int m = 0; m < nL && m < 32; m++) fluidPerLevel[m] = H.levels[m].nFluid;
  // (1) level-0 operator in block layout
  if (xPacked && yPacked) {
    Packing P;
    P.bsx0 = H.bsx0;
    P.nbx = H.nb1x;
    P.nby = H.nb1y;
    const int64_t nb = (int64_t)H.nb1x * H.nb1y * H.nb1z;
    P.boff.assign(nb + 1, 0);
    for (int64_t b = 0; b < nb; b++) {
      const int bs = H.bsx0 >> H.blockLevel[b];
      P.boff[b + 1] = P.boff[b] + (int64_t)bs * bs * bs;
    }
    const Level& L = H.levels[0];
    std::vector<float> x(L.nCells, 0.f);
    std::vector<int64_t> map(L.nCells);
    for (const Tile& t : L.tiles)
      for (int k = 0; k < t.ts; k++)
        for (int j = 0; j < t.ts; j++)
          for (int i = 0; i < t.ts; i++) {
            const int64_t c = t.off + tidx(t.ts, i, j, k);
            map[c] = P.index(t.level, t.ox + i, t.oy + j, t.oz + k);
            x[c] = L.diag[c] > 0 ? xPacked[map[c]] : 0.f;
          }
    std::vector<double> y;
    host_apply(L, x, y);
    std::memset(yPacked, 0, sizeof(double) * P.boff[nb]);
    for (int64_t c = 0; c < L.nCells; c++) yPacked[map[c]] = y[c];
  }
  // (2) Galerkin consistency per coarse level
  if (galerkinErr) {
    std::mt19937_64 rng(7);
    std::uniform_real_distribution<float> U(-1.f, 1.f);
    for (int m = 0; m + 1 < nL && m < 32; m++) {
      const Level& F = H.levels[m];
      const Level& G = H.levels[m + 1];
      std::vector<float> xc(G.nCells, 0.f);
      for (int64_t c = 0; c < G.nCells; c++) xc[c] = G.diag[c] > 0 ? U(rng) : 0.f;
      std::vector<float> xf;
      host_prolong(F, G, xc, xf);
      std::vector<double> yf, ptApf, yc;
      host_apply(F, xf, yf);
      host_restrict(F, G, yf, ptApf);
      host_apply(G, xc, yc);
      double emax = 0, ymax = 0;
      // every coarse cell: one that P^T A P reaches but A_c leaves empty
      // (a liquid cell built without its children) shows here too
      for (int64_t c = 0; c < G.nCells; c++) {
        emax = std::max(emax, std::fabs(ptApf[c] - yc[c]));
        ymax = std::max(ymax, std::fabs(ptApf[c]));
      }
      galerkinErr[m] = ymax > 0 ? emax / ymax : 0.0;
    }
  }
  return MSBG_OK;
}

extern "C" int msbg_gpu_pressure_host_check(const msbg_topo_desc* topo,
                                            const msbg_pressure_callbacks* cb,
                                            const float* xPacked, double* yPacked,
                                            int* nMgLevels, int64_t* fluidPerLevel,
                                            double* galerkinErr) {
  if (!topo || !cb) return MSBG_EINVARG;
  return host_check(topo, cb, nullptr, xPacked, yPacked, nMgLevels, fluidPerLevel, galerkinErr);
}

// The same from the per-cell arrays of msbg_gpu_pressure_prepare_arrays.
extern "C" int msbg_gpu_pressure_host_check_arrays(const msbg_topo_desc* topo,
                                                   const uint16_t* flags, const float* faceX,
                                                   const float* faceY, const float* faceZ,
                                                   const float* rhs, const float* xPacked,
                                                   double* yPacked, int* nMgLevels,
                                                   int64_t* fluidPerLevel, double* galerkinErr) {
  if (!topo || !flags || !faceX || !faceY || !faceZ) return MSBG_EINVARG;
  const ArrayInput A{flags, {faceX, faceY, faceZ}, rhs};
  return host_check(topo, nullptr, &A, xPacked, yPacked, nMgLevels, fluidPerLevel, galerkinErr);
}
