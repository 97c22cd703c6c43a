/*
 * msbg_oracle_pressure.c — FP64 oracle of the FLIP pressure system.
 *
 * TEST INFRASTRUCTURE ONLY (the checker; see msbg_oracle.h).  An independent
 * cell-by-cell restatement of the discretisation, assembled as a CSR matrix
 * and solved with Jacobi-preconditioned CG in FP64.  It shares nothing with
 * the GPU library but the formulas:
 *   same-level face coupling  h * beta            (src/msbg3.cpp:1269-1275)
 *   level-jump face coupling  (2/3) * h_f * beta  (src/msbg3.cpp:59-161,
 *                                                   DPMR_GRAD_COEFF_FC src/msbg.h:87)
 *   a_ii = sum of its face couplings (the reference's 1/D is the face sum,
 *          src/msbg3.cpp:2686-2731), b_i = rhs * h^3.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "msbg_oracle.h"

#define NONFLUID (0x1 | 0x2 | 0x1000)

typedef struct {
  int sx, sy, sz, bsx0, nbx, nby, nbz;
  const int* lev;
  const int* dbc; /* six domain faces: 0 open, 1 solid; NULL: the reference's rule */
  int64_t* boff;
  oracle_cell_type_fn ct;
  oracle_face_fn fc;
  void* user;
} Grid;

static int inside(const Grid* g, const int f[3]) {
  return f[0] >= 0 && f[1] >= 0 && f[2] >= 0 && f[0] < g->sx && f[1] < g->sy && f[2] < g->sz;
}

/* index of the level-L cell with level-L coordinates P (in block layout) */
static int64_t cell_index(const Grid* g, int L, const int P[3]) {
  const int bs = g->bsx0 >> L;
  const int bx = P[0] / bs, by = P[1] / bs, bz = P[2] / bs;
  const int64_t b = bx + (int64_t)g->nbx * (by + (int64_t)g->nby * bz);
  return g->boff[b] + (P[0] % bs) + (int64_t)bs * ((P[1] % bs) + (int64_t)bs * (P[2] % bs));
}

static int block_level(const Grid* g, const int f[3]) {
  return g->lev[f[0] / g->bsx0 + g->nbx * (f[1] / g->bsx0 + g->nby * (f[2] / g->bsx0))];
}

static int is_fluid(const Grid* g, int L, const int P[3]) {
  return !(g->ct(g->user, P[0] << L, P[1] << L, P[2] << L) & NONFLUID);
}

static double face_beta(const Grid* g, int L, int dir, const int P[3]) {
  return g->fc(g->user, dir, P[0] << L, P[1] << L, P[2] << L);
}

/* For one cell: diagonal and up to 24 off-diagonal (col, coupling) pairs. */
static double cell_row(const Grid* g, int L, const int P[3], int64_t* cols, double* vals,
                       int* nnz) {
  const double h = (double)(1 << L);
  double diag = 0;
  int n = 0;
  for (int dir = 0; dir < 3; dir++) {
    const int ax = dir == 0 ? 1 : 0, bx = dir == 2 ? 1 : 2;
    for (int side = 0; side < 2; side++) {
      int fv[3] = {P[0] << L, P[1] << L, P[2] << L};
      fv[dir] = side ? (P[dir] + 1) << L : (P[dir] << L) - 1;
      int q[3] = {P[0], P[1], P[2]};
      if (side) q[dir] += 1;
      if (!inside(g, fv)) {
        /* p = 0 outside.  Solid: no coupling.  Open: the callback's lower
         * face coefficient, 1 on an upper face.  No spec: the reference's
         * diagonal (src/msbg3.cpp:2714-2722) reads faces past the grid as 0,
         * so the lower faces count and the upper ones do not. */
        const int bc = g->dbc ? g->dbc[2 * dir + side] : -1;
        if (bc == 1 || (bc == -1 && side))
          ;
        else if (side)
          diag += h;
        else
          diag += h * face_beta(g, L, dir, q);
        continue;
      }
      const int L2 = block_level(g, fv);
      if (L2 == L) {
        const double c = h * face_beta(g, L, dir, q);
        int P2[3] = {P[0], P[1], P[2]};
        P2[dir] += side ? 1 : -1;
        diag += c;
        if (c != 0 && is_fluid(g, L, P2)) {
          cols[n] = cell_index(g, L, P2);
          vals[n++] = c;
        }
      } else if (L2 == L + 1) {
        const double c = (2.0 / 3.0) * h * face_beta(g, L, dir, q);
        int P2[3];
        for (int k = 0; k < 3; k++) P2[k] = fv[k] >> (L + 1);
        diag += c;
        if (c != 0 && is_fluid(g, L + 1, P2)) {
          cols[n] = cell_index(g, L + 1, P2);
          vals[n++] = c;
        }
      } else {
        for (int u = 0; u < 2; u++)
          for (int v = 0; v < 2; v++) {
            int f[3];
            f[dir] = side ? (P[dir] + 1) * 2 : P[dir] * 2 - 1;
            f[ax] = P[ax] * 2 + u;
            f[bx] = P[bx] * 2 + v;
            int qf[3] = {f[0], f[1], f[2]};
            if (!side) qf[dir] += 1; /* shared face is the fine cell's upper face */
            const double c = (2.0 / 3.0) * (h / 2) * face_beta(g, L - 1, dir, qf);
            diag += c;
            if (c != 0 && is_fluid(g, L - 1, f)) {
              cols[n] = cell_index(g, L - 1, f);
              vals[n++] = c;
            }
          }
      }
    }
  }
  *nnz = n;
  return diag;
}

typedef struct {
  int64_t n;
  int64_t* rowptr;
  int64_t* col;
  double* val;  /* off-diagonal couplings (positive; A_ij = -val) */
  double* diag; /* 0 for non-liquid rows */
} Csr;

static int assemble(Grid* g, Csr* A, oracle_rhs_fn rhs, double* b) {
  const int64_t nb = (int64_t)g->nbx * g->nby * g->nbz;
  int64_t n = g->boff[nb];
  A->n = n;
  A->rowptr = (int64_t*)calloc(n + 1, sizeof(int64_t));
  A->diag = (double*)calloc(n, sizeof(double));
  int* cnt = (int*)calloc(n, sizeof(int));
  int64_t* tc = (int64_t*)malloc(sizeof(int64_t) * n * 24);
  double* tv = (double*)malloc(sizeof(double) * n * 24);
  if (!A->rowptr || !A->diag || !cnt || !tc || !tv) return 2;
#pragma omp parallel for schedule(dynamic, 1)
  for (int64_t blk = 0; blk < nb; blk++) {
    const int L = g->lev[blk], bs = g->bsx0 >> L;
    const int bx = (int)(blk % g->nbx), by = (int)((blk / g->nbx) % g->nby),
              bz = (int)(blk / ((int64_t)g->nbx * g->nby));
    for (int vz = 0; vz < bs; vz++)
      for (int vy = 0; vy < bs; vy++)
        for (int vx = 0; vx < bs; vx++) {
          const int P[3] = {bx * bs + vx, by * bs + vy, bz * bs + vz};
          const int64_t c = g->boff[blk] + vx + (int64_t)bs * (vy + (int64_t)bs * vz);
          if (!is_fluid(g, L, P)) {
            cnt[c] = 0;
            A->diag[c] = 0;
            if (b) b[c] = 0;
            continue;
          }
          int nnz = 0;
          A->diag[c] = cell_row(g, L, P, tc + c * 24, tv + c * 24, &nnz);
          cnt[c] = nnz;
          if (b) {
            const double h = (double)(1 << L);
            b[c] = (double)rhs(g->user, P[0] << L, P[1] << L, P[2] << L) * h * h * h;
          }
        }
  }
  for (int64_t i = 0; i < n; i++) A->rowptr[i + 1] = A->rowptr[i] + cnt[i];
  A->col = (int64_t*)malloc(sizeof(int64_t) * (A->rowptr[n] + 1));
  A->val = (double*)malloc(sizeof(double) * (A->rowptr[n] + 1));
  for (int64_t i = 0; i < n; i++) {
    memcpy(A->col + A->rowptr[i], tc + i * 24, sizeof(int64_t) * cnt[i]);
    memcpy(A->val + A->rowptr[i], tv + i * 24, sizeof(double) * cnt[i]);
  }
  free(cnt);
  free(tc);
  free(tv);
  return 0;
}

static void csr_free(Csr* A) {
  free(A->rowptr);
  free(A->col);
  free(A->val);
  free(A->diag);
}

static void spmv(const Csr* A, const double* x, double* y) {
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < A->n; i++) {
    if (A->diag[i] == 0) {
      y[i] = 0;
      continue;
    }
    double s = A->diag[i] * x[i];
    for (int64_t k = A->rowptr[i]; k < A->rowptr[i + 1]; k++) s -= A->val[k] * x[A->col[k]];
    y[i] = s;
  }
}

static double dot(const double* a, const double* b, int64_t n) {
  double s = 0;
#pragma omp parallel for reduction(+ : s) schedule(static)
  for (int64_t i = 0; i < n; i++) s += a[i] * b[i];
  return s;
}

static int make_grid(Grid* g, int sx, int sy, int sz, int bsx0, const int* lev, const int* dbc,
                     oracle_cell_type_fn ct, oracle_face_fn fc, void* user) {
  g->sx = sx;
  g->sy = sy;
  g->sz = sz;
  g->bsx0 = bsx0;
  g->nbx = sx / bsx0;
  g->nby = sy / bsx0;
  g->nbz = sz / bsx0;
  g->lev = lev;
  g->dbc = dbc;
  g->ct = ct;
  g->fc = fc;
  g->user = user;
  const int64_t nb = (int64_t)g->nbx * g->nby * g->nbz;
  g->boff = (int64_t*)malloc(sizeof(int64_t) * (nb + 1));
  if (!g->boff) return 2;
  g->boff[0] = 0;
  for (int64_t b = 0; b < nb; b++) {
    const int bs = bsx0 >> lev[b];
    g->boff[b + 1] = g->boff[b] + (int64_t)bs * bs * bs;
  }
  return 0;
}

int oracle_pressure_apply(int sx, int sy, int sz, int bsx0, const int* blockLevel,
                          const int* domainBc, oracle_cell_type_fn cellType, oracle_face_fn face,
                          void* user, const double* x, double* y) {
  Grid g;
  Csr A;
  if (make_grid(&g, sx, sy, sz, bsx0, blockLevel, domainBc, cellType, face, user)) return 2;
  int rc = assemble(&g, &A, NULL, NULL);
  if (!rc) spmv(&A, x, y);
  csr_free(&A);
  free(g.boff);
  return rc;
}

int oracle_pressure_solve(int sx, int sy, int sz, int bsx0, const int* blockLevel,
                          const int* domainBc, oracle_cell_type_fn cellType, oracle_face_fn face,
                          oracle_rhs_fn rhs, void* user, double tol, int maxIter, double* x,
                          double* b, int* itersOut, double* relResOut) {
  Grid g;
  Csr A;
  if (sx % bsx0 || sy % bsx0 || sz % bsx0) return 5;
  if (make_grid(&g, sx, sy, sz, bsx0, blockLevel, domainBc, cellType, face, user)) return 2;
  int rc = assemble(&g, &A, rhs, b);
  if (rc) return rc;
  const int64_t n = A.n;
  double* r = (double*)malloc(sizeof(double) * n);
  double* z = (double*)malloc(sizeof(double) * n);
  double* d = (double*)malloc(sizeof(double) * n);
  double* q = (double*)malloc(sizeof(double) * n);
  for (int64_t i = 0; i < n; i++) {
    x[i] = 0;
    r[i] = b[i];
    z[i] = A.diag[i] > 0 ? r[i] / A.diag[i] : 0;
    d[i] = z[i];
  }
  const double bb = dot(b, b, n);
  double rho = dot(r, z, n), rr = bb;
  int it = 0;
  while (it < maxIter && rr > tol * tol * bb && bb > 0) {
    spmv(&A, d, q);
    const double alpha = rho / dot(d, q, n);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; i++) {
      x[i] += alpha * d[i];
      r[i] -= alpha * q[i];
      z[i] = A.diag[i] > 0 ? r[i] / A.diag[i] : 0;
    }
    rr = dot(r, r, n);
    const double rhoNew = dot(r, z, n);
    const double beta = rhoNew / rho;
    rho = rhoNew;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; i++) d[i] = z[i] + beta * d[i];
    it++;
  }
  /* true residual */
  spmv(&A, x, q);
  double t = 0;
  for (int64_t i = 0; i < n; i++) t += (b[i] - q[i]) * (b[i] - q[i]);
  if (itersOut) *itersOut = it;
  if (relResOut) *relResOut = bb > 0 ? sqrt(t / bb) : 0;
  free(r);
  free(z);
  free(d);
  free(q);
  csr_free(&A);
  free(g.boff);
  return 0;
}

/* ---- array-backed scene ----------------------------------------------------
 * Callbacks that read per-cell arrays in the packed block layout of MG level 0
 * (blocks in bid order, (bsx0>>L)^3 cells each at the block's level L): cell
 * flags, the LOWER face coefficient per direction and the rhs.  A fine voxel
 * maps to the level-L cell that contains it.  Outside the domain a cell is
 * solid and a face has coefficient 0 (the reference's getValueGen_ reads 0
 * there, src/msbg3.cpp:2700-2708).  Used to feed the reference's own prepared
 * channels (preparePressureSolveFLIPLevel0_, src/msbg3.cpp:2472-2584) to the
 * oracle, so both assemble from identical inputs. */
typedef struct {
  int sx, sy, sz, bsx0, nbx, nby;
  const int* lev;
  const int* dbc; /* six domain faces: 0 open, 1 solid; NULL: the reference's rule */
  int64_t* boff;
  const unsigned short* flags;
  const float* face[3];
  const float* rhs;
} ArrayScene;

static int64_t array_cell(const ArrayScene* a, int x, int y, int z) {
  if (x < 0 || y < 0 || z < 0 || x >= a->sx || y >= a->sy || z >= a->sz) return -1;
  const int64_t b = (x / a->bsx0) + (int64_t)a->nbx * ((y / a->bsx0) + (int64_t)a->nby * (z / a->bsx0));
  const int L = a->lev[b], bs = a->bsx0 >> L;
  const int vx = (x % a->bsx0) >> L, vy = (y % a->bsx0) >> L, vz = (z % a->bsx0) >> L;
  return a->boff[b] + vx + (int64_t)bs * (vy + (int64_t)bs * vz);
}

void* oracle_array_scene_create(int sx, int sy, int sz, int bsx0, const int* lev,
                                const unsigned short* flags, const float* fx, const float* fy,
                                const float* fz, const float* rhs) {
  ArrayScene* a = (ArrayScene*)calloc(1, sizeof(ArrayScene));
  if (!a) return NULL;
  a->sx = sx;
  a->sy = sy;
  a->sz = sz;
  a->bsx0 = bsx0;
  a->nbx = sx / bsx0;
  a->nby = sy / bsx0;
  const int64_t nb = (int64_t)a->nbx * a->nby * (sz / bsx0);
  a->boff = (int64_t*)malloc(sizeof(int64_t) * (nb + 1));
  if (!a->boff) {
    free(a);
    return NULL;
  }
  a->boff[0] = 0;
  for (int64_t b = 0; b < nb; b++) {
    const int bs = bsx0 >> lev[b];
    a->boff[b + 1] = a->boff[b] + (int64_t)bs * bs * bs;
  }
  a->lev = lev;
  a->flags = flags;
  a->face[0] = fx;
  a->face[1] = fy;
  a->face[2] = fz;
  a->rhs = rhs;
  return a;
}

void oracle_array_scene_destroy(void* p) {
  ArrayScene* a = (ArrayScene*)p;
  if (!a) return;
  free(a->boff);
  free(a);
}

unsigned short oracle_array_cell_type(void* p, int x, int y, int z) {
  const ArrayScene* a = (const ArrayScene*)p;
  const int64_t c = array_cell(a, x, y, z);
  return c < 0 ? (unsigned short)0x1 : a->flags[c];
}

float oracle_array_face(void* p, int dir, int x, int y, int z) {
  const ArrayScene* a = (const ArrayScene*)p;
  const int64_t c = array_cell(a, x, y, z);
  return c < 0 ? 0.f : a->face[dir][c];
}

float oracle_array_rhs(void* p, int x, int y, int z) {
  const ArrayScene* a = (const ArrayScene*)p;
  const int64_t c = array_cell(a, x, y, z);
  return c < 0 || !a->rhs ? 0.f : a->rhs[c];
}
