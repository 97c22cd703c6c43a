/*
 * msbg_oracle.h — CPU restatement of the reference MSBG solver path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker the GPU path is compared
 * with; it is never linked into, called by, or used as a fallback for the
 * product library.  Only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg load it.
 *
 * Parity pinned: each routine is checked against the compiled reference
 * (oracle/_ref/libmsbg_ref.so, built from the reference sources by
 * oracle/Makefile) on seeded inputs, and against the golden fixtures in
 * tests/golden/ that were generated from that compiled reference.
 */
#ifndef MSBG_ORACLE_H
#define MSBG_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* 8-colour in-place mean-curvature flow on a single-level FP32 channel.
 * Same arguments as the reference harness ref_mcf: kind[nb] per block
 * (0 NULL, 1 value, 2 empty, 3 full), values = packed value blocks in
 * ascending bid order, update = block list.  numIter is rounded up to even
 * unless exactIter != 0 (then exactly numIter sweeps run; used to compare
 * single iterations).  Follows src/msbg4.cpp:348-851 and
 * src/halo.cpp:266-479 with src/halo.h:266-280 (OPT_BC_NEUMANN). */
int oracle_mcf(int nbx, int nby, int nbz, int bsx, const int8_t* kind,
               float emptyVal, float fullVal, float* values, const int* update,
               int nUpdate, int numIter, float dt, int clamp01, int exactIter);

/* FP64 reference solution of the FLIP pressure system on an adaptive block
 * grid (the system the GPU MGPCG solves):
 *   cells: every block b holds (bsx0>>L)^3 cells of edge h = 2^L, L = map[b];
 *   cell type, face coefficient beta and rhs come from the callbacks at the
 *   fine-voxel coordinates of the cell's lowest corner voxel;
 *   coupling across a face: same level h*beta; level jump (2/3)*h_fine*beta
 *   with beta of the fine cell's face (src/msbg.h:82-87, src/msbg3.cpp:59-161);
 *   a_ii = sum of the face couplings of cell i (air / outside = p 0);
 *   b_i = rhs * h^3.
 * Solved with Jacobi-preconditioned CG in FP64 to |r| <= tol |b|.
 * x, b: outputs in the reference block layout (blocks in bid order, each
 * (bsx0>>L)^3 values, vid = x + y*bs + z*bs*bs).  Returns 0 on success. */
typedef unsigned short (*oracle_cell_type_fn)(void*, int, int, int);
typedef float (*oracle_face_fn)(void*, int, int, int, int);
typedef float (*oracle_rhs_fn)(void*, int, int, int);
/* domainBc: six domain faces (-x, +x, -y, +y, -z, +z), 0 open, 1 solid, or
 * NULL for the reference's rule (lower faces open, upper faces no coupling). */
int oracle_pressure_solve(int sx, int sy, int sz, int bsx0, const int* blockLevel,
                          const int* domainBc, oracle_cell_type_fn cellType, oracle_face_fn face,
                          oracle_rhs_fn rhs, void* user, double tol, int maxIter, double* x,
                          double* b, int* itersOut, double* relResOut);

/* y = A x for the same system (x, y in the block layout, FP64). */
int oracle_pressure_apply(int sx, int sy, int sz, int bsx0, const int* blockLevel,
                          const int* domainBc, oracle_cell_type_fn cellType, oracle_face_fn face,
                          void* user, const double* x, double* y);

/* Callbacks over per-cell arrays in the packed block layout of MG level 0:
 * flags, lower-face coefficient per direction, rhs (see
 * msbg_oracle_pressure.c).  The user pointer comes from
 * oracle_array_scene_create; the arrays must outlive it. */
void* oracle_array_scene_create(int sx, int sy, int sz, int bsx0, const int* lev,
                                const unsigned short* flags, const float* fx, const float* fy,
                                const float* fz, const float* rhs);
void oracle_array_scene_destroy(void* scene);
unsigned short oracle_array_cell_type(void* scene, int x, int y, int z);
float oracle_array_face(void* scene, int dir, int x, int y, int z);
float oracle_array_rhs(void* scene, int x, int y, int z);

/* ---- FLIP transfers (msbg_oracle_flip.c, src/flip_sim.cpp) ---- */
/* FlipParticle (src/flip_sim.h:48) */
typedef struct {
  float pos[3], vel[3];
  int phase; /* 0 liquid, 1 air */
} oracle_flip_particle;
/* the FlipConfig fields the transfers read (src/flip_sim.h:29-45) */
typedef struct {
  float rhoL, rhoG, massEps, betaMin, alphaPhi;
  int particlesPerVoxel;
} oracle_flip_params;
/* vel, beta: 3 floats per voxel (lower-face u, v, w); mass: 1; block layout;
 * activeBlock[nBlocks]: 1 where a voxel has mass > massEps. */
int oracle_flip_p2g(int sx, int sy, int sz, int bsx, const oracle_flip_particle* p, int64_t np,
                    const oracle_flip_params* c, float* vel, float* mass, float* beta,
                    uint8_t* activeBlock);
void oracle_flip_gravity(int sx, int sy, int sz, int bsx, float* vel, float* velOld,
                         const float* mass, float gravity, float dt, float massEps);
void oracle_flip_gradient(int sx, int sy, int sz, int bsx, float* vel, const float* mass,
                          const float* beta, const float* pressure, float dt, float massEps);
void oracle_flip_g2p(int sx, int sy, int sz, int bsx, oracle_flip_particle* p, int64_t np,
                     const float* vel, const float* velOld, float alpha);

/* ---- mixed-resolution G2P interpolation (msbg_oracle_flip_mr.c,
 * src/flip_sim.cpp:1354-1545, src/msbg.cpp:1887-1960, src/sbg.h:3111-3420) ----
 * level[b]: resolution level of block b; packed layout: per block in bid
 * order its (bsx0>>level)^3 voxels at its level, off[b] its first voxel
 * (oracle_mr_layout returns the total).  dist: the value blocks of
 * CH_DIST_FINECOARSE, packed; kind[l*nBlocks + b]: block b's kind in the
 * channel of level l (0 empty, 1 value, 2 full = dTransRes*1024). */
int64_t oracle_mr_layout(int nbx, int nby, int nbz, int bsx0, const int* level, int64_t* off);
void oracle_mr_dist(int nbx, int nby, int nbz, int bsx0, const int* level, int nLevels,
                    int dTransRes, uint16_t* dist, int8_t* kind);
void oracle_mr_dist_interp(int sx, int sy, int sz, int bsx0, int nbx, int nby, int nbz,
                           const int* level, const int64_t* off, const uint16_t* dist,
                           const int8_t* kind, int dTransRes, int lv, const float* pos,
                           int64_t n, float* out);
void oracle_mr_g2p(int sx, int sy, int sz, int bsx0, const int* level, int dTransRes,
                   oracle_flip_particle* p, int64_t np, const float* vel, const float* velOld,
                   const uint16_t* dist, const int8_t* kind, float alpha);

/* downsampleVelocity (src/msbg4.cpp:2035-2270), MG level m-1 -> m: src/dst
 * packed at those MG levels (3 floats per voxel), flags packed at MG level m. */
void oracle_mr_downsample_velocity(int sx, int sy, int sz, int bsx0, const int* level0, int m,
                                   const uint16_t* flags, const float* src, float* dst);

/* ---- particle splatting (msbg_oracle_splat.c, src/msbg_demo.cpp) ---- */
/* pos: 3 floats per particle; kind/active: one byte per block (1 = value);
 * out: the value blocks packed in bid order, 16-bit render density
 * (finalize = 0: the quantised squared distances before finalisation). */
void oracle_splat_domain(int sx, int sy, int sz, float lo[3], float hi[3]);
int oracle_splat_mark(int sx, int sy, int sz, int bsx, const float* pos, int64_t n,
                      float rParticle, float nbDist, int8_t* active);
int oracle_splat(int sx, int sy, int sz, int bsx, const int8_t* kind, const float* pos,
                 int64_t n, float rParticle, float nbDist, int finalize, uint16_t* out);
uint16_t oracle_splat_finalize_value(uint16_t q, float rParticle, float nbDist);

#ifdef __cplusplus
}
#endif

#endif
