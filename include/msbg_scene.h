/*
 * msbg_scene.h — seeded synthetic workloads for the sparse block-grid solver.
 *
 * Host-only (C++/OpenMP) generators shared by the tests, the benchmark and the
 * CPU baselines, so every side sees identical inputs.  They have no
 * counterpart in the reference: its own inputs come from particle splatting
 * (src/msbg_demo.cpp:519-684) and the FLIP simulation (src/flip_sim.cpp),
 * which are outside this path.  Random numbers: splitmix64 -> [0,1) doubles.
 */
#ifndef MSBG_SCENE_H
#define MSBG_SCENE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Signed distance to a union of random spheres on a single-level block grid.
 *   res^3 domain, bsx^3 blocks, nSpheres centres U[0,res)^3, radii
 *   U[rmin,rmax]; phi(x) = min_i(|x - c_i| - r_i) at voxel centres (x+0.5).
 *   Value blocks: blocks holding any voxel with |phi| <= band, dilated by
 *   `dilate` blocks.  Other blocks are const: MSBG_BLOCK_EMPTY (phi > 0 side,
 *   value +band) or MSBG_BLOCK_FULL (phi < 0 side, value -band).
 *   kind[nb] is always written; values (packed value blocks, ascending bid)
 *   only when non-NULL.  *nValueBlocks receives the count. */
int msbg_scene_sphere_sdf(int res, int bsx, int nSpheres, float rmin, float rmax,
                          float band, int dilate, uint64_t seed, int8_t* kind,
                          float* values, int64_t* nValueBlocks);

/* Free-surface pressure problem (adaptive MSBG, FLIP pressure solve).
 *   Domain res^3 (fine voxels), base blocks bsx0^3, nLevels resolution levels.
 *   Liquid = {z < zLiquid*res} U nSpheres spheres (centres U[0,res)^3, radii
 *   U[rMin,rMax]*res); nCuboids axis-aligned solid cuboids (sides
 *   U[0.05,0.15]*res) override liquid; everything else is air.
 *   Refinement map: level 0 for blocks whose centre lies within `band` fine
 *   voxels (+ half a block diagonal) of the liquid surface, coarser levels in
 *   further bands of width 2*band, 4*band ...; then 2:1 graded.
 *   RHS = discrete MAC divergence (per unit volume) of
 *   u = sum_k a_k sin(2 pi k.x/res + phi_k) over nModes modes, |k|_inf in
 *   1..kMax, a_k ~ N(0,1) per component.
 * The callbacks below sample it at fine-voxel coordinates like the
 * reference's FlipPressureCallbacks (src/msbg.h:829-835, src/flip_sim.cpp:313-338):
 *   cell type: 0 liquid, CELL_SOLID (1) solid or outside, CELL_VOID (0x1000) air;
 *   face coefficient: 1 inside the box, 0 on faces touching a solid cell or a
 *   box wall; rhs: divergence in liquid cells, 0 elsewhere. */
typedef struct msbg_pressure_scene msbg_pressure_scene;

msbg_pressure_scene* msbg_scene_pressure_create(int res, int bsx0, int nLevels, float zLiquid,
                                                int nSpheres, float rMin, float rMax,
                                                int nCuboids, int nModes, int kMax, float band,
                                                uint64_t seed);
/* Same problem with a wavy free surface: liquid below
 *   z = res * (zLiquid + waveAmp * sum_i a_i sin(2 pi (kx_i x + ky_i y)/res + phi_i))
 * with nWaves seeded sinusoids (|kx|, ky in 1..3, a_i > 0 summing to 1), plus
 * the spheres (up to 4096).  nWaves = 0 gives msbg_scene_pressure_create. */
msbg_pressure_scene* msbg_scene_pressure_create_wavy(int res, int bsx0, int nLevels,
                                                     float zLiquid, float waveAmp, int nWaves,
                                                     int nSpheres, float rMin, float rMax,
                                                     int nCuboids, int nModes, int kMax,
                                                     float band, uint64_t seed);
void msbg_scene_pressure_destroy(msbg_pressure_scene* s);
/* Refinement map (levels per base block, bid order). */
int msbg_scene_pressure_block_levels(const msbg_pressure_scene* s, int* levels);
/* The scene as per-cell arrays in the packed layout msbg_gpu_pressure_prepare_arrays
 * takes: for every base block in bid order, (bsx0 >> level)^3 cells
 * (vid = x + y*bs + z*bs*bs), each sampled by the callbacks below at the fine
 * voxel of its lowest corner: cell type, lower-face coefficient per direction,
 * rhs.  Each array holds the sum over blocks of (bsx0 >> level)^3 values. */
int msbg_scene_pressure_arrays(const msbg_pressure_scene* s, uint16_t* flags, float* faceX,
                               float* faceY, float* faceZ, float* rhs);
uint16_t msbg_scene_cell_type(void* scene, int x, int y, int z);
float msbg_scene_face_coeff(void* scene, int dir, int x, int y, int z);
float msbg_scene_rhs(void* scene, int x, int y, int z);

#ifdef __cplusplus
}
#endif

#endif /* MSBG_SCENE_H */
