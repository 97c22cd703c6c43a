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

#ifdef __cplusplus
}
#endif

#endif /* MSBG_SCENE_H */
