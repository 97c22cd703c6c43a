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

#ifdef __cplusplus
}
#endif

#endif
