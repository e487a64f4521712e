/*
 * CPU oracle for the batched symmetric eigensolver -- TEST INFRASTRUCTURE.
 *
 * A scalar C restatement of the reference's per-matrix algorithm
 * (EigenG-Batched: tred1_tiled.hpp, tql2_tiled.hpp, imtql2_tiled.hpp,
 * hhtr2sy_tiled.hpp, jac_tiled.hpp, eigen_GPU_check.cu, main.cpp
 * generators), with OpenMP over the matrices of a batch.  It is the checker
 * for the CUDA library and the timed CPU baseline; only tests/, the smoke
 * entry and bench.py's CPU legs load it.
 *
 * Pinning: the Frank-matrix analytic eigenvalues (eigen_GPU_check.cu:17-32),
 * scipy's LAPACK dsyev/ssyev, and outputs of the reference's own GPU build
 * (oracle/_ref, fixtures under tests/golden/) check this restatement.
 *
 * Deliberate difference: for n == 2 the reference's n<=32 path returns the
 * input matrix unchanged in `a` (tred1_tiled.hpp:25-34 skips the reduction
 * and hhtr2sy_tiled.hpp:27-35 returns before the copy-back); the oracle runs
 * the general algorithm and returns the eigenvectors.
 */
#include <math.h>
#include <omp.h>
#include <stddef.h>
#include <stdint.h>
#include <stdlib.h>

/* ---------------- double ---------------- */
#define T double
#define SFX(x) x##_d
static inline double o_eps_d(void) { return 2.220446049250313080847e-16; }
#include "eigen_oracle_body.h"
#undef T
#undef SFX

/* ---------------- float ----------------- */
#define T float
#define SFX(x) x##_f
static inline float o_eps_f(void) { return 1.1920928955078125e-07f; }
#include "eigen_oracle_body.h"
#undef T
#undef SFX

int oracle_num_threads(void) { return omp_get_max_threads(); }
