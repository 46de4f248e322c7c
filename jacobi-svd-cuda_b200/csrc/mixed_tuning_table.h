/* Built-in choices of the blocked mixed-precision path by matrix width:
 * {largest column count the entry covers (0 = any), tensor-core sweep cap,
 * inner sweeps of the block eigen-solve, Gram row splits (0 = automatic)}.
 * The first entry whose column bound covers the input applies.
 *
 * Generated by jacobi-svd-cuda_b200/mixed_autotune.py on NVIDIA B200,
 * 2026-12-04: A = U diag(sigma) V^T, Haar U and V, sigma geometric 1 .. 1e-6, epsilon 1e-14; 2 timed solves per
 * candidate after a warm-up, minimum kept; candidates with sigma off by
 * more than 1e-12 normwise rejected; a candidate replaces the previous
 * choice only when it is more than 2% faster.
 *
 * width: shape, candidates tried (rejected), ms with the previous table -> chosen
 *   256: 1024 x 256, 15 (0), 6.3 -> 5.9
 *   512: 2048 x 512, 15 (0), 13.2 -> 13.2
 *   1024: 4096 x 1024, 15 (0), 32.1 -> 32.1
 *   2048: 8192 x 2048, 15 (0), 112.5 -> 105.5
 *   4096: 8192 x 4096, 15 (0), 537.4 -> 523.4
 */
#pragma once

#define JSVD_MIXED_TUNING_TABLE \
    { {256, 0, 1, 4}, {512, 4, 1, 0}, {1024, 4, 1, 0}, {2048, 6, 1, 8}, {0, 6, 2, 4} }
