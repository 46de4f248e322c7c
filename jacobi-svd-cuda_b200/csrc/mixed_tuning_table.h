/* Built-in choices of the blocked mixed-precision path by matrix width:
 * {largest column count the entry covers (0 = any), tensor-core sweep cap,
 * inner sweeps of the block eigen-solve, Gram row splits (0 = automatic)}.
 * The first entry whose column bound covers the input applies.
 *
 * Hand-set from measurements on a B200 (4096 x 1024: a cap of 4 sweeps and one
 * inner sweep 31.6 ms against 34.6 ms with 10; 8192 x 4096: 10 sweeps 6% faster
 * than 4); regenerate with jacobi-svd-cuda_b200/mixed_autotune.py.
 */
#pragma once

#define JSVD_MIXED_TUNING_TABLE \
    { {2048, 4, 1, 0}, {0, 10, 1, 0} }
