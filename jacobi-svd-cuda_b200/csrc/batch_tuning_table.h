/* Built-in launch shapes of the batched solver, one entry per size class:
 * {threads per CTA, persistent CTAs per SM, grid cap (0 = none)}.
 * Classes: A and V in <= 48 KiB / <= 100 KiB / <= ~226 KiB of shared memory;
 * A alone in shared memory; A and V in global memory.
 *
 * Source: hand-picked from launch-shape sweeps of the 20,000-matrix mixed
 * batch (m ~ U{16..256}, n ~ U{8..m}, FP32-stored, seed 3) on one B200.
 * jacobi-svd-cuda_b200/batch_autotune.py regenerates this file from
 * jsvd_batch_autotune on the device it runs on. */
#pragma once

#define JSVD_BATCH_TUNING_TABLE \
    { {256, 4, 0}, {256, 2, 0}, {512, 1, 0}, {512, 1, 0}, {512, 1, 0} }
