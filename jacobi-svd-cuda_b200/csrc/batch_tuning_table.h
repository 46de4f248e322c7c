/* Built-in launch shapes of the batched solver, one entry per size class:
 * {threads per CTA, persistent CTAs per SM, grid cap (0 = none)}.
 *
 * Generated by jacobi-svd-cuda_b200/batch_autotune.py on NVIDIA B200
 * (148 SMs), 2026-12-03, from jsvd_batch_autotune over 4000 FP32-stored matrices m ~ U{16..256}, n ~ U{8..m} (seed 3);
 * 2 runs per shape, L2 flushed before each, minimum kept.  A shape
 * replaces the previous built-in one only when it is more than 2% faster.
 *
 * class: members timed / in batch, shapes tried, ms previous -> chosen
 *   0 (A and V in <= 48 KiB of shared memory): 1535 / 1535, 9 shapes, 6.40 -> 6.40
 *   1 (A and V in <= 100 KiB of shared memory): 630 / 630, 6 shapes, 12.43 -> 12.43
 *   2 (A and V in <= ~226 KiB of shared memory): 844 / 844, 3 shapes, 46.86 -> 46.86
 *   3 (A in shared memory, V in global memory): 485 / 485, 9 shapes, 76.49 -> 76.49
 *   4 (A and V in global memory): 506 / 506, 9 shapes, 240.89 -> 240.89
 *
 * CTAs per matrix: the classes whose bit is set in JSVD_BATCH_CLUSTER_CLASSES
 * are solved by a thread-block cluster per matrix (2, 4 or 8 CTAs, the
 * smallest that holds it), the others by one CTA per matrix; a class goes
 * over only when that is more than 2% faster.
 * Timed on NVIDIA B200 (148 SMs), 2026-12-04, over 20000 FP32-stored matrices (seed 3), all classes, mean of 3 runs, L2 flushed.
 * class: ms one CTA per matrix, ms clusters -> chosen
 *   2: 209.9, 220.0 -> one CTA
 *   3: 362.9, 334.5 -> clusters
 *   4: 1134.1, 956.9 -> clusters
 */
#pragma once

#define JSVD_BATCH_TUNING_TABLE \
    { {256, 4, 0}, {256, 2, 0}, {512, 1, 0}, {512, 1, 0}, {512, 1, 0} }

#define JSVD_BATCH_CLUSTER_CLASSES 0x18
