"""Ring bookkeeping of the batched solver's cluster kernel, on the CPU.

batch_cluster_kernel (jacobi-svd-cuda_b200/csrc/batched.cu) keeps a member's
columns in the distributed shared memory of a C-CTA cluster laid out as the
round-robin circle: CTA i owns the pair slots [i*half/C, (i+1)*half/C), its
top slots are a ring of S+1 buffers indexed (j - jt0 - g) mod (S+1 - jt0) at
round g, its bottom slots a ring indexed (j + g) mod (S+1), and per round it
sends its last top column to the right neighbour's spare top buffer and its
first bottom column to the left neighbour's spare bottom buffer (the end
CTAs turn the circle into their own spare buffers).  The kernel tracks
these indices incrementally; this test restates that bookkeeping step for
step and checks, with column ids in place of data, that
  * every slot of every round reads the ordered pair (p, q) that the
    reference's round-robin schedule gives for that round (src/kernels.cu:
    637-678, through the oracle's jo_schedule), dummy slots of odd n skipped;
  * a moved column lands only in a buffer nobody reads in that round, and no
    buffer is written twice;
  * every buffer index stays inside the CTA's (2 * smax + 3) buffers;
  * after whole sweeps position p holds column p again (where the kernel
    reads sigma, U and V from).
"""
import pytest

import oracle as O


def _simulate(n, C, sweeps, nwarps=16, slots_per_warp=4):
    ne = n + (n & 1)
    half, L = ne // 2, ne - 1
    rounds = L if n >= 2 else 0
    smax = (half + C - 1) // C
    nbuf = 2 * smax + 3  # buffer 0: column 0 (CTA 0); 1..smax+1: top ring; smax+2..: bottom ring
    top0, bot0 = 1, smax + 2
    sched = O.schedule(n)
    ctas = []
    for rank in range(C):
        k0, k1 = rank * half // C, (rank + 1) * half // C
        S = k1 - k0
        assert S >= 2
        jt0 = 1 if rank == 0 else 0
        c = dict(k0=k0, S=S, jt0=jt0, rt=S - jt0 + 1, rb=S + 1,
                 sr=(rank + 2) * half // C - k1 if rank < C - 1 else 0,
                 sl=k0 - (rank - 1) * half // C if rank > 0 else 0, slots=[])
        c["o_top"] = c["sr"] if rank < C - 1 else S
        c["o_bot"] = c["sl"] if rank > 0 else c["rt"] - 1
        for w in range(nwarps):
            for t in range(slots_per_warp):
                j = w + t * nwarps
                if j < S:
                    k = k0 + j
                    c["slots"].append(dict(j=j, pv=k, qv=ne - 1 - k, tb=-1 if (rank == 0 and j == 0) else j - jt0,
                                           bb=j))
        ctas.append(c)

    def top_buf(c, tb):
        return 0 if tb < 0 else top0 + tb

    mem = [dict() for _ in range(C)]
    for rank, c in enumerate(ctas):  # round 0: position p holds column p
        for sl in c["slots"]:
            for val, buf in ((sl["pv"], top_buf(c, sl["tb"])), (sl["qv"], bot0 + sl["bb"])):
                if val != n:
                    mem[rank][buf] = val
    for _ in range(sweeps):
        for r in range(rounds):
            seen, writes, reads = [], [], set()
            for rank, c in enumerate(ctas):
                S = c["S"]
                for sl in c["slots"]:
                    j = sl["j"]
                    xt, xb = (rank, top_buf(c, sl["tb"])), (rank, bot0 + sl["bb"])
                    if j == S - 1:
                        dt = (rank + 1, top0 + c["o_top"]) if rank < C - 1 else (rank, bot0 + c["o_top"])
                    else:
                        dt = xt
                    if j == 0:
                        db = (rank - 1, bot0 + c["o_bot"]) if rank > 0 else (rank, top0 + c["o_bot"])
                    else:
                        db = xb
                    for buf in (xt, xb, dt, db):
                        assert 0 <= buf[1] < nbuf
                    p = None if sl["pv"] == n else mem[rank].get(xt[1])
                    q = None if sl["qv"] == n else mem[rank].get(xb[1])
                    if p is not None and q is not None:
                        seen.append((p, q))
                    reads.update((xt, xb))
                    if p is not None:
                        writes.append((dt, p, xt))
                    if q is not None:
                        writes.append((db, q, xb))
                    # the kernel's incremental updates
                    if sl["pv"] != 0:
                        sl["pv"] = L if sl["pv"] == 1 else sl["pv"] - 1
                    sl["qv"] = L if sl["qv"] == 1 else sl["qv"] - 1
                    if sl["tb"] >= 0:
                        sl["tb"] = c["rt"] - 1 if sl["tb"] == 0 else sl["tb"] - 1
                    sl["bb"] = 0 if sl["bb"] == c["rb"] - 1 else sl["bb"] + 1
                if rank < C - 1:
                    c["o_top"] = c["sr"] if c["o_top"] == 0 else c["o_top"] - 1
                else:
                    c["o_top"] = 0 if c["o_top"] == c["rb"] - 1 else c["o_top"] + 1
                if rank > 0:
                    c["o_bot"] = 0 if c["o_bot"] == c["sl"] else c["o_bot"] + 1
                else:
                    c["o_bot"] = c["rt"] - 1 if c["o_bot"] == 0 else c["o_bot"] - 1
            assert sorted(seen) == sorted(sched[r]), (n, C, r)
            dsts = [w[0] for w in writes]
            assert len(set(dsts)) == len(dsts)
            for dst, _, src in writes:
                assert dst == src or dst not in reads
            for dst, val, _ in writes:
                mem[dst[0]][dst[1]] = val
    for rank, c in enumerate(ctas):  # a whole sweep turns the circle once
        for sl in c["slots"]:
            k = c["k0"] + sl["j"]
            assert sl["pv"] == k and sl["qv"] == ne - 1 - k
            if k != n:
                assert mem[rank][top_buf(c, sl["tb"])] == k
            if ne - 1 - k != n:
                assert mem[rank][bot0 + sl["bb"]] == ne - 1 - k


@pytest.mark.parametrize("C", [2, 4, 8])
@pytest.mark.parametrize("n", [15, 16, 17, 31, 32, 33, 64, 65, 113, 120, 131, 150, 199, 229, 256])
def test_cluster_ring_follows_the_schedule(n, C):
    half = (n + (n & 1)) // 2
    if half < 2 * C:  # the host sends such members to a smaller cluster or none
        pytest.skip("fewer than two slots per CTA")
    _simulate(n, C, sweeps=2 if n <= 64 else 1)
