#!/usr/bin/env python3
"""Generate pair_tables.inc: the sector order of the pair layout for N <= 8.

An ADO (N x N complex) is stored as P = N(N-1)/2 + ceil(N/2) sectors of
32 B; each sector holds a symmetric pair (w(i,j), w(j,i)) or two diagonal
elements.  The stage kernel for N <= 8 runs one warp per ADO and computes the
commutator with FP64 m8n8k4 MMAs on the tile zero-padded to 8 x 8: lane
l = 4r + t reads, for k-slice s, the sector of the pair {r, 4s+t}, whose two
halves are exactly its A-fragment element (r, 4s+t) and its B-fragment
element (4s+t, r).  The MMA result (r, 2t), (r, 2t+1) goes through a
swizzled row-major tile in shared memory (chunk = 8 r + (c ^ swz(r))) to the
lane that owns the sector.

This script searches (simulated annealing) the sector numbering and the
orientation of each pair so that
  * the fragment reads of every quarter warp hit 8 different 16-byte bank
    groups (no shared-memory bank conflicts),
  * the exchange reads (owner lane p reading C(e1), C(e2)) are conflict free,
  * secondarily, the sectors of each bath's cross (row b and column b) fall
    into as few 128-byte lines as possible.
The result is deterministic for the fixed seeds below.

Usage: python gen_pair_tables.py OUT.inc
"""
import random
import sys
from collections import Counter


def swz(r):
    return ((r & 1) << 2) | (r & 1) | (((r >> 1) & 1) << 1)


def items_of(n):
    off = [(i, j) for i in range(n) for j in range(i + 1, n)]
    diag = [(2 * k, min(2 * k + 1, n - 1)) for k in range((n + 1) // 2)]
    return off, diag


def build(n, perm, orient):
    off, diag = items_of(n)
    table = [None] * len(perm)
    for it, (a, b) in enumerate(off + diag):
        if it < len(off):
            e1, e2 = (a, b), (b, a)
        else:
            e1, e2 = (a, a), (b, b)
        if orient[it] and e1 != e2:
            e1, e2 = e2, e1
        table[perm[it]] = (e1, e2)
    return table


def cost(n, perm, orient, w_lines=0.05):
    table = build(n, perm, orient)
    loc = {}
    for sec, (e1, e2) in enumerate(table):
        loc.setdefault(e1, (sec, 0))
        loc.setdefault(e2, (sec, 1))
    c = 0
    for q in range(4):
        for s in range(2):
            for which in (0, 1):
                ch = []
                for rr in (2 * q, 2 * q + 1):
                    for t in range(4):
                        col = 4 * s + t
                        if rr >= n or col >= n:
                            continue
                        e = (rr, col) if which == 0 else (col, rr)
                        if rr == col and which == 1:
                            continue
                        sec, h = loc[e]
                        ch.append((2 * sec + h) % 8)
                if ch:
                    c += max(Counter(ch).values()) - 1
    P = len(table)
    for k in range(0, P, 8):
        for which in (0, 1):
            ch = [table[p][which][1] ^ swz(table[p][which][0]) for p in range(k, min(P, k + 8))]
            c += max(Counter(ch).values()) - 1
    lines = 0
    for b in range(n):
        secs = [p for p, (e1, e2) in enumerate(table) if b in e1 or b in e2]
        lines += len({p // 4 for p in secs})
    return c + w_lines * lines, c, lines


def search(n, seed):
    off, diag = items_of(n)
    P = len(off) + len(diag)
    rng = random.Random(seed)
    best = None
    for restart in range(40):
        perm = list(range(P))
        rng.shuffle(perm)
        orient = [rng.randint(0, 1) for _ in range(P)]
        cur = cost(n, perm, orient)[0]
        T = 2.0
        for _ in range(30000):
            if rng.random() < 0.6 and P > 1:
                a, b = rng.sample(range(P), 2)
                perm[a], perm[b] = perm[b], perm[a]
                nc = cost(n, perm, orient)[0]
                if nc <= cur or rng.random() < 2.718 ** ((cur - nc) / T):
                    cur = nc
                else:
                    perm[a], perm[b] = perm[b], perm[a]
            else:
                a = rng.randrange(P)
                orient[a] ^= 1
                nc = cost(n, perm, orient)[0]
                if nc <= cur or rng.random() < 2.718 ** ((cur - nc) / T):
                    cur = nc
                else:
                    orient[a] ^= 1
            T = max(0.02, T * 0.9997)
        tot, c, lines = cost(n, perm, orient)
        if best is None or tot < best[0]:
            best = (tot, c, lines, perm[:], orient[:])
        if c == 0 and lines <= 4 * n:
            break
    tot, c, lines, perm, orient = best
    return build(n, perm, orient), c, lines


def main():
    out = sys.argv[1]
    rows = []
    for n in range(1, 9):
        if n == 1:
            table, c, lines = [((0, 0), (0, 0))], 0, 1
        else:
            table, c, lines = search(n, 1000 + n)
        e1 = [a[0] * n + a[1] for a, b in table]
        e2 = [b[0] * n + b[1] for a, b in table]
        rows.append((n, e1, e2, c, lines))
        print(f"N={n}: P={len(table)} conflicts={c} lines={lines}", flush=True)
    with open(out, "w") as f:
        f.write("/* Generated by gen_pair_tables.py: sector order of the pair layout for N <= 8.\n"
                " * kPairE1[N][p], kPairE2[N][p] = row-major element index of the two halves of\n"
                " * sector p (equal for the padding half of an odd N's last diagonal sector). */\n")
        f.write("static const signed char kPairE1[9][32] = {\n    {0},\n")
        for n, e1, e2, c, lines in rows:
            f.write("    {" + ", ".join(map(str, e1)) + "}, /* N=%d conflicts=%d lines=%d */\n" % (n, c, lines))
        f.write("};\nstatic const signed char kPairE2[9][32] = {\n    {0},\n")
        for n, e1, e2, c, lines in rows:
            f.write("    {" + ", ".join(map(str, e2)) + "},\n")
        f.write("};\n")


if __name__ == "__main__":
    main()
