"""Block connectivity: Gridgen ``bc3d.inp`` records and the reference's internal ``.inc`` form.

``convert_inp_inc`` restates sub_convert_inp.f90:25-248 (Convert_bc + the partner-subface
search); the 21-int ``.inc`` record order is sub_IO.f90:700-705:
ib,ie,jb,je,kb,ke,bc,face,f_no, ib1,ie1,jb1,je1,kb1,ke1,nb1,face1,f_no1,L1,L2,L3.

``Interface`` builds the pair of signed ``.inp`` records for a block-to-block connection from a
plain node-index correspondence, the way a mesh generator (Gridgen) would write them.
"""
from dataclasses import dataclass, field
from typing import List, Optional, Tuple

import numpy as np

BC_WALL, BC_SYMMETRY, BC_FARFIELD, BC_INFLOW, BC_OUTFLOW, BC_INNER = 2, 3, 4, 5, 6, -1


@dataclass
class InpSub:
    rng: Tuple[int, int, int, int, int, int]  # signed ib,ie,jb,je,kb,ke as in bc3d.inp
    bc: int
    rng1: Optional[Tuple[int, int, int, int, int, int]] = None  # partner range (inner only)
    nb1: int = 0  # partner block, 1-based


@dataclass
class InpBlock:
    nx: int
    ny: int
    nz: int
    subs: List[InpSub] = field(default_factory=list)


def _convert_bc(kb, ke, bc, kb1, ke1, nb1):
    """Convert_bc (sub_convert_inp.f90:131-248) for one subface; returns the 21-int record
    without f_no / f_no1 (filled by the caller)."""
    s = [0, 0, 0]
    for k in range(3):
        if kb[k] == ke[k]:
            s[k] = 0
        elif kb[k] > 0:
            s[k] = 1
        else:
            s[k] = -1
    ib, ie = min(abs(kb[0]), abs(ke[0])), max(abs(kb[0]), abs(ke[0]))
    jb, je = min(abs(kb[1]), abs(ke[1])), max(abs(kb[1]), abs(ke[1]))
    kb_, ke_ = min(abs(kb[2]), abs(ke[2])), max(abs(kb[2]), abs(ke[2]))
    if s[0] == 0:
        face = 1 if ib == 1 else 4
    elif s[1] == 0:
        face = 2 if jb == 1 else 5
    else:
        face = 3 if kb_ == 1 else 6
    rec = [ib, ie, jb, je, kb_, ke_, bc, face, 0]
    if bc >= 0:
        return rec + [0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0]
    p = [0, 0, 0]
    for k in range(3):
        if kb1[k] == ke1[k]:
            p[k] = 0
        elif kb1[k] > 0:
            p[k] = 1
        else:
            p[k] = -1
    ib1, ie1 = min(abs(kb1[0]), abs(ke1[0])), max(abs(kb1[0]), abs(ke1[0]))
    jb1, je1 = min(abs(kb1[1]), abs(ke1[1])), max(abs(kb1[1]), abs(ke1[1]))
    kb1_, ke1_ = min(abs(kb1[2]), abs(ke1[2])), max(abs(kb1[2]), abs(ke1[2]))
    if p[0] == 0:
        face1 = 1 if ib1 == 1 else 4
    elif p[1] == 0:
        face1 = 2 if jb1 == 1 else 5
    else:
        face1 = 3 if kb1_ == 1 else 6
    Lp = [0, 0, 0]
    for k in range(3):
        for j in range(3):
            if s[k] == p[j]:
                Lp[k] = j + 1
    for k in range(3):
        k1 = Lp[k] - 1
        if s[k] != 0:
            if (ke[k] - kb[k]) * (ke1[k1] - kb1[k1]) < 0:
                Lp[k] = -Lp[k]
        else:
            if (face - 1) // 3 == (face1 - 1) // 3:
                Lp[k] = -Lp[k]
    return rec + [ib1, ie1, jb1, je1, kb1_, ke1_, nb1, face1, 0] + Lp


def convert_inp_inc(blocks: List[InpBlock]) -> List[List[List[int]]]:
    """convert_inp_inc (sub_convert_inp.f90:25-122): list (per block) of 21-int records."""
    inc = []
    for b in blocks:
        recs = []
        for ksub, s in enumerate(b.subs, start=1):
            kb = [s.rng[0], s.rng[2], s.rng[4]]
            ke = [s.rng[1], s.rng[3], s.rng[5]]
            if s.bc < 0:
                kb1 = [s.rng1[0], s.rng1[2], s.rng1[4]]
                ke1 = [s.rng1[1], s.rng1[3], s.rng1[5]]
                r = _convert_bc(kb, ke, s.bc, kb1, ke1, s.nb1)
            else:
                r = _convert_bc(kb, ke, s.bc, None, None, 0)
            r[8] = ksub
            recs.append(r)
        inc.append(recs)
    for m, recs in enumerate(inc, start=1):
        for r in recs:
            if r[6] < 0:
                found = 0
                for ks1, r1 in enumerate(inc[r[15] - 1], start=1):
                    if r[9:15] == r1[0:6] and r1[15] == m:
                        found = ks1
                        break
                if found == 0:
                    raise ValueError("partner subface not found (block %d)" % m)
                r[17] = found
    return inc


def interface(nbA, rngA, nbB, mapping):
    """Signed .inp records for the connection of block A's face to block B's face.

    rngA: ((i0,i1),(j0,j1),(k0,k1)) node ranges of A's face (one dim constant).
    mapping: callable (i,j,k) of A -> (i,j,k) of B for the nodes of the face (affine per dim).
    Returns (InpSub for A, InpSub for B).
    """
    const = [d for d in range(3) if rngA[d][0] == rngA[d][1]]
    assert len(const) == 1, rngA
    cA = const[0]
    tan = [d for d in range(3) if d != cA]
    lo = [rngA[d][0] for d in range(3)]
    hi = [rngA[d][1] for d in range(3)]
    pB0 = mapping(*lo)
    pB1 = mapping(*hi)
    # the B dimension that varies with each tangential A dimension
    corr = {}
    for t in tan:
        q = list(lo)
        q[t] = hi[t]
        pq = mapping(*q)
        diff = [pq[d] - pB0[d] for d in range(3)]
        dB = [d for d in range(3) if diff[d] != 0]
        assert len(dB) == 1, (diff, rngA)
        corr[t] = dB[0]
    cB = [d for d in range(3) if d not in corr.values()][0]
    assert pB0[cB] == pB1[cB]
    sign = {tan[0]: 1, tan[1]: -1}
    rA = []
    for d in range(3):
        a, b = rngA[d]
        s = sign.get(d, 1)
        rA += [s * a, s * b]
    rB = [0] * 6
    for d in range(3):
        if d == cB:
            rB[2 * d] = rB[2 * d + 1] = pB0[d]
    for t in tan:
        dB = corr[t]
        s = sign[t]
        rB[2 * dB] = s * pB0[dB]
        rB[2 * dB + 1] = s * pB1[dB]
    return (InpSub(tuple(rA), BC_INNER, tuple(rB), nbB), InpSub(tuple(rB), BC_INNER, tuple(rA), nbA))


def flat_inc(inc):
    """(nsub int32 array, concatenated int32 .inc array) for the C-ABI."""
    nsub = np.array([len(r) for r in inc], dtype=np.int32)
    flat = np.array([v for recs in inc for r in recs for v in r], dtype=np.int32)
    return nsub, flat


def write_bc3d_inp(path, blocks: List[InpBlock]):
    """Gridgen generic bc3d.inp as read by sub_convert_inp.f90:46-72."""
    with open(path, "w") as f:
        f.write(" 1\n%d\n" % len(blocks))
        for m, b in enumerate(blocks, start=1):
            f.write("%d %d %d\n" % (b.nx, b.ny, b.nz))
            f.write("Block %d\n" % m)
            f.write("%d\n" % len(b.subs))
            for s in b.subs:
                f.write("%6d%6d%6d%6d%6d%6d%6d\n" % (*s.rng, s.bc))
                if s.bc < 0:
                    f.write("%6d%6d%6d%6d%6d%6d%6d\n" % (*s.rng1, s.nb1))


def read_bc3d_inp(path) -> List[InpBlock]:
    toks = []
    with open(path) as f:
        lines = f.read().splitlines()
    it = iter(lines)
    next(it)
    nb = int(next(it).split()[0])
    blocks = []
    for _ in range(nb):
        nx, ny, nz = [int(v) for v in next(it).split()[:3]]
        next(it)
        ns = int(next(it).split()[0])
        b = InpBlock(nx, ny, nz)
        for _ in range(ns):
            v = [int(x) for x in next(it).split()[:7]]
            if v[6] < 0:
                w = [int(x) for x in next(it).split()[:7]]
                b.subs.append(InpSub(tuple(v[:6]), v[6], tuple(w[:6]), w[6]))
            else:
                b.subs.append(InpSub(tuple(v[:6]), v[6]))
        blocks.append(b)
    del toks
    return blocks
