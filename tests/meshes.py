"""Small analytic meshes used only by the tests."""
import numpy as np

from ocfd_b200.connectivity import BC_FARFIELD, BC_SYMMETRY, InpBlock, InpSub, interface
from ocfd_b200.meshgen import Case


def wavy_box(nx=17, ny=13, nz=9, amp=0.02, seed=7, nblk=1, cuts=None):
    """Unit box with smooth sinusoidal node displacement (closed-form, so shared node planes of
    split blocks coincide exactly), far-field on every physical face; cut into nblk blocks in i."""
    rng = np.random.default_rng(seed)
    ph = rng.uniform(0, 2 * np.pi, 3)
    x = np.linspace(0.0, 1.0, nx)
    y = np.linspace(0.0, 1.0, ny) ** 1.2
    z = np.linspace(0.0, 0.5, nz)
    Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
    s = np.sin(np.pi * X) * np.sin(np.pi * Y) * np.sin(2 * np.pi * Z)
    P = np.stack([X + amp * s * np.cos(ph[0]), Y + amp * s * np.cos(ph[1]), Z + amp * s * np.cos(ph[2])])
    if cuts is None:
        cuts = [int(round(1 + (nx - 1) * q / nblk)) for q in range(1, nblk)]
    cuts = [1] + list(cuts) + [nx]
    nblk = len(cuts) - 1
    xyz, inp = [], []
    for b in range(nblk):
        i0, i1 = cuts[b], cuts[b + 1]
        n = i1 - i0 + 1
        B = InpBlock(n, ny, nz)
        if b == 0:
            B.subs.append(InpSub((1, 1, 1, ny, 1, nz), BC_FARFIELD))
        B.subs.append(InpSub((1, n, 1, 1, 1, nz), BC_FARFIELD))
        B.subs.append(InpSub((1, n, ny, ny, 1, nz), BC_FARFIELD))
        B.subs.append(InpSub((1, n, 1, ny, 1, 1), BC_FARFIELD))
        B.subs.append(InpSub((1, n, 1, ny, nz, nz), BC_FARFIELD))
        if b == nblk - 1:
            B.subs.append(InpSub((n, n, 1, ny, 1, nz), BC_FARFIELD))
        xyz.append(np.ascontiguousarray(P[:, :, :, i0 - 1:i1]))
        inp.append(B)
    for b in range(nblk - 1):
        nA = inp[b].nx
        sA, sB = interface(b + 1, ((nA, nA), (1, ny), (1, nz)), b + 2, lambda i, j, k: (1, j, k))
        inp[b].subs.append(sA)
        inp[b + 1].subs.insert(0, sB)
    return Case("wavy_box_%dx%dx%d_b%d" % (nx, ny, nz, nblk), xyz, inp)


def mirrored_bump(ni=33, nj=17, nk=9):
    """The channel-bump mesh mirrored in z about its mid plane (k -> nk+1-k gives the same nodes
    with z -> 0.25 - z); used for the symmetry pin."""
    from ocfd_b200 import meshgen
    return meshgen.channel_bump(ni, nj, nk)
