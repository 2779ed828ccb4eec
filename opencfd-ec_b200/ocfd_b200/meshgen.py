"""Analytic, seeded structured meshes for the benchmark configurations.

Every mesh is returned as a ``Case``: per-block node coordinates (shape (3, nz, ny, nx), i.e.
Fortran x(1:nx,1:ny,1:nz) with i fastest), the Gridgen-style ``bc3d.inp`` records and the
derived ``.inc`` records.  No external mesh or dataset is used: these generators stand in for the
reference's case files, whose meshes are not shipped (.MISSING_LARGE_BLOBS:1).

* ``channel_bump``   -- config 1: 129x65x17 channel with a sin^2 bump, optionally cut in i.
* ``airfoil_omesh``  -- NACA 4-digit O-mesh extruded over k (config 4's 2-D airfoils).
* ``swept_wing``     -- config 2: O-H mesh around a tapered, swept NACA 0012 wing (8 blocks);
                        config 3 adds an ellipsoidal fuselage at the root (24 blocks).
"""
import math
from dataclasses import dataclass, field
from typing import List

import numpy as np

from .connectivity import (BC_FARFIELD, BC_INFLOW, BC_OUTFLOW, BC_SYMMETRY, BC_WALL, InpBlock,
                           InpSub, convert_inp_inc, flat_inc, interface)


@dataclass
class Case:
    name: str
    xyz: List[np.ndarray]                      # per block (3, nz, ny, nx) float64
    inp: List[InpBlock]
    inc: List[List[List[int]]] = field(default_factory=list)
    meta: dict = field(default_factory=dict)

    def __post_init__(self):
        if not self.inc:
            self.inc = convert_inp_inc(self.inp)

    @property
    def dims(self):
        return [(a.shape[3], a.shape[2], a.shape[1]) for a in self.xyz]

    @property
    def ncells(self):
        return sum((nx - 1) * (ny - 1) * (nz - 1) for nx, ny, nz in self.dims)

    def flat(self):
        nijk = np.array([v for d in self.dims for v in d], dtype=np.int32)
        nsub, inc = flat_inc(self.inc)
        xyz = [np.ascontiguousarray(a, dtype=np.float64) for a in self.xyz]
        return nijk, xyz, nsub, inc


def _stretch(n, ratio):
    """n-1 intervals with geometric ratio, normalised to [0,1]."""
    if abs(ratio - 1.0) < 1e-12:
        return np.linspace(0.0, 1.0, n)
    d = ratio ** np.arange(n - 1)
    s = np.concatenate([[0.0], np.cumsum(d)])
    return s / s[-1]


def _split_points(n, cuts):
    """node index boundaries 1..n for given cut node indices."""
    return [1] + list(cuts) + [n]


def channel_bump(ni=129, nj=65, nk=17, cuts_i=(), name="bump"):
    """Config 1: x in [-1.5,2.5], height 1, lower wall y = 0.05 sin^2(pi x) on [0,1], z in
    [0,0.25] with symmetry planes, j stretched from the lower wall with ratio 1.05; inflow at
    i-, outflow at i+ (far-field BC), slip walls at j-/j+ (inviscid).  cuts_i splits the
    channel into blocks at the given node indices (shared node planes)."""
    x1 = np.linspace(-1.5, 2.5, ni)
    ybot = np.where((x1 >= 0.0) & (x1 <= 1.0), 0.05 * np.sin(np.pi * x1) ** 2, 0.0)
    eta = _stretch(nj, 1.05)
    z1 = np.linspace(0.0, 0.25, nk)
    X = np.empty((3, nk, nj, ni))
    X[0] = x1[None, None, :]
    X[1] = ybot[None, None, :] + (1.0 - ybot[None, None, :]) * eta[None, :, None]
    X[2] = z1[:, None, None]
    bnds = _split_points(ni, cuts_i)
    nb = len(bnds) - 1
    xyz, inp = [], []
    for b in range(nb):
        i0, i1 = bnds[b], bnds[b + 1]
        blk = np.ascontiguousarray(X[:, :, :, i0 - 1:i1])
        nx = i1 - i0 + 1
        B = InpBlock(nx, nj, nk)
        if b == 0:
            B.subs.append(InpSub((1, 1, 1, nj, 1, nk), BC_FARFIELD))
        B.subs.append(InpSub((1, nx, 1, 1, 1, nk), BC_WALL))
        B.subs.append(InpSub((1, nx, nj, nj, 1, nk), BC_WALL))
        B.subs.append(InpSub((1, nx, 1, nj, 1, 1), BC_SYMMETRY))
        B.subs.append(InpSub((1, nx, 1, nj, nk, nk), BC_SYMMETRY))
        if b == nb - 1:
            B.subs.append(InpSub((nx, nx, 1, nj, 1, nk), BC_FARFIELD))
        xyz.append(blk)
        inp.append(B)
    for b in range(nb - 1):
        nxA = inp[b].nx
        sA, sB = interface(b + 1, ((nxA, nxA), (1, nj), (1, nk)), b + 2, lambda i, j, k: (1, j, k))
        inp[b].subs.append(sA)
        inp[b + 1].subs.insert(0, sB)
    return Case(name, xyz, inp, meta=dict(kind="bump", ni=ni, nj=nj, nk=nk))


def naca4(m, p, t, n_half, cluster=True):
    """Closed-trailing-edge NACA 4-digit section (closed-form thickness law with the -0.1036
    coefficient).  Returns (x, y) of 2*n_half-1 points, TE(lower) -> LE -> TE(upper), clockwise
    seen from +z so that the O-mesh i index runs around the section."""
    beta = np.linspace(0.0, np.pi, n_half)
    xc = 0.5 * (1.0 - np.cos(beta)) if cluster else np.linspace(0.0, 1.0, n_half)
    yt = 5.0 * t * (0.2969 * np.sqrt(xc) - 0.1260 * xc - 0.3516 * xc ** 2 + 0.2843 * xc ** 3 - 0.1036 * xc ** 4)
    if m > 0 and p > 0:
        yc = np.where(xc < p, m / p ** 2 * (2 * p * xc - xc ** 2), m / (1 - p) ** 2 * ((1 - 2 * p) + 2 * p * xc - xc ** 2))
        dyc = np.where(xc < p, 2 * m / p ** 2 * (p - xc), 2 * m / (1 - p) ** 2 * (p - xc))
    else:
        yc = np.zeros_like(xc)
        dyc = np.zeros_like(xc)
    th = np.arctan(dyc)
    xu, yu = xc - yt * np.sin(th), yc + yt * np.cos(th)
    xl, yl = xc + yt * np.sin(th), yc - yt * np.cos(th)
    # lower surface TE->LE then upper LE->TE
    x = np.concatenate([xl[::-1], xu[1:]])
    y = np.concatenate([yl[::-1], yu[1:]])
    return x, y


def _surface_normals(xs, ys):
    """Unit outward normals of a closed clockwise section polyline (first point == last point);
    the trailing-edge point gets the bisector of its two neighbours."""
    n = xs.size
    ip = np.r_[1:n, 1]          # next index (periodic, skipping the duplicate last point)
    im = np.r_[n - 2, 0:n - 1]  # previous index
    tx, ty = xs[ip] - xs[im], ys[ip] - ys[im]
    nx_, ny_ = -ty, tx          # left of the clockwise direction of travel = outward
    nrm = np.hypot(nx_, ny_)
    return nx_ / nrm, ny_ / nrm


def _omesh_plane(xs, ys, nxs, nys, nj, ds, radius, center):
    """O-mesh in one plane.  Surface points (xs, ys) with outward normals (nxs, nys) are joined to
    a circle of `radius` around `center`; the outer points are spread uniformly in angle
    (clockwise from the +x axis, like the section ordering).  Wall-normal rays near the wall blend
    into straight lines to the outer points; node spacing is geometric with first step `ds`."""
    n = xs.size
    ang = -2.0 * np.pi * np.arange(n) / (n - 1)
    xo = center[0] + radius * np.cos(ang)
    yo = center[1] + radius * np.sin(ang)
    s = _stretch(nj, _growth_for(nj, ds / radius))
    t = np.minimum(s / 0.05, 1.0)
    b = t * t * (3.0 - 2.0 * t)
    Xn = xs[None, :] + nxs[None, :] * radius * s[:, None]
    Yn = ys[None, :] + nys[None, :] * radius * s[:, None]
    Xl = xs[None, :] + (xo - xs)[None, :] * s[:, None]
    Yl = ys[None, :] + (yo - ys)[None, :] * s[:, None]
    X = (1.0 - b[:, None]) * Xn + b[:, None] * Xl
    Y = (1.0 - b[:, None]) * Yn + b[:, None] * Yl
    return X, Y  # (nj, n)


def _growth_for(n, ds):
    """ratio r such that the first of n-1 geometric intervals is ds of the total."""
    lo, hi = 1.0 + 1e-9, 2.0
    for _ in range(200):
        mid = 0.5 * (lo + hi)
        first = (mid - 1.0) / (mid ** (n - 1) - 1.0)
        if first > ds:
            lo = mid
        else:
            hi = mid
    return 0.5 * (lo + hi)


def airfoil_omesh(ni=129, nj=33, nk=3, m=0.0, p=0.0, t=0.12, radius=20.0, ds=2e-6, dz=0.1,
                  viscous=True, name="airfoil"):
    """2-D-extruded O-mesh around a NACA 4-digit section: i around the section (i=1 and i=ni
    are the same trailing-edge line, joined as a periodic inner boundary), j from the wall to a
    circular far field of `radius` chords, k extruded over dz with symmetry planes."""
    assert ni % 2 == 1
    xs, ys = naca4(m, p, t, (ni + 1) // 2)
    nxs, nys = _surface_normals(xs, ys)
    # first wall-normal step ds chords (y+ ~ 1 at Re ~ 6e6 when ds ~ 2e-6)
    X2, Y2 = _omesh_plane(xs, ys, nxs, nys, nj, ds, radius, (0.5, 0.0))
    X = np.empty((3, nk, nj, ni))
    X[0] = X2[None]
    X[1] = Y2[None]
    X[2] = np.linspace(0.0, dz, nk)[:, None, None]
    B = InpBlock(ni, nj, nk)
    B.subs.append(InpSub((1, ni, 1, 1, 1, nk), BC_WALL if viscous else BC_WALL))
    B.subs.append(InpSub((1, ni, nj, nj, 1, nk), BC_FARFIELD))
    B.subs.append(InpSub((1, ni, 1, nj, 1, 1), BC_SYMMETRY))
    B.subs.append(InpSub((1, ni, 1, nj, nk, nk), BC_SYMMETRY))
    sA, sB = interface(1, ((1, 1), (1, nj), (1, nk)), 1, lambda i, j, k: (ni, j, k))
    B.subs.insert(0, sA)
    B.subs.insert(1, sB)
    return Case(name, [X], [B], meta=dict(kind="airfoil", ni=ni, nj=nj, nk=nk, m=m, p=p, t=t))


def fuselage_lift(x, y, length=4.0, fineness=8.0, xc=0.5):
    """Height above the symmetry plane of a half ellipsoid of revolution about the x axis
    (length `length`, maximum diameter length / fineness, centred at x = xc), 0 outside it."""
    a, b = 0.5 * length, 0.5 * length / fineness
    q = 1.0 - ((x - xc) / a) ** 2 - (y / b) ** 2
    return b * np.sqrt(np.maximum(q, 0.0))


def swept_wing(ni=257, nj=97, nk_wing=61, nk_tip=26, i_cut=49, sweep_deg=30.0, taper=0.56,
               semi_span=1.5, radius=20.0, ds=4.5e-6, tip_far=15.0, name="wing", j_cuts=(), fuselage=None):
    """Config 2 stand-in: O-H mesh around a swept, tapered NACA 0012 wing.

    i runs around each spanwise section (O-type, periodic trailing-edge seam), j from the wall
    to a cylindrical far field of `radius` root chords, k from the root symmetry plane (z=0) over
    the wing (nk_wing nodes, tip clustered, elliptic tip rounding over the last 5 % of the span)
    and on to a far field `tip_far` chords beyond the tip (nk_tip nodes).  Beyond the tip the
    section collapses to its chord line and the j=1 surface becomes a sheet joining the lower and
    upper sides (an inner boundary i <-> ni+1-i).  Blocks: i cut at i_cut, the leading edge and
    ni+1-i_cut; k cut at the tip -> 8 uneven blocks; optional wall-normal cuts at the node
    indices j_cuts multiply that by len(j_cuts)+1.

    fuselage (dict of fuselage_lift's arguments, or None): the root surface k = 1 is lifted onto a
    half ellipsoid of revolution about the x axis (a wing-body configuration: the wing root sits on
    the body's side); every k line (i, j) is lifted by the ellipsoid's height above its root node,
    fading linearly to zero at 60 % of the semi-span, so every node keeps its order in k.  The root face keeps its symmetry condition, which on the lifted part makes the
    body a slip (inviscid) surface.
    """
    assert ni % 2 == 1
    mid = (ni + 1) // 2
    nk = nk_wing + nk_tip - 1
    # spanwise nodes
    zw = semi_span * np.sin(np.linspace(0.0, np.pi / 2, nk_wing))  # clustered toward the tip
    dz_tip = zw[-1] - zw[-2]
    gt = _growth_for(nk_tip, dz_tip / tip_far)
    zt = semi_span + tip_far * _stretch(nk_tip, gt)
    z = np.concatenate([zw, zt[1:]])
    xs0, ys0 = naca4(0.0, 0.0, 0.12, mid)
    nx0, ny0 = _surface_normals(xs0, ys0)
    tanL = math.tan(math.radians(sweep_deg))
    X = np.empty((3, nk, nj, ni))
    z0 = 0.95 * semi_span
    for k in range(nk):
        zk = min(z[k], semi_span)
        chord = 1.0 - (1.0 - taper) * zk / semi_span
        xle = zk * tanL
        if z[k] <= z0:
            th = 1.0
        elif z[k] < semi_span:
            th = math.sqrt(max(0.0, 1.0 - ((z[k] - z0) / (semi_span - z0)) ** 2))
        else:
            th = 0.0
        xs = xle + chord * xs0
        ys = chord * ys0 * th
        X2, Y2 = _omesh_plane(xs, ys, nx0, ny0, nj, ds, radius, (xle + 0.5 * chord, 0.0))
        X[0, k] = X2
        X[1, k] = Y2
        X[2, k] = z[k]
    if fuselage is not None:
        # one lift per (i, j) line, from the root plane's node: z stays monotone along every k line
        zb = 0.6 * semi_span
        lift = fuselage_lift(X[0, 0], X[1, 0], **fuselage)
        X[2] = X[2] + lift[None] * np.maximum(0.0, 1.0 - X[2] / zb)
    kt = nk_wing  # node index of the tip plane
    ibnd = [1, i_cut, mid, ni + 1 - i_cut, ni]
    jbnd = [1] + list(j_cuts) + [nj]
    kbnd = [1, kt, nk]
    njb = len(jbnd) - 1
    xyz, inp = [], []
    bid = {}
    for kb in range(2):
        for jb in range(njb):
            for ib in range(4):
                bid[(ib, jb, kb)] = len(xyz) + 1
                i0, i1 = ibnd[ib], ibnd[ib + 1]
                j0, j1 = jbnd[jb], jbnd[jb + 1]
                k0, k1 = kbnd[kb], kbnd[kb + 1]
                xyz.append(np.ascontiguousarray(X[:, k0 - 1:k1, j0 - 1:j1, i0 - 1:i1]))
                inp.append(InpBlock(i1 - i0 + 1, j1 - j0 + 1, k1 - k0 + 1))
    for kb in range(2):
        for jb in range(njb):
            for ib in range(4):
                b = bid[(ib, jb, kb)]
                B = inp[b - 1]
                nx, ny, nzb = B.nx, B.ny, B.nz
                # i faces
                if ib == 0:  # TE seam: i=1 of block ib0 <-> i=ni of block ib3
                    o = bid[(3, jb, kb)]
                    sA, sB = interface(b, ((1, 1), (1, ny), (1, nzb)), o, lambda i, j, k, n3=inp[o - 1].nx: (n3, j, k))
                    B.subs.append(sA)
                    inp[o - 1].subs.append(sB)
                if ib < 3:
                    nb = bid[(ib + 1, jb, kb)]
                    sA, sB = interface(b, ((nx, nx), (1, ny), (1, nzb)), nb, lambda i, j, k: (1, j, k))
                    B.subs.append(sA)
                    inp[nb - 1].subs.append(sB)
                # j faces
                if jb == 0:
                    if kb == 0:
                        B.subs.append(InpSub((1, nx, 1, 1, 1, nzb), BC_WALL))
                    elif ib < 2:  # sheet beyond the tip: block ib <-> block 3-ib with i reversed
                        ob = bid[(3 - ib, jb, kb)]
                        i0 = ibnd[ib]
                        o0 = ibnd[3 - ib]
                        sA, sB = interface(b, ((1, nx), (1, 1), (1, nzb)), ob,
                                           lambda i, j, k, i0=i0, o0=o0: ((ni + 1 - (i0 + i - 1)) - o0 + 1, 1, k))
                        B.subs.append(sA)
                        inp[ob - 1].subs.append(sB)
                if jb == njb - 1:
                    B.subs.append(InpSub((1, nx, ny, ny, 1, nzb), BC_FARFIELD))
                else:  # wall-normal cut: top face of this block <-> bottom face of the next
                    nb = bid[(ib, jb + 1, kb)]
                    sA, sB = interface(b, ((1, nx), (ny, ny), (1, nzb)), nb, lambda i, j, k: (i, 1, k))
                    B.subs.append(sA)
                    inp[nb - 1].subs.append(sB)
                # k faces
                if kb == 0:
                    B.subs.append(InpSub((1, nx, 1, ny, 1, 1), BC_SYMMETRY))
                    nb = bid[(ib, jb, 1)]
                    sA, sB = interface(b, ((1, nx), (1, ny), (nzb, nzb)), nb, lambda i, j, k: (i, j, 1))
                    B.subs.append(sA)
                    inp[nb - 1].subs.append(sB)
                else:
                    B.subs.append(InpSub((1, nx, 1, ny, nzb, nzb), BC_FARFIELD))
    return Case(name, xyz, inp, meta=dict(kind="wing", ni=ni, nj=nj, nk=nk, nk_wing=nk_wing, ref_s=None))


def wing_ref_area(semi_span=1.5, taper=0.56):
    return semi_span * (1.0 + taper) / 2.0
