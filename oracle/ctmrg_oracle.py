"""CPU oracle of the double-layer SequentialCTMRG (the simple update is in
simple_update_oracle.py) -- TEST INFRASTRUCTURE ONLY.

A numpy restatement of frostspin/ctmrg (ctm_contract.py, ctm_renormalize.py,
ctm_environment.py, sequential_ctmrg.py, rdm.py) on the oracle tensors of
frostspin_oracle.py (U(1)/Z2) or su2_oracle.py (SU(2)), every sector SVD on the
dense path
(robust_svd, misc_tools/svd_tools.py:116-151).  Only tests/ and bench.py's
CPU-baseline leg use it, as the checker and the timed CPU baseline.
"""

import numpy as np

from . import frostspin_oracle as fo
from . import su2_oracle as so


def module_of(o):
    """The oracle module implementing the symmetry of an oracle tensor."""
    return so if isinstance(o, so.OTensor) else fo


class OT:
    """Method wrapper so the contraction recipes read like the reference."""

    __slots__ = ("o", "m")

    def __init__(self, o, m=None):
        self.o = o
        self.m = module_of(o) if m is None else m

    def permute(self, r, c):
        return OT(self.m.permute(self.o, r, c), self.m)

    def __matmul__(self, other):
        return OT(self.m.matmul(self.o, other.o), self.m)

    def transpose(self):
        return OT(self.m.transpose(self.o), self.m)

    def dagger(self):
        return OT(self.m.dagger(self.o), self.m)

    def norm(self):
        return self.m.norm(self.o)

    def normalized(self):
        return OT(self.m.scale(self.o, 1.0 / self.m.norm(self.o)), self.m)

    def full_contract(self, other):
        return self.m.full_contract(self.o, other.o)

    def trace(self):
        return self.m.trace(self.o)

    @property
    def shape(self):
        return self.o.shape


# ------------------------------------------------------ contractions (ctm_contract.py)


def enlarged_corner(C, Tx, Ty, A):
    ul = Tx @ C
    ul = ul @ Ty
    ul = ul.permute((0, 3), (1, 4, 2, 5))
    ul = A @ ul
    ul = ul.permute((0, 1, 4, 5), (2, 3, 6, 7))
    ul = A.permute((0, 1, 4, 5), (2, 3)).dagger() @ ul
    return ul.permute((2, 0, 4), (3, 1, 5))


def corner_ul(C1, T1, T4, A):
    return enlarged_corner(C1, T1.permute((1, 2, 0), (3,)), T4.permute((0,), (1, 2, 3)),
                           A.permute((0, 1, 3, 4), (2, 5)))


def corner_ur(T1, C2, A, T2):
    return enlarged_corner(C2, T2.permute((2, 3, 1), (0,)), T1.permute((0,), (1, 2, 3)),
                           A.permute((0, 1, 4, 5), (3, 2)))


def corner_dr(A, T2, T3, C3):
    return enlarged_corner(C3.transpose(), T3.permute((0, 1, 3), (2,)),
                           T2.permute((1,), (2, 3, 0)), A.permute((0, 1, 5, 2), (4, 3)))


def corner_dl(T4, A, C4, T3):
    return enlarged_corner(C4, T4.permute((1, 2, 0), (3,)), T3.permute((3,), (0, 1, 2)),
                           A.permute((0, 1, 2, 3), (5, 4)))


# ------------------------------------------------ projectors (ctm_renormalize.py)


def projectors(c1, c2, c3, c4, chi, rtol, degen_ratio):
    """Dense-SVD construct_projectors (ctm_renormalize.py:6-136)."""
    m = c1.m
    o1, o2, o3, o4 = c1.o, c2.o, c3.o, c4.o
    shared = np.intersect1d(np.intersect1d(o1.block_irreps, o2.block_irreps),
                            np.intersect1d(o3.block_irreps, o4.block_irreps))
    idx = [np.searchsorted(o.block_irreps, shared) for o in (o1, o2, o3, o4)]
    rs, rts, us, ss, vs = [], [], [], [], []
    for k in range(shared.size):
        r = o1.blocks[idx[0][k]] @ o2.blocks[idx[1][k]]
        rt = o3.blocks[idx[2][k]] @ o4.blocks[idx[3][k]]
        u, s, v = np.linalg.svd(r @ rt, full_matrices=False)
        rs.append(r)
        rts.append(rt)
        us.append(u)
        ss.append(s)
        vs.append(v)
    cuts = fo.find_block_cuts(ss, chi, dims=m.irrep_dims(shared), rtol=rtol,
                              degen_ratio=degen_ratio)
    keep = np.flatnonzero(cuts)
    p_blocks, pt_blocks = [], []
    for k in keep:
        c = cuts[k]
        s12 = 1.0 / np.sqrt(ss[k][:c])
        p_blocks.append(s12[:, None] * us[k][:, :c].T @ rs[k])
        pt_blocks.append(rts[k] @ vs[k][:c].T * s12)
    irr = o2.block_irreps[idx[1][keep]]
    mid = m.init_representation(cuts[keep], irr)
    n2 = o2.nrr
    sp = np.zeros(n2 + 1, dtype=bool)
    sp[1:] = o2.signature[n2:]
    spt = np.ones(n2 + 1, dtype=bool)
    spt[:-1] = ~o2.signature[n2:]
    P = OT(m.transpose(m.OTensor((mid,), o2.col_reps, p_blocks, irr, sp)), m)
    Pt = OT(m.OTensor(o2.col_reps, (mid,), pt_blocks, irr, spt), m)
    return P, Pt


def ren_T(Pt, T, A, P):
    nT = T @ P.permute((2,), (0, 1, 3))
    nT = nT.permute((0, 3), (1, 4, 2, 5))
    nT = A @ nT
    nT = nT.permute((0, 1, 4, 5), (2, 3, 6, 7))
    nT = A.permute((0, 1, 4, 5), (2, 3)).dagger() @ nT
    nT = nT.permute((3, 1, 4), (2, 0, 5))
    return (Pt.transpose() @ nT).normalized()


def ren_corner(C, T, X):
    return ((T @ C).permute((0,), (1, 2, 3)) @ X).normalized()


# ------------------------------------------------------------ environment & driver


def dummy_env(A):
    """ctm_environment.py:6-34 on oracle tensors."""
    m = A.m
    z = m.singlet()
    one = (z,)
    s = A.o.signature
    r = A.o.col_reps
    sh = A.o.shape

    def fa(arr, rr, cr, sig=None):
        return OT(m.from_array(arr, rr, cr, sig), m)

    return {
        "C1": fa(np.eye(1), one, one),
        "C2": fa(np.eye(1), one, one),
        "C3": fa(np.eye(1), one, one, [True, False]),
        "C4": fa(np.eye(1), one, one),
        "T1": fa(np.eye(sh[4])[None, :, :, None], one, (r[2], r[2], z),
                 np.array([False, s[4], ~s[4], True])),
        "T2": fa(np.eye(sh[5])[None, None, :, :], one, (z, r[3], r[3]),
                 np.array([True, False, s[5], ~s[5]])),
        "T3": fa(np.eye(sh[2])[:, :, None, None], (r[0], r[0], z), one,
                 np.array([s[2], ~s[2], True, False])),
        "T4": fa(np.eye(sh[3])[None, :, :, None], one, (r[1], r[1], z),
                 np.array([False, s[3], ~s[3], True])),
    }


class SequentialCTMRG:
    """sequential_ctmrg.py:19-211 with the checkerboard AB/BA cell only."""

    def __init__(self, A, B, chi, *, cutoff=1e-11, degen_ratio=0.9999):
        self.As = [OT(A), OT(B)]
        self.chi = chi
        self.rtol = cutoff
        self.degen = degen_ratio
        envs = [dummy_env(a) for a in self.As]
        self.t = {k: [e[k] for e in envs] for k in envs[0]}
        self.coords = [(0, 0), (1, 0)]
        self.corners = {k: [None, None] for k in ("ul", "ur", "dl", "dr")}

    @staticmethod
    def idx(x, y):
        return (x + y) % 2

    def g(self, name, x, y):
        return self.t[name][self.idx(x, y)]

    def A(self, x, y):
        return self.As[self.idx(x, y)]

    def corner(self, kind, x, y, free=False):
        i = self.idx(x, y)
        c = self.corners[kind][i]
        if c is None:
            g, A = self.g, self.A
            if kind == "ul":
                c = corner_ul(g("C1", x, y), g("T1", x + 1, y), g("T4", x, y + 1), A(x + 1, y + 1))
            elif kind == "ur":
                c = corner_ur(g("T1", x + 2, y), g("C2", x + 3, y), A(x + 2, y + 1),
                              g("T2", x + 3, y + 1))
            elif kind == "dl":
                c = corner_dl(g("T4", x, y + 2), A(x + 1, y + 2), g("C4", x, y + 3),
                              g("T3", x + 1, y + 3))
            else:
                c = corner_dr(A(x + 2, y + 2), g("T2", x + 3, y + 2), g("T3", x + 2, y + 3),
                              g("C3", x + 3, y + 3))
            if not free:
                self.corners[kind][i] = c
        elif free:
            self.corners[kind][i] = None
        return c

    def _proj(self, c1, c2, c3, c4):
        return projectors(c1, c2, c3, c4, self.chi, self.rtol, self.degen)

    def iterate(self):
        g, A = self.g, self.A
        # up
        pr = {}
        for x, y in self.coords:
            pr[self.idx(x + 2, y)] = self._proj(self.corner("dr", x, y), self.corner("ur", x, y, True),
                                                self.corner("ul", x, y, True), self.corner("dl", x, y))
        new = [None, None]
        for x, y in self.coords:
            P, Pt = pr[self.idx(x + 1, y)][0], pr[self.idx(x, y)][1]
            nC1 = ren_corner(g("C1", x, y).transpose(), g("T4", x, y + 1).permute((3, 1, 2), (0,)),
                             P).transpose()
            nT1 = ren_T(Pt, g("T1", x, y).permute((1, 2, 3), (0,)),
                        A(x, y + 1).permute((0, 1, 4, 5), (2, 3)), P).permute((3,), (1, 2, 0))
            nC2 = ren_corner(g("C2", x, y), g("T2", x, y + 1).permute((1, 2, 3), (0,)), Pt)
            new[self.idx(x, y + 1)] = (nC1, nT1, nC2)
        self._commit(("C1", "T1", "C2"), new)
        # right
        pr = {}
        for x, y in self.coords:
            pr[self.idx(x + 3, y + 2)] = self._proj(
                self.corner("dl", x, y), self.corner("dr", x, y, True),
                self.corner("ur", x, y, True), self.corner("ul", x, y))
        new = [None, None]
        for x, y in self.coords:
            P, Pt = pr[self.idx(x, y + 1)][0], pr[self.idx(x, y)][1]
            nC2 = ren_corner(g("C2", x, y).transpose(), g("T1", x - 1, y).permute((3, 1, 2), (0,)),
                             P).transpose()
            nT2 = ren_T(Pt, g("T2", x, y).permute((2, 3, 0), (1,)),
                        A(x - 1, y).permute((0, 1, 5, 2), (3, 4)), P).permute((0,), (3, 1, 2))
            nC3 = ren_corner(g("C3", x, y).transpose(), g("T3", x - 1, y).permute((3, 0, 1), (2,)),
                             Pt).transpose()
            new[self.idx(x - 1, y)] = (nC2, nT2, nC3)
        self._commit(("C2", "T2", "C3"), new)
        # down
        pr = {}
        for x, y in self.coords:
            pr[self.idx(x + 1, y + 3)] = self._proj(
                self.corner("ul", x, y), self.corner("dl", x, y, True),
                self.corner("dr", x, y, True), self.corner("ur", x, y))
        new = [None, None]
        for x, y in self.coords:
            P, Pt = pr[self.idx(x - 1, y)][0], pr[self.idx(x, y)][1]
            nC3 = ren_corner(g("C3", x, y), g("T2", x, y - 1).permute((0, 2, 3), (1,)), P)
            nT3 = ren_T(Pt, g("T3", x, y).permute((0, 1, 2), (3,)),
                        A(x, y - 1).permute((0, 1, 2, 3), (4, 5)), P).permute((1, 2, 0), (3,))
            nC4 = ren_corner(g("C4", x, y), g("T4", x, y - 1).permute((0, 1, 2), (3,)), Pt)
            new[self.idx(x, y - 1)] = (nC3, nT3, nC4)
        self._commit(("C3", "T3", "C4"), new)
        # left
        pr = {}
        for x, y in self.coords:
            pr[self.idx(x, y + 1)] = self._proj(
                self.corner("ur", x, y), self.corner("ul", x, y, True),
                self.corner("dl", x, y, True), self.corner("dr", x, y))
        new = [None, None]
        for x, y in self.coords:
            P, Pt = pr[self.idx(x, y - 1)][0], pr[self.idx(x, y)][1]
            nC4 = ren_corner(g("C4", x, y).transpose(), g("T3", x + 1, y).permute((2, 0, 1), (3,)),
                             P).transpose()
            nT4 = ren_T(Pt, g("T4", x, y).permute((1, 2, 3), (0,)),
                        A(x + 1, y).permute((0, 1, 3, 4), (5, 2)), P).permute((3,), (1, 2, 0))
            nC1 = ren_corner(g("C1", x, y), g("T1", x + 1, y).permute((0, 1, 2), (3,)), Pt)
            new[self.idx(x + 1, y)] = (nC4, nT4, nC1)
        self._commit(("C4", "T4", "C1"), new)

    def _commit(self, names, new):
        for k, name in enumerate(names):
            self.t[name] = [n[k] for n in new]


# ---------------------------------------------------------------- rdm (rdm.py)


def _open_corner(C1, T1, T4, A):
    ul = T1.permute((1, 2, 0), (3,)) @ C1
    ul = ul @ T4.permute((0,), (1, 2, 3))
    ul = ul.permute((0, 3), (1, 4, 2, 5))
    ul = A.permute((1, 0, 3, 4), (2, 5)) @ ul
    ul = ul.permute((0, 4, 5), (1, 2, 3, 6, 7))
    ul = A.permute((1, 2, 5), (0, 3, 4)).dagger() @ ul
    return ul.permute((3, 0, 4, 1, 6), (5, 2, 7))


def _open_corner_mirror(T1, C2, A, T2):
    ur = C2 @ T1.permute((0,), (1, 2, 3))
    ur = ur.transpose() @ T2.permute((0,), (2, 3, 1))
    ur = ur.permute((0, 3), (1, 4, 2, 5))
    ur = A.permute((1, 0, 4, 5), (2, 3)) @ ur
    ur = ur.permute((0, 4, 5), (1, 2, 3, 6, 7))
    return A.permute((1, 2, 3), (0, 4, 5)).dagger() @ ur


def rdm_1x2(C1, T1l, T1r, C2, T4, Al, Ar, T2, C4, T3l, T3r, C3):
    """rdm.py:90-137, normalised by the trace; returns a dense array."""
    left = T4.permute((0, 1, 2), (3,)) @ C4
    left = _open_corner(C1, T1l, left, Al)
    left = left @ T3l.permute((0, 1, 3), (2,))
    left = left.permute((0, 1), (2, 3, 4, 5))
    right = T2.permute((0, 2, 3), (1,)) @ C3
    right = right.permute((0, 3), (1, 2))
    right = _open_corner_mirror(T1r, C2, Ar, right)
    right = right.permute((3, 0, 5, 2, 6), (4, 1, 7))
    right = right @ T3r.permute((0, 1, 2), (3,))
    right = right.permute((2, 3, 4, 5), (0, 1))
    r = (left @ right).permute((1, 3), (0, 2))
    return r.m.toarray(r.o) / r.trace()


def ctm_rdm1x2(ctm, x, y):
    g, A = ctm.g, ctm.A
    return rdm_1x2(g("C1", x, y), g("T1", x + 1, y), g("T1", x + 2, y), g("C2", x + 3, y),
                   g("T4", x, y + 1), A(x + 1, y + 1), A(x + 2, y + 1), g("T2", x + 3, y + 1),
                   g("C4", x, y + 2), g("T3", x + 1, y + 2), g("T3", x + 2, y + 2),
                   g("C3", x + 3, y + 2))


def ctm_rdm2x1(ctm, x, y):
    g, A = ctm.g, ctm.A
    return rdm_1x2(
        g("C2", x + 2, y), g("T2", x + 2, y + 1).permute((1, 2, 3), (0,)),
        g("T2", x + 2, y + 2).permute((1,), (2, 3, 0)), g("C3", x + 2, y + 3).transpose(),
        g("T1", x + 1, y), A(x + 1, y + 1).permute((0, 1), (3, 4, 5, 2)),
        A(x + 1, y + 2).permute((0, 1), (3, 4, 5, 2)),
        g("T3", x + 1, y + 3).permute((2, 3, 0), (1,)), g("C1", x, y),
        g("T4", x, y + 1).permute((1, 2, 3), (0,)), g("T4", x, y + 2).permute((1, 2, 3), (0,)),
        g("C4", x, y + 3).transpose(),
    )


def ren_quadrant(P, quadrant, Pt):
    """ctm_renormalize.py:219-225."""
    return (P.transpose() @ quadrant @ Pt).normalized()


class SimultaneousCTMRG(SequentialCTMRG):
    """simultaneous_ctmrg.py:14-132 with the checkerboard AB/BA cell: every
    enlarged corner, then the projectors of the four directions, then every
    corner (from the enlarged corners) and edge of every site at once."""

    def iterate(self):
        g, A = self.g, self.A
        idx = self.idx
        for x, y in self.coords:
            for kind in ("dr", "ur", "ul", "dl"):
                self.corner(kind, x, y)
        pr = {d: {} for d in ("up", "right", "down", "left")}
        for x, y in self.coords:
            dl, dr, ur, ul = (self.corner(k, x, y) for k in ("dl", "dr", "ur", "ul"))
            pr["up"][idx(x + 2, y)] = self._proj(dr, ur, ul, dl)
            pr["right"][idx(x + 3, y + 2)] = self._proj(dl, dr, ur, ul)
            pr["down"][idx(x + 1, y + 3)] = self._proj(ul, dl, dr, ur)
            pr["left"][idx(x, y + 1)] = self._proj(ur, ul, dl, dr)

        def P(d, x, y):
            return pr[d][idx(x, y)][0]

        def Pt(d, x, y):
            return pr[d][idx(x, y)][1]

        names = ("C1", "C2", "C3", "C4", "T1", "T2", "T3", "T4")
        new = {k: [None, None] for k in names}
        for x, y in self.coords:
            i = idx(x, y)
            a = A(x, y)
            new["C1"][i] = ren_quadrant(P("up", x + 1, y - 1), self.corner("ul", x - 1, y - 1),
                                        Pt("left", x - 1, y))
            new["T1"][i] = ren_T(Pt("up", x, y - 1), g("T1", x, y - 1).permute((1, 2, 3), (0,)),
                                 a.permute((0, 1, 4, 5), (2, 3)),
                                 P("up", x + 1, y - 1)).permute((3,), (1, 2, 0))
            new["C2"][i] = ren_quadrant(P("right", x + 1, y + 1), self.corner("ur", x - 2, y - 1),
                                        Pt("up", x, y - 1))
            new["T2"][i] = ren_T(Pt("right", x + 1, y), g("T2", x + 1, y).permute((2, 3, 0), (1,)),
                                 a.permute((0, 1, 5, 2), (3, 4)),
                                 P("right", x + 1, y + 1)).permute((0,), (3, 1, 2))
            new["C3"][i] = ren_quadrant(P("down", x - 1, y + 1), self.corner("dr", x - 2, y - 2),
                                        Pt("right", x + 1, y)).transpose()
            new["T3"][i] = ren_T(Pt("down", x, y + 1), g("T3", x, y + 1).permute((0, 1, 2), (3,)),
                                 a.permute((0, 1, 2, 3), (4, 5)),
                                 P("down", x - 1, y + 1)).permute((1, 2, 0), (3,))
            new["C4"][i] = ren_quadrant(P("left", x - 1, y - 1), self.corner("dl", x - 1, y - 2),
                                        Pt("down", x, y + 1))
            new["T4"][i] = ren_T(Pt("left", x - 1, y), g("T4", x - 1, y).permute((1, 2, 3), (0,)),
                                 a.permute((0, 1, 3, 4), (5, 2)),
                                 P("left", x - 1, y - 1)).permute((3,), (1, 2, 0))
        self.t = new
        self.corners = {k: [None, None] for k in ("ul", "ur", "dl", "dr")}
