"""Symmetrized CTMRG on device tensors (frostspin/ctmrg/symmetrized_ctmrg.py:19-274).

For the AB/BA cell with B the rotated dagger of A (B = A.dagger().permute((4, 5),
(2, 3, 0, 1))), the environment of B is a leg permutation of the environment
of A.  Only the enlarged corners of site (0, 0) are contracted; each is stored
with its partner at (1, 0), a leg permutation.  The four projector pairs of an
iteration come from those corners, and each pair also serves, permuted, in
the opposite direction.  Only A's eight environment tensors are renormalised;
B's are their permutations.  Reduced density matrices reuse the same symmetry
(rdm_symmetrized_1x2 / 2x1).
"""

from . import rdm
from .ctm_contract import contract_dl, contract_dr, contract_ul, contract_ur
from .ctm_environment import CTMEnvironment
from .ctm_renormalize import (
    renormalize_quadrant,
    renormalize_T1,
    renormalize_T2,
    renormalize_T3,
    renormalize_T4,
)
from .sequential_ctmrg import SequentialCTMRG

_PARTNER = {"ul": "dr", "dr": "ul", "ur": "dl", "dl": "ur"}


class SymmetrizedCTMRG(SequentialCTMRG):
    def __repr__(self):
        return (f"{self.symmetry()} symmetric SymmetrizedCTMRG with Dmax = {self.Dmax}"
                f" and chi_target = {self.chi_target}")

    # ------------------------------------------------------ enlarged corners
    def _enlarged(self, kind, x, y, free_memory):
        """symmetrized_ctmrg.py:20-115: the corner, cached together with its
        partner at (x + 1, y), the same tensor with legs (1, 0, 2 | 4, 3, 5)."""
        e = self._env
        partner = _PARTNER[kind]
        c = e.get_corner(kind, x, y)
        if c is None:
            if kind == "ul":
                c = contract_ul(e.get_C1(x, y), e.get_T1(x + 1, y), e.get_T4(x, y + 1),
                                e.get_A(x + 1, y + 1))
            elif kind == "ur":
                c = contract_ur(e.get_T1(x + 2, y), e.get_C2(x + 3, y), e.get_A(x + 2, y + 1),
                                e.get_T2(x + 3, y + 1))
            elif kind == "dl":
                c = contract_dl(e.get_T4(x, y + 2), e.get_A(x + 1, y + 2), e.get_C4(x, y + 3),
                                e.get_T3(x + 1, y + 3))
            else:
                c = contract_dr(e.get_A(x + 2, y + 2), e.get_T2(x + 3, y + 2),
                                e.get_T3(x + 2, y + 3), e.get_C3(x + 3, y + 3))
            if not free_memory:
                e.set_corner(kind, x, y, c)
                e.set_corner(partner, x + 1, y, c.permute((1, 0, 2), (4, 3, 5)))
        elif free_memory:
            e.set_corner(kind, x, y, None)
            e.set_corner(partner, x + 1, y, None)
        return c

    # ------------------------------------------------------------ iteration
    def iterate(self):
        """symmetrized_ctmrg.py:121-127."""
        self.compute_projectors()
        self.renormalize_tensors()

    def compute_projectors(self):
        """symmetrized_ctmrg.py:129-171."""
        e = self._env
        dl = self.construct_enlarged_dl(0, 0)
        dr = self.construct_enlarged_dr(0, 0)
        ur = self.construct_enlarged_ur(0, 0)
        ul = self.construct_enlarged_ul(0, 0)

        def store(direction, xy, mirror, mxy, P, Pt):
            e.store_projectors(direction, *xy, P, Pt)
            e.store_projectors(mirror, *mxy, P.permute((1, 0, 2), (3,)),
                               Pt.permute((1, 0, 2), (3,)))

        store("up", (0, 0), "down", (0, 1), *self._projectors(dr, ur, ul, dl, e.get_C2(0, 1)))
        store("right", (1, 0), "left", (0, 0),
              *self._projectors(dl, dr, ur, ul, e.get_C3(0, 0).transpose()))
        store("down", (1, 1), "up", (0, 1), *self._projectors(ul, dl, dr, ur, e.get_C4(1, 0)))
        store("left", (0, 1), "right", (0, 0), *self._projectors(ur, ul, dl, dr, e.get_C1(1, 1)))

    def renormalize_tensors(self):
        """symmetrized_ctmrg.py:173-234."""
        e = self._env
        A = e.get_A(0, 0)
        nC1 = renormalize_quadrant(e.get_P("up", 1, 1), self.construct_enlarged_ul(1, 1),
                                   e.get_Pt("left", 1, 0))
        nT1 = renormalize_T1(e.get_Pt("up", 0, 1), e.get_T1(0, 1), A, e.get_P("up", 1, 1))
        nC2 = renormalize_quadrant(e.get_P("right", 1, 1), self.construct_enlarged_ur(0, 1),
                                   e.get_Pt("up", 0, 1))
        nT2 = renormalize_T2(e.get_Pt("right", 1, 0), e.get_T2(1, 0), A,
                             e.get_P("right", 1, 1))
        nC3 = renormalize_quadrant(e.get_P("down", 1, 1), self.construct_enlarged_dr(0, 0),
                                   e.get_Pt("right", 1, 0)).transpose()
        nT3 = renormalize_T3(e.get_Pt("down", 0, 1), e.get_T3(0, 1), A, e.get_P("down", 1, 1))
        nC4 = renormalize_quadrant(e.get_P("left", 1, 1), self.construct_enlarged_dl(1, 0),
                                   e.get_Pt("down", 0, 1))
        nT4 = renormalize_T4(e.get_Pt("left", 1, 0), e.get_T4(1, 0), A, e.get_P("left", 1, 1))
        envs = {
            "C1": [nC1, nC3.transpose()],
            "C2": [nC2, nC4],
            "C3": [nC3, nC1.transpose()],
            "C4": [nC4, nC2],
            "T1": [nT1, nT3.permute((3,), (1, 0, 2))],
            "T2": [nT2, nT4.permute((3,), (0, 2, 1))],
            "T3": [nT3, nT1.permute((2, 1, 3), (0,))],
            "T4": [nT4, nT2.permute((1,), (3, 2, 0))],
        }
        self._env = CTMEnvironment(e.cell, [A, e.get_A(0, 1)], envs)

    # --------------------------------------------------------- observables
    def compute_rdm1x2(self, x, y):
        """symmetrized_ctmrg.py:236-246."""
        e = self._env
        return rdm.rdm_symmetrized_1x2(e.get_C1(x, y), e.get_T1(x + 1, y), e.get_T4(x, y + 1),
                                       e.get_A(x + 1, y + 1), e.get_C4(x, y + 2),
                                       e.get_T3(x + 1, y + 2))

    def compute_rdm2x1(self, x, y):
        """symmetrized_ctmrg.py:248-258."""
        e = self._env
        return rdm.rdm_symmetrized_2x1(e.get_C1(x, y), e.get_T1(x + 1, y), e.get_C2(x + 2, y),
                                       e.get_T4(x, y + 1), e.get_A(x + 1, y + 1),
                                       e.get_T2(x + 2, y + 1))

    def compute_rdm_2nd_neighbor_cell(self, *, free_memory=True):
        """symmetrized_ctmrg.py:260-274: the diagonals of site (0, 0); those of
        the other site are their transposes."""
        if free_memory:
            self._env.reset_constructed_corners()
        dr = self.compute_rdm_diag_dr(0, 0, free_memory=free_memory)
        ur = self.compute_rdm_diag_ur(0, 0, free_memory=free_memory)
        return [dr, dr.transpose()], [ur, ur.transpose()]
