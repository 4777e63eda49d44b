"""Simultaneous CTMRG on device tensors (frostspin/ctmrg/simultaneous_ctmrg.py:14-132).

One iteration builds every enlarged corner of every unique site, then the
projectors of the four directions from them, then renormalises every corner
(from the enlarged corners, with two projectors) and every edge of every site
at once; the new environment replaces the old one.  Parameters, observables
and checkpoint I/O are those of SequentialCTMRG.
"""

from .ctm_environment import CTMEnvironment
from .ctm_renormalize import (
    renormalize_quadrant,
    renormalize_T1,
    renormalize_T2,
    renormalize_T3,
    renormalize_T4,
)
from .sequential_ctmrg import SequentialCTMRG

_NAMES = ("C1", "C2", "C3", "C4", "T1", "T2", "T3", "T4")


class SimultaneousCTMRG(SequentialCTMRG):
    def __repr__(self):
        return (f"{self.symmetry()} symmetric SimultaneousCTMRG with Dmax = {self.Dmax}"
                f" and chi_target = {self.chi_target}")

    def iterate(self):
        """simultaneous_ctmrg.py:19-26."""
        self.construct_enlarged_corners()
        self.compute_projectors()
        self.renormalize_tensors()

    def construct_enlarged_corners(self):
        """simultaneous_ctmrg.py:28-36."""
        for x, y in self.site_coords:
            self.construct_enlarged_dr(x, y)
            self.construct_enlarged_ur(x, y)
            self.construct_enlarged_ul(x, y)
            self.construct_enlarged_dl(x, y)

    def compute_projectors(self):
        """simultaneous_ctmrg.py:38-77: for every site, the up, right, down and
        left projectors from its four enlarged corners."""
        e = self._env
        for x, y in self.site_coords:
            dl = self.construct_enlarged_dl(x, y)
            dr = self.construct_enlarged_dr(x, y)
            ur = self.construct_enlarged_ur(x, y)
            ul = self.construct_enlarged_ul(x, y)
            P, Pt = self._projectors(dr, ur, ul, dl, e.get_C2(x + 2, y + 1))
            e.store_projectors("up", x + 2, y, P, Pt)
            P, Pt = self._projectors(dl, dr, ur, ul, e.get_C3(x + 2, y + 2).transpose())
            e.store_projectors("right", x + 3, y + 2, P, Pt)
            P, Pt = self._projectors(ul, dl, dr, ur, e.get_C4(x + 1, y + 2))
            e.store_projectors("down", x + 1, y + 3, P, Pt)
            P, Pt = self._projectors(ur, ul, dl, dr, e.get_C1(x + 1, y + 1))
            e.store_projectors("left", x, y + 1, P, Pt)

    def renormalize_tensors(self):
        """simultaneous_ctmrg.py:79-132."""
        e = self._env
        new = {k: [None] * self.n_sites for k in _NAMES}
        for i, (x, y) in enumerate(self.site_coords):
            A = e.get_A(x, y)
            new["C1"][i] = renormalize_quadrant(e.get_P("up", x + 1, y - 1),
                                                self.construct_enlarged_ul(x - 1, y - 1),
                                                e.get_Pt("left", x - 1, y))
            new["T1"][i] = renormalize_T1(e.get_Pt("up", x, y - 1), e.get_T1(x, y - 1), A,
                                          e.get_P("up", x + 1, y - 1))
            new["C2"][i] = renormalize_quadrant(e.get_P("right", x + 1, y + 1),
                                                self.construct_enlarged_ur(x - 2, y - 1),
                                                e.get_Pt("up", x, y - 1))
            new["T2"][i] = renormalize_T2(e.get_Pt("right", x + 1, y), e.get_T2(x + 1, y), A,
                                          e.get_P("right", x + 1, y + 1))
            new["C3"][i] = renormalize_quadrant(e.get_P("down", x - 1, y + 1),
                                                self.construct_enlarged_dr(x - 2, y - 2),
                                                e.get_Pt("right", x + 1, y)).transpose()
            new["T3"][i] = renormalize_T3(e.get_Pt("down", x, y + 1), e.get_T3(x, y + 1), A,
                                          e.get_P("down", x - 1, y + 1))
            new["C4"][i] = renormalize_quadrant(e.get_P("left", x - 1, y - 1),
                                                self.construct_enlarged_dl(x - 1, y - 2),
                                                e.get_Pt("down", x, y + 1))
            new["T4"][i] = renormalize_T4(e.get_Pt("left", x - 1, y), e.get_T4(x - 1, y), A,
                                          e.get_P("left", x - 1, y - 1))
        self._env = CTMEnvironment(e.cell, e.elementary_tensors, new)
