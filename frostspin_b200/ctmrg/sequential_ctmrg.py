"""Sequential CTMRG on device tensors.

Same algorithm and parameters as frostspin/ctmrg/abstract_ctmrg.py:17-668 and
sequential_ctmrg.py:19-211: one iteration is an up, right, down and left move;
each move builds the projectors of every unique site from four enlarged corners
(cached and reused across moves until the tensors they depend on change), then
renormalises the corner-edge-corner triple of the absorbed side.
"""

import numpy as np

from . import observables, rdm
from .ctm_contract import (
    contract_C1234,
    contract_dl,
    contract_dr,
    contract_norm,
    contract_T1T3,
    contract_T2T4,
    contract_ul,
    contract_ur,
)
from .ctm_environment import CTMEnvironment
from .ctm_renormalize import (
    construct_projectors,
    renormalize_C1_left,
    renormalize_C1_up,
    renormalize_C2_right,
    renormalize_C2_up,
    renormalize_C3_down,
    renormalize_C3_right,
    renormalize_C4_down,
    renormalize_C4_left,
    renormalize_T1,
    renormalize_T2,
    renormalize_T3,
    renormalize_T4,
)


class SequentialCTMRG:
    def __init__(self, env, chi_target, *, verbosity=0, **ctm_params):
        self.verbosity = verbosity
        self._env = env
        self.chi_target = int(chi_target)
        self.block_chi_ratio = float(ctm_params.get("block_chi_ratio", 1.1))
        self.ncv_ratio = float(ctm_params.get("ncv_ratio", 2.0))
        self.cutoff = float(ctm_params.get("cutoff", 1e-11))
        self.degen_ratio = float(ctm_params.get("degen_ratio", 0.9999))
        if self.chi_target < 2:
            raise ValueError("chi must be larger than 2")
        if self.block_chi_ratio < 1.0:
            raise ValueError("block_chi_ratio must be larger than 1.0")
        if self.ncv_ratio < 2.0:
            raise ValueError("ncv_ratio must be larger than 2.0")
        if not (0.0 <= self.cutoff < 1.0):
            raise ValueError("cutoff must me obey 0.0 <= self.cutoff < 1.0")
        if not (0.0 < self.degen_ratio <= 1.0):
            raise ValueError("degen_ratio must obey 0.0 <= self.degen_ratio <= 1.0")

    @classmethod
    def from_elementary_tensors(cls, tiling, tensors, chi_target, *, verbosity=0, **ctm_params):
        env = CTMEnvironment.from_elementary_tensors(tiling, tensors)
        return cls(env, chi_target, verbosity=verbosity, **ctm_params)

    @classmethod
    def load_from_file(cls, filename, *, verbosity=0):
        with np.load(filename) as fin:
            chi_target = int(fin["_CTM_chi_target"])
            params = {k: float(fin[f"_CTM_{k}"]) for k in
                      ("block_chi_ratio", "ncv_ratio", "cutoff", "degen_ratio")}
        return cls(CTMEnvironment.load_from_file(filename), chi_target, verbosity=verbosity,
                   **params)

    def save_to_file(self, filename, **additional_data):
        data = {
            "_CTM_chi_target": self.chi_target,
            "_CTM_block_chi_ratio": self.block_chi_ratio,
            "_CTM_ncv_ratio": self.ncv_ratio,
            "_CTM_cutoff": self.cutoff,
            "_CTM_degen_ratio": self.degen_ratio,
        }
        data |= self._env.get_data_dic()
        np.savez_compressed(filename, **data, **additional_data)

    def copy(self):
        """Independent copy (environment tensors copied, parameters shared)."""
        return type(self)(self._env.copy(), self.chi_target, verbosity=self.verbosity,
                          block_chi_ratio=self.block_chi_ratio, ncv_ratio=self.ncv_ratio,
                          cutoff=self.cutoff, degen_ratio=self.degen_ratio)

    def set_tensors(self, tensors):
        """abstract_ctmrg.py:158-166."""
        self._env.set_tensors(tensors)

    @property
    def environment(self):
        return self._env

    # -------------------------------------------------------------- properties
    @property
    def Lx(self):
        return self._env.Lx

    @property
    def Ly(self):
        return self._env.Ly

    @property
    def cell(self):
        return self._env.cell

    @property
    def chi_values(self):
        return self._env.chi_values

    @property
    def Dmax(self):
        return self._env.Dmax

    @property
    def Dmin(self):
        return self._env.Dmin

    @property
    def n_sites(self):
        return self._env.n_sites

    @property
    def site_coords(self):
        return self._env.site_coords

    @property
    def elementary_tensors(self):
        return self._env.elementary_tensors

    @property
    def tiling(self):
        return "\n".join("".join(s) for s in self.cell)

    def symmetry(self):
        return self._env.symmetry()

    def __repr__(self):
        return (f"{self.symmetry()} symmetric SequentialCTMRG with Dmax = {self.Dmax}"
                f" and chi_target = {self.chi_target}")

    # --------------------------------------------------------- enlarged corners
    def _enlarged(self, kind, x, y, free_memory):
        e = self._env
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
        elif free_memory:
            e.set_corner(kind, x, y, None)
        return c

    def construct_enlarged_ul(self, x, y, *, free_memory=False):
        return self._enlarged("ul", x, y, free_memory)

    def construct_enlarged_ur(self, x, y, *, free_memory=False):
        return self._enlarged("ur", x, y, free_memory)

    def construct_enlarged_dl(self, x, y, *, free_memory=False):
        return self._enlarged("dl", x, y, free_memory)

    def construct_enlarged_dr(self, x, y, *, free_memory=False):
        return self._enlarged("dr", x, y, free_memory)

    def _projectors(self, c1, c2, c3, c4, last):
        return construct_projectors(
            c1, c2, c3, c4, self.chi_target, last,
            block_chi_ratio=self.block_chi_ratio, ncv_ratio=self.ncv_ratio,
            rtol=self.cutoff, degen_ratio=self.degen_ratio,
        )

    # -------------------------------------------------------------------- moves
    def iterate(self):
        self.up_move()
        self.right_move()
        self.down_move()
        self.left_move()

    def up_move(self):
        e = self._env
        for x, y in self.site_coords:
            P, Pt = self._projectors(
                self.construct_enlarged_dr(x, y),
                self.construct_enlarged_ur(x, y, free_memory=True),
                self.construct_enlarged_ul(x, y, free_memory=True),
                self.construct_enlarged_dl(x, y),
                e.get_C2(x + 2, y + 1),
            )
            e.store_projectors("up", x + 2, y, P, Pt)
        for x, y in self.site_coords:
            P = e.get_P("up", x + 1, y)
            Pt = e.get_Pt("up", x, y)
            nC1 = renormalize_C1_up(e.get_C1(x, y), e.get_T4(x, y + 1), P)
            nT1 = renormalize_T1(Pt, e.get_T1(x, y), e.get_A(x, y + 1), P)
            nC2 = renormalize_C2_up(e.get_C2(x, y), e.get_T2(x, y + 1), Pt)
            e.store_renormalized(x, y + 1, (nC1, nT1, nC2))
        e.commit(("C1", "T1", "C2"))

    def right_move(self):
        e = self._env
        for x, y in self.site_coords:
            P, Pt = self._projectors(
                self.construct_enlarged_dl(x, y),
                self.construct_enlarged_dr(x, y, free_memory=True),
                self.construct_enlarged_ur(x, y, free_memory=True),
                self.construct_enlarged_ul(x, y),
                e.get_C3(x + 2, y + 2).transpose(),
            )
            e.store_projectors("right", x + 3, y + 2, P, Pt)
        for x, y in self.site_coords:
            P = e.get_P("right", x, y + 1)
            Pt = e.get_Pt("right", x, y)
            nC2 = renormalize_C2_right(e.get_C2(x, y), e.get_T1(x - 1, y), P)
            nT2 = renormalize_T2(Pt, e.get_T2(x, y), e.get_A(x - 1, y), P)
            nC3 = renormalize_C3_right(e.get_C3(x, y), e.get_T3(x - 1, y), Pt)
            e.store_renormalized(x - 1, y, (nC2, nT2, nC3))
        e.commit(("C2", "T2", "C3"))

    def down_move(self):
        e = self._env
        for x, y in self.site_coords:
            P, Pt = self._projectors(
                self.construct_enlarged_ul(x, y),
                self.construct_enlarged_dl(x, y, free_memory=True),
                self.construct_enlarged_dr(x, y, free_memory=True),
                self.construct_enlarged_ur(x, y),
                e.get_C4(x + 1, y + 2),
            )
            e.store_projectors("down", x + 1, y + 3, P, Pt)
        for x, y in self.site_coords:
            P = e.get_P("down", x - 1, y)
            Pt = e.get_Pt("down", x, y)
            nC3 = renormalize_C3_down(e.get_C3(x, y), e.get_T2(x, y - 1), P)
            nT3 = renormalize_T3(Pt, e.get_T3(x, y), e.get_A(x, y - 1), P)
            nC4 = renormalize_C4_down(e.get_C4(x, y), e.get_T4(x, y - 1), Pt)
            e.store_renormalized(x, y - 1, (nC3, nT3, nC4))
        e.commit(("C3", "T3", "C4"))

    def left_move(self):
        e = self._env
        for x, y in self.site_coords:
            P, Pt = self._projectors(
                self.construct_enlarged_ur(x, y),
                self.construct_enlarged_ul(x, y, free_memory=True),
                self.construct_enlarged_dl(x, y, free_memory=True),
                self.construct_enlarged_dr(x, y),
                e.get_C1(x + 1, y + 1),
            )
            e.store_projectors("left", x, y + 1, P, Pt)
        for x, y in self.site_coords:
            P = e.get_P("left", x, y - 1)
            Pt = e.get_Pt("left", x, y)
            nC4 = renormalize_C4_left(e.get_C4(x, y), e.get_T3(x + 1, y), P)
            nT4 = renormalize_T4(Pt, e.get_T4(x, y), e.get_A(x + 1, y), P)
            nC1 = renormalize_C1_left(e.get_C1(x, y), e.get_T1(x + 1, y), Pt)
            e.store_renormalized(x + 1, y, (nC4, nT4, nC1))
        e.commit(("C4", "T4", "C1"))

    # ---------------------------------------------------------- observables
    def compute_PEPS_norm_log(self):
        """abstract_ctmrg.py:337-387."""
        e = self._env
        logZ = 0.0
        for x, y in self.site_coords:
            nc = contract_C1234(e.get_C1(x, y), e.get_C2(x + 1, y), e.get_C4(x, y + 1),
                                e.get_C3(x + 1, y + 1))
            nt13 = contract_T1T3(e.get_C1(x, y), e.get_T1(x + 1, y), e.get_C2(x + 2, y),
                                 e.get_C4(x, y + 1), e.get_T3(x + 1, y + 1),
                                 e.get_C3(x + 2, y + 1))
            nt24 = contract_T2T4(e.get_C1(x, y), e.get_C2(x + 1, y), e.get_T4(x, y + 1),
                                 e.get_T2(x + 1, y + 1), e.get_C4(x, y + 2),
                                 e.get_C3(x + 1, y + 2))
            n1234 = contract_norm(e.get_C1(x, y), e.get_T1(x + 1, y), e.get_C2(x + 2, y),
                                  e.get_T4(x, y + 1), e.get_A(x + 1, y + 1),
                                  e.get_T2(x + 2, y + 1), e.get_C4(x, y + 2),
                                  e.get_T3(x + 1, y + 2), e.get_C3(x + 2, y + 2))
            if nc * nt13 * nt24 * n1234 < 0:
                return np.nan
            logZ += (np.log(abs(n1234)) + np.log(abs(nc)) - np.log(abs(nt13))
                     - np.log(abs(nt24)))
        return logZ / self.n_sites

    def compute_rdm1x1(self, x, y):
        e = self._env
        return rdm.rdm_1x1(e.get_C1(x, y), e.get_T1(x + 1, y), e.get_C2(x + 2, y),
                           e.get_T4(x, y + 1), e.get_A(x + 1, y + 1), e.get_T2(x + 2, y + 1),
                           e.get_C4(x, y + 2), e.get_T3(x + 1, y + 2), e.get_C3(x + 2, y + 2))

    def compute_rdm1x2(self, x, y):
        e = self._env
        return rdm.rdm_1x2(
            e.get_C1(x, y), e.get_T1(x + 1, y), e.get_T1(x + 2, y), e.get_C2(x + 3, y),
            e.get_T4(x, y + 1), e.get_A(x + 1, y + 1), e.get_A(x + 2, y + 1),
            e.get_T2(x + 3, y + 1), e.get_C4(x, y + 2), e.get_T3(x + 1, y + 2),
            e.get_T3(x + 2, y + 2), e.get_C3(x + 3, y + 2),
        )

    def compute_rdm2x1(self, x, y):
        e = self._env
        return rdm.rdm_2x1(
            e.get_C1(x, y), e.get_T1(x + 1, y), e.get_C2(x + 2, y), e.get_T4(x, y + 1),
            e.get_A(x + 1, y + 1), e.get_T2(x + 2, y + 1), e.get_T4(x, y + 2),
            e.get_A(x + 1, y + 2), e.get_T2(x + 2, y + 2), e.get_C4(x, y + 3),
            e.get_T3(x + 1, y + 3), e.get_C3(x + 2, y + 3),
        )

    def compute_transfer_spectrum_h(self, y, nvals, *, dmax_full=200, maxiter=1000,
                                    arpack_tol=0):
        """abstract_ctmrg.py:519-538: nvals largest eigenvalues of the horizontal
        transfer matrix at cell row y."""
        e = self._env
        T1s = [e.get_T1(-x, y) for x in range(self.Lx)]
        T3s = [e.get_T3(-x, y + 1) for x in range(self.Lx)]
        return observables.compute_mps_transfer_spectrum(
            T1s, T3s, nvals, dmax_full=dmax_full, maxiter=maxiter, arpack_tol=arpack_tol,
            verbosity=self.verbosity)

    def compute_transfer_spectrum_v(self, x, nvals, *, dmax_full=200, maxiter=1000,
                                    arpack_tol=0):
        """abstract_ctmrg.py:540-559 (vertical transfer matrix at cell column x)."""
        e = self._env
        T1s = [e.get_T2(x + 1, -y).permute((1,), (2, 3, 0)) for y in range(self.Ly)]
        T3s = [e.get_T4(x, -y).permute((1, 2), (3, 0)) for y in range(self.Ly)]
        return observables.compute_mps_transfer_spectrum(
            T1s, T3s, nvals, dmax_full=dmax_full, maxiter=maxiter, arpack_tol=arpack_tol,
            verbosity=self.verbosity)

    def compute_corr_length_h(self, y, *, maxiter=1000, arpack_tol=0):
        """abstract_ctmrg.py:561-568: -Lx / ln |lambda_2 / lambda_1|."""
        _, v2 = self.compute_transfer_spectrum_h(y, 2, maxiter=maxiter, arpack_tol=arpack_tol)
        return -self.Lx / np.log(np.abs(v2))

    def compute_corr_length_v(self, x, *, maxiter=1000, arpack_tol=0):
        """abstract_ctmrg.py:570-577."""
        _, v2 = self.compute_transfer_spectrum_v(x, 2, maxiter=maxiter, arpack_tol=arpack_tol)
        return -self.Ly / np.log(np.abs(v2))

    def compute_rdm_1st_neighbor_cell(self):
        r12 = [self.compute_rdm1x2(x, y) for x, y in self.site_coords]
        r21 = [self.compute_rdm2x1(x, y) for x, y in self.site_coords]
        return r12, r21

    def compute_rdm1x1_cell(self):
        """abstract_ctmrg.py:476-483."""
        return [self.compute_rdm1x1(x, y) for x, y in self.site_coords]

    def compute_rdm_diag_dr(self, x, y, *, free_memory=False):
        """abstract_ctmrg.py:438-455: sites (x + 1, y + 1) and (x + 2, y + 2)."""
        e = self._env
        return rdm.rdm_diag_dr(
            e.get_C1(x, y), e.get_T1(x + 1, y),
            self.construct_enlarged_ur(x, y, free_memory=free_memory),
            e.get_T4(x, y + 1), e.get_A(x + 1, y + 1),
            self.construct_enlarged_dl(x, y, free_memory=free_memory),
            e.get_A(x + 2, y + 2), e.get_T2(x + 3, y + 2), e.get_T3(x + 2, y + 3),
            e.get_C3(x + 3, y + 3),
        )

    def compute_rdm_diag_ur(self, x, y, *, free_memory=False):
        """abstract_ctmrg.py:457-474: sites (x + 1, y + 2) and (x + 2, y + 1)."""
        e = self._env
        return rdm.rdm_diag_ur(
            self.construct_enlarged_ul(x, y, free_memory=free_memory),
            e.get_T1(x + 2, y), e.get_C2(x + 3, y), e.get_A(x + 2, y + 1),
            e.get_T2(x + 3, y + 1), e.get_T4(x, y + 2), e.get_A(x + 1, y + 2),
            self.construct_enlarged_dr(x, y, free_memory=free_memory),
            e.get_C4(x, y + 3), e.get_T3(x + 1, y + 3),
        )

    def compute_rdm_2nd_neighbor_cell(self, *, free_memory=True):
        """abstract_ctmrg.py:501-517: both diagonals of every unique site.  With
        free_memory the cached enlarged corners are dropped first and each is
        freed after use (the contraction peaks at 3 d^2 chi^2 D^4)."""
        if free_memory:
            self._env.reset_constructed_corners()
        dr, ur = [], []
        for x, y in self.site_coords:
            dr.append(self.compute_rdm_diag_dr(x, y, free_memory=free_memory))
            ur.append(self.compute_rdm_diag_ur(x, y, free_memory=free_memory))
        return dr, ur
