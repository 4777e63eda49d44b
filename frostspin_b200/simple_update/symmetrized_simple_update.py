"""Symmetrized simple update on device tensors
(frostspin/simple_update/symmetrized_simple_update.py:10-271).

Two-site checkerboard cell where the second tensor is the rotated dagger of
the first (B = A.dagger().permute((4, 5), (2, 3, 0, 1))), so only A is stored
and evolved.  A bond update contracts A with its own dagger through the bond
weight, applies the gate and keeps the leading eigenvectors of the resulting
Hermitian matrix (truncated eigh instead of SVD).  One second-order cycle
updates bonds 0, 1, 2, 3, 2, 1 with the end gates doubled, as in the
reference; the evolution loop and the file format are SimpleUpdate's.
"""

import numpy as np

from ..symmetric_tensor import DiagonalTensor
from ..symmetric_tensor.tools import get_symmetric_tensor_type
from .simple_update import SimpleUpdate, check_hamiltonians


class _FixedSchedule:
    """Leg swaps of the single tensor between default order (-1, -2, bonds)
    and the cycle (symmetrized_simple_update.py:11-30)."""

    initial_swap = [((1, 2, 4, 5), (3, 0))]
    final_swap = [((5, 0), (4, 1, 2, 3))]
    lperm = [
        ((0, 4, 2, 3), (1, 5)),
        ((0, 4, 2, 3), (1, 5)),
        ((0, 1, 4, 3), (2, 5)),
        ((0, 1, 2, 4), (3, 5)),
        ((0, 1, 2, 4), (3, 5)),
        ((0, 1, 4, 3), (2, 5)),
        ((0, 4, 2, 3), (1, 5)),
    ]
    bond = [0, 1, 2, 3, 2, 1, 0]
    gate = [1, 0, 0, 2, 0, 0, 0]
    n_updates = 6


class SymmetrizedSimpleUpdate(SimpleUpdate):
    _classname = "SymmetrizedSimpleUpdate"

    def __init__(self, D, beta, tau, rcutoff, degen_ratio, A, raw_hamilts, weights, logZ, *,
                 verbosity=0):
        if len(weights) != 4:
            raise ValueError("Invalid weight length")
        raw_hamilts = list(raw_hamilts)
        check_hamiltonians(raw_hamilts)
        self.verbosity = int(verbosity)
        self._sched = _FixedSchedule()
        if len(raw_hamilts) == 1:
            h = raw_hamilts[0]
            self._hamiltonians = [h, 2 * h, 2 * h]
        elif len(raw_hamilts) == 4:
            h = raw_hamilts
            self._hamiltonians = [h[0], h[1], h[2], 2 * h[3], 2 * h[0]]
        else:
            raise ValueError("Invalid raw_hamiltonians")
        self._beta = float(beta)
        self._n_bonds = 4
        self._n_updates = self._sched.n_updates
        self._n_tensors = 1
        self._symmetry = raw_hamilts[0].symmetry()
        self._tensor_bond_indices = [np.array([0, 1, 2, 3])]
        self._tensors = [A]
        self._weights = list(weights)
        self.D = int(D)
        self._logZ = float(logZ)
        self.rcutoff = float(rcutoff)
        self.degen_ratio = float(degen_ratio)
        self.tau = float(tau)
        self._raw_update_data = np.zeros((0, 0), dtype=int)
        self._raw_hamilts = raw_hamilts

    def __repr__(self):
        return (f"SymmetrizedSimpleUpdate with {self._symmetry} symmetry and D = {self.D}"
                f" at beta = {self._beta:.10g}")

    @classmethod
    def from_infinite_temperature(cls, D, tau, raw_hamilts, *, rcutoff=1e-14,
                                  degen_ratio=0.99999, verbosity=0):
        """symmetrized_simple_update.py:96-152: identity between physical and
        ancilla legs, trivial virtual legs, unit weights."""
        ST = type(raw_hamilts[0])
        h = raw_hamilts[0]
        if not (h.signature[0] ^ h.signature[1]):
            raise ValueError("the gate must act on a site and its dual")
        phys = h.row_reps[0]
        d = ST.representation_dimension(phys)
        s0 = bool(h.signature[0])
        A = ST.from_array(np.eye(d).reshape(d, d, 1, 1, 1, 1), (phys, phys),
                          (ST.singlet(),) * 4, signature=[not s0, s0, 1, 1, 1, 1])
        weights = [DiagonalTensor([np.ones((1,))], ST.singlet(), A.block_irreps, [1],
                                  ST.symmetry()) for _ in range(4)]
        return cls(D, 0.0, tau, rcutoff, degen_ratio, A, raw_hamilts, weights, 0.0,
                   verbosity=verbosity)

    @property
    def logZ(self):
        # the cell holds two tensors, A and its rotated dagger
        return self._logZ / 2

    def get_tensors(self):
        """symmetrized_simple_update.py:154-167: A with sqrt(weights) on its
        virtual legs, and its rotated dagger."""
        t = self._tensors[0]
        for w in self._weights:
            t = t.permute((0, 1, 3, 4, 5), (2,)) * w**-0.5
        t = t.permute((0, 1), (2, 3, 4, 5))
        return [t, t.dagger().permute((4, 5), (2, 3, 0, 1))]

    def update_first_neighbor(self, left, weights, gate):
        """symmetrized_simple_update.py:169-204: theta = effL effL^dagger
        through the bond weight, gate, truncated eigh."""
        cstL, effL = left.qr()
        effL = effL.permute((0, 2), (1,)) * weights**-0.5
        theta = effL @ effL.dagger()
        theta = theta.permute((0, 2), (1, 3)) @ gate
        theta = theta.permute((0, 2), (1, 3))
        new_weights, new_effL = theta.truncated_eigh(self.D, rtol=self.rcutoff,
                                                     degen_ratio=self.degen_ratio)
        new_weights /= new_weights.sum()
        lognf = np.log(theta.norm() / new_weights.norm())
        new_effL = (new_effL * new_weights).permute((0,), (2, 1))
        return cstL @ new_effL, new_weights, lognf

    def _elementary_update(self, i):
        """symmetrized_simple_update.py:206-219."""
        s = self._sched
        left = self._tensors[0].permute(*s.lperm[i])
        b = s.bond[i]
        new_left, nw, lognf = self.update_first_neighbor(left, self._weights[b],
                                                         self._gates[s.gate[i]])
        self._logZ += lognf
        self._weights[b] = nw
        self._tensors[0] = new_left

    @classmethod
    def load_from_file(cls, savefile, *, verbosity=0):
        """symmetrized_simple_update.py:221-271."""
        with np.load(savefile) as fin:
            if fin["_SimpleUpdate_classname"] != cls._classname:
                raise ValueError(f"Savefile '{savefile}' does not match class '{cls._classname}'")
            ST = get_symmetric_tensor_type(fin["_SimpleUpdate_symmetry"][()])
            hs = [ST.load_from_dic(fin, prefix=f"_SimpleUpdate_hamiltonian_{i}")
                  for i in range(int(fin["_SimpleUpdate_n_hamiltonians"]))]
            A = ST.load_from_dic(fin, prefix="_SimpleUpdate_tensor_0")
            weights = [DiagonalTensor.load_from_dic(fin, prefix=f"_SimpleUpdate_weights_{i}")
                       for i in range(4)]
            return cls(fin["_SimpleUpdate_D"][()], fin["_SimpleUpdate_beta"][()],
                       fin["_SimpleUpdate_tau"][()], fin["_SimpleUpdate_rcutoff"][()],
                       fin["_SimpleUpdate_degen_ratio"][()], A, hs, weights,
                       fin["_SimpleUpdate_logZ"][()], verbosity=verbosity)
