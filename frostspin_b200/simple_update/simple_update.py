"""Finite-temperature simple update on device tensors.

Same algorithm, conventions and file format as frostspin/simple_update/
(simple_update.py:11-790, abstract_simple_update.py:1-187): imaginary-time
second-order Trotter evolution of a purification (physical and ancilla leg on
every tensor), bond weights as DiagonalTensors, truncation to a target bond
dimension D keeping whole multiplets, beta counted on the bilayer
(dbeta = 4 tau per cycle).  Every tensor operation is a device permute, grouped
GEMM, diagonal product, QR or truncated SVD.
"""

import numpy as np

from ..symmetric_tensor import DiagonalTensor
from ..symmetric_tensor.tools import get_symmetric_tensor_type
from .su_models import TENSOR_BOND_INDICES, j1_j2_models


def check_tensor_bond_indices(tensor_bond_indices):
    """Every bond on exactly two tensors, no bond twice on one tensor
    (simple_update_tools.py:4-31)."""
    n_bonds = max(max(t) for t in tensor_bond_indices) + 1
    count = np.zeros(n_bonds, dtype=int)
    for i, tbi in enumerate(tensor_bond_indices):
        tbi = list(tbi)
        for j, leg in enumerate(tbi):
            if not 0 <= leg < n_bonds:
                raise ValueError("Bond indices must be 0 to n_bonds - 1")
            if leg in tbi[j + 1 :]:
                raise ValueError(f"Leg {leg} apperars twice in tensor {i}")
            count[leg] += 1
    for i, c in enumerate(count):
        if c != 2:
            raise ValueError(f"Virtual bond {i} appears {c} times")


def check_hamiltonians(hamiltonians):
    """simple_update_tools.py:34-42."""
    ST = type(hamiltonians[0])
    for i, h in enumerate(hamiltonians):
        if type(h) is not ST:
            raise ValueError(f"Invalid type for Hamiltonian {i}")
        if h.ndim != 4 or h.n_row_reps != 2:
            raise ValueError(f"Hamiltonian {i} has invalid shape")
        for a in range(2):
            if not np.array_equal(h.row_reps[a], h.col_reps[a]):
                raise ValueError(f"Hamiltonian {i} has invalid representations")
            if not h.signature[a] ^ h.signature[a + 2]:
                raise ValueError(f"Hamiltonian {i} has invalid signature")


def _swap(init, end):
    """(row_axes, col_axes) taking leg labels `init` to `end`, last two legs as
    columns."""
    p = [init.index(x) for x in end]
    return tuple(p[:-2]), tuple(p[-2:])


class UpdateSchedule:
    """Update sequence and leg bookkeeping (simple_update.py:11-184).

    Legs are labelled -1 (physical), -2 (ancilla) and by bond index.  Between
    the updates of one cycle a tensor keeps its two active legs last (columns);
    lperm/rperm/mperm move each tensor from its previous active pair to the one
    of the next update, initial_swap/final_swap convert from/to the default
    order (-1, -2, *bonds).  A second-order cycle is the forward sequence
    followed by its reverse without the end points; the end points use a doubled
    gate, and a final extra step (a copy of step 0 with the plain gate) opens and
    closes the evolution.
    """

    def __init__(self, tensor_bond_indices, raw_update_data, raw_hamilts, second_order=True):
        data = np.asarray(raw_update_data, dtype=int)
        if second_order:
            data = np.vstack((data, data[-2:0:-1]))
        self.bond1 = list(data[:, 0])
        self.bond2 = list(data[:, 1])
        self.gate = list(data[:, 2])
        self.left = list(data[:, 3])
        self.right = list(data[:, 4])
        self.middle = [u[5] if u[0] != u[1] else None for u in data]
        n_up = len(self.bond1)
        n_t = len(tensor_bond_indices)
        self.hamiltonians = list(raw_hamilts)

        def active_after(upto):
            state = [None] * n_t
            for i in upto:
                state[self.left[i]] = [-1, self.bond1[i]]
                state[self.right[i]] = [-1, self.bond2[i]]
                if self.bond1[i] != self.bond2[i]:
                    state[self.middle[i]] = [self.bond1[i], self.bond2[i]]
            return state

        eff = active_after(range(n_up))
        legs = [None] * n_t
        self.initial_swap = [None] * n_t
        for i in range(n_t):
            init = [-1, -2, *tensor_bond_indices[i]]
            end = sorted(set(init) - set(eff[i])) + eff[i]
            self.initial_swap[i] = _swap(init, end)
            legs[i] = end

        self.lperm, self.rperm, self.mperm = [None] * n_up, [None] * n_up, [None] * n_up
        for i in range(n_up):
            for side, bond, perms in ((self.left[i], self.bond1[i], self.lperm),
                                      (self.right[i], self.bond2[i], self.rperm)):
                init = legs[side]
                end = [*sorted(set(init) - {-1, bond}), -1, bond]
                perms[i] = _swap(init, end)
                legs[side] = end
            if self.bond1[i] != self.bond2[i]:
                m = self.middle[i]
                b12 = [self.bond1[i], self.bond2[i]]
                init = legs[m]
                end = sorted(set(init) - set(b12)) + b12
                self.mperm[i] = _swap(init, end)
                legs[m] = end

        for lst in (self.bond1, self.bond2, self.gate, self.left, self.right, self.middle,
                    self.lperm, self.rperm, self.mperm):
            lst.append(lst[0])

        if second_order:
            eff[self.left[0]] = [-1, self.bond1[0]]
            eff[self.right[0]] = [-1, self.bond2[0]]
            if self.bond1[0] != self.bond2[0]:
                eff[self.middle[0]] = [self.bond1[0], self.bond2[0]]
            self.hamiltonians.append(2 * raw_hamilts[self.gate[0]])
            self.gate[0] = len(raw_hamilts)
            self.hamiltonians.append(2 * raw_hamilts[self.gate[n_up // 2]])
            self.gate[n_up // 2] = len(raw_hamilts) + 1

        self.final_swap = [None] * n_t
        for i in range(n_t):
            end = [-1, -2, *tensor_bond_indices[i]]
            init = sorted(set(end) - set(eff[i])) + eff[i]
            p = [init.index(x) for x in end]
            self.final_swap[i] = (tuple(p[:2]), tuple(p[2:]))
        self.n_updates = n_up


class SimpleUpdate:
    _classname = "SimpleUpdate"
    _is_second_order = True

    def __init__(self, D, beta, tau, rcutoff, degen_ratio, tensor_bond_indices, tensors,
                 raw_update_data, raw_hamilts, weights, logZ, *, verbosity=0):
        tensor_bond_indices = [np.array(t, dtype=int) for t in tensor_bond_indices]
        raw_hamilts = list(raw_hamilts)
        check_tensor_bond_indices(tensor_bond_indices)
        check_hamiltonians(raw_hamilts)
        if len(tensors) != len(tensor_bond_indices):
            raise ValueError("Invalid tensor number")
        self.verbosity = int(verbosity)
        self._sched = UpdateSchedule([list(t) for t in tensor_bond_indices],
                                     raw_update_data, raw_hamilts)
        self._hamiltonians = self._sched.hamiltonians
        self._beta = float(beta)
        self._n_bonds = len(weights)
        self._n_updates = self._sched.n_updates
        self._n_tensors = len(tensors)
        self._symmetry = raw_hamilts[0].symmetry()
        self._tensor_bond_indices = tensor_bond_indices
        self._tensors = list(tensors)
        self._weights = list(weights)
        self.D = int(D)
        self._logZ = float(logZ)
        self.rcutoff = float(rcutoff)
        self.degen_ratio = float(degen_ratio)
        self.tau = float(tau)
        self._raw_update_data = np.asarray(raw_update_data, dtype=int)
        self._raw_hamilts = raw_hamilts

    def __repr__(self):
        return (f"SimpleUpdate with {self._symmetry} symmetry and D = {self.D}"
                f" at beta = {self._beta:.10g}")

    # ----------------------------------------------------------- constructors
    @classmethod
    def square_lattice_first_neighbor(cls, h1, D, tau, *, rcutoff=1e-10, degen_ratio=1.0,
                                      verbosity=0):
        """simple_update.py:338-363: 2-site checkerboard cell, 4 bonds."""
        tensor_bond_indices = [[0, 1, 2, 3], [2, 3, 0, 1]]
        update_data = np.array([[b, b, 0, 0, 1, -1] for b in range(4)])
        return cls.from_infinite_temperature(D, tau, rcutoff, degen_ratio,
                                             tensor_bond_indices, update_data, [h1],
                                             verbosity=verbosity)

    @classmethod
    def square_lattice_second_neighbor(cls, h1, h2, D, tau, *, model="J1-J2", rcutoff=1e-10,
                                       degen_ratio=1.0, verbosity=0):
        """simple_update.py:366-407: AB//CD plaquette, 8 bonds, first-neighbour
        gates h1 and second-neighbour gates h2 / 2 applied through both
        intermediate sites; ``model`` is "J1-J2", "checkerboard" or
        "Shastry-Sutherland" (su_models.py)."""
        if model not in j1_j2_models:
            raise KeyError(f"Unknown model: {model}")
        return cls.from_infinite_temperature(D, tau, rcutoff, degen_ratio,
                                             TENSOR_BOND_INDICES, j1_j2_models[model],
                                             [h1, h2 / 2], verbosity=verbosity)

    @classmethod
    def from_infinite_temperature(cls, D, tau, rcutoff, degen_ratio, tensor_bond_indices,
                                  raw_update_data, raw_hamilts, *, verbosity=0):
        """beta = 0 product state (simple_update.py:409-535): identity between the
        physical and ancilla legs, trivial virtual legs, unit weights."""
        check_tensor_bond_indices(tensor_bond_indices)
        n_t = len(tensor_bond_indices)
        n_bonds = max(max(t) for t in tensor_bond_indices) + 1
        ST = type(raw_hamilts[0])
        sched = UpdateSchedule([list(t) for t in tensor_bond_indices], raw_update_data,
                               raw_hamilts)
        phys = [ST.singlet() for _ in range(n_t)]
        sigs = [[None] * (2 + len(t)) for t in tensor_bond_indices]
        for j, b1 in enumerate(sched.bond1):
            b2 = sched.bond2[j]
            h = sched.hamiltonians[sched.gate[j]]
            iL, iR = sched.left[j], sched.right[j]
            phys[iL] = h.row_reps[0]
            sigs[iL][0], sigs[iL][1] = ~h.signature[0], h.signature[0]
            sigs[iL][2 + list(tensor_bond_indices[iL]).index(b1)] = True
            phys[iR] = h.row_reps[1]
            sigs[iR][0], sigs[iR][1] = ~h.signature[1], h.signature[1]
            sigs[iR][2 + list(tensor_bond_indices[iR]).index(b2)] = False
            if b2 != b1:
                im = sched.middle[j]
                sigs[im][2 + list(tensor_bond_indices[im]).index(b1)] = False
                sigs[im][2 + list(tensor_bond_indices[im]).index(b2)] = True
        tensors = []
        t = None
        for i in range(n_t):
            d = ST.representation_dimension(phys[i])
            mat = np.eye(d).reshape((d, d) + (1,) * len(tensor_bond_indices[i]))
            t = ST.from_array(mat, (phys[i], phys[i]), (ST.singlet(),) * len(tensor_bond_indices[i]),
                              signature=sigs[i])
            tensors.append(t)
        weights = [DiagonalTensor([np.ones((1,))], ST.singlet(), t.block_irreps, [1],
                                  ST.symmetry()) for _ in range(n_bonds)]
        return cls(D, 0.0, tau, rcutoff, degen_ratio, tensor_bond_indices, tensors,
                   raw_update_data, raw_hamilts, weights, 0.0, verbosity=verbosity)

    # ------------------------------------------------------------- properties
    @property
    def Dmax(self):
        return max(max(t.shape[2:]) for t in self._tensors)

    @property
    def beta(self):
        return self._beta

    @property
    def n_bonds(self):
        return self._n_bonds

    @property
    def n_tensors(self):
        return self._n_tensors

    @property
    def logZ(self):
        return self._logZ / self._n_tensors

    @property
    def tau(self):
        return self._tau

    @tau.setter
    def tau(self, tau):
        """Gates exp(-tau h) on the device (abstract_simple_update.py:29-36)."""
        self._tau = tau
        self._gates = tuple((-tau * h).expm() for h in self._hamiltonians)
        self._dbeta = 2 * (1 + self._is_second_order) * tau

    def symmetry(self):
        return self._symmetry

    def get_bond_representation(self, i):
        for j in range(self._n_tensors):
            ind = np.flatnonzero(self._tensor_bond_indices[j] == i)
            if ind.size:
                return self._tensors[j].col_reps[ind[0]]
        raise ValueError(f"Unknown bond {i}")

    def get_bond_representations(self):
        return [self.get_bond_representation(i) for i in range(self._n_bonds)]

    def get_weights(self, *, sort=True):
        return [w.toarray(sort=sort) for w in self._weights]

    def bond_entanglement_entropy(self):
        return np.array([-w @ np.log(w) for w in self.get_weights()])

    def get_tensors(self):
        """Tensors with sqrt(weights) on every virtual leg
        (abstract_simple_update.py:73-92)."""
        sqw = [w**-0.5 for w in self._weights]
        out = []
        for i, t0 in enumerate(self._tensors):
            rswap = (0, 1, *range(3, t0.ndim))
            t = t0
            for leg in self._tensor_bond_indices[i]:
                t = t.permute(rswap, (2,)) * sqw[leg]
            out.append(t.permute((0, 1), tuple(range(2, t0.ndim))))
        return out

    # --------------------------------------------------------------- evolution
    def evolve(self, beta_evolve):
        """abstract_simple_update.py:94-147."""
        if beta_evolve < -1e-12:
            raise ValueError("Cannot evolve for negative imaginary time")
        if beta_evolve < 0.9 * self._dbeta:
            return
        niter = round(beta_evolve / self._dbeta)
        s = self._sched
        for i in range(self._n_tensors):
            self._tensors[i] = self._tensors[i].permute(*s.initial_swap[i])
        self._elementary_update(self._n_updates)
        for j in range(1, self._n_updates):
            self._elementary_update(j)
        for _ in range(niter - 1):
            for j in range(self._n_updates):
                self._elementary_update(j)
        self._elementary_update(self._n_updates)
        for i in range(self._n_tensors):
            self._tensors[i] = self._tensors[i].permute(*s.final_swap[i])
        self._beta += niter * self._dbeta

    def _elementary_update(self, i):
        """simple_update.py:599-631."""
        s = self._sched
        left = self._tensors[s.left[i]].permute(*s.lperm[i])
        right = self._tensors[s.right[i]].permute(*s.rperm[i])
        b1, b2 = s.bond1[i], s.bond2[i]
        gate = self._gates[s.gate[i]]
        if b1 == b2:
            left, right, nw1, lognf = self.update_first_neighbor(left, right,
                                                                 self._weights[b1], gate)
        else:
            mid = self._tensors[s.middle[i]].permute(*s.mperm[i])
            left, mid, right, nw1, nw2, lognf = self.update_through_proxy(
                left, mid, right, self._weights[b1], self._weights[b2], gate)
            self._weights[b2] = nw2
            self._tensors[s.middle[i]] = mid
        self._logZ += lognf
        self._weights[b1] = nw1
        self._tensors[s.left[i]] = left
        self._tensors[s.right[i]] = right

    def _truncated_svd(self, theta):
        return theta.truncated_svd(self.D, rtol=self.rcutoff, degen_ratio=self.degen_ratio)

    def update_first_neighbor(self, left, right, weights, gate):
        """simple_update.py:633-698: QR off the constant parts, absorb the inverse
        weights, apply the gate, truncated SVD, renormalise the new weights to sum
        1 and absorb them back."""
        cstL, effL = left.qr()
        cstR, effR = right.qr()
        effL = effL.permute((0, 1), (2,)) * weights**-1
        effR = effR.permute((2,), (0, 1))
        theta = (effL @ effR).permute((0, 2), (1, 3)) @ gate
        theta = theta.permute((0, 2), (1, 3))
        effL, new_weights, effR = self._truncated_svd(theta)
        new_weights /= new_weights.sum()
        lognf = np.log(theta.norm() / new_weights.norm())
        effL = (effL * new_weights).permute((0,), (1, 2))
        effR = (new_weights * effR).permute((1,), (2, 0))
        return cstL @ effL, cstR @ effR, new_weights, lognf

    def update_through_proxy(self, left, mid, right, weightsL, weightsR, gate):
        """simple_update.py:700-790: gate between two tensors through a middle one,
        two successive truncated SVDs."""
        cstL, effL = left.qr()
        effL = effL.permute((0, 1), (2,)) * weightsL**-1
        cstm, effm = mid.qr()
        effm = effm.permute((1,), (2, 0))
        cstR, effR = right.qr()
        effR = effR.permute((0, 1), (2,)) * weightsR**-1
        theta = (effL @ effm).permute((0, 1, 3), (2,)) @ effR.transpose()
        theta = theta.permute((0, 2, 3), (1, 4)) @ gate
        theta = theta.permute((4, 2), (0, 3, 1))
        norm0 = theta.norm()
        effR, new_weightsR, theta = self._truncated_svd(theta)
        new_weightsR /= new_weightsR.sum()
        effR = effR * new_weightsR
        theta = (new_weightsR * theta).permute((1, 2), (3, 0))
        effL, new_weightsL, effm = self._truncated_svd(theta)
        new_weightsL /= new_weightsL.sum()
        lognf = np.log(norm0 / new_weightsL.norm())
        effm = (new_weightsL * effm).permute((1,), (0, 2))
        effL = (effL * new_weightsL).permute((0,), (1, 2))
        effR = effR.permute((1,), (0, 2))
        return cstL @ effL, cstm @ effm, cstR @ effR, new_weightsL, new_weightsR, lognf

    # ---------------------------------------------------------------------- I/O
    def save_to_file(self, savefile, **additional_data):
        """Same keys as abstract_simple_update.py:149-187."""
        data = {
            "_SimpleUpdate_symmetry": self._symmetry,
            "_SimpleUpdate_classname": self._classname,
            "_SimpleUpdate_D": self.D,
            "_SimpleUpdate_beta": self._beta,
            "_SimpleUpdate_tau": self._tau,
            "_SimpleUpdate_logZ": self._logZ,
            "_SimpleUpdate_is_second_order": self._is_second_order,
            "_SimpleUpdate_rcutoff": self.rcutoff,
            "_SimpleUpdate_degen_ratio": self.degen_ratio,
            "_SimpleUpdate_raw_update_data": self._raw_update_data,
            "_SimpleUpdate_n_bonds": self._n_bonds,
            "_SimpleUpdate_n_hamiltonians": len(self._raw_hamilts),
            "_SimpleUpdate_n_tensors": self._n_tensors,
        }
        for i, h in enumerate(self._raw_hamilts):
            data |= h.get_data_dic(prefix=f"_SimpleUpdate_hamiltonian_{i}")
        for i, tbi in enumerate(self._tensor_bond_indices):
            data |= self._tensors[i].get_data_dic(prefix=f"_SimpleUpdate_tensor_{i}")
            data[f"_SimpleUpdate_tensor_bond_indices_{i}"] = tbi
        for i, w in enumerate(self._weights):
            data |= w.get_data_dic(prefix=f"_SimpleUpdate_weights_{i}")
        np.savez_compressed(savefile, **data, **additional_data)

    @classmethod
    def load_from_file(cls, savefile, *, verbosity=0):
        """simple_update.py:538-597."""
        with np.load(savefile) as fin:
            if fin["_SimpleUpdate_classname"] != cls._classname:
                raise ValueError(f"Savefile '{savefile}' does not match class '{cls._classname}'")
            ST = get_symmetric_tensor_type(fin["_SimpleUpdate_symmetry"][()])
            hs = [ST.load_from_dic(fin, prefix=f"_SimpleUpdate_hamiltonian_{i}")
                  for i in range(int(fin["_SimpleUpdate_n_hamiltonians"]))]
            tensors, tbis = [], []
            for i in range(int(fin["_SimpleUpdate_n_tensors"])):
                tensors.append(ST.load_from_dic(fin, prefix=f"_SimpleUpdate_tensor_{i}"))
                tbis.append(fin[f"_SimpleUpdate_tensor_bond_indices_{i}"])
            weights = [DiagonalTensor.load_from_dic(fin, prefix=f"_SimpleUpdate_weights_{i}")
                       for i in range(int(fin["_SimpleUpdate_n_bonds"]))]
            return cls(fin["_SimpleUpdate_D"][()], fin["_SimpleUpdate_beta"][()],
                       fin["_SimpleUpdate_tau"][()], fin["_SimpleUpdate_rcutoff"][()],
                       fin["_SimpleUpdate_degen_ratio"][()], tbis, tensors,
                       fin["_SimpleUpdate_raw_update_data"], hs, weights,
                       fin["_SimpleUpdate_logZ"][()], verbosity=verbosity)
