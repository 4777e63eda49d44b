"""CPU oracle of the finite-temperature simple update -- TEST INFRASTRUCTURE ONLY.

A numpy restatement of frostspin/simple_update (abstract_simple_update.py:
94-147, simple_update.py:338-363, 409-535, 599-700) for the square-lattice
first-neighbour model on the 2-site checkerboard cell, over the oracle
tensors of frostspin_oracle.py (U(1)) or su2_oracle.py (SU(2)).

The reference keeps every tensor in a rotating leg order between updates
(initial_swap, lperm, rperm, final_swap) to save permutes.  Here each tensor
stays in its default leg order (physical, ancilla, bonds in
tensor_bond_indices order) and is permuted into the update's form and back
around every update: the same updates in the same order on the same tensors
(permutes are exact up to the rounding of the SU(2) recoupling), so beta,
logZ, bond representations and weights agree with the reference's run to
rounding.  The sequence per evolve(beta) follows abstract_simple_update.py:
94-147: niter = round(beta / (4 tau)); one half step (plain gate on bond 0),
the rest of the first cycle, niter - 1 full cycles whose end points (bonds 0
and 3) use the doubled gate, and a closing half step on bond 0.

Only tests/ and bench.py's CPU-baseline leg use this module.
"""

import numpy as np
import scipy.linalg as sla

from . import frostspin_oracle as fo
from . import su2_oracle as so

# first-neighbour square lattice (simple_update.py:338-363): tensor 0 carries
# bonds (0, 1, 2, 3), tensor 1 bonds (2, 3, 0, 1); every update is on bond b
# between tensor 0 (left) and tensor 1 (right)
TENSOR_BONDS = ((0, 1, 2, 3), (2, 3, 0, 1))


# ------------------------------------------------------------------ blocks


def _irrep_dims(m, irreps):
    return np.asarray(m.irrep_dims(irreps), dtype=np.int64)


def expm_tensor(m, h, x):
    """exp(x h) blockwise (SymmetricTensor.expm on every irrep block)."""
    return m.OTensor(h.row_reps, h.col_reps, [sla.expm(x * b) for b in h.blocks],
                     h.block_irreps, h.signature)


def qr(m, t):
    """symmetric_tensor.py:655-670: economic QR of every block; the middle leg
    has min(rows, cols) states per irrep."""
    qs, rs = [], []
    for b in t.blocks:
        q, r = np.linalg.qr(b, mode="reduced")
        qs.append(q)
        rs.append(r)
    mid = m.init_representation(np.array([r.shape[0] for r in rs]), t.block_irreps)
    nrr = t.nrr
    Q = m.OTensor(t.row_reps, (mid,), qs, t.block_irreps, np.r_[t.signature[:nrr], True])
    R = m.OTensor((mid,), t.col_reps, rs, t.block_irreps, np.r_[False, t.signature[nrr:]])
    return Q, R


def truncated_svd(m, t, cut, rtol, degen_ratio):
    """symmetric_tensor.py:835-877 with the dense per-block SVD: values kept
    by find_block_cuts counting each value of irrep block i dims[i] times;
    returns (U, (weight blocks, irreps), V)."""
    us, ss, vs = [], [], []
    for b in t.blocks:
        u, s, v = np.linalg.svd(b, full_matrices=False)
        us.append(u)
        ss.append(s)
        vs.append(v)
    cuts = fo.find_block_cuts(ss, cut, dims=_irrep_dims(m, t.block_irreps), rtol=rtol,
                              degen_ratio=degen_ratio)
    keep = np.flatnonzero(cuts)
    irr = t.block_irreps[keep]
    mid = m.init_representation(cuts[keep], irr)
    nrr = t.nrr
    U = m.OTensor(t.row_reps, (mid,), [us[i][:, : cuts[i]] for i in keep], irr,
                  np.r_[t.signature[:nrr], True])
    V = m.OTensor((mid,), t.col_reps, [vs[i][: cuts[i]] for i in keep], irr,
                  np.r_[False, t.signature[nrr:]])
    return U, ([ss[i][: cuts[i]].copy() for i in keep], irr), V


def weights_sum(m, w):
    """DiagonalTensor.sum (diagonal_tensor.py:195-199): irrep-dimension weighted."""
    blocks, irr = w
    return float(sum(d * b.sum() for d, b in zip(_irrep_dims(m, irr), blocks, strict=True)))


def weights_norm(m, w):
    """DiagonalTensor.norm (diagonal_tensor.py:201-205)."""
    blocks, irr = w
    return float(np.sqrt(sum(d * (b @ b) for d, b in zip(_irrep_dims(m, irr), blocks,
                                                         strict=True))))


def diag_mul(m, t, w, *, left):
    """t * w (left=False: the column leg of a one-column-leg matrix) or w * t
    (left=True: the row leg), symmetric_tensor.py:1189-1248."""
    blocks, irr = w
    if m is fo:
        return fo.diagonal_mul(t, blocks, irr, left=left)
    # SU(2) irreps are self-conjugate: blocks meet by irrep
    pos = {int(q): i for i, q in enumerate(irr)}
    out, out_irr = [], []
    for b, q in zip(t.blocks, t.block_irreps, strict=True):
        i = pos.get(int(q))
        if i is None:
            continue
        d = blocks[i]
        out.append(b * (d[:, None] if left else d))
        out_irr.append(q)
    return m.OTensor(t.row_reps, t.col_reps, out, np.asarray(out_irr, dtype=t.block_irreps.dtype),
                     t.signature)


# ------------------------------------------------------------------ update


def update_first_neighbor(m, left, right, weights, gate, D, rcutoff, degen_ratio):
    """simple_update.py:633-697.  left / right: rows = the legs the gate does
    not touch, columns = (physical, updated bond); returns the new left and
    right in the same form, the new weights and log of the normalisation."""
    cstL, effL = qr(m, left)
    cstR, effR = qr(m, right)
    inv = ([1.0 / b for b in weights[0]], weights[1])
    effL = diag_mul(m, m.permute(effL, (0, 1), (2,)), inv, left=False)
    effR = m.permute(effR, (2,), (0, 1))
    theta = m.matmul(effL, effR)
    theta = m.matmul(m.permute(theta, (0, 2), (1, 3)), gate)
    theta = m.permute(theta, (0, 2), (1, 3))
    effL, nw, effR = truncated_svd(m, theta, D, rcutoff, degen_ratio)
    s = weights_sum(m, nw)
    nw = ([b / s for b in nw[0]], nw[1])
    lognf = float(np.log(m.norm(theta) / weights_norm(m, nw)))
    effL = m.permute(diag_mul(m, effL, nw, left=False), (0,), (1, 2))
    effR = m.permute(diag_mul(m, effR, nw, left=True), (1,), (2, 0))
    return m.matmul(cstL, effL), m.matmul(cstR, effR), nw, lognf


def _to_update_form(t, bond_pos):
    """Default legs (physical, ancilla, bonds...) -> rows (ancilla, the other
    bonds in order), columns (physical, the updated bond); the axes and the
    inverse permutation back."""
    rest = [1] + [2 + j for j in range(4) if j != bond_pos]
    axes = rest + [0, 2 + bond_pos]
    back = tuple(int(i) for i in np.argsort(axes))
    return (tuple(rest), (0, 2 + bond_pos)), (back[:2], back[2:])


class SimpleUpdate:
    """Square-lattice first-neighbour simple update on the AB checkerboard cell
    (simple_update.py:338-363), second-order Trotter (abstract_simple_update.py:
    94-147): tensors in their default leg order between updates."""

    def __init__(self, h, D, tau, *, rcutoff=1e-10, degen_ratio=1.0):
        m = so if isinstance(h, so.OTensor) else fo
        self.m = m
        self.D = int(D)
        self.tau = float(tau)
        self.rcutoff = float(rcutoff)
        self.degen_ratio = float(degen_ratio)
        self.beta = 0.0
        self._logZ = 0.0   # summed over updates; logZ is per tensor (abstract_simple_update.py:26-27)
        self.gate = expm_tensor(m, h, -self.tau)          # plain step
        self.gate2 = expm_tensor(m, h, -2.0 * self.tau)   # doubled end points
        # from_infinite_temperature (simple_update.py:409-535): identity between
        # the physical leg and its ancilla, trivial virtual legs, unit weights;
        # the left tensor's bonds are outgoing, the right tensor's incoming
        phys = h.row_reps[0]
        d = int(np.prod(h.shape[:1]))
        one = m.singlet()
        self.tensors = []
        for i in range(2):
            sig = [not bool(h.signature[i]), bool(h.signature[i])] + [i == 0] * 4
            mat = np.eye(d).reshape((d, d, 1, 1, 1, 1))
            self.tensors.append(m.from_array(mat, (phys, phys), (one,) * 4, signature=sig))
        singlet_irrep = np.array([1], dtype=np.int64) if m is so else np.zeros(1, dtype=np.int8)
        self.weights = [([np.ones(1)], singlet_irrep) for _ in range(4)]

    def _update(self, bond, gate):
        m = self.m
        lf, lb = _to_update_form(self.tensors[0], TENSOR_BONDS[0].index(bond))
        rf, rb = _to_update_form(self.tensors[1], TENSOR_BONDS[1].index(bond))
        left = m.permute(self.tensors[0], *lf)
        right = m.permute(self.tensors[1], *rf)
        nl, nr, nw, lognf = update_first_neighbor(m, left, right, self.weights[bond], gate,
                                                  self.D, self.rcutoff, self.degen_ratio)
        self.tensors[0] = m.permute(nl, *lb)
        self.tensors[1] = m.permute(nr, *rb)
        self.weights[bond] = nw
        self._logZ += lognf

    def evolve(self, beta_evolve):
        """abstract_simple_update.py:94-147 for the sequence bonds 0, 1, 2, 3,
        2, 1 (forward, then back without the end points)."""
        dbeta = 4.0 * self.tau
        if beta_evolve < 0.9 * dbeta:
            return
        niter = round(beta_evolve / dbeta)
        seq = (0, 1, 2, 3, 2, 1)
        self._update(0, self.gate)
        for j in range(1, len(seq)):
            self._update(seq[j], self.gate2 if j == 3 else self.gate)
        for _ in range(niter - 1):
            for j, b in enumerate(seq):
                self._update(b, self.gate2 if j in (0, 3) else self.gate)
        self._update(0, self.gate)
        self.beta += niter * dbeta

    @property
    def logZ(self):
        return self._logZ / len(self.tensors)

    def bond_representation(self, bond):
        """The bond leg's representation on the left tensor."""
        return self.tensors[0].col_reps[TENSOR_BONDS[0].index(bond)]

    def sorted_weights(self, bond):
        """All weights of a bond, each repeated by its irrep dimension, in
        decreasing order (get_weights(sort=True))."""
        blocks, irr = self.weights[bond]
        dims = _irrep_dims(self.m, irr)
        return np.sort(np.concatenate([np.repeat(b, d) for b, d in zip(blocks, dims, strict=True)]))[::-1]
