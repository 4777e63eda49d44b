"""Update tables of the second-neighbour simple-update models
(frostspin/simple_update/su_models.py:8-86).

All three live on the AB//CD plaquette of the square lattice: four site
tensors, eight bonds, tensor_bond_indices [[0, 1, 2, 3], [4, 3, 5, 1],
[2, 6, 0, 7], [5, 7, 4, 6]].  A row is (bond1, bond2, hamiltonian, left tensor,
right tensor, middle tensor); a first-neighbour gate has bond1 == bond2 and no
middle tensor (-1), a second-neighbour gate acts through the middle tensor
between its two bonds.  Hamiltonian 0 is h1, hamiltonian 1 is h2 / 2 (every
diagonal is updated twice, through both intermediate sites).  The row order
is the Trotter order, so it is part of the model.
"""

import numpy as np

# the eight first-neighbour bonds: (bond, left tensor, right tensor)
_FIRST = [(0, 0, 2), (1, 0, 1), (2, 0, 2), (3, 0, 1), (4, 3, 1), (5, 3, 1), (6, 3, 2),
          (7, 3, 2)]

# the sixteen second-neighbour gates of the J1-J2 model:
# (bond1, bond2, left tensor, right tensor, middle tensor)
_DIAGONAL = [
    (0, 7, 0, 3, 2), (4, 3, 3, 0, 1), (6, 0, 3, 0, 2), (1, 4, 0, 3, 1),
    (5, 1, 3, 0, 1), (2, 6, 0, 3, 2), (7, 2, 3, 0, 2), (3, 5, 0, 3, 1),
    (4, 6, 1, 2, 3), (0, 1, 2, 1, 0), (3, 0, 1, 2, 0), (7, 4, 2, 1, 3),
    (5, 7, 1, 2, 3), (2, 3, 2, 1, 0), (1, 2, 1, 2, 0), (6, 5, 2, 1, 3),
]

# diagonals present in each model, in Trotter order
_MODEL_DIAGONALS = {
    "J1-J2": list(range(16)),
    "checkerboard": [0, 1, 4, 5, 10, 11, 14, 15],
    "Shastry-Sutherland": [0, 1, 14, 15],
}

TENSOR_BOND_INDICES = [[0, 1, 2, 3], [4, 3, 5, 1], [2, 6, 0, 7], [5, 7, 4, 6]]


def _table(diagonals):
    rows = [(b, b, 0, left, right, -1) for b, left, right in _FIRST]
    rows += [(b1, b2, 1, left, right, mid)
             for b1, b2, left, right, mid in (_DIAGONAL[i] for i in diagonals)]
    return np.array(rows, dtype=np.int64)


j1_j2_models = {name: _table(d) for name, d in _MODEL_DIAGONALS.items()}
