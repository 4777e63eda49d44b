"""CTMRG environment container (frostspin/ctmrg/ctm_environment.py:6-460).

Unit cells are given as tiling strings ("A", "AB\\nBA", ...).  Site (x, y) maps
to the unique tensor index indices[x mod Lx, y mod Ly]; every unique site owns
C1..C4, T1..T4 and the four enlarged corners built from it.  The .npz keys are
the reference's (`_CTM_cell`, `_CTM_symmetry`, `_CTM_A_i`, `_CTM_C1_i`, ...).
"""

import numpy as np

from ..symmetric_tensor.tools import get_symmetric_tensor_type

_NAMES = ("C1", "C2", "C3", "C4", "T1", "T2", "T3", "T4")


def initialize_dummy_env(A):
    """1x1 identity corners and layer-identity edges (ctm_environment.py:6-34)."""
    ST = type(A)
    one = (ST.singlet(),)
    C1 = ST.from_array(np.eye(1), one, one)
    C2 = ST.from_array(np.eye(1), one, one)
    C3 = ST.from_array(np.eye(1), one, one, signature=[True, False])
    C4 = ST.from_array(np.eye(1), one, one)
    s = A.signature
    r = A.col_reps
    T1 = ST.from_array(np.eye(A.shape[4])[None, :, :, None], one, (r[2], r[2], ST.singlet()),
                       signature=np.array([False, s[4], ~s[4], True]))
    T2 = ST.from_array(np.eye(A.shape[5])[None, None, :, :], one, (ST.singlet(), r[3], r[3]),
                       signature=np.array([True, False, s[5], ~s[5]]))
    T3 = ST.from_array(np.eye(A.shape[2])[:, :, None, None], (r[0], r[0], ST.singlet()), one,
                       signature=np.array([s[2], ~s[2], True, False]))
    T4 = ST.from_array(np.eye(A.shape[3])[None, :, :, None], one, (r[1], r[1], ST.singlet()),
                       signature=np.array([False, s[3], ~s[3], True]))
    return {"C1": C1, "C2": C2, "C3": C3, "C4": C4, "T1": T1, "T2": T2, "T3": T3, "T4": T4}


def parse_tiling(tiling):
    rows = [list(r.strip().replace(" ", "")) for r in tiling.strip().splitlines()]
    if any(len(r) != len(rows[0]) for r in rows):
        raise ValueError("tiling rows must have equal length")
    return np.array(rows, dtype="U1")


def unique_coords(cell):
    """Unique letters in order of appearance; site_coords[i] = (x, y) of the
    first occurrence; indices[x, y] = i (ctm_environment.py:37-59)."""
    letters = []
    for c in cell.flat:
        if c not in letters:
            letters.append(c)
    site_coords = np.empty((len(letters), 2), dtype=np.int8)
    indices_t = np.empty(cell.shape, dtype=int)
    for i, c in enumerate(letters):
        where = cell == c
        ys, xs = where.nonzero()
        site_coords[i] = xs[0], ys[0]
        indices_t[where] = i
    return site_coords, indices_t.T.copy()


class CTMEnvironment:
    def __init__(self, cell, As, envs):
        self._cell = cell
        self._site_coords, self._indices = unique_coords(cell)
        self._n_sites = self._site_coords.shape[0]
        self._Ly, self._Lx = cell.shape
        self._As = tuple(As)
        if len(self._As) != self._n_sites:
            raise ValueError("Incompatible cell and tensor number")
        self._t = {k: list(envs[k]) for k in _NAMES}
        self._symmetry = type(As[0]).symmetry()
        self._check()
        self.reset_constructed_corners()
        self._reset_temp()

    def _check(self):
        for x, y in self._site_coords:
            A = self.get_A(x, y)
            Ay = self.get_A(x, y - 1)
            if A.signature[2] == Ay.signature[4]:
                raise ValueError(f"signature mismatch between {(x, y)} and {(x, y - 1)}")
            if not np.array_equal(A.col_reps[0], Ay.col_reps[2]):
                raise ValueError(f"rep mismatch between {(x, y)} and {(x, y - 1)}")
            Ax = self.get_A(x + 1, y)
            if A.signature[3] == Ax.signature[5]:
                raise ValueError(f"signature mismatch between {(x + 1, y)} and {(x, y)}")
            if not np.array_equal(A.col_reps[1], Ax.col_reps[3]):
                raise ValueError(f"rep mismatch between {(x + 1, y)} and {(x, y)}")

    @classmethod
    def from_elementary_tensors(cls, tiling, tensors):
        cell = parse_tiling(tiling)
        if len(tensors) != len(set(cell.flat)):
            raise ValueError("Incompatible cell and tensor number")
        envs = {k: [] for k in _NAMES}
        for A in tensors:
            d = initialize_dummy_env(A)
            for k in _NAMES:
                envs[k].append(d[k])
        return cls(cell, tensors, envs)

    def copy(self):
        """Independent environment: every tensor's blocks are copied."""
        envs = {k: [t.copy() for t in self._t[k]] for k in _NAMES}
        return type(self)(self._cell, self._As, envs)

    def set_tensors(self, tensors):
        """New elementary tensors with the same representations; the environment
        is kept and the enlarged corners are reset (ctm_environment.py:299-312)."""
        if len(tensors) != self._n_sites:
            raise ValueError("Incompatible cell and tensors")
        for i, A in enumerate(tensors):
            if not A.match_representations(self._As[i]):
                raise ValueError("Incompatible representation for new tensor")
        self._As = tuple(tensors)
        self.reset_constructed_corners()

    def tensors(self, name):
        return list(self._t[name])

    # ------------------------------------------------------------ accessors
    def _index(self, x, y):
        return self._indices[x % self._Lx, y % self._Ly]

    def get(self, name, x, y):
        return self._t[name][self._index(x, y)]

    def get_A(self, x, y):
        return self._As[self._index(x, y)]

    def get_C1(self, x, y):
        return self.get("C1", x, y)

    def get_C2(self, x, y):
        return self.get("C2", x, y)

    def get_C3(self, x, y):
        return self.get("C3", x, y)

    def get_C4(self, x, y):
        return self.get("C4", x, y)

    def get_T1(self, x, y):
        return self.get("T1", x, y)

    def get_T2(self, x, y):
        return self.get("T2", x, y)

    def get_T3(self, x, y):
        return self.get("T3", x, y)

    def get_T4(self, x, y):
        return self.get("T4", x, y)

    @property
    def Lx(self):
        return self._Lx

    @property
    def Ly(self):
        return self._Ly

    @property
    def cell(self):
        return self._cell

    @property
    def n_sites(self):
        return self._n_sites

    @property
    def site_coords(self):
        return self._site_coords

    @property
    def elementary_tensors(self):
        return self._As

    @property
    def Dmax(self):
        return max(max(A.shape[2:]) for A in self._As)

    @property
    def Dmin(self):
        return min(min(A.shape[2:]) for A in self._As)

    @property
    def chi_values(self):
        s = set()
        for C in self._t["C1"] + self._t["C3"]:
            s.update(C.shape)
        return sorted(s)

    def symmetry(self):
        return self._symmetry

    # ------------------------------------------------------ enlarged corners
    def reset_constructed_corners(self):
        self._corners = {k: [None] * self._n_sites for k in ("ul", "ur", "dl", "dr")}

    def get_corner(self, kind, x, y):
        return self._corners[kind][self._index(x, y)]

    def set_corner(self, kind, x, y, value):
        self._corners[kind][self._index(x, y)] = value

    # --------------------------------------------------- projectors and moves
    def _reset_temp(self):
        self._proj = {}
        self._new = [None] * self._n_sites

    def store_projectors(self, direction, x, y, P, Pt):
        self._proj[(direction, self._index(x, y))] = (P, Pt)

    def get_P(self, direction, x, y):
        return self._proj[(direction, self._index(x, y))][0]

    def get_Pt(self, direction, x, y):
        return self._proj[(direction, self._index(x, y))][1]

    def store_renormalized(self, x, y, triple):
        self._new[self._index(x, y)] = triple

    def commit(self, names):
        """Replace (corner, edge, corner) of every unique site by the
        renormalised tensors; all are computed before any is stored, since a
        move reads C[x, y] while writing C[x, y + 1]."""
        for k, name in enumerate(names):
            self._t[name] = [t[k] for t in self._new]
        self._reset_temp()

    # ------------------------------------------------------------------- I/O
    def get_data_dic(self):
        data = {"_CTM_cell": self._cell, "_CTM_symmetry": self._symmetry}
        for i in range(self._n_sites):
            data |= self._As[i].get_data_dic(prefix=f"_CTM_A_{i}")
            for k in _NAMES:
                data |= self._t[k][i].get_data_dic(prefix=f"_CTM_{k}_{i}")
        return data

    @classmethod
    def load_from_file(cls, savefile):
        with np.load(savefile) as data:
            cell = data["_CTM_cell"]
            ST = get_symmetric_tensor_type(data["_CTM_symmetry"][()])
            n = len(set(cell.flat))
            As = [ST.load_from_dic(data, prefix=f"_CTM_A_{i}") for i in range(n)]
            envs = {k: [ST.load_from_dic(data, prefix=f"_CTM_{k}_{i}") for i in range(n)]
                    for k in _NAMES}
        return cls(cell, As, envs)
