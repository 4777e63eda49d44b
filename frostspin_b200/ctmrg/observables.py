"""Transfer-matrix spectrum of a CTMRG environment (correlation lengths).

Restates frostspin/ctmrg/observables.py:4-154.  The transfer operator adds one
row of edge tensors (and optionally of site tensors) to a left edge state; its
action is a chain of device permutes and grouped GEMMs, and its leading
eigenvalues come from SymmetricTensor.eigs (dense sector eig on the device for
small sectors, ARPACK with device matvecs for large ones).
"""

import numpy as np


def compute_mps_transfer_spectrum(T1s, T3s, nvals, *, A_list=None, dmax_full=200, rng=None,
                                  maxiter=4000, arpack_tol=0, verbosity=0):
    """observables.py:4-154.  T1s / T3s: top and bottom edge tensors of one cell
    row, from right to left (leg order 3-Tup-0 with 1, 2 down; 3-Tdown-2 with
    0, 1 up).  Returns the nvals largest eigenvalues by magnitude, normalised by
    the first (real when their imaginary parts are negligible)."""
    ST = type(T1s[0])
    Ts_up = [T.permute((3, 1, 2), (0,)) for T in T1s]
    Ts_down = [T.permute((3,), (2, 0, 1)) for T in T3s]
    if A_list is None:
        reps = (Ts_up[0].col_reps[0], Ts_down[0].col_reps[0])
        sig0 = np.array([~Ts_up[0].signature[3], ~Ts_down[0].signature[1]], dtype=bool)

        def matmat(st0):
            st = st0.permute((0,), (1, 2))
            for mu, md in zip(Ts_up, Ts_down, strict=True):
                st = mu @ st
                st = st.permute((3, 1, 2), (0, 4))
                st = md @ st
                st = st.permute((1,), (0, 2))
            return st.permute((0, 1), (2,))

    else:
        As = [A.permute((0, 1, 4, 5), (3, 2)) for A in A_list]
        Acs = [A.dagger().permute((2, 3), (4, 5, 1, 0)) for A in A_list]
        reps = (Ts_up[0].col_reps[0], As[0].col_reps[0], Acs[0].col_reps[2],
                Ts_down[0].col_reps[0])
        sig0 = np.array([~Ts_up[0].signature[3], ~As[0].signature[4], ~Acs[0].signature[4],
                         ~Ts_down[0].signature[1]], dtype=bool)

        def matmat(st0):
            st = st0.permute((0,), (1, 2, 3, 4))
            for mu, md, A, Ac in zip(Ts_up, Ts_down, As, Acs, strict=True):
                st = mu @ st
                st = st.permute((3, 1), (0, 2, 4, 5, 6))
                st = A @ st
                st = st.permute((0, 1, 6, 5), (2, 3, 4, 7, 8))
                st = Ac @ st
                st = st.permute((5, 2, 0), (1, 3, 4, 6))
                st = md @ st
                st = st.permute((3,), (2, 1, 0, 4))
            return st.permute((0, 1, 2, 3), (4,))

    try:
        vals = ST.eigs(matmat, nvals, reps, sig0, dmax_full=dmax_full, rng=rng,
                       maxiter=maxiter, arpack_tol=arpack_tol)
    except Exception as err:  # the reference also returns NaNs on failure (:138-141)
        if verbosity > 0:
            print("WARNING: transfer matrix spectrum computation failed:", err)
        return np.nan * np.ones((nvals,))
    sortperm = np.abs(vals).argsort()[: -nvals - 1 : -1]
    vals = vals[sortperm]
    vals = vals / vals[0]
    if np.iscomplexobj(vals) and np.linalg.norm(vals.imag) < 1e-6:
        vals = vals.real
    elif np.iscomplexobj(vals) and verbosity > 0:
        print("Info: CTMRG transfer matrix eigenvalues are not real")
    return vals
