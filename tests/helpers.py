"""Shared test helpers: tolerances, error metrics and a SOL 105 consumer.

The consumer restates, for tests only, what the reference does with the
assembled matrices (src/solver/boundary_conditions.jl:457-528 free dofs,
src/solver/solve_case.jl:845-871 static solve, :1905-2052 buckling):
remove SPC and dependent (MPC) dofs, solve K_ff u_f = F_f, recover the
dependent dofs from their independent images, assemble KG from u, and solve
K_ff phi = lambda (-Kg_ff) phi with a shift-invert Lanczos (scipy eigsh).
"""
import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as sla

ROW_TOL = 1e-12      # |K_gpu - K_oracle| per nonzero / max |K| of its row (the parity bound)
LAMBDA_TOL = 1e-9    # relative, first buckling load factors


def rowmax_rel_err(colptr, ref, got):
    """Max over nonzeros of |got - ref| / max|ref| of the same column (== row, symmetric)."""
    n = len(colptr) - 1
    starts = colptr[:-1] - 1
    lens = np.diff(colptr)
    col = np.repeat(np.arange(n), lens)
    absref = np.abs(ref)
    colmax = np.zeros(n)
    np.maximum.at(colmax, col, absref)
    colmax[colmax == 0] = 1.0
    return float((np.abs(got - ref) / colmax[col]).max()) if len(ref) else 0.0


def to_csc(colptr, rowval, nzval, n):
    return sp.csc_matrix((nzval, rowval - 1, colptr - 1), shape=(n, n))


def free_dofs(model, dep_dofs_1based, K):
    n = model.ndof
    mask = np.ones(n, bool)
    if model.spc_dofs is not None:
        mask[model.spc_dofs] = False
    if len(dep_dofs_1based):
        mask[np.asarray(dep_dofs_1based) - 1] = False
    diag = K.diagonal()
    mask &= np.abs(diag) > 0.0   # AUTOSPC of empty rows (e.g. the RBE2 centre node's unused dofs)
    return np.nonzero(mask)[0]


def static_solution(model, K, cmap):
    dep, ptr, ind, coef = cmap
    free = free_dofs(model, dep, K)
    Kf = K[free][:, free].tocsc()
    u = np.zeros(model.ndof)
    u[free] = sla.spsolve(Kf, model.force[free])
    for i, d in enumerate(dep):
        u[d - 1] = sum(coef[t] * u[ind[t] - 1] for t in range(ptr[i], ptr[i + 1]))
    return u, free


def load_factors(K, KG, free, k=5, sigma=None):
    """Smallest positive buckling load factors of K phi = lambda (-KG) phi.

    Solved as the definite problem (-KG) phi = mu K phi (K_ff positive
    definite), lambda = 1 / mu for the largest positive mu.
    """
    del sigma
    Kf = K[free][:, free].tocsc()
    Gf = KG[free][:, free].tocsc()
    Kf = 0.5 * (Kf + Kf.T)
    Gf = 0.5 * (Gf + Gf.T)
    v0 = np.ones(Kf.shape[0])
    mu = sla.eigsh(-Gf, k=k, M=Kf, which="LA", return_eigenvectors=False, tol=1e-15, v0=v0, ncv=max(4 * k, 40))
    mu = np.sort(mu[mu > 0])[::-1]
    return 1.0 / mu
