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
# Where an entry sums terms far larger than its row's max (the rows of an RBE2
# master, whose images carry lever arms of metres), its value is fixed only to
# a few eps * sum|terms| by ANY summation order: the reference iterates its
# elements in Dict order, and the oracle reordered against itself already
# differs by up to 7 eps * sum|terms| there (tests/test_oracle.py).  The bound
# per entry is therefore max(ROW_TOL * rowmax, SUM_TOL * eps * sum|terms|); it
# equals ROW_TOL * rowmax wherever sum|terms| < ~280 rowmax.
SUM_TOL = 16.0
EPS = 2.0 ** -52


def rowmax_rel_err(colptr, ref, got):
    """Max over nonzeros of |got - ref| / max|ref| of the same column (== row, symmetric)."""
    if not len(ref):
        return 0.0
    cm = _colmax_per_entry(colptr, ref)
    cm[cm == 0] = 1.0
    return float((np.abs(got - ref) / cm).max())


def _colmax_per_entry(colptr, ref):
    """max|ref| of each stored entry's column, expanded to one value per entry."""
    lens = np.diff(colptr)
    starts = colptr[:-1] - 1
    nonempty = lens > 0
    colmax = np.zeros(len(lens))
    colmax[nonempty] = np.maximum.reduceat(np.abs(ref), starts[nonempty])
    return np.repeat(colmax, lens)


def parity_ratio(colptr, ref, got, abs_sums):
    """Max over nonzeros of |got - ref| / max(ROW_TOL * rowmax, SUM_TOL * EPS * sum|terms|).

    abs_sums is the oracle's per-entry sum of |term| (oracle.assemble_k with
    abs_sums=True).  A value <= 1 passes the parity bound."""
    if not len(ref):
        return 0.0
    bound = np.maximum(ROW_TOL * _colmax_per_entry(colptr, ref), SUM_TOL * EPS * abs_sums)
    bound[bound == 0] = ROW_TOL
    return float((np.abs(got - ref) / bound).max())


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
