"""Anderson acceleration with a QR-updated least-squares problem (TEST ORACLE).

Restates ``aasol`` of the reference, src/utils/anderson.jl:301-443, with its
helpers ``aa_point!`` (:470-481), ``betafix!`` (:488-491), ``BuildDG!``
(:450-461), ``aa_qr_update!`` (:498-512), ``Orthogonalize!`` CGS2 (:525-540),
``update_aaqr!`` (:542-550), ``downdate_aaqr!`` (:552-583) and ``AndersonOK``
(:727-737).  Pinned against the Toth--Kelley histories of :116-160.

Only the large-storage layout (Vstore with >= 3m+3 columns) is restated; the
low-storage block path of ``downdate_aaqr!`` computes the same product.
"""
import numpy as np
import scipy.linalg


class AASolResult:
    def __init__(self, solution, functionval, history, condhist, alphanorm, idid, errcode):
        self.solution = solution
        self.functionval = functionval
        self.history = history
        self.condhist = condhist
        self.alphanorm = alphanorm
        self.idid = idid
        self.errcode = errcode


def _betafix(gx, sol, beta):
    # anderson.jl:488-491: gx <- (1-beta)*sol + beta*gx
    return (1.0 - beta) * sol + beta * gx


def _householder_qr(A):
    """Thin QR of A (m x n, m >= n) with LAPACK's dlarfg sign convention.

    Equivalent to Julia's ``qr!`` + ``Matrix(G.Q)`` / ``Matrix(G.R)`` used by
    downdate_aaqr! (anderson.jl:557-559).
    """
    A = np.array(A, dtype=np.float64, copy=True)
    m, n = A.shape
    taus = np.zeros(n)
    vs = []
    for j in range(n):
        x = A[j:, j].copy()
        alpha = x[0]
        xnorm = np.linalg.norm(x[1:]) if m - j > 1 else 0.0
        if xnorm == 0.0:
            tau = 0.0
            v = np.zeros_like(x)
            v[0] = 1.0
        else:
            beta = -np.copysign(np.hypot(alpha, xnorm), alpha)
            tau = (beta - alpha) / beta
            v = x * (1.0 / (alpha - beta))   # dlarfg scales by the reciprocal
            v[0] = 1.0
            A[j, j] = beta
            A[j + 1:, j] = 0.0
            # apply H = I - tau v v^T to the trailing columns
            if j + 1 < n:
                w = v @ A[j:, j + 1:]
                A[j:, j + 1:] -= tau * np.outer(v, w)
        taus[j] = tau
        vs.append(v)
    R = np.triu(A[:n, :n])
    # form thin Q by applying the reflectors to the first n columns of I
    Q = np.zeros((m, n))
    Q[:n, :n] = np.eye(n)
    for j in range(n - 1, -1, -1):
        v = vs[j]
        w = v @ Q[j:, :]
        Q[j:, :] -= taus[j] * np.outer(v, w)
    return Q, R


def _gemv_sub(y, A, x):
    """y - A x accumulated column by column, as BLAS gemv with alpha=-1, beta=1."""
    y = y.copy()
    for j in range(A.shape[1]):
        y += (-x[j]) * A[:, j]
    return y


def _orthogonalize(Qkm, vnew):
    """CGS2 of anderson.jl:525-540; returns (hv, vnew_normalized)."""
    k = Qkm.shape[1]
    hv = np.zeros(k + 1)
    if k > 0:
        h1 = Qkm.T @ vnew
        vnew = _gemv_sub(vnew, Qkm, h1)
        h2 = Qkm.T @ vnew
        vnew = _gemv_sub(vnew, Qkm, h2)
        hv[:k] = h1 + h2
    hv[k] = np.linalg.norm(vnew)
    vnew = vnew / hv[k]
    return hv, vnew


def _aa_qr_update(Q, R, vnew, m, k):
    """anderson.jl:498-512 (in place on Q, R)."""
    if k == 0:
        nrm = np.linalg.norm(vnew)
        R[0, 0] = nrm
        Q[:, 0] = vnew / nrm
    else:
        if k > m - 1:
            # downdate_aaqr!, anderson.jl:552-583
            Rp = R[:, 1:m].copy()
            Qx, Rd = _householder_qr(Rp)
            R[: m - 1, : m - 1] = Rd
            R[:, m - 1] = 0.0
            Q[:, : m - 1] = Q @ Qx
            Q[:, m - 1] = 0.0
        kq = min(k, m - 1)
        hv, qn = _orthogonalize(Q[:, :kq], vnew.copy())
        R[: kq + 1, kq] = hv
        Q[:, kq] = qn


def _solve_R(RA, tres):
    # Julia's `\` on a square matrix takes the triangular path when the matrix is
    # upper triangular (the Anderson R always is, see downdate analysis in the
    # module docstring of the CUDA Anderson kernels) and LU otherwise.
    if np.allclose(np.tril(RA, -1), 0.0, atol=0.0):
        return scipy.linalg.solve_triangular(RA, tres, lower=False)
    return np.linalg.solve(RA, tres)


def aasol(gfix, x0, m, maxit=20, rtol=1e-10, atol=1e-10, beta=1.0,
          picard_maxit=0, picard_beta=1.0, picard_rtol=1e-2, picard_atol=1e-2,
          callback=None):
    """Restatement of aasol(GFix!, x0, method) (anderson.jl:301-443).

    ``gfix(x) -> G(x)`` returns a new array.  ``callback(phase, k, resnorm)``
    is called after every evaluation (used by tests to compare histories).
    """
    if not (0 < abs(beta) <= 1):
        raise ValueError("abs(beta) must be in (0,1]")
    n = x0.size
    sol = np.array(x0, dtype=np.float64, copy=True).ravel()
    k = 0
    gx = gfix(sol).ravel().astype(np.float64)
    if beta != 1:
        gx = _betafix(gx, sol, beta)
    res = gx - sol
    resnorm = np.linalg.norm(res)
    resnorm_up_bd = 1.0e4 * resnorm
    tol = rtol * resnorm + atol
    picard_tol = picard_rtol * resnorm + picard_atol
    history = [resnorm]
    condhist, alphanorm = [], []
    toosoon = resnorm <= tol
    if callback:
        callback("init", 0, resnorm)

    if (not toosoon) and picard_maxit > 0:
        sol = gx.copy()
        for _ in range(picard_maxit - 1):
            gx = gfix(sol).ravel().astype(np.float64)
            if picard_beta != 1:
                gx = _betafix(gx, sol, picard_beta)
            res = gx - sol
            resnorm = np.linalg.norm(res)
            history.append(resnorm)
            if callback:
                callback("picard", k + 1, resnorm)
            if resnorm <= picard_tol or resnorm >= resnorm_up_bd:
                break
            sol = gx.copy()
        toosoon = resnorm <= tol

    Q = np.zeros((n, max(m, 1)))
    R = np.zeros((max(m, 1), max(m, 1)))
    DG = np.zeros((n, max(m, 1)))
    dg = np.zeros(n)
    df = np.zeros(n)

    def aa_point(gx, sol, res):
        dg = -gx
        gnew = gfix(sol).ravel().astype(np.float64)
        if beta != 1:
            gnew = _betafix(gnew, sol, beta)
        dg = dg + gnew
        df = -res
        res = gnew - sol
        df = df + res
        return gnew, dg, df, res, np.linalg.norm(res)

    if not toosoon:
        sol = gx.copy()
        k += 1
        gx, dg, df, res, resnorm = aa_point(gx, sol, res)
        history.append(resnorm)
        if callback:
            callback("anderson", k, resnorm)

    while (k < maxit + picard_maxit) and (resnorm > tol) and (not toosoon) and (resnorm < resnorm_up_bd):
        if m == 0:
            alphanrm, condit = 1.0, 1.0
            sol = gx.copy()
        else:
            # BuildDG!(DG, m, k+1, dg), anderson.jl:450-461
            kk = k + 1
            if m == 1:
                DG[:, 0] = dg
            elif kk > m + 1:
                DG[:, : m - 1] = DG[:, 1:m].copy()
                DG[:, m - 1] = dg
            else:
                DG[:, kk - 2] = dg
            _aa_qr_update(Q, R, df.copy(), m, k - 1)
            mk = min(m, k)
            QA = Q[:, :mk]
            RA = R[:mk, :mk]
            tres = QA.T @ res
            theta = _solve_R(RA, tres)
            condit = np.linalg.cond(RA)
            alpha = np.zeros(mk + 1)
            alpha[0] = theta[0]
            for ia in range(1, mk):
                alpha[ia] = theta[ia] - theta[ia - 1]
            alpha[mk] = 1 - theta[mk - 1]
            alphanrm = np.sum(np.abs(alpha))
            sol = _gemv_sub(gx, DG[:, :mk], theta)
        condhist.append(condit)
        alphanorm.append(alphanrm)
        k += 1
        gx, dg, df, res, resnorm = aa_point(gx, sol, res)
        history.append(resnorm)
        if callback:
            callback("anderson", k, resnorm)

    # AndersonOK, anderson.jl:727-737
    if toosoon:
        idid, errcode = True, -1
    elif resnorm >= resnorm_up_bd:
        idid, errcode = False, -2
    elif resnorm <= tol:
        idid, errcode = True, 0
    else:
        idid, errcode = False, 10
    return AASolResult(sol, gx, np.array(history), np.array(condhist), np.array(alphanorm), idid, errcode)
