"""CPU oracle for the expm(-iHt) hot path.

TEST INFRASTRUCTURE ONLY.  Only ``tests/``, ``__graft_entry__.smoke()`` and the
``cpu_baseline`` / ``--impl reference`` legs of ``bench.py`` may import this module, and
only as the checker or the timed CPU baseline.  The product path (``fastctqw_b200``) never
imports it and has no CPU fallback.

What it restates
----------------
The reference's runnable path is ``Operator.buildExpmOperator`` with ``device="cpu"``
(FastCTQW/Operator.py:70-78), which calls ``scipy.linalg.expm`` on ``X = -1j*H*t``
(FastCTQW/Operator.py:55-56, :76).  The arithmetic lives in the third-party dependency
scipy (pinned here at 1.18.1; the reference asks for ``scipy>=1.14``, pyproject.toml:30),
whose dense ``expm`` is compiled.  Its algorithm of record is Al-Mohy & Higham, "A New
Scaling and Squaring Algorithm for the Matrix Exponential", SIAM J. Matrix Anal. Appl.
31(3), 2009, with the Higham & Tisseur (2000) block 1-norm estimator.  This module
restates that published algorithm in FP64 numpy, following the step structure of the
pure-Python statement of the same algorithm that scipy ships in
``scipy/sparse/linalg/_matfuncs.py`` (selection ``_expm`` :593-680, Pade-13 ``pade13_scaled``
:522-541, ``_solve_P_Q`` :683-712, ``_ell`` :819-862).

Deliberate, documented differences from scipy (the device pipeline makes the same choices,
so that (m, s) can be compared one to one):
  * d4 and d6 are always exact (the device materialises A^4 and A^6 anyway); d8 and d10
    use a deterministic block 1-norm estimate (t = 2, fixed +-1 second column) instead of
    scipy's randomised one.
  * optional preprocessing shifts (trace shift, Higham 2005 sec. 2; and the rank-one
    "commuting shift" along the all-ones vector when every row sum and column sum of A is
    the same number).  Both are exact identities of the exponential.

Parity is pinned (see tests/test_oracle.py): against scipy.linalg.expm in FP64 on the
golden fixtures generated from the reference's own CPU path (tests/golden/), against the
FP64 eigendecomposition propagator V exp(-i L t) V^T, and against scipy's own known-answer
tests for expm, run with this oracle substituted.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

# Al-Mohy & Higham (2009), Table 3.1 / Algorithm 6.1: largest 2^-s-scaled norm for which
# the Pade degree m meets double-precision backward error (theta_13 = 4.25 in the 2009
# algorithm).  Same numbers as scipy/sparse/linalg/_matfuncs.py:644-662.
THETA = {3: 1.495585217958292e-2, 5: 2.539398330063230e-1, 7: 9.504178996162932e-1,
         9: 2.097847961257068e0, 13: 4.25}
PADE_DEGREES = (3, 5, 7, 9, 13)
# Matrix products needed to evaluate the [m/m] Pade numerator/denominator pair.
PADE_PRODUCTS = {3: 2, 5: 3, 7: 4, 9: 5, 13: 6}
UNIT_ROUNDOFF = 2.0 ** -53


def pade_coefficients(m: int) -> list[float]:
    """Coefficients b_0..b_m of the [m/m] Pade approximant to exp, scaled so b_m = 1.

    b_j = (2m - j)! / (j! (m - j)!)  (Higham 2005, eq. 2.1 up to a common factor).  For
    m = 13 this gives 64764752532480000, ..., 182, 1 (scipy/sparse/linalg/_matfuncs.py:524).
    """
    f = math.factorial
    return [float(f(2 * m - j) // (f(j) * f(m - j))) for j in range(m + 1)]


def ell_constant(m: int) -> float:
    """1/|c_{2m+1}|, c_{2m+1} = (-1)^m (m!)^2 / ((2m)! (2m+1)!): the leading coefficient of
    the Pade error series exp(x) - r_m(x) (Al-Mohy & Higham 2009, eq. 5.2; the table of
    these values is scipy/sparse/linalg/_matfuncs.py:840-845)."""
    f = math.factorial
    return float(f(2 * m) * f(2 * m + 1) // (f(m) ** 2))


def onenorm(A: np.ndarray) -> float:
    """Exact induced 1-norm: max column sum of |A|."""
    if A.size == 0:
        return 0.0
    return float(np.abs(A).sum(axis=0).max())


def second_probe_sign(n: int) -> np.ndarray:
    """Deterministic +-1 column used as the second probe of the t=2 block estimator.

    sign_i = +1 when bit 31 of (i * 0x9E3779B1 mod 2^32) is clear, else -1.  The device
    estimator builds the same column.
    """
    i = np.arange(n, dtype=np.uint64)
    h = (i * np.uint64(0x9E3779B1)) & np.uint64(0xFFFFFFFF)
    return np.where((h >> np.uint64(31)) & np.uint64(1), -1.0, 1.0)


def normest1(apply, apply_h, n: int, itmax: int = 5) -> float:
    """Deterministic Higham-Tisseur block 1-norm estimate with t = 2 columns.

    ``apply(X)`` returns A @ X and ``apply_h(S)`` returns A^H @ S for (n, 2) blocks.  This
    follows Higham & Tisseur (2000), Algorithm 2.4, minus the random resampling of
    parallel sign columns: the first probe is ones/n, the second the fixed +-1/n column
    from :func:`second_probe_sign`; each round moves to the unit vectors of the two largest
    entries of max_j |(A^H S)_ij| not visited before.  Returns a lower bound of ||A||_1.
    """
    if n == 0:
        return 0.0
    t = 2 if n > 1 else 1
    X = np.ones((n, t), dtype=np.complex128) / n
    if t == 2:
        X[:, 1] = second_probe_sign(n) / n
    est_old = 0.0
    visited: set[int] = set()
    ind_best = 0
    for k in range(1, itmax + 1):
        Y = apply(X)
        col = np.abs(Y).sum(axis=0)
        j = int(np.argmax(col))
        est = float(col[j])
        if k >= 2 and est <= est_old:
            return est_old
        est_old = est
        if k == itmax:
            break
        absY = np.abs(Y)
        S = np.where(absY > 0, Y / np.where(absY > 0, absY, 1.0), 1.0)
        Z = apply_h(S)
        h = np.abs(Z).max(axis=1)
        if k >= 2 and h.max() <= h[ind_best]:
            break
        order = np.argsort(-h, kind="stable")
        picks = [int(i) for i in order if int(i) not in visited][:t]
        if len(picks) < t:
            break
        ind_best = picks[0]
        visited.update(picks)
        X = np.zeros((n, t), dtype=np.complex128)
        for c, i in enumerate(picks):
            X[i, c] = 1.0
    return est_old


def normest_product(mats: list[np.ndarray]) -> float:
    """Estimate ||M_1 M_2 ... M_k||_1 without forming the product."""
    n = mats[0].shape[0]

    def apply(X):
        for M in reversed(mats):
            X = M @ X
        return X

    def apply_h(S):
        for M in mats:
            S = M.conj().T @ S
        return S

    return normest1(apply, apply_h, n)


def abs_power_onenorm(A: np.ndarray, p: int) -> float:
    """Exact ||(|A|)^p||_1 = max(1^T |A|^p) for the non-negative matrix |A|
    (scipy/sparse/linalg/_matfuncs.py:_onenorm_matrix_power_nnm)."""
    absA = np.abs(A)
    v = np.ones(A.shape[0])
    for _ in range(p):
        v = v @ absA
    return float(v.max()) if v.size else 0.0


def ell(A: np.ndarray, m: int, anorm: float | None = None,
        abs_pow_norm: float | None = None) -> int:
    """Backward-error correction l(A, m) of Al-Mohy & Higham (2009), eq. 5.3
    (scipy/sparse/linalg/_matfuncs.py:819-862)."""
    if abs_pow_norm is None:
        abs_pow_norm = abs_power_onenorm(A, 2 * m + 1)
    if abs_pow_norm == 0.0:
        return 0
    if anorm is None:
        anorm = onenorm(A)
    alpha = abs_pow_norm / (anorm * ell_constant(m))
    return max(int(math.ceil(math.log2(alpha / UNIT_ROUNDOFF) / (2 * m))), 0)


def ell_log2(log2_abs_pow_norm: float, log2_anorm: float, m: int, s: int) -> int:
    """l(2^-s A, m) from log2 ||(|A|)^(2m+1)||_1 and log2 ||A||_1.

    Scaling A by 2^-s scales the first norm by 2^-(2m+1)s and the second by 2^-s, so
    log2 alpha(2^-s A) = log2 alpha(A) - 2 m s.  This is how the device evaluates l without
    overflow (|A|^27 overflows FP32 for ||A|| of a few hundred).
    """
    if not math.isfinite(log2_abs_pow_norm):
        return 0
    log2_alpha = log2_abs_pow_norm - log2_anorm - math.log2(ell_constant(m)) - 2 * m * s
    return max(int(math.ceil((log2_alpha + 53.0) / (2 * m))), 0)


@dataclass
class Selection:
    """Pade degree m and squaring count s, plus the norms that decided them."""
    m: int
    s: int
    d: dict = field(default_factory=dict)


def is_skew_hermitian(A: np.ndarray) -> bool:
    """Exact test A^H == -A (then A, and every shift of it by i*real, is normal)."""
    return bool(np.array_equal(A.conj().T, -A))


def select_pade(A: np.ndarray, normal: bool = False) -> Selection:
    """Choose (m, s) by Al-Mohy & Higham (2009) Algorithm 6.1, in the order of
    scipy/sparse/linalg/_matfuncs.py:636-670 (exact d4/d6, estimated d8/d10).

    ``normal=True`` drops the l(A, m) correction.  l bounds the Pade backward error through
    ||(|A|)^(2m+1)||, which guards against non-normality; for a normal A the error of
    r_m(A) is max over the spectrum of |r_m(z) - e^z|, and every d_p bounds the spectral
    radius, so the theta_m test on the d_p alone is already rigorous.
    """
    n = A.shape[0]
    anorm = onenorm(A)
    A2 = A @ A
    A4 = A2 @ A2
    A6 = A4 @ A2
    d4 = onenorm(A4) ** 0.25
    d6 = onenorm(A6) ** (1.0 / 6.0)
    info = {"norm1": anorm, "d4": d4, "d6": d6}
    eta1 = max(d4, d6)
    def ell0(m):
        return True if normal else ell(A, m, anorm) == 0

    if eta1 < THETA[3] and ell0(3):
        return Selection(3, 0, info)
    eta2 = max(d4, d6)
    if eta2 < THETA[5] and ell0(5):
        return Selection(5, 0, info)
    d8 = normest_product([A4, A4]) ** 0.125 if n else 0.0
    info["d8"] = d8
    eta3 = max(d6, d8)
    if eta3 < THETA[7] and ell0(7):
        return Selection(7, 0, info)
    if eta3 < THETA[9] and ell0(9):
        return Selection(9, 0, info)
    d10 = normest_product([A4, A6]) ** 0.1 if n else 0.0
    info["d10"] = d10
    eta4 = max(d8, d10)
    eta5 = min(eta3, eta4)
    s = 0 if eta5 == 0 else max(int(math.ceil(math.log2(eta5 / THETA[13]))), 0)
    if normal:
        return Selection(13, s, info)
    apn = abs_power_onenorm(A, 27)
    info["abs27"] = apn
    if apn > 0 and anorm > 0:
        s += ell_log2(math.log2(apn), math.log2(anorm), 13, s)
    return Selection(13, s, info)


def pade_uv(A: np.ndarray, m: int, s: int = 0) -> tuple[np.ndarray, np.ndarray]:
    """Numerator-odd part U and even part V of r_m(2^-s A) = (V+U)/(V-U)
    (scipy/sparse/linalg/_matfuncs.py:488-541)."""
    n = A.shape[0]
    b = pade_coefficients(m)
    I = np.eye(n, dtype=A.dtype)
    B = A * 2.0 ** (-s)
    B2 = B @ B
    if m == 13:
        B4 = B2 @ B2
        B6 = B4 @ B2
        U = B @ (B6 @ (b[13] * B6 + b[11] * B4 + b[9] * B2)
                 + b[7] * B6 + b[5] * B4 + b[3] * B2 + b[1] * I)
        V = B6 @ (b[12] * B6 + b[10] * B4 + b[8] * B2) + b[6] * B6 + b[4] * B4 + b[2] * B2 + b[0] * I
        return U, V
    pw = [I, B2]
    for _ in range(2, m // 2 + 1):
        pw.append(pw[-1] @ B2)
    U = B @ sum(b[2 * k + 1] * pw[k] for k in range(m // 2 + 1))
    V = sum(b[2 * k] * pw[k] for k in range(m // 2 + 1))
    return U, V


def solve_pq(U: np.ndarray, V: np.ndarray) -> np.ndarray:
    """r_m = Q^-1 P with P = V + U, Q = V - U (scipy/sparse/linalg/_matfuncs.py:683-712)."""
    return np.linalg.solve(V - U, V + U)


@dataclass
class Shift:
    """Exact preprocessing: A = mu I + nu J/n + Y with J the all-ones matrix.

    ``nu`` is used only when every row sum and every column sum of A equal the same c
    (then J commutes with A and Y 1 = 0), giving exp(A) = e^mu (exp(Y) + (e^nu - 1) J/n).
    """
    mu: complex = 0.0
    nu: complex = 0.0
    rank1: bool = False


def common_line_sum(A: np.ndarray):
    """Return c (row 0's sum) if every row sum and column sum of A equals it within the
    rounding of a sum, 4 n 2^-53 max_i sum_j (|Re A_ij| + |Im A_ij|); else None.

    Exact equality of floating-point sums depends on the order of summation (row sums of a
    weighted regular graph with non-representable weights differ in the last bit), so the test
    is made at rounding level; the device makes the same test.
    """
    if A.shape[0] == 0:
        return None
    n = A.shape[0]
    A = A.astype(np.complex128)
    r = A.sum(axis=1)
    c = A.sum(axis=0)
    scale = float(np.max(np.abs(A.real).sum(axis=1) + np.abs(A.imag).sum(axis=1)))
    tol = 4.0 * n * 2.0 ** -53 * scale
    dev = max(np.max(np.abs(r.real - r[0].real)), np.max(np.abs(r.imag - r[0].imag)),
              np.max(np.abs(c.real - r[0].real)), np.max(np.abs(c.imag - r[0].imag)))
    if dev <= tol:
        return complex(r[0])
    return None


def preprocess(A: np.ndarray, mode: str = "auto") -> tuple[np.ndarray, Shift]:
    """Apply the exact shifts the device applies.  ``mode``: 'none', 'trace', 'auto'
    ('auto' = trace shift, plus the rank-one shift when the line sums are all equal)."""
    n = A.shape[0]
    A = A.astype(np.complex128)
    if mode == "none" or n == 0:
        return A, Shift()
    mu = complex(np.trace(A) / n)
    Y = A - mu * np.eye(n)
    sh = Shift(mu=mu)
    if mode == "auto":
        c = common_line_sum(A)
        if c is not None and n > 1:
            nu = c - mu
            Y = Y - (nu / n) * np.ones((n, n))
            sh.nu, sh.rank1 = nu, True
    return Y, sh


def postprocess(E: np.ndarray, sh: Shift) -> np.ndarray:
    """Undo :func:`preprocess`: exp(A) = e^mu (exp(Y) + (e^nu - 1) J / n)."""
    n = E.shape[0]
    if sh.rank1:
        E = E + (np.exp(sh.nu) - 1.0) / n
    return np.exp(sh.mu) * E


def expm(A: np.ndarray, shift: str = "none", return_selection: bool = False,
         structure: bool = False):
    """FP64 scaling-and-squaring Pade exponential (Al-Mohy & Higham 2009).

    ``shift``: 'none' (scipy's behaviour), 'trace' or 'auto' (see :func:`preprocess`).
    ``structure``: drop l(A, m) when the shifted matrix is exactly skew-Hermitian, as the
    device does (see :func:`select_pade`).
    """
    A = np.asarray(A)
    if A.ndim != 2 or A.shape[0] != A.shape[1]:
        raise ValueError("expected a square matrix")
    n = A.shape[0]
    real_in = not np.iscomplexobj(A)
    if n == 0:
        out = np.zeros((0, 0), dtype=np.float64 if real_in else np.complex128)
        return (out, Selection(3, 0)) if return_selection else out
    Y, sh = preprocess(A, shift)
    sel = select_pade(Y, normal=structure and is_skew_hermitian(Y))
    U, V = pade_uv(Y, sel.m, sel.s)
    R = solve_pq(U, V)
    for _ in range(sel.s):
        R = R @ R
    R = postprocess(R, sh)
    if real_in and shift == "none":
        R = R.real
    return (R, sel) if return_selection else R


def reference_cpu_expm(X: np.ndarray) -> np.ndarray:
    """The reference's CPU path itself: ``scipy.linalg.expm(X)`` exactly as
    ``Operator.buildExpmOperator`` calls it for device="cpu" (FastCTQW/Operator.py:74-76).
    Used as the timed CPU baseline; it runs in X's precision on all host BLAS threads."""
    import scipy.linalg
    return scipy.linalg.expm(X)


# ---------------------------------------------------------------- walk-level helpers

def build_hamiltonian(A: np.ndarray, gamma: float = 1.0, laplacian: bool = False,
                      dtype=np.complex128) -> np.ndarray:
    """H = -gamma A, or -gamma (D - A) (FastCTQW/Operator.py:49-53)."""
    if laplacian:
        return -gamma * np.asarray(np.diag(A.sum(axis=1)) - A, dtype=dtype)
    return -gamma * np.asarray(A, dtype=dtype)


def walk_generator(H: np.ndarray, t: float, dtype=np.complex128) -> np.ndarray:
    """X = -1j H t (FastCTQW/Operator.py:55-56)."""
    return np.asarray(-1j * H * t, dtype=dtype)


def propagator_eigh(H: np.ndarray, t: float) -> np.ndarray:
    """Exact FP64 propagator exp(-i H t) = V diag(e^{-i lambda t}) V^H for Hermitian H."""
    lam, Vec = np.linalg.eigh(np.asarray(H, dtype=np.complex128))
    return (Vec * np.exp(-1j * lam * t)) @ Vec.conj().T


def state_eigh(H: np.ndarray, t: float, psi0: np.ndarray) -> np.ndarray:
    """exp(-i H t) psi0 in FP64 from the eigendecomposition."""
    lam, Vec = np.linalg.eigh(np.asarray(H, dtype=np.complex128))
    return Vec @ (np.exp(-1j * lam * t) * (Vec.conj().T @ psi0.astype(np.complex128)))


def infidelity(psi: np.ndarray, psi_ref: np.ndarray) -> float:
    """1 - |<psi_ref|psi>|^2 with both states upcast to FP64 and normalised."""
    a = np.asarray(psi, dtype=np.complex128)
    b = np.asarray(psi_ref, dtype=np.complex128)
    na, nb = np.linalg.norm(a), np.linalg.norm(b)
    if na == 0 or nb == 0:
        return 1.0
    ov = np.vdot(b, a) / (na * nb)
    return float(max(0.0, 1.0 - abs(ov) ** 2))


def unitarity_residual(U: np.ndarray) -> float:
    """||U^H U - I||_F / sqrt(N) in FP64."""
    U = np.asarray(U, dtype=np.complex128)
    n = U.shape[0]
    if n == 0:
        return 0.0
    return float(np.linalg.norm(U.conj().T @ U - np.eye(n)) / math.sqrt(n))


def rel_error(U: np.ndarray, U_ref: np.ndarray) -> float:
    """||U - U_ref||_F / ||U_ref||_F in FP64."""
    d = np.linalg.norm(np.asarray(U, np.complex128) - np.asarray(U_ref, np.complex128))
    r = np.linalg.norm(np.asarray(U_ref, np.complex128))
    return float(d / r) if r > 0 else float(d)


def flops_expm(n: int, m: int, s: int) -> float:
    """Algorithmic real flops of one complex expm: 8n^3 (pi_m + s) + (8/3) n^3 + 8 n^3."""
    return 8.0 * n ** 3 * (PADE_PRODUCTS[m] + s) + (8.0 / 3.0) * n ** 3 + 8.0 * n ** 3


# ---------------------------------------------------------------- spectral radius (selection)

def tridiag_radius(alpha, beta) -> float:
    """Largest |eigenvalue| of the symmetric tridiagonal (alpha on the diagonal, beta beside it)
    by Sturm-sequence bisection inside the Gershgorin interval -- the step the engine runs on the
    host after its device Lanczos iterations (fx_batch.cu, tridiag_radius).  A zero beta_j ends
    the matrix after row j (the Krylov space ran out)."""
    a = [float(x) for x in alpha]
    b = [float(x) for x in beta]
    k = len(a)
    for j in range(k - 1):
        if not b[j] > 0.0:
            k = j + 1
            break
    a, b = a[:k], b[:k - 1]
    off = [(abs(b[i - 1]) if i > 0 else 0.0) + (abs(b[i]) if i + 1 < k else 0.0) for i in range(k)]
    lo = min(a[i] - off[i] for i in range(k))
    hi = max(a[i] + off[i] for i in range(k))

    def below(x):
        cnt, q = 0, 1.0
        for i in range(k):
            q = a[i] - x - (b[i - 1] ** 2 / q if i > 0 else 0.0)
            if q == 0.0:
                q = -1e-300
            cnt += q < 0.0
        return cnt

    def kth(want):
        x0, x1 = lo, hi
        for _ in range(200):
            if x1 - x0 <= 1e-14 * max(abs(x0), abs(x1)):
                break
            mid = 0.5 * (x0 + x1)
            if below(mid) >= want:
                x1 = mid
            else:
                x0 = mid
        return 0.5 * (x0 + x1)

    return max(abs(kth(1)), abs(kth(k)))


def lanczos_radius(B: np.ndarray, steps: int = 30, starts: int = 2, seed: int = 0) -> float:
    """Spectral-radius estimate of a real symmetric B: `starts` Lanczos runs of `steps` steps from
    random sign vectors, no reorthogonalisation, the largest radius of their tridiagonals (the
    algorithm of the engine's estimate; its Ritz values lie inside the spectrum)."""
    n = B.shape[0]
    rng = np.random.default_rng(seed)
    best = 0.0
    for _ in range(starts):
        v = rng.choice([-1.0, 1.0], n) / np.sqrt(n)
        vp = np.zeros(n)
        bprev = 0.0
        alpha, beta = [], []
        for _j in range(steps):
            t = B @ v
            a = float(t @ v)
            w = t - a * v - bprev * vp
            bb = float(np.linalg.norm(w))
            alpha.append(a)
            beta.append(bb)
            vp, v = v, (w / bb if bb > 1e-300 else np.zeros(n))
            bprev = bb
        best = max(best, tridiag_radius(alpha, beta[:-1]))
    return best
