"""CPU statement of the Chebyshev-Bessel approximant of the walk propagator.

TEST INFRASTRUCTURE ONLY.  Only ``tests/`` may import this module, as the checker of the
device pipeline's Chebyshev plan and of its arithmetic.  The product path
(``fastctqw_b200``) never imports it.

What it states
--------------
The reference computes ``U = expm(X)``, ``X = -iHt``, by scaling and squaring with Pade
approximants (FastCTQW/Operator.py:70-78; include/MatrixExpCalculator.h:52-68).  For walk
generators ``X = iB`` with ``B`` real symmetric the device pipeline can replace the Pade
stage and its solve by a polynomial: the Chebyshev expansion of ``e^{iaz}`` on ``[-1, 1]``
(Jacobi-Anger; Tal-Ezer & Kosloff, J. Chem. Phys. 81, 1984),

    e^{iaz} = J_0(a) + 2 sum_{k>=1} i^k J_k(a) T_k(z),

applied to ``Z = B / rho`` with ``rho`` an upper bound of the spectral radius of ``B`` and
``a = rho / 2^s``, then ``s`` squarings.  Truncated after degree ``D`` the error on the
spectrum is at most ``2 sum_{k>D} |J_k(a)|``, and ``2^s`` times that after the squarings.

The device evaluates the series with products of real symmetric commuting matrices only:
  * even part ``sum_j e_j T_j(C)`` with ``C = T_2(Z) = 2Z^2 - I`` (``T_2j(Z) = T_j(C)``),
  * odd part ``Z sum_j b_j T_j(C)`` (the odd coefficients moved onto ``Z T_j(C)`` with
    ``Z T_j(C) = (T_2j+1(Z) + T_2j-1(Z)) / 2``),
  * each part as ``sum_g T_g(G) r_g(C)`` with ``G = T_m(C)`` and ``deg r_g < m`` (baby steps
    ``T_1..T_m`` of ``C``), summed by Clenshaw's recurrence in ``G``.
This module restates every step of that plan in FP64 so that tests can check the device's
plan (``fx_chebyshev_plan``) one to one and the device's result against the same
arithmetic and against the FP64 eigendecomposition.
"""
from __future__ import annotations

import math

import numpy as np

# largest baby-step count of the device plan (arenas for T_1..T_m of C)
MAX_BABY = 5
# products of one squaring in the cost model of the plan
SQUARING_PRODUCTS = 3
# scalings that leave a above this are skipped (they would need hundreds of products)
MAX_A = 1024.0


def bessel_j(a: float, kmax: int) -> np.ndarray:
    """J_0(a) .. J_kmax(a) for a >= 0 by Miller's backward recurrence.

    J_{k-1} = (2k / a) J_k - J_{k+1} from a start far above max(kmax, a), normalised by
    J_0 + 2 sum_{k>=1} J_2k = 1 (Abramowitz & Stegun 9.1.27 and 9.1.46).
    """
    out = np.zeros(kmax + 1)
    if a == 0.0:
        out[0] = 1.0
        return out
    top = max(kmax, int(a)) + 20 + int(math.sqrt(40.0 * max(kmax, a)))
    top += top & 1
    jp, j = 0.0, 1e-300
    vals = np.zeros(top + 1)
    vals[top] = j
    norm = 0.0
    for k in range(top, 0, -1):
        jm = (2.0 * k / a) * j - jp
        jp, j = j, jm
        vals[k - 1] = j
        if abs(j) > 1e250:
            vals[k - 1:] *= 1e-250
            jp *= 1e-250
            j *= 1e-250
    norm = vals[0] + 2.0 * vals[2::2].sum()
    return vals[:kmax + 1] / norm


def degree(a: float, tol: float) -> int:
    """Smallest D with 2 sum_{k>D} |J_k(a)| <= tol."""
    kmax = int(a) + 40 + int(8.0 * max(a, 1.0) ** (1.0 / 3.0)) + 40
    j = np.abs(bessel_j(a, kmax))
    tail = np.cumsum(j[::-1])[::-1]   # tail[k] = sum_{i >= k} |J_i|
    for d in range(kmax):
        if 2.0 * tail[d + 1] <= tol:
            return d
    return kmax


def parts(D: int) -> tuple[int, int]:
    """Degrees in C of the even part and of the odd part's cofactor (-1: no odd part)."""
    je = D // 2
    jo = (D - 1) // 2 if D >= 1 else -1
    return je, jo


def chain_products(j: int, m: int) -> int:
    """Products of a Clenshaw chain of degree j in C with G = T_m(C): floor(j / m)."""
    return j // m if j >= 0 else 0


def baby_top(D: int, m: int) -> int:
    """Highest baby step T_k(C) the plan needs: T_m (= G) when a chain has a giant step,
    else the parts' own degree (their sums are then linear combinations of T_0..T_top)."""
    je, jo = parts(D)
    if D <= 1:
        return 0
    if je // m >= 1 or (jo >= 0 and jo // m >= 1):
        return m
    return max(je, jo)


def plan_cost(D: int, m: int) -> int:
    """Matrix products of the polynomial stage: baby steps T_2..T_top of C, both chains, and
    the product by Z of the odd chain (a multiple of I when its degree is 0: no product)."""
    je, jo = parts(D)
    if D <= 1:
        return 0
    return max(baby_top(D, m) - 1, 0) + chain_products(je, m) + (chain_products(jo, m) + 1 if jo >= 1 else 0)


def best_baby(D: int) -> tuple[int, int]:
    """(cost, m) minimising plan_cost over m = 1..MAX_BABY (ties to the smaller m)."""
    best = None
    for m in range(1, MAX_BABY + 1):
        c = plan_cost(D, m)
        if best is None or c < best[0]:
            best = (c, m)
    return best


def plan(rho: float, tol: float = 1e-6, smax: int = 60) -> dict:
    """The cheapest (s, D, m) for a spectral bound rho: products of the polynomial stage plus
    SQUARING_PRODUCTS per squaring, the error 2^s * 2 sum_{k>D} |J_k(rho / 2^s)| <= tol; ties
    to the smaller s."""
    best = None
    for s in range(smax + 1):
        a = math.ldexp(rho, -s)
        if a > MAX_A:
            continue
        D = degree(a, math.ldexp(tol, -s))
        c, m = best_baby(D)
        tot = c + SQUARING_PRODUCTS * s
        if best is None or tot < best["cost"]:
            best = {"s": s, "degree": D, "baby": m, "cost": tot, "a": a}
        if a < 1e-3:
            break
    return best


def split_coefficients(a: float, D: int) -> tuple[np.ndarray, np.ndarray]:
    """(e, b): e_j of the even part sum_j e_j T_j(C), b_j of the odd part Z sum_j b_j T_j(C)."""
    J = bessel_j(a, max(D, 1))
    je, jo = parts(D)
    e = np.array([J[0]] + [2.0 * (-1) ** j * J[2 * j] for j in range(1, je + 1)])
    if jo < 0:
        return e, np.zeros(0)
    o = np.array([2.0 * (-1) ** k * J[2 * k + 1] for k in range(jo + 1)])
    b = np.zeros(jo + 2)
    for k in range(jo, 0, -1):
        b[k] = 2.0 * o[k] - b[k + 1]
    b[0] = o[0] - 0.5 * b[1]
    return e, b[:jo + 1]


def blocks(x: np.ndarray, m: int) -> np.ndarray:
    """r[g, j] with sum_k x_k T_k(C) = sum_g T_g(T_m(C)) sum_{j<m} r[g, j] T_j(C).

    T_gm T_j = (T_gm+j + T_gm-j) / 2 for g, j >= 1, so from the top degree down:
    r[g, j] = 2 x_k and x_{gm-j} -= x_k (g, j >= 1), r[g, j] = x_k otherwise.
    """
    x = np.array(x, dtype=np.float64)
    L = (len(x) - 1) // m
    r = np.zeros((L + 1, m))
    for k in range(len(x) - 1, -1, -1):
        g, j = divmod(k, m)
        if g == 0 or j == 0:
            r[g, j] = x[k]
        else:
            r[g, j] = 2.0 * x[k]
            x[g * m - j] -= x[k]
    return r


def baby_steps(C: np.ndarray, top: int) -> list[np.ndarray]:
    """[I, T_1(C), .., T_top(C)] by T_k = 2 T_i T_j - T_(j-i), (i, j) = (1, 1), (1, 2), (2, 2),
    (2, 3) for k = 2..5: T_2 = 2C^2 - I, T_3 = 2 C T_2 - C, T_4 = 2 T_2^2 - I, T_5 = 2 T_2 T_3 - C."""
    n = C.shape[0]
    T = [np.eye(n), C]
    pairs = {2: (1, 1), 3: (1, 2), 4: (2, 2), 5: (2, 3)}
    for k in range(2, top + 1):
        i, j = pairs[k]
        T.append(2.0 * T[i] @ T[j] - T[j - i])
    return T


def clenshaw(r: np.ndarray, T: list[np.ndarray], m: int) -> np.ndarray:
    """sum_g T_g(G) r_g(C) with G = T_m(C): b_g = r_g + 2 G b_{g+1} - b_{g+2}, result
    r_0 + G b_1 - b_2."""
    L = r.shape[0] - 1

    def rg(g):
        return sum(r[g, j] * T[j] for j in range(min(m, len(T))) if r[g, j] != 0.0)

    if L == 0:
        return rg(0)
    G = T[m]
    b2 = np.zeros_like(G)
    b1 = rg(L)
    for g in range(L - 1, 0, -1):
        b1, b2 = 2.0 * G @ b1 - b2 + rg(g), b1
    return G @ b1 - b2 + rg(0)


def polynomial(B: np.ndarray, rho: float, s: int, D: int, m: int) -> np.ndarray:
    """R = p(B / rho) ~ exp(i B / 2^s) by the device's sequence of steps (FP64)."""
    n = B.shape[0]
    a = math.ldexp(rho, -s)
    e, b = split_coefficients(a, D)
    Z = B / rho if rho > 0 else np.zeros_like(B)
    if D <= 1:
        return e[0] * np.eye(n) + 1j * (b[0] * Z if len(b) else 0.0)
    C = 2.0 * Z @ Z - np.eye(n)
    T = baby_steps(C, baby_top(D, m))
    re = clenshaw(blocks(e, m), T, m)
    if len(b) == 0:
        return re.astype(np.complex128)
    if len(b) == 1:
        im = b[0] * Z
    else:
        im = Z @ clenshaw(blocks(b, m), T, m)
    return re + 1j * im


def walk_propagator(B: np.ndarray, rho: float, tol: float = 1e-6) -> tuple[np.ndarray, dict]:
    """exp(iB) by the plan for rho, the polynomial stage and s squarings (FP64)."""
    p = plan(rho, tol)
    R = polynomial(B, rho, p["s"], p["degree"], p["baby"])
    for _ in range(p["s"]):
        R = R @ R
    return R, p
