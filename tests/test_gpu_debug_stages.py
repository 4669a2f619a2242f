"""The intermediate outputs of FX_OPT_DEBUG_STAGE (needs a GPU).

With debug_stage = k the general pipeline writes intermediate k instead of U and stops:
1 the shifted Y, 2-4 A2, A4, A6, 5 / 6 the Pade odd / even parts U, V of the scaled Y, 7 the
solve R = (V - U)^-1 (V + U), 8 + j the iterate after j squarings (E = R - I in I + E form).
Each is compared with the FP64 oracle's step (oracle/expm_oracle.py: pade_uv, solve_pq) on a
general complex input, within the complex64 tolerance of the parity tests (1e-5 relative).
"""
import numpy as np
import pytest

from oracle import expm_oracle as eo

pytestmark = pytest.mark.gpu

REL = 1e-5


def _stage(X, k, m, s):
    from fastctqw_b200._native import Engine
    e = Engine(X.shape[0], X.dtype)
    e.configure(shift=1, debug_stage=k, force_m=m, force_s=s)
    out = e.run_host(X)
    e.close()
    return out.astype(np.complex128)


def test_debug_stages_follow_the_oracle():
    rng = np.random.default_rng(8)
    n = 96
    X = ((rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))) * 0.4).astype(np.complex64)
    X64 = X.astype(np.complex128)
    Y = X64 - np.trace(X64) / n * np.eye(n)          # trace shift only (shift = 1)
    m, s = 13, 3
    refs = {1: Y, 2: Y @ Y}
    refs[3] = refs[2] @ refs[2]
    refs[4] = refs[3] @ refs[2]
    U, V = eo.pade_uv(Y, m, s)
    refs[5], refs[6] = U, V
    R = eo.solve_pq(U, V)
    refs[7] = R
    E = R - np.eye(n)
    refs[8] = E                                       # before the first squaring (I + E form)
    refs[9] = 2 * E + E @ E
    for k, ref in refs.items():
        got = _stage(X, k, m, s)
        assert eo.rel_error(got, ref) <= REL, (k, eo.rel_error(got, ref))
