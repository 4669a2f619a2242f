"""The int8 slicer of the product kernels (needs a GPU).

Every FP64 row is scaled by 2^(7S - e), e the row exponent (frexp of the row maximum, raised by
one when the mantissa would round to 128 at 7 bits), and cut into S signed digits from the top
with round-half-even: d_0 = rint(v / 2^7(S-1)), then the remainders.  The two kernels (a warp per
row that reads the row twice; and the two passes the products use, row exponents by a warp per
row and then the digits over a block plan of the rows' elements) must give the same digits, bit
for bit, and both must equal this rule restated in numpy below; the product kernels rely on it
(exactness of the int32 level sums, symmetric digits).  Rows cover zero, tiny (the two-step
scaling), ragged widths (K not a multiple of 4 included), exact half-way values and the
split-off diagonal.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _digits(x: np.ndarray, S: int, split_diag: bool):
    """Row exponents and digits of the rows of x (float64), the restated rule."""
    x = x.copy()
    dg = None
    if split_diag:
        idx = np.arange(min(x.shape))
        dg = x[idx, idx].copy()
        x[idx, idx] = 0.0
    mx = np.abs(x).max(axis=1)
    m, e = np.frexp(mx)
    e = np.where(mx > 0, e + (m * 128.0 >= 127.5), 0).astype(np.int64)
    r = np.rint(np.ldexp(x, (7 * S - e)[:, None]))
    d = []
    for q in range(S - 1):
        k = 7 * (S - 1 - q)
        t = np.rint(np.ldexp(r, -k))
        r = r - np.ldexp(t, k)
        d.append(t)
    d.append(r)
    return e, np.stack(d).astype(np.int8), dg


def _rows(rows, K, seed):
    rng = np.random.default_rng(seed)
    x = rng.standard_normal((rows, K)) * np.exp2(rng.integers(-40, 40, size=(rows, 1)))
    x[1] = 0.0                                          # zero row
    x[2] = rng.standard_normal(K) * 1e-300              # tiny row: two-step scaling
    x[3] = (np.arange(K) % 97 + 0.5) * 2.0 ** -35       # half-way values at S = 5 (e = 0)
    x[3, 0] = 0.99
    x[4, ::7] *= 1e6                                    # a few dominant entries
    return x


@pytest.mark.parametrize("K", [1024, 3000, 2050, 96, 4097])
@pytest.mark.parametrize("S", [3, 4, 5])
def test_slicers_agree_with_the_digit_rule(K, S):
    import torch
    from fastctqw_b200 import _native
    dev = torch.device("cuda", 0)
    rows = 40
    x = _rows(rows, K, seed=K + S)
    X = torch.from_numpy(x).to(dev)
    for split in (False, True):
        e_ref, d_ref, dg_ref = _digits(x, S, split)
        outs = [_native.slice_rows(X, S=S, kind=k, split_diag=split) for k in (0, 1)]
        for o in outs:
            assert np.array_equal(o["exp"].cpu().numpy(), e_ref), (S, K, split)
            assert np.array_equal(o["re"].cpu().numpy(), d_ref), (S, K, split)
            if split:
                assert np.array_equal(o["dg"].cpu().numpy(), dg_ref)
        assert torch.equal(outs[0]["re"], outs[1]["re"])


@pytest.mark.parametrize("K", [2048, 1100])
def test_two_plane_slices_share_the_row_exponent(K):
    """re and im of a complex row share one exponent (the maximum over both planes); -im's
    digits are the negated digits of im."""
    import torch
    from fastctqw_b200 import _native
    dev = torch.device("cuda", 0)
    S = 5
    xr, xi = _rows(24, K, 1), _rows(24, K, 2)[::-1].copy()
    both = np.concatenate([xr, xi], axis=1)
    e_ref, _, _ = _digits(both, S, False)
    for kind in (0, 1):
        o = _native.slice_rows(torch.from_numpy(xr).to(dev), torch.from_numpy(xi).to(dev), S=S, kind=kind, neg=True)
        assert np.array_equal(o["exp"].cpu().numpy(), e_ref)
        for x, key in ((xr, "re"), (xi, "im")):
            r = np.rint(np.ldexp(x, (7 * S - e_ref)[:, None]))
            got = o[key].cpu().numpy().astype(np.int64)
            val = sum(got[q] * 2.0 ** (7 * (S - 1 - q)) for q in range(S))
            assert np.array_equal(val, r), key
        assert np.array_equal(o["neg_im"].cpu().numpy().astype(np.int16), -o["im"].cpu().numpy().astype(np.int16))
