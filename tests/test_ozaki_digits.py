"""The digit arithmetic of the FP64 form's tensor-core contraction (ozaki.cu),
restated on the CPU with exact integer products: 7 truncation digits of 7
bits per row of b_l and per column of C5, the 28 digit products with
i + j < 7, recombined in FP64.  The restated product is within 1e-12 of the
largest |tmp| of an FP64 GEMM (the bound tests/test_gpu_ozaki.py asserts for
the kernel), while 6 digits would not leave that margin."""
import numpy as np
import pytest

from donof_b200 import workload

S = 7


def digits(X, axis, s=S):
    """Truncation digits of X along `axis` (the contraction axis): X ~= 2^e sum_i d_i 2^(-7(i+1))."""
    mx = np.max(np.abs(X), axis=axis, keepdims=True)
    e = np.where(mx > 0, np.frexp(mx)[1], 0)
    y = X * np.ldexp(1.0, -e)
    assert np.all(np.abs(y) < 1.0)
    out = []
    for _ in range(s):
        y = y * 128.0
        t = np.trunc(y)
        out.append(t.astype(np.int64))
        y = y - t
    return out, e


def t1_digits(b, C5, s=S):
    """tmp[l, m, q] = sum_n b[m, n, l] C5[n, q] through the digit products."""
    A = np.moveaxis(b, 2, 0)                 # (l, m, n)
    Ad, ea = digits(A, axis=2, s=s)          # ea: (l, m, 1)
    Bd, eb = digits(C5, axis=0, s=s)         # eb: (1, q)
    acc = [np.zeros((A.shape[0], A.shape[1], C5.shape[1]), dtype=np.int64) for _ in range(s)]
    for i in range(s):
        for j in range(s - i):
            acc[i + j] += np.matmul(Ad[i], Bd[j])        # exact: int64 (int32 on the device)
    for g in range(s):
        assert np.max(np.abs(acc[g])) < 2 ** 31          # the device's int32 accumulators cannot overflow
    v = acc[s - 1].astype(np.float64)
    for g in range(s - 2, -1, -1):
        v = v * 2.0 ** -7 + acc[g]
    return v * np.ldexp(1.0, ea) * np.ldexp(1.0, eb - 14)


@pytest.mark.parametrize("nbf,naux,nbf5,seed", [(24, 16, 12, 1), (48, 8, 48, 2), (96, 4, 40, 3)])
def test_seven_digits_reach_the_stated_bound(nbf, naux, nbf5, seed):
    rng = np.random.default_rng(seed)
    b = workload.make_b(nbf, naux, rng)
    C = np.linalg.qr(rng.standard_normal((nbf, nbf)))[0]
    ref = np.einsum("mnl,nq->lmq", b, C[:, :nbf5])
    out = t1_digits(b, C[:, :nbf5])
    err = np.max(np.abs(out - ref)) / np.max(np.abs(ref))
    assert err <= 1e-12
    six = t1_digits(b, C[:, :nbf5], s=6)
    assert np.max(np.abs(six - ref)) / np.max(np.abs(ref)) > 1e-12


def test_digits_are_exact_and_bounded():
    rng = np.random.default_rng(5)
    x = rng.standard_normal((7, 33)) * np.ldexp(1.0, rng.integers(-30, 30, size=(7, 1)))
    d, e = digits(x, axis=1)
    assert all(np.max(np.abs(di)) <= 127 for di in d)
    back = sum(di * 2.0 ** (-7 * (i + 1)) for i, di in enumerate(d)) * np.ldexp(1.0, e)
    # the truncation residual is below 2^(-7S) of the row's power of two
    assert np.all(np.abs(back - x) <= np.ldexp(1.0, e - 7 * S))


def test_int32_bound_at_the_largest_supported_basis():
    """|acc_g| <= 7 * 127^2 * nbf < 2^31 for nbf <= 16384 (ozaki_shape_ok): the
    device's int32 accumulators are exact."""
    assert 7 * 127 ** 2 * 16384 < 2 ** 31
