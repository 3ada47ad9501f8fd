"""The integer split behind the complex128 tensor-core blocks, restated in
numpy (CPU): rows of the real-embedded 64 x 64 block unitary W and rows of a
state supertile S are scaled by powers of two to 55-bit integers and cut into
seven 8-bit digits (W: balanced digits, rounded on the host; S: the two's-
complement bytes, truncated on the device).  The 28 digit products of weight
i + j >= 6 are summed exactly per weight and combined in FP64.  Checked here:
every digit fits its int8 / uint8 operand type, every per-weight sum fits an
int32 accumulator, and the result matches W @ S to 2^-48 relative."""
import numpy as np
import pytest

from subquokka_dev_b200 import circuits

DIGITS = 7


def biased_exponent(x):
    return ((np.abs(x).view(np.uint64) >> np.uint64(52)) & np.uint64(0x7FF)).astype(np.int64)


def w_digits(row):
    """Balanced base-256 digits (low first) of round(row 2^(1076 - e)) and e."""
    e = int(biased_exponent(row).max())
    v = np.rint(np.ldexp(row, 1076 - e)).astype(np.int64)
    out = []
    for _ in range(DIGITS - 1):
        d = ((v + 128) & 255) - 128
        out.append(d)
        v = (v - d) // 256
    out.append(v)
    return np.array(out), e


def s_digits(row):
    """Two's-complement bytes (low first; the top one signed) of
    trunc(row 2^(1076 - e)) and e."""
    e = int(biased_exponent(row).max())
    v = np.trunc(np.ldexp(row, 1076 - e)).astype(np.int64)
    out = [(v >> (8 * j)) & 255 for j in range(DIGITS - 1)]
    out.append(v >> 48)
    return np.array(out), e


def contract(W, S):
    """D[m][n] = sum_k W[m][k] S[n][k] through the digit products."""
    wd = [w_digits(W[m]) for m in range(W.shape[0])]
    sd = [s_digits(S[n]) for n in range(S.shape[0])]
    D = np.zeros((W.shape[0], S.shape[0]))
    amax = 0
    for m, (w, ew) in enumerate(wd):
        assert np.all((w[:-1] >= -128) & (w[:-1] <= 127)) and np.abs(w[-1]).max() <= 65
        for n, (s, es) in enumerate(sd):
            assert np.all((s[:-1] >= 0) & (s[:-1] <= 255)) and np.all((s[-1] >= -64) & (s[-1] <= 63))
            acc = 0.0
            for d in range(6, 13):
                a = sum(int(w[i] @ s[d - i]) for i in range(d - 6, 7))
                amax = max(amax, abs(a))
                acc += a * 2.0 ** (8 * (d - 12))
            D[m, n] = acc * 2.0 ** (ew - 1028) * 2.0 ** (es - 1028) if es >= 6 else 0.0
    return D, amax


def embed(U):
    W = np.zeros((128, 128))
    W[0::2, 0::2], W[0::2, 1::2] = U.real, -U.imag
    W[1::2, 0::2], W[1::2, 1::2] = U.imag, U.real
    return W


@pytest.mark.parametrize("seed,scale", [(1, 0), (2, -40), (3, -900)])
def test_digit_products_match_fp64(seed, scale):
    rng = np.random.default_rng(seed)
    z = rng.standard_normal((64, 64)) + 1j * rng.standard_normal((64, 64))
    U = np.linalg.qr(z)[0]
    W = embed(U)
    X = circuits.random_state(12, seed).reshape(64, 64) * 2.0 ** scale   # X[n][i]
    X[3] = 0                                                            # a row of zeros
    S = np.stack([X.real, X.imag], axis=2).reshape(64, 128)             # S[n][2i + c]
    D, amax = contract(W, S)
    ref = W @ S.T
    assert amax < 2 ** 25                                               # int32 accumulators
    err = np.abs(D - ref).max() / np.abs(ref).max()
    assert err <= 2.0 ** -48
    assert np.all(D[:, 3] == 0)
