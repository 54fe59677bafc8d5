"""Evaluation of an integer-slice form of the split GEMMs (CPU, exact integer arithmetic).

The mixed-precision path cuts each FP64 operand, scaled by a power of two per
weight row / field column into (-1, 1), into S digits of 8 bits that BF16 holds
exactly, and sums the slice products with qa + qb <= S - 1 (split_gemm.cu).
The integer form evaluated here follows Ootomo, Ozaki and Yokota, "DGEMM on
integer matrix multiplication unit" (IJHPCA, 2024): the same power-of-two
scaling, digits of 7 bits plus sign (int8, |digit| <= 127), the products of
each level L = qa + qb summed exactly in int32 (tcgen05.mma kind::i8), and the
levels combined in FP64 with weights 2^-7(L+2).

The operands are the RTRAN(+1) products of a real grid: the orthonormal
Legendre table PF of the oracle (one m, one parity) times random field rows.
The checks pin what such a kernel would need: the int32 level sums stay exact,
7 int8 digits (28 digit pairs) match the accuracy of the 6 BF16 digits
(21 pairs) that meet the step's error bound, and 6 int8 digits do not.
"""

import numpy as np
import pytest

from oracle.grid import Grid


def _digits(M, axis, base_bits, S):
    """Power-of-two scaling of each row (axis=1) or column (axis=0) into (-1, 1)
    and S signed digits in base 2^base_bits: M = 2^e * sum_q D[q] 2^-b(q+1)
    up to the truncation below the last digit.  Returns (D[S], e)."""
    amax = np.max(np.abs(M), axis=axis, keepdims=True)
    e = np.where(amax > 0, np.floor(np.log2(np.where(amax > 0, amax, 1.0))) + 1, 0).astype(np.int64)
    scaled = M * np.exp2(-e.astype(np.float64))  # exact (power of two); |scaled| < 1
    fix = np.trunc(np.ldexp(scaled, base_bits * S)).astype(np.int64)  # |fix| < 2^(b S) <= 2^56
    sign, mag = np.sign(fix), np.abs(fix)
    mask = (1 << base_bits) - 1
    D = np.stack([sign * ((mag >> (base_bits * (S - 1 - q))) & mask) for q in range(S)])
    return D, e


def _sliced_product(A, B, base_bits, S):
    """sum_{qa + qb <= S-1} 2^-b(qa+qb+2) (Da[qa] Db[qb]) 2^(ea+eb), the level sums in
    exact integers; returns (C, the largest |level sum|)."""
    Da, ea = _digits(A, 1, base_bits, S)
    Db, eb = _digits(B, 0, base_bits, S)
    C = np.zeros((A.shape[0], B.shape[1]))
    peak = 0
    for L in range(S):
        acc = np.zeros((A.shape[0], B.shape[1]), dtype=np.int64)
        for qa in range(L + 1):
            acc += Da[qa] @ Db[L - qa]
        peak = max(peak, int(np.max(np.abs(acc))))
        C += np.ldexp(acc.astype(np.float64), -base_bits * (L + 2))
    return C * np.exp2(ea.astype(np.float64)) * np.exp2(eb.astype(np.float64)), peak


def _rel(C, R):
    return float(np.linalg.norm(C - R) / np.linalg.norm(R))


@pytest.fixture(scope="module")
def operands():
    """RTRAN(+1) operands at 96x64x64 (NRCHOP 64): for m = 0, 20, 40 and both
    parities, A = PF rows (NRH x K) and B = random field rows (K x 2 NXCHOPDIM)."""
    g = Grid(96, 64, 64, 64, 42, 21)
    rng = np.random.default_rng(3)
    out = []
    for m in (0, 20, 40):
        nn = int(g.NRCHOPS[m])
        for p in (0, 1):
            A = g.PF[:, p:nn:2, m]
            B = rng.standard_normal((A.shape[1], 2 * g.NXCHOPDIM)) * np.exp2(rng.integers(-20, 1, (1, 2 * g.NXCHOPDIM)))
            R = (A.astype(np.longdouble) @ B.astype(np.longdouble)).astype(np.float64)
            out.append((A, B, R))
    return out


def test_int32_levels_exact(operands):
    """Each level sum of int8 digit products fits int32 (|digit| <= 127)."""
    for A, B, _ in operands:
        _, peak = _sliced_product(A, B, 7, 7)
        assert peak < 2 ** 31
        # the bound for any K: (L + 1) K 127^2 < 2^31 holds for K below 2^31 / (7 * 127^2) ~ 19,000
        assert 7 * A.shape[1] * 127 ** 2 < 2 ** 31


def test_int8_digits_needed(operands):
    """7 int8 digits match 6 BF16 digits; 6 int8 digits are about 2^6 worse."""
    e_bf16_6 = max(_rel(_sliced_product(A, B, 8, 6)[0], R) for A, B, R in operands)
    e_i8_6 = max(_rel(_sliced_product(A, B, 7, 6)[0], R) for A, B, R in operands)
    e_i8_7 = max(_rel(_sliced_product(A, B, 7, 7)[0], R) for A, B, R in operands)
    assert e_bf16_6 < 1e-13
    assert e_i8_7 < 2 * e_bf16_6
    assert e_i8_6 > 8 * e_bf16_6
