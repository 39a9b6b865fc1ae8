"""Setup numerics against the reference's own code (golden vectors generated
by tests/golden/make_golden.py from the reference compiled from source)."""
from __future__ import annotations

from fractions import Fraction
from pathlib import Path

import numpy as np
import pytest

import bfam_b200 as bf
from oracle import oracle as orc

GOLD = np.load(Path(__file__).parent / "golden" / "reference_ops.npz")


@pytest.mark.parametrize("N", range(1, 9))
def test_product_lgl_bit_exact(N):
    r, w, wi, D = bf.lgl_operators(N)
    assert np.array_equal(r, GOLD[f"r_{N}"])
    assert np.array_equal(w, GOLD[f"w_{N}"])
    assert np.array_equal(wi, GOLD[f"wi_{N}"])
    assert np.array_equal(D, GOLD[f"Dr_{N}"])


@pytest.mark.parametrize("pair", [(n, n) for n in range(1, 9)] + [(3, 5), (5, 3), (5, 7), (7, 5)])
def test_product_mortar_ops_bit_exact(pair):
    a, b = pair
    assert np.array_equal(bf.mortar_operators(a, b), GOLD[f"prj_{a}_to_{b}"])


@pytest.mark.parametrize("N", range(1, 9))
def test_oracle_lgl_pinned(N):
    """The oracle computes its operators by a different algorithm; pin it."""
    r, w, D = orc.lgl(N)
    scale = max(1.0, np.abs(GOLD[f"Dr_{N}"]).max())
    assert np.abs(r - GOLD[f"r_{N}"]).max() < 1e-14
    assert np.abs(w - GOLD[f"w_{N}"]).max() < 1e-14
    assert np.abs(D - GOLD[f"Dr_{N}"]).max() < 1e-14 * scale * 4


@pytest.mark.parametrize("N", range(1, 9))
def test_oracle_mortar_pinned(N):
    Ib, It, Pb, Pt = orc.mortar(N)
    g = GOLD[f"prj_{N}_to_{N}"]
    for mine, k in ((Pb, 1), (Pt, 2), (Ib, 3), (It, 4)):
        assert np.abs(mine - g[k]).max() < 1e-14


@pytest.mark.parametrize("N", range(1, 9))
def test_mortar_operator_identities(N):
    """Projection after interpolation reproduces a polynomial; the two
    halves' projections sum to the identity on the full interval."""
    n = N + 1
    g = GOLD[f"prj_{N}_to_{N}"].reshape(5, n, n).transpose(0, 2, 1)  # row-major
    Pb, Pt, Ib, It = g[1], g[2], g[3], g[4]
    assert np.abs(Pb @ Ib + Pt @ It - np.eye(n)).max() < 1e-12


def test_pcg32_stream_matches_reference():
    for seed, seq in ((0, 1), (42, 54), (1, 2)):
        ref = GOLD[f"pcg32_{seed}_{seq}"]
        g = bf.PCG32(seed, seq)
        assert [g.next() for _ in range(len(ref))] == [int(x) for x in ref]


def test_lsrk_kc54_coefficients_exact():
    A, B, C = bf.lsrk_coefficients(bf.LSRK_KC54)
    exact_A = [0, Fraction(-567301805773, 1357537059087), Fraction(-2404267990393, 2016746695238),
               Fraction(-3550918686646, 2091501179385), Fraction(-1275806237668, 842570457699)]
    exact_B = [Fraction(1432997174477, 9575080441755), Fraction(5161836677717, 13612068292357),
               Fraction(1720146321549, 2090206949498), Fraction(3134564353537, 4481467310338),
               Fraction(2277821191437, 14882151754819)]
    for got, ex in zip(A, exact_A):
        assert got == float(ex)
    for got, ex in zip(B, exact_B):
        assert got == float(ex)
    assert C[0] == 0.0 and C[-1] == 1.0 and len(C) == 6


def test_lsrk_methods_consistency():
    """sum of stage weights: 2N-storage schemes integrate dq/dt = 1 exactly."""
    for m in (bf.LSRK_KC54, bf.LSRK_W33, bf.LSRK_HEUN, bf.LSRK_FE):
        A, B, C = bf.lsrk_coefficients(m)
        q, dq, t = 0.0, 0.0, 0.0
        for s in range(len(A)):
            dq = A[s] * dq + 1.0
            q += B[s] * dq
        assert abs(q - 1.0) < 1e-14
