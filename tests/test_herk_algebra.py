"""The Hermitian product's tile algebra, restated in numpy (host only, no GPU).

The tensor-core product (matvis_b200/csrc/herk.cu) fills each upper 128 x 128
tile (I, J) of V = conj(Z) Z^T from split-term products (pa, pb) of the panel's
real and imaginary planes:

    Re  = sum_(pa,pb) Zr_I^pa Zr_J^pb^T + Zi_I^pa Zi_J^pb^T
    Imc = sum_(pa,pb) Zr_I^pa Zi_J^pb^T - Zi_I^pa Zr_J^pb^T

A diagonal tile (I = J) skips the Zr . Zi^T products and keeps only
W = -sum Zi^pa Zr^pb^T in its imaginary half; the reduction forms W - W^T.
That equals Imc exactly when the set of split-term products is symmetric under
pa <-> pb, which these tests check for every split mode's product table and
against the reference's own product, z.conj().dot(z.T) (cpu/matprod.py:11-32),
in exact (float64) arithmetic on split panels.
"""

import numpy as np
import pytest

# the split-term products of each mode, as the kernel issues them (product_terms)
PRODUCTS = {
    "fp16x3": [(0, 1), (1, 0), (0, 0)],
    "bf16x3": [(0, 1), (1, 0), (0, 0)],
    "tf32x3": [(0, 1), (1, 0), (0, 0)],
    "bf16x6": [(1, 1), (0, 2), (2, 0), (0, 1), (1, 0), (0, 0)],
}


def _round(x, mode):
    """x rounded to the mode's operand type, to nearest even: fp16, or float32 with
    its mantissa cut to 7 bits (bf16) or 10 bits (tf32)."""
    if mode == "fp16x3":
        return x.astype(np.float16).astype(np.float64)
    drop = 16 if mode.startswith("bf16") else 13
    b = x.astype(np.float32).view(np.uint32).astype(np.uint64)
    b = (b + (1 << (drop - 1)) - 1 + ((b >> drop) & 1)) >> drop << drop
    return b.astype(np.uint32).view(np.float32).astype(np.float64)


def _split(x, terms, mode):
    """x = sum of `terms` planes, each rounded to the mode's operand type (the panel's split)."""
    out, rest = [], x.astype(np.float64)
    for _ in range(terms):
        p = _round(rest, mode)
        out.append(p)
        rest = rest - p
    return out


def _tile_sums(zr, zi, rows_i, rows_j, prods, diag_form):
    re = np.zeros((len(rows_i), len(rows_j)))
    im = np.zeros_like(re)
    for pa, pb in prods:
        ar, ai = zr[pa][rows_i], zi[pa][rows_i]
        br, bi = zr[pb][rows_j], zi[pb][rows_j]
        re += ar @ br.T + ai @ bi.T
        im -= ai @ br.T
        if not diag_form:
            im += ar @ bi.T
    return re, im


@pytest.mark.parametrize("mode", sorted(PRODUCTS))
def test_product_tables_are_swap_symmetric(mode):
    prods = PRODUCTS[mode]
    assert sorted(prods) == sorted((b, a) for a, b in prods)


@pytest.mark.parametrize("mode", sorted(PRODUCTS))
def test_diagonal_tile_imaginary_half_is_w_minus_w_transpose(mode):
    rng = np.random.default_rng(7)
    M, K, B = 40, 96, 16  # 40 rows in blocks of 16 (the last block ragged)
    z = rng.normal(size=(M, K)) + 1j * rng.normal(size=(M, K))
    terms = 3 if mode == "bf16x6" else 2
    zr, zi = _split(z.real, terms, mode), _split(z.imag, terms, mode)
    # the product of the split panel, computed as the reference does
    zs = sum(zr) + 1j * sum(zi)
    full = zs.conj() @ zs.T
    prods = PRODUCTS[mode]
    nb = -(-M // B)
    for I in range(nb):
        ri = np.arange(I * B, min((I + 1) * B, M))
        re, imc = _tile_sums(zr, zi, ri, ri, prods, diag_form=False)
        re_d, w = _tile_sums(zr, zi, ri, ri, prods, diag_form=True)
        np.testing.assert_array_equal(re_d, re)
        np.testing.assert_allclose(w - w.T, imc, rtol=0, atol=1e-10)
        # the split terms only reach the reference's product where both terms of
        # the pair are kept: compare the tile with the kept products alone
        kept = np.zeros((len(ri), len(ri)), complex)
        for pa, pb in prods:
            a = zr[pa][ri] + 1j * zi[pa][ri]
            b = zr[pb][ri] + 1j * zi[pb][ri]
            kept += a.conj() @ b.T
        np.testing.assert_allclose(re + 1j * (w - w.T), kept, rtol=0, atol=1e-10)
        # and those products are the reference's own up to the dropped small terms
        auto = np.diag(full).real[ri]
        scale = np.sqrt(np.outer(auto, auto))
        tol = {"fp16x3": 2e-6, "bf16x3": 1e-4, "tf32x3": 1e-5, "bf16x6": 1e-6}[mode]
        assert np.max(np.abs(re + 1j * (w - w.T) - full[np.ix_(ri, ri)]) / scale) < tol
        # off-diagonal tiles keep both products of the imaginary half
        for J in range(I + 1, nb):
            rj = np.arange(J * B, min((J + 1) * B, M))
            re_o, im_o = _tile_sums(zr, zi, ri, rj, prods, diag_form=False)
            a_full = np.zeros((len(ri), len(rj)), complex)
            for pa, pb in prods:
                a_full += (zr[pa][ri] + 1j * zi[pa][ri]).conj() @ (zr[pb][rj] + 1j * zi[pb][rj]).T
            np.testing.assert_allclose(re_o + 1j * im_o, a_full, rtol=0, atol=1e-10)
