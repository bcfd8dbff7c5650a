"""The digit-slice schemes behind the two int8 tensor-core emulations, restated in numpy and
checked on CPU against exact products, so that the slice and level counts the kernels use are
pinned by a test and not only by the GPU comparisons:

  * the plain form's trailing update (kernels_oz.cu): 6 rounded (balanced) 7-bit digits per panel
    row against a power-of-two row scale, products of levels s + t <= 8 (26 per K step): the
    product of two panel rows within ~1e-12 of ||P_r|| ||P_c||, far inside what the FP64 DMMA
    comparison (1e-12 on the forms) allows, and as close as 7 truncated digits at 28 products;
  * the refined mixed form's Gram term (kernels_gram_oz.cu): C^T in 7 and y in 4 rounded
    (balanced) digits, levels s + t <= 9: the corrected forms at the FP64 product's accuracy,
    where truncated digits or 3 y digits are not.

The emulation is exact integer arithmetic on the digits (int64 matrix products) with the level sums
combined in extended precision, i.e. what the tensor cores compute.  Systems come from the seeded
generator and the oracle's V_ph; the panels are those of a real Cholesky factorisation of eps.
"""
from __future__ import annotations

import numpy as np
import pytest


def _digits(m: np.ndarray, nd: int, base_bits: int, rounded: bool) -> tuple[np.ndarray, np.ndarray]:
    """Row-scaled digits of m: truncated (|v| < 1, trunc) or balanced (|v| < 1/2, rint)."""
    mx = np.abs(m).max(axis=1)
    e = np.frexp(np.where(mx > 0, mx, 1.0))[1] + (1 if rounded else 0)
    v = m * np.ldexp(1.0, -e)[:, None]
    base = float(1 << base_bits)
    out = []
    for _ in range(nd):
        t = v * base
        d = np.rint(t) if rounded else np.trunc(t)
        v = t - d
        out.append(d.astype(np.int64))
    return np.array(out), e


def _product(a: np.ndarray, b: np.ndarray, nd_a: int, nd_b: int, lmax: int, rounded: bool):
    """a @ b.T from digit products of levels s + t <= lmax (1-based digits), level sums exact."""
    da, ea = _digits(a, nd_a, 7, rounded)
    db, eb = _digits(b, nd_b, 7, rounded)
    g = np.zeros((a.shape[0], b.shape[0]), dtype=np.longdouble)
    levels: dict[int, np.ndarray] = {}
    for s in range(nd_a):
        for t in range(nd_b):
            lv = s + t + 2
            if lv <= lmax:
                levels[lv] = levels.get(lv, 0) + da[s] @ db[t].T
    for lv in sorted(levels, reverse=True):
        g += levels[lv].astype(np.longdouble) * np.longdouble(2.0) ** (-7 * lv)
    scale = np.ldexp(1.0, ea)[:, None].astype(np.longdouble) * np.ldexp(1.0, eb)[None, :].astype(np.longdouble)
    return (g * scale).astype(np.float64), db, eb


def _system(nmo: int, nocc: int, seed: int):
    import oracle
    from minigw_b200.synthetic import make_input

    o = oracle.Oracle()
    inp = make_input(nmo, nocc, seed=seed)
    _, _, de = o.ph_map(nmo, nocc, inp.mo_energy)
    return inp, de, o.vph(inp)


@pytest.mark.parametrize("omega", [0.05, 1.0, 20.0])
def test_update_scheme_product_error(omega):
    """6 rounded digits, levels <= 8 (26 products): the trailing-update product of two panel rows
    of a real eps factorisation within 1e-12 of ||P_r|| ||P_c|| (measured ~2e-13; an FP64 dot
    product ~3e-16), within 3x of 7 truncated digits at 28 products, while cutting the levels to
    <= 7 (21 products) or truncating the 6 digits costs an order of magnitude."""
    _, de, v = _system(40, 12, seed=117)
    n = v.shape[0]
    d = 4 * de / (de * de + omega ** 2)
    dh = np.sqrt(d)
    chol = np.linalg.cholesky(np.eye(n) + dh[:, None] * v * dh[None, :])
    panel = chol[128:, :128]
    exact = panel.astype(np.longdouble) @ panel.T.astype(np.longdouble)
    scale = np.sqrt((panel * panel).sum(1)).max() ** 2

    def err(nd, lmax, rounded):
        got, _, _ = _product(panel, panel, nd, nd, lmax, rounded)
        return float(np.abs(got - exact).max() / scale)

    e = err(6, 8, True)
    assert e <= 1e-12, e
    assert e <= 3 * err(7, 8, False)
    assert err(6, 7, True) > 5 * e
    assert err(6, 7, False) > 10 * e


def _blocked_forms(tall: np.ndarray, n: int, scheme) -> np.ndarray:
    """-||w||^2 of the right-hand-side rows after a right-looking blocked Cholesky of the tall
    matrix [eps; (D^1/2 X)^T] with K = 128 outer blocks (the kernels' blocking): each panel
    factored in FP64, the trailing update from the emulated digit products (`scheme` = (digits,
    level cut, rounded)) or in FP64 (scheme None)."""
    a = tall.copy()
    for k0 in range(0, n, 128):
        k1 = min(k0 + 128, n)
        lkk = np.linalg.cholesky(a[k0:k1, k0:k1])
        a[k0:k1, k0:k1] = lkk
        a[k1:, k0:k1] = np.linalg.solve(lkk, a[k1:, k0:k1].T).T
        p = a[k1:, k0:k1]
        if p.shape[0] == 0 or k1 >= n:
            continue
        if scheme is None:
            upd = p @ p[: n - k1].T
        else:
            pp = np.zeros((p.shape[0], 128))
            pp[:, : k1 - k0] = p
            nd, lmax, rounded = scheme
            upd, _, _ = _product(pp, pp[: n - k1], nd, nd, lmax, rounded)
        a[k1:, k1:n] -= upd
    w = a[n:, :n]
    return -np.sum(w * w, axis=1)


def test_update_scheme_inside_the_blocked_factorisation():
    """The screened forms from the whole blocked factorisation with the emulated trailing updates
    (6 rounded digits, levels <= 8) within 2e-13 relative of the FP64 factorisation at low, middle
    and high frequency (measured 5e-14 to 9e-14, and ~7e-16 at high frequency), and within 3x of
    the 7 truncated digits the kernel used before."""
    inp, de, v = _system(40, 12, seed=117)
    nmo, nocc = 40, 12
    n = v.shape[0]
    eri = inp.eri_mo.reshape(nmo, nmo, nmo, nmo)
    io = np.repeat(np.arange(nocc), nmo - nocc)
    av = np.tile(np.arange(nocc, nmo), nocc)
    x = np.concatenate([eri[s, :, io, av].T for s in (10, 11, 12, 13)])  # (4 nmo) x n right-hand sides
    for omega in (0.05, 1.0, 30.0):
        d = 4 * de / (de * de + omega ** 2)
        dh = np.sqrt(d)
        tall = np.concatenate([np.eye(n) + dh[:, None] * v * dh[None, :], x * dh[None, :]])
        ref = _blocked_forms(tall, n, None)
        scale = np.abs(ref).max()
        e6 = np.abs(_blocked_forms(tall, n, (6, 8, True)) - ref).max() / scale
        e7 = np.abs(_blocked_forms(tall, n, (7, 8, False)) - ref).max() / scale
        assert e6 <= 2e-13, (omega, e6)
        assert e6 <= 3 * e7 + 1e-16, (omega, e6, e7)


def _pchol(v: np.ndarray, tau_rel: float = 1e-13) -> np.ndarray:
    n = v.shape[0]
    diag = np.diag(v).copy()
    tau = tau_rel * diag.max()
    c = np.zeros((n, n))
    piv: list[int] = []
    for k in range(n):
        p = int(np.argmax(diag))
        if diag[p] < tau:
            break
        col = (v[:, p] - c[:, :k] @ c[p, :k]) / np.sqrt(diag[p])
        c[:, k] = col
        diag -= col * col
        piv.append(p)
        diag[piv] = 0.0
    return c[:, :len(piv)]


def test_refined_gram_scheme_forms_error():
    """The refined form's t3 = ||C^T y||^2 from 7 x 4 rounded digits (levels <= 9), with t1, t2
    from the same rounded y: forms within 2e-13 relative of the exact q (the exact-product
    refinement gives ~2e-14; truncated 7 x 3 digits 1e-11, rounded 7 x 3 digits 1e-11)."""
    inp, de, v = _system(40, 12, seed=117)
    nmo, nocc = 40, 12
    n = v.shape[0]
    c = _pchol(v)
    ct = c.T.copy()
    eri = inp.eri_mo.reshape(nmo, nmo, nmo, nmo)
    io = np.repeat(np.arange(nocc), nmo - nocc)
    av = np.tile(np.arange(nocc, nmo), nocc)
    x = eri[11, :, io, av]  # n x nmo right-hand sides of state 11
    errs = {}
    for omega in (0.05, 2.0):
        d = 4 * de / (de * de + omega ** 2)
        dh = np.sqrt(d)
        eps = np.eye(n) + dh[:, None] * v * dh[None, :]
        b = dh[:, None] * x
        q_exact = -np.sum(b * np.linalg.solve(eps, b), axis=0)
        z = np.linalg.solve(eps.astype(np.float32), b.astype(np.float32)).astype(np.float64)  # FP32 solve
        y = dh[:, None] * z
        for name, nd_b, lmax, rounded in (("7x4 rounded", 4, 9, True), ("7x3 rounded", 3, 9, True),
                                          ("7x3 truncated", 3, 8, False)):
            g, db, eb = _product(ct, y.T, 7, nd_b, lmax, rounded)
            # the y the digits represent, for t1 and t2
            yh = sum(db[t].astype(np.float64) * 2.0 ** (-7 * (t + 1)) for t in range(nd_b))
            yh = (yh * np.ldexp(1.0, eb)[:, None]).T
            zh = yh / dh[:, None]
            q = -(2 * np.sum(x * yh, 0) - np.sum(zh * zh, 0) - np.sum(g * g, 0))
            errs[name] = max(errs.get(name, 0.0), float(np.abs(q - q_exact).max() / np.abs(q_exact).max()))
    assert errs["7x4 rounded"] <= 2e-13, errs
    assert errs["7x3 rounded"] > 10 * errs["7x4 rounded"], errs
    assert errs["7x3 truncated"] > 10 * errs["7x4 rounded"], errs
