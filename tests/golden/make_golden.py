"""Generate the golden fixtures under tests/golden/ (committed).

Two kinds of fixture:

* numax's own golden values, ported verbatim from the reference's tests:
  tests/linalg/test_lu_plu.mojo:15-109 (SciPy's P, L, U of a 4x4 whose first
  pivot is zero) and the hand-written matrices of
  tests/linalg/test_tensor_linalg.mojo / test_panel.mojo / test_linalg.mojo.
* independent LAPACK answers (SciPy 1.18 / OpenBLAS) on seeded inputs, to pin
  the oracle where numax itself has no golden data: LU factors and pivots,
  the Cholesky factor, Householder QR in LAPACK's packed form, and symmetric
  eigenvalues.

Inputs come from numpy's PCG64 with fixed seeds.  Run:
    python tests/golden/make_golden.py
"""
import os

import numpy as np
import scipy.linalg as sl

HERE = os.path.dirname(os.path.abspath(__file__))


def numax_fixtures():
    # tests/linalg/test_lu_plu.mojo:15-109
    a = np.array([0.0, 2.0, 1.0, 3.0, 4.0, 1.0, -2.0, 1.0, 2.0, 5.0, 3.0, -1.0,
                  1.0, -3.0, 2.0, 6.0]).reshape(4, 4)
    p = np.array([0.0, 0.0, 0.0, 1.0, 1.0, 0.0, 0.0, 0.0, 0.0, 1.0, 0.0, 0.0,
                  0.0, 0.0, 1.0, 0.0]).reshape(4, 4)
    l = np.array([1.0, 0.0, 0.0, 0.0, 0.5, 1.0, 0.0, 0.0, 0.25, -0.7222222222222222, 1.0, 0.0,
                  0.0, 0.4444444444444444, -0.14432989690721645, 1.0]).reshape(4, 4)
    u = np.array([4.0, 1.0, -2.0, 1.0, 0.0, 4.5, 4.0, -1.5, 0.0, 0.0, 5.388888888888889,
                  4.666666666666667, 0.0, 0.0, 0.0, 4.34020618556701]).reshape(4, 4)
    # tests/linalg/test_tensor_linalg.mojo:816-832 (exchange matrix)
    exchange = np.array([[0.0, 1.0], [1.0, 0.0]])
    exchange_b = np.array([3.0, 5.0])
    exchange_x = np.array([5.0, 3.0])
    # tests/linalg/test_tensor_linalg.mojo:700-741 (fails at index 3)
    later_block = np.array([4.0, 1.0, 0.0, 0.0, 1.0, 4.0, 0.0, 0.0, 0.0, 0.0, 1.0, 3.0,
                            0.0, 0.0, 3.0, 1.0]).reshape(4, 4)
    not_spd_2x2 = np.array([[1.0, 2.0], [2.0, 1.0]])
    # tests/linalg/test_panel.mojo:258-275 (column (0, 4, 7) pivots on row 2)
    panel3 = np.array([0.0, 1.0, 2.0, 4.0, 5.0, 6.0, 7.0, 8.0, 10.0]).reshape(3, 3)
    # tests/linalg/test_tensor_linalg.mojo:505-531 (hand-made SPD 5x5)
    spd5 = np.array([9.0, 3.0, 1.0, 2.0, 0.0, 3.0, 10.0, 2.0, 1.0, 1.0, 1.0, 2.0, 8.0, 3.0, 2.0,
                     2.0, 1.0, 3.0, 11.0, 4.0, 0.0, 1.0, 2.0, 4.0, 7.0]).reshape(5, 5)
    # tests/linalg/test_linalg.mojo:65-71 (spd3)
    spd3 = np.array([4.0, 2.0, 1.0, 2.0, 5.0, 3.0, 1.0, 3.0, 6.0]).reshape(3, 3)
    np.savez(os.path.join(HERE, "numax_fixtures.npz"), lu_a=a, lu_p=p, lu_l=l, lu_u=u,
             exchange=exchange, exchange_b=exchange_b, exchange_x=exchange_x,
             later_block=later_block, not_spd_2x2=not_spd_2x2, panel3=panel3, spd5=spd5,
             spd3=spd3)


def lapack_fixtures():
    rng = np.random.Generator(np.random.PCG64(20260101))
    out = {}
    for n in (17, 64):
        a = rng.standard_normal((n, n))
        lu, piv = sl.lu_factor(a)
        out[f"lu{n}_a"], out[f"lu{n}_lu"], out[f"lu{n}_piv"] = a, lu, piv.astype(np.int32)
    g = rng.standard_normal((40, 40))
    spd = g @ g.T / 40 + np.eye(40)
    out["chol40_a"], out["chol40_l"] = spd, np.linalg.cholesky(spd)
    q = rng.standard_normal((70, 40))
    (packed, tau), _ = sl.qr(q, mode="raw")
    out["qr70_a"], out["qr70_packed"], out["qr70_tau"] = q, np.ascontiguousarray(packed), tau
    g = rng.standard_normal((24, 24))
    sym = (g + g.T) / 2
    out["eig24_a"], out["eig24_w"] = sym, np.linalg.eigvalsh(sym)
    # The harmonic well of examples/advanced/quantum_well.mojo:66-75 at w = 1.
    n, dx = 24, 8.0 / 23
    h = np.zeros((n, n))
    x = -4.0
    for i in range(n):
        h[i, i] = 1.0 / dx ** 2 + x * x / 2
        if i + 1 < n:
            h[i, i + 1] = h[i + 1, i] = -0.5 / dx ** 2
        x += dx
    out["well24_a"], out["well24_w"] = h, np.linalg.eigvalsh(h)
    np.savez(os.path.join(HERE, "lapack_fixtures.npz"), **out)


if __name__ == "__main__":
    numax_fixtures()
    lapack_fixtures()
    print("wrote", sorted(f for f in os.listdir(HERE) if f.endswith(".npz")))
