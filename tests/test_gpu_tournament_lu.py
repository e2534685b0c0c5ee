"""Tournament-pivoting FP32 LU, the panels of the mixed-precision
factorization (no numax counterpart; opted into for nmx_getrf_f32 by the
"lu.tournament" knob): P A = L U to FP32 accuracy with LAPACK-style
interchanges, for panels that one CTA, one group of CTAs and several groups
pick pivots for, unblocked and over look-ahead panels; an exactly zero
column is reported in info as by partial pivoting; and the refinement
converges with tournament pivoting on and off."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


def _factor(a, tournament, lookahead=-1):
    from numax_b200 import _lib, linalg
    lib = _lib.load()
    ctx = _lib.context(torch.cuda.current_device())
    lib.nmx_tune_set(ctx, b"lu.tournament", 1 if tournament else -1)
    lib.nmx_tune_set(ctx, b"lu.lookahead", lookahead)
    try:
        return linalg.lu_factor(a)
    finally:
        lib.nmx_tune_set(ctx, b"lu.tournament", -1)
        lib.nmx_tune_set(ctx, b"lu.lookahead", -1)


def _residual(a, f):
    """max |P A - L U| / max |A|, in FP64 on the device; and max |L|."""
    n = a.shape[0]
    piv = f.pivots.cpu().numpy()
    perm = np.arange(n)
    for j, p in enumerate(piv):
        assert j <= p < n
        perm[j], perm[p] = perm[p], perm[j]
    lu = f.factored.double()
    low = torch.tril(lu, -1) + torch.eye(n, dtype=torch.float64, device=lu.device)
    up = torch.triu(lu)
    pa = a.double()[torch.from_numpy(perm).to(a.device)]
    r = ((pa - low @ up).abs().max() / a.double().abs().max()).item()
    return r, low.abs().max().item()


# n = 7 and 33: one CTA; 1500: one group of 3 CTAs; 9000: two groups and a
# third level; odd orders take the unaligned-row loads.
@pytest.mark.parametrize("n", [7, 33, 500, 1500, 4099, 9000])
def test_tournament_lu_reconstructs(n):
    g = torch.Generator(device="cuda")
    g.manual_seed(n)
    a = torch.randn((n, n), generator=g, dtype=torch.float32, device="cuda")
    ft = _factor(a, True)
    fp = _factor(a, False)
    assert ft.info == 0 and fp.info == 0
    rt, lt = _residual(a, ft)
    rp, lp = _residual(a, fp)
    assert lp <= 1.0 + 1e-6
    # A stable factorization: within a small factor of partial pivoting's.
    assert rt <= 10 * rp + 1e-6, (rt, rp)
    assert lt <= 1e3, lt
    same = np.array_equal(ft.pivots.cpu().numpy(), fp.pivots.cpu().numpy())
    # Up to 512 rows one CTA picks every pivot: partial pivoting itself.
    # Past that the tournament picks others.
    assert same == (n <= 512)


# Look-ahead panels (orders >= 2 panels): ragged last panels, the smallest
# and the widest panel width, and one matrix with look-ahead off.
@pytest.mark.parametrize("n,nb", [(700, 64), (1500, 96), (3000, 512), (5000, 1024), (3000, 0)])
def test_tournament_lu_lookahead_panels(n, nb):
    g = torch.Generator(device="cuda")
    g.manual_seed(n + nb)
    a = torch.randn((n, n), generator=g, dtype=torch.float32, device="cuda")
    ft = _factor(a, True, nb)
    fp = _factor(a, False)
    assert ft.info == 0
    rt, lt = _residual(a, ft)
    rp, _ = _residual(a, fp)
    assert rt <= 10 * rp + 1e-6, (rt, rp)
    assert lt <= 1e3, lt


def test_tournament_lu_zero_column_and_ties():
    n = 700
    g = torch.Generator(device="cuda")
    g.manual_seed(3)
    a = torch.randn((n, n), generator=g, dtype=torch.float32, device="cuda")
    a[:, 45] = 0.0
    a[[10] + list(range(600, 610)), 0] = 10.0     # tied largest entries: the lower row
    ft = _factor(a, True)
    fp = _factor(a, False)
    assert fp.info == 46 and ft.info == 46
    assert int(ft.pivots[0]) == 10 and int(fp.pivots[0]) == 10
    assert torch.isfinite(ft.factored).all()
    rt, _ = _residual(a, ft)
    assert rt <= 1e-4, rt


@pytest.mark.parametrize("tournament,lookahead", [(True, -1), (True, 0), (False, -1)])
def test_ir_with_and_without_tournament(tournament, lookahead):
    from numax_b200 import _lib, linalg
    lib = _lib.load()
    ctx = _lib.context(torch.cuda.current_device())
    n = 2500
    rng = np.random.Generator(np.random.PCG64(17))
    a = rng.standard_normal((n, n)) / np.sqrt(n) + 2 * np.eye(n)
    b = rng.standard_normal(n)
    lib.nmx_tune_set(ctx, b"lu.tournament", -1 if tournament else 0)
    lib.nmx_tune_set(ctx, b"lu.lookahead", lookahead)
    try:
        x, st = linalg.solve_ir(torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda(),
                                precision="bf16x3", tol=1e-14)
    finally:
        lib.nmx_tune_set(ctx, b"lu.tournament", -1)
        lib.nmx_tune_set(ctx, b"lu.lookahead", -1)
    x = x.cpu().numpy()
    assert st["converged"] == 1, st
    berr = np.abs(b - a @ x).max() / (np.abs(a).sum(1).max() * np.abs(x).max() + np.abs(b).max())
    assert berr <= 1e-14
