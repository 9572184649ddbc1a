"""GPU checks of the batched persistent solver (configuration 3 shapes):
every problem of a mixed-size set solved to its FP64 true residual, with the
per-problem iteration counts of the single-problem CG."""
import numpy as np
import pytest

from oracle import oracle as O
from qex_b200 import _lib as L
from qex_b200 import fields as F
from qex_b200 import stag as S

pytestmark = pytest.mark.gpu

SHAPES = [(8, 8, 8, 8), (4, 4, 4, 8), (6, 6, 6, 6), (8, 8, 4, 4), (4, 6, 8, 4), (8, 4, 4, 8)]


def make_set(naik=False):
    rng = np.random.default_rng(7)
    probs = []
    for i, dims in enumerate(SHAPES):
        eps = rng.uniform(0.1, 0.5)
        g = F.fat_naik_links(dims, 50 + i) if naik else F.apply_phases(dims, F.gauge_warm(dims, eps, 50 + i))
        m = rng.uniform(0.02, 0.2)
        b = F.even_source(dims, 70 + i)
        probs.append((dims, g, m, b))
    return probs


@pytest.mark.parametrize("naik", [False, True])
def test_batched_matches_single_solves(cuda, naik):
    probs = make_set(naik)
    stags = [S.Staggered(S.Layout(d), g) for d, g, m, b in probs]
    xs = [np.zeros_like(b) for d, g, m, b in probs]
    sp = S.SolverParams(r2req=1e-20)
    out = S.solve_batched(stags, xs, [b for *_, b in probs], [m for _, _, m, _ in probs], sp)
    assert out["graph"]
    for (d, g, m, b), s, x, its, r2 in zip(probs, stags, xs, out["iterations"], out["r2"]):
        V = F.volume(d)
        o = O.Oracle(d, g)
        ax = o.vec()
        o.stagD2ee(ax, x, m * m)
        res = np.linalg.norm(ax[: V // 2] - b[: V // 2]) ** 2 / np.linalg.norm(b[: V // 2]) ** 2
        assert res <= 1e-20 and abs(res - r2) <= 1e-3 * r2
        assert not np.any(x[V // 2:])
        y = np.zeros_like(b)
        sp1 = S.SolverParams(r2req=1e-20)
        s.solveEE(y, b, m, sp1)
        assert abs(its - sp1.iterations) <= 1, (d, its, sp1.iterations)
        assert np.abs(x - y).max() / np.abs(y).max() < 1e-8


def test_batched_deterministic_and_device_path(cuda):
    torch = cuda
    probs = make_set(False)
    stags = [S.Staggered(S.Layout(d), S.to_device_links(g)) for d, g, m, b in probs]
    bs = [S.to_device_vector(b) for *_, b in probs]
    ms = [m for _, _, m, _ in probs]
    runs = []
    for _ in range(2):
        xs = [torch.zeros_like(b) for b in bs]
        out = S.solve_batched(stags, xs, bs, ms, S.SolverParams(r2req=1e-18))
        runs.append([x.cpu().numpy() for x in xs])
        assert (out["r2"] <= 1e-18).all()
    for a, b in zip(*runs):
        assert np.array_equal(a, b)


def test_batched_rejects_bad_input(cuda):
    probs = make_set(False)[:2]
    stags = [S.Staggered(S.Layout(d), g) for d, g, m, b in probs]
    xs = [np.zeros_like(b) for *_, b in probs]
    with pytest.raises(S.L.QexStagError):
        S.solve_batched([stags[0], stags[0]], xs, [b for *_, b in probs], [0.1, 0.1],
                        S.SolverParams(r2req=1e-20))
    with pytest.raises(S.L.QexStagError):
        S.solve_batched(stags, xs, [b for *_, b in probs], [0.1, 0.1],
                        S.SolverParams(r2req=1e-20, sloppySolve=S.L.SLOPPY_HALF))


def test_barrier_timeout_is_reported(cuda):
    """Failure detection without a GPU fault: the batched solver's grid
    barrier waits for a block that never arrives, gives up after its time
    limit, and the call reports QEXSTAG_ERR_TIMEOUT; the context stays
    usable (the barrier and a solve run afterwards)."""
    import time
    lib = L.load()
    assert lib.qexstag_barrier_selftest(0, 1000.0) == L.OK
    t0 = time.perf_counter()
    rc = lib.qexstag_barrier_selftest(1, 50.0)
    dt = time.perf_counter() - t0
    assert rc == L.ERR_TIMEOUT, rc
    assert "timed out" in lib.qexstag_last_error().decode()
    assert dt < 5.0, dt
    assert lib.qexstag_barrier_selftest(0, 1000.0) == L.OK
    assert lib.qexstag_barrier_selftest(-1, 50.0) == L.ERR_ARG
    dims = (4, 4, 4, 4)
    g = F.naive_links(dims, 0.3, 2)
    s = S.Staggered(S.Layout(dims), g)
    b = F.even_source(dims, 3)
    x = np.zeros_like(b)
    sp = S.SolverParams(r2req=1e-20)
    s.solveEE(x, b, 0.1, sp)
    assert sp.status == L.OK
