"""The multi-shift and batched workloads at their stated sizes.

Multi-shift (a rational term of RHMC, src/solvers/cgm.nim:68-246 driven as
src/physics/stagSolve.nim:560-668): 24^3 x 48, fat+Naik fields of the solver
workload's recipe, m = 0.01, 12 shifts log-spaced from 1e-4 to 1, 8 Gaussian
right-hand sides, FP32 inner iterations with FP64 residuals, tolerance 1e-9
per shift (r2 <= 1e-18) for every (right-hand side, shift).

Batched: 64 independent naive staggered lattices drawn (seeded) from {8^4,
12^4, 16^4, 8^3 x 16}, each with its own warmSU(eps) field (eps ~ U[0.1,
0.5]) and mass (~ U[0.02, 0.2]), solved in one persistent launch under a
CUDA graph to r2 <= 1e-20, each checked with the oracle's stagD2ee.
"""
import numpy as np
import pytest

from oracle import oracle as O
from qex_b200 import _lib as L
from qex_b200 import fields as F
from qex_b200 import stag as S
from qex_b200.batched_bench import problem_set
from qex_b200.multishift_bench import shifts

pytestmark = pytest.mark.gpu


def test_multishift_24x24x24x48_12_shifts_8_rhs(cuda):
    torch = cuda
    dims = (24, 24, 24, 48)
    V = F.volume(dims)
    h = V // 2
    m = 0.01
    r2req = 1e-18
    g = F.fat_naik_links(dims, 21)
    s = S.Staggered(S.Layout(dims), S.to_device_links(g))
    sig = shifts(12)
    bs_h = [F.even_source(dims, 100 + j) for j in range(8)]
    bs = [S.to_device_vector(b) for b in bs_h]
    ys = [[torch.zeros((3, V), dtype=torch.complex128, device="cuda") for _ in sig] for _ in bs]
    sp = S.SolverParams(r2req=r2req, sloppySolve=L.SLOPPY_SINGLE)
    r2 = s.cgm_ee(m, sig, bs, ys, sp)
    assert sp.status == L.OK and r2.shape == (8, 12)
    assert (r2 <= r2req).all(), r2.max()
    # every (j, k) true residual again, with the FP64 operator
    ay = torch.zeros_like(ys[0][0])
    for j, b in enumerate(bs):
        b2 = (b[:, :h].abs() ** 2).sum().item()
        for k, sg in enumerate(sig):
            s.stagD2ee(ay, ys[j][k], m * m)
            res = ((ay[:, :h] + sg * ys[j][k][:, :h] - b[:, :h]).abs() ** 2).sum().item() / b2
            assert res <= r2req, (j, k, res)
            assert not ys[j][k][:, h:].any()
    # and with the oracle's operator for a few (right-hand side, shift)
    o = O.Oracle(dims, g)
    for j, k in ((0, 0), (7, 11), (3, 5)):
        y = S.to_host_vector(ys[j][k])
        a = o.vec()
        o.stagD2ee(a, y, m * m)
        b = bs_h[j]
        res = np.linalg.norm(a[:h] + sig[k] * y[:h] - b[:h]) ** 2 / np.linalg.norm(b[:h]) ** 2
        assert res <= r2req, (j, k, res)


def test_batched_64_uneven_lattices(cuda):
    torch = cuda
    probs = problem_set(64)
    assert {p[0] for p in probs} == {(8, 8, 8, 8), (12, 12, 12, 12), (16, 16, 16, 16), (8, 8, 8, 16)}
    stags = [S.Staggered(S.Layout(d), S.to_device_links(g)) for d, g, m, b in probs]
    bs = [S.to_device_vector(b) for *_, b in probs]
    ms = [m for _, _, m, _ in probs]
    for rep in range(2):  # the first call tunes the launch, the second replays the graph
        xs = [torch.zeros_like(b) for b in bs]
        sp = S.SolverParams(r2req=1e-20)
        out = S.solve_batched(stags, xs, bs, ms, sp)
        assert out["graph"] and sp.status == L.OK
    for (d, g, m, b), x, r2 in zip(probs, xs, out["r2"]):
        V = F.volume(d)
        o = O.Oracle(d, g)
        xh = S.to_host_vector(x)
        ax = o.vec()
        o.stagD2ee(ax, xh, m * m)
        res = np.linalg.norm(ax[: V // 2] - b[: V // 2]) ** 2 / np.linalg.norm(b[: V // 2]) ** 2
        assert res <= 1e-20 and abs(res - r2) <= 1e-3 * r2, (d, res, r2)
        assert not np.any(xh[V // 2:])
