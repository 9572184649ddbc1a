"""The library against QEX's own logged output, on the GPU.

The same three start-of-trajectory solves as test_oracle_qex_regression.py
(QEX's HISQ HMC regression runs, 8^3 x 16 cold start, m = 0.005 with a
Hasenbusch mass of 0.6; tests/golden/qex_alphas_regression_8x8x8x16.json),
here with every step in the library through the C ABI: the phased unit links
smeared by qexstag_hisq_smear, D by qexstag_D and the solves by
qexstag_solve (FP64).  QEX logged 26, 26 and 34 iterations.
"""
import json
from pathlib import Path

import numpy as np
import pytest

from qex_b200 import fields as F
from qex_b200 import smear as SM
from qex_b200 import stag as S

pytestmark = pytest.mark.gpu

GOLDEN = json.loads((Path(__file__).resolve().parent / "golden" / "qex_alphas_regression_8x8x8x16.json").read_text())


@pytest.mark.parametrize("seed", [0, 1])
def test_library_start_of_trajectory_solves_match_qex_log(cuda, seed):
    p = GOLDEN["params"]
    dims = tuple(p["lattice"])
    m, mh, r2req = p["mass"], p["hasenbusch_mass"], p["action_r2req"]
    V = F.volume(dims)
    lay = S.Layout(dims)
    thin = np.broadcast_to(np.eye(3, dtype=np.complex128), (4, V, 3, 3)).copy()
    fat, lng = SM.hisq_smear(lay, F.apply_phases(dims, thin), SM.newHISQ(lepage=0.0, naik=1.0))
    assert np.allclose(np.abs(fat[:, :, 0, 0]), 1.125, atol=1e-14)
    assert np.allclose(np.abs(lng[:, :, 0, 0]), 1.0 / 24.0, atol=1e-15)
    s = S.Staggered(lay, F.interleave(fat, lng), long_coeff=p["naik"])
    rng = np.random.default_rng(2000 + seed)

    def gaussian():
        return rng.standard_normal((V, 3)) + 1j * rng.standard_normal((V, 3))

    def vec():
        return np.zeros((V, 3), dtype=np.complex128)

    def solve(x, b, mass):
        sp = S.SolverParams(r2req=r2req)
        s.solve(x, b, mass, sp)
        return sp.iterations, sp.r2

    # pseudofermion heatbath (alphas.nim:722-745)
    hpsi, psi = gaussian(), gaussian()
    phi, hphit, hphi = vec(), vec(), vec()
    s.D(phi, psi, -mh)
    s.D(hphit, hpsi, -m)
    runs = [solve(hphi, hphit, -mh)]
    phi[V // 2:] = 0
    hphi[V // 2:] = 0
    # fermion action (alphas.nim:694-707)
    hpsit, x1, x2 = vec(), vec(), vec()
    s.D(hpsit, hphi, -mh)
    runs.append(solve(x1, phi, -mh))
    runs.append(solve(x2, hpsit, -m))
    for (its, r2), want in zip(runs, GOLDEN["solves"]):
        assert its == want["iterations"], (want["what"], its)
        lo, hi = want["r2_over_b2"]
        assert r2 <= r2req and lo / 4 <= r2 <= hi * 4, (want["what"], r2, lo, hi)
