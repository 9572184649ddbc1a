"""The oracle against QEX's own logged output (CPU only).

QEX's HISQ HMC regression runs (src/alphas/regression/*/*.log; the numbers
are in tests/golden/qex_alphas_regression_8x8x8x16.json, extracted by the
script beside it) start an 8^3 x 16 lattice cold, so the three solves made
before any molecular dynamics act on the HISQ smearing of unit links:
  1. the ratio pseudofermion's heatbath, D(-0.6)^-1 D(-0.005) eta
     (alphas.nim:722-745),
  2. the heavy action term, D(-0.6)^-1 phi with phi = D(-0.6) psi, odd half
     zeroed (alphas.nim:694-707),
  3. the ratio action term, D(-0.005)^-1 D(-0.6) hphi, hphi the heatbath's
     result with its odd half zeroed,
each through QEX's full-lattice solve (stagSolve.nim:469-557: left or right
even-odd preconditioning as the source's parities decide, CG on the even
Schur system, defect correction to r2 <= 1e-20 |b|^2).  QEX logged 26, 26
and 34 iterations in every run.  The sources came from QEX's MILC generator,
which is not restated here; on the free field every Gaussian source of the
same distribution sees the same spectrum, so the oracle, fed seeded numpy
Gaussians through the same sequence, must take the same iteration counts and
end at residuals of the same size.  This pins, against QEX itself: the
rephase before smearing (alphas/extra/qexsmear.nim:90-98), both fat7 levels,
projectU and the Naik term (9/8 and -1/24 times the phases on unit links),
the phases and the antiperiodic boundary, D and its Schur operator with
their normalisation, the solve's choice of preconditioning, and the CG's
stopping rule.  The fermion action QEX logged after those solves (24323)
lies within the spread of the oracle's over sources, which pins the
Gaussian draws' normalisation and the action's.
"""
import json
from pathlib import Path

import numpy as np
import pytest

from oracle import oracle as O
from qex_b200 import fields as F

GOLDEN = json.loads((Path(__file__).resolve().parent / "golden" / "qex_alphas_regression_8x8x8x16.json").read_text())


def _free_hisq_oracle(dims):
    V = int(np.prod(dims))
    thin = np.broadcast_to(np.eye(3, dtype=np.complex128), (4, V, 3, 3)).copy()
    phased = O.apply_phases(dims, thin)
    fat, lng = O.hisq_smear(dims, phased, lepage=0.0, naik=1.0)
    return phased, fat, lng, O.Oracle(dims, F.interleave(fat, lng))


def test_golden_params_are_this_workload():
    p = GOLDEN["params"]
    assert p["lattice"] == [8, 8, 8, 16] and p["gauge_start"] == "cold"
    assert (p["mass"], p["hasenbusch_mass"], p["action_r2req"]) == (0.005, 0.6, 1e-20)
    assert p["naik"] == pytest.approx(-1.0 / 24.0)
    assert [s["iterations"] for s in GOLDEN["solves"]] == [26, 26, 34]


def test_free_hisq_links():
    dims = tuple(GOLDEN["params"]["lattice"])
    phased, fat, lng, _ = _free_hisq_oracle(dims)
    eye = np.eye(3)
    # fat link 9/8 times the link's phase, long link -1/24 times the
    # product of the three phases it spans (boundary sign of the 3-hop)
    assert np.allclose(fat, 1.125 * phased[:, :, 0, 0][:, :, None, None] * eye, atol=1e-14)
    ratio = lng[:, :, 0, 0] / phased[:, :, 0, 0]
    assert np.allclose(np.abs(ratio), 1.0 / 24.0, atol=1e-15)
    assert np.allclose(lng, lng[:, :, 0, 0][:, :, None, None] * eye, atol=1e-15)


def _start_of_trajectory(o, V, p, seed):
    """The pseudofermion heatbath (alphas.nim:722-745) and the fermion action
    (alphas.nim:694-707) on seeded Gaussians with unit variance in each real
    component: ((iterations, r2/b2) of the three solves, S_F)."""
    m, mh, r2req = p["mass"], p["hasenbusch_mass"], p["action_r2req"]
    rng = np.random.default_rng(1000 + seed)

    def gaussian():
        return rng.standard_normal((V, 3)) + 1j * rng.standard_normal((V, 3))

    hpsi, psi = gaussian(), gaussian()
    phi, hphit, hphi = o.vec(), o.vec(), o.vec()
    o.D(phi, psi, -mh)
    o.D(hphit, hpsi, -m)
    runs = [o.solve(hphi, hphit, -mh, r2req)]
    phi[V // 2:] = 0
    hphi[V // 2:] = 0
    hpsit, x1, x2 = o.vec(), o.vec(), o.vec()
    o.D(hpsit, hphi, -mh)
    runs.append(o.solve(x1, phi, -mh, r2req))
    runs.append(o.solve(x2, hpsit, -m, r2req))
    return runs, 0.5 * (np.vdot(x1, x1).real + np.vdot(x2, x2).real)


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_start_of_trajectory_solves_match_qex_log(seed):
    p = GOLDEN["params"]
    dims = tuple(p["lattice"])
    _, _, _, o = _free_hisq_oracle(dims)
    runs, _ = _start_of_trajectory(o, int(np.prod(dims)), p, seed)
    for (its, r2), want in zip(runs, GOLDEN["solves"]):
        assert its == want["iterations"], (want["what"], its)
        lo, hi = want["r2_over_b2"]
        # the same size of final residual as QEX's (its sources differ)
        assert r2 <= p["action_r2req"] and lo / 4 <= r2 <= hi * 4, (want["what"], r2, lo, hi)


def test_start_of_trajectory_fermion_action_matches_qex_log():
    """S_F = (|psi|^2 + |hpsi|^2)/2 after the three solves.  Over Gaussian
    sources it spreads by about 165 (0.7 %) around 24600; QEX's one sample
    is 24323.  A factor in the normalisation of the Gaussian draws (QEX's
    randomComplexGaussian: unit variance in each real component) or of the
    action would move it by 50 % or more, so the oracle's mean over four
    sources must lie within 750 (4 standard deviations of the difference)."""
    p = GOLDEN["params"]
    dims = tuple(p["lattice"])
    _, _, _, o = _free_hisq_oracle(dims)
    actions = [_start_of_trajectory(o, int(np.prod(dims)), p, seed)[1] for seed in range(10, 14)]
    qex = float(np.mean(p["start_fermion_action"]))
    assert abs(np.mean(actions) - qex) <= 750.0, (actions, qex)
    assert p["start_gauge_action"] == 0.0  # the cold configuration


def test_fixture_is_what_the_logs_hold():
    """The committed fixture equals a fresh extraction from QEX's logs, where
    the QEX source tree is at hand (skipped elsewhere)."""
    import importlib.util
    path = Path(__file__).resolve().parent / "golden" / "extract_alphas_regression.py"
    spec = importlib.util.spec_from_file_location("extract_alphas_regression", path)
    ex = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(ex)
    if not (ex.DEFAULT_ROOT / "src/alphas/regression").is_dir():
        pytest.skip("QEX source tree not present")
    assert ex.extract() == GOLDEN
