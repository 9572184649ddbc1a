"""Molecular dynamics on the device through the C ABI (scope row F4): QEX's
HMC step (src/hmc/hmcAction.nim:248-304: kineticAction, mdt = axexpmuly,
mdv = p -= forces) with every field operation a library kernel.
  - gauge action and force: qexstag_gauge_action / qexstag_gauge_force
    (Wilson, or plaquette + rectangle via gaugeActRect);
  - link update U <- expAH(eps p) U: qexstag_link_update;
  - momenta: qexstag_momenta_heatbath (randomTAH), qexstag_momenta_update,
    qexstag_kinetic_action;
  - fermion (optional): one staggered pseudofermion of the HISQ-smeared
    operator, or of the thin-link fat + Naik operator (fat = U, long =
    naik U U U, as smearing coefficients with one-link terms only), action
    by the library's solve and force by qexstag_hisq_force.
Fields: device complex128 tensors (4, 3, 3, V) in the library's link layout
(thin links without phases; the phases are folded in for the fermion).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L
from . import fields as F
from . import smear as SM
from . import stag as S


def _p(t):
    return C.c_void_p(t.data_ptr())


class GaugeAction:
    """GaugeActionCoeffs (gaugeAction.nim:14-19)."""

    def __init__(self, layout: S.Layout, beta: float, c1: float = 0.0):
        self.l = layout
        self.c = L.GaugeCoefsC()
        L.load().qexstag_gauge_coefs_rect(C.byref(self.c), float(beta), float(c1))

    def action(self, U) -> float:
        out = C.c_double()
        L.check(L.load().qexstag_gauge_action(self.l.handle, C.byref(self.c), _p(U), L.MEM_DEVICE, C.byref(out)),
                "gauge_action")
        return out.value

    def force(self, U, f) -> None:
        L.check(L.load().qexstag_gauge_force(self.l.handle, C.byref(self.c), _p(U), _p(f), L.MEM_DEVICE),
                "gauge_force")


def link_update(layout, U, P, eps: float) -> None:
    L.check(L.load().qexstag_link_update(layout.handle, _p(U), _p(P), float(eps), L.MEM_DEVICE), "link_update")


def momenta_update(layout, P, f, a: float) -> None:
    L.check(L.load().qexstag_momenta_update(layout.handle, _p(P), _p(f), float(a), L.MEM_DEVICE),
            "momenta_update")


def momenta_heatbath(layout, P, seed: int, counter: int) -> None:
    L.check(L.load().qexstag_momenta_heatbath(layout.handle, _p(P), int(seed), int(counter), L.MEM_DEVICE),
            "momenta_heatbath")


def kinetic_action(layout, P) -> float:
    out = C.c_double()
    L.check(L.load().qexstag_kinetic_action(layout.handle, _p(P), L.MEM_DEVICE, C.byref(out)), "kinetic_action")
    return out.value


class StaggeredPseudofermion:
    """S_F = 0.5 |D(-m)^-1 phi|^2 with the fat/long links smeared from the
    phased thin links (hmcAction.nim:794-885)."""

    def __init__(self, layout: S.Layout, mass: float, hisq: bool = True, naik: float = -1.0 / 24.0,
                 r2req_action=1e-20, r2req_force=1e-20, sloppy=L.SLOPPY_HALF):
        import torch
        self.l = layout
        self.mass = mass
        self.sm = SM.Smear(layout)
        if hisq:
            self.coef = SM.newHISQ()
        else:
            one = SM.Fat7lCoefs(1.0, 0.0, 0.0, 0.0, 0.0)
            self.coef = SM.HisqCoefs(one, SM.Fat7lCoefs(1.0, 0.0, 0.0, 0.0, 0.0), naik, 1e-20)
        V = layout.V
        eye = torch.eye(3, dtype=torch.complex128, device="cuda").reshape(1, 3, 3, 1).expand(8, 3, 3, V)
        self.stag = S.Staggered(layout, eye.contiguous(), long_coeff=self.coef.naik or 1.0)
        signs = np.stack([F.link_signs(layout.dims, mu, 1) for mu in range(4)])
        self.signs = torch.from_numpy(signs).to("cuda").reshape(4, 1, 1, V).to(torch.complex128)
        self.r2a, self.r2f, self.sloppy = r2req_action, r2req_force, sloppy
        self.phi = None
        self.solver_iterations = 0

    def phased(self, U):
        return (U * self.signs).contiguous()

    def heatbath(self, U, gen) -> None:
        import torch
        V = self.l.V
        self.sm.smear_into(self.stag, self.coef, self.phased(U))
        psi = torch.complex(torch.randn((3, V), dtype=torch.float64, device="cuda", generator=gen),
                            torch.randn((3, V), dtype=torch.float64, device="cuda", generator=gen))
        phi = torch.zeros_like(psi)
        self.stag.D(phi, psi, -self.mass)
        phi[:, V // 2:] = 0
        self.phi = phi

    def action(self, U) -> float:
        import torch
        self.sm.smear_into(self.stag, self.coef, self.phased(U))
        psi = torch.zeros_like(self.phi)
        sp = S.SolverParams(r2req=self.r2a, sloppySolve=self.sloppy)
        self.stag.solve(psi, self.phi, -self.mass, sp)
        self.solver_iterations += sp.iterations
        return 0.5 * float((psi.abs() ** 2).sum())

    def force(self, U, f) -> None:
        """f = the MD force, 0.25 times QEX's fermForce output (addForce(gf,
        0.25*dtau, f))."""
        sp = S.SolverParams(r2req=self.r2f, sloppySolve=self.sloppy)
        self.sm.force(self.stag, self.coef, self.phased(U), f, self.phi, self.mass, sp)
        self.solver_iterations += sp.iterations
        f.mul_(0.25)


class MD:
    def __init__(self, layout: S.Layout, gauge: GaugeAction, fermion: StaggeredPseudofermion | None = None):
        import torch
        self.l = layout
        self.gauge = gauge
        self.ferm = fermion
        self._fg = torch.empty((4, 3, 3, layout.V), dtype=torch.complex128, device="cuda")
        self._ff = torch.empty_like(self._fg)

    def potential(self, U) -> float:
        v = self.gauge.action(U)
        if self.ferm is not None:
            v += self.ferm.action(U)
        return v

    def hamiltonian(self, U, P) -> float:
        return kinetic_action(self.l, P) + self.potential(U)

    def mdv(self, U, P, eps: float) -> None:
        """p -= eps F (QEX's mdv: forces summed, p -= f)."""
        self.gauge.force(U, self._fg)
        momenta_update(self.l, P, self._fg, -eps)
        if self.ferm is not None:
            self.ferm.force(U, self._ff)
            momenta_update(self.l, P, self._ff, -eps)

    def leapfrog(self, U, P, tau: float, nsteps: int) -> None:
        """In place: half step in p, nsteps of (U, p), last p step halved."""
        eps = tau / nsteps
        self.mdv(U, P, 0.5 * eps)
        for i in range(nsteps):
            link_update(self.l, U, P, eps)
            self.mdv(U, P, eps if i < nsteps - 1 else 0.5 * eps)

    def omelyan(self, U, P, tau: float, nsteps: int, lam: float = 0.1931833275037836) -> None:
        """In place: Omelyan's second-order minimum-norm integrator (Omelyan,
        Mryglod and Folk, Comput. Phys. Commun. 151 (2003) 272), QEX's
        default "2MN" (hmcAction.nim:230, from the mdevolve package).  Per
        step p += lam eps F, U by eps/2, p += (1 - 2 lam) eps F, U by eps/2,
        p += lam eps F, the closing kick merged with the next step's opening
        one: two force evaluations per step."""
        eps = tau / nsteps
        self.mdv(U, P, lam * eps)
        for i in range(nsteps):
            link_update(self.l, U, P, 0.5 * eps)
            self.mdv(U, P, (1.0 - 2.0 * lam) * eps)
            link_update(self.l, U, P, 0.5 * eps)
            self.mdv(U, P, 2.0 * lam * eps if i < nsteps - 1 else lam * eps)

    def integrate(self, U, P, tau: float, nsteps: int, integrator: str = "leapfrog") -> None:
        if integrator == "leapfrog":
            self.leapfrog(U, P, tau, nsteps)
        elif integrator == "omelyan":
            self.omelyan(U, P, tau, nsteps)
        else:
            raise ValueError(f"unknown integrator {integrator!r}")


def plaquette(layout, U) -> float:
    """Average plaquette Re Tr P / 3 from the Wilson action at beta = 3."""
    return -GaugeAction(layout, 3.0).action(U) / (6.0 * layout.V * 3.0)


def hmc(layout, U, beta, fermion, ntraj, tau=1.0, nsteps=20, integrator="omelyan", seed=7, counter0=0,
        accept_seed=11):
    """ntraj HMC trajectories from U (QEX's hmc loop: momenta heatbath,
    pseudofermion heatbath, molecular dynamics, Metropolis accept/reject with
    probability min(1, exp(-dH))).  Returns the final links and one record
    per trajectory (dH, accepted, plaquette after)."""
    import torch
    md = MD(layout, GaugeAction(layout, beta), fermion)
    rng = np.random.default_rng(accept_seed)
    gen = torch.Generator(device="cuda")
    gen.manual_seed(seed)
    P = torch.empty_like(U)
    out = []
    for t in range(ntraj):
        momenta_heatbath(layout, P, seed, counter0 + t)
        if fermion is not None:
            fermion.heatbath(U, gen)
        h0 = md.hamiltonian(U, P)
        U1 = U.clone()
        md.integrate(U1, P, tau, nsteps, integrator)
        dh = md.hamiltonian(U1, P) - h0
        acc = bool(dh <= 0 or rng.random() < np.exp(-dh))
        if acc:
            U = U1
        out.append({"dH": dh, "accepted": acc, "plaquette": plaquette(layout, U)})
    return U, out


def trajectory_with_reversal(layout, U0, beta, tau, nsteps, fermion=None, seed=7, counter=0, P0=None):
    """One trajectory from (U0, P0) and back with flipped momenta."""
    import torch
    md = MD(layout, GaugeAction(layout, beta), fermion)
    U = U0.clone()
    if P0 is None:
        P = torch.empty_like(U)
        momenta_heatbath(layout, P, seed, counter)
    else:
        P = P0.clone()
    Pstart = P.clone()
    h0 = md.hamiltonian(U, P)
    md.leapfrog(U, P, tau, nsteps)
    h1 = md.hamiltonian(U, P)
    P.neg_()
    md.leapfrog(U, P, tau, nsteps)
    h2 = md.hamiltonian(U, P)
    return {"H0": h0, "H1": h1, "dH": h1 - h0, "dH_reversed": h2 - h0,
            "max_dU": float((U - U0).abs().max()), "max_dp": float((P + Pstart).abs().max())}


def time_gauge_kernels(dims, reps=5):
    """Device times of the gauge force, action and link update at dims."""
    import torch
    lay = S.Layout(dims)
    U = S.to_device_links(F.gauge_warm(dims, 0.3, 3))
    P = torch.empty_like(U)
    f = torch.empty_like(U)
    momenta_heatbath(lay, P, 1, 0)
    out = {}
    for name, c1 in (("wilson", 0.0), ("symanzik", -1.0 / 12)):
        ga = GaugeAction(lay, 5.6, c1)
        for what, fn in (("force", lambda: ga.force(U, f)), ("action", lambda: ga.action(U))):
            fn()
            torch.cuda.synchronize()
            ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
            ev[0].record()
            for _ in range(reps):
                fn()
            ev[1].record()
            torch.cuda.synchronize()
            out[f"{what}_{name}_ms"] = ev[0].elapsed_time(ev[1]) / reps
    V0 = U.clone()
    link_update(lay, V0, P, 0.01)
    torch.cuda.synchronize()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    ev[0].record()
    for _ in range(reps):
        link_update(lay, V0, P, 0.01)
    ev[1].record()
    torch.cuda.synchronize()
    out["link_update_ms"] = ev[0].elapsed_time(ev[1]) / reps
    return out


def main():
    """Config-4-shaped run with the device MD: 16^4, beta 5.6 Wilson (or
    Symanzik with --c1), one pseudofermion (HISQ, or thin fat + Naik with
    --thin), m = 0.05, tau = 1, 20 leapfrog steps, and the reversed
    trajectory; plus the gauge kernels' device times at --kdims."""
    import argparse
    import json
    import time
    import torch
    ap = argparse.ArgumentParser()
    ap.add_argument("--dims", default="16,16,16,16")
    ap.add_argument("--kdims", default="32,32,32,32")
    ap.add_argument("--beta", type=float, default=5.6)
    ap.add_argument("--c1", type=float, default=0.0)
    ap.add_argument("--mass", type=float, default=0.05)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--thin", action="store_true")
    ap.add_argument("--hmc", type=int, default=0,
                    help="run this many HMC trajectories with accept/reject instead (after --therm)")
    ap.add_argument("--therm", type=int, default=20, help="pure-gauge trajectories before --hmc")
    ap.add_argument("--settle", type=int, default=3, help="trajectories with the fermion before measuring")
    ap.add_argument("--integrator", default="omelyan", choices=["leapfrog", "omelyan"])
    a = ap.parse_args()
    dims = tuple(int(v) for v in a.dims.split(","))
    S.init(0)
    lay = S.Layout(dims)
    U0 = S.to_device_links(F.gauge_warm(dims, 0.3, 41))
    ferm = StaggeredPseudofermion(lay, a.mass, hisq=not a.thin)
    if a.hmc > 0:
        t0 = time.perf_counter()
        U, th = hmc(lay, U0, a.beta, None, a.therm, nsteps=a.steps, integrator=a.integrator, seed=3)
        U, st = hmc(lay, U, a.beta, ferm, a.settle, nsteps=a.steps, integrator=a.integrator, seed=5,
                    counter0=10000)
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        U, rec = hmc(lay, U, a.beta, ferm, a.hmc, nsteps=a.steps, integrator=a.integrator, seed=9, counter0=20000)
        torch.cuda.synchronize()
        t2 = time.perf_counter()
        dh = np.array([r["dH"] for r in rec])
        ex = np.exp(-dh)
        print(json.dumps({
            "dims": dims, "beta": a.beta, "mass": a.mass, "fermion": "thin fat+Naik" if a.thin else "hisq",
            "integrator": a.integrator, "steps": a.steps, "tau": 1.0,
            "thermalization": {"pure_gauge": a.therm, "accepted": sum(r["accepted"] for r in th),
                               "with_fermion": a.settle, "plaquette": th[-1]["plaquette"] if th else None},
            "trajectories": rec, "acceptance": float(np.mean([r["accepted"] for r in rec])),
            "mean_abs_dH": float(np.abs(dh).mean()), "mean_exp_minus_dH": float(ex.mean()),
            "exp_minus_dH_stderr": float(ex.std(ddof=1) / np.sqrt(len(ex))) if len(ex) > 1 else None,
            "seconds_per_trajectory": (t2 - t1) / a.hmc, "seconds_thermalization": t1 - t0}))
        return
    gen = torch.Generator(device="cuda")
    gen.manual_seed(7)
    ferm.heatbath(U0, gen)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    m = MD(lay, GaugeAction(lay, a.beta, a.c1), ferm)
    U = U0.clone()
    P = torch.empty_like(U)
    momenta_heatbath(lay, P, 7, 0)
    P0 = P.clone()
    h0 = m.hamiltonian(U, P)
    m.leapfrog(U, P, 1.0, a.steps)
    h1 = m.hamiltonian(U, P)
    P.neg_()
    m.leapfrog(U, P, 1.0, a.steps)
    h2 = m.hamiltonian(U, P)
    torch.cuda.synchronize()
    secs = time.perf_counter() - t0
    out = {"dims": dims, "fermion": "thin fat+Naik" if a.thin else "hisq", "dH": h1 - h0, "dH_reversed": h2 - h0,
           "max_dU": float((U - U0).abs().max()), "max_dp": float((P + P0).abs().max()),
           "solver_iterations": ferm.solver_iterations, "seconds_two_trajectories": secs,
           "kernels": time_gauge_kernels(tuple(int(v) for v in a.kdims.split(",")))}
    print(json.dumps(out))


if __name__ == "__main__":
    main()
