"""Test harness: an eager-torch HMC around the library's fermion force
(QEX src/hmc/hmcAction.nim), used by the GPU tests as an independent
restatement to check the device MD driver qex_b200/md.py against.

The fermion parts go through the library: the pseudofermion heatbath
(D(-m) psi, hmcAction.nim:794-823), the action (solve, 825-849), the force
solve and fermForce's outer products (669-790).  The gauge parts around them
are restated here in torch on the GPU, which is test and driver glue, not
the hot path:
  - Wilson action S_G = -(beta/3) sum_{x, mu<nu} Re Tr P_munu(x)
    (src/gauge/gaugeAction.nim:487-571) and its force;
  - fermion operator from thin links U: fat = U, long = c U(x)U(x+mu)U(x+2mu)
    (the Naik term of src/gauge/fat7l.nim:145-154, c = -1/24 for HISQ), phases
    folded in, and the chain rule of the long links back to U;
  - kinetic energy 0.5 |p|^2 - 16 V and leapfrog with U <- exp(eps p) U
    (hmcAction.nim:248-304, gaugeUtils.nim:453-475), reversibility check
    (hmcAction.nim:340-380).

Conventions.  For U -> exp(eps T) U with T anti-Hermitian, dS/deps =
Re Tr[T G^dagger]; the MD force is F = TAH(G) and p <- p - dtau F, which is
QEX's mdv with addForce(gf, 0.25*dtau, f) for the fermion part.  Link fields
here are complex128 torch tensors (nfields, V, 3, 3) in QEX's V=1 site order.
"""
from __future__ import annotations

import numpy as np
import torch

from qex_b200 import fields as F
from qex_b200 import stag as S


def dagger(m):
    return m.conj().transpose(-1, -2)


def tah(m):
    """projectTAH: traceless anti-Hermitian part."""
    a = 0.5 * (m - dagger(m))
    tr = torch.diagonal(a, dim1=-2, dim2=-1).sum(-1) / 3.0
    return a - tr[..., None, None] * torch.eye(3, dtype=m.dtype, device=m.device)


def exp_ah(x):
    """exp(x) for a batch of 3x3 matrices by scaling and squaring: x / 2^s has
    max-row-sum norm <= 1/2, its exponential is the Taylor series to order 16
    (truncation < 1e-20), then squared s times.  Batched matmuls only (the
    batched Hermitian eigensolver refuses batches of a 16^4 lattice's links)."""
    nrm = x.abs().sum(-1).amax().item()
    s = 0
    while nrm > 0.5:
        nrm *= 0.5
        s += 1
    y = x / float(2 ** s)
    eye = torch.eye(3, dtype=x.dtype, device=x.device).expand_as(y)
    r = eye + y / 16.0
    for k in range(15, 0, -1):
        r = eye + (y @ r) / float(k)
    for _ in range(s):
        r = r @ r
    return r


class Lattice:
    """Index tables of a 4-d lattice in QEX's V=1 site order, on the GPU."""

    def __init__(self, dims, device="cuda"):
        self.dims = tuple(int(d) for d in dims)
        self.V = F.volume(self.dims)
        c = F.coords(self.dims)
        self.device = device
        self.coords = c
        self.fwd, self.bck = {}, {}
        for mu in range(4):
            for n in (1, 2, 3):
                x = c.copy()
                x[:, mu] = (x[:, mu] + n) % self.dims[mu]
                self.fwd[(mu, n)] = torch.from_numpy(F.index_of(self.dims, x)).to(device)
                x = c.copy()
                x[:, mu] = (x[:, mu] - n) % self.dims[mu]
                self.bck[(mu, n)] = torch.from_numpy(F.index_of(self.dims, x)).to(device)
        self.sign1 = torch.stack([torch.from_numpy(F.link_signs(self.dims, mu, 1)) for mu in range(4)]).to(device)
        self.sign3 = torch.stack([torch.from_numpy(F.link_signs(self.dims, mu, 3)) for mu in range(4)]).to(device)

    def up(self, f, mu, n=1):
        """g(x) = f(x + n mu)"""
        return f[self.fwd[(mu, n)]]

    def dn(self, f, mu, n=1):
        """g(x) = f(x - n mu)"""
        return f[self.bck[(mu, n)]]


# ---------------------------------------------------------------------------
# Wilson gauge action
# ---------------------------------------------------------------------------

def staple_sum(lat: Lattice, U, mu):
    """Sum_nu of the staples closing U_mu(x) into plaquettes, so that the
    plaquettes through U_mu(x) sum to Re Tr[U_mu(x) Sigma_mu(x)]."""
    s = torch.zeros_like(U[0])
    for nu in range(4):
        if nu == mu:
            continue
        # U_nu(x+mu) U_mu(x+nu)^dag U_nu(x)^dag
        s = s + lat.up(U[nu], mu) @ dagger(lat.up(U[mu], nu)) @ dagger(U[nu])
        # U_nu(x+mu-nu)^dag U_mu(x-nu)^dag U_nu(x-nu)
        a = lat.dn(lat.up(U[nu], mu), nu)
        s = s + dagger(a) @ dagger(lat.dn(U[mu], nu)) @ lat.dn(U[nu], nu)
    return s


def wilson_action(lat: Lattice, U, beta: float) -> float:
    tot = 0.0
    for mu in range(4):
        for nu in range(mu):
            p = U[mu] @ lat.up(U[nu], mu) @ dagger(lat.up(U[mu], nu)) @ dagger(U[nu])
            tot += torch.diagonal(p, dim1=-2, dim2=-1).sum(-1).real.sum().item()
    return -(beta / 3.0) * tot


def wilson_force(lat: Lattice, U, beta: float):
    """F_mu = TAH(G), G = -(beta/3) (U Sigma)^dagger, i.e. (beta/3) TAH(U Sigma)."""
    return torch.stack([(beta / 3.0) * tah(U[mu] @ staple_sum(lat, U, mu)) for mu in range(4)])


# ---------------------------------------------------------------------------
# staggered fermion from thin links
# ---------------------------------------------------------------------------

class StaggeredFermion:
    """One pseudofermion with the fat+Naik operator built from thin links U:
    fat_mu = U_mu, long_mu = c U_mu(x) U_mu(x+mu) U_mu(x+2mu), phases folded.
    naik = None gives the naive operator (fat only)."""

    def __init__(self, lat: Lattice, mass: float, naik: float | None = -1.0 / 24.0,
                 r2req_action=1e-20, r2req_force=1e-18, sloppy=S.L.SLOPPY_HALF, hisq: bool = False):
        self.lat = lat
        self.mass = mass
        self.naik = naik
        self.lay = S.Layout(lat.dims)
        self.stag = None
        self.phi = None
        self.r2a, self.r2f, self.sloppy = r2req_action, r2req_force, sloppy
        self.solver_iterations = 0
        # HISQ: the operator's fat and long links are the library's HISQ
        # smearing of the phased thin links (hmcAction.nim:540-555), and the
        # force is its qexstag_hisq_force (smearing chain rule included)
        self.hisq = hisq
        if hisq:
            from qex_b200 import smear as SM
            self.sm = SM.Smear(self.lay)
            self.coef = SM.newHISQ()
            self.smear_seconds = 0.0

    def links(self, U):
        lat = self.lat
        fat = U * lat.sign1[:, :, None, None]
        if self.naik is None:
            return fat
        lng = torch.stack([U[mu] @ lat.up(U[mu], mu, 1) @ lat.up(U[mu], mu, 2) for mu in range(4)])
        lng = self.naik * lng * lat.sign3[:, :, None, None]
        g = torch.empty((8,) + tuple(U.shape[1:]), dtype=U.dtype, device=U.device)
        g[0::2] = fat
        g[1::2] = lng
        return g

    def phased_thin(self, U):
        return (U * self.lat.sign1[:, :, None, None]).permute(0, 2, 3, 1).contiguous()

    def set_links(self, U):
        if self.hisq:
            if self.stag is None:
                eye = torch.eye(3, dtype=U.dtype, device=U.device)
                init = eye.reshape(1, 3, 3, 1).expand(8, 3, 3, self.lat.V).contiguous()
                self.stag = S.Staggered(self.lay, init, long_coeff=self.coef.naik)
            self.sm.smear_into(self.stag, self.coef, self.phased_thin(U))
            return
        dev = self.links(U).permute(0, 2, 3, 1).contiguous()
        if self.stag is None:
            self.stag = S.Staggered(self.lay, dev, long_coeff=self.naik if self.naik else 1.0)
        else:
            self.stag.update_links(dev)

    def heatbath(self, U, gen: torch.Generator):
        """phi = D(-m) psi with psi Gaussian, odd sites zeroed (hmcAction.nim:794-823)."""
        self.set_links(U)
        V = self.lat.V
        psi = torch.complex(torch.randn((3, V), dtype=torch.float64, device="cuda", generator=gen),
                            torch.randn((3, V), dtype=torch.float64, device="cuda", generator=gen))
        phi = torch.zeros_like(psi)
        self.stag.D(phi, psi, -self.mass)
        phi[:, V // 2:] = 0
        self.phi = phi

    def action(self, U) -> float:
        """0.5 |D(-m)^-1 phi|^2 (hmcAction.nim:825-849)."""
        self.set_links(U)
        psi = torch.zeros_like(self.phi)
        sp = S.SolverParams(r2req=self.r2a, sloppySolve=self.sloppy)
        self.stag.solve(psi, self.phi, -self.mass, sp)
        self.solver_iterations += sp.iterations
        return 0.5 * (psi.abs() ** 2).sum().item()

    def outer(self, U):
        """fermForce's f1/f3 for the current phi (device layout -> matrix layout)."""
        self.set_links(U)
        psi = torch.zeros_like(self.phi)
        sp = S.SolverParams(r2req=self.r2f, sloppySolve=self.sloppy)
        self.stag.force_solve(psi, self.phi, self.mass, sp)
        self.solver_iterations += sp.iterations
        f = torch.zeros((self.stag.nlinks, 3, 3, self.lat.V), dtype=torch.complex128, device="cuda")
        self.stag.ferm_outer(f, psi)
        return f.permute(0, 3, 1, 2).contiguous()

    def force(self, U):
        """F = TAH(G) with dS_F/deps = Re Tr[T G^dagger]; S_F = 0.5|D(-m)^-1 phi|^2
        changes by Re Tr[dW f^dagger]/4 for a change dW of a phased link W."""
        lat = self.lat
        if self.hisq:
            if self.stag is None:
                self.set_links(U)
            f = torch.empty((4, 3, 3, lat.V), dtype=torch.complex128, device="cuda")
            sp = S.SolverParams(r2req=self.r2f, sloppySolve=self.sloppy)
            self.sm.force(self.stag, self.coef, self.phased_thin(U), f, self.phi, self.mass, sp)
            self.solver_iterations += sp.iterations
            # the generator acting on W = eta U acts on U the same way
            return 0.25 * f.permute(0, 3, 1, 2)
        f = self.outer(U)
        nl = f.shape[0]
        out = []
        for mu in range(4):
            k = 2 * mu if nl == 8 else mu
            # fat: W = eta U
            gd = U[mu] @ dagger(f[k] * lat.sign1[mu][:, None, None])
            if nl == 8:
                w = (self.naik * f[k + 1]) * lat.sign3[mu][:, None, None]  # dS/dL with L = U U U
                u0, u1, u2 = U[mu], lat.up(U[mu], mu, 1), lat.up(U[mu], mu, 2)
                gd = gd + u0 @ u1 @ u2 @ dagger(w)
                # y = x - mu: L(y) = U(y) U(x) U(x+mu)
                gd = gd + u0 @ u1 @ dagger(lat.dn(w, mu, 1)) @ lat.dn(U[mu], mu, 1)
                # y = x - 2mu: L(y) = U(y) U(y+mu) U(x)
                gd = gd + u0 @ dagger(lat.dn(w, mu, 2)) @ lat.dn(U[mu], mu, 2) @ lat.dn(U[mu], mu, 1)
            out.append(tah(dagger(gd)) * 0.25)
        return torch.stack(out)


# ---------------------------------------------------------------------------
# HMC
# ---------------------------------------------------------------------------

class HMC:
    def __init__(self, lat: Lattice, beta: float, fermion: StaggeredFermion | None):
        self.lat = lat
        self.beta = beta
        self.ferm = fermion

    def kinetic(self, p) -> float:
        return 0.5 * (p.abs() ** 2).sum().item() - 16.0 * self.lat.V

    def potential(self, U) -> float:
        v = wilson_action(self.lat, U, self.beta)
        if self.ferm is not None:
            v += self.ferm.action(U)
        return v

    def hamiltonian(self, U, p) -> float:
        return self.kinetic(p) + self.potential(U)

    def force(self, U):
        f = wilson_force(self.lat, U, self.beta)
        if self.ferm is not None:
            f = f + self.ferm.force(U)
        return f

    def leapfrog(self, U, p, tau: float, nsteps: int):
        eps = tau / nsteps
        p = p - 0.5 * eps * self.force(U)
        for i in range(nsteps):
            U = exp_ah(eps * p) @ U
            p = p - (eps if i < nsteps - 1 else 0.5 * eps) * self.force(U)
        return U, p


def random_momenta(lat: Lattice, gen: np.random.Generator):
    """randTah3 momenta on every link (gaugeUtils.nim:1466-1493)."""
    return torch.from_numpy(F.rand_tah(4 * lat.V, gen).reshape(4, lat.V, 3, 3)).to("cuda")


def trajectory_with_reversal(lat, U0, beta, mass, naik, tau, nsteps, seed=7, sloppy=S.L.SLOPPY_HALF,
                             r2req_action=1e-20, r2req_force=1e-20, hisq=False):
    """One trajectory from (U0, p0) and its reversal (flip p, evolve back).
    Returns a dict with H values, dH, and the reversibility errors."""
    gen = torch.Generator(device="cuda")
    gen.manual_seed(seed)
    ferm = StaggeredFermion(lat, mass, naik, r2req_action=r2req_action, r2req_force=r2req_force,
                            sloppy=sloppy, hisq=hisq)
    ferm.heatbath(U0, gen)
    hmc = HMC(lat, beta, ferm)
    p0 = random_momenta(lat, np.random.default_rng(seed))
    h0 = hmc.hamiltonian(U0, p0)
    U1, p1 = hmc.leapfrog(U0, p0, tau, nsteps)
    h1 = hmc.hamiltonian(U1, p1)
    U2, p2 = hmc.leapfrog(U1, -p1, tau, nsteps)
    h2 = hmc.hamiltonian(U2, p2)
    du = (U2 - U0).abs().max().item()
    dp = (p2 + p0).abs().max().item()
    return {"H0": h0, "H1": h1, "dH": h1 - h0, "H_reversed": h2, "dH_reversed": h2 - h0,
            "max_dU": du, "max_dp": dp, "plaquette_action": wilson_action(lat, U1, beta),
            "solver_iterations": ferm.solver_iterations}


def thermalize(lat, U, beta, ntraj, tau=1.0, nsteps=20, seed=11):
    """Pure-gauge HMC trajectories with Metropolis accept/reject
    (src/hmc/metropolis.nim) to bring a warm start near equilibrium."""
    rng = np.random.default_rng(seed)
    hmc = HMC(lat, beta, None)
    acc = 0
    for _ in range(ntraj):
        p = random_momenta(lat, rng)
        h0 = hmc.hamiltonian(U, p)
        U1, p1 = hmc.leapfrog(U, p, tau, nsteps)
        dh = hmc.hamiltonian(U1, p1) - h0
        if dh <= 0 or rng.random() < np.exp(-dh):
            U, acc = U1, acc + 1
    return U, acc
