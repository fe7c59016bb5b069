"""Synthetic EGSnrc-style physics tables for the transport kernels.

The reference builds its tables in HATCH from PEGS4 files and the EGSnrc data
files ``si_*.data``, ``pgs4form.dat``, ``msnew.data``, ``incoh.data``,
``photo_relax.data``, ``photo_cs.data`` and ``eii_ik.data``
(``media.cu:332-1292``, ``PhysicsInit.cu:187-2047``).  None of those files is
available, so this module computes every table from documented closed-form
models and writes them in the reference's in-memory layout
(:mod:`gegs_b200.physics_layout`).  The CUDA kernels and the CPU oracle read
the same block, so GPU/CPU parity is exact; parity against real EGSnrc data is
unpinned.

Models (all per atom unless noted):

* Compton: Klein-Nishina total cross section x Z.
* Photo-absorption: ``c_Z E^-3.5`` above the K edge, divided by shell jump
  ratios below each edge (edges from screened Moseley scaling).
* Rayleigh: hydrogen-like form factor ``Z (1+(x/x0)^2)^-2`` with
  ``x0 = 0.3 Z^(1/3)`` 1/Angstrom; total cross section by quadrature.
* Pair (+triplet): ``alpha r0^2 Z(Z+1) (28/9 ln 2k - 218/27)`` with a cubic
  threshold taper.
* Electrons: restricted collision stopping power (ICRU 37 / Berger-Seltzer
  form with Sternheimer density effect), bremsstrahlung from the EGS4 screening
  fits (same functions the sampler uses), Moller / Bhabha / Heitler
  annihilation totals, Moliere ``b_c`` and ``chi_c`` (Bethe 1953).
* Multiple scattering: Goudsmit-Saunderson distribution of the screened
  Rutherford cross section (Legendre series, moments via Legendre functions of
  the second kind), minus its no- and single-scattering terms, tabulated in the
  reference's ``u`` variable with alias tables (Kawrakow & Bielajew 1998).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from . import physics_layout as L

RM = 0.5110034          # electron rest energy used by the reference (CUDA_EGS.h:141)
R0 = 2.8179403e-13      # classical electron radius, cm
ALPHA = 1.0 / 137.035999
BARN = 1e-24
INV_1P66 = 1.0 / 1.6605655   # barn * N_A (reference con2, media.cu:873)
HC_INV = 80.65506856998      # 1/(Angstrom MeV) (CUDA_EGS.h:143)

# ---------------------------------------------------------------------------
# elements and media
# ---------------------------------------------------------------------------
ELEMENTS = {  # Z: (symbol, atomic weight, mean excitation energy eV)
    1: ("H", 1.00794, 19.2), 6: ("C", 12.011, 78.0), 7: ("N", 14.0067, 82.0),
    8: ("O", 15.9994, 95.0), 15: ("P", 30.9738, 173.0), 18: ("AR", 39.948, 188.0),
    20: ("CA", 40.078, 191.0), 74: ("W", 183.84, 727.0),
}


@dataclass
class Medium:
    name: str
    rho: float                     # standard density g/cm^3
    mass_fractions: dict           # Z -> mass fraction
    gas: bool = False
    ae: float = 0.7                # total-energy electron cut (MeV)
    ap: float = 0.01               # photon cut (MeV)
    ue: float = 20.0 + RM
    up: float = 20.0

    @property
    def elements(self):
        zs = sorted(self.mass_fractions)
        w = np.array([self.mass_fractions[z] for z in zs], float)
        w = w / w.sum()
        a = np.array([ELEMENTS[z][1] for z in zs])
        pz = w / a          # moles of atoms per gram: sum(pz*A) == 1
        return np.array(zs, float), pz, a


MEDIA = {
    "AIR700ICRU": Medium("AIR700ICRU", 0.00120479, {6: 0.000124, 7: 0.755268, 8: 0.231781, 18: 0.012827}, gas=True),
    "H2O700ICRU": Medium("H2O700ICRU", 1.0, {1: 0.111894, 8: 0.888106}),
    "LUNG700ICRU": Medium("LUNG700ICRU", 1.05, {1: 0.103, 6: 0.105, 7: 0.031, 8: 0.761}),
    "ICRUTISSUE700ICRU": Medium("ICRUTISSUE700ICRU", 1.0, {1: 0.101, 6: 0.111, 7: 0.026, 8: 0.762}),
    "ICRPBONE700ICRU": Medium("ICRPBONE700ICRU", 1.85, {1: 0.047234, 6: 0.14433, 7: 0.04199, 8: 0.446096,
                                                        15: 0.10497, 20: 0.20993}),
    "W700ICRU": Medium("W700ICRU", 19.3, {74: 1.0}),
}

SHELLS = ("K", "L1", "L2", "L3", "M", "N")
JUMP = np.array([6.0, 1.15, 1.4, 2.6, 3.0, 1.5])


def binding_energies(z: int) -> np.ndarray:
    """K, L1, L2, L3, M, N binding energies in MeV (screened Moseley scaling)."""
    ry = 13.6e-6
    b = np.zeros(6)
    b[0] = ry * max(z - 1.0, 1.0) ** 2 if z > 1 else ry
    if z >= 3:
        b[1] = ry * (z - 4.15) ** 2 / 4.0 if z > 5 else ry * 0.25
    if z >= 5:
        b[2] = 0.93 * b[1]
        b[3] = 0.85 * b[1]
    if z >= 11:
        b[4] = ry * (z - 11.25) ** 2 / 9.0
    if z >= 19:
        b[5] = ry * (z - 21.15) ** 2 / 16.0
    return b


def shell_electrons(z: int):
    """(binding MeV, electrons, J0 in atomic units) for the Compton shells of element z."""
    b = binding_energies(z)
    out = []
    left = z
    # shell capacities and Slater-like screening constants
    spec = [(b[0], 2, 0.3, 1), (np.mean(b[1:4]) if z >= 3 else 0.0, 8, 4.15, 2),
            (b[4], 18, 11.25, 3), (b[5], 32, 21.15, 4)]
    for be, cap, s, n in spec:
        if left <= 0:
            break
        ne = min(cap, left)
        left -= ne
        zeff = max(z - s, 1.0)
        j0 = 0.849 * n / zeff          # hydrogenic J(0) scaling
        out.append((max(be, 1e-6), ne, j0))
    if left > 0:  # outermost electrons of heavy atoms
        out.append((5e-6, left, 0.849 * 5 / 1.5))
    return out


# ---------------------------------------------------------------------------
# photon cross sections (barns per atom)
# ---------------------------------------------------------------------------
def sigma_kn(e):
    """Klein-Nishina total cross section per electron (barns)."""
    k = np.asarray(e, float) / RM
    l2k = np.log1p(2 * k)
    s = ((1 + k) / k ** 2 * (2 * (1 + k) / (1 + 2 * k) - l2k / k) + l2k / (2 * k)
         - (1 + 3 * k) / (1 + 2 * k) ** 2)
    return 2 * math.pi * R0 ** 2 * s / BARN


def photo_c(z):
    return 2.66e-5 * (z / 8.0) ** 4.5


def sigma_photo(z, e):
    e = np.asarray(e, float)
    b = binding_energies(int(z))
    jump = np.ones_like(e)
    for s in range(6):
        if b[s] > 0:
            jump = np.where(e < b[s], jump * JUMP[s], jump)
    return photo_c(z) * e ** -3.5 / jump


def form_factor(z, x):
    x0 = 0.3 * z ** (1.0 / 3.0)
    return z / (1 + (x / x0) ** 2) ** 2


def sigma_rayleigh(z, e):
    e = np.atleast_1d(np.asarray(e, float))
    mu, w = np.polynomial.legendre.leggauss(400)
    # refine near mu=1 (forward peak): integrate in t=(1-mu)/2 on a log grid
    t = np.logspace(-12, 0, 1200)
    out = np.empty_like(e)
    for i, ee in enumerate(e):
        x = ee * HC_INV * np.sqrt(t)
        f = (1 + (1 - 2 * t) ** 2) * form_factor(z, x) ** 2
        out[i] = math.pi * R0 ** 2 * 2 * np.trapezoid(f, t) / BARN
    return out


def sigma_pair(z, e):
    k = np.asarray(e, float) / RM
    p = 28.0 / 9.0 * np.log(2 * np.maximum(k, 4.0)) - 218.0 / 27.0
    p4 = 28.0 / 9.0 * math.log(8.0) - 218.0 / 27.0
    p = np.where(k < 4.0, p4 * np.clip((k - 2.0) / 2.0, 0, None) ** 3, p)
    return ALPHA * R0 ** 2 * z * (z + 1) * np.maximum(p, 0.0) / BARN


# ---------------------------------------------------------------------------
# electron helpers
# ---------------------------------------------------------------------------
def fcoulc(z):
    """Coulomb correction f_c(Z) (Davies, Bethe & Maximon 1954)."""
    a2 = (ALPHA * z) ** 2
    return a2 * (1 / (1 + a2) + 0.20206 - 0.0369 * a2 + 0.0083 * a2 ** 2 - 0.002 * a2 ** 3)


def xsif(z):
    """Tsai's ratio of atomic-electron to nuclear bremsstrahlung."""
    return math.log(1440 * z ** (-2.0 / 3.0)) / (math.log(183 * z ** (-1.0 / 3.0)) - fcoulc(z))


def phi12(delta):
    """EGS4 fits of the Thomas-Fermi screening functions (SLAC-265)."""
    d = np.asarray(delta, float)
    lo = d <= 1
    p1 = np.where(lo, 20.863 - 3.242 * d + 0.625 * d * d, 21.12 - 4.184 * np.log(d + 0.952))
    p2 = np.where(lo, 20.029 - 1.930 * d - 0.086 * d * d, 21.12 - 4.184 * np.log(d + 0.952))
    return p1, p2


@dataclass
class MediumTables:
    med: Medium
    z: np.ndarray
    pz: np.ndarray
    a: np.ndarray
    extras: dict = field(default_factory=dict)


def _line_fit(values, loge, nbins):
    """Log-linear pairs: bin j spans points j..j+1; last bin copies the slope."""
    out = np.zeros((nbins, 2))
    values = np.asarray(values, float)
    loge = np.asarray(loge, float)
    nfit = min(len(values) - 1, nbins)
    b = (values[1:nfit + 1] - values[:nfit]) / (loge[1:nfit + 1] - loge[:nfit])
    out[:nfit, 1] = b
    out[:nfit, 0] = values[1:nfit + 1] - b * loge[1:nfit + 1]
    for j in range(nfit, nbins):
        out[j, 1] = out[j - 1, 1]
        out[j, 0] = values[j] - out[j, 1] * loge[j]
    return out


def density_effect(med: Medium, beta_gamma, i_ev, ne_per_g):
    """Sternheimer density-effect correction delta(beta*gamma)."""
    hw = 28.816 * math.sqrt(med.rho * ne_per_g / 6.02214e23)       # plasma energy eV
    cbar = 2 * math.log(i_ev / hw) + 1
    if med.gas:
        x0 = 1.6 if cbar < 10 else 0.326 * cbar - 1.5
        x1 = 4.0
    else:
        if i_ev < 100:
            x0 = 0.2 if cbar < 3.681 else 0.326 * cbar - 1.0
            x1 = 2.0
        else:
            x0 = 0.2 if cbar < 5.215 else 0.326 * cbar - 1.5
            x1 = 3.0
    m = 3.0
    a = (cbar - 4.606 * x0) / (x1 - x0) ** m
    x = np.log10(beta_gamma)
    d = np.where(x >= x1, 4.606 * x - cbar,
                 np.where(x >= x0, 4.606 * x - cbar + a * (x1 - x) ** m, 0.0))
    return np.maximum(d, 0.0)


def electron_quantities(mt: MediumTables, t):
    """Restricted dE/dx and discrete cross sections (per cm, standard density)."""
    med = mt.med
    z, pz = mt.z, mt.pz
    ne_per_g = 6.02214e23 * np.sum(pz * z)          # electrons per gram
    n_el = med.rho * ne_per_g
    kconst = 2 * math.pi * R0 ** 2 * RM * n_el     # MeV/cm
    te = med.ae - RM
    lnI = np.sum(pz * z * np.log([ELEMENTS[int(q)][2] for q in z])) / np.sum(pz * z)
    i_ev = math.exp(lnI)
    tau = t / RM
    g = tau + 1
    b2 = tau * (tau + 2) / g ** 2
    bg = np.sqrt(tau * (tau + 2))
    dens = density_effect(med, bg, i_ev, ne_per_g)
    delta = te / RM
    lnterm = np.log(2 * (tau + 2) / (i_ev * 1e-6 / RM) ** 2)
    # electrons
    dm = np.minimum(delta, tau / 2)
    fm = (-1 - b2 + np.log((tau - dm) * dm) + tau / (tau - dm)
          + (dm ** 2 / 2 + (2 * tau + 1) * np.log(1 - dm / tau)) / g ** 2)
    scol_m = kconst / b2 * (lnterm + fm - dens)
    # positrons
    dp = np.minimum(delta, tau)
    y = 1 / (tau + 2)
    fp = (np.log(tau * dp) - b2 / tau * (tau + 2 * dp - 1.5 * dp ** 2 * y - (dp - dp ** 3 / 3) * y ** 2
                                          - (dp ** 2 / 2 - tau * dp ** 3 / 3 + dp ** 4 / 4) * y ** 3))
    scol_p = kconst / b2 * (lnterm + fp - dens)
    # bremsstrahlung (same screening functions as the sampler)
    zz = z * (z + np.array([xsif(q) for q in z]))
    zt = np.sum(pz * zz)
    zg = np.sum(pz * zz * (-np.log(z) / 3)) / zt
    delcm = 136 * RM * math.exp(zg)
    ar = ALPHA * R0 ** 2 * zt * 6.02214e23 * med.rho     # 1/cm
    srad = np.zeros_like(t)
    sbr = np.zeros_like(t)
    for i, tt in enumerate(t):
        e = tt + RM
        kc = min(med.ap, tt)
        # restricted radiative: integral of k dsigma/dk from 0 to kc
        kk = np.linspace(0, kc, 200)[1:]
        ep = e - kk
        eps = ep / e
        dl = delcm * kk / (e * ep)
        p1, p2 = phi12(dl)
        f = (1 + eps ** 2) * (p1 + 4 * zg) - 2.0 / 3.0 * eps * (p2 + 4 * zg)
        srad[i] = ar * np.trapezoid(np.concatenate([[f[0]], f]), np.concatenate([[0.0], kk]))
        if tt > med.ap:
            kk = np.exp(np.linspace(math.log(med.ap), math.log(tt * 0.999999), 300))
            ep = e - kk
            eps = ep / e
            dl = delcm * kk / (e * ep)
            p1, p2 = phi12(dl)
            f = (1 + eps ** 2) * (p1 + 4 * zg) - 2.0 / 3.0 * eps * (p2 + 4 * zg)
            sbr[i] = ar * np.trapezoid(f, np.log(kk))
    sbr = np.maximum(sbr, 0.0)
    # Moller (T > 2 te)
    e0 = np.clip(te / t, 1e-12, 0.5)
    smol = np.where(t > 2 * te,
                    kconst / (b2 * t) * (1 / e0 - 1 / (1 - e0) + (tau / g) ** 2 * (0.5 - e0)
                                          - (2 * tau + 1) / g ** 2 * np.log((1 - e0) / e0)), 0.0)
    smol = np.maximum(smol, 0.0)
    # Bhabha (T > te)
    e0b = np.clip(te / t, 1e-12, 1.0)
    yp = 1 - 2 * y
    b4 = yp ** 3
    b3 = b4 + yp ** 2
    bb2 = yp * (3 + y ** 2)
    b1 = 2 - y ** 2
    sbh = np.where(t > te, kconst / (b2 * t) * (1 / e0b - 1 - b2 * (b1 * np.log(1 / e0b) - bb2 * (1 - e0b)
                                                                 + b3 * (1 - e0b ** 2) / 2 - b4 * (1 - e0b ** 3) / 3)), 0.0)
    sbh = np.maximum(sbh, 0.0)
    # annihilation in flight (Heitler)
    gg = g
    san = math.pi * R0 ** 2 / (gg + 1) * ((gg ** 2 + 4 * gg + 1) / (gg ** 2 - 1) * np.log(gg + np.sqrt(gg ** 2 - 1))
                                          - (gg + 3) / np.sqrt(gg ** 2 - 1)) * n_el
    # restricted radiative loss by the collision-loss-cut brems below AP
    dedx_m = scol_m + srad
    dedx_p = scol_p + srad
    sig_m = smol + sbr
    sig_p = sbh + sbr + san
    return dict(dedx_m=dedx_m, dedx_p=dedx_p, sig_m=sig_m, sig_p=sig_p, sbr=sbr, smol=smol,
                sbh=sbh, san=san, delcm=delcm, zg=zg, n_el=n_el)


def moliere(mt: MediumTables):
    """Moliere b_c (1/cm) and chi_c (MeV cm^-1/2) at standard density (Bethe 1953)."""
    z, pz = mt.z, mt.pz
    zz = z * (z + 1)
    zs = np.sum(pz * zz)
    ze = np.sum(pz * zz * np.log(z ** (-2.0 / 3.0)))
    zx = np.sum(pz * zz * np.log(1 + 3.34 * (ALPHA * z) ** 2))
    rho = mt.med.rho
    blcc = 6680.0 * rho * zs * math.exp(ze / zs) / math.exp(zx / zs)
    xcc = math.sqrt(0.157 * rho * zs)
    return blcc, xcc


# ---------------------------------------------------------------------------
# Goudsmit-Saunderson tables (the msnew.data surfaces)
# ---------------------------------------------------------------------------
def _sr_moments(eta, lmax):
    """<P_l> of the screened Rutherford distribution, l=0..lmax (vector over eta).

    f(mu) = 2 eta (1+eta) / (1 + 2 eta - mu)^2 on [-1, 1]; with z = 1 + 2 eta,
    <P_l> = l (Q_{l-1}(z) - z Q_l(z)), Q_l the Legendre functions of the second
    kind, obtained by Miller's backward recurrence normalised to Q_0.
    """
    eta = np.atleast_1d(eta).astype(float)
    zz = 1 + 2 * eta
    lstart = int(lmax + 60 + 40 / np.sqrt(eta.min()))
    lstart = min(lstart, 400000)
    q = np.zeros((lmax + 2, eta.size))
    qn1 = np.zeros_like(eta)
    qn = np.full_like(eta, 1e-200)
    for l in range(lstart, 0, -1):
        # (l+1) Q_{l+1} = (2l+1) z Q_l - l Q_{l-1}  ->  Q_{l-1}
        qm1 = ((2 * l + 1) * zz * qn - (l + 1) * qn1) / l
        qn1, qn = qn, qm1
        if l - 1 <= lmax + 1:
            q[l - 1] = qm1
        big = np.abs(qn) > 1e200
        if big.any():
            qn[big] *= 1e-200
            qn1[big] *= 1e-200
            q[:, big] *= 1e-200
    q0 = 0.5 * np.log((1 + eta) / eta)
    q *= (q0 / q[0])[None, :]
    mom = np.ones((lmax + 1, eta.size))
    ls = np.arange(1, lmax + 1)[:, None]
    mom[1:] = ls * (q[0:lmax] - zz[None, :] * q[1:lmax + 1])
    return mom


def _g1(eta):
    return 2 * eta * ((1 + eta) * np.log1p(1 / eta) - 1)


def _eta_from_g1(g1):
    lo, hi = np.full_like(g1, 1e-14), np.full_like(g1, 1e3)
    for _ in range(200):
        mid = np.sqrt(lo * hi)
        v = _g1(mid)
        hi = np.where(v > g1, mid, hi)
        lo = np.where(v > g1, lo, mid)
    return np.sqrt(lo * hi)


def _omega2(lam, chia2):
    """Width parameter of the u transform (electron.cu:199-202, same fit)."""
    ll = math.log(lam)
    if ll < 2.2299:
        p = 1.347006 + ll * (0.209364 - ll * (0.45525 - ll * (0.50142 - 0.081234 * ll)))
    else:
        p = -2.77164 + ll * (2.94874 - ll * (0.1535754 - ll * 0.00552888))
    return chia2 * (lam + 4) * p


def _alias(p):
    """Walker alias table for len(p) equiprobable bins: (keep fraction, alias index)."""
    n = len(p)
    prob = np.asarray(p, float) * n / np.sum(p)
    w = np.ones(n)
    alias = np.arange(n)
    small = [i for i in range(n) if prob[i] < 1]
    large = [i for i in range(n) if prob[i] >= 1]
    while small and large:
        s = small.pop()
        l_ = large.pop()
        w[s] = prob[s]
        alias[s] = l_
        prob[l_] = prob[l_] - (1 - prob[s])
        (small if prob[l_] < 1 else large).append(l_)
    return w, alias


def build_ms_tables():
    nl, nq, nu = L.MAXL_MS + 1, L.MAXQ_MS + 1, L.MAXU_MS + 1
    llammin = math.log(1.0)
    llammax = math.log(1e5)
    dllamb = (llammax - llammin) / L.MAXL_MS
    dqms = 0.5 / L.MAXQ_MS
    ums = np.zeros((nu, nq, nl))
    fms = np.zeros((nu, nq, nl))
    wms = np.zeros((nu, nq, nl))
    ims = np.zeros((nu, nq, nl), np.int64)
    ugrid = np.linspace(0.0, 1.0, nu)
    for i in range(nl):
        lam = math.exp(llammin + i * dllamb)
        qs = np.array([max(j * dqms, 0.5e-3) for j in range(nq)])
        g1 = np.minimum(qs / lam, 0.999)
        etas = _eta_from_g1(g1)
        for j in range(nq):
            eta = etas[j]
            lmax = int(min(6000, 60 + 40 / math.sqrt(max(qs[j], 1e-3) / max(lam, 1.0)) / 4 + 30 / math.sqrt(eta) / 10))
            lmax = max(lmax, 200)
            mom = _sr_moments(np.array([eta]), lmax)[:, 0]
            gl = 1 - mom
            el = math.exp(-lam)
            norm = 1 - el * (1 + lam)
            c = (np.exp(-lam * gl) - el - lam * el * mom) / norm
            om2 = _omega2(lam, eta)
            # density in mu at the u grid points
            xi = om2 * ugrid / (1 + 0.5 * om2 - ugrid)
            mu = np.clip(1 - xi, -1, 1)
            p_prev = np.ones_like(mu)
            p_cur = mu.copy()
            dens = 0.5 * c[0] * p_prev + 1.5 * c[1] * p_cur
            for l in range(1, lmax):
                p_next = ((2 * l + 1) * mu * p_cur - l * p_prev) / (l + 1)
                dens += (l + 1.5) * c[l + 1] * p_next
                p_prev, p_cur = p_cur, p_next
            jac = om2 * (1 + 0.5 * om2) / (1 + 0.5 * om2 - ugrid) ** 2
            fu = np.maximum(dens * jac, 0.0)
            fu = np.maximum(fu, fu.max() * 1e-6)
            mass = 0.5 * (fu[1:] + fu[:-1]) * np.diff(ugrid)
            w, al = _alias(mass)
            ums[:, j, i] = ugrid
            a = fu[1:] / fu[:-1] - 1
            fms[:nu - 1, j, i] = a
            fms[nu - 1, j, i] = a[-1]
            wms[:nu - 1, j, i] = w
            ims[:nu - 1, j, i] = al
    return dict(ums=ums, fms=fms, wms=wms, ims=ims, llammin=llammin, llammax=llammax,
                dllamb=dllamb, dqms=dqms)


_MS_CACHE = {}


MS_DATA_FILE = __import__("pathlib").Path(__file__).with_name("data") / "ms_sr_tables.npz"


def ms_tables(rebuild: bool = False):
    """GS surfaces; loaded from the packaged file (``build_ms_tables`` takes ~4 min).

    ``python -m gegs_b200.physics_data --ms`` regenerates the file.
    """
    if "t" not in _MS_CACHE:
        if MS_DATA_FILE.exists() and not rebuild:
            d = np.load(MS_DATA_FILE)
            _MS_CACHE["t"] = {k: (d[k] if d[k].ndim else float(d[k])) for k in d.files}
        else:
            _MS_CACHE["t"] = build_ms_tables()
    return _MS_CACHE["t"]


def write_ms_file():
    t = build_ms_tables()
    np.savez_compressed(MS_DATA_FILE, ums=t["ums"].astype(np.float32), fms=t["fms"].astype(np.float32),
                        wms=t["wms"].astype(np.float32), ims=t["ims"].astype(np.int32),
                        llammin=t["llammin"], llammax=t["llammax"], dllamb=t["dllamb"], dqms=t["dqms"])


# ---------------------------------------------------------------------------
# block assembly
# ---------------------------------------------------------------------------
K_FLUO = [(4, 0.50), (3, 0.26), (5, 0.20), (6, 0.04)]


def relaxation_probs(z: int) -> np.ndarray:
    """39 transition probabilities (K:1-19, L1:20-26, L2:27-32, L3:33-37, M:38-39)."""
    p = np.zeros(L.MXTRANS)
    wk = z ** 4 / (z ** 4 + 1.06e6)
    wl = z ** 4 / (z ** 4 + 8.9e7)
    wm = z ** 4 / (z ** 4 + 1.2e9)
    p[0:4] = wk * np.array([0.50, 0.26, 0.20, 0.04])
    p[4:19] = (1 - wk) / 15.0
    # L1: 13, 14 (Coster-Kronig), 5, 6 (fluorescence), 505, 605, 606 (Auger)
    p[19:26] = [0.25, 0.45, wl * 0.7 * 0.3, wl * 0.3 * 0.3, 0, 0, 0]
    rest = 1 - p[19:23].sum()
    p[23:26] = rest * np.array([0.6, 0.3, 0.1])
    # L2: 14, 5, 6, 505, 605, 606
    p[26:28] = [0.15, wl * 0.8]
    p[28] = wl * 0.2
    rest = 1 - p[26:29].sum()
    p[29:32] = rest * np.array([0.6, 0.3, 0.1])
    # L3: 5, 6, 505, 605, 606
    p[32:34] = [wl * 0.8, wl * 0.2]
    rest = 1 - p[32:34].sum()
    p[34:37] = rest * np.array([0.6, 0.3, 0.1])
    # M: 6, 606
    p[37] = wm
    p[38] = 1 - wm
    return p


def _eno_alias(weights):
    """Shell-selection alias (reference init_compton layout, PhysicsInit.cu:1400-1490).

    Sampling: r = 1 + U*n; i = int(r); if r > eno[i-1]: i = atbin[i-1].
    """
    n = len(weights)
    w, al = _alias(np.asarray(weights, float))
    eno = np.arange(1, n + 1) + w          # keep bin i (1-based) when r <= i + w
    atbin = al + 1
    return eno, atbin


def build_block(media_names, mlc_media=(), overrides=None):
    """Build the physics block for the listed media (order = medium index).

    ``mlc_media``: media names that get range rejection (the reference turns it
    on for the MLC region's medium only, init.cu:922).
    """
    overrides = overrides or {}
    if len(media_names) > L.MXMED:
        raise ValueError(f"at most {L.MXMED} media, got {len(media_names)}")
    blk = L.new_block()
    nmed = len(media_names)
    blk["nmed"] = nmed
    blk["rm"] = RM
    blk["prm"] = RM
    blk["rmt2"] = np.float32(2 * np.float32(RM))
    blk["rmsq"] = np.float32(np.float32(RM) * np.float32(RM))
    blk["estepe"] = 0.25
    blk["ximax"] = 0.5
    blk["transport_algorithm"] = 1    # PRESTA-I (CUDA_EGS.h:38)
    blk["exact_bca"] = 0              # BCA_EXACT off (CUDA_EGS.h:33)
    blk["spin_effects"] = 0           # SPIN_FLAG off (CUDA_EGS.h:40)
    blk["ibrdst"] = 1                 # BAS_KM (CUDA_EGS.h:41)
    blk["iprdst"] = 1                 # IPRDST (CUDA_EGS.h:43)
    blk["nbr_split"] = 1
    mts = []
    for m, name in enumerate(media_names):
        med = MEDIA[name]
        if name in overrides:
            for k, v in overrides[name].items():
                setattr(med, k, v)
        z, pz, a = med.elements
        mts.append(MediumTables(med, z, pz, a))

    # ---- element data (edges, relaxation) -------------------------------
    all_z = sorted({int(q) for mt in mts for q in mt.z})
    for zi in all_z:
        be = binding_energies(zi)
        blk["binding_energies"][L.MXSHELL * (zi - 1): L.MXSHELL * zi] = be
        ip = np.where(be > 0, (JUMP - 1) / JUMP, 0.0)
        if zi == 1:
            ip[0] = 1.0
        ip[5] = 1.01
        blk["interaction_prob"][L.MXSHELL * (zi - 1): L.MXSHELL * zi] = ip
        blk["relaxation_prob"][L.MXTRANS * (zi - 1): L.MXTRANS * zi] = relaxation_probs(zi)
        edges = [(be[s], s) for s in range(6) if be[s] > 1e-3]
        edges.sort(key=lambda t: -t[0])
        ne = len(edges)
        blk["edge_number"][zi - 1] = ne
        base = L.MXEDGE * (zi - 1)
        cz = photo_c(zi)
        jump = 1.0
        for m in range(ne + 1):
            if m == 0:
                blk["edge_c"][base] = cz
            else:
                jump *= JUMP[edges[m - 1][1]]
                blk["edge_a"][base + m] = math.log(cz / jump)
                blk["edge_b"][base + m] = -3.5
            if m < ne:
                blk["edge_energies"][base + m] = edges[m][0]

    # ---- per medium -------------------------------------------------------
    ms = ms_tables()
    shell_list = []        # global Compton shells: (z, shn, ne, j0, be)
    shell_index = {}
    eii_rows = []
    e_eii_min = min(min(mt.med.ae - RM, mt.med.ap) for mt in mts)
    eii_shells_of = {}
    for zi in all_z:
        be = binding_energies(zi)
        eii_shells_of[zi] = [s for s in range(4) if be[s] > e_eii_min]
    eii_first_of = {}
    cnt = 0
    for zi in all_z:
        if eii_shells_of[zi]:
            eii_first_of[zi] = cnt + 1
            cnt += len(eii_shells_of[zi])
    if cnt > L.MAX_EII_SHELLS:
        raise ValueError("too many EII shells")
    blk["eii_flag"] = 1 if cnt > 0 else 0

    ecutmn = min(mt.med.ae for mt in mts)
    tstbmn = 1e30
    for m, mt in enumerate(mts):
        med = mt.med
        z, pz, a = mt.z, mt.pz, mt.a
        ne_ = len(z)
        blk["nne"][m] = ne_
        for k in range(ne_):
            blk["zelem"][k * L.MXMED + m] = z[k]
            blk["pz"][k * L.MXMED + m] = pz[k]
            blk["wa"][k * L.MXMED + m] = a[k]
        blk["rho"][m] = med.rho
        blk["ae"][m] = med.ae
        blk["ap"][m] = med.ap
        blk["ue"][m] = med.ue
        blk["up"][m] = med.up
        te = med.ae - RM
        blk["te"][m] = te
        blk["thmoll"][m] = te * 2 + RM
        blk["smaxir"][m] = 1e10
        blk["e_max_rr"][m] = 0.8
        blk["i_do_rr"][m] = 1 if med.name in mlc_media else 0
        con2 = med.rho / (np.sum(pz * a)) * INV_1P66
        # photon tables (init_user_photon, media.cu:832-1058)
        gy = (L.MXGE - 1) / math.log(med.up / med.ap)
        gx = -gy * math.log(med.ap)
        blk["ge"][m] = (gx, gy)
        gle = (np.arange(L.MXGE) - gx) / gy
        eg = np.exp(gle)
        sig_kn = np.sum(pz * z) * sigma_kn(eg)
        sig_ph = sum(pz[k] * sigma_photo(z[k], eg) for k in range(ne_))
        sig_pp = sum(pz[k] * sigma_pair(z[k], eg) for k in range(ne_))
        sig_ry = sum(pz[k] * sigma_rayleigh(z[k], eg) for k in range(ne_))
        sigma = sig_kn + sig_pp + sig_ph
        gmfp = 1.0 / (sigma * con2)
        gbr1 = sig_pp / sigma
        gbr2 = gbr1 + sig_kn / sigma
        cohe = sigma / (sig_ry + sigma)
        for nm, v in (("gmfp", gmfp), ("gbr1", gbr1), ("gbr2", gbr2), ("cohe", cohe)):
            blk[nm][m * L.MXGE:(m + 1) * L.MXGE] = _line_fit(v, gle, L.MXGE)
        _rayleigh_tables(blk, m, mt, gx, gy)
        # bound Compton shells of this medium
        wts, ids = [], []
        for k in range(ne_):
            zi = int(z[k])
            for s, (be, nel, j0) in enumerate(shell_electrons(zi)):
                key = (zi, s)
                if key not in shell_index:
                    shell_list.append((zi, s + 1, nel, j0, be))
                    shell_index[key] = len(shell_list)
                wts.append(pz[k] * nel)
                ids.append(shell_index[key])
        nsh = len(ids)
        if nsh > L.MXMDSH:
            raise ValueError("too many Compton shells in medium")
        eno, atbin = _eno_alias(np.array(wts) / np.sum(wts))
        blk["n_shell"][m] = nsh
        blk["shell_array"][m * L.MXMDSH: m * L.MXMDSH + nsh] = ids
        blk["eno_array"][m * L.MXMDSH: m * L.MXMDSH + nsh] = eno
        blk["eno_atbin_array"][m * L.MXMDSH: m * L.MXMDSH + nsh] = atbin

        # electron tables
        ey = (L.MXEKE - 1) / math.log((med.ue - RM) / te)
        ex = 1 - ey * math.log(te)
        blk["eke01"][m] = (ex, ey)
        idx = np.arange(1, L.MXEKE + 2)
        elke = (idx - ex) / ey
        ek = np.exp(elke)
        q = electron_quantities(mt, ek)
        for qel, (dd, ss) in enumerate(((q["dedx_m"], q["sig_m"]), (q["dedx_p"], q["sig_p"]))):
            base = qel * L.MXEKE * L.MXMED + m * L.MXEKE
            blk["dedx"][base: base + L.MXEKE] = _line_fit(dd[:L.MXEKE + 1], elke[:L.MXEKE + 1], L.MXEKE)
            blk["sig"][base: base + L.MXEKE] = _line_fit(ss[:L.MXEKE + 1], elke[:L.MXEKE + 1], L.MXEKE)
        with np.errstate(invalid="ignore", divide="ignore"):
            ebr1 = np.nan_to_num(q["sbr"] / q["sig_m"])
            pbr1 = np.nan_to_num(q["sbr"] / q["sig_p"])
            pbr2 = np.nan_to_num((q["sbr"] + q["sbh"]) / q["sig_p"])
        for nm, v in (("ebr1", ebr1), ("pbr1", pbr1), ("pbr2", pbr2)):
            blk[nm][m * L.MXEKE:(m + 1) * L.MXEKE] = _line_fit(v[:L.MXEKE + 1], elke[:L.MXEKE + 1], L.MXEKE)
        blk["delcm"][m] = q["delcm"]
        blcc, xcc = moliere(mt)
        mt.extras.update(blcc_raw=blcc, xcc_raw=xcc)
        # bremsstrahlung screening coefficients (fix_brems, PhysicsInit.cu:1552-1640)
        _fix_brems(blk, m, mt)
        # EII bookkeeping (eii_init, PhysicsInit.cu:1643-1800)
        nsh_med = 0
        for k in range(ne_):
            zi = int(z[k])
            nsh_e = len(eii_shells_of[zi])
            blk["eii_no"][k * L.MXMED + m] = nsh_e
            blk["eii_first"][L.MXMED * k + m] = eii_first_of.get(zi, 0)
            nsh_med += nsh_e
        blk["eii_nsh"][m] = nsh_med
        blk["eii_cons"][m] = med.rho / np.sum(pz * a) * INV_1P66
        # default BLCMIN for the PRESTA-I boundary crossing (mscati, PhysicsInit.cu:955-990)
        r1 = ecutmn
        tstbm = (ecutmn - RM) * (ecutmn + RM) / (r1 * r1)
        r1 = ecutmn / xcc
        tstbm = blcc * tstbm * r1 * r1
        aux = math.log(tstbm)
        tstbm = math.log(tstbm / aux)
        tstbmn = min(tstbmn, tstbm)
    blk["skindepth_for_bca"] = math.exp(tstbmn)

    for m, mt in enumerate(mts):
        blk["blcc"][m] = mt.extras["blcc_raw"] * 1.16699413758864573
        blk["xcc"][m] = mt.extras["xcc_raw"] ** 2
    for m, mt in enumerate(mts):
        _mscati_tables(blk, m)

    # Compton shell arrays
    for i, (zi, shn, nel, j0, be) in enumerate(shell_list):
        blk["iz_array"][i] = zi
        blk["shn_array"][i] = shn
        blk["ne_array"][i] = nel
        jo = j0 * 137.0
        blk["jo_array"][i] = jo
        blk["be_array"][i] = be / RM
        blk["erfjo_array"][i] = 0.82436063535 * math.erf(0.70710678119 * (1.0 + 0.3 * jo))

    # EII shells
    for zi in all_z:
        if not eii_shells_of[zi]:
            continue
        blk["eii_nshells"][zi - 1] = len(eii_shells_of[zi])
        be = binding_energies(zi)
        for n, s in enumerate(eii_shells_of[zi]):
            jj = eii_first_of[zi] + n          # 1-based global shell index
            blk["eii_z"][jj - 1] = zi
            blk["eii_sh"][jj - 1] = s + 1
            uj = be[s]
            emax = max(m.med.ue for m in mts) - RM
            lo, hi = math.log(uj), math.log(emax)
            b = (L.N_EII_BINS - 1) / (hi - lo)
            blk["eii"][jj - 1] = (b, 1 - b * lo)        # .x slope, .y intercept (moller.cu:93)
            le = lo + np.arange(L.N_EII_BINS + 1) / b
            tt = np.exp(le)
            nel = 2 if s == 0 else (2 if s < 3 else 4)
            nel = [2, 2, 2, 4][s]
            tau = tt / RM
            b2 = tau * (tau + 2) / (tau + 1) ** 2
            sg = 0.05 * nel * 2 * math.pi * R0 ** 2 * RM / b2 * (1 / uj) * np.clip(1 - uj / tt, 0, None) / BARN
            fit = _line_fit(sg, le, L.N_EII_BINS + 1)[:L.N_EII_BINS]
            rows = blk["eii_xsection"][(jj - 1) * L.N_EII_BINS: jj * L.N_EII_BINS]
            rows[:, 0] = fit[:, 1]    # .x slope
            rows[:, 1] = fit[:, 0]    # .y intercept

    # multiple scattering surfaces
    blk["llammin"] = ms["llammin"]
    blk["llammax"] = ms["llammax"]
    blk["dllamb"] = ms["dllamb"]
    blk["dllambi"] = 1.0 / ms["dllamb"]
    blk["dqms"] = ms["dqms"]
    blk["dqmsi"] = 1.0 / ms["dqms"]
    blk["ums_array"] = ms["ums"].reshape(-1)
    blk["fms_array"] = ms["fms"].reshape(-1)
    blk["wms_array"] = ms["wms"].reshape(-1)
    blk["ims_array"] = ms["ims"].reshape(-1)
    return blk


def _fix_brems(blk, m, mt):
    z, pz = mt.z, mt.pz
    zt = zb = zf = 0.0
    for zi, pi in zip(z, pz):
        fc = fcoulc(zi)
        xi = xsif(zi)
        aux = pi * zi * (zi + xi)
        zt += aux
        zb -= aux * math.log(zi) / 3
        zf += aux * fc
    zv = (zb - zf) / zt
    zg = zb / zt
    fmax1 = 2 * (20.863 + 4 * zg) - 2 * (20.029 + 4 * zg) / 3
    fmax2 = 2 * (20.863 + 4 * zv) - 2 * (20.029 + 4 * zv) / 3
    rows = [
        ((20.863 + 4 * zg) / fmax1, -3.242 / fmax1, 0.625 / fmax1, (21.12 + 4 * zg) / fmax1, -4.184 / fmax1, 0.952),
        ((20.029 + 4 * zg) / fmax1, -1.93 / fmax1, -0.086 / fmax1, (21.12 + 4 * zg) / fmax1, -4.184 / fmax1, 0.952),
        ((20.863 + 4 * zv) / fmax2, -3.242 / fmax2, 0.625 / fmax2, (21.12 + 4 * zv) / fmax2, -4.184 / fmax2, 0.952),
        ((20.029 + 4 * zv) / fmax2, -1.93 / fmax2, -0.086 / fmax2, (21.12 + 4 * zv) / fmax2, -4.184 / fmax2, 0.952),
        (3 * (20.863 + 4 * zg) - (20.029 + 4 * zg), 3 * -3.242 + 1.930, 3 * 0.625 + 0.086, 2 * 21.12 + 8 * zg, 2 * -4.184, 0.952),
        (3 * (20.863 + 4 * zg) + (20.029 + 4 * zg), 3 * -3.242 - 1.930, 3 * 0.625 - 0.086, 4 * 21.12 + 16 * zg, 4 * -4.184, 0.952),
        (3 * (20.863 + 4 * zv) - (20.029 + 4 * zv), 3 * -3.242 + 1.930, 3 * 0.625 + 0.086, 2 * 21.12 + 8 * zv, 2 * -4.184, 0.952),
        (3 * (20.863 + 4 * zv) + (20.029 + 4 * zv), 3 * -3.242 - 1.930, 3 * 0.625 - 0.086, 4 * 21.12 + 16 * zv, 4 * -4.184, 0.952),
    ]
    for l, r in enumerate(rows):
        for nm, v in zip(("dl1", "dl2", "dl3", "dl4", "dl5", "dl6"), r):
            blk[nm][m * 8 + l] = v
    blk["bpar"][m * 2 + 1] = blk["dl1"][m * 8 + 6] / (3 * blk["dl1"][m * 8 + 7] + blk["dl1"][m * 8 + 6])
    blk["bpar"][m * 2 + 0] = 12 * blk["dl1"][m * 8 + 7] / (3 * blk["dl1"][m * 8 + 7] + blk["dl1"][m * 8 + 6])
    blk["log_ap"][m] = math.log(blk["ap"][m])
    zz = np.sum(pz * z * (z + 1)) / np.sum(pz)
    zbr = 8.116224e-05 * zz ** (1.0 / 3.0)
    blk["zbrang"][m] = zbr
    blk["lzbrang"][m] = -math.log(zbr)


def _ev(tab, i, x):
    return tab[i, 0] + tab[i, 1] * x


def _mscati_tables(blk, m):
    """sig_e, monotonicity, e_array, range_ep, expeke1, tmxs (PhysicsInit.cu:1007-1180)."""
    ex, ey = (float(v) for v in blk["eke01"][m])
    rm = RM
    dedx = [blk["dedx"][q * L.MXEKE * L.MXMED + m * L.MXEKE: q * L.MXEKE * L.MXMED + (m + 1) * L.MXEKE].astype(float) for q in (0, 1)]
    sig = [blk["sig"][q * L.MXEKE * L.MXMED + m * L.MXEKE: q * L.MXEKE * L.MXMED + (m + 1) * L.MXEKE].astype(float) for q in (0, 1)]
    neke = L.MXEKE
    for qel in (0, 1):
        smax, mono, old = 1e-15, True, -1.0
        for i in range(1, neke + 1):
            eil = (i - ex) / ey
            s = _ev(sig[qel], i - 1, eil) / _ev(dedx[qel], i - 1, eil)
            smax = max(smax, s)
            if s < old:
                mono = False
            old = s
        blk["sig_e"][qel * L.MXMED + m] = smax
        blk["sig_ismonotone"][2 * m + qel] = 1 if mono else 0
    base = m * L.MXEKE
    ei = math.exp((1 - ex) / ey)
    blk["e_array"][base] = ei
    blk["expeke1"][m] = math.exp(1.0 / ey) - 1
    rng = np.zeros((L.MXEKE, 2))
    for i in range(1, neke):
        eip1 = math.exp((i + 1 - ex) / ey)
        blk["e_array"][base + i] = eip1
        eke = (eip1 + ei) * 0.5
        elke = math.log(eke)
        lelke = int(ey * elke + ex)
        for qel in (1, 0):
            ededx = _ev(dedx[qel], lelke - 1, elke)
            aux = dedx[qel][i - 1, 1] / ededx
            r1 = (eip1 - ei) / eke
            rng[i, qel] = rng[i - 1, qel] + (eip1 - ei) / ededx * (1 + aux * (1 + 2 * aux) * r1 * r1 / 24)
        ei = eip1
    blk["range_ep"][2 * base: 2 * (base + L.MXEKE)] = rng.reshape(-1)
    xcc = float(blk["xcc"][m])
    blcc = float(blk["blcc"][m])
    ximax, estepe = float(blk["ximax"]), float(blk["estepe"])
    e_arr = blk["e_array"][base: base + L.MXEKE].astype(float)
    eil = (1 - ex) / ey
    ei = math.exp(eil)
    p2 = ei * (ei + rm * 2)
    beta2 = p2 / (p2 + rm * rm)
    chi_a2 = xcc / (p2 * 4 * blcc)
    dedx0 = _ev(dedx[0], 0, eil)
    estepx = p2 * 2 * beta2 * dedx0 / ei / xcc / (math.log(1.0 / chi_a2 + 1) * (chi_a2 + 1) - 1)
    estepx = min(estepx * ximax, estepe)
    si = estepx * ei / dedx0
    tm = np.zeros((L.MXEKE, 2))
    for i in range(1, neke):
        elke = (i + 1 - ex) / ey
        eke = math.exp(elke)
        lelke = i + 1
        p2 = eke * (eke + rm * 2)
        beta2 = p2 / (p2 + rm * rm)
        chi_a2 = xcc / (p2 * 4 * blcc)
        ededx = _ev(dedx[0], lelke - 1, elke)
        estepx = p2 * 2 * beta2 * ededx / eke / xcc / (math.log(1.0 / chi_a2 + 1) * (chi_a2 + 1) - 1)
        estepx = min(estepx * ximax, estepe)
        ekef = (1 - estepx) * eke
        if ekef <= e_arr[0]:
            sip1 = (e_arr[0] - ekef) / dedx0
            lelkef = 1
        else:
            elkef = math.log(ekef)
            lelkef = int(ey * elkef + ex)
            leip1l = lelkef + 1
            eip1l = (leip1l - ex) / ey
            eip1 = e_arr[leip1l - 1]
            aux = (eip1 - ekef) / eip1
            elktmp = 0.5 * (elkef + eip1l + 0.25 * aux * aux * (1 + aux * (1 + 0.875 * aux)))
            ektmp = (ekef + eip1) * 0.5
            ededx = _ev(dedx[0], lelkef - 1, elktmp)
            aux = dedx[0][lelkef - 1, 1] / ededx
            r1 = (eip1 - ekef) / ektmp
            sip1 = (eip1 - ekef) / ededx * (1 + aux * (aux * 2 + 1) * r1 * r1 / 24)
        sip1 = sip1 + rng[lelke - 1, 0] - rng[lelkef, 0]
        tm[i - 1, 1] = (sip1 - si) * ey
        tm[i - 1, 0] = sip1 - tm[i - 1, 1] * elke
        si = sip1
    tm[neke - 1] = tm[neke - 2]
    blk["tmxs"][base: base + L.MXEKE] = tm


def _rayleigh_tables(blk, m, mt, gx, gy):
    """Form-factor CDF, pmax and uniform-bin index (init_rayleigh_data, media.cu:1060-1292)."""
    nff = L.MXRAYFF
    med = mt.med
    xg = np.logspace(-4, 3.5, nff)
    ff = np.sqrt(sum(mt.pz[k] * form_factor(mt.z[k], xg) ** 2 for k in range(len(mt.z))))
    ff = np.maximum(ff, 1e-300)
    bb = np.zeros(nff)
    fcum = np.zeros(nff)
    s0 = 0.0
    for j in range(nff - 1):
        b = math.log(ff[j + 1] / ff[j]) / math.log(xg[j + 1] / xg[j])
        bb[j] = b
        x1, x2 = xg[j], xg[j + 1]
        s0 += ff[j] ** 2 * (x2 * x2 * x2 ** (2 * b) - x1 * x1 * x1 ** (2 * b)) / ((1 + b) * x1 ** (2 * b))
        fcum[j + 1] = s0
    emin = math.exp(-gx / gy)
    emax = math.exp((L.MXGE - 1.0 - gx) / gy)
    dle = math.log(emax / emin) / (L.MXGE - 1.0)
    pe = np.zeros(L.MXGE)
    idx = 1
    for j in range(1, L.MXGE + 1):
        e = emin * math.exp(dle * (j - 1.0))
        xmax = 20.607544 * 2.0 * e / RM
        k = 1
        while k <= nff - 1:
            if xg[k - 1] <= xmax < xg[k]:
                break
            k += 1
        idx = min(k, nff - 1)
        b = bb[idx - 1]
        x1 = xg[idx - 1]
        pe[j - 1] = fcum[idx - 1] + ff[idx - 1] ** 2 * (xmax * xmax * xmax ** (2 * b) - x1 * x1 * x1 ** (2 * b)) / ((1 + b) * x1 ** (2 * b))
    anorm = 1.0 / math.sqrt(pe[-1])
    anorm1 = 1.005 / pe[-1]
    anorm2 = 1.0 / pe[-1]
    pe = np.minimum(pe * anorm1, 1.0)
    ff = ff * anorm
    fcum = fcum * anorm2
    carr = (1.0 + bb) / (xg * ff) ** 2
    iarr = np.zeros(L.RAYCDFSIZE, np.int64)
    iarr[L.RAYCDFSIZE - 1] = idx
    dw = 1.0 / (L.RAYCDFSIZE - 1.0)
    xold = xg[0]
    ibin = 1
    b = bb[0]
    pow_x1 = xg[0] ** (2 * b)
    iarr[0] = 1
    for j in range(2, L.RAYCDFSIZE):
        w = dw
        while True:
            x1 = xold
            x2 = xg[ibin]
            t = x1 * x1 * x1 ** (2 * b)
            aux = ff[ibin - 1] ** 2 * (x2 * x2 * x2 ** (2 * b) - t) / ((1 + b) * pow_x1)
            if aux > w:
                xold = math.exp(math.log(t + w * (1 + b) * pow_x1 / ff[ibin - 1] ** 2) / (2 + 2 * b))
                iarr[j - 1] = ibin
                break
            w -= aux
            xold = x2
            ibin += 1
            b = bb[ibin - 1]
            pow_x1 = xold ** (2 * b)
    bfin = 0.5 / (1.0 + bb)
    rd = blk["rayleigh_data"][m * nff:(m + 1) * nff]
    rd[:, 0] = xg
    rd[:, 1] = fcum
    rd[:, 2] = bfin
    rd[:, 3] = carr
    blk["i_array"][m * L.RAYCDFSIZE:(m + 1) * L.RAYCDFSIZE] = iarr
    pm = np.zeros((L.MXGE, 2))
    for j in range(L.MXGE - 1):
        gle = (j - gx) / gy
        pm[j, 1] = (pe[j + 1] - pe[j]) * gy
        pm[j, 0] = pe[j] - pm[j, 1] * gle
    pm[-1] = pm[-2]
    blk["pmax"][m * L.MXGE:(m + 1) * L.MXGE] = pm


if __name__ == "__main__":
    import sys
    if "--ms" in sys.argv:
        write_ms_file()
        print("wrote", MS_DATA_FILE)


PHYSICS_FILE_MAGIC = b"GEGSPHY1"


def write_physics_file(path, media, block):
    """Write a physics block for C/C++ callers (read by gegs_plan_load,
    include/gegs_plan.h): the magic "GEGSPHY1", the block size and the number
    of media (uint32 each), each medium's name NUL-padded to 32 bytes, then the
    block as it lies in memory. `media` names the block's media in index order."""
    import struct
    blk = np.ascontiguousarray(block)
    nmed = int(np.asarray(blk["nmed"]).reshape(-1)[0])
    if nmed != len(media):
        raise ValueError(f"{len(media)} media names for a block of {nmed}")
    with open(path, "wb") as f:
        f.write(PHYSICS_FILE_MAGIC + struct.pack("<II", blk.dtype.itemsize, len(media)))
        for m in media:
            b = m.encode("ascii")
            if len(b) >= 32:
                raise ValueError(f"medium name {m!r} longer than 31 characters")
            f.write(b + b"\0" * (32 - len(b)))
        f.write(blk.tobytes())
