"""Project-written known answers that pin the oracle (and so the GPU path,
which matches it bit for bit) to physics and geometry, independent of the
reference's missing test data:

* the Compton sampler without binding follows the Klein-Nishina cross
  section (chi-square over the scattering cosine) and the Compton relation
  between energy and angle;
* the photoelectron leaves along Sauter's angular distribution;
* the Moller sampler follows the Moller cross section above the delta-ray
  threshold and the two-body relation between energy and angle;
* direction rotations keep unit length and the requested polar angle;
* the voxel walk of howfar_phantom visits the voxels an exact ray traversal
  visits, with step lengths adding up to the chord;
* the electron and positron range tables are the integral of the inverse
  stopping power of the same tables (CSDA-range consistency).
"""
import numpy as np
import pytest

from gegs_b200 import physics_data as PD
from gegs_b200 import workloads as W

RM = 0.51099895


def _kn_bin_probs(k, edges):
    """Klein-Nishina probability of each cos(theta) bin (numerical integration)."""
    c = np.linspace(-1.0, 1.0, 400001)
    r = 1.0 / (1.0 + k * (1.0 - c))
    f = r * r * (r + 1.0 / r - (1.0 - c * c))
    cdf = np.concatenate([[0.0], np.cumsum((f[1:] + f[:-1]) / 2 * np.diff(c))])
    at = np.interp(edges, c, cdf)
    p = np.diff(at)
    return p / p.sum()


@pytest.mark.parametrize("energy", [0.3, 1.25, 6.0])
def test_compton_sampler_follows_klein_nishina(oracle, energy):
    media = ["H2O700ICRU"]
    phys = PD.build_block(media)
    n = 200_000
    e, c, err = oracle.probe_compton(phys, 0, 0, energy, n, seed=7)
    assert err == 0
    ok = c <= 1.0
    assert ok.mean() > 0.999
    k = energy / RM
    # energy-angle relation of free-electron Compton scattering
    np.testing.assert_allclose(e[ok], energy / (1.0 + k * (1.0 - c[ok])), rtol=3e-5)
    edges = np.linspace(-1.0, 1.0, 41)
    obs, _ = np.histogram(c[ok], bins=edges)
    exp = _kn_bin_probs(k, edges) * ok.sum()
    chi2 = float(((obs - exp) ** 2 / exp).sum())
    assert chi2 < 40 + 4 * np.sqrt(2 * 40), chi2        # 40 bins: chi2 well inside 40 +- 4 sigma


def test_rotations_keep_unit_length_and_polar_angle(oracle):
    a, b = oracle.probe_rotate(100_000, seed=3)
    assert np.abs(a).max() < 4e-6
    assert np.abs(b).max() < 4e-6


def _to_patient(sh, pos, d, field=0):
    s = sh.scene
    f = sh.fields_arr[field]
    x, y, z = pos
    u, v, w = d
    if s.change_xyz:
        p = np.array([y, z - s.source_to_isocenter, x], np.float64)
        q = np.array([v, w, u], np.float64)
    else:
        p = np.array([x, y, z - s.source_to_isocenter], np.float64)
        q = np.array([u, v, w], np.float64)
    c, sn = f.cos_angle, f.sin_angle
    p[:2] = [p[0] * c - p[1] * sn, p[0] * sn + p[1] * c]
    q[:2] = [q[0] * c - q[1] * sn, q[0] * sn + q[1] * c]
    return p + np.array(s.iso[:3], np.float64), q


def _exact_walk(bounds, p, d):
    """Voxels crossed by the ray p + t d (float64), with the crossing distances."""
    lo = np.array([b[0] for b in bounds]); hi = np.array([b[-1] for b in bounds])
    with np.errstate(divide="ignore", invalid="ignore"):
        t1 = (lo - p) / d
        t2 = (hi - p) / d
    tmin = np.nanmax(np.minimum(t1, t2)); tmax = np.nanmin(np.maximum(t1, t2))
    if not tmin < tmax:
        return [], []
    cross = [tmin]
    for a in range(3):
        if d[a] != 0:
            t = (bounds[a][1:-1] - p[a]) / d[a]
            cross.extend(t[(t > tmin) & (t < tmax)])
    cross = np.sort(np.array(cross + [tmax]))
    mids = (cross[:-1] + cross[1:]) / 2
    vox = []
    for t in mids:
        q = p + t * d
        idx = [int(np.searchsorted(bounds[a], q[a]) - 1) for a in range(3)]
        vox.append(idx[0] + len(bounds[0][:-1]) * (idx[1] + len(bounds[1][:-1]) * idx[2]))
    return vox, cross


def test_voxel_walk_matches_exact_traversal(oracle):
    job = W.config1(histories=10, n=20, voxel=1.5)
    sh = job.scene()
    bounds = [np.asarray(job.phantom[k], np.float64) for k in ("x_bounds", "y_bounds", "z_bounds")]
    rng = np.random.default_rng(11)
    checked = 0
    for _ in range(200):
        pos = np.array([rng.uniform(-5, 5), rng.uniform(-5, 5), 50.0], np.float32)
        d = np.array([rng.normal(0, 0.15), rng.normal(0, 0.15), 1.0])
        d = (d / np.linalg.norm(d)).astype(np.float32)
        p, q = _to_patient(sh, pos, d)
        vox, cross = _exact_walk(bounds, p, q)
        if len(vox) < 3 or np.min(np.diff(cross)) < 1e-3:
            continue                                            # a near-corner crossing: float ties
        regs, steps = oracle.probe_walk(job.physics, sh, pos, d)
        inside = regs >= 6
        got = (regs[inside] - 6).tolist()
        assert got == vox
        # steps inside the phantom add up to the chord
        k = np.flatnonzero(inside)
        assert abs(steps[k[0] + 1:k[-1] + 2].sum() - (cross[-1] - cross[0])) < 1e-3
        checked += 1
    assert checked > 100


@pytest.mark.parametrize("qel", [0, 1])
def test_range_table_is_the_integral_of_the_inverse_stopping_power(qel):
    """range_ep (the CSDA range from the lowest table energy, built as in
    PhysicsInit.cu:1007-1180 with its second-order bin correction) against a
    fine numerical integral of dE / (dE/dx) over the same log-linear
    stopping-power table, for electrons (qel 0) and positrons (qel 1)."""
    blk = PD.build_block(["H2O700ICRU"])
    from gegs_b200 import physics_layout as L
    m = 0
    ex, ey = (float(v) for v in blk["eke01"][m])
    dedx = blk["dedx"][qel * L.MXEKE * L.MXMED + m * L.MXEKE: qel * L.MXEKE * L.MXMED + (m + 1) * L.MXEKE].astype(float)
    e_arr = blk["e_array"][m * L.MXEKE: (m + 1) * L.MXEKE].astype(float)
    rng = blk["range_ep"][2 * m * L.MXEKE: 2 * (m + 1) * L.MXEKE].reshape(-1, 2)[:, qel].astype(float)

    def stopping(e):
        le = np.log(e)
        i = np.clip((ex + ey * le).astype(int), 1, L.MXEKE) - 1
        return dedx[i, 0] + dedx[i, 1] * le

    checked = 0
    for k in range(8, L.MXEKE - 1, 9):
        e = np.exp(np.linspace(np.log(e_arr[0]), np.log(e_arr[k]), 20001))
        f = 1.0 / stopping(e)
        integral = float(np.sum((f[1:] + f[:-1]) / 2 * np.diff(e)))
        assert rng[k] == pytest.approx(integral, rel=2e-3), k
        checked += 1
    assert checked >= 10
    assert (np.diff(rng[:L.MXEKE - 1]) > 0).all()      # a range grows with energy


def _moller_bin_probs(t, eps_min, edges):
    """Moller cross section over the slower electron's fraction eps of the kinetic
    energy, tau = T / mc^2: (1/eps^2)[1 + g2 eps^2 + r^2 - g3 r], r = eps / (1 - eps),
    g2 = tau^2/(tau+1)^2, g3 = (2 tau + 1)/(tau+1)^2; probability per bin."""
    tau = t / RM
    g2 = tau * tau / (tau + 1) ** 2
    g3 = (2 * tau + 1) / (tau + 1) ** 2
    e = np.linspace(eps_min, 0.5, 400001)
    r = e / (1 - e)
    f = (1 + g2 * e * e + r * (r - g3)) / (e * e)
    cdf = np.concatenate([[0.0], np.cumsum((f[1:] + f[:-1]) / 2 * np.diff(e))])
    p = np.diff(np.interp(edges, e, cdf))
    return p / p.sum()


@pytest.mark.parametrize("ekin", [0.6, 2.0, 8.0])
def test_moller_sampler_follows_the_moller_cross_section(oracle, ekin):
    """The Moller sampler (without impact ionisation) against the Moller cross
    section above the delta-ray threshold (chi-square over the energy fraction
    of the slower electron), and the two-body relation between its energy and
    its angle."""
    phys = PD.build_block(["H2O700ICRU"], overrides={"eii_flag": 0})
    te = float(phys["te"][0])
    n = 200_000
    frac, cos, err = oracle.probe_moller(phys, 0, ekin, n, seed=11)
    assert err == 0 and (frac > 0).all()
    eps_min = te / ekin
    assert frac.min() >= eps_min * (1 - 1e-5) and frac.max() <= 0.5 + 1e-6
    edges = np.linspace(eps_min, 0.5, 41)
    obs, _ = np.histogram(frac, bins=edges)
    exp = _moller_bin_probs(ekin, eps_min, edges) * n
    chi2 = float(((obs - exp) ** 2 / exp).sum())
    assert chi2 < 40 + 4 * np.sqrt(2 * 40), chi2
    # cos^2 = (T + 2 mc^2) / T * T2 / (T2 + 2 mc^2) for the electron of kinetic energy T2
    t2 = frac.astype(np.float64) * ekin
    want = (ekin + 2 * RM) / ekin * t2 / (t2 + 2 * RM)
    np.testing.assert_allclose(cos.astype(np.float64) ** 2, want, rtol=2e-4, atol=2e-6)


def _sauter_bin_probs(ekin, edges):
    """Sauter's K-shell photoelectron angular distribution over cos(theta):
    sin^2 / (1 - beta c)^4 * [1 + gamma (gamma - 1)(gamma - 2) (1 - beta c) / 2]."""
    g = 1.0 + ekin / RM
    b = np.sqrt(1.0 - 1.0 / (g * g))
    c = np.linspace(-1.0, 1.0, 400001)
    f = (1 - c * c) / (1 - b * c) ** 4 * (1 + 0.5 * g * (g - 1) * (g - 2) * (1 - b * c))
    cdf = np.concatenate([[0.0], np.cumsum((f[1:] + f[:-1]) / 2 * np.diff(c))])
    p = np.diff(np.interp(edges, c, cdf))
    return p / p.sum()


@pytest.mark.parametrize("energy", [0.03, 0.1, 0.5])
def test_photoelectron_direction_follows_sauter(oracle, energy):
    """With photoelectron angular sampling on and atomic relaxation off, the
    photoelectron takes the photon's energy and leaves along Sauter's
    distribution (chi-square over the cosine)."""
    phys = PD.build_block(["H2O700ICRU"])
    n = 200_000
    ekin, cos, err = oracle.probe_photo(phys, 0, 0x20, energy, n, seed=13)
    assert err == 0 and (cos <= 1.0).all()
    np.testing.assert_allclose(ekin, energy, rtol=1e-5)
    edges = np.linspace(-1.0, 1.0, 41)
    obs, _ = np.histogram(cos, bins=edges)
    exp = _sauter_bin_probs(energy, edges) * n
    keep = exp > 5
    chi2 = float(((obs[keep] - exp[keep]) ** 2 / exp[keep]).sum())
    dof = int(keep.sum())
    assert chi2 < dof + 4 * np.sqrt(2 * dof), (chi2, dof)
