"""Dose interpolation, 3-D gamma and the CT ramp on the GPU against their
CPU counterparts (bit for bit: the same float operations in the same order),
and the point-dose read-out."""
import numpy as np
import pytest

from gegs_b200 import workloads as W


def _grid(rng, n=(18, 14, 10), sp=(0.3, 0.25, 0.5)):
    nx, ny, nz = n
    b = [np.cumsum(np.r_[-3.0, np.full(k, s)]).astype(np.float32) for k, s in zip(n, sp)]
    z, y, x = np.meshgrid(*(np.arange(k) for k in (nz, ny, nx)), indexing="ij")
    dose = (np.exp(-((x - 9) ** 2 + (y - 7) ** 2) / 30.0) * (1 + 0.1 * z) + rng.uniform(0, 0.02, (nz, ny, nx)))
    return dose.astype(np.float32), b


def _gamma_ref(r, e, sp, dta, dd_abs, cut_abs, search):
    """Brute-force minimum over all voxels within search*dta, in float32."""
    f = np.float32
    nz, ny, nx = r.shape
    rmax = f(search) * f(dta)
    R = [int(rmax / f(s)) for s in sp]
    offs = []
    for k in range(-R[2], R[2] + 1):
        for j in range(-R[1], R[1] + 1):
            for i in range(-R[0], R[0] + 1):
                px, py, pz = f(sp[0]) * f(i), f(sp[1]) * f(j), f(sp[2]) * f(k)
                d2 = f(f(f(px * px) + f(py * py)) + f(pz * pz))
                if d2 <= f(rmax * rmax):
                    offs.append((i, j, k, d2))
    inv_dta2 = f(1) / f(f(dta) * f(dta))
    inv_dd2 = f(1) / f(f(dd_abs) * f(dd_abs))
    g = np.full(r.shape, -1.0, np.float32)
    for (z, y, x), rv in np.ndenumerate(r):
        if not rv >= f(cut_abs):
            continue
        best = np.float32(np.inf)
        for i, j, k, d2 in offs:
            xx, yy, zz = x + i, y + j, z + k
            if 0 <= xx < nx and 0 <= yy < ny and 0 <= zz < nz:
                dd = f(e[zz, yy, xx] - rv)
                v = f(f(d2 * inv_dta2) + f(f(dd * dd) * inv_dd2))
                best = min(best, v)
        g[z, y, x] = np.sqrt(best)
    return g


def test_point_dose_interpolates_between_centres():
    from gegs_b200.postprocess import point_dose
    rng = np.random.default_rng(3)
    dose, b = _grid(rng)
    c = [(bb[:-1] + bb[1:]) / 2 for bb in b]
    # at a voxel centre the interpolated dose is that voxel's dose
    assert point_dose(dose, *b, (c[0][5], c[1][4], c[2][3])) == pytest.approx(float(dose[3, 4, 5]), rel=1e-6)
    mid = ((c[0][5] + c[0][6]) / 2, c[1][4], c[2][3])
    assert point_dose(dose, *b, mid) == pytest.approx(float(dose[3, 4, 5] + dose[3, 4, 6]) / 2, rel=1e-5)


@pytest.mark.gpu
def test_interp_dose_matches_the_oracle():
    from gegs_b200.postprocess import interp_dose
    from oracle.post_oracle import interp_dose as ref_interp
    rng = np.random.default_rng(1)
    dose, b = _grid(rng)
    args = ((-3.1, -3.05, -3.2), (0.11, 0.09, 0.2), (50, 40, 27))
    np.testing.assert_array_equal(interp_dose(dose, *b, *args), ref_interp(dose, *b, *args))


@pytest.mark.gpu
def test_gamma3d_matches_brute_force():
    from gegs_b200.postprocess import gamma3d
    rng = np.random.default_rng(2)
    ref, b = _grid(rng, n=(14, 12, 8))
    ev = (ref * (1 + rng.normal(0, 0.02, ref.shape))).astype(np.float32)
    ev = np.roll(ev, 1, axis=2)                     # a one-voxel shift in x
    sp = (0.3, 0.25, 0.5)
    g, rate = gamma3d(ref, ev, sp, dta=0.3, dd=0.03, cutoff=0.1, search=2.0)
    want = _gamma_ref(ref, ev, sp, 0.3, 0.03 * ref.max(), 0.1 * ref.max(), 2.0)
    np.testing.assert_array_equal(g, want)
    sel = want >= 0
    assert rate == pytest.approx(float((want[sel] <= 1).mean()))
    g0, rate0 = gamma3d(ref, ref, sp)
    assert rate0 == 1.0 and g0.max() == 0.0


@pytest.mark.gpu
def test_ct_ramp_matches_the_host_ramp():
    from gegs_b200.postprocess import ct_ramp
    rng = np.random.default_rng(4)
    media = ["AIR700ICRU", "LUNG700ICRU", "ICRUTISSUE700ICRU", "ICRPBONE700ICRU"]
    hu = rng.integers(-1100, 2600, 200_000).astype(np.int16)
    hu[:6] = [-1025, -1024, -974, -973, 1976, 1977]
    seg = [(media.index(n), ub, lo, hi) for n, ub, lo, hi in W.CT_RAMP]
    med, dens = ct_ramp(hu, seg, W.CT_LOWER)
    m_ref, d_ref = W.hu_to_material(hu, media)
    np.testing.assert_array_equal(med, m_ref)
    np.testing.assert_array_equal(dens, d_ref)
