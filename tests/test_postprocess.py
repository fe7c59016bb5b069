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


def _plane(dose, b, start, sizes, dims):
    """The voxel whose centre is nearest each point of the comparison plane (ties never occur here)."""
    c = [(bb[:-1].astype(np.float64) + bb[1:]) / 2 for bb in b]
    out = []
    for k in range(dims[2]):
        for j in range(dims[1]):
            for i in range(dims[0]):
                p = [start[a] + sizes[a] * (i, j, k)[a] for a in range(3)]
                idx = [int(np.argmin(np.abs(c[a] - p[a]))) for a in range(3)]
                out.append(dose[idx[2], idx[1], idx[0]])
    return np.array(out, np.float32)


def test_relative_dose_samples_and_grades_like_the_detector_array_comparison():
    from gegs_b200.postprocess import relative_dose, sample_plane
    rng = np.random.default_rng(5)
    dose, b = _grid(rng)
    c = [(bb[:-1] + bb[1:]) / 2 for bb in b]
    start, sizes, dims = (float(c[0][2]), float(c[1][7]), float(c[2][1])), (0.3, 0.0, 0.5), (12, 1, 6)
    calc = sample_plane(dose, *b, start, sizes, dims)
    np.testing.assert_array_equal(calc, _plane(dose, b, start, sizes, dims))
    lines, tot, ok = relative_dose(dose, *b, start, sizes, dims)
    assert lines == [f"{v:f}" for v in calc] and tot == ok == 0
    with pytest.raises(ValueError, match="outside"):
        sample_plane(dose, *b, (float(c[0][-1]) + 1.0, 0.0, 0.0), sizes, (1, 1, 1))

    # measured values in cGy (x100 when not normalised): identical except planted misses
    meas = calc / np.float32(100)
    meas[[5, 20, 40]] *= np.float32(1.08)
    meas[30] = np.float32(0.0)                                # below 10 % of the maximum: not compared
    lines, tot, ok = relative_dose(dose, *b, start, sizes, dims, meas, norm_type=0, array_type=1,
                                   gamma_len_cm=0.3, gamma_dos=0.03)
    assert tot == calc.size - 1 and ok == tot - 3
    flags = [int(l.split()[2]) for l in lines[:-1]]
    assert flags[5] == flags[20] == flags[40] == -1 and flags[30] == 0
    assert lines[-1] == f"Totally {tot} points compared, {ok} passed, percentage = {ok / tot * 100:.0f} %"

    # normalised to the maximum: a uniform scale of the measurement changes nothing
    _, tot1, ok1 = relative_dose(dose, *b, start, sizes, dims, meas * np.float32(3.7), norm_type=1,
                                 array_type=1, gamma_dos=0.03)
    assert (tot1, ok1) == (tot, ok)

    # the 1000-chamber array: a miss passes when a neighbour on the row (x) or across rows (z) agrees
    row = np.full(12 * 6, 2.0, np.float32)
    calc2 = row.copy()
    calc2[13] = np.float32(2.2)                                # 10 % off; every neighbour agrees
    d2 = np.zeros((10, 14, 18), np.float32)
    lines, tot, ok = relative_dose(_embed(d2, b, start, sizes, dims, calc2), *b, start, sizes, dims,
                                   row / np.float32(100), array_type=2, gamma_len_cm=0.3, gamma_dos=0.03)
    assert ok == tot == row.size
    # with a 2 mm distance criterion the neighbour's 0.25 cm offset alone exceeds it
    lines, tot, ok = relative_dose(_embed(d2, b, start, sizes, dims, calc2), *b, start, sizes, dims,
                                   row / np.float32(100), array_type=2, gamma_len_cm=0.2, gamma_dos=0.03)
    assert ok == tot - 1 and int(lines[13].split()[2]) == -1


def _embed(d, b, start, sizes, dims, vals):
    """A dose grid whose comparison-plane samples are `vals`."""
    d = d.copy()
    c = [(bb[:-1].astype(np.float64) + bb[1:]) / 2 for bb in b]
    n = 0
    for k in range(dims[2]):
        for j in range(dims[1]):
            for i in range(dims[0]):
                p = [start[a] + sizes[a] * (i, j, k)[a] for a in range(3)]
                idx = [int(np.argmin(np.abs(c[a] - p[a]))) for a in range(3)]
                d[idx[2], idx[1], idx[0]] = vals[n]
                n += 1
    return d


def test_measured_data_file_takes_the_first_number_of_each_line(tmp_path):
    from gegs_b200.postprocess import read_measured
    (tmp_path / "m.txt").write_text("1.5 x y\n2.5\n\n3.5 7\n4.5\n")
    np.testing.assert_array_equal(read_measured(tmp_path / "m.txt", 3), np.float32([1.5, 2.5, 3.5]))
    with pytest.raises(ValueError):
        read_measured(tmp_path / "m.txt", 5)


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
