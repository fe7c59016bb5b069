"""The package's transport against the reference's own, statistically.

``oracle/ref`` runs whole transports with the reference's ten stage kernels,
compiled from its sources (photon.cu, compton.cu, ..., electron.cu, with
geom.cu and the samplers): one CPU thread, every random number from a seeded
generator of its own, primaries put on the photon stack as the reference
loads them, the stage kernels run until every stack is empty
(``ref_transport`` in oracle/ref/ref_harness.cpp). The oracle transports
other histories of the same plan -- the CUDA path equals the oracle bit for
bit for any history range (tests/test_gpu_parity.py), so this compares the
GPU's dose with the reference's. Every field's histories are split in
halves, one for each side, so that both sides sample every field and no
phase-space record twice.

Per configuration, 20 batches on each side, the dose summed over blocks of
voxels; per block the batch mean and its standard error. Over the blocks
above 10 % of the maximum, the normalised differences
z = (a - b) / sqrt(sa^2 + sb^2) must behave like a consistent pair's: at
least 88 % within 2 (about 94 % is expected: Student t with 19 degrees of
freedom) and a mean square between 0.7 and 1.4. The total energy deposited
agrees within 3 combined standard errors."""
import numpy as np
import pytest

from gegs_b200 import workloads as W

NB = 20


def _refpin():
    from oracle import oracle as O
    from oracle import refpin as R
    O.build()
    R.build()
    if not R.available():
        pytest.skip("reference harness not built (reference sources absent)")
    return O, R


def _blocks(e, dims, f):
    nx, ny, nz = dims
    a = e.reshape(nz, ny, nx)
    a = a[: nz // f[2] * f[2], : ny // f[1] * f[1], : nx // f[0] * f[0]]
    return a.reshape(nz // f[2], f[2], ny // f[1], f[1], nx // f[0], f[0]).sum(axis=(1, 3, 5)).reshape(-1)


CASES = {
    # name: (job, histories per side, block of voxels)
    "c1": (lambda n: W.config1(histories=2 * n), 150_000, (5, 5, 5)),
    "c2": (lambda n: W.config2(histories=2 * n, nphsp=2 * n), 150_000, (10, 10, 10)),
    "c3": (lambda n: W.config3(histories=2 * n, nphsp=2 * n), 150_000, (16, 16, 8)),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_dose_agrees_with_the_reference_transport(name):
    O, R = _refpin()
    mk, n, blk = CASES[name]
    job = mk(n)
    sh = job.scene()
    dims = (sh.scene.nx, sh.scene.ny, sh.scene.nz)
    pair = R.Pair(job.physics, sh)
    ref, ora = [], []
    for b in range(NB):
        # each field's histories (and phase-space records) split in halves: the
        # first half for the reference, the second for the oracle; batch b takes
        # the b-th part of every field's half
        e_ref = np.zeros(dims[0] * dims[1] * dims[2])
        e_ora = np.zeros_like(e_ref)
        for fd in job.fields:
            hb, he = int(fd["hist_begin"]), int(fd["hist_end"])
            s = (he - hb) // 2 // NB
            e_ref += pair.transport(hb + b * s, hb + (b + 1) * s, seed=1000 + b)
            mid = hb + (he - hb) // 2
            t, _ = O.run(job.physics, sh, mid + b * s, mid + (b + 1) * s)
            e_ora += t.astype(np.float64) * 2.0 ** -30
        ref.append(_blocks(e_ref, dims, blk))
        ora.append(_blocks(e_ora, dims, blk))
    ref, ora = np.array(ref), np.array(ora)
    ma, mb = ref.mean(0), ora.mean(0)
    sa, sb = ref.std(0, ddof=1) / np.sqrt(NB), ora.std(0, ddof=1) / np.sqrt(NB)
    sel = (ma > 0.1 * ma.max()) & (mb > 0.1 * mb.max())
    assert sel.sum() >= 30, f"{name}: only {sel.sum()} blocks above 10 % of the maximum"
    z = (ma[sel] - mb[sel]) / np.sqrt(sa[sel] ** 2 + sb[sel] ** 2)
    within = float(np.mean(np.abs(z) < 2.0))
    msq = float(np.mean(z * z))
    ta, tb = ref.sum(1), ora.sum(1)
    zt = (ta.mean() - tb.mean()) / np.sqrt(ta.var(ddof=1) / NB + tb.var(ddof=1) / NB)
    print(f"{name}: {sel.sum()} blocks, {within:.3f} within 2 sigma, mean z^2 {msq:.3f}, "
          f"total energy z {zt:.2f} (ratio {ta.mean() / tb.mean():.4f})")
    assert within >= 0.88, f"{name}: {within:.3f} of the blocks within 2 sigma"
    assert 0.7 < msq < 1.4, f"{name}: mean z^2 {msq:.3f}"
    assert abs(zt) < 3.0, f"{name}: total energy differs by {zt:.2f} sigma"
