"""Gradient of a dose objective with respect to per-beamlet fluence weights.

The dose is linear in the weights: every tagged primary's statistical weight
is multiplied by the weight of its beamlet. ``BeamletDose`` is a
``torch.autograd.Function``: its forward runs the transport with the weights
and returns the dose per voxel; its backward calls the engine's replay
(``gegs_backward``), which re-runs the same histories from their RNG
counters with unit weights and adds, for every energy deposit, energy x
dL/d(energy in that voxel) to the deposit's beamlet -- nothing per history is
stored. Objectives are ordinary torch expressions of the dose.

Finite differences with common random numbers (the same histories, so the
same random numbers, at w + d e_b and w - d e_b) check the gradient.
"""
from __future__ import annotations

import numpy as np
import torch

FIXED = 2.0 ** -30          # tally unit: MeV * 2^30 per voxel


class BeamletModel:
    """An engine holding a scene with a beamlet grid, the histories to run and
    the tally-to-dose conversion (dose = energy * unit / mass)."""

    def __init__(self, engine, job, hist_begin=0, hist_end=None, dose_unit=1.0, batch=0):
        self.engine = engine
        self.job = job
        self.h0 = hist_begin
        self.h1 = job.histories if hist_end is None else hist_end
        self.mass = job.voxel_mass()
        self.unit = float(dose_unit)
        self.batch = batch
        self.nb = engine.nbeamlets
        if self.nb == 0:
            raise ValueError("the engine's scene has no beamlet grid")
        self.forward_ms = self.backward_ms = 0.0

    def dose(self, w) -> np.ndarray:
        e = self.engine
        e.set_beamlet_weights(np.asarray(w, np.float32))
        e.reset_tally()
        st = e.run(self.h0, self.h1, batch=self.batch)
        self.forward_ms = st["device_ms"]
        return e.tally().astype(np.float64) * (FIXED * self.unit) / self.mass

    def launch_dose(self, w):
        """Queue the forward transport at weights w and return at once; dose
        plans on other engines can be queued before finish_dose."""
        e = self.engine
        e.set_beamlet_weights(np.asarray(w, np.float32))
        e.reset_tally()
        e.launch(self.h0, self.h1, batch=self.batch)

    def finish_dose(self) -> np.ndarray:
        st = self.engine.wait()
        self.forward_ms = st["device_ms"]
        return self.engine.tally().astype(np.float64) * (FIXED * self.unit) / self.mass

    def vjp(self, dL_dD) -> np.ndarray:
        """dL/dw from dL/dD (per voxel)."""
        g = np.asarray(dL_dD, np.float64).reshape(-1) * (self.unit / self.mass)
        out = self.engine.backward(self.h0, self.h1, g, batch=self.batch)
        self.backward_ms = self.engine.stats()["device_ms"]
        return out

    def calibrate(self, w, mask, value):
        """Set the dose unit so that the mean dose over `mask` at weights w is `value`."""
        self.unit = 1.0
        d = self.dose(w)
        m = d[mask].mean()
        if not m > 0:
            raise ValueError("no dose in the calibration region")
        self.unit = value / m
        return self.unit


class BeamletDose(torch.autograd.Function):
    @staticmethod
    def forward(ctx, w, model):
        ctx.model = model
        d = model.dose(w.detach().cpu().numpy())
        return torch.from_numpy(d).to(w.device)

    @staticmethod
    def backward(ctx, grad_dose):
        g = ctx.model.vjp(grad_dose.detach().cpu().numpy())
        return torch.from_numpy(g).to(grad_dose.device, torch.float64), None


def beamlet_dose(w: torch.Tensor, model: BeamletModel) -> torch.Tensor:
    return BeamletDose.apply(w, model)


def objective(dose: torch.Tensor, target, organ, prescription=60.0, limit=20.0) -> torch.Tensor:
    """mean over the target of (D - prescription)^2 plus the mean over the organ
    of max(D - limit, 0)^2."""
    t = torch.as_tensor(target, device=dose.device)
    o = torch.as_tensor(organ, device=dose.device)
    return ((dose[t] - prescription) ** 2).mean() + (torch.clamp(dose[o] - limit, min=0.0) ** 2).mean()


def fd_gradient(model: BeamletModel, w, beamlets, loss, delta=0.05):
    """Central differences of loss(dose) for the listed beamlets with common random numbers."""
    w = np.asarray(w, np.float64)
    out = []
    for b in beamlets:
        wp, wm = w.copy(), w.copy()
        wp[b] += delta
        wm[b] -= delta
        lp = loss(torch.from_numpy(model.dose(wp))).item()
        lm = loss(torch.from_numpy(model.dose(wm))).item()
        out.append((lp - lm) / (2 * delta))
    return np.array(out)


def beamlet_doses(model: BeamletModel, beamlets):
    """Dose of each listed beamlet alone at unit weight (the untagged part removed)."""
    zero = np.zeros(model.nb, np.float32)
    base = model.dose(zero)
    out = []
    for b in beamlets:
        w = zero.copy()
        w[b] = 1.0
        out.append(model.dose(w) - base)
    return out


def optimize_weights(model: BeamletModel, w0, target, organ, iterations=20, lr=0.05, prescription=60.0,
                     limit=20.0):
    """Projected gradient descent on the beamlet weights (kept >= 0): each
    iteration is one forward transport and one replay backward. Returns the
    final weights and the objective per iteration."""
    w = torch.tensor(np.asarray(w0, np.float64), requires_grad=True)
    history = []
    for _ in range(iterations):
        w.grad = None
        loss = objective(beamlet_dose(w, model), target, organ, prescription, limit)
        loss.backward()
        history.append(float(loss.detach()))
        with torch.no_grad():
            g = w.grad
            step = lr * float(w.abs().mean()) / max(float(g.abs().max()), 1e-30)
            w -= step * g
            w.clamp_(min=0.0)
    return w.detach().numpy(), history


def optimize_weights_batch(models, w0s, targets, organs, iterations=20, lr=0.05, prescription=60.0, limit=20.0):
    """optimize_weights on several plans at once: every iteration queues the
    forward transport of all plans (each engine on its own stream, so they run
    concurrently on the device), then takes each plan's objective, its replay
    backward and its projected step. Returns the final weights and the
    objective history of every plan."""
    ws = [np.asarray(w, np.float64).copy() for w in w0s]
    hist = [[] for _ in models]
    for _ in range(iterations):
        for m, w in zip(models, ws):
            m.launch_dose(w)
        doses = [m.finish_dose() for m in models]
        for k, (m, d) in enumerate(zip(models, doses)):
            dt = torch.from_numpy(d).requires_grad_(True)
            loss = objective(dt, targets[k], organs[k], prescription, limit)
            loss.backward()
            hist[k].append(float(loss.detach()))
            g = m.vjp(dt.grad.numpy())
            step = lr * float(np.abs(ws[k]).mean()) / max(float(np.abs(g).max()), 1e-30)
            ws[k] = np.maximum(ws[k] - step * g, 0.0)
    return ws, hist
