"""Learned interface preconditioner for FETI-DP: data, training, evaluation.

The network itself (one 3-layer MLP per subdomain, width 256, BF16 weights,
FP32 accumulation) and its training step run in the library's own kernels
(``emg_fetidp_learned_*``); this module generates what it learns from:

* random permeability fields: log mu_r a Gaussian random field (Gaussian
  covariance, correlation length 0.1, sigma 1.5) per hex cell, clipped to
  mu_r in [1, 2000];
* random divergence-free currents J = curl T, T a Gaussian random vector
  field (correlation length 0.15), entering as F_i = int (curl N_i) . T
  (T constant per tet), so F is orthogonal to every discrete gradient;
* (residual, wanted correction) pairs that the FETI-DP solver itself
  produces: residuals r of deluxe-preconditioned multiplier CG runs, and
  t = F^-1 r - M_D r from an accurate inner solve, so that M_D + L approaches
  F^-1.

Evaluation solves held-out fields with the plain deluxe preconditioner and
with deluxe + learned (flexible CG); the true FP64 residual decides
convergence in both.
"""
from __future__ import annotations

import ctypes as C
import time

import numpy as np

from . import _abi, fetidp, mesh

NED_A = np.array([0, 1, 2, 0, 1, 2])
NED_B = np.array([1, 2, 0, 3, 3, 3])


def grf(n: int, corr: float, sigma: float, rng, components: int = 1) -> np.ndarray:
    """Gaussian random field on the n^3 cells of the unit cube (periodic FFT
    synthesis, Gaussian covariance of length `corr`), scaled to standard
    deviation `sigma`; shape (components, n, n, n), index [c][k][j][i]."""
    k = 2.0 * np.pi * np.fft.fftfreq(n, d=1.0 / n)
    kk = k[:, None, None] ** 2 + k[None, :, None] ** 2 + k[None, None, :] ** 2
    amp = np.exp(-0.25 * kk * corr ** 2)
    out = np.empty((components, n, n, n))
    for c in range(components):
        w = np.fft.fftn(rng.standard_normal((n, n, n)))
        f = np.real(np.fft.ifftn(w * amp))
        out[c] = sigma * (f - f.mean()) / max(f.std(), 1e-300)
    return out


def random_mu(n: int, rng, sigma: float = 1.5, corr: float = 0.1, lo: float = 1.0, hi: float = 2000.0):
    """mu_r per hex cell (n^3, cell index i + n (j + n k))."""
    return np.clip(np.exp(grf(n, corr, sigma, rng)[0]), lo, hi).ravel()


def tet_curls(xyz: np.ndarray, tets: np.ndarray):
    """Physical curls (T, 6, 3) of the Whitney functions in the Nedelec local
    order, with the global edge signs applied, and |det J| (T,)."""
    x = xyz[tets]                              # (T, 4, 3)
    d = x[:, :3, :] - x[:, 3:4, :]             # rows d0, d1, d2
    det = np.einsum("ti,ti->t", d[:, 0], np.cross(d[:, 1], d[:, 2]))
    a = d / det[:, None, None]
    c = np.stack([-2 * a[:, 2], -2 * a[:, 0], -2 * a[:, 1], -2 * a[:, 1] + 2 * a[:, 2],
                  2 * a[:, 0] - 2 * a[:, 2], -2 * a[:, 0] + 2 * a[:, 1]], axis=1)
    sg = np.where(tets[:, NED_B] < tets[:, NED_A], 1.0, -1.0)
    return c * sg[:, :, None], np.abs(det)


def curl_t_rhs(m, l2g: np.ndarray, T_cell: np.ndarray, n_dofs: int) -> np.ndarray:
    """F_i = sum over tets of |det|/6 (s_i curl_i) . T_t with T constant per
    hex cell (T_cell: (3, n^3)); the tets of cell c are 6c .. 6c+5."""
    c, adet = tet_curls(m.xyz, np.asarray(m.tets, np.int64))
    T = T_cell[:, np.arange(m.n_tets) // 6].T            # (T, 3)
    fe = (adet / 6.0)[:, None] * np.einsum("tkc,tc->tk", c, T)
    F = np.zeros(n_dofs)
    ok = l2g >= 0
    np.add.at(F, l2g[ok], fe[ok])
    return F


class Trainer:
    """FETI-DP on the n^3 cube split into parts^3 jittered boxes, one material
    per hex cell (so every field is a new nu array), with the learned
    preconditioner attached."""

    def __init__(self, n: int = 32, parts: int = 4, seed: int = 0, stream=None):
        import torch
        self.torch = torch
        base = mesh.plain_scale(n)
        self.n = n
        self.m = mesh.CubeMesh(**{**base.__dict__, "material": (np.arange(base.n_tets) // 6).astype(np.int32),
                                  "nu": np.ones(n ** 3), "sigma": np.zeros(n ** 3), "sources": []})
        self.fd = fetidp.FetiDP(self.m, mesh.jittered_partition(base, parts), parts ** 3, stream)
        self.nl = self.fd.info()["n_lambda"]
        self.n_dofs = self.fd.map.n_dofs
        self.dev = torch.device("cuda")
        _abi.check(_abi.lib().emg_fetidp_learned_init(self.fd.h, seed), "emg_fetidp_learned_init")
        self.L = _abi.lib()

    # -- multiplier-space helpers -------------------------------------------------
    def _ptr(self, t):
        return C.c_void_p(t.data_ptr())

    def op(self, which: int, v):
        out = self.torch.empty_like(v)
        _abi.check(self.L.emg_fetidp_apply(self.fd.h, which, self._ptr(v), self._ptr(out)), "emg_fetidp_apply")
        return out

    def field(self, rng):
        """Factor for a random mu field; returns the global right-hand side (device)."""
        mu = random_mu(self.n, rng)
        rc = self.fd.factor(nu=1.0 / mu, sigma=np.zeros(self.n ** 3))
        if rc:
            raise RuntimeError(f"factor {rc}: {self.L.emg_last_error().decode()}")
        T = grf(self.n, 0.15, 1.0, rng, components=3).reshape(3, -1)
        b = curl_t_rhs(self.m, self.fd.map.l2g, T, self.n_dofs)
        return self.torch.tensor(b, device=self.dev)

    def lambda_rhs(self, b):
        out = self.torch.empty(self.nl, dtype=self.torch.float64, device=self.dev)
        _abi.check(self.L.emg_fetidp_lambda_rhs(self.fd.h, self._ptr(b), self._ptr(out)), "emg_fetidp_lambda_rhs")
        return out

    def pcg(self, rhs, tol: float, max_it: int = 500, record=None):
        """Deluxe-preconditioned CG on F lam = rhs; residuals appended to `record`."""
        lam = self.torch.zeros_like(rhs)
        r = rhs.clone()
        z = self.op(1, r)
        p = z.clone()
        rz = float(r @ z)
        r0 = float(r.norm())
        for it in range(max_it):
            if record is not None:
                record.append(r.clone())
            q = self.op(0, p)
            a = rz / float(p @ q)
            lam += a * p
            r -= a * q
            if float(r.norm()) < tol * r0:
                return lam, it + 1
            z = self.op(1, r)
            rzn = float(r @ z)
            p = z + (rzn / rz) * p
            rz = rzn
        return lam, max_it

    def pairs(self, rng, per_solve: int = 8, stride: int = 3):
        """(residual, F^-1 r - M_D r) pairs from one random field."""
        b = self.field(rng)
        rec = []
        self.pcg(self.lambda_rhs(b), 1e-8, record=rec)
        rs = rec[::stride][:per_solve]
        R, T = [], []
        for r in rs:
            y, _ = self.pcg(r, 1e-9)
            R.append(r)
            T.append(y - self.op(1, r))
        return R, T

    def train(self, R, T, epochs: int = 20, batch: int = 32, lr: float = 1e-3, seed: int = 0):
        torch = self.torch
        Rm = torch.stack(R)
        Tm = torch.stack(T)
        g = np.random.default_rng(seed)
        losses = []
        loss = C.c_double()
        for _ in range(epochs):
            order = g.permutation(len(R))
            for s in range(0, len(order), batch):
                idx = torch.tensor(order[s:s + batch], device=self.dev)
                rb = Rm[idx].contiguous()
                tb = Tm[idx].contiguous()
                _abi.check(self.L.emg_fetidp_learned_train(self.fd.h, len(idx), self._ptr(rb), self._ptr(tb),
                                                           C.c_float(lr), C.byref(loss)), "learned_train")
                losses.append(loss.value)
        return losses

    def evaluate(self, rng, tol: float = 1e-8):
        """Solve one held-out field with deluxe (2) and deluxe + learned (4)."""
        b = self.field(rng).cpu().numpy()
        self.torch.cuda.synchronize()
        out = {}
        for pc in (2, 4):
            self.torch.cuda.synchronize()
            t0 = time.perf_counter()
            x, rc, res = self.fd.solve_rhs(b, tol=tol, max_iter=2000, precond=pc)
            dt = (time.perf_counter() - t0) * 1e3
            out[pc] = {"status": rc, "iterations": res.iterations, "residual": res.residual_norm, "ms": dt,
                       "x": x}
        return out
