"""Learned interface preconditioner: data generation on the CPU (random
fields, divergence-free curl-T sources) and, on the GPU, the MLP inference
kernel against a NumPy restatement with BF16-rounded weights, training and
flexible-CG solves checked by the true FP64 residual."""
import ctypes as C

import numpy as np
import pytest

from emagddm_b200 import _abi, learned, mesh
from oracle import oracle as O


def test_random_fields_statistics():
    rng = np.random.default_rng(1)
    f = learned.grf(16, 0.1, 1.5, rng, components=2)
    assert f.shape == (2, 16, 16, 16)
    assert abs(f[0].std() - 1.5) < 1e-9 and abs(f[0].mean()) < 1e-9
    mu = learned.random_mu(16, np.random.default_rng(2))
    assert mu.min() >= 1.0 and mu.max() <= 2000.0 and mu.size == 16 ** 3


def test_curl_t_source_is_orthogonal_to_gradients():
    """F_i = int curl(N_i) . T annihilates the discrete gradient of every
    interior nodal hat function (exactly, T constant per tet)."""
    m = mesh.perturbed(mesh.plain_small(6), 0.2, seed=1)
    d = O.dof_build(m.tets, m.dirichlet, gauge=O.GAUGE_NONE)
    T = learned.grf(6, 0.15, 1.0, np.random.default_rng(3), components=3).reshape(3, -1)
    F = learned.curl_t_rhs(m, d["l2g"], T, int(d["n_dofs"]))
    en = d["edge_nodes"].reshape(-1, 2)
    ed = d["edge_dof"].ravel()
    g = np.zeros(m.n_nodes)
    free = ed >= 0
    np.add.at(g, en[free, 1], F[ed[free]])   # +1 at the head (higher node)
    np.add.at(g, en[free, 0], -F[ed[free]])  # -1 at the tail
    interior = np.all((m.xyz > 1e-12) & (m.xyz < 1 - 1e-12), axis=1)
    assert np.abs(g[interior]).max() <= 1e-12 * np.abs(F).max()


def bf16(a):
    u = np.asarray(a, np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


@pytest.mark.gpu
def test_learned_preconditioner_kernels_and_solves():
    import torch
    tr = learned.Trainer(n=8, parts=2, seed=5)
    L = _abi.lib()
    rng = np.random.default_rng(0)
    b = tr.field(rng)
    rhs = tr.lambda_rhs(b)
    # untrained network (W3 = 0): the learned correction is zero
    z2 = tr.op(2, rhs)
    assert float(z2.abs().max()) == 0.0
    _, rc2, o2 = tr.fd.solve_rhs(b.cpu().numpy(), tol=1e-10, precond=2)
    x4, rc4, o4 = tr.fd.solve_rhs(b.cpu().numpy(), tol=1e-10, precond=4)
    assert rc2 == rc4 == 0 and abs(o2.iterations - o4.iterations) <= 2
    # inference against NumPy with random weights (BF16 forward)
    n = C.c_int64()
    L.emg_fetidp_learned_params(tr.fd.h, None, C.byref(n), 0)
    W = np.random.default_rng(1).normal(scale=0.05, size=n.value).astype(np.float32)
    _abi.check(L.emg_fetidp_learned_params(tr.fd.h, _abi.ptr(W), C.byref(n), 1), "load")
    z = tr.op(2, rhs).cpu().numpy()
    from emagddm_b200 import fetidp
    r = rhs.cpu().numpy()
    lay = fetidp.dual_layout(tr.fd)
    c = np.zeros(lay["n_entries"])
    off = 0
    for s in range(lay["n_parts"]):
        e0, e1 = lay["dual_off"][s], lay["dual_off"][s + 1]
        k = int(e1 - e0)
        x = lay["dual_sign"][e0:e1] * r[lay["dual_lam"][e0:e1]]
        nm = np.linalg.norm(x) or 1.0
        x = (x / nm).astype(np.float32)
        P = bf16(W[off:off + 2 * 256 * k + 2 * 256 + 256 * 256 + k])
        w1 = P[:256 * k].reshape(256, k); b1 = P[256 * k:256 * k + 256]
        w2 = P[256 * k + 256:256 * k + 256 + 65536].reshape(256, 256); b2 = P[256 * k + 65792:256 * k + 66048]
        w3t = P[256 * k + 66048:512 * k + 66048].reshape(256, k); b3 = P[512 * k + 66048:]
        h1 = np.maximum(w1 @ x + b1, 0)
        h2 = np.maximum(w2 @ h1 + b2, 0)
        c[e0:e1] = nm * (w3t.T @ h2 + b3)
        off += P.size
    le = lay["lam_entry"]
    zref = 0.5 * (c[le[:, 0]] - c[le[:, 1]])
    assert np.abs(z - zref).max() <= 1e-4 * np.abs(zref).max()
    # training on pairs lowers the loss; learned solves still converge to the same x
    _abi.check(L.emg_fetidp_learned_init(tr.fd.h, 7), "init")
    R, T = tr.pairs(rng, per_solve=6, stride=2)
    losses = tr.train(R, T, epochs=15, batch=6, lr=1e-3)
    assert losses[-1] < 0.7 * losses[0], (losses[0], losses[-1])
    # (pairs() factored a new field: compare both preconditioners on it)
    x6, rc6, o6 = tr.fd.solve_rhs(b.cpu().numpy(), tol=1e-10, precond=2)
    x5, rc5, o5 = tr.fd.solve_rhs(b.cpu().numpy(), tol=1e-10, precond=4)
    assert rc5 == rc6 == 0 and o5.residual_norm <= 1e-10
    assert np.linalg.norm(x5 - x6) <= 1e-8 * np.linalg.norm(x6)
