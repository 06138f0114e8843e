"""CPU oracle of the learned initial guess of the Crank-Nicolson solve.

Test infrastructure only: the tests use it to check the CUDA kernels of the
learned form (features, per-sample statistics, the MLP forward and backward
passes and Adam).  The reference has no learned component, so nothing here
follows a reference file; the guess it serves replaces the extrapolated start
x0 = 2 RHS - psi of the Crank-Nicolson solve (RHS = A psi, solve A^H x = RHS,
src/nrqcd.f90:1112-1123).

Learned guess.  Per sample (site, species) with psi (36 complex), the
right-hand side b = A psi, u = b - psi and the history v1, v2 = what the
extrapolation 2 b - psi missed in the previous two steps
(t = x - (2 b - psi) of those steps):

    x0 = 2 b - psi + w0 s0 u + w1 v1 + w2 v2,   (w0, w1, w2) complex = MLP(features)

a per-site linear prediction of this step's miss t; s0 = |tau| (tau = dt a0 / 2)
scales u = O(tau H psi) to the size of the misses.  The MLP is
16 -> 64 -> 64 -> 6 with ReLU, BF16 weights and activations and FP32
accumulation.  Training minimises sum_s |sum_j w_j e_j - t|^2 (e = s0 u, v1, v2)
from exact solves; per sample only the Gram statistics G_jk = <e_j, e_k>,
g_j = <e_j, t> and |t|^2 enter.

Rounding points (mirrored by the kernels): features, weights, hidden
activations and backward gradients are rounded to BF16 (round to nearest
even) where they feed a matrix product; sums accumulate in FP64 here and in
FP32 on the device; biases and their gradients stay FP32.
"""
from __future__ import annotations

import numpy as np

NIN, NH, NOUT = 16, 64, 6
NBASIS = 3  # u, v1, v2
# the output bias is per group b3[group]: species (sign of feature 9) x history
# depth (2 x feature 10): group = 3 * (species) + depth
NGROUP = 6
SIZES = (("w1", (NH, NIN)), ("b1", (NH,)), ("w2", (NH, NH)), ("b2", (NH,)), ("w3", (NOUT, NH)),
         ("b3", (NGROUP, NOUT)))
FEAT_SPECIES, FEAT_DEPTH = 9, 10
NPARAMS = sum(int(np.prod(s)) for _, s in SIZES)
# G00, G11, G22, Re/Im G01, Re/Im G02, Re/Im G12, Re/Im g0, Re/Im g1, Re/Im g2, Gtt
NSTATS = 16


def gram(stats):
    """(n, 3, 3) hermitian G, (n, 3) g and (n,) |t|^2 from the statistics rows."""
    s = np.asarray(stats, dtype=np.float64)
    n = s.shape[0]
    G = np.zeros((n, 3, 3), dtype=np.complex128)
    G[:, 0, 0], G[:, 1, 1], G[:, 2, 2] = s[:, 0], s[:, 1], s[:, 2]
    for (j, k), c in (((0, 1), 3), ((0, 2), 5), ((1, 2), 7)):
        G[:, j, k] = s[:, c] + 1j * s[:, c + 1]
        G[:, k, j] = np.conj(G[:, j, k])
    g = np.stack([s[:, 9] + 1j * s[:, 10], s[:, 11] + 1j * s[:, 12], s[:, 13] + 1j * s[:, 14]], 1)
    return G, g, s[:, 15]


def unpack(p):
    out, o = {}, 0
    for name, shape in SIZES:
        k = int(np.prod(shape))
        out[name] = np.asarray(p[o:o + k], dtype=np.float64).reshape(shape)
        o += k
    return out


def pack(d):
    return np.concatenate([np.asarray(d[name], dtype=np.float32).ravel() for name, _ in SIZES])


def bf16(a):
    """Round to BF16 (nearest even), returned as float64 values."""
    f = np.ascontiguousarray(np.asarray(a, dtype=np.float32))
    u = f.view(np.uint32).astype(np.uint64)
    u = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def f32(a):
    return np.asarray(a, dtype=np.float32).astype(np.float64)


def forward(p, feat):
    """Outputs (n, 6) and the intermediates of the backward pass."""
    w = unpack(p)
    X = bf16(feat)
    W1, W2, W3 = bf16(w["w1"]), bf16(w["w2"]), bf16(w["w3"])
    H1 = f32(np.maximum(X @ W1.T + w["b1"], 0.0))
    H1b = bf16(H1)
    H2 = f32(np.maximum(H1b @ W2.T + w["b2"], 0.0))
    H2b = bf16(H2)
    gr = group_of(feat)
    Y = f32(H2b @ W3.T + w["b3"][gr])
    return Y, (X, W1, W2, W3, H1b, H2b)


def group_of(feat):
    f = np.asarray(feat, dtype=np.float32)
    depth = np.clip(np.rint(2.0 * f[:, FEAT_DEPTH]), 0, 2).astype(int)
    return 3 * (f[:, FEAT_SPECIES] < 0).astype(int) + depth


def _bias_grad(dY, gr):
    g = np.zeros((NGROUP, dY.shape[1]))
    for k in range(NGROUP):
        g[k] = dY[gr == k].sum(0)
    return g


def _loss_dw(Y, stats):
    G, g, Gtt = gram(stats)
    w = Y[:, 0::2] + 1j * Y[:, 1::2]
    Gw = np.einsum("njk,nk->nj", G, w)
    L = np.real(np.einsum("nj,nj->n", np.conj(w), Gw)) - 2 * np.real(np.einsum("nj,nj->n", np.conj(w), g)) + Gtt
    d = Gw - g  # dL/d conj(w)
    dY = np.zeros_like(Y, dtype=np.float64)
    dY[:, 0::2] = 2 * d.real
    dY[:, 1::2] = 2 * d.imag
    return L, dY


def loss_and_dy(Y, stats, nbatch):
    """Mean over the batch of |sum_j w_j e_j - t|^2 (stats pre-normalised) and dL/dY."""
    L, dY = _loss_dw(np.asarray(Y, dtype=np.float64), stats)
    return float(L.sum() / nbatch), f32(dY / nbatch)


def loss_grad(p, feat, stats, nbatch=None):
    """Loss and gradient (NPARAMS) with the kernels' rounding points."""
    n = feat.shape[0]
    nbatch = n if nbatch is None else nbatch
    Y, (X, W1, W2, W3, H1b, H2b) = forward(p, feat)
    loss, dY = loss_and_dy(Y, stats, nbatch)
    dYb = bf16(dY)
    g = {"b3": _bias_grad(dY, group_of(feat)), "w3": dYb.T @ H2b}
    dH2 = f32((dYb @ W3) * (H2b > 0))
    g["b2"] = dH2.sum(0)
    dH2b = bf16(dH2)
    g["w2"] = dH2b.T @ H1b
    dH1 = f32((dH2b @ W2) * (H1b > 0))
    g["b1"] = dH1.sum(0)
    dH1b = bf16(dH1)
    g["w1"] = dH1b.T @ X
    return loss, pack(g)


def loss_grad_exact(p, feat, stats):
    """FP64 loss and gradient without rounding (finite-difference reference)."""
    w = unpack(p)
    X = np.asarray(feat, dtype=np.float64)
    A1 = X @ w["w1"].T + w["b1"]
    H1 = np.maximum(A1, 0)
    A2 = H1 @ w["w2"].T + w["b2"]
    H2 = np.maximum(A2, 0)
    gr = group_of(feat)
    Y = H2 @ w["w3"].T + w["b3"][gr]
    n = X.shape[0]
    L, dY = _loss_dw(Y, stats)
    dY = dY / n
    g = {"b3": _bias_grad(dY, gr), "w3": dY.T @ H2}
    dA2 = (dY @ w["w3"]) * (A2 > 0)
    g["b2"] = dA2.sum(0)
    g["w2"] = dA2.T @ H1
    dA1 = (dA2 @ w["w2"]) * (A1 > 0)
    g["b1"] = dA1.sum(0)
    g["w1"] = dA1.T @ X
    return float(L.sum() / n), np.concatenate([np.asarray(g[k]).ravel() for k, _ in SIZES])


def adam(p, g, m, v, step, lr, b1=0.9, b2=0.999, eps=1e-8):
    """One Adam step (step counts from 1); returns new (p, m, v)."""
    m = b1 * m + (1 - b1) * g
    v = b2 * v + (1 - b2) * g * g
    mh = m / (1 - b1 ** step)
    vh = v / (1 - b2 ** step)
    return p - lr * mh / (np.sqrt(vh) + eps), m, v


# ---------------------------------------------------------------- features
def _plaquette_retr(links, n, i, j):
    """Re Tr U_i(x) U_j(x+i) U_i(x+j)^dag U_j(x)^dag / 3 at every site.
    links: (V, 3, 3, 3) [site, dir, col, row] (Fortran links(row, col, dir, site))."""
    nx, ny, nz = n
    U = np.transpose(links, (0, 1, 3, 2))  # [site, dir, row, col]
    idx = np.arange(nx * ny * nz).reshape(nz, ny, nx)

    def shift(d):
        ax = {0: 2, 1: 1, 2: 0}[d]
        return np.roll(idx, -1, axis=ax).ravel()
    Ui, Uj = U[:, i], U[:, j]
    P = Ui @ Uj[shift(i)] @ np.conj(np.transpose(Ui[shift(j)], (0, 2, 1))) @ np.conj(np.transpose(Uj, (0, 2, 1)))
    return np.real(np.trace(P, axis1=1, axis2=2)) / 3.0


def features(n, links, efield, psi, b, v1, v2, mass, tau, species):
    """(V, 16) features of one species: psi, b (V, 6, 6) complex, history
    v1 (last step) and v2 (the one before) (V, 6, 6) or None, efield (V, 3, 8)."""
    V = psi.shape[0]
    ps = psi.reshape(V, 36)
    u = (b - psi).reshape(V, 36)
    h1 = np.zeros_like(ps) if v1 is None else v1.reshape(V, 36)
    h2 = np.zeros_like(ps) if v2 is None else v2.reshape(V, 36)
    nps = np.sum(np.abs(ps) ** 2, 1)
    nu = np.sum(np.abs(u) ** 2, 1)
    n1 = np.sum(np.abs(h1) ** 2, 1)
    n2 = np.sum(np.abs(h2) ** 2, 1)
    cpu = np.sum(np.conj(ps) * u, 1)
    cu1 = np.sum(np.conj(u) * h1, 1)
    c21 = np.sum(np.conj(h2) * h1, 1)
    f = np.zeros((V, 16))
    ok = nps > 0
    f[ok, 0] = cpu[ok].real / (nps[ok] * tau)
    f[ok, 1] = cpu[ok].imag / (nps[ok] * tau)
    f[ok, 2] = np.sqrt(nu[ok] / nps[ok]) / abs(tau)
    ok2 = (nu > 0) & (n1 > 0)
    den = np.sqrt(nu[ok2] * n1[ok2])
    f[ok2, 3] = cu1[ok2].real / den
    f[ok2, 4] = cu1[ok2].imag / den
    f[ok2, 5] = np.minimum(np.sqrt(n1[ok2] / nu[ok2]) / abs(tau), 50.0)
    ok3 = (n1 > 0) & (n2 > 0)
    den = np.sqrt(n1[ok3] * n2[ok3])
    f[ok3, 6] = c21[ok3].real / den
    f[ok3, 7] = c21[ok3].imag / den
    f[ok3, 8] = np.minimum(np.sqrt(n1[ok3] / n2[ok3]), 10.0)
    f[:, 9] = 1.0 if species == 0 else -1.0
    f[:, 10] = 0.5 * ((v1 is not None) + (v2 is not None))
    f[:, 11] = 1.0 - _plaquette_retr(links, n, 0, 1)
    f[:, 12] = 1.0 - _plaquette_retr(links, n, 1, 2)
    f[:, 13] = 1.0 - _plaquette_retr(links, n, 2, 0)
    f[:, 14] = np.sum(np.asarray(efield).reshape(V, 24) ** 2, 1)
    f[:, 15] = 1.0 / mass
    return f


def stats(psi, b, v1, v2, x, s0=1.0):
    """(V, 16) Gram statistics of one species for the basis (s0 u, v1, v2),
    t = x - (2 b - psi)."""
    V = psi.shape[0]
    e = [s0 * (b - psi).reshape(V, 36)]
    for h in (v1, v2):
        e.append(np.zeros((V, 36), dtype=np.complex128) if h is None else h.reshape(V, 36))
    t = (x - (2 * b - psi)).reshape(V, 36)
    G = lambda j, k: np.sum(np.conj(e[j]) * e[k], 1)  # noqa: E731
    gg = [np.sum(np.conj(e[j]) * t, 1) for j in range(3)]
    return np.stack([G(0, 0).real, G(1, 1).real, G(2, 2).real, G(0, 1).real, G(0, 1).imag, G(0, 2).real,
                     G(0, 2).imag, G(1, 2).real, G(1, 2).imag, gg[0].real, gg[0].imag, gg[1].real, gg[1].imag,
                     gg[2].real, gg[2].imag, np.sum(np.abs(t) ** 2, 1)], axis=1)
