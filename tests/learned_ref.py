"""CPU reference of the learned preconditioner network (test infrastructure).

Mirrors src_b200/csrc/learned.cuh: the same parameter layout, the same face couplings and node
features, and — with ``bf16=True`` — rounding to BF16 at the points where the GPU stores BF16
(activations, layer inputs, layer weights, the upstream gradient of a layer).  Forward and
backward are written out explicitly; ``torch_forward`` restates the forward pass in torch so the
explicit backward can be checked against autograd in FP64.
"""
from __future__ import annotations

import numpy as np

C, FIN, K3, NL = 32, 4, 96, 3
OFF_WIN = 0
OFF_BIN = OFF_WIN + C * FIN
OFF_L0 = OFF_BIN + C
LSTRIDE = C * K3 + C
OFF_WOUT = OFF_L0 + NL * LSTRIDE
OFF_BOUT = OFF_WOUT + C
NPARAM = OFF_BOUT + 1


def bf16(x):
    """Round float32 values to bfloat16 (nearest even), returned as float32."""
    a = np.ascontiguousarray(x, np.float32)
    u = a.view(np.uint32)
    r = ((u >> 16) & 1) + np.uint32(0x7FFF)
    return ((u + r) & np.uint32(0xFFFF0000)).view(np.float32)


class Geometry:
    """Face couplings and node features of the network for a reference-layout mesh."""

    def __init__(self, rm, rh0, vol, coefw, dt):
        i1, i2 = rm.iedge[:, 0].astype(np.int64), rm.iedge[:, 1].astype(np.int64)
        S = rm.sn
        vert = (rm.coord[i1, 0] == rm.coord[i2, 0]) & (rm.coord[i1, 1] == rm.coord[i2, 1])
        rhof = 0.5 * (rh0[i1] + rh0[i2])
        volf = 0.5 * (vol[i1] + vol[i2])
        cwf = 0.5 * (coefw[i1] + coefw[i2])
        s2h = S[:, 0] ** 2 + S[:, 1] ** 2 + S[:, 2] ** 2
        s2v = S[:, 0] ** 2 + S[:, 1] ** 2 + S[:, 2] ** 2 * cwf
        T = np.where(vert, 0.5 * dt * s2v * rhof / volf, 0.5 * dt * s2h * rhof / volf).astype(np.float32)
        n = rm.npoin
        self.n, self.i1, self.i2, self.vert, self.T = n, i1, i2, vert, T
        Dh = np.zeros(n, np.float32)
        Dv = np.zeros(n, np.float32)
        for D, m in ((Dh, ~vert), (Dv, vert)):
            np.add.at(D, i1[m], T[m])
            np.add.at(D, i2[m], T[m])
        self.iDh = np.where(Dh > 0, 1.0 / np.maximum(Dh, 1e-30), 0).astype(np.float32)
        self.iDv = np.where(Dv > 0, 1.0 / np.maximum(Dv, 1e-30), 0).astype(np.float32)
        self.feat2 = np.where((Dh > 0) & (Dv > 0), np.log(np.maximum(Dv, 1e-30) / np.maximum(Dh, 1e-30)) / 8.0,
                              0).astype(np.float32)
        # top/bottom nodes = nodes with exactly one vertical face
        nv = np.zeros(n, np.int64)
        np.add.at(nv, i1[vert], 1)
        np.add.at(nv, i2[vert], 1)
        self.bnd = (nv == 1).astype(np.float32)
        # |diagonal| of the line matrix (impfl = 1), the restatement of the library's set-up
        hx = np.zeros(n)
        for d in range(3):
            s2 = S[:, d] ** 2
            m = ~vert
            np.add.at(hx, i1[m], s2[m] * rh0[i2[m]] / vol[i2[m]])
            np.add.at(hx, i2[m], s2[m] * rh0[i1[m]] / vol[i1[m]])
        Tl = (0.5 * dt) * ((S[:, 0] ** 2 + S[:, 1] ** 2) + (S[:, 2] ** 2) * cwf) * rhof / volf
        av_ = np.zeros(n)
        np.add.at(av_, i1[vert], Tl[vert])
        np.add.at(av_, i2[vert], Tl[vert])
        vr = vol * rh0
        dh = -((0.5 * dt) * hx) / ((4.0 * vol) * rh0)
        b = dh - av_ / vr
        self.bdiag = np.abs(b).astype(np.float32)

    def aggregate(self, h, mode):
        """A_h (mode 'h') or A_v ('v') of node features h [n, C] in float32."""
        m = self.vert if mode == "v" else ~self.vert
        iD = self.iDv if mode == "v" else self.iDh
        dt = h.dtype
        a = np.zeros_like(h)
        i1, i2, T = self.i1[m], self.i2[m], self.T[m].astype(dt)
        w1 = T * iD[i1].astype(dt)
        w2 = T * iD[i2].astype(dt)
        np.add.at(a, i1, w1[:, None] * (h[i2] - h[i1]))
        np.add.at(a, i2, w2[:, None] * (h[i1] - h[i2]))
        return a

    def spread(self, G, mode):
        """Transpose of the weights of `aggregate` applied to per-node G (already scaled by iD)."""
        m = self.vert if mode == "v" else ~self.vert
        out = np.zeros_like(G, dtype=np.float64)
        i1, i2, T = self.i1[m], self.i2[m], self.T[m].astype(np.float64)
        np.add.at(out, i1, T[:, None] * G[i2])
        np.add.at(out, i2, T[:, None] * G[i1])
        return out


def unpack(prm):
    p = np.asarray(prm, np.float64)
    Win = p[OFF_WIN:OFF_WIN + C * FIN].reshape(C, FIN)
    bin_ = p[OFF_BIN:OFF_BIN + C]
    Ws = [p[OFF_L0 + l * LSTRIDE: OFF_L0 + l * LSTRIDE + C * K3].reshape(C, K3) for l in range(NL)]
    bs = [p[OFF_L0 + l * LSTRIDE + C * K3: OFF_L0 + (l + 1) * LSTRIDE] for l in range(NL)]
    return Win, bin_, Ws, bs, p[OFF_WOUT:OFF_WOUT + C], p[OFF_BOUT]


def forward(prm, r, z, geo: Geometry, rnd=True):
    R = bf16 if rnd else (lambda a: np.asarray(a, np.float64))
    Win, bin_, Ws, bs, wout, bout = unpack(prm)
    s = np.abs(r).max()
    s = s if s > 0 else 1.0
    x = np.stack([r / s, z * geo.bdiag.astype(np.float64) / s, geo.feat2, geo.bnd], axis=1)
    x = x.astype(np.float32) if rnd else x
    H = [R(np.maximum(x @ Win.T + bin_, 0))]
    Xs = []
    for l in range(NL):
        h = H[-1]
        hc = np.asarray(h, np.float32 if rnd else np.float64)
        X = np.concatenate([hc, geo.aggregate(hc, "h"), geo.aggregate(hc, "v")], axis=1)
        X = R(X)
        Xs.append(X)
        W = R(Ws[l]) if rnd else Ws[l]
        H.append(R(np.maximum(X.astype(np.float64) @ W.T.astype(np.float64) + bs[l], 0)))
    y = H[-1].astype(np.float64) @ wout + bout
    q = z + y * s / geo.bdiag.astype(np.float64)
    return {"s": s, "x": x, "H": H, "Xs": Xs, "y": y, "q": q}


def backward(prm, fw, t, z, geo: Geometry, rnd=True, dy=None):
    """Gradient of the error loss for target t, or, with `dy` given, of any loss whose
    derivative w.r.t. the network output y is dy (the loss is then returned as None)."""
    R = bf16 if rnd else (lambda a: np.asarray(a, np.float64))
    Win, bin_, Ws, bs, wout, bout = unpack(prm)
    g = np.zeros(NPARAM)
    if dy is None:
        n = len(t)
        ystar = (t - z) * geo.bdiag.astype(np.float64) / fw["s"]
        e = fw["y"] - ystar
        loss = 0.5 * np.sum(e * e) / n
        dy = e / n
    else:
        loss = None
    H = fw["H"]
    g[OFF_WOUT:OFF_WOUT + C] = dy @ H[3].astype(np.float64)
    g[OFF_BOUT] = dy.sum()
    dH = np.outer(dy, wout)
    for l in range(NL - 1, -1, -1):
        du = np.where(H[l + 1] > 0, dH, 0.0)
        du = R(du).astype(np.float64) if rnd else du
        W = (R(Ws[l]) if rnd else Ws[l]).astype(np.float64)
        X = fw["Xs"][l].astype(np.float64)
        g[OFF_L0 + l * LSTRIDE: OFF_L0 + l * LSTRIDE + C * K3] = (du.T @ X).ravel()
        g[OFF_L0 + l * LSTRIDE + C * K3: OFF_L0 + (l + 1) * LSTRIDE] = du.sum(0)
        dX = du @ W
        dself, dah, dav = dX[:, :C], dX[:, C:2 * C], dX[:, 2 * C:]
        dah = np.where(geo.iDh[:, None] > 0, dah, 0)
        dav = np.where(geo.iDv[:, None] > 0, dav, 0)
        Gh = dah * geo.iDh[:, None]
        Gv = dav * geo.iDv[:, None]
        dH = dself - dah - dav + geo.spread(Gh, "h") + geo.spread(Gv, "v")
    du0 = np.where(H[0] > 0, dH, 0.0)
    g[OFF_WIN:OFF_WIN + C * FIN] = (du0.T @ fw["x"].astype(np.float64)).ravel()
    g[OFF_BIN:OFF_BIN + C] = du0.sum(0)
    return loss, g


def torch_loss(prm, r, z, t, geo: Geometry):
    """The same network and loss in torch FP64 without rounding (for autograd)."""
    import torch
    P = torch.tensor(np.asarray(prm, np.float64), requires_grad=True)
    Win = P[OFF_WIN:OFF_WIN + C * FIN].reshape(C, FIN)
    bin_ = P[OFF_BIN:OFF_BIN + C]
    s = float(np.abs(r).max())
    bd = torch.tensor(geo.bdiag.astype(np.float64))
    x = torch.stack([torch.tensor(r / s), torch.tensor(z) * bd / s, torch.tensor(geo.feat2.astype(np.float64)),
                     torch.tensor(geo.bnd.astype(np.float64))], 1)
    h = torch.relu(x @ Win.T + bin_)

    def agg(h, mode):
        m = geo.vert if mode == "v" else ~geo.vert
        iD = torch.tensor((geo.iDv if mode == "v" else geo.iDh).astype(np.float64))
        i1, i2 = torch.tensor(geo.i1[m]), torch.tensor(geo.i2[m])
        T = torch.tensor(geo.T[m].astype(np.float64))
        a = torch.zeros_like(h)
        a = a.index_add(0, i1, (T * iD[i1])[:, None] * (h[i2] - h[i1]))
        a = a.index_add(0, i2, (T * iD[i2])[:, None] * (h[i1] - h[i2]))
        return a

    for l in range(NL):
        W = P[OFF_L0 + l * LSTRIDE: OFF_L0 + l * LSTRIDE + C * K3].reshape(C, K3)
        b = P[OFF_L0 + l * LSTRIDE + C * K3: OFF_L0 + (l + 1) * LSTRIDE]
        X = torch.cat([h, agg(h, "h"), agg(h, "v")], 1)
        h = torch.relu(X @ W.T + b)
    y = h @ P[OFF_WOUT:OFF_WOUT + C] + P[OFF_BOUT]
    ystar = torch.tensor((t - z) * geo.bdiag.astype(np.float64) / s)
    loss = 0.5 * torch.sum((y - ystar) ** 2) / len(t)
    loss.backward()
    return float(loss.detach()), P.grad.numpy()


def init_params(seed=0, out_scale=0.0):
    """Same initialisation law as mpg_learned_init (values differ: numpy RNG)."""
    rng = np.random.default_rng(seed)
    p = np.zeros(NPARAM, np.float32)
    p[OFF_WIN:OFF_WIN + C * FIN] = rng.normal(0, np.sqrt(2 / FIN), C * FIN)
    p[OFF_BIN:OFF_BIN + C] = 0.01
    for l in range(NL):
        p[OFF_L0 + l * LSTRIDE: OFF_L0 + l * LSTRIDE + C * K3] = rng.normal(0, np.sqrt(2 / K3), C * K3)
        p[OFF_L0 + l * LSTRIDE + C * K3: OFF_L0 + (l + 1) * LSTRIDE] = 0.01
    p[OFF_WOUT:OFF_WOUT + C] = rng.normal(0, out_scale, C) if out_scale else 0.0
    return p
