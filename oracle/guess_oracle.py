"""CPU oracle for the learned-guess networks (test infrastructure only).

A numpy float64 restatement of the three-layer MLP the engine trains and runs
on the GPU: Z1 = X W1 + b1, H1 = silu(Z1), Z2 = H1 W2 + b2, H2 = silu(Z2),
Y = H2 W3 + b3, loss = mean((Y - T)^2) over all rows and outputs, and its
gradient by reverse-mode differentiation written out by hand. Parameters are
one flat vector laid out W1[din][hid], b1, W2[hid][hid], b2, W3[hid][dout], b3.
There is no reference counterpart (the reference's guess is SAD,
TinySCF.c:324-364); the oracle is pinned by central finite differences.
"""
import numpy as np


def param_count(din, hid, dout):
    return din * hid + hid + hid * hid + hid + hid * dout + dout


def split(p, din, hid, dout):
    o = 0
    out = []
    for shape in ((din, hid), (hid,), (hid, hid), (hid,), (hid, dout), (dout,)):
        size = int(np.prod(shape))
        out.append(p[o:o + size].reshape(shape))
        o += size
    return out


def silu(z):
    return z / (1.0 + np.exp(-z))


def dsilu(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def forward(p, X, din, hid, dout):
    W1, b1, W2, b2, W3, b3 = split(np.asarray(p, dtype=np.float64), din, hid, dout)
    Z1 = X @ W1 + b1
    H1 = silu(Z1)
    Z2 = H1 @ W2 + b2
    H2 = silu(Z2)
    return H2 @ W3 + b3, (Z1, H1, Z2, H2)


def loss_grad(p, X, T, din, hid, dout):
    X = np.asarray(X, dtype=np.float64)
    T = np.asarray(T, dtype=np.float64)
    W1, b1, W2, b2, W3, b3 = split(np.asarray(p, dtype=np.float64), din, hid, dout)
    Y, (Z1, H1, Z2, H2) = forward(p, X, din, hid, dout)
    R = Y - T
    loss = float(np.mean(R * R))
    dY = 2.0 * R / R.size
    gW3 = H2.T @ dY
    gb3 = dY.sum(0)
    dZ2 = (dY @ W3.T) * dsilu(Z2)
    gW2 = H1.T @ dZ2
    gb2 = dZ2.sum(0)
    dZ1 = (dZ2 @ W2.T) * dsilu(Z1)
    gW1 = X.T @ dZ1
    gb1 = dZ1.sum(0)
    g = np.concatenate([a.ravel() for a in (gW1, gb1, gW2, gb2, gW3, gb3)])
    return loss, g
