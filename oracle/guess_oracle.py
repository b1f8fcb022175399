"""CPU oracle for the learned-guess networks (test infrastructure only).

A numpy float64 restatement of the three-layer MLP the engine trains and runs
on the GPU: Z1 = X W1 + b1, H1 = silu(Z1), Z2 = H1 W2 + b2, H2 = silu(Z2),
Y = H2 W3 + b3, loss = mean((Y - T)^2) over all rows and outputs, and its
gradient by reverse-mode differentiation written out by hand. Parameters are
one flat vector laid out W1[din][hid], b1, W2[hid][hid], b2, W3[hid][dout], b3.
There is no reference counterpart (the reference's guess is SAD,
TinySCF.c:324-364); the oracle is pinned by central finite differences.

It also restates, in scalar Python, the network inputs: the atom-pair blocks,
their local frames and invariant features (pair_blocks), pinned by the
frame's own invariants (orthonormal rows, e_z along the pair) and by the
rotation invariance of the features checked in the tests.
"""
import math

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


# ---------------------------------------------------------------------------
# Pair blocks, local frames and invariant features of the learned guess,
# restated in scalar Python (double precision, the library's order of
# operations) from the definition: one block per atom (diagonal) and per pair
# closer than 4 A; a diagonal block's frame has e_z towards the nearest atom,
# an off-diagonal block's e_z runs from its first atom (the one with more
# basis functions) to the second with the origin at the midpoint; e_x points
# to the nearest atom more than 0.25 A off that axis; distances are ordered by
# (round(r / 1e-4 A), atom index). Features: element one-hots of both atoms,
# a diagonal flag, 8 Gaussians of the pair distance, and the 12 nearest other
# atoms within 5 A of the origin (local coordinates scaled by the cosine
# cutoff / 5 A, element one-hot and cutoff weight).

BOHR2A = 0.52917720859
PAIR_CUT = 4.0
ENV_CUT = 5.0
N_ENV = 12
DIN = 128
_SLOT = {0: 0, 5: 1, 6: 2, 7: 3}
_LAYOUT = {(0, 0, 1): 5, (0, 0, 0, 1, 1, 2): 15}


def _sub(a, b):
    return [a[0] - b[0], a[1] - b[1], a[2] - b[2]]


def _dot(a, b):
    return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]


def _unit(a):
    n = math.sqrt(_dot(a, a))
    if n < 1e-12:
        return a
    return [a[0] / n, a[1] / n, a[2] / n]


def _key(r_angstrom, idx):
    return (math.floor(r_angstrom * 1e4 + 0.5), idx)   # round half away from zero (r >= 0)


def _frame(origin, z, x_atom):
    if x_atom is not None:
        v = _sub(x_atom, origin)
        t = _dot(v, z)
        ex = _unit([v[k] - t * z[k] for k in range(3)])
    else:
        m = 0
        for k in (1, 2):
            if abs(z[k]) < abs(z[m]):
                m = k
        e = [0.0, 0.0, 0.0]
        e[m] = 1.0
        t = _dot(e, z)
        ex = _unit([e[k] - t * z[k] for k in range(3)])
    ey = [z[1] * ex[2] - z[2] * ex[1], z[2] * ex[0] - z[0] * ex[2], z[0] * ex[1] - z[1] * ex[0]]
    return [ex, ey, list(z)]


def _x_atom(xyz, origin, z, skip):
    best = None
    for c in range(len(xyz)):
        if c in skip:
            continue
        v = _sub(xyz[c], origin)
        key = _key(math.sqrt(_dot(v, v)) * BOHR2A, c)
        t = _dot(v, z)
        w = [v[k] - t * z[k] for k in range(3)]
        if math.sqrt(_dot(w, w)) * BOHR2A > 0.25 and (best is None or key < best[0]):
            best = (key, c)
    return None if best is None else xyz[best[1]]


def _features(elem, xyz, a, b, origin, Q):
    f = [0.0] * DIN
    f[_SLOT[elem[a]]] = 1.0
    f[4 + _SLOT[elem[b]]] = 1.0
    f[8] = 1.0 if a == b else 0.0
    if a != b:
        v = _sub(xyz[b], xyz[a])
        r = math.sqrt(_dot(v, v)) * BOHR2A
        for k in range(8):
            d = (r - (0.5 + 0.5 * k)) / 0.5
            f[9 + k] = math.exp(-d * d)
    env = []
    for c in range(len(xyz)):
        if c == a or c == b:
            continue
        v = _sub(xyz[c], origin)
        r = math.sqrt(_dot(v, v)) * BOHR2A
        if r < ENV_CUT:
            env.append(_key(r, c))
    env.sort()
    for k, (_, c) in enumerate(env[:N_ENV]):
        v = _sub(xyz[c], origin)
        r = math.sqrt(_dot(v, v)) * BOHR2A
        fc = 0.5 * (math.cos(math.pi * r / ENV_CUT) + 1.0) if r < ENV_CUT else 0.0
        o = 17 + 8 * k
        for d in range(3):
            f[o + d] = fc * _dot(Q[d], v) * BOHR2A / ENV_CUT
        f[o + 3 + _SLOT[elem[c]]] = fc
        f[o + 7] = fc
    return f


def pair_blocks(elem, xyz_bohr, shell_am):
    """[(a, b, type, Q (3x3 rows e_x e_y e_z), features (128 floats as float64))]
    in the library's block order, or None when an element or layout is not
    covered (H: s s p; C, N, O: s s s p p d)."""
    xyz = [list(map(float, r)) for r in xyz_bohr]
    na = len(xyz)
    nf = []
    for a in range(na):
        if elem[a] not in _SLOT or tuple(shell_am[a]) not in _LAYOUT:
            return None
        nf.append(_LAYOUT[tuple(shell_am[a])])
    out = []
    for a in range(na):
        near = None
        for c in range(na):
            if c != a:
                v = _sub(xyz[c], xyz[a])
                key = _key(math.sqrt(_dot(v, v)) * BOHR2A, c)
                if near is None or key < near[0]:
                    near = (key, c)
        if near is None:
            Q = [[1.0, 0.0, 0.0], [0.0, 1.0, 0.0], [0.0, 0.0, 1.0]]
        else:
            z = _unit(_sub(xyz[near[1]], xyz[a]))
            Q = _frame(xyz[a], z, _x_atom(xyz, xyz[a], z, (a, near[1])))
        out.append((a, a, 0 if nf[a] == 15 else 1, Q, _features(elem, xyz, a, a, xyz[a], Q)))
    cut = PAIR_CUT / BOHR2A
    for i in range(na):
        for j in range(i + 1, na):
            v = _sub(xyz[j], xyz[i])
            if math.sqrt(_dot(v, v)) >= cut:
                continue
            a, b = (j, i) if nf[j] > nf[i] else (i, j)
            t = 2 if (nf[a] == 15 and nf[b] == 15) else (3 if nf[a] == 15 else 4)
            mid = [0.5 * (xyz[a][k] + xyz[b][k]) for k in range(3)]
            z = _unit(_sub(xyz[b], xyz[a]))
            Q = _frame(mid, z, _x_atom(xyz, mid, z, (a, b)))
            out.append((a, b, t, Q, _features(elem, xyz, a, b, mid, Q)))
    return out
