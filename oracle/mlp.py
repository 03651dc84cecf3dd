"""CPU oracle of the learned start's network and descriptors (test
infrastructure only): the same layout, activation and loss as the
library's kernels (include/imago_learned.h), in float64 numpy, with
finite-difference gradients to check the analytic ones."""
import math

import numpy as np


def unpack(p, n_in, nh, n_out):
    p = np.asarray(p, np.float64)
    o = 0
    out = []
    for shape in ((n_in, nh), (nh,), (nh, nh), (nh,), (nh, n_out), (n_out,)):
        n = int(np.prod(shape))
        out.append(p[o:o + n].reshape(shape))
        o += n
    return out


def forward(p, x, n_in, nh, n_out):
    w1, b1, w2, b2, w3, b3 = unpack(p, n_in, nh, n_out)
    h1 = np.tanh(x @ w1 + b1)
    h2 = np.tanh(h1 @ w2 + b2)
    return h2 @ w3 + b3, (h1, h2)


def loss(p, x, t, m, n_in, nh, n_out):
    y, _ = forward(p, x, n_in, nh, n_out)
    return float((m * (y - t) ** 2).sum() / max(m.sum(), 1.0))


def grad(p, x, t, m, n_in, nh, n_out):
    """Analytic gradient of the masked MSE, in the library's parameter
    order."""
    w1, b1, w2, b2, w3, b3 = unpack(p, n_in, nh, n_out)
    y, (h1, h2) = forward(p, x, n_in, nh, n_out)
    dy = 2.0 * m * (y - t) / max(m.sum(), 1.0)
    gw3, gb3 = h2.T @ dy, dy.sum(axis=0)
    d2 = (dy @ w3.T) * (1.0 - h2 ** 2)
    gw2, gb2 = h1.T @ d2, d2.sum(axis=0)
    d1 = (d2 @ w2.T) * (1.0 - h1 ** 2)
    gw1, gb1 = x.T @ d1, d1.sum(axis=0)
    return np.concatenate([a.ravel() for a in (gw1, gb1, gw2, gb2, gw3, gb3)])


def finite_difference(p, x, t, m, n_in, nh, n_out, idx, h=1e-6):
    out = []
    for i in idx:
        q = np.array(p, np.float64)
        q[i] += h
        lp = loss(q, x, t, m, n_in, nh, n_out)
        q[i] -= 2 * h
        lm = loss(q, x, t, m, n_in, nh, n_out)
        out.append((lp - lm) / (2 * h))
    return np.array(out)


def adam(p, g, mo, v, step, lr, b1=0.9, b2=0.999, eps=1e-8):
    mo = b1 * mo + (1 - b1) * g
    v = b2 * v + (1 - b2) * g * g
    c1, c2 = 1 - b1 ** step, 1 - b2 ** step
    return p - lr * (mo / c1) / (np.sqrt(v / c2) + eps), mo, v


def descriptors(real_vectors, pos, species, nspecies, cutoff, nrad, width):
    """The radial descriptors of include/imago_learned.h by brute force over
    lattice images."""
    rv = np.asarray(real_vectors, float)
    pos = np.asarray(pos, float)
    vol = abs(np.linalg.det(rv))
    rec = np.linalg.inv(rv).T
    diag = np.linalg.norm(rv.sum(axis=0))
    reps = [int(math.ceil((cutoff + diag) / (vol / (vol * np.linalg.norm(rec[i])))))
            for i in range(3)]
    mu = cutoff * np.arange(1, nrad + 1) / nrad
    out = np.zeros((len(pos), nrad + nspecies))
    for i in range(len(pos)):
        for a in range(-reps[0], reps[0] + 1):
            for b in range(-reps[1], reps[1] + 1):
                for c in range(-reps[2], reps[2] + 1):
                    R = a * rv[0] + b * rv[1] + c * rv[2]
                    d = pos + R - pos[i]
                    r = np.sqrt((d * d).sum(axis=1))
                    r = r[(r > 0) & (r < cutoff)]
                    fc = 0.5 * (np.cos(np.pi * r / cutoff) + 1.0)
                    out[i, :nrad] += (np.exp(-(r[:, None] - mu) ** 2 / (2 * width * width))
                                      * fc[:, None]).sum(axis=0)
        out[i, nrad + species[i]] = 1.0
    return out
