"""Python mirror of the seeded synthetic generators (csrc/synth.cpp).

The benchmark configurations are generated matrices; this module restates
the generator definitions independently (SplitMix64 counter RNG, stencil
assembly, random SPD assembly, the filtered lognormal field) so that the
tests pin the C++ generators to their written definition bit for bit.
Pure Python: meant for small sizes.
"""
from __future__ import annotations

import math

import numpy as np

M64 = (1 << 64) - 1
GAMMA = 0x9E3779B97F4A7C15
S_XSTAR, S_ROWSCALE, S_SIZE, S_ROWLEN, S_COL, S_VAL, S_FIELD = 1, 2, 3, 4, 5, 6, 7


def mix64(z: int) -> int:
    z &= M64
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M64
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M64
    return z ^ (z >> 31)


def stream_key(seed: int, stream: int) -> int:
    return mix64(((seed * GAMMA) & M64) ^ mix64(stream + GAMMA))


def u01(key: int, i: int) -> float:
    return (mix64(key + (i + 1) * GAMMA) >> 11) * 2.0 ** -53


def normal01(key: int, m: int) -> float:
    a, b = u01(key, 2 * m), u01(key, 2 * m + 1)
    return math.sqrt(-2.0 * math.log(1.0 - a)) * math.cos(6.283185307179586 * b)


def xstar(seed: int, n: int) -> np.ndarray:
    k = stream_key(seed, S_XSTAR)
    return np.array([-1.0 + 2.0 * u01(k, i) for i in range(n)])


def _csr(rows):
    rp, ci, v = [0], [], []
    for r in rows:
        for c, x in r:
            ci.append(c)
            v.append(x)
        rp.append(len(ci))
    return np.array(rp, np.int32), np.array(ci, np.int32), np.array(v, np.float64)


def laplace2d(nx: int, ny: int):
    rows = []
    for i in range(nx * ny):
        x, y = i % nx, i // nx
        r = []
        if y > 0:
            r.append((i - nx, -1.0))
        if x > 0:
            r.append((i - 1, -1.0))
        r.append((i, 4.0))
        if x < nx - 1:
            r.append((i + 1, -1.0))
        if y < ny - 1:
            r.append((i + nx, -1.0))
        rows.append(r)
    return _csr(rows)


def _stencil3d(g, off, diag):
    st = (g * g, g, 1)
    rows = []
    for i in range(g ** 3):
        co = (i // (g * g), (i // g) % g, i % g)  # z, y, x
        r, offsum = [], 0.0
        for d in range(3):
            if co[d] > 0:
                a = off(i, i - st[d], d, 0)
                r.append((i - st[d], a))
                offsum += abs(a)
        dpos = len(r)
        r.append((i, 0.0))
        for d in (2, 1, 0):
            if co[d] < g - 1:
                a = off(i, i + st[d], d, 1)
                r.append((i + st[d], a))
                offsum += abs(a)
        r[dpos] = (i, diag(i, offsum, co))
        rows.append(r)
    return _csr(rows)


def poisson3d_scaled(g: int, seed: int):
    k = stream_key(seed, S_ROWSCALE)
    f = [math.pow(10.0, -3.0 + 3.0 * u01(k, i)) for i in range(g ** 3)]
    return _stencil3d(g, lambda i, j, d, up: -(f[i] + f[j]) * 0.5, lambda i, s, co: s + 1e-3)


def convdiff3d(g: int, peclet=10.0, v=(1.0, 0.5, 0.25)):
    vx, vy, vz = v
    gam = 2.0 * peclet / max(v) if max(v) > 0 else 0.0
    vel = (vz, vy, vx)
    return _stencil3d(g, lambda i, j, d, up: -1.0 if up else -(1.0 + gam * vel[d]),
                      lambda i, s, co: 6.0 + gam * (vx + vy + vz))


def random_spd_size(seed: int) -> int:
    u = u01(stream_key(seed, S_SIZE), 0)
    x = math.exp(math.log(1000.0) + u * (math.log(64000.0) - math.log(1000.0)))
    return int(math.floor(x + 0.5))  # llround for positive values


def random_spd(seed: int, n: int = 0):
    if n <= 0:
        n = random_spd_size(seed)
    kl, ks, kc, kv = (stream_key(seed, s) for s in (S_ROWLEN, S_ROWSCALE, S_COL, S_VAL))
    tr = []
    for i in range(n):
        k = 8 + int(math.floor(25.0 * u01(kl, i)))
        sc = math.pow(10.0, -4.0 + 8.0 * u01(ks, i))
        for e in range(k):
            j = int(math.floor(u01(kc, i * 32 + e) * n))
            j = min(j, n - 1)
            if j == i:
                continue
            a = normal01(kv, i * 32 + e) * sc * 0.5
            tr.append((i * n + j, len(tr), a))
            tr.append((j * n + i, len(tr), a))
    tr.sort(key=lambda t: (t[0], t[1]))
    keys, vals = [], []
    for key, _, a in tr:
        if keys and keys[-1] == key:
            vals[-1] += a
        else:
            keys.append(key)
            vals.append(a)
    rowabs = [0.0] * n
    for key, a in zip(keys, vals):
        rowabs[key // n] += abs(a)
    rows, q = [], 0
    for i in range(n):
        r, diag_done = [], False
        while q < len(keys) and keys[q] // n == i:
            j = keys[q] % n
            if not diag_done and j > i:
                r.append((i, rowabs[i] + 1.0))
                diag_done = True
            r.append((j, vals[q]))
            q += 1
        if not diag_done:
            r.append((i, rowabs[i] + 1.0))
        rows.append(r)
    return _csr(rows)


def aniso3d(g: int, seed: int, log_sigma=2.0, corr_len=8.0, aniso=100.0):
    n = g ** 3
    kf = stream_key(seed, S_FIELD)
    w = [normal01(kf, i) for i in range(n)]
    t = [0.0] * n
    R = int(math.ceil(3.0 * corr_len))
    h = [math.exp(-float(d) * d / (corr_len * corr_len)) for d in range(-R, R + 1)]
    h2 = 0.0
    for x in h:
        h2 += x * x
    idx = lambda x, y, z: x + g * (y + g * z)
    for p in range(3):
        src, dst = (t, w) if p == 1 else (w, t)
        for z in range(g):
            for y in range(g):
                for x in range(g):
                    s = 0.0
                    for d in range(-R, R + 1):
                        if p == 0:
                            j = idx((x + d) % g, y, z)
                        elif p == 1:
                            j = idx(x, (y + d) % g, z)
                        else:
                            j = idx(x, y, (z + d) % g)
                        s += h[d + R] * src[j]
                    dst[idx(x, y, z)] = s
    norm = math.pow(h2, 1.5)
    kc = [math.exp(log_sigma * t[i] / norm) for i in range(n)]
    an = (aniso, 1.0, 1.0)

    def diag(i, offsum, co):
        bnd = 0.0
        for d in range(3):
            if co[d] == 0:
                bnd += an[d] * kc[i]
            if co[d] == g - 1:
                bnd += an[d] * kc[i]
        return offsum + bnd

    return _stencil3d(g, lambda i, j, d, up: -an[d] * 2.0 * kc[i] * kc[j] / (kc[i] + kc[j]), diag)
