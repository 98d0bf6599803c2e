"""Seeded synthetic initial conditions for the benchmark and parity workloads.

No public dataset is involved: every input is an analytic field plus uniform
noise drawn from a SplitMix64 stream (seed = workload index), in i-j-k order.
Fields are returned as primitive variables [rho, p, u, v, w] in the reference
host layout (halo'd AoS, src/containers/array_4d.hpp:64-71) with zero halos,
as testcases::* leave them (src/testcases.cpp writes the interior only).
"""
import math

import numpy as np

from .abi import NS_NGC, halo_shape

_GOLDEN = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)


def splitmix64_uniform(seed, n, start=0):
    """n uniforms in [0,1) from SplitMix64 (Steele, Lea, Flood 2014), stream position start."""
    with np.errstate(over="ignore"):
        idx = np.arange(start + 1, start + n + 1, dtype=np.uint64)
        z = np.uint64(seed) + idx * _GOLDEN
        z = (z ^ (z >> np.uint64(30))) * _M1
        z = (z ^ (z >> np.uint64(27))) * _M2
        z = z ^ (z >> np.uint64(31))
    return (z >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def _noise_slabs(seed, nx, ny, nz, ncomp, slab=16):
    """Uniform [-1,1) draws, ncomp per cell in i-j-k order, one i-slab at a time
    (the same stream as splitmix64_uniform(seed, nx*ny*nz*ncomp), bounded memory)."""
    per = ny * nz * ncomp
    for i0 in range(0, nx, slab):
        i1 = min(nx, i0 + slab)
        r = splitmix64_uniform(seed, (i1 - i0) * per, start=i0 * per)
        yield i0, i1, r.reshape(i1 - i0, ny, nz, ncomp) * 2.0 - 1.0


def cell_centres(n, L):
    """Cell-centred coordinates x = dx/2 + i dx (src/grid.cpp:48)."""
    d = L / n
    return d * 0.5 + np.arange(n) * d


def _empty(p):
    return np.zeros(halo_shape(p), dtype=np.float64)


def _interior(W):
    g = NS_NGC
    return W[g:-g, g:-g, g:-g, :]


def random_field(p, seed, smooth=True, amp=0.05):
    """Positive-density, positive-pressure random field for operator parity tests.

    smooth=True adds a few Fourier modes; smooth=False adds a density/pressure jump
    along every axis so the WENO weights leave the linear regime.
    """
    W = _empty(p)
    nx, ny, nz = p.nx, p.ny, p.nz
    x = cell_centres(nx, 1.0)[:, None, None]
    y = cell_centres(ny, 1.0)[None, :, None]
    z = cell_centres(nz, 1.0)[None, None, :]
    r = splitmix64_uniform(seed, nx * ny * nz * 5).reshape(nx, ny, nz, 5) * 2.0 - 1.0
    base = (np.sin(2 * math.pi * x) * np.cos(2 * math.pi * y) * np.sin(2 * math.pi * z + 0.3))
    I = _interior(W)
    I[..., 0] = 1.0 + 0.2 * base + amp * r[..., 0]
    I[..., 1] = 1.5 + 0.3 * np.cos(2 * math.pi * (x + y + z)) + amp * r[..., 1]
    I[..., 2] = 0.4 * np.sin(2 * math.pi * y) + amp * r[..., 2]
    I[..., 3] = -0.3 * np.cos(2 * math.pi * z) + amp * r[..., 3]
    I[..., 4] = 0.2 * np.sin(2 * math.pi * x) + amp * r[..., 4]
    if not smooth:
        jump = ((x > 0.5) ^ (y > 0.4) ^ (z > 0.6)).astype(np.float64)
        I[..., 0] += 0.8 * jump
        I[..., 1] += 1.2 * jump
    return W


def shear_layer(p, seed=1, mach=0.5, noise=1e-3):
    """Double temporal shear layer on [0,2pi]^3 (periodic).

    rho = 1, p = 1/(gamma M^2), u = tanh((y-pi/2)/d) - tanh((y-3pi/2)/d) - 1 with
    d = 0.05*2pi, v = 0.05 sin(x) sum_l exp(-(y-y_l)^2/d^2) + noise, w = noise.
    """
    W = _empty(p)
    nx, ny, nz = p.nx, p.ny, p.nz
    x = cell_centres(nx, p.Lx)[:, None, None]
    y = cell_centres(ny, p.Ly)[None, :, None]
    d = 0.05 * 2.0 * math.pi
    y1, y2 = 0.5 * math.pi, 1.5 * math.pi
    r = splitmix64_uniform(seed, nx * ny * nz * 2).reshape(nx, ny, nz, 2) * 2.0 - 1.0
    I = _interior(W)
    I[..., 0] = 1.0
    I[..., 1] = 1.0 / (p.gamma * mach * mach)
    I[..., 2] = np.broadcast_to(np.tanh((y - y1) / d) - np.tanh((y - y2) / d) - 1.0, (nx, ny, nz))
    g = np.exp(-((y - y1) ** 2) / d ** 2) + np.exp(-((y - y2) ** 2) / d ** 2)
    I[..., 3] = 0.05 * np.sin(x) * g + noise * r[..., 0]
    I[..., 4] = noise * r[..., 1]
    return W


def sod(p, seed=3, amp=0.01):
    """3D Sod problem along x with interface x = 0.5 + amp sin(2pi y) sin(2pi z)."""
    W = _empty(p)
    nx, ny, nz = p.nx, p.ny, p.nz
    x = cell_centres(nx, p.Lx)[:, None, None]
    y = cell_centres(ny, p.Ly)[None, :, None]
    z = cell_centres(nz, p.Lz)[None, None, :]
    left = x < 0.5 + amp * np.sin(2 * math.pi * y) * np.sin(2 * math.pi * z)
    I = _interior(W)
    I[..., 0] = np.where(left, 1.0, 0.125)
    I[..., 1] = np.where(left, 1.0, 0.1)
    I[..., 2:] = 0.0
    return W


def taylor_green(p, seed=5, mach=0.1, noise=1e-4):
    """Compressible Taylor-Green vortex on [0,2pi]^3 with seeded velocity noise.

    rho = 1, p = 1/(gamma M^2) + (cos 2x + cos 2y)(cos 2z + 2)/16,
    u = sin x cos y cos z, v = -cos x sin y cos z, w = 0, plus uniform noise of
    amplitude `noise` on u, v, w (three draws per cell in i-j-k order).
    Generated one i-slab at a time, so 512^3 needs little more than the array."""
    W = _empty(p)
    nx, ny, nz = p.nx, p.ny, p.nz
    x = cell_centres(nx, p.Lx)
    y = cell_centres(ny, p.Ly)[None, :, None]
    z = cell_centres(nz, p.Lz)[None, None, :]
    I = _interior(W)
    p0 = 1.0 / (p.gamma * mach * mach)
    cy, sy, c2y = np.cos(y), np.sin(y), np.cos(2 * y)
    cz, c2z = np.cos(z), np.cos(2 * z)
    for i0, i1, r in _noise_slabs(seed, nx, ny, nz, 3):
        xs = x[i0:i1, None, None]
        S = I[i0:i1]
        S[..., 0] = 1.0
        S[..., 1] = p0 + (np.cos(2 * xs) + c2y) * (c2z + 2.0) / 16.0
        S[..., 2] = np.sin(xs) * cy * cz + noise * r[..., 0]
        S[..., 3] = -np.cos(xs) * sy * cz + noise * r[..., 1]
        S[..., 4] = noise * r[..., 2]
    return W
