"""Seeded synthetic initial conditions of the benchmark problems (host-side numpy).

The reference builds its initial conditions with Matlab initializers
(experiment/RiemannProblem/RiemannProblemInitializer.m, experiment/KelvinHelmholtzInitializer.m);
no datasets are involved.  These generators produce the same physical set-ups with a fixed-seed
counter-based generator (numpy Philox), so the CPU oracle and the GPU library start from
bit-identical states.

All arrays are returned in the library's layout: (5, slab) float64 = [rho, E, px, py, pz],
x fastest, slab = numel rounded up to a multiple of 32.
"""
import numpy as np


def slab_pitch(nx, ny, nz):
    n = nx * ny * nz
    return ((n + 31) // 32) * 32


def pack(shape, rho, E, px, py, pz):
    nx, ny, nz = shape
    n = nx * ny * nz
    q = np.zeros((5, slab_pitch(nx, ny, nz)))
    for k, a in enumerate((rho, E, px, py, pz)):
        q[k, :n] = np.broadcast_to(np.asarray(a, dtype=np.float64), (nz, ny, nx)).reshape(-1)
    return q


def sod(n=1024, gamma=1.4, x0=0.5, left=(1.0, 0.0, 1.0), right=(0.125, 0.0, 0.1)):
    """1-D Sod shock tube on [0,1]: (rho, u, P) left | right of x0."""
    x = (np.arange(n) + 0.5) / n
    L = x < x0
    rho = np.where(L, left[0], right[0])
    u = np.where(L, left[1], right[1])
    P = np.where(L, left[2], right[2])
    E = P / (gamma - 1) + 0.5 * rho * u * u
    return pack((n, 1, 1), rho, E, rho * u, 0.0, 0.0)


def kelvin_helmholtz(shape, gamma=5.0 / 3.0, P0=2.5, amp=1e-2, seed=12345):
    """Periodic unit-cube shear layer: rho=2, vx=+0.5 for |y-1/2| < 1/4, else rho=1, vx=-0.5;
    P uniform; vx, vy, vz get i.i.d. U(-amp, amp) perturbations from a seeded Philox stream."""
    nx, ny, nz = shape
    y = (np.arange(ny) + 0.5) / ny
    band = (np.abs(y - 0.5) < 0.25)[None, :, None]
    rho = np.where(band, 2.0, 1.0) * np.ones((nz, ny, nx))
    vx = np.where(band, 0.5, -0.5) * np.ones((nz, ny, nx))
    rng = np.random.Generator(np.random.Philox(seed))
    vx = vx + rng.uniform(-amp, amp, size=(nz, ny, nx))
    vy = rng.uniform(-amp, amp, size=(nz, ny, nx))
    vz = rng.uniform(-amp, amp, size=(nz, ny, nx)) if nz > 1 else np.zeros((nz, ny, nx))
    E = P0 / (gamma - 1) + 0.5 * rho * (vx * vx + vy * vy + vz * vz)
    return pack(shape, rho, E, rho * vx, rho * vy, rho * vz)


def random_smooth(shape, gamma=1.4, seed=7, amp=0.2):
    """Smooth random positive state (sum of a few random Fourier modes) for parity tests."""
    nx, ny, nz = shape
    rng = np.random.Generator(np.random.Philox(seed))
    zz, yy, xx = np.meshgrid(np.arange(nz) / nz, np.arange(ny) / ny, np.arange(nx) / nx, indexing="ij")

    def field(base, a):
        f = np.full((nz, ny, nx), base)
        for _ in range(4):
            kx, ky, kz = rng.integers(0, 3, size=3)
            ph = rng.uniform(0, 2 * np.pi)
            f = f + a * rng.uniform(-1, 1) * np.cos(2 * np.pi * (kx * xx + ky * yy + kz * zz) + ph)
        return f

    rho = field(1.0, amp * 0.5)
    P = field(1.0, amp * 0.5)
    vx, vy, vz = field(0.0, amp), field(0.0, amp), field(0.0, amp)
    E = P / (gamma - 1) + 0.5 * rho * (vx * vx + vy * vy + vz * vz)
    return pack(shape, rho, E, rho * vx, rho * vy, rho * vz)


def random_jumpy(shape, gamma=1.4, seed=11):
    """Piecewise-constant random blocks with strong jumps (exercises all HLLC wave modes and the
    limiters' zero branches)."""
    nx, ny, nz = shape
    rng = np.random.Generator(np.random.Philox(seed))
    def blocks(lo, hi):
        b = rng.uniform(lo, hi, size=(max(1, nz // 2 + 1), max(1, ny // 2 + 1), max(1, nx // 3 + 1)))
        iz = (np.arange(nz) * b.shape[0]) // nz
        iy = (np.arange(ny) * b.shape[1]) // ny
        ix = (np.arange(nx) * b.shape[2]) // nx
        return b[np.ix_(iz, iy, ix)]
    rho = blocks(0.2, 3.0)
    P = blocks(0.1, 5.0)
    vx, vy, vz = blocks(-1.5, 1.5), blocks(-1.0, 1.0), blocks(-1.0, 1.0)
    E = P / (gamma - 1) + 0.5 * rho * (vx * vx + vy * vy + vz * vz)
    return pack(shape, rho, E, rho * vx, rho * vy, rho * vz)


def rotating_annulus(shape, r_inner=1.0, dr=0.05, gamma=1.4, seed=31, amp=0.05):
    """Cylindrical test state (x = r, y = theta, z = z): a rotating annulus with v_theta = r^-1/2,
    a radial pressure gradient and seeded smooth perturbations of every field, for the cylindrical
    parity tests.  The radial cell i has its centre at r_inner + i dr."""
    nx, ny, nz = shape
    rng = np.random.Generator(np.random.Philox(seed))
    r = (r_inner + dr * np.arange(nx))[None, None, :]
    th = (np.arange(ny) / ny)[None, :, None]
    z = (np.arange(nz) / nz)[:, None, None]

    def noise():
        f = np.zeros((nz, ny, nx))
        for _ in range(3):
            k, m, l = rng.integers(1, 4), rng.integers(0, 3), rng.integers(0, 2)
            ph = rng.uniform(0, 2 * np.pi)
            f = f + rng.uniform(-1, 1) * np.cos(2 * np.pi * (k * (r - r_inner) / (dr * nx) + m * th + l * z) + ph)
        return f

    rho = (1.0 + 0.5 * (r - r_inner)) * (1.0 + amp * noise())
    P = 1.0 / r * (1.0 + amp * noise())
    vr = amp * noise()
    vth = r ** -0.5 * (1.0 + amp * noise())
    vz = amp * noise()
    E = P / (gamma - 1) + 0.5 * rho * (vr * vr + vth * vth + vz * vz)
    return pack(shape, rho, E, rho * vr, rho * vth, rho * vz)
