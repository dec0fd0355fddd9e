"""Initial states of the workloads this library is measured and checked on.

All generators return the five primitive fields (rho, vx, vy, vz, p) as
FP64 arrays of the ghosted shape (n+4 per axis), filled on every cell
(ghosts included, as the reference's init_* functions do, e.g.
src/rs/src/init.rs:401-444); only interior values matter because ghosts are
refilled by the boundary rules.  Cell centres of interior cell i are at
(i - 2 + 1/2) * ds from the lower domain edge.

Workloads
  kelvin_helmholtz   3D KH shear layer, periodic unit box (gamma 1.4)
  sod                3D Sod shock tube along x, outflow on all faces
  isentropic_vortex  Shu's isentropic vortex advected along (1, 1, 0),
                     periodic box [-5, 5]^3, strength 5
  riemann_random     random two-state Riemann problem split by a plane
The reference's own KH set-up shears in z and has no noise; these follow
the workload definitions instead (shear in y, seeded noise).
"""
from __future__ import annotations

import numpy as np

PERIODIC, OUTFLOW, WALL = 0, 1, 2

_MASK64 = (1 << 64) - 1


def splitmix64(x: np.ndarray) -> np.ndarray:
    """SplitMix64 finaliser on uint64 arrays (Steele, Lea & Flood 2014)."""
    x = (x + np.uint64(0x9E3779B97F4A7C15)) & np.uint64(_MASK64)
    x = (x ^ (x >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
    x = (x ^ (x >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return x ^ (x >> np.uint64(31))


def counter_uniform(seed: int, index: np.ndarray, comp: int) -> np.ndarray:
    """Uniform [0, 1) from (seed, cell index, component), counter-based."""
    with np.errstate(over="ignore"):
        key = np.uint64(seed & _MASK64) * np.uint64(0x9E3779B97F4A7C15) + index.astype(np.uint64) * np.uint64(3) \
            + np.uint64(comp)
        r = splitmix64(key)
    return (r >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def centres(n_int: int, ds: float, lo: float = 0.0) -> np.ndarray:
    """Cell-centre coordinates of all n_int + 4 ghosted cells along an axis."""
    return lo + (np.arange(n_int + 4, dtype=np.float64) - 2 + 0.5) * ds


def _splitmix64_t(x):
    """splitmix64 on int64 torch tensors holding uint64 bit patterns
    (multiplication wraps modulo 2^64 as on uint64; right shifts made
    logical by masking)."""
    import torch

    def srl(v, k):
        return (v >> k) & ((1 << (64 - k)) - 1)

    def c(u):  # uint64 constant as the int64 with the same bits
        return torch.tensor(u - (1 << 64) if u >= 1 << 63 else u, dtype=torch.int64, device=x.device)

    x = x + c(0x9E3779B97F4A7C15)
    x = (x ^ srl(x, 30)) * c(0xBF58476D1CE4E5B9)
    x = (x ^ srl(x, 27)) * c(0x94D049BB133111EB)
    return x ^ srl(x, 31)


def _counter_uniform_t(seed: int, index, comp: int):
    """counter_uniform on an int64 torch index tensor, bit for bit."""
    import torch
    s = seed & _MASK64
    k0 = (s * 0x9E3779B97F4A7C15) & _MASK64
    k0 = torch.tensor(k0 - (1 << 64) if k0 >= 1 << 63 else k0, dtype=torch.int64, device=index.device)
    r = _splitmix64_t(k0 + index * 3 + comp)
    return ((r >> 11) & ((1 << 53) - 1)).to(torch.float64) * (1.0 / 9007199254740992.0)


def _kh_noise_device(vels, seed, noise, shape, n, ny, nz, device):
    """The noise of kelvin_helmholtz added on a torch device (same bits as
    the NumPy path: integer hashing, then one multiply and adds per value)."""
    import torch
    dev = torch.device(device)
    ii = (torch.arange(shape[0], device=dev) - 2).remainder(n).view(-1, 1, 1)
    jj = (torch.arange(shape[1], device=dev) - 2).remainder(ny).view(1, -1, 1)
    kk = (torch.arange(shape[2], device=dev) - 2).remainder(nz).view(1, 1, -1)
    idx = ((ii * ny + jj) * nz + kk).to(torch.int64)
    out = []
    for comp, v in enumerate(vels):
        t = torch.from_numpy(v).to(dev)
        t += noise * (2.0 * _counter_uniform_t(seed, idx, comp) - 1.0)
        out.append(t.cpu().numpy())
    return out


def kelvin_helmholtz(n: int = 64, seed: int = 1, noise: float = 1e-3, ny: int | None = None,
                     nz: int | None = None, shear: float = 0.5, ratio: float = 2.0, p0: float = 2.5,
                     device: str | None = None):
    """KH layer: rho=ratio, vx=+shear for |y-0.5|<0.25, else rho=1,
    vx=-shear; p=p0; vy=0.01 sin(4 pi x)(exp(-(y-0.25)^2/0.005)+exp(-(y-0.75)^2/0.005));
    vz=0; plus uniform noise in [-noise, noise] on vx, vy, vz.  The defaults
    (shear 0.5, ratio 2, p 2.5) are the 64^3 periodic parity workload.
    `device` (a torch device) computes the noise there, with the same bits.
    Returns (prims, ds, bcs)."""
    ny = ny or n
    nz = nz or n
    ds = 1.0 / n
    x = centres(n, ds)[:, None, None]
    y = centres(ny, ds)[None, :, None]
    shape = (n + 4, ny + 4, nz + 4)
    inner = np.abs(y - 0.5) < 0.25
    rho = np.broadcast_to(np.where(inner, float(ratio), 1.0), shape).copy()
    vx = np.broadcast_to(np.where(inner, float(shear), -float(shear)), shape).copy()
    vy = np.broadcast_to(0.01 * np.sin(4 * np.pi * x) * (np.exp(-(y - 0.25) ** 2 / 0.005)
                                                          + np.exp(-(y - 0.75) ** 2 / 0.005)), shape).copy()
    vz = np.zeros(shape)
    p = np.full(shape, float(p0))
    if noise and device is not None:
        vx, vy, vz = _kh_noise_device((vx, vy, vz), seed, noise, shape, n, ny, nz, device)
    elif noise:
        # noise indexed by interior cell (i, j, k) -> (i*ny + j)*nz + k
        ii = np.arange(shape[0])[:, None, None] - 2
        jj = np.arange(shape[1])[None, :, None] - 2
        kk = np.arange(shape[2])[None, None, :] - 2
        idx = ((np.mod(ii, n) * ny + np.mod(jj, ny)) * nz + np.mod(kk, nz)).astype(np.int64)
        idx = np.broadcast_to(idx, shape)
        for comp, v in enumerate((vx, vy, vz)):
            v += noise * (2.0 * counter_uniform(seed, idx, comp) - 1.0)
    return [rho, vx, vy, vz, p], ds, (PERIODIC,) * 6


def fourier_modes(n: int, seed: int, modes: int = 8, amp: float = 0.1, kmax: int = 4, device: str | None = None):
    """Smooth periodic state on the unit cube: rho = 1, p = 1, v = 0 plus
    `modes` random Fourier modes sin(2 pi k.x + phase), integer wave vectors
    k in [-kmax, kmax]^3 (not 0), each with its own amplitude in
    [-amp, amp] on rho, p, vx, vy and vz.  `device` (a torch device) runs the
    3-D products and sums there (values within one FP64 unit in the last
    place of the NumPy path's).  Returns (prims, ds, bcs)."""
    rng = np.random.default_rng(seed)
    ds = 1.0 / n
    c = centres(n, ds)
    shape = (n + 4,) * 3
    if device is not None:
        return _fourier_device(rng, c, shape, modes, amp, kmax, device), ds, (PERIODIC,) * 6
    prim = [np.ones(shape), np.zeros(shape), np.zeros(shape), np.zeros(shape), np.ones(shape)]
    for _ in range(modes):
        k = np.zeros(3, dtype=np.int64)
        while not k.any():
            k = rng.integers(-kmax, kmax + 1, 3)
        phase = rng.uniform(0.0, 2.0 * np.pi)
        a = rng.uniform(-amp, amp, 5)
        # sin(2 pi k.x + phase) = Im(e^{i phase} e^{i 2 pi kx x} e^{i 2 pi ky y} e^{i 2 pi kz z})
        ex = np.exp(1j * (2 * np.pi * k[0] * c + phase))[:, None, None]
        ey = np.exp(1j * 2 * np.pi * k[1] * c)[None, :, None]
        ez = np.exp(1j * 2 * np.pi * k[2] * c)[None, None, :]
        s = np.imag((ex * ey) * ez)
        order = (0, 4, 1, 2, 3)          # amplitudes for rho, p, vx, vy, vz
        for f, j in zip(order, range(5)):
            prim[f] += a[j] * s
    return prim, ds, (PERIODIC,) * 6


def _fourier_device(rng, c, shape, modes, amp, kmax, device):
    """fourier_modes' fields on a torch device: the 1-D and 2-D factors in
    NumPy as there, the 3-D imaginary part as Re(exy) Im(ez) + Im(exy) Re(ez)
    and the sums on the device."""
    import torch
    dev = torch.device(device)
    prim = [torch.ones(shape, dtype=torch.float64, device=dev), torch.zeros(shape, dtype=torch.float64, device=dev),
            torch.zeros(shape, dtype=torch.float64, device=dev), torch.zeros(shape, dtype=torch.float64, device=dev),
            torch.ones(shape, dtype=torch.float64, device=dev)]
    for _ in range(modes):
        k = np.zeros(3, dtype=np.int64)
        while not k.any():
            k = rng.integers(-kmax, kmax + 1, 3)
        phase = rng.uniform(0.0, 2.0 * np.pi)
        a = rng.uniform(-amp, amp, 5)
        ex = np.exp(1j * (2 * np.pi * k[0] * c + phase))[:, None]
        ey = np.exp(1j * 2 * np.pi * k[1] * c)[None, :]
        ez = np.exp(1j * 2 * np.pi * k[2] * c)
        exy = ex * ey
        xr = torch.from_numpy(np.ascontiguousarray(exy.real)).to(dev)[:, :, None]
        xi = torch.from_numpy(np.ascontiguousarray(exy.imag)).to(dev)[:, :, None]
        zr = torch.from_numpy(np.ascontiguousarray(ez.real)).to(dev)[None, None, :]
        zi = torch.from_numpy(np.ascontiguousarray(ez.imag)).to(dev)[None, None, :]
        sn = xr * zi + xi * zr
        order = (0, 4, 1, 2, 3)
        for f, j in zip(order, range(5)):
            prim[f] += float(a[j]) * sn
    return [t.cpu().numpy() for t in prim]


def sod(n: int = 64, ny: int | None = None, nz: int | None = None):
    """rho=1, p=1 for x<0.5; rho=0.125, p=0.1 otherwise; v=0; outflow."""
    ny = ny or n
    nz = nz or n
    ds = 1.0 / n
    x = centres(n, ds)[:, None, None]
    shape = (n + 4, ny + 4, nz + 4)
    left = np.broadcast_to(x < 0.5, shape)
    rho = np.where(left, 1.0, 0.125)
    p = np.where(left, 1.0, 0.1)
    z = np.zeros(shape)
    return [rho, z.copy(), z.copy(), z.copy(), p], ds, (OUTFLOW,) * 6


def isentropic_vortex(n: int = 64, beta: float = 5.0, gamma: float = 1.4, ny: int | None = None,
                      nz: int | None = None, half_width: float = 5.0):
    """Shu's isentropic vortex (tube along z) on [-L, L]^3, background
    rho=1, p=1, v=(1, 1, 0), periodic."""
    ny = ny or n
    nz = nz or n
    ds = 2.0 * half_width / n
    x = centres(n, ds, -half_width)[:, None, None]
    y = centres(ny, ds, -half_width)[None, :, None]
    shape = (n + 4, ny + 4, nz + 4)
    r2 = x * x + y * y
    e = np.exp(0.5 * (1.0 - r2))
    du = -beta / (2 * np.pi) * e * y
    dv = beta / (2 * np.pi) * e * x
    T = 1.0 - (gamma - 1.0) * beta * beta / (8.0 * gamma * np.pi * np.pi) * e * e
    rho = np.broadcast_to(T ** (1.0 / (gamma - 1.0)), shape).copy()
    p = rho ** gamma
    vx = np.broadcast_to(1.0 + du, shape).copy()
    vy = np.broadcast_to(1.0 + dv, shape).copy()
    vz = np.zeros(shape)
    return [rho, vx, vy, vz, p], ds, (PERIODIC,) * 6


def riemann_random(shape, seed: int, bcs=(OUTFLOW,) * 6):
    """Two constant states split by a plane through a random point with a
    random unit normal; rho, p log-uniform in [0.1, 10], velocities uniform
    in [-1, 1].  ``shape`` is the interior shape; the box is [0, shape*ds]
    with ds = 1 / max(shape)."""
    rng = np.random.default_rng(seed)
    nx, ny, nz = shape
    ds = 1.0 / max(shape)
    states = []
    for _ in range(2):
        rho = float(np.exp(rng.uniform(np.log(0.1), np.log(10.0))))
        p = float(np.exp(rng.uniform(np.log(0.1), np.log(10.0))))
        v = rng.uniform(-1.0, 1.0, 3)
        states.append((rho, v, p))
    point = rng.uniform(0.25, 0.75, 3) * np.array(shape) * ds
    normal = rng.normal(size=3)
    normal /= np.linalg.norm(normal)
    x = centres(nx, ds)[:, None, None]
    y = centres(ny, ds)[None, :, None]
    z = centres(nz, ds)[None, None, :]
    side = ((x - point[0]) * normal[0] + (y - point[1]) * normal[1] + (z - point[2]) * normal[2]) < 0
    full = (nx + 4, ny + 4, nz + 4)
    side = np.broadcast_to(side, full)
    (r0, v0, p0), (r1, v1, p1) = states
    prim = [np.where(side, r0, r1), np.where(side, v0[0], v1[0]), np.where(side, v0[1], v1[1]),
            np.where(side, v0[2], v1[2]), np.where(side, p0, p1)]
    return prim, ds, tuple(bcs)


def conserved_from_primitives(prim, ds, gamma):
    """calc_conserved (src/rs/src/physics.rs:143-175) in NumPy, any dtype."""
    rho, vx, vy, vz, p = prim
    T = rho.dtype.type
    V = T(ds) * T(ds) * T(ds)
    gm1 = T(gamma) - T(1.0)
    return [rho * V, vx * rho * V, vy * rho * V, vz * rho * V,
            V * (rho * (vx * vx + vy * vy + vz * vz) / T(2.0) + p / gm1)]
