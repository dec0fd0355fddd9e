"""Learned coarse-grid correction: training pairs made by the solver, the
training loop, and corrected coarse solves (include/deepgreen_net.h).

Everything numerical runs in libdeepgreen.so: the Euler steps, coarsening,
the network's input and target crops, the tensor-core convolutions, Adam and
the corrector.  torch provides device buffers only.

Pairs (one per coarse step): a fine periodic grid F (2n cells per axis) and
a coarse grid C (n) that starts as the 2x2x2 sums of F.  F takes two steps
(dt1, dt2, its own CFL dts); C takes one plain step of dt1 + dt2.  The pair
is (C before, C after, truth = coarsened F after): the network learns
truth - C_after from (C_before, C_after), in flux form -- it predicts face
fluxes whose divergence is the correction, so the correction conserves the
totals exactly and vanishes for uniform states.
"""
from __future__ import annotations

import ctypes
import json
import math
import time
from dataclasses import dataclass, field

import numpy as np

from . import capi, setups
from .net import IO_CHANNELS, Net

INPUTS = 14
OUTPUTS = 15          # face fluxes: the correction is their divergence
GAMMA = 1.4
CFL = 0.4


class Norm(ctypes.Structure):
    _fields_ = [("in_mean", ctypes.c_float * 16), ("in_inv_std", ctypes.c_float * 16),
                ("out_std", ctypes.c_float * 16)]

    @classmethod
    def identity(cls):
        n = cls()
        for c in range(16):
            n.in_mean[c] = 0.0
            n.in_inv_std[c] = 1.0
            n.out_std[c] = 1.0
        return n

    def to_dict(self):
        return {k: list(getattr(self, k)) for k, _ in self._fields_}

    @classmethod
    def from_dict(cls, d):
        n = cls()
        for k, _ in cls._fields_:
            for i, v in enumerate(d[k]):
                getattr(n, k)[i] = float(v)
        return n


class Stats(ctypes.Structure):
    _fields_ = [("steps", ctypes.c_uint64), ("fallback_steps", ctypes.c_uint64), ("masked_cells", ctypes.c_uint64),
                ("cells", ctypes.c_uint64), ("max_drift", ctypes.c_double), ("last_drift", ctypes.c_double),
                ("violations", ctypes.c_uint64)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


def _lib():
    return capi.load()


def _check(rc, msg_fn):
    if rc != capi.DG_OK:
        raise capi.DgError(rc, msg_fn())


def grid(n: int, device: int = 0) -> capi.Context:
    """A periodic FP32 grid of n^3 cells on the unit cube (minmod, CFL 0.4, gamma 1.4)."""
    return capi.Context((n, n, n), 1.0 / n, (capi.PERIODIC,) * 6, gamma=GAMMA, cfl=CFL,
                        limiter=capi.LIMITER_MINMOD, precision=capi.F32, device=device)


def coarsen(fine: capi.Context, coarse: capi.Context):
    lib = _lib()
    _check(lib.dg_coarsen(fine.h, coarse.h), lambda: lib.dg_last_error(coarse.h).decode())


class PackPool:
    """Dense state packs on the device: slots x 5 x (n+4)^3 FP32."""

    def __init__(self, n: int, slots: int, device: int = 0):
        import torch
        self.n = n
        self.cells = (n + 4) ** 3
        self.data = torch.empty((slots, 5, self.cells), dtype=torch.float32, device=torch.device("cuda", device))

    def ptr(self, slot: int) -> int:
        return self.data[slot].data_ptr()

    def store(self, ctx: capi.Context, slot: int):
        base = self.ptr(slot)
        ctx.get_conserved_device([base + 4 * f * self.cells for f in range(5)])
        ctx.synchronize()   # the copy runs on the grid's stream; later users may be on others


def features(norm: Norm, before: int, after: int, n: int, origin, ext: int, out_ptr: int, stream=None):
    lib = _lib()
    ds = 1.0 / n
    _check(lib.dg_learned_features(ctypes.byref(norm), before, after, n, ds, GAMMA, int(origin[0]), int(origin[1]),
                                   int(origin[2]), ext, out_ptr, stream),
           lambda: lib.dg_last_error(None).decode())


def targets(norm: Norm, after: int, truth: int, n: int, origin, ext: int, out_ptr: int, stream=None):
    lib = _lib()
    ds = 1.0 / n
    _check(lib.dg_learned_targets(ctypes.byref(norm), after, truth, n, ds, int(origin[0]), int(origin[1]),
                                  int(origin[2]), ext, out_ptr, stream),
           lambda: lib.dg_last_error(None).decode())


class Corrector:
    """dg_corrector: plain step + learned correction on a coarse grid."""

    def __init__(self, ctx: capi.Context, net: Net, norm: Norm, tolerance: float | None = None):
        self.lib = _lib()
        self.ctx, self.net, self.norm = ctx, net, norm
        h = ctypes.c_void_p()
        _check(self.lib.dg_corrector_create(ctx.h, net.h, ctypes.byref(norm), ctypes.byref(h)),
               lambda: self.lib.dg_corrector_last_error(None).decode())
        self.h = h
        if tolerance is not None:
            _check(self.lib.dg_corrector_set_tolerance(self.h, float(tolerance)), self._err)

    def _err(self):
        return self.lib.dg_corrector_last_error(self.h).decode()

    def step(self, nsteps: int = 1):
        _check(self.lib.dg_corrector_step(self.h, int(nsteps)), self._err)

    def stats(self) -> dict:
        s = Stats()
        _check(self.lib.dg_corrector_stats(self.h, ctypes.byref(s)), self._err)
        return s.as_dict()

    def close(self):
        if getattr(self, "h", None):
            self.lib.dg_corrector_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------------------
# Initial states of the training and evaluation workloads
# ---------------------------------------------------------------------------
def _setup_device():
    """The GPU builds the large initial states (same values as the NumPy path)."""
    import torch
    return "cuda" if torch.cuda.is_available() else None


def initial_state(kind: str, n: int, seed: int, **kw):
    """'kh': KH layer with shear / ratio (kw, else drawn from seed: shear in
    [0.2, 0.8], density ratio in [1, 4]); 'fourier': 8 random modes."""
    if kind == "kh":
        rng = np.random.default_rng(seed)
        shear = kw.get("shear", rng.uniform(0.2, 0.8))
        ratio = kw.get("ratio", rng.uniform(1.0, 4.0))
        prim, _, _ = setups.kelvin_helmholtz(n, seed=seed, shear=shear, ratio=ratio, device=_setup_device())
        return prim, {"kind": "kh", "seed": seed, "shear": float(shear), "ratio": float(ratio)}
    if kind == "fourier":
        prim, _, _ = setups.fourier_modes(n, seed, device=_setup_device())
        return prim, {"kind": "fourier", "seed": seed}
    raise ValueError(kind)


def device_initial_conserved(kind: str, n: int, seed: int, device: int = 0, **kw):
    """initial_state's fields built on the GPU and returned as the five
    conserved totals (mass, momenta, energy; FP32 CUDA tensors of the ghosted
    shape) for dg_set_conserved_device: the large grids of the evaluation
    (1024^3: 43 GB of FP64 primitives) never pass through host memory.  The
    primitives are the same functions of the cell centres as initial_state's
    (KH noise by the same counter-based generator); they are converted to
    totals in FP64 (calc_conserved, physics.rs:143-175) and rounded once."""
    import torch
    dev = torch.device("cuda", device)
    f64 = torch.float64
    ds = 1.0 / n
    m = n + 4
    c = (torch.arange(m, dtype=f64, device=dev) - 2 + 0.5) * ds
    meta = {"kind": kind, "seed": seed}
    if kind == "kh":
        rng = np.random.default_rng(seed)
        shear = kw.get("shear", rng.uniform(0.2, 0.8))
        ratio = kw.get("ratio", rng.uniform(1.0, 4.0))
        meta.update(shear=float(shear), ratio=float(ratio))
        y = c.view(1, m, 1)
        inner = (torch.abs(y - 0.5) < 0.25).expand(m, m, m)
        rho = torch.where(inner, float(ratio), 1.0).to(f64)
        vel = [torch.where(inner, float(shear), -float(shear)).to(f64),
               (0.01 * torch.sin(4 * np.pi * c.view(m, 1, 1))
                * (torch.exp(-(y - 0.25) ** 2 / 0.005) + torch.exp(-(y - 0.75) ** 2 / 0.005))).expand(m, m, m)
               .contiguous(),
               torch.zeros((m, m, m), dtype=f64, device=dev)]
        # the noise of setups.kelvin_helmholtz, indexed by interior cell
        ii = (torch.arange(m, device=dev) - 2).remainder(n).view(-1, 1, 1)
        jj = (torch.arange(m, device=dev) - 2).remainder(n).view(1, -1, 1)
        kk = (torch.arange(m, device=dev) - 2).remainder(n).view(1, 1, -1)
        idx = ((ii * n + jj) * n + kk).to(torch.int64)
        for comp in range(3):
            vel[comp] = vel[comp] + 1e-3 * (2.0 * setups._counter_uniform_t(seed, idx, comp) - 1.0)
        del idx
        p = torch.full((m, m, m), 2.5, dtype=f64, device=dev)
    elif kind == "fourier":
        rng = np.random.default_rng(seed)
        rho = torch.ones((m, m, m), dtype=f64, device=dev)
        p = torch.ones((m, m, m), dtype=f64, device=dev)
        vel = [torch.zeros((m, m, m), dtype=f64, device=dev) for _ in range(3)]
        cn = c.cpu().numpy()
        for _ in range(8):
            k = np.zeros(3, dtype=np.int64)
            while not k.any():
                k = rng.integers(-4, 5, 3)
            phase = rng.uniform(0.0, 2.0 * np.pi)
            a = rng.uniform(-0.1, 0.1, 5)
            exy = np.exp(1j * (2 * np.pi * k[0] * cn + phase))[:, None] * np.exp(1j * 2 * np.pi * k[1] * cn)[None, :]
            ez = np.exp(1j * 2 * np.pi * k[2] * cn)
            xr = torch.from_numpy(np.ascontiguousarray(exy.real)).to(dev)[:, :, None]
            xi = torch.from_numpy(np.ascontiguousarray(exy.imag)).to(dev)[:, :, None]
            zr = torch.from_numpy(np.ascontiguousarray(ez.real)).to(dev)[None, None, :]
            zi = torch.from_numpy(np.ascontiguousarray(ez.imag)).to(dev)[None, None, :]
            sn = xr * zi + xi * zr
            rho += float(a[0]) * sn
            p += float(a[1]) * sn
            for comp in range(3):
                vel[comp] += float(a[2 + comp]) * sn
            del sn
    else:
        raise ValueError(kind)
    vol = ds ** 3
    cons = [(rho * vol).to(torch.float32)]
    ke = torch.zeros_like(rho)
    for v in vel:
        cons.append((rho * v * vol).to(torch.float32))
        ke += v * v
    cons.append((vol * (0.5 * rho * ke + p / (GAMMA - 1.0))).to(torch.float32))
    del rho, vel, p, ke
    out = [t.contiguous() for t in cons]
    # dg_set_conserved_device copies on the context's own (non-blocking)
    # stream: the fields must be complete before they are handed over
    torch.cuda.synchronize(dev)
    return out, meta


# ---------------------------------------------------------------------------
# Pairs
# ---------------------------------------------------------------------------
@dataclass
class PairSet:
    n: int                                   # coarse cells per axis
    before: PackPool
    after: PackPool
    truth: PackPool
    count: int = 0
    meta: list = field(default_factory=list)


def make_pairs(n_coarse: int, trajectories, pairs_per_trajectory: int, spacing: int, warmup_max: int, seed: int,
               device: int = 0, log=print) -> PairSet:
    """trajectories: list of (kind, seed).  Per trajectory: a fine grid
    (2 n_coarse) from that initial state, a random warm-up of 0..warmup_max
    fine steps, then pairs every `spacing` fine steps."""
    total = len(trajectories) * pairs_per_trajectory
    ps = PairSet(n_coarse, PackPool(n_coarse, total, device), PackPool(n_coarse, total, device),
                 PackPool(n_coarse, total, device))
    rng = np.random.default_rng(seed)
    fine = grid(2 * n_coarse, device)
    coarse = grid(n_coarse, device)
    for kind, s in trajectories:
        prim, meta = initial_state(kind, 2 * n_coarse, s)
        fine.set_primitives(prim)
        del prim
        w = int(rng.integers(0, warmup_max + 1))
        if w:
            fine.compute_step(w)
        t0 = time.time()
        for k in range(pairs_per_trajectory):
            slot = ps.count
            coarsen(fine, coarse)
            ps.before.store(coarse, slot)
            dts = fine.compute_step(2)
            coarse.compute_step_dt(float(dts[0] + dts[1]))
            ps.after.store(coarse, slot)
            coarsen(fine, coarse)
            ps.truth.store(coarse, slot)
            ps.count += 1
            ps.meta.append(dict(meta, fine_step=w + k * (spacing + 2)))
            if k + 1 < pairs_per_trajectory and spacing:
                fine.compute_step(spacing)
        log(f"pairs: {meta} warm-up {w}: {pairs_per_trajectory} pairs in {time.time() - t0:.2f}s")
    fine.close()
    coarse.close()
    return ps


# ---------------------------------------------------------------------------
# Training
# ---------------------------------------------------------------------------
class Batcher:
    """Random crops of the pair set into device batch buffers."""

    def __init__(self, ps: PairSet, batch: int, crop: int, seed: int, device: int = 0):
        import torch
        self.ps, self.batch, self.crop = ps, batch, crop
        self.ext = crop + 9        # network output crop + 1: the divergence needs the lower faces
        dev = torch.device("cuda", device)
        self.feat = torch.zeros((batch, self.ext, self.ext, self.ext, IO_CHANNELS), dtype=torch.bfloat16, device=dev)
        self.tgt = torch.zeros((batch, crop, crop, crop, IO_CHANNELS), dtype=torch.float32, device=dev)
        self.rng = np.random.default_rng(seed)

    def fill(self, norm: Norm, stream=None):
        n = self.ps.n
        fstride = self.ext ** 3 * IO_CHANNELS * 2
        tstride = self.crop ** 3 * IO_CHANNELS * 4
        for i in range(self.batch):
            slot = int(self.rng.integers(0, self.ps.count))
            o = self.rng.integers(0, n, 3)
            features(norm, self.ps.before.ptr(slot), self.ps.after.ptr(slot), n, o - 5, self.ext,
                     self.feat.data_ptr() + i * fstride, stream)
            targets(norm, self.ps.after.ptr(slot), self.ps.truth.ptr(slot), n, o, self.crop,
                    self.tgt.data_ptr() + i * tstride, stream)


# Input channels holding the three components of one vector (momentum, its
# change over the step, velocity) and the target channels of the momentum.
VECTOR_INPUTS = ((1, 2, 3), (6, 7, 8), (10, 11, 12))
VECTOR_TARGETS = ((1, 2, 3),)


def fit_norm(ps: PairSet, samples: int = 16, crop: int = 48, seed: int = 0) -> Norm:
    """Per-channel mean / std of the inputs and std of the targets over random
    crops of the pair set (host statistics of device-made crops).  The three
    components of a vector share one scale, the largest: a flow whose
    training states move along x only (a shear layer) still gets a sensible
    scale for the y and z components, which grow once it rolls up."""
    import torch
    ident = Norm.identity()
    b = Batcher(ps, samples, crop, seed)
    b.fill(ident)
    torch.cuda.synchronize()
    f = b.feat.float().reshape(-1, IO_CHANNELS).cpu().numpy().astype(np.float64)
    t = b.tgt.reshape(-1, IO_CHANNELS).cpu().numpy().astype(np.float64)
    in_sd = f.std(axis=0)
    out_sd = t.std(axis=0)
    for grp in VECTOR_INPUTS:
        in_sd[list(grp)] = in_sd[list(grp)].max()
    for grp in VECTOR_TARGETS:
        out_sd[list(grp)] = out_sd[list(grp)].max()
    norm = Norm.identity()
    for c in range(16):
        if c < INPUTS:
            norm.in_mean[c] = float(f[:, c].mean())
            norm.in_inv_std[c] = 1.0 / float(in_sd[c]) if in_sd[c] > 0 else 1.0
        else:
            norm.in_mean[c] = 0.0
            norm.in_inv_std[c] = 0.0
        norm.out_std[c] = float(out_sd[c]) if c < 5 and out_sd[c] > 0 else 1.0
    return norm


def train(net: Net, ps: PairSet, norm: Norm, steps: int, batch: int = 8, crop: int = 64, lr: float = 1e-3,
          lr_min: float = 1e-5, seed: int = 0, log_every: int = 100, log=print, balance: bool = True):
    """Adam on the MSE of the normalised correction, each crop weighted by the
    inverse power of its target when `balance` (so that crops of smooth flow,
    whose corrections are small, count as much as crops of shear layers);
    cosine learning-rate decay from lr to lr_min.  Returns the loss history."""
    b = Batcher(ps, batch, crop, seed)
    hist = []
    t0 = time.time()
    for it in range(steps):
        b.fill(norm)
        loss = net.forward_backward_flux(b.feat, b.tgt, balance)
        rate = lr_min + 0.5 * (lr - lr_min) * (1.0 + math.cos(math.pi * it / max(steps, 1)))
        net.adam_step(rate)
        hist.append(loss)
        if log_every and (it % log_every == 0 or it == steps - 1):
            log(f"train step {it}: loss {loss:.5f} lr {rate:.2e} ({time.time() - t0:.1f}s)")
    return hist


def save(path, net: Net, norm: Norm, extra=None):
    params = [(w.tolist(), b.tolist()) for w, b in net.params()]
    with open(path, "w") as fh:
        json.dump({"norm": norm.to_dict(), "params": params, "extra": extra or {}}, fh)


def load(path, device: int = 0):
    with open(path) as fh:
        d = json.load(fh)
    net = Net(INPUTS, OUTPUTS, device=device)
    net.set_params([(np.asarray(w, np.float32), np.asarray(b, np.float32)) for w, b in d["params"]])
    return net, Norm.from_dict(d["norm"]), d.get("extra", {})


# ---------------------------------------------------------------------------
# Corrected and plain solves to a given time
# ---------------------------------------------------------------------------
def solve_to_time(ctx: capi.Context, t_end: float, corrector: Corrector | None = None, max_steps: int = 100000,
                  batch: int = 16, growth: float = 1.1):
    """Advance ctx from time 0 to t_end: CFL steps (plain, or corrected when a
    corrector is given) while they stay short of t_end, then one plain step
    of the remaining time.  Far from t_end the steps go to the device in
    batches of up to `batch` without a host round trip: a batch of m steps
    is enqueued only if m steps whose dt grew by `growth` each step would
    still end short of t_end, and the dts the steps used are read back after
    it.  Near t_end every step reads its dt first.  Returns (steps, seconds)."""
    import torch
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    t = 0.0
    steps = 0
    while steps < max_steps:
        dt = ctx.next_dt()
        if t + dt >= t_end:
            if t_end > t:
                ctx.compute_step_dt(t_end - t)
                steps += 1
            break
        m, reach, d = 0, 0.0, dt
        while m < min(batch, max_steps - steps) and t + reach + d < t_end:
            reach += d
            d *= growth
            m += 1
        m = max(m, 1)
        if corrector is not None:
            corrector.step(m)
        else:
            ctx.enqueue_steps(m)
        t += float(np.sum(ctx.get_dts(m))) if m > 1 else dt
        steps += m
    ctx.synchronize()
    return steps, time.perf_counter() - t0
