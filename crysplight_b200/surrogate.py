"""Learned light-response surrogate: an MLP from an emission point (x, y, z) to
the 64 per-SiPM detection probabilities and the 64 (mean, log sigma) pairs of
the detected photons' arrival times, trained on the GPU by the library's own
tcgen05 kernels (``csrc/cl_mlp.cu``: BF16 weights and activations, FP32
accumulation, Adam on FP32 master weights).

The reference has no surrogate; this is new in this framework.  The training
data is generated by the CUDA Monte Carlo itself (``scan_dataset``).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

from . import _lib
from .params import Box, Readout, TimeBinning

D_IN, D_H, D_OUT = 3, 256, 192
N_CELLS = 64


def _declare(lib):
    if getattr(lib, "_mlp_declared", False):
        return
    P = C.c_void_p
    lib.cl_mlp_param_count.restype = C.c_int
    lib.cl_mlp_create.argtypes = [C.POINTER(C.c_void_p), C.c_int, C.c_int]
    lib.cl_mlp_create.restype = C.c_int
    lib.cl_mlp_destroy.argtypes = [P]
    lib.cl_mlp_destroy.restype = None
    lib.cl_mlp_last_error.argtypes = [P]
    lib.cl_mlp_last_error.restype = C.c_char_p
    lib.cl_mlp_set_max_ctas.argtypes = [P, C.c_int]
    lib.cl_mlp_set_max_ctas.restype = C.c_int
    lib.cl_mlp_set_params.argtypes = [P, P]
    lib.cl_mlp_get_params.argtypes = [P, P]
    lib.cl_mlp_set_data.argtypes = [P, P, P, C.c_int64]
    lib.cl_mlp_train.argtypes = [P, C.c_int, C.c_int, C.c_float, C.c_uint32, C.c_uint32,
                                 C.POINTER(C.c_float)]
    lib.cl_mlp_forward.argtypes = [P, P, P, C.c_int64]
    lib.cl_mlp_gradient.argtypes = [P, P, P, C.c_int, P, C.POINTER(C.c_float)]
    for n in ("cl_mlp_set_params", "cl_mlp_get_params", "cl_mlp_set_data", "cl_mlp_train",
              "cl_mlp_forward", "cl_mlp_gradient"):
        getattr(lib, n).restype = C.c_int
    lib._mlp_declared = True


def init_params(seed: int) -> np.ndarray:
    """U(-1/sqrt(fan_in), 1/sqrt(fan_in)) for weights and biases (the usual
    linear-layer initialisation), in the cl_mlp parameter layout."""
    rng = np.random.default_rng(seed)
    parts = []
    for fan_out, fan_in in ((D_H, D_IN), (D_H, D_H), (D_H, D_H), (D_OUT, D_H)):
        b = 1.0 / np.sqrt(fan_in)
        parts.append(rng.uniform(-b, b, size=fan_out * fan_in))
        parts.append(rng.uniform(-b, b, size=fan_out))
    return np.concatenate(parts).astype(np.float32)


class MLP:
    """One network on one GPU (not re-entrant)."""

    def __init__(self, device: int = 0, max_batch: int = 65536, seed: int = 0):
        self.lib = _lib.load()
        _declare(self.lib)
        h = C.c_void_p()
        rc = self.lib.cl_mlp_create(C.byref(h), int(device), int(max_batch))
        if rc != 0:
            raise _lib.CudaTransportError(rc, "cl_mlp_create failed")
        self.h = h
        self.device = device
        self.max_batch = max_batch
        self.n_params = int(self.lib.cl_mlp_param_count())
        self.step = 0
        self.set_params(init_params(seed))

    def close(self):
        if getattr(self, "h", None):
            self.lib.cl_mlp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc):
        if rc != 0:
            raise _lib.CudaTransportError(rc, self.lib.cl_mlp_last_error(self.h).decode())

    def set_max_ctas(self, n: int):
        self._check(self.lib.cl_mlp_set_max_ctas(self.h, int(n)))

    def set_params(self, p: np.ndarray):
        p = np.ascontiguousarray(p, np.float32)
        assert p.size == self.n_params
        self._check(self.lib.cl_mlp_set_params(self.h, C.c_void_p(p.ctypes.data)))

    def get_params(self) -> np.ndarray:
        p = np.empty(self.n_params, np.float32)
        self._check(self.lib.cl_mlp_get_params(self.h, C.c_void_p(p.ctypes.data)))
        return p

    def set_data(self, x, t):
        """x [n][3], t [n][192]: float32 CUDA tensors kept referenced here."""
        self._data = (x.contiguous(), t.contiguous())
        self._check(self.lib.cl_mlp_set_data(self.h, C.c_void_p(self._data[0].data_ptr()),
                                             C.c_void_p(self._data[1].data_ptr()), x.shape[0]))

    def train(self, steps: int, batch: int = 65536, lr: float = 1e-3, seed: int = 0) -> float:
        loss = C.c_float()
        self._check(self.lib.cl_mlp_train(self.h, int(steps), int(batch), float(lr), int(seed) & 0xFFFFFFFF,
                                          self.step & 0xFFFFFFFF, C.byref(loss)))
        self.step += steps
        return float(loss.value)

    def forward(self, x):
        import torch
        x = x.contiguous()
        out = torch.empty((x.shape[0], D_OUT), dtype=torch.float32, device=x.device)
        self._check(self.lib.cl_mlp_forward(self.h, C.c_void_p(x.data_ptr()), C.c_void_p(out.data_ptr()),
                                            x.shape[0]))
        return out

    def forward_into(self, x, out) -> None:
        """out[n][192] (float32 CUDA tensor, contiguous) = network(x[n][3])."""
        self._check(self.lib.cl_mlp_forward(self.h, C.c_void_p(x.data_ptr()), C.c_void_p(out.data_ptr()),
                                            x.shape[0]))

    def gradient(self, x, t):
        g = np.empty(self.n_params, np.float32)
        loss = C.c_float()
        self._check(self.lib.cl_mlp_gradient(self.h, C.c_void_p(x.data_ptr()), C.c_void_p(t.data_ptr()),
                                             x.shape[0], C.c_void_p(g.ctypes.data), C.byref(loss)))
        return float(loss.value), g


# ---------------------------------------------------------------------------
# Training data: a point scan through the CUDA Monte Carlo
# ---------------------------------------------------------------------------
def depth_warp(t, a: float):
    """Warped depth w(t) = (1 - a) t + a (1 - sqrt(1 - t)) of t = z / Lz in
    [0, 1] (the readout face at t = 1): monotonic, w(0) = 0, w(1) = 1, and
    with a > 0 stretched near the readout face, where the light of a point
    concentrates under one SiPM.  a = 0 is the identity."""
    t = np.clip(np.asarray(t, np.float64), 0.0, 1.0)
    return (1.0 - a) * t + a * (1.0 - np.sqrt(1.0 - t))


def depth_unwarp(w, a: float):
    """The t with depth_warp(t, a) = w (bisection; w in [0, 1])."""
    w = np.asarray(w, np.float64)
    lo, hi = np.zeros_like(w), np.ones_like(w)
    for _ in range(60):
        mid = 0.5 * (lo + hi)
        below = depth_warp(mid, a) < w
        lo = np.where(below, mid, lo)
        hi = np.where(below, hi, mid)
    return 0.5 * (lo + hi)


def grid_points(box: Box, shape=(48, 48, 24), z_warp: float = 0.0, z_range=None) -> np.ndarray:
    """Cell centres of a regular nx x ny x nz grid over the crystal, (P, 3)
    float32 in mm, x fastest; with ``z_warp`` the z levels are the cell
    centres of a regular grid in the warped depth (denser towards the readout
    face); ``z_range`` = (z0, z1) mm restricts the grid to that slab."""
    nx, ny, nz = shape
    L = [float(box.L[i]) for i in range(3)]
    z0, z1 = (0.0, L[2]) if z_range is None else (float(z_range[0]), float(z_range[1]))
    ax = [(np.arange(n, dtype=np.float64) + 0.5) * (L[i] / n) for i, n in enumerate((nx, ny))]
    ax.append(z0 + (np.arange(nz, dtype=np.float64) + 0.5) * ((z1 - z0) / nz))
    if z_warp:
        ax[2] = z0 + depth_unwarp((np.arange(nz, dtype=np.float64) + 0.5) / nz, z_warp) * (z1 - z0)
    z, y, x = np.meshgrid(ax[2], ax[1], ax[0], indexing="ij")
    return np.stack([x.ravel(), y.ravel(), z.ravel()], axis=1).astype(np.float32)


@dataclass
class ScanResult:
    points: np.ndarray          # (P, 3) float32 mm
    photons_per_point: int
    counts: np.ndarray          # (P, cells) int64, cell = i + nx*j
    tsum: np.ndarray            # (P, cells) uint64 fixed-point sums of t
    tsum2: np.ndarray           # (P, cells) uint64 fixed-point sums of t^2
    tmin: np.ndarray            # (P, cells) float32
    counters: dict = field(default_factory=dict)
    seconds: float = 0.0


def scan_light(engine, box: Box, op, ro, *, points: np.ndarray, photons_per_point: int, seed: int,
               pid_offset: int = 0, batch_points: int = 4096, max_bounces: int = 100_000,
               tau_ns: float = 0.0) -> ScanResult:
    """Transport ``photons_per_point`` photons from each point (emitted at
    t = 0, no decay-time delay by default, so the times are transit times) and
    collect per-point SiPM counts and arrival-time moments on the GPU."""
    import time
    import torch
    ro = ro if isinstance(ro, Readout) else Readout(ro)
    cells = ro.grid.nx * ro.grid.ny
    pts = np.ascontiguousarray(points, np.float32).reshape(-1, 3)
    P = pts.shape[0]
    npp = int(photons_per_point)
    dev = torch.device("cuda", engine.device if hasattr(engine, "device") else 0)
    counts = np.zeros((P, cells), np.int64)
    tsum = np.zeros((P, cells), np.uint64)
    tsum2 = np.zeros((P, cells), np.uint64)
    tmin = np.zeros((P, cells), np.float32)
    tot = None
    tb = TimeBinning(100.0, 80)
    stream = torch.cuda.Stream(device=dev)
    t0 = time.perf_counter()
    with torch.cuda.stream(stream):
        for b0 in range(0, P, batch_points):
            nb = min(batch_points, P - b0)
            src = torch.from_numpy(pts[b0:b0 + nb]).to(dev)
            sx, sy, sz = (src[:, i].contiguous() for i in range(3))
            off = torch.arange(nb + 1, dtype=torch.int64, device=dev) * npp
            segid = torch.arange(nb, dtype=torch.int32, device=dev)
            maps = torch.empty(nb * cells, dtype=torch.int32, device=dev)
            tm = torch.empty(nb * cells, dtype=torch.float32, device=dev)
            npe = torch.empty(nb, dtype=torch.int32, device=dev)
            ctr = torch.zeros(9, dtype=torch.int64, device=dev)
            s1 = torch.empty(nb * cells, dtype=torch.int64, device=dev)
            s2 = torch.empty(nb * cells, dtype=torch.int64, device=dev)
            engine.run_segments_moments_device(
                box, op, ro, tb, sx=sx.data_ptr(), sy=sy.data_ptr(), sz=sz.data_ptr(), st=None,
                src_offsets=off.data_ptr(), src_segment=segid.data_ptr(), n_src=nb, n_segments=nb,
                n_photons=nb * npp, seed=seed, pid_offset=pid_offset + b0 * npp, tau_ns=tau_ns,
                max_bounces=max_bounces, maps=maps.data_ptr(), tmin=tm.data_ptr(), npe=npe.data_ptr(),
                counters=ctr.data_ptr(), tsum=s1.data_ptr(), tsum2=s2.data_ptr(),
                stream=stream.cuda_stream)
            engine.sync(stream.cuda_stream)
            counts[b0:b0 + nb] = maps.view(nb, cells).cpu().numpy().astype(np.uint32)
            tsum[b0:b0 + nb] = s1.view(nb, cells).cpu().numpy().view(np.uint64)
            tsum2[b0:b0 + nb] = s2.view(nb, cells).cpu().numpy().view(np.uint64)
            tmin[b0:b0 + nb] = tm.view(nb, cells).cpu().numpy()
            c = ctr.cpu().numpy()
            tot = c if tot is None else tot + c
    from .params import COUNTER_NAMES
    return ScanResult(pts, npp, counts, tsum, tsum2, tmin,
                      {n: int(v) for n, v in zip(COUNTER_NAMES, tot)} if tot is not None else {},
                      time.perf_counter() - t0)


MIN_TIME_COUNTS = 20       # below this a cell's time moments are replaced by column medians
FIRST_PASS_FLOOR = 1e-6    # floor of a training target's probability minus its first-pass term
SIGMA_FLOOR_NS = 1e-3


def light_targets(scan: ScanResult) -> np.ndarray:
    """Network targets (P, 192): log detection probability, mean arrival time
    (ns) and log of its standard deviation, per SiPM."""
    n = float(scan.photons_per_point)
    c = scan.counts.astype(np.float64)
    logp = np.log((c + 0.5) / (n + 1.0))
    with np.errstate(divide="ignore", invalid="ignore"):
        m1 = scan.tsum.astype(np.float64) / _lib.MOMENT_T_SCALE / c
        m2 = scan.tsum2.astype(np.float64) / _lib.MOMENT_T2_SCALE / c
        var = np.maximum(m2 - m1 * m1, SIGMA_FLOOR_NS ** 2)
        logs = 0.5 * np.log(var)
    ok = c >= MIN_TIME_COUNTS
    for a in (m1, logs):
        med = np.array([np.median(a[ok[:, j], j]) if ok[:, j].any() else 0.0 for j in range(a.shape[1])])
        a[~ok] = np.broadcast_to(med, a.shape)[~ok]
    return np.concatenate([logp, m1, logs], axis=1).astype(np.float32)


def members_of_rank(members: int, rank: int, world: int) -> list:
    """Ensemble members trained by ``rank`` of ``world`` (one GPU each):
    rank, rank + world, ..."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("need 0 <= rank < world")
    return list(range(rank, int(members), world))


def _gather_members(trained: dict, members: int, world: int, group):
    """All ranks receive every member's parameters and loss history, in member
    order (all_gather of a (members per rank, P) block, padded)."""
    import torch
    import torch.distributed as dist
    per = -(-members // world)
    some = next(iter(trained.values()))[0] if trained else None
    n_par = np.zeros(1, np.int64)
    if some is not None:
        n_par[0] = np.asarray(some).size
    dev = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend(group) == "nccl" \
        else torch.device("cpu")
    t = torch.from_numpy(n_par).to(dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    P = int(t.item())
    n_hist = max((len(h) for _, h in trained.values()), default=0)
    t = torch.tensor([n_hist], dtype=torch.int64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    H = int(t.item())
    block = np.zeros((per, P + H), np.float32)
    rank = dist.get_rank(group)
    for i, k in enumerate(members_of_rank(members, rank, world)):
        p, h = trained[k]
        block[i, :P] = np.asarray(p, np.float32)
        block[i, P:P + len(h)] = np.asarray(h, np.float32)
    src = torch.from_numpy(block).to(dev)
    out = [torch.empty_like(src) for _ in range(world)]
    dist.all_gather(out, src, group=group)
    blocks = [o.cpu().numpy() for o in out]
    params, history = [], []
    for k in range(members):
        r, i = k % world, k // world
        params.append(blocks[r][i, :P].copy())
        history.append([float(v) for v in blocks[r][i, P:P + H]])
    return params, history


def split_holdout(n_points: int, frac: float = 0.1, seed: int = 11):
    """Deterministic train / held-out split of point indices."""
    rng = np.random.default_rng(seed)
    perm = rng.permutation(n_points)
    n_hold = int(round(frac * n_points))
    return np.sort(perm[n_hold:]), np.sort(perm[:n_hold])


# ---------------------------------------------------------------------------
# First-pass light
# ---------------------------------------------------------------------------
def first_pass_optics(op, ro) -> tuple:
    """The optics the first-pass term depends on: (n_crystal, n_coupling,
    abs_len_mm, rayleigh_mm, pitch_mm, nx, ny)."""
    ro = ro if isinstance(ro, Readout) else Readout(ro)
    return (float(op.n_crystal), float(op.n_coupling), float(op.abs_len_mm), float(op.rayleigh_mm),
            float(ro.grid.pitch_mm), int(ro.grid.nx), int(ro.grid.ny))


def first_pass_light(xyz, box: Box, optics: tuple, device: int = 0, stream=None):
    """First-pass detection probabilities (cl_surrogate_direct) of emission
    points xyz ((n, 3) float32 CUDA tensor or array, mm): torch tensor
    (n, 64) on the GPU.  A photon reaches the readout face without a bulk
    interaction, is transmitted and lands in the SiPM's pixel; PDE 1."""
    import torch
    from .params import OpticalParams, SipmGrid
    from .transport import stream_arg
    x = torch.as_tensor(np.asarray(xyz, np.float32) if not isinstance(xyz, torch.Tensor) else xyz,
                        dtype=torch.float32, device=f"cuda:{device}").contiguous()
    n1, n2, ab, ray, pitch, nx, ny = optics
    op = OpticalParams(n1, n2, ab, ray, 1.0, True, True, 0.0, 1.0)
    ro = Readout(SipmGrid(pitch, int(nx), int(ny)))
    out = torch.empty((x.shape[0], N_CELLS), dtype=torch.float32, device=x.device)
    rc = _lib.load().cl_surrogate_direct(C.c_void_p(x.data_ptr()), int(x.shape[0]), C.byref(box),
                                         C.byref(op), C.byref(ro), C.c_void_p(out.data_ptr()),
                                         stream_arg(stream))
    if rc != 0:
        raise _lib.CudaTransportError(rc, "cl_surrogate_direct failed")
    return out


# ---------------------------------------------------------------------------
# Ensemble
# ---------------------------------------------------------------------------
@dataclass
class LightSurrogate:
    """K networks plus the input scaling and the target standardisation."""
    box_mm: np.ndarray          # (3,)
    y_mean: np.ndarray          # (192,)
    y_std: np.ndarray           # (192,)
    members: list               # K parameter vectors (float32)
    cells: int = N_CELLS
    meta: dict = field(default_factory=dict)
    z_warp: float = 0.0         # network input depth: 2 depth_warp((z - z0) / (z1 - z0)) - 1
    z_range: Optional[tuple] = None   # (z0, z1) mm of a slab ensemble; None: the whole crystal
    # optics of the first-pass term (first_pass_optics) when the members were
    # trained on the light response minus it; None: on the whole response
    first_pass: Optional[tuple] = None

    def depth_range(self) -> tuple:
        """(z0, z1) in mm: the depths the network's input spans."""
        if self.z_range is None:
            return 0.0, float(self.box_mm[2])
        return float(self.z_range[0]), float(self.z_range[1])

    def normalise(self, xyz: np.ndarray) -> np.ndarray:
        """Network inputs: x and y scaled to [-1, 1]; z through the depth warp
        of its position in the ensemble's depth range (clamped to it)."""
        q = np.asarray(xyz, np.float64).reshape(-1, 3)
        L = self.box_mm.astype(np.float64)
        out = 2.0 * q / L - 1.0
        z0, z1 = self.depth_range()
        out[:, 2] = 2.0 * depth_warp((q[:, 2] - z0) / (z1 - z0), self.z_warp) - 1.0
        return out.astype(np.float32)

    @classmethod
    def train(cls, box: Box, xyz: np.ndarray, targets: np.ndarray, *, members: int = 5, steps: int = 20000,
              batch: int = 65536, lr: float = 1e-3, lr_final: Optional[float] = None,
              time_weight: float = 1.0, z_warp: float = 0.0, z_range=None, seed: int = 0,
              device: int = 0, chunk: int = 250, log=None, group=None, member_trainer=None,
              first_pass: Optional[tuple] = None):
        """Train ``members`` networks on standardised targets.

        ``lr_final``: cosine decay of the Adam step size from ``lr`` to
        ``lr_final`` over the steps (piecewise constant per ``chunk`` steps);
        None keeps ``lr``.  ``time_weight``: weight of the 128 arrival-time
        outputs in the squared-error loss relative to the 64 log-probabilities
        (applied by standardising those targets with std / sqrt(time_weight)).

        With a ``torch.distributed`` process ``group`` the members are spread
        over its ranks, one GPU each (rank r trains members r, r + world, ...
        on ``device``) and every rank returns the whole ensemble (one
        all_gather of the parameter vectors).  Member k's initialisation and
        minibatch stream depend on k only, so the ensemble is the same for
        any number of ranks.  ``member_trainer(k, x, y) -> (params, losses)``
        replaces the tensor-core trainer (tests).  ``first_pass``: the optics
        of the first-pass term (first_pass_optics) when ``targets`` hold the
        light response minus it (prediction adds it back)."""
        import math
        import time
        L = np.array([float(box.L[i]) for i in range(3)], np.float64)
        y_mean = targets.mean(0).astype(np.float64)
        y_std = np.maximum(targets.std(0), 1e-6).astype(np.float64)
        y_std[N_CELLS:] /= math.sqrt(time_weight)
        obj = cls(L, y_mean.astype(np.float32), y_std.astype(np.float32), [], z_warp=float(z_warp),
                  z_range=None if z_range is None else (float(z_range[0]), float(z_range[1])),
                  first_pass=None if first_pass is None else tuple(first_pass))
        xn = obj.normalise(xyz)
        yn = ((targets - y_mean) / y_std).astype(np.float32)
        if member_trainer is None:
            import torch
            x = torch.from_numpy(xn).to(f"cuda:{device}")
            y = torch.from_numpy(yn).to(f"cuda:{device}")

            def member_trainer(k, x, y):
                net = MLP(device, max_batch=batch, seed=seed * 1000 + k)
                try:
                    net.set_data(x, y)
                    hist = []
                    for s0 in range(0, steps, chunk):
                        ns = min(chunk, steps - s0)
                        if lr_final is None:
                            lr_now = lr
                        else:
                            mid = (s0 + 0.5 * ns) / steps
                            lr_now = lr_final + 0.5 * (lr - lr_final) * (1.0 + math.cos(math.pi * mid))
                        hist.append(net.train(ns, batch=batch, lr=lr_now, seed=seed * 1000 + k))
                        if log and ((s0 + ns) % 2000 == 0 or s0 + ns == steps):
                            log(f"member {k} step {s0 + ns}: lr {lr_now:.2e} loss {hist[-1]:.5f}")
                    return net.get_params(), hist
                finally:
                    net.close()
        else:
            x, y = xn, yn
        rank, world = 0, 1
        if group is not None:
            import torch.distributed as dist
            rank, world = dist.get_rank(group), dist.get_world_size(group)
        mine = members_of_rank(members, rank, world)
        t0 = time.perf_counter()
        trained = {k: member_trainer(k, x, y) for k in mine}
        if group is None:
            params = [trained[k][0] for k in range(members)]
            history = [trained[k][1] for k in range(members)]
        else:
            params, history = _gather_members(trained, members, world, group)
        obj.members = [np.asarray(p, np.float32) for p in params]
        obj.meta = {"steps": steps, "batch": batch, "lr": lr, "lr_final": lr_final,
                    "time_weight": time_weight, "z_warp": z_warp, "z_range": obj.z_range, "seed": seed,
                    "train_seconds": time.perf_counter() - t0, "loss_history": history,
                    "ranks": world}
        return obj

    def raw_outputs(self, xyz: np.ndarray, device: int = 0):
        """Standardised outputs of every member: torch tensor (K, n, 192) on the GPU."""
        import torch
        x = torch.from_numpy(self.normalise(xyz)).to(f"cuda:{device}")
        outs = []
        net = MLP(device, max_batch=65536, seed=0)
        try:
            for p in self.members:
                net.set_params(p)
                outs.append(net.forward(x))
        finally:
            net.close()
        return torch.stack(outs)

    def predict(self, xyz: np.ndarray, device: int = 0) -> dict:
        """Ensemble means (numpy): p (n, cells), t_mean, t_sigma (ns), and the
        count-weighted relative spread of the members' p (n,)."""
        raw = self.raw_outputs(xyz, device).double().cpu().numpy()
        y = raw * self.y_std.astype(np.float64) + self.y_mean.astype(np.float64)
        c = self.cells
        p = np.exp(y[:, :, :c])
        if self.first_pass is not None:
            # the same first-pass term for every member: it moves the mean, not the spread
            box = Box(tuple(float(v) for v in self.box_mm))
            p = p + first_pass_light(np.asarray(xyz, np.float32).reshape(-1, 3), box, self.first_pass,
                                     device).double().cpu().numpy()[None]
        pm = p.mean(0)
        spread = p.std(0).sum(1) / np.maximum(pm.sum(1), 1e-30)
        return {"p": pm, "t_mean": y[:, :, c:2 * c].mean(0), "t_sigma": np.exp(y[:, :, 2 * c:].mean(0)),
                "spread": spread, "p_members": p}

    def save(self, path: str):
        np.savez_compressed(path, box_mm=self.box_mm, y_mean=self.y_mean, y_std=self.y_std,
                            members=np.stack(self.members), cells=self.cells, z_warp=np.float64(self.z_warp),
                            z_range=np.float64(self.depth_range() if self.z_range is not None else (np.nan, np.nan)),
                            first_pass=np.float64(self.first_pass if self.first_pass is not None else [np.nan] * 7),
                            meta=np.array(repr({k: v for k, v in self.meta.items() if k != "loss_history"})))

    @classmethod
    def load(cls, path: str):
        z = np.load(path, allow_pickle=False)
        zr = None
        if "z_range" in z.files and np.all(np.isfinite(z["z_range"])):
            zr = (float(z["z_range"][0]), float(z["z_range"][1]))
        fp = None
        if "first_pass" in z.files and not np.any(np.isnan(z["first_pass"])):
            f = [float(v) for v in z["first_pass"]]
            fp = (f[0], f[1], f[2], f[3], f[4], int(f[5]), int(f[6]))
        return cls(z["box_mm"], z["y_mean"], z["y_std"], list(z["members"]), int(z["cells"]),
                   {"saved": str(z["meta"])}, float(z["z_warp"]) if "z_warp" in z.files else 0.0, zr, fp)
