"""Differentiable rollout: forward + hand-written adjoint of the fixed-corotated
CK-MPM substep as a torch.autograd.Function.

No counterpart in the reference.  The CUDA library runs the forward on a dense
grid of the scene's domain with exact fixed-point deposits and keeps a
checkpoint every `checkpoint_every` substeps; backward recomputes one segment
at a time from its checkpoint and runs the adjoint of P2G, the grid update,
G2P and the SVD-based stress (ckmpm_b200/csrc/diff_math.cuh).  By default the
interval is the smallest whose checkpoints and tape fit in half of the free
device memory: 1 (the whole rollout kept, nothing recomputed) whenever it fits.  Inputs and
outputs are CUDA float32 tensors; the work is ordered on torch's current
stream.

    sim = DiffRollout(cfg, n, mass, volume, nu=0.3, nsteps=200, dt=1e-4)
    xT, FT = rollout(sim, x0, v0, logE)        # x0, v0: [n, 3]; logE: [n]
    loss = ((xT.mean(0) - target) ** 2).sum()
    loss.backward()                            # gradients for x0, v0, logE
"""
from __future__ import annotations

import ctypes as C

import torch

from . import _capi as capi
from .engine import MPMConfig


def _lib():
    L = capi.lib()
    if not getattr(L, "_diff_bound", False):
        P = C.c_void_p
        L.ckmpm_diff_create.argtypes = [C.POINTER(capi.SceneDesc), C.c_uint32, C.c_float, C.c_float, C.c_float,
                                        C.c_uint32, C.c_float, C.c_uint32, C.POINTER(P)]
        L.ckmpm_diff_forward.argtypes = [P, P, P, P, P, P, P]
        L.ckmpm_diff_backward.argtypes = [P, P, P, P, P, P, P]
        L.ckmpm_diff_timing.argtypes = [P, C.POINTER(C.c_float), C.POINTER(C.c_uint64)]
        L.ckmpm_diff_last_error.argtypes = [P]
        L.ckmpm_diff_last_error.restype = C.c_char_p
        L.ckmpm_diff_destroy.argtypes = [P]
        for name in ("ckmpm_diff_create", "ckmpm_diff_forward", "ckmpm_diff_backward", "ckmpm_diff_timing",
                     "ckmpm_diff_destroy"):
            getattr(L, name).restype = C.c_int
        L._diff_bound = True
    return L


def _check(code: int, where: str, handle) -> None:
    if code != capi.CKMPM_OK:
        msg = _lib().ckmpm_diff_last_error(handle)
        raise capi.CkmpmError(code, where, msg.decode() if msg else "")


def _ptr(t: torch.Tensor | None):
    if t is None:
        return None
    assert t.is_cuda and t.dtype == torch.float32 and t.is_contiguous()
    return C.c_void_p(t.data_ptr())


def rollout_bytes(config: MPMConfig, n: int, nsteps: int, every: int) -> int:
    """Device bytes of the checkpoints and the recomputation tape of a rollout of n
    particles over nsteps substeps with a checkpoint every `every` substeps: each
    checkpoint holds x and F (48 B per particle) and the node velocities (16 B per
    node of both staggered grids of the domain); the tape holds every - 1 states
    and every node-velocity slots."""
    nodes = 2
    for b in config.domain_blocks:
        nodes *= 4 * int(b)
    state, vel = 48 * n, 16 * nodes
    nseg = -(-nsteps // every)
    return nseg * (state + vel) + max(every - 1, 1) * state + every * vel


def auto_checkpoint_interval(config: MPMConfig, n: int, nsteps: int, budget_bytes: int) -> int:
    """The smallest checkpoint interval whose checkpoints and tape fit in budget_bytes;
    when none does, the interval that needs the least memory."""
    for every in range(1, nsteps + 1):
        if rollout_bytes(config, n, nsteps, every) <= budget_bytes:
            return every
    return min(range(1, nsteps + 1), key=lambda k: (rollout_bytes(config, n, nsteps, k), k))


class DiffRollout:
    """A differentiable rollout of n fixed-corotated particles (ckmpm_diff_* handle).
    checkpoint_every None picks the interval by memory (auto_checkpoint_interval
    over half of the device's free memory)."""

    def __init__(self, config: MPMConfig, n: int, mass: float, volume: float, nu: float = 0.3, nsteps: int = 200,
                 dt: float = 1e-4, checkpoint_every: int | None = None):
        self.config, self.n, self.nsteps, self.dt = config, n, nsteps, dt
        if checkpoint_every is None:
            free, _ = torch.cuda.mem_get_info(config.device)
            checkpoint_every = auto_checkpoint_interval(config, n, nsteps, free // 2)
        self.checkpoint_every = checkpoint_every
        self._h = C.c_void_p()
        desc = config.to_c()
        _check(_lib().ckmpm_diff_create(C.byref(desc), n, mass, volume, nu, nsteps, dt, checkpoint_every,
                                        C.byref(self._h)), "ckmpm_diff_create", None)

    def forward(self, x0: torch.Tensor, v0: torch.Tensor, logE: torch.Tensor) -> tuple[torch.Tensor, torch.Tensor]:
        xT = torch.empty((self.n, 3), device=x0.device, dtype=torch.float32)
        FT = torch.empty((self.n, 3, 3), device=x0.device, dtype=torch.float32)
        stream = C.c_void_p(torch.cuda.current_stream(x0.device).cuda_stream)
        _check(_lib().ckmpm_diff_forward(self._h, _ptr(x0), _ptr(v0), _ptr(logE), _ptr(xT), _ptr(FT), stream),
               "ckmpm_diff_forward", self._h)
        return xT, FT

    def backward(self, gxT: torch.Tensor | None, gFT: torch.Tensor | None, device):
        gx0 = torch.empty((self.n, 3), device=device, dtype=torch.float32)
        gv0 = torch.empty((self.n, 3), device=device, dtype=torch.float32)
        glogE = torch.empty((self.n,), device=device, dtype=torch.float32)
        stream = C.c_void_p(torch.cuda.current_stream(device).cuda_stream)
        _check(_lib().ckmpm_diff_backward(self._h, _ptr(gxT), _ptr(gFT), _ptr(gx0), _ptr(gv0), _ptr(glogE), stream),
               "ckmpm_diff_backward", self._h)
        return gx0, gv0, glogE

    def generation(self) -> int:
        ms = (C.c_float * 2)()
        g = C.c_uint64()
        _check(_lib().ckmpm_diff_timing(self._h, ms, C.byref(g)), "ckmpm_diff_timing", self._h)
        return g.value

    def timing_ms(self) -> tuple[float, float]:
        """Device time of the last forward and backward (ms)."""
        ms = (C.c_float * 2)()
        g = C.c_uint64()
        _check(_lib().ckmpm_diff_timing(self._h, ms, C.byref(g)), "ckmpm_diff_timing", self._h)
        return ms[0], ms[1]

    def close(self) -> None:
        if self._h:
            _lib().ckmpm_diff_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class _Rollout(torch.autograd.Function):
    @staticmethod
    def forward(ctx, sim: DiffRollout, x0, v0, logE):
        x0c, v0c, lc = (t.detach().contiguous().float() for t in (x0, v0, logE))
        xT, FT = sim.forward(x0c, v0c, lc)
        ctx.sim = sim
        ctx.gen = sim.generation()
        ctx.device = x0.device
        return xT, FT

    @staticmethod
    def backward(ctx, gxT, gFT):
        sim = ctx.sim
        if sim.generation() != ctx.gen:
            raise RuntimeError("DiffRollout ran another forward since this graph was built; its checkpoints are gone")
        gxT = None if gxT is None else gxT.contiguous().float()
        gFT = None if gFT is None else gFT.contiguous().float()
        gx0, gv0, glogE = sim.backward(gxT, gFT, ctx.device)
        return None, gx0, gv0, glogE


def rollout(sim: DiffRollout, x0: torch.Tensor, v0: torch.Tensor, logE: torch.Tensor):
    """(xT [n, 3], FT [n, 3, 3]) after sim.nsteps substeps, differentiable in x0, v0 and logE."""
    return _Rollout.apply(sim, x0, v0, logE)
