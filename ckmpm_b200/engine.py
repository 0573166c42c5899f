"""Python host interface mirroring the reference's engine/material/model/config API.

Names and call order follow AppledoreM/CKMPM:
  * MPMConfig        <- MPMConfigBase<Derived> getters (include/mpm_config.h:12-124)
                        plus the domain extent of MPMDomainRange (include/mpm_domain.h:17-30)
  * MPMMaterial      <- MPMMaterial<k> and its MaterialParameter_ (include/mpm_material.cuh:20-175)
  * MPMModel         <- MPMModel(mass, volume, x, v, material, freezeTime) (include/mpm_model.h:11-59)
  * MPMEngine        <- MPMEngine<GridConfig>: Initialize, InitializeParticle,
                        InitialSetup, Simulate (include/mpm_engine.cuh:29-974)

Differences, all at the boundary: scene constants are run-time values instead
of compile-time CRTP getters; the engine is an ordinary object (several per
process) instead of a per-GridConfig singleton; failures raise CkmpmError
instead of calling exit()/abort(); Simulate returns instead of ending the
process.  All arithmetic runs in the CUDA library (ckmpm_b200/_lib).
"""
from __future__ import annotations

import ctypes as C
import json
import math
from dataclasses import dataclass, field
from pathlib import Path
from typing import Sequence

import numpy as np

from . import _capi as capi

ConstitutiveModel = {"fixed_corotated": capi.FIXED_COROTATED, "linear": capi.LINEAR,
                     "drucker_prager": capi.DRUCKER_PRAGER, "fluid": capi.FLUID, "von_mises": capi.VON_MISES,
                     "nacc": capi.NACC}


def compute_lame_parameters(E: float, nu: float) -> tuple[float, float]:
    """(lambda, mu) from Young's modulus and Poisson ratio (include/mpm_material.cuh:277-283)."""
    lam = E * nu / ((1 + nu) * (1 - 2 * nu))
    mu = E / (2 * (1 + nu))
    return lam, mu


def evaluate_sound_speed(E: float, nu: float, rho: float) -> float:
    """include/mpm_test_base.h:15-19."""
    return math.sqrt(E * (1 - nu) / ((1 + nu) * (1 - 2 * nu) * rho))


def evaluate_timestep(dx: float, E: float, nu: float, rho: float, cfl: float = 0.5) -> float:
    """cfl * dx / sound speed (include/mpm_test_base.h:21-24)."""
    return cfl * dx / evaluate_sound_speed(E, nu, rho)


@dataclass
class MPMMaterial:
    """One constitutive model and its parameters, as MaterialParameter_ of
    MPMMaterial<k> (include/mpm_material.cuh:24-257):

    * 'fixed_corotated' | 'drucker_prager' | 'linear': lambda_, mu_;
    * 'fluid': bulk_, gamma_, viscosity_, J0_;
    * 'von_mises': mu_, lambda_, yield_stress_;
    * 'nacc' (non-associated Cam-clay): mu_, lambda_, alpha0_, beta_,
      hardening_factor_, m_, hardening_on_.
    """
    kind: str
    lambda_: float = 0.0
    mu_: float = 0.0
    bulk_: float = 0.0
    gamma_: float = 0.0
    viscosity_: float = 0.0
    J0_: float = 1.0
    yield_stress_: float = 0.0
    alpha0_: float = 0.0
    beta_: float = 0.0
    hardening_factor_: float = 0.0
    m_: float = 0.0
    hardening_on_: bool = True

    @staticmethod
    def fixed_corotated(lambda_: float, mu_: float) -> "MPMMaterial":
        return MPMMaterial("fixed_corotated", lambda_=lambda_, mu_=mu_)

    @staticmethod
    def drucker_prager(lambda_: float, mu_: float) -> "MPMMaterial":
        return MPMMaterial("drucker_prager", lambda_=lambda_, mu_=mu_)

    @staticmethod
    def linear(lambda_: float, mu_: float) -> "MPMMaterial":
        return MPMMaterial("linear", lambda_=lambda_, mu_=mu_)

    @staticmethod
    def fluid(bulk: float, gamma: float, viscosity: float, J0: float = 1.0) -> "MPMMaterial":
        return MPMMaterial("fluid", bulk_=bulk, gamma_=gamma, viscosity_=viscosity, J0_=J0)

    @staticmethod
    def von_mises(mu: float, lambda_: float, yield_stress: float) -> "MPMMaterial":
        return MPMMaterial("von_mises", mu_=mu, lambda_=lambda_, yield_stress_=yield_stress)

    @staticmethod
    def nacc(mu: float, lambda_: float, alpha0: float, beta: float, hardening_factor: float, m: float,
             hardening_on: bool = True) -> "MPMMaterial":
        return MPMMaterial("nacc", mu_=mu, lambda_=lambda_, alpha0_=alpha0, beta_=beta,
                           hardening_factor_=hardening_factor, m_=m, hardening_on_=hardening_on)

    @property
    def kind_code(self) -> int:
        return ConstitutiveModel[self.kind]

    def params(self) -> list[float]:
        """The 8 parameter slots of ckmpm_material.p, in the reference's field order."""
        if self.kind == "fluid":
            p = [self.bulk_, self.gamma_, self.viscosity_, self.J0_]
        elif self.kind == "von_mises":
            p = [self.mu_, self.lambda_, self.yield_stress_]
        elif self.kind == "nacc":
            p = [self.mu_, self.lambda_, self.alpha0_, self.beta_, self.hardening_factor_, self.m_,
                 1.0 if self.hardening_on_ else 0.0]
        else:
            p = [self.lambda_, self.mu_]
        return [float(v) for v in p] + [0.0] * (capi.MATERIAL_PARAMS - len(p))

    def to_c(self) -> capi.Material:
        m = capi.Material()
        m.kind = self.kind_code
        for i, v in enumerate(self.params()):
            m.p[i] = float(v)
        return m


@dataclass
class MPMModel:
    """Particles of one material: MPMModel(mass, volume, x, v, material, freezeTime)."""
    particle_mass: float
    particle_volume: float
    particle_position: np.ndarray
    particle_velocity: np.ndarray
    material: MPMMaterial
    freeze_time: float = 0.0

    def __post_init__(self):
        self.particle_position = np.ascontiguousarray(self.particle_position, dtype=np.float32).reshape(-1, 3)
        self.particle_velocity = np.ascontiguousarray(self.particle_velocity, dtype=np.float32).reshape(-1, 3)
        n, nv = len(self.particle_position), len(self.particle_velocity)
        if nv not in (1, n):
            raise ValueError("particle_velocity must hold 1 or n velocities (include/mpm_model.h:31-32)")

    def GetParticleMass(self) -> float:
        return self.particle_mass

    def GetParticleVolume(self) -> float:
        return self.particle_volume

    def GetParticleCount(self) -> int:
        return len(self.particle_position)

    def GetParticleMaterial(self) -> MPMMaterial:
        return self.material

    def IsFreezed(self, elapsed_seconds: float) -> bool:
        return elapsed_seconds < self.freeze_time


@dataclass
class MPMConfig:
    """Scene constants: the MPMConfigBase getters plus the domain extent in blocks."""
    dx: float
    domain_blocks: tuple[int, int, int]
    gravity: float = -9.8
    mass_clamp: float = 0.0
    dt: float = 1e-4
    cfl: float = 0.5
    fps: int = 48
    total_frames: int = 1
    boundary: str = "sticky_blocks"
    floor_cells: float = 8.0
    max_particles_per_block: int = 4096
    track_ids: bool = True
    device: int = 0
    block_size: int = 4
    particles_per_cell_cap: int = 64
    # Rigid particles (GetExistRigidParticle / GetRigidParticleCount /
    # GetRigidParticleVelocity(frame), include/mpm_config.h:92-106): the first
    # rigid_particle_count particles of every von Mises model are rigid;
    # rigid_particle_velocity is (vx, vy, vz) or a callable frame -> (vx, vy, vz).
    exist_rigid_particle: bool = False
    rigid_particle_count: int = 0
    rigid_particle_velocity: object = (0.0, 0.0, 0.0)
    # boundary == "field": (rule, param) per grid cell, the irregular-boundary hook
    # (GetExistIrregularBoundary / ProcessGridCellVelocity, include/mpm_config.h:108-117)
    # evaluated into data; see ckmpm_b200.boundary.
    boundary_field: object = None

    # MPMConfigBase getter names (include/mpm_config.h:17-123)
    def GetDx(self) -> float:
        return self.dx

    def GetInvDx(self) -> float:
        return 1.0 / self.dx

    def GetBlockSize(self) -> int:
        return self.block_size

    def GetBlockVolume(self) -> int:
        return self.block_size ** 3

    def GetMaxParticleCountPerCell(self) -> int:
        return self.particles_per_cell_cap

    def GetMaxParticleCountPerBlock(self) -> int:
        return self.max_particles_per_block

    def GetFps(self) -> int:
        return self.fps

    def GetDt(self) -> float:
        return self.dt

    def GetCfl(self) -> float:
        return self.cfl

    def GetTotalSimulatedFrameCount(self) -> int:
        return self.total_frames

    def GetGravity(self) -> float:
        return self.gravity

    def GetMassClamp(self) -> float:
        return self.mass_clamp

    def GetExistRigidParticle(self) -> bool:
        return self.exist_rigid_particle

    def GetRigidParticleCount(self) -> int:
        return self.rigid_particle_count

    def GetRigidParticleVelocity(self, frame: int = 0) -> tuple[float, float, float]:
        v = self.rigid_particle_velocity
        v = v(frame) if callable(v) else v
        return tuple(float(c) for c in v)

    def to_c(self) -> capi.SceneDesc:
        d = capi.SceneDesc()
        d.dx = self.dx
        for i in range(3):
            d.domain_blocks[i] = int(self.domain_blocks[i])
        d.gravity = self.gravity
        d.mass_clamp = self.mass_clamp
        d.boundary = {"sticky_blocks": capi.BOUNDARY_STICKY_BLOCKS, "slip_floor": capi.BOUNDARY_SLIP_FLOOR,
                      "field": capi.BOUNDARY_FIELD}[self.boundary]
        d.floor_cells = self.floor_cells
        d.max_particles_per_block = self.max_particles_per_block
        d.device = self.device
        d.flags = capi.FLAG_TRACK_IDS if self.track_ids else 0
        return d


@dataclass
class ParticleState:
    x: np.ndarray
    v: np.ndarray
    F: np.ndarray
    aux: np.ndarray
    id: np.ndarray


class Scene:
    """Owner of one ckmpm_scene handle (one simulation on one GPU)."""

    def __init__(self, config: MPMConfig):
        self.config = config
        self._h = C.c_void_p()
        L = capi.lib()
        desc = config.to_c()
        capi.check(L.ckmpm_create(C.byref(desc), C.byref(self._h)), "ckmpm_create", None)
        self.models: list[MPMModel] = []
        self._exports_in_flight: list[np.ndarray] = []  # host buffers of unfinished exports
        if config.exist_rigid_particle:
            self.set_rigid(config.rigid_particle_count, config.GetRigidParticleVelocity(0))
        if config.boundary == "field" and config.boundary_field is not None:
            self.set_boundary_field(*config.boundary_field)

    def set_boundary_field(self, rule, param=None) -> None:
        """Per-cell boundary rules of a boundary="field" scene: rule (uint8, one per
        cell, shape (Nx, Ny, Nz) or flat x-major) and param (3 floats per cell: the
        normal of SLIP / SEPARATE cells, the velocity of VELOCITY cells)."""
        r = np.ascontiguousarray(rule, np.uint8).ravel()
        p = None if param is None else np.ascontiguousarray(param, np.float32).reshape(-1)
        capi.check(capi.lib().ckmpm_set_boundary_field(self._h, r.ctypes.data_as(C.POINTER(C.c_uint8)),
                                                       capi.fptr(p)), "ckmpm_set_boundary_field", self._h)

    def set_rigid(self, count: int, velocity) -> None:
        """Rigid particles on (before setup): the first `count` particles of
        every von Mises model start rigid and move with `velocity`."""
        v = np.ascontiguousarray(velocity, np.float32).reshape(3)
        capi.check(capi.lib().ckmpm_set_rigid(self._h, int(count), capi.fptr(v)), "ckmpm_set_rigid", self._h)

    def set_rigid_velocity(self, velocity) -> None:
        """Velocity of the rigid particles for the substeps enqueued from now on."""
        v = np.ascontiguousarray(velocity, np.float32).reshape(3)
        capi.check(capi.lib().ckmpm_set_rigid_velocity(self._h, capi.fptr(v)), "ckmpm_set_rigid_velocity", self._h)

    def add_model(self, model: MPMModel) -> int:
        L = capi.lib()
        mat = model.material.to_c()
        idx = C.c_int32()
        x, v = model.particle_position, model.particle_velocity
        capi.check(L.ckmpm_add_model(self._h, C.byref(mat), len(x), capi.fptr(x), capi.fptr(v), len(v),
                                     model.particle_mass, model.particle_volume, C.byref(idx)),
                   "ckmpm_add_model", self._h)
        self.models.append(model)
        return idx.value

    def setup(self) -> None:
        capi.check(capi.lib().ckmpm_setup(self._h), "ckmpm_setup", self._h)

    def set_stream(self, stream_handle: int | None) -> None:
        capi.check(capi.lib().ckmpm_set_stream(self._h, C.c_void_p(stream_handle or 0)), "ckmpm_set_stream", self._h)

    def step(self, nsteps: int, dt: float) -> None:
        capi.check(capi.lib().ckmpm_step(self._h, nsteps, dt), "ckmpm_step", self._h)

    def step_async(self, nsteps: int, dt: float) -> None:
        capi.check(capi.lib().ckmpm_step_async(self._h, nsteps, dt), "ckmpm_step_async", self._h)

    def status_check(self) -> None:
        capi.check(capi.lib().ckmpm_status_check(self._h), "ckmpm_status_check", self._h)

    def step_adaptive(self, max_steps: int, dt_max: float, cfl: float, frame_time: float) -> float:
        """Advance one frame of frame_time with the reference's dt rule; returns the time advanced."""
        el = C.c_double()
        capi.check(capi.lib().ckmpm_step_adaptive(self._h, max_steps, dt_max, cfl, frame_time, C.byref(el)),
                   "ckmpm_step_adaptive", self._h)
        return el.value

    def time(self) -> tuple[float, float]:
        """(simulated time, end of the current adaptive frame), both in double."""
        out = (C.c_double * 2)()
        capi.check(capi.lib().ckmpm_get_time(self._h, out), "ckmpm_get_time", self._h)
        return out[0], out[1]

    def conservation_metric(self, model: int = 0) -> np.ndarray:
        """The reference's conservation metric of one model (CollectConservationMetric,
        include/mpm_algorithm.cuh:1082-1361, written per substep by Simulate,
        include/mpm_engine.cuh:573-603): rows Eulerian linear and angular
        momentum (left at zero, as the reference leaves them), Lagrangian linear
        momentum sum(v) and angular momentum sum(x cross v), per unit particle mass,
        with v the velocity the next G2P interpolates (zero for rigid particles).
        Summed in double here; the reference adds floats with atomics."""
        st = self.state(model)
        x, v = st.x.astype(np.float64), st.v.astype(np.float64)
        out = np.zeros((4, 3))
        out[2] = v.sum(axis=0)
        out[3] = np.cross(x, v).sum(axis=0)
        return out

    def step_profiled(self, nsteps: int, dt: float) -> tuple[float, float, int]:
        out = (C.c_double * 3)()
        capi.check(capi.lib().ckmpm_step_profiled(self._h, nsteps, dt, out), "ckmpm_step_profiled", self._h)
        return out[0], out[1], int(out[2])

    def count(self, model: int = 0) -> int:
        n = C.c_uint32()
        capi.check(capi.lib().ckmpm_get_count(self._h, model, C.byref(n)), "ckmpm_get_count", self._h)
        return n.value

    def export_positions_async(self, model: int, x: np.ndarray) -> None:
        """Enqueue a positions export of `model` into x (float32, C-contiguous, at
        least the model's particle count rows of 3), as state(model).x would hold
        it; returns at once.  With x in pinned memory (torch's pin_memory) the
        copy overlaps the substeps enqueued after this call.  x is filled when
        export_wait() returns, which gives the number of valid leading rows; read
        nothing from x before that."""
        if x.dtype != np.float32 or not x.flags.c_contiguous or x.ndim != 2 or x.shape[1] != 3:
            raise ValueError("x must be a C-contiguous float32 array of shape (n, 3)")
        capi.check(capi.lib().ckmpm_export_positions_async(self._h, model, capi.fptr(x), x.shape[0]),
                   "ckmpm_export_positions_async", self._h)
        self._exports_in_flight.append(x)

    def export_wait(self) -> int:
        """Wait for the exports enqueued so far; returns the live count of the last one."""
        n = C.c_uint32()
        capi.check(capi.lib().ckmpm_export_wait(self._h, C.byref(n)), "ckmpm_export_wait", self._h)
        self._exports_in_flight.clear()
        return n.value

    def state(self, model: int = 0) -> ParticleState:
        n = self.count(model)
        x = np.zeros((n, 3), np.float32)
        v = np.zeros((n, 3), np.float32)
        F = np.zeros((n, 3, 3), np.float32)
        aux = np.zeros(n, np.float32)
        ids = np.zeros(n, np.uint32)
        nout = C.c_uint32()
        capi.check(capi.lib().ckmpm_get_state(self._h, model, capi.fptr(x), capi.fptr(v), capi.fptr(F),
                                              capi.fptr(aux), capi.uptr(ids), n, C.byref(nout)),
                   "ckmpm_get_state", self._h)
        return ParticleState(x, v, F, aux, ids)

    def blocks(self, model: int = -1, which: int = 0) -> tuple[np.ndarray, np.ndarray]:
        n = C.c_uint32()
        L = capi.lib()
        code = L.ckmpm_get_blocks(self._h, model, which, None, None, 0, C.byref(n))
        if code not in (capi.CKMPM_OK, 6):
            capi.check(code, "ckmpm_get_blocks", self._h)
        keys = np.zeros((n.value, 3), np.int32)
        counts = np.zeros(n.value, np.uint32)
        capi.check(L.ckmpm_get_blocks(self._h, model, which, capi.iptr(keys), capi.uptr(counts), n.value,
                                      C.byref(n)), "ckmpm_get_blocks", self._h)
        return keys, counts

    def counters(self) -> dict:
        out = (C.c_uint64 * 5)()
        capi.check(capi.lib().ckmpm_get_counters(self._h, out), "ckmpm_get_counters", self._h)
        return {"steps": int(out[0]), "lost": int(out[1]), "window_skips": int(out[2]), "status": int(out[3]),
                "timeouts": int(out[4])}

    # Launch shape, autotuner and checkpoints (no counterpart in the reference).
    def tuning(self) -> dict:
        t = capi.Tuning()
        occ = (C.c_uint32 * 2)()
        capi.check(capi.lib().ckmpm_get_tuning(self._h, C.byref(t), occ), "ckmpm_get_tuning", self._h)
        d = t.as_dict()
        d["max_ctas_per_sm"] = {128: int(occ[0]), 256: int(occ[1])}
        return d

    def set_tuning(self, threads: int, ctas_per_sm: int, graph_chunk: int) -> None:
        t = capi.Tuning(threads, ctas_per_sm, graph_chunk, 0.0)
        capi.check(capi.lib().ckmpm_set_tuning(self._h, C.byref(t)), "ckmpm_set_tuning", self._h)

    def set_reorder_interval(self, substeps: int) -> None:
        """Substeps between re-layouts of each block's particles into the setup order
        (default 128, 0 = never); the results do not depend on it."""
        capi.check(capi.lib().ckmpm_set_reorder_interval(self._h, substeps), "ckmpm_set_reorder_interval", self._h)

    def autotune(self, probe_steps: int, dt: float) -> tuple[dict, list[dict]]:
        """Time every launch shape on this scene and keep the fastest; the
        simulation state is left unchanged.  Returns (best, all candidates)."""
        cap = 64
        res = (capi.Tuning * cap)()
        n = C.c_uint32()
        best = capi.Tuning()
        capi.check(capi.lib().ckmpm_autotune(self._h, probe_steps, dt, res, cap, C.byref(n), C.byref(best)),
                   "ckmpm_autotune", self._h)
        return best.as_dict(), [res[i].as_dict() for i in range(min(cap, n.value))]

    def checkpoint_bytes(self) -> int:
        b = C.c_uint64()
        capi.check(capi.lib().ckmpm_checkpoint_bytes(self._h, C.byref(b)), "ckmpm_checkpoint_bytes", self._h)
        return b.value

    def checkpoint_save(self, device_ptr: int) -> None:
        capi.check(capi.lib().ckmpm_checkpoint_save(self._h, C.c_void_p(device_ptr)), "ckmpm_checkpoint_save",
                   self._h)

    def checkpoint_restore(self, device_ptr: int) -> None:
        capi.check(capi.lib().ckmpm_checkpoint_restore(self._h, C.c_void_p(device_ptr)),
                   "ckmpm_checkpoint_restore", self._h)

    def dt_pair(self) -> tuple[float, float]:
        out = (C.c_float * 2)()
        capi.check(capi.lib().ckmpm_get_dt(self._h, out), "ckmpm_get_dt", self._h)
        return out[0], out[1]

    def close(self) -> None:
        if self._h:
            capi.lib().ckmpm_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class MPMEngine:
    """Reference-shaped driver: Initialize -> InitializeParticle -> InitialSetup -> Simulate.

    Mirrors MPMEngine<GridConfig> (include/mpm_engine.cuh:29-974): dt is
    min(config dt, 1/fps) (:178) and shrunk by the initial CFL bound (:109-117);
    Simulate runs frames of substeps.  With a fixed step size every substep
    uses that dt; the first substep after InitialSetup advects with dt = 0, as
    in the reference (:479-480).
    """

    def __init__(self):
        self.scene: Scene | None = None
        self.dt_ = 0.0
        self.config: MPMConfig | None = None

    def Initialize(self, config: MPMConfig) -> None:
        self.config = config
        self.scene = Scene(config)
        self.dt_ = min(config.GetDt(), 1.0 / config.GetFps())

    def InitializeParticle(self, config: MPMConfig, models: Sequence[MPMModel]) -> None:
        assert self.scene is not None, "Initialize first"
        for m in models:
            vmax = float(np.max(np.linalg.norm(m.particle_velocity, axis=1))) if len(m.particle_velocity) else 0.0
            if vmax > 0.0:
                self.dt_ = min(self.dt_, config.GetDx() * config.GetCfl() / vmax)
            self.scene.add_model(m)

    def InitialSetup(self, config: MPMConfig) -> None:
        assert self.scene is not None
        self.scene.setup()

    def ExportParticleToModel(self, export_root: str | Path, frame: int) -> list[Path]:
        """Raw binary export as the reference writes it with exportParticlePositionAsBinary
        (include/mpm_engine.cuh:433-444): float32 xyz triples per model in
        <root>/model_<i>_particle_frame_<frame>.txt."""
        assert self.scene is not None
        root = Path(export_root)
        root.mkdir(parents=True, exist_ok=True)
        out = []
        for i in range(len(self.scene.models)):
            x = self.scene.state(i).x
            f = root / f"model_{i}_particle_frame_{frame}.txt"
            np.ascontiguousarray(x, np.float32).tofile(f)
            out.append(f)
        return out

    def Simulate(self, config: MPMConfig, export_callback=None, fixed_substeps_per_frame: int | None = None,
                 export_root: str | Path | None = None, collect_conservation_metric: bool = False) -> int:
        """Run GetTotalSimulatedFrameCount() frames; returns the substeps taken.

        As the reference's Simulate (include/mpm_engine.cuh:457-909): every
        substep takes nextDt = min(dt_, time left in the frame, dx cfl / max|v|)
        on the device, the first substep advects with 0, and each frame ends
        exactly on its boundary.  With fixed_substeps_per_frame every substep
        uses dt_ instead.  export_callback(frame_index, scene) runs after every
        frame (the reference's ExportParticleToModel point, :880-883).

        collect_conservation_metric records the conservation metric of every
        model before every substep (:573-603), stepping one substep at a time
        (same results, slower): `self.conservation_records[i]` holds rows of 13
        values (time, then the four vectors of Scene.conservation_metric), and
        with export_root they are also written, float32, to
        <root>/conservationMetric_model_<i>.bin as the reference writes them.
        """
        assert self.scene is not None
        start = self.scene.counters()["steps"]
        nmodels = len(self.scene.models)
        if collect_conservation_metric:
            self.conservation_records = [[] for _ in range(nmodels)]

        def record():
            t = self.scene.time()[0]
            for i in range(nmodels):
                self.conservation_records[i].append(np.concatenate([[t], self.scene.conservation_metric(i).ravel()]))

        for frame in range(config.GetTotalSimulatedFrameCount()):
            if config.GetExistRigidParticle():  # the hook is evaluated per frame (mpm_algorithm.cuh:1614)
                self.scene.set_rigid_velocity(config.GetRigidParticleVelocity(frame))
            if not collect_conservation_metric:
                if fixed_substeps_per_frame:
                    self.scene.step(fixed_substeps_per_frame, self.dt_)
                else:
                    self.scene.step_adaptive(1 << 30, self.dt_, config.GetCfl(), 1.0 / config.GetFps())
            elif fixed_substeps_per_frame:
                for _ in range(fixed_substeps_per_frame):
                    record()
                    self.scene.step(1, self.dt_)
            else:
                # One substep per call; frame_time 0 continues the frame the first call opened.
                frame_time = 1.0 / config.GetFps()
                while True:
                    if frame_time == 0.0:
                        t, frame_end = self.scene.time()
                        if not frame_end - t > 0.0:
                            break
                    record()
                    self.scene.step_adaptive(1, self.dt_, config.GetCfl(), frame_time)
                    frame_time = 0.0
            if export_root is not None:
                self.ExportParticleToModel(export_root, frame)
            if export_callback is not None:
                export_callback(frame, self.scene)
        if collect_conservation_metric and export_root is not None:
            root = Path(export_root)
            root.mkdir(parents=True, exist_ok=True)
            for i, rows in enumerate(self.conservation_records):
                np.asarray(rows, np.float32).reshape(-1, 13).tofile(root / f"conservationMetric_model_{i}.bin")
        return self.scene.counters()["steps"] - start


def load_raw_positions(path: str | Path) -> np.ndarray:
    """Particle positions from a raw float32 xyz file (the reference's asset/*.bin format)."""
    a = np.fromfile(path, dtype=np.float32)
    if a.size % 3:
        raise ValueError(f"{path}: {a.size} floats is not a whole number of xyz triples")
    return a.reshape(-1, 3)


def load_scene_json(path: str | Path) -> tuple[MPMConfig, list[MPMModel]]:
    """JSON scene files (a project addition; the reference's importer at
    include/mpm_io.h:168-199 is commented out).  Schema:
      {"config": {MPMConfig fields}, "models": [{"material": {...}, "mass": m,
       "volume": v, "positions": "file.npy" | "file.bin" | [[x,y,z],...], "velocity": [[vx,vy,vz]]}],
       "boundary_rules": [{"slip_walls": width} | {"sticky_walls": width} | {"fixed_box": [lo, hi]} |
                          {"velocity_box": [lo, hi, velocity]} |
                          {"rotating_box": [lo, hi, center, axis, factor]} |
                          {"separate_below": [cell_y, normal]}, ...]}
    A ".bin" file is raw float32 xyz triples, the reference's asset format
    (asset/*.bin, read by the scenes' SetupModel, e.g.
    tests/sand_armadillo/test_sand_armadillo.cuh:137-192).  boundary_rules
    (with config "boundary": "field") build the per-cell boundary with
    ckmpm_b200.boundary.BoundaryField, applying the rules in order.  A material
    gives MPMMaterial's fields, or "E" and "nu" for lambda_ and mu_
    (ComputeLameParameters, include/mpm_material.cuh:277-283).
    """
    path = Path(path)
    spec = json.loads(path.read_text())
    cfgd = dict(spec["config"])
    if "domain_blocks" in cfgd:
        cfgd["domain_blocks"] = tuple(cfgd["domain_blocks"])
    cfg = MPMConfig(**cfgd)
    if spec.get("boundary_rules"):
        from .boundary import BoundaryField
        if cfg.boundary != "field":
            raise ValueError('boundary_rules need config "boundary": "field"')
        bf = BoundaryField(cfg)
        for rule in spec["boundary_rules"]:
            (name, args), = rule.items()
            if name not in ("slip_walls", "sticky_walls", "fixed_box", "velocity_box", "rotating_box",
                            "separate_below"):
                raise ValueError(f"unknown boundary rule {name!r}")
            getattr(bf, name)(*(args if isinstance(args, list) else [args]))
        cfg.boundary_field = bf.arrays()
    models = []
    for md in spec["models"]:
        matd = dict(md["material"])
        if "E" in matd:  # Young's modulus and Poisson ratio, as the reference's scenes give them
            lam, mu = compute_lame_parameters(matd.pop("E"), matd.pop("nu"))
            matd.setdefault("lambda_", lam)
            matd.setdefault("mu_", mu)
        mat = MPMMaterial(**matd)
        pos = md["positions"]
        if isinstance(pos, str):
            pos = load_raw_positions(path.parent / pos) if pos.endswith(".bin") else np.load(path.parent / pos)
        models.append(MPMModel(md["mass"], md["volume"], np.asarray(pos, np.float32),
                               np.asarray(md.get("velocity", [[0, 0, 0]]), np.float32), mat,
                               md.get("freeze_time", 0.0)))
    return cfg, models
