"""Python host mirror of BirdFlowSimulation over the bfx C ABI.

``Lattice`` is a thin owner of one ``bfx_sim`` handle, configured with the raw
``bfx_config`` fields (lattice units).  ``BirdFlowSimulation`` mirrors the
reference class (Sources/BirdFlowMetal/BirdFlowSimulation.swift:410-2096):
same construction from a ``SimulationConfiguration`` + ``BirdParameters`` +
``BirdBodyState``, same ``advance(steps, batch_size, field_capture,
record_run_samples)`` semantics and the same error kinds (``BirdFlowError``).
"""
from __future__ import annotations

import ctypes as ct
import math
from dataclasses import dataclass, field

import numpy as np

from . import _lib as L
from .config import BirdBodyState, BirdParameters, SimulationConfiguration


class BirdFlowError(RuntimeError):
    """BirdFlowError (Sources/BirdFlowMetal/BirdFlowError.swift:3-55) with the C status code."""

    def __init__(self, status: int, message: str):
        super().__init__(f"{L.STATUS_NAMES.get(status, status)}: {message}")
        self.status = status
        self.kind = L.STATUS_NAMES.get(status, str(status))


def _check(status: int, handle=None):
    if status != L.BFX_OK:
        raise BirdFlowError(status, L.last_error(handle))


def _fp(a):
    return a.ctypes.data_as(ct.POINTER(ct.c_float))


@dataclass
class AdvanceResult:
    """AdvanceResult (Sources/BirdFlowMetal/GPUFieldObservation.swift:90-108)."""
    run_samples: list = field(default_factory=list)
    field_frame_published: bool = False
    dropped_field_frame_count: int = 0
    runtime_safety: dict | None = None


def _capture_mode(mode) -> int:
    """FieldCaptureMode (GPUFieldObservation.swift:4-13) by name, or a bool
    (True: required, False: disabled)."""
    if isinstance(mode, bool):
        return L.FIELD_CAPTURE_REQUIRED if mode else L.FIELD_CAPTURE_DISABLED
    if mode in L.FIELD_CAPTURE_MODES:
        return L.FIELD_CAPTURE_MODES[mode]
    raise ValueError(f"unknown field capture mode {mode!r}")


class _DeviceArray:
    """__cuda_array_interface__ over a leased slot's device memory, so torch
    (torch.as_tensor(view, device="cuda")) reads it without a copy."""

    def __init__(self, ptr: int, shape, typestr: str = "<f4"):
        self.__cuda_array_interface__ = {"shape": tuple(shape), "typestr": typestr, "data": (int(ptr), False),
                                         "version": 3, "strides": None}


class FieldFrameLease:
    """GPUFieldFrameLease (GPUFieldObservation.swift:205-262): a read-only
    view of one published field frame.  The slot stays out of the capture
    rotation until the lease is released (explicitly, on leaving a ``with``
    block, after a CUDA stream's work completes, or when the object is
    collected)."""

    def __init__(self, lattice: "Lattice", frame: L.FieldFrame, metadata: dict):
        self._lattice = lattice
        self._frame = frame
        self.lease = int(frame.lease)
        self.metadata = metadata

    @property
    def step(self) -> int:
        return int(self._frame.snapshot.step)

    def copy(self):
        """(density[n], velocity[n, 3]) in lattice units, copied to the host."""
        n = self._lattice.n
        rho = np.empty(n, np.float32)
        vel = np.empty(3 * n, np.float32)
        _check(self._lattice.lib.bfx_field_frame_copy(self._lattice.handle, self.lease, _fp(rho), _fp(vel), n),
               self._lattice.handle)
        return rho, vel.reshape(-1, 3)

    def flow_diagnostics(self):
        """deriveFlowDiagnostics (Visualization.metal:270-308) of this frame:
        (vorticity[n, 4] = curl xyz and |curl| in 1/s, q[n] in 1/s^2, valid[n])."""
        n = self._lattice.n
        vort = np.empty((n, 4), np.float32)
        q = np.empty(n, np.float32)
        valid = np.empty(n, np.uint8)
        _check(self._lattice.lib.bfx_flow_diagnostics(self._lattice.handle, self.lease, vort.ctypes.data,
                                                      q.ctypes.data, valid.ctypes.data, n, 0), self._lattice.handle)
        return vort, q, valid

    def device_views(self):
        """bindMacroscopicFields: (density[nz, ny, nx], velocity[nz, ny, nx, 4])
        as __cuda_array_interface__ objects over the slot.  Read only by
        contract: nothing may write through them."""
        c = self._lattice.config
        return (_DeviceArray(self._frame.density, (c.nz, c.ny, c.nx)),
                _DeviceArray(self._frame.velocity, (c.nz, c.ny, c.nx, 4)))

    def release(self):
        """releaseImmediately (GPUFieldObservation.swift:247-249); releasing twice is a no-op."""
        if self.lease and self._lattice.handle:
            self._lattice.lib.bfx_release_field_frame(self._lattice.handle, self.lease)
        self.lease = 0

    def release_after(self, stream=None):
        """releaseAfterCompletion(of:) (GPUFieldObservation.swift:241-245): the
        slot is released once the work queued so far on ``stream`` (a
        torch.cuda.Stream, a raw cudaStream_t, or None for the simulation's
        own stream) has completed."""
        if not self.lease:
            return
        raw = getattr(stream, "cuda_stream", stream)
        _check(self._lattice.lib.bfx_release_field_frame_after(self._lattice.handle, self.lease,
                                                               ct.c_void_p(raw) if raw else None),
               self._lattice.handle)
        self.lease = 0

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.release()

    def __del__(self):
        try:
            self.release()
        except Exception:
            pass


def default_config(nx: int, ny: int, nz: int, **kw) -> L.Config:
    c = L.Config()
    c.nx, c.ny, c.nz = nx, ny, nz
    c.device = 0
    c.cell_size = 1.0
    c.time_step = 1.0
    c.velocity_to_lattice = 1.0
    c.force_to_physical = 1.0
    c.omega_plus = c.omega_minus = 1.0
    c.sponge_width = 4.0
    c.far_field[:] = [0.0, 0.0, 0.0, 1.0]
    c.body_substeps = 1
    c.accumulate_loads = 1
    c.force_estimator = 6
    for k, v in kw.items():
        cur = getattr(c, k)
        if isinstance(cur, ct.Array):
            if isinstance(v, (list, tuple)) and len(v) and isinstance(v[0], (list, tuple)):
                for i, row in enumerate(v):
                    cur[i][:] = list(row)
            else:
                cur[:] = list(v)
        else:
            setattr(c, k, v)
    return c


def bird_struct(rows) -> L.Bird:
    b = L.Bird()
    for name, row in zip(L.BIRD_FIELDS, rows):
        getattr(b, name).v[:] = [float(x) for x in row]
    return b


def body_struct(state: BirdBodyState | None) -> L.BodyState:
    s = L.BodyState()
    if state is None:
        s.orientation[:] = [0.0, 0.0, 0.0, 1.0]
        return s
    s.position[:] = list(state.position_meters)
    s.orientation[:] = list(state.orientation_body_to_world)
    s.velocity[:] = list(state.linear_velocity_meters_per_second)
    s.omega_body[:] = list(state.angular_velocity_body_radians_per_second)
    return s


class Lattice:
    """One simulation handle on the GPU (bfx_create / bfx_destroy)."""

    def __init__(self, config: L.Config, bird: L.Bird | None = None, body: L.BodyState | None = None,
                 mesh: dict | None = None, wing: L.FlappingWing | None = None):
        """bird / body / mesh: bfx_create; wing (with geometry
        GEOMETRY_FLAPPING_WING): bfx_create_flapping_wing, the prescribed wing of
        MetalFlappingWingValidator held at its root."""
        self.lib = L.load()
        self.config = config
        self.bird = bird
        self.wing = wing
        self.n = int(config.nx) * int(config.ny) * int(config.nz)
        self._mesh_keep = None
        if wing is not None:
            handle = ct.c_void_p()
            _check(self.lib.bfx_create_flapping_wing(ct.byref(config), ct.byref(wing), ct.byref(handle)), None)
            self.handle = handle
            return
        mesh_ptr = None
        if mesh is not None:
            local = np.ascontiguousarray(mesh["local"], np.float32)
            seg = np.ascontiguousarray(mesh["segment"], np.uint8)
            tris = np.ascontiguousarray(mesh["tris"], np.uint32)
            parts = np.ascontiguousarray(mesh["tri_part"], np.uint8)
            self._mesh_keep = (local, seg, tris, parts)
            m = L.Mesh()
            m.local_vertices = local.ctypes.data_as(ct.POINTER(ct.c_float))
            m.vertex_segment = seg.ctypes.data_as(ct.POINTER(ct.c_uint8))
            m.vertex_count = local.shape[0]
            m.triangles = tris.ctypes.data_as(ct.POINTER(ct.c_uint32))
            m.triangle_part = parts.ctypes.data_as(ct.POINTER(ct.c_uint8))
            m.triangle_count = tris.shape[0]
            joints = mesh.get("joints") or []
            if joints:
                arr = (L.Joint * len(joints))()
                for j, d in enumerate(joints):
                    arr[j].origin[:] = [float(v) for v in d["origin"]]
                    arr[j].axis[:] = [float(v) for v in d["axis"]]
                    arr[j].bias, arr[j].amplitude, arr[j].phase = d["bias"], d["amplitude"], d["phase"]
                m.joint_count = len(joints)
                m.joints = arr
                self._mesh_joints = arr
            if mesh.get("kf_times") is not None:
                # keyframe replay: times (s) and frames x vertices x 3 body-frame offsets (m)
                kt = np.ascontiguousarray(mesh["kf_times"], np.float32)
                kp = np.ascontiguousarray(mesh["kf_points"], np.float32)
                m.keyframe_count = kt.shape[0]
                m.keyframe_times = kt.ctypes.data_as(ct.POINTER(ct.c_float))
                m.keyframe_points = kp.ctypes.data_as(ct.POINTER(ct.c_float))
                self._mesh_keyframes = (kt, kp)
            mesh_ptr = ct.byref(m)
            self._mesh_struct = m
        handle = ct.c_void_p()
        st = self.lib.bfx_create(ct.byref(config), ct.byref(bird) if bird is not None else None,
                                 ct.byref(body) if body is not None else None, mesh_ptr, ct.byref(handle))
        _check(st, None)
        self.handle = handle

    def close(self):
        if getattr(self, "handle", None):
            self.lib.bfx_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- stepping ---------------------------------------------------------
    def advance(self, steps: int, batch_size: int = 32, capture_fields=False, record_samples: bool = False):
        """capture_fields: a FieldCaptureMode name ("required", "bestEffort",
        "disabled") or a bool (True: required)."""
        mode = _capture_mode(capture_fields)
        flags = ({L.FIELD_CAPTURE_REQUIRED: L.ADVANCE_CAPTURE_FIELDS,
                  L.FIELD_CAPTURE_BEST_EFFORT: L.ADVANCE_CAPTURE_BEST_EFFORT}.get(mode, 0) |
                 (L.ADVANCE_RECORD_SAMPLES if record_samples else 0))
        samples = (L.RunSample * max(steps, 1))() if record_samples else None
        res = L.AdvanceResult()
        st = self.lib.bfx_advance(self.handle, steps, batch_size, flags, samples, steps if record_samples else 0,
                                  ct.byref(res))
        _check(st, self.handle)
        return res, samples

    # -- read-back ----------------------------------------------------------
    def populations(self) -> np.ndarray:
        out = np.empty(19 * self.n, np.float32)
        _check(self.lib.bfx_copy_populations(self.handle, _fp(out), out.size), self.handle)
        return out.reshape(19, self.config.nz, self.config.ny, self.config.nx)

    def set_populations(self, pops: np.ndarray):
        a = np.ascontiguousarray(pops, np.float32).ravel()
        _check(self.lib.bfx_set_populations(self.handle, _fp(a), a.size), self.handle)

    def fields(self):
        rho = np.empty(self.n, np.float32)
        vel = np.empty(3 * self.n, np.float32)
        _check(self.lib.bfx_copy_fields(self.handle, _fp(rho), _fp(vel), self.n), self.handle)
        return rho, vel.reshape(-1, 3)

    # -- field observation (BirdFlowSimulation.swift:1148-1210, 1806-1918) ----
    def set_observation_buffers(self, count: int, wait_limit_ms: int = 0):
        _check(self.lib.bfx_set_observation_buffers(self.handle, count, wait_limit_ms), self.handle)

    def acquire_field_frame(self, after_step: int | None = None) -> FieldFrameLease | None:
        frame = L.FieldFrame()
        _check(self.lib.bfx_acquire_field_frame(self.handle, int(after_step is not None), after_step or 0,
                                                ct.byref(frame)), self.handle)
        if frame.lease == 0:
            return None
        meta = {
            "step": int(frame.snapshot.step), "time_seconds": float(frame.snapshot.time),
            "body": frame.snapshot.body, "aerodynamic_load": frame.snapshot.loads,
            "grid": tuple(frame.grid), "slot": int(frame.slot), "domain_origin_meters": tuple(frame.domain_origin),
            "cell_size_meters": float(frame.cell_size), "velocity_to_physical": float(frame.velocity_to_physical),
            "geometry": {name: tuple(getattr(frame.geometry, name)) for name in L.GEOMETRY_FRAME_FIELDS},
            "publication_uptime_seconds": float(frame.publication_uptime_seconds),
        }
        return FieldFrameLease(self, frame, meta)

    def capture_current_fields(self, mode="required") -> bool:
        published = ct.c_uint32(0)
        _check(self.lib.bfx_capture_current_fields(self.handle, _capture_mode(mode), ct.byref(published)),
               self.handle)
        return bool(published.value)

    def observation_counters(self):
        """(droppedFieldFrameCount, fieldCaptureWaitCount)."""
        d, w = ct.c_uint64(0), ct.c_uint64(0)
        _check(self.lib.bfx_observation_counters(self.handle, ct.byref(d), ct.byref(w)), self.handle)
        return int(d.value), int(w.value)

    def mask(self) -> np.ndarray:
        out = np.empty(self.n, np.uint8)
        _check(self.lib.bfx_copy_mask(self.handle, out.ctypes.data_as(ct.POINTER(ct.c_uint8)), self.n), self.handle)
        return out

    def wall(self) -> np.ndarray:
        out = np.empty(4 * self.n, np.float32)
        _check(self.lib.bfx_copy_wall(self.handle, _fp(out), self.n), self.handle)
        return out.reshape(-1, 4)

    def links(self):
        count = ct.c_size_t()
        _check(self.lib.bfx_copy_links(self.handle, None, None, None, 0, ct.byref(count)), self.handle)
        n = count.value
        cell = np.empty(max(n, 1), np.uint32)
        d = np.empty(max(n, 1), np.uint8)
        q = np.empty(max(n, 1), np.float32)
        _check(self.lib.bfx_copy_links(self.handle, cell.ctypes.data_as(ct.POINTER(ct.c_uint32)),
                                       d.ctypes.data_as(ct.POINTER(ct.c_uint8)), _fp(q), n, ct.byref(count)),
               self.handle)
        return cell[:n], d[:n], q[:n]

    def loads(self) -> L.Loads:
        out = L.Loads()
        _check(self.lib.bfx_last_loads(self.handle, ct.byref(out)), self.handle)
        return out

    def snapshot(self) -> L.Snapshot:
        out = L.Snapshot()
        _check(self.lib.bfx_snapshot(self.handle, ct.byref(out)), self.handle)
        return out

    def safety(self) -> L.SafetyRecord:
        out = L.SafetyRecord()
        _check(self.lib.bfx_runtime_safety(self.handle, ct.byref(out)), self.handle)
        return out

    def body(self) -> L.BodyState:
        out = L.BodyState()
        _check(self.lib.bfx_get_body(self.handle, ct.byref(out)), self.handle)
        return out

    def set_body(self, body: L.BodyState):
        _check(self.lib.bfx_set_body(self.handle, ct.byref(body)), self.handle)

    def mass_momentum(self) -> np.ndarray:
        out = np.zeros(4, np.float64)
        _check(self.lib.bfx_fluid_mass_momentum(self.handle, out.ctypes.data_as(ct.POINTER(ct.c_double))), self.handle)
        return out

    def step_index(self):
        step = ct.c_uint64()
        t = ct.c_double()
        _check(self.lib.bfx_step_index(self.handle, ct.byref(step), ct.byref(t)), self.handle)
        return step.value, t.value

    def save_state(self) -> bytes:
        size = ct.c_size_t()
        _check(self.lib.bfx_save_state(self.handle, None, 0, ct.byref(size)), self.handle)
        buf = ct.create_string_buffer(size.value)
        _check(self.lib.bfx_save_state(self.handle, buf, size.value, ct.byref(size)), self.handle)
        return buf.raw

    def restore_state(self, data: bytes):
        buf = ct.create_string_buffer(data, len(data))
        _check(self.lib.bfx_restore_state(self.handle, buf, len(data)), self.handle)

    def advance_ledger(self, steps: int):
        """Advances `steps` steps one at a time with the coupled momentum
        ledger (bfx_advance_ledger): one L.LedgerSample per step, impulses in
        kg m / s.  A safety violation raises after the samples written so far
        are kept in ``self.last_ledger``."""
        samples = (L.LedgerSample * max(steps, 1))()
        done = ct.c_uint64()
        st = self.lib.bfx_advance_ledger(self.handle, steps, samples, max(steps, 1), ct.byref(done))
        self.last_ledger = [samples[i] for i in range(done.value)]
        _check(st, self.handle)
        return self.last_ledger

    def save_archive(self, destination: str, extra: dict | None = None):
        """Writes a checkpoint archive (bfx.checkpoint): the canonical FP32
        populations, the current solid mask and the exact restart state, with
        their SHA-256 digests, configuration, bird, step, time, body and loads
        in the manifest.  `extra` adds manifest entries."""
        from . import checkpoint as C
        step, time = self.step_index()
        manifest = {"configuration": C.struct_dict(self.config),
                    "bird": C.struct_dict(self.bird) if self.bird is not None else None,
                    "step": int(step), "timeSeconds": float(time), "body": C.struct_dict(self.body()),
                    "load": C.struct_dict(self.loads())}
        if extra:
            manifest.update(extra)
        files = {C.POPULATIONS: self.populations().tobytes(), C.SOLID_MASK: self.mask().tobytes(),
                 C.RESTART_STATE: self.save_state()}
        C.write_archive(destination, manifest, files)

    @classmethod
    def from_archive(cls, source: str, mesh=None) -> "Lattice":
        """init(checkpointURL:observationBufferCount:) (BirdFlowSimulation.swift:661-672):
        a new simulation built from an archive's configuration, bird and body
        and restored to its exact state.  A mesh configuration needs its mesh,
        which the archive does not hold."""
        from . import checkpoint as C
        manifest, _ = C.read_archive(source)
        cfg = C.struct_from_dict(L.Config, manifest["configuration"])
        bird = C.struct_from_dict(L.Bird, manifest["bird"]) if manifest.get("bird") else None
        body = C.struct_from_dict(L.BodyState, manifest["body"]) if manifest.get("body") else None
        if cfg.geometry == L.GEOMETRY_MESH and mesh is None:
            raise C.CheckpointError("a mesh configuration needs its mesh (meshes are not archived)")
        lat = cls(cfg, bird, body, mesh)
        try:
            lat.restore_archive(source)
        except BaseException:
            lat.close()  # the handle and its device memory are not leaked on a refused archive
            raise
        return lat

    def restore_archive(self, source: str) -> dict:
        """Restores a checkpoint archive written by save_archive after checking
        every digest; the restored populations must equal the archive's
        populations file byte for byte.  Returns the manifest."""
        from . import checkpoint as C
        manifest, files = C.read_archive(source)
        self.restore_state(files[C.RESTART_STATE])
        if self.populations().tobytes() != files[C.POPULATIONS]:
            raise C.CheckpointError("populations file does not match the restart state")
        if self.mask().tobytes() != files[C.SOLID_MASK]:
            raise C.CheckpointError("solid-mask file does not match the restart state")
        return manifest

    def replay_topology(self, mode: int, device_masks_ptr: int = 0, capacity_steps: int = 0):
        """bfx_test_replay_topology: 1 records each following step's occupancy
        into the device buffer at device_masks_ptr (capacity_steps x n bytes), 2
        replays a recording, 0 turns the hook off."""
        _check(self.lib.bfx_test_replay_topology(self.handle, int(mode), ct.c_void_p(int(device_masks_ptr) or None),
                                                 int(capacity_steps)), self.handle)

    def adjoint(self, steps: int, force_weight=(0.0, 0.0, 0.0), power_weight: float = 0.0, window=None,
                checkpoint_interval: int = 0) -> L.AdjointResult:
        """Advances `steps` steps and runs the discrete adjoint backward
        (bfx_adjoint).  The result holds J (the window mean of
        force_weight . F + power_weight * P) and dJ/dtheta for
        theta = (stroke amplitude, pitch amplitude, pitch phase, deviation
        amplitude)."""
        obj = L.AdjointObjective()
        for k in range(3):
            obj.force_weight[k] = float(force_weight[k])
        obj.power_weight = float(power_weight)
        if window is not None:
            obj.window_first, obj.window_last = int(window[0]), int(window[1])
        res = L.AdjointResult()
        _check(self.lib.bfx_adjoint(self.handle, int(steps), ct.byref(obj), int(checkpoint_interval), ct.byref(res)),
               self.handle)
        return res

    def set_kernel_timing(self, enabled: bool):
        _check(self.lib.bfx_set_kernel_timing(self.handle, int(enabled)), self.handle)

    def kernel_timing(self):
        ms = ct.c_double()
        n = ct.c_uint64()
        _check(self.lib.bfx_kernel_timing(self.handle, ct.byref(ms), ct.byref(n)), self.handle)
        return ms.value, n.value

    def timer_begin(self):
        _check(self.lib.bfx_timer_begin(self.handle), self.handle)

    def timer_end(self) -> float:
        ms = ct.c_double()
        _check(self.lib.bfx_timer_end(self.handle, ct.byref(ms)), self.handle)
        return ms.value

    def launch_count(self) -> int:
        n = ct.c_uint64()
        _check(self.lib.bfx_launch_count(self.handle, ct.byref(n)), self.handle)
        return n.value

    def device_bytes(self) -> int:
        n = ct.c_uint64()
        _check(self.lib.bfx_device_bytes(self.handle, ct.byref(n)), self.handle)
        return n.value


class BirdFlowSimulation:
    """BirdFlowSimulation (BirdFlowSimulation.swift:410-2096) on the CUDA backend.

    Production defaults of the reference: analytic bird geometry, halfway
    moving bounce-back, TRT collision, estimator 6, far-field + sponge faces.
    ``storage``, ``collision``, ``wall_rule`` expose the typed operator
    selection that the reference overloads onto caseParameters.w.
    """

    def __init__(self, configuration: SimulationConfiguration, bird: BirdParameters,
                 initial_body_state: BirdBodyState, observation_buffer_count: int = 1, *, storage: int = L.STORAGE_F32,
                 collision: int = L.COLLISION_TRT, device: int = 0, field_wait_limit_ms: int = 0):
        if not 1 <= observation_buffer_count <= 4:
            raise BirdFlowError(8,
                                f"invalidObservationBufferCount({observation_buffer_count})")
        bird.validate(configuration)
        self.configuration = configuration
        self.bird = bird
        sc = configuration.scaling
        far = configuration.far_field_velocity_meters_per_second
        v2l = sc.velocity_to_lattice
        cfg = default_config(
            configuration.grid.x, configuration.grid.y, configuration.grid.z,
            device=device, origin=configuration.domain_origin_meters, cell_size=sc.cell_size_meters,
            time_step=sc.time_step_seconds, velocity_to_lattice=v2l, force_to_physical=sc.force_to_physical,
            omega_plus=sc.omega_plus, omega_minus=sc.omega_minus, sponge_strength=configuration.sponge_strength,
            sponge_width=float(configuration.sponge_width_cells),
            far_field=[float(np.float32(far[0]) * np.float32(v2l)), float(np.float32(far[1]) * np.float32(v2l)),
                       float(np.float32(far[2]) * np.float32(v2l)), 1.0],
            gravity=configuration.gravity_meters_per_second_squared, body_substeps=configuration.body_substeps,
            collision=collision, wall_rule=L.WALL_HALFWAY, storage=storage, geometry=L.GEOMETRY_BIRD,
            free_flight=int(configuration.free_flight), accumulate_loads=1)
        self.lattice = Lattice(cfg, bird_struct(bird.packed()), body_struct(initial_body_state))
        if observation_buffer_count != 1 or field_wait_limit_ms:
            self.lattice.set_observation_buffers(observation_buffer_count, field_wait_limit_ms)
        self.step_index = 0
        self.time_seconds = 0.0

    def advance(self, steps: int, batch_size: int = 32, field_capture: str = "required",
                record_run_samples: bool = False) -> AdvanceResult:
        if steps < 0 or batch_size <= 0:
            raise BirdFlowError(3, f"invalid advance request steps={steps} batchSize={batch_size}")
        mode = _capture_mode(field_capture)
        if steps == 0:
            return AdvanceResult(dropped_field_frame_count=self.dropped_field_frame_count,
                                 runtime_safety=self.runtime_safety_report() if self.configuration.free_flight else None)
        res, samples = self.lattice.advance(steps, batch_size, field_capture, record_run_samples)
        self.step_index, self.time_seconds = self.lattice.step_index()
        out = AdvanceResult(field_frame_published=bool(res.field_frame_published),
                            dropped_field_frame_count=int(res.dropped_field_frames))
        if record_run_samples:
            out.run_samples = [samples[i] for i in range(steps)]
        if self.configuration.free_flight:
            out.runtime_safety = self.runtime_safety_report()
        return out

    def snapshot(self):
        return self.lattice.snapshot()

    def copy_macroscopic_fields(self):
        """copyMacroscopicFields (BirdFlowSimulation.swift:1107-1130): density
        and velocity in m/s (lattice velocity x velocityToPhysical) of the
        newest published frame."""
        rho, vel = self.lattice.fields()
        return rho, (vel * np.float32(self.configuration.scaling.velocity_to_physical)).astype(np.float32)

    def copy_gauge_pressure_field_pascals(self):
        rho, _ = self.lattice.fields()
        sc = self.configuration.scaling
        return (np.float32(1.0 / 3.0) * (rho - np.float32(1.0)) * np.float32(sc.pressure_scale_pascals)).astype(np.float32)

    def acquire_latest_gpu_field_frame(self, after_step: int | None = None) -> FieldFrameLease | None:
        """acquireLatestGPUFieldFrame(afterStep:) (BirdFlowSimulation.swift:1145-1171)
        with the GPUFieldFrameMetadata scales (GPUFieldObservation.swift:162-203)."""
        lease = self.lattice.acquire_field_frame(after_step)
        if lease is not None:
            sc = self.configuration.scaling
            v2p = np.float32(sc.velocity_to_physical)
            lease.metadata.update(
                velocity_to_physical=float(v2p),
                pressure_scale_pascals=float(np.float32(sc.pressure_scale_pascals)),
                reference_dynamic_pressure_pascals=float(
                    np.float32(0.5) * np.float32(self.configuration.physical_air_density) *
                    (np.float32(sc.lattice_reference_speed) * v2p) ** 2),
                physical_air_density=float(np.float32(self.configuration.physical_air_density)),
                bird=self.bird)
        return lease

    def capture_current_macroscopic_field(self, mode: str = "required") -> bool:
        """captureCurrentMacroscopicField(mode:) (BirdFlowSimulation.swift:1173-1210)."""
        return self.lattice.capture_current_fields(mode)

    @property
    def dropped_field_frame_count(self) -> int:
        return self.lattice.observation_counters()[0]

    @property
    def field_capture_wait_count(self) -> int:
        return self.lattice.observation_counters()[1]

    def runtime_safety_report(self) -> dict:
        r = self.lattice.safety()
        return {"maximum_mach": r.metrics[0], "minimum_clearance_meters": r.metrics[1],
                "first_violation_step": (r.event[1] << 32) | r.event[0] if r.event[2] else None,
                "flags": int(r.event[2]), "passed": r.event[2] == 0}

    def save_checkpoint(self) -> bytes:
        return self.lattice.save_state()

    def restore_checkpoint(self, data: bytes):
        self.lattice.restore_state(data)
        self.step_index, self.time_seconds = self.lattice.step_index()

    def advance_with_coupled_momentum_ledger(self, steps: int, maximum_relative_residual: float = 0.005) -> dict:
        """advanceWithCoupledMomentumLedger (BirdFlowSimulation.swift:806-1085):
        steps one at a time recording the total-system linear-momentum
        balance, and gates it: the boundary closure (aerodynamic impulse +
        fluid boundary impulse) and the external-system closure (total
        momentum change - far field - sponge - gravity) must each stay within
        `maximum_relative_residual` in RMS, relative to the RMS aerodynamic
        impulse (and the RMS external impulse for the system closure)."""
        if not self.configuration.free_flight:
            raise BirdFlowError(10, "the total-system ledger requires freeFlight=true")
        if steps <= 0 or not math.isfinite(maximum_relative_residual) or maximum_relative_residual <= 0:
            raise BirdFlowError(3, f"invalid advance request steps={steps} batchSize=1")
        samples = self.lattice.advance_ledger(steps)
        self.step_index, self.time_seconds = self.lattice.step_index()
        return ledger_report(samples, self.configuration.scaling.time_step_seconds, maximum_relative_residual)

    def save_checkpoint_archive(self, destination: str):
        """CheckpointArchive.write (CheckpointArchive.swift:45-80): a directory
        with manifest.json, the populations, the solid mask and the exact
        restart state, each with its SHA-256 digest (bfx.checkpoint)."""
        self.lattice.save_archive(destination)

    def restore_checkpoint_archive(self, source: str):
        """CheckpointArchive.read (CheckpointArchive.swift:82-110): verifies the
        schema, sizes and digests, then restores."""
        manifest = self.lattice.restore_archive(source)
        self.step_index, self.time_seconds = self.lattice.step_index()
        return manifest

    def close(self):
        self.lattice.close()


def ledger_report(samples, time_step_seconds: float, maximum_relative_residual: float = 0.005) -> dict:
    """CoupledMomentumLedgerReport (CoupledMomentumLedger.swift:36-60) from
    ledger samples: RMS and maximum residuals, their relative values and the
    verdict of the two closure gates."""
    rows = []
    for s in samples:
        d = {"step": int(s.step), "time_seconds": float(s.time)}
        for n in L.LEDGER_VECTORS:
            d[n] = [float(v) for v in getattr(s, n)]
        for n in L.LEDGER_COUNTS:
            d[n] = int(getattr(s, n))
        rows.append(d)

    def rms(key):
        return math.sqrt(sum(sum(v * v for v in r[key]) for r in rows) / len(rows)) if rows else 0.0

    def maximum(key):
        return max((math.sqrt(sum(v * v for v in r[key])) for r in rows), default=0.0)

    aero, external = rms("aerodynamic_impulse"), rms("external_impulse")
    boundary, system = rms("boundary_residual"), rms("system_residual")
    rel_boundary = boundary / max(aero, 1.0e-30)
    rel_system = system / max(max(aero, external), 1.0e-30)
    finite = all(math.isfinite(v) for r in rows for n in L.LEDGER_VECTORS for v in r[n])
    passed = bool(rows) and finite and rel_boundary <= maximum_relative_residual and rel_system <= maximum_relative_residual
    return {
        "schema_version": 1, "steps": len(rows), "time_step_seconds": time_step_seconds,
        "momentum_definition": "direct population momentum + whole-bird translational momentum + prescribed-wing "
                               "momentum relative to the registered body frame; external impulse = open far field + "
                               "sponge + gravity",
        "topology_definition": "fluid boundary impulse minus the persistent-link exchange reconstructed from the "
                               "pre-step populations; the remainder includes cover / uncover conversion",
        "samples": rows, "rms_aerodynamic_impulse": aero, "rms_external_impulse": external,
        "rms_boundary_closure_residual": boundary, "rms_external_system_closure_residual": system,
        "maximum_boundary_closure_residual": maximum("boundary_residual"),
        "maximum_external_system_closure_residual": maximum("system_residual"),
        "relative_rms_boundary_closure_residual": rel_boundary,
        "relative_rms_external_system_closure_residual": rel_system,
        "maximum_allowed_relative_rms_residual": maximum_relative_residual,
        "finite": finite, "passed": passed,
        "scientific_verdict": "coupled external linear-momentum and fluid/boundary impulse gates passed" if passed
        else "coupled momentum closure failed; do not accept quantitative free-flight loads",
    }

