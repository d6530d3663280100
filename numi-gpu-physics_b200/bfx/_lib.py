"""ctypes binding of libbfx.so (include/bfx.h).

The library is the only execution path: if libbfx.so is missing or cannot be
loaded, importing a simulation raises ``BirdFlowError`` — there is no CPU
fallback.  Structures below mirror include/bfx.h field for field; their sizes
are asserted against the C layout in tests/test_abi.py.
"""
from __future__ import annotations

import ctypes as ct
import os

_PKG_DIR = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(_PKG_DIR, "libbfx.so")

BFX_OK = 0
STATUS_NAMES = {
    0: "ok", 1: "deviceUnavailable", 2: "allocationFailed", 3: "invalidAdvanceRequest",
    4: "commandBufferFailed", 5: "runtimeSafetyViolation", 6: "simulationStateInvalidated",
    7: "invalidConfiguration", 8: "invalidArgument", 9: "capacity", 10: "unsupported", 11: "timeout",
}

COLLISION_TRT, COLLISION_TRT_LIMITER, COLLISION_REGULARIZED, COLLISION_RR3 = 0, 1, 2, 3
WALL_HALFWAY, WALL_INTERPOLATED = 0, 1
STORAGE_F32, STORAGE_F16_DEVIATION, STORAGE_BF16_DEVIATION, STORAGE_F64 = 0, 1, 2, 3
BC_FARFIELD, BC_PERIODIC, BC_VELOCITY, BC_OUTFLOW = 0, 1, 2, 3
GEOMETRY_NONE, GEOMETRY_BIRD, GEOMETRY_ELLIPSOID, GEOMETRY_MESH, GEOMETRY_FLAPPING_WING = 0, 1, 2, 3, 4
LINK_LINEAR, LINK_RAY_ROOT = 0, 1
INIT_EQUILIBRIUM, INIT_SHEAR_WAVE_Y, INIT_SHEAR_WAVE_Z = 0, 1, 2
ADVANCE_CAPTURE_FIELDS, ADVANCE_RECORD_SAMPLES, ADVANCE_CAPTURE_BEST_EFFORT = 1, 2, 4
FIELD_CAPTURE_REQUIRED, FIELD_CAPTURE_BEST_EFFORT, FIELD_CAPTURE_DISABLED = 0, 1, 2
FIELD_CAPTURE_MODES = {"required": FIELD_CAPTURE_REQUIRED, "bestEffort": FIELD_CAPTURE_BEST_EFFORT,
                       "disabled": FIELD_CAPTURE_DISABLED}

STORAGE_BYTES = {STORAGE_F32: 4, STORAGE_F16_DEVIATION: 2, STORAGE_BF16_DEVIATION: 2, STORAGE_F64: 8}
STORAGE_NAMES = {STORAGE_F32: "f32", STORAGE_F16_DEVIATION: "f16dev", STORAGE_BF16_DEVIATION: "bf16dev",
                 STORAGE_F64: "f64"}


class Config(ct.Structure):
    _fields_ = [
        ("nx", ct.c_uint32), ("ny", ct.c_uint32), ("nz", ct.c_uint32), ("device", ct.c_int32),
        ("origin", ct.c_float * 3), ("cell_size", ct.c_float),
        ("time_step", ct.c_float), ("velocity_to_lattice", ct.c_float), ("force_to_physical", ct.c_float),
        ("fast_math", ct.c_uint32),
        ("omega_plus", ct.c_float), ("omega_minus", ct.c_float),
        ("sponge_strength", ct.c_float), ("sponge_width", ct.c_float),
        ("far_field", ct.c_float * 4), ("gravity", ct.c_float * 3), ("body_substeps", ct.c_uint32),
        ("face_bc", ct.c_int32 * 6), ("face_velocity", (ct.c_float * 3) * 6),
        ("collision", ct.c_int32), ("wall_rule", ct.c_int32), ("storage", ct.c_int32), ("geometry", ct.c_int32),
        ("link_rule", ct.c_int32), ("force_estimator", ct.c_int32), ("load_component", ct.c_int32),
        ("selected_part", ct.c_int32),
        ("free_flight", ct.c_uint32), ("accumulate_loads", ct.c_uint32),
        ("moving_wall_local_density", ct.c_uint32), ("static_geometry", ct.c_uint32),
        ("init", ct.c_int32), ("link_capacity", ct.c_uint32),
        ("init_amplitude", ct.c_float), ("mesh_half_thickness", ct.c_float),
    ]


class Float4(ct.Structure):
    _fields_ = [("v", ct.c_float * 4)]


BIRD_FIELDS = ("body_radii_mass", "inertia", "wing_geometry0", "wing_geometry1", "tail_geometry",
               "wing_kinematics0", "wing_kinematics1", "safety_geometry", "safety_limits",
               "left_wing_mass_com", "left_wing_inertia", "right_wing_mass_com", "right_wing_inertia")


class Bird(ct.Structure):
    _fields_ = [(name, Float4) for name in BIRD_FIELDS]


class FlappingWing(ct.Structure):
    """bfx_flapping_wing (GPUFlappingWingParameters, GPUData.swift:383-388)."""
    _fields_ = [(name, Float4) for name in ("root_and_chord", "geometry", "kinematics0", "kinematics1")]


class BodyState(ct.Structure):
    _fields_ = [("position", ct.c_double * 3), ("orientation", ct.c_double * 4),
                ("velocity", ct.c_double * 3), ("omega_body", ct.c_double * 3)]


class Joint(ct.Structure):
    _fields_ = [("origin", ct.c_float * 3), ("axis", ct.c_float * 3), ("bias", ct.c_float),
                ("amplitude", ct.c_float), ("phase", ct.c_float), ("_reserved", ct.c_float)]


class Mesh(ct.Structure):
    _fields_ = [("local_vertices", ct.POINTER(ct.c_float)), ("vertex_segment", ct.POINTER(ct.c_uint8)),
                ("vertex_count", ct.c_uint32), ("triangles", ct.POINTER(ct.c_uint32)),
                ("triangle_part", ct.POINTER(ct.c_uint8)), ("triangle_count", ct.c_uint32),
                ("joint_count", ct.c_uint32), ("joints", ct.POINTER(Joint)),
                ("keyframe_count", ct.c_uint32), ("keyframe_times", ct.POINTER(ct.c_float)),
                ("keyframe_points", ct.POINTER(ct.c_float))]


class Loads(ct.Structure):
    _fields_ = [("force", ct.c_double * 3), ("torque", ct.c_double * 3), ("force_lattice", ct.c_double * 3),
                ("limiter_activations", ct.c_double), ("max_restriction", ct.c_double),
                ("link_count", ct.c_int64), ("covered_count", ct.c_int64), ("uncovered_count", ct.c_int64),
                ("power", ct.c_double)]


class RunSample(ct.Structure):
    _fields_ = [("time", ct.c_double), ("position", ct.c_double * 3), ("orientation", ct.c_double * 4),
                ("velocity", ct.c_double * 3), ("omega_body", ct.c_double * 3), ("force", ct.c_double * 3),
                ("torque", ct.c_double * 3), ("left_hinge_force", ct.c_float * 3),
                ("left_hinge_torque", ct.c_float * 3), ("right_hinge_force", ct.c_float * 3),
                ("right_hinge_torque", ct.c_float * 3), ("step", ct.c_uint64)]


class SafetyRecord(ct.Structure):
    _fields_ = [("metrics", ct.c_float * 4), ("event", ct.c_uint32 * 4)]


class Snapshot(ct.Structure):
    _fields_ = [("step", ct.c_uint64), ("time", ct.c_double), ("body", BodyState), ("loads", Loads)]


class AdvanceResult(ct.Structure):
    _fields_ = [("steps_done", ct.c_uint64), ("field_frame_published", ct.c_uint32),
                ("safety_passed", ct.c_uint32), ("safety", SafetyRecord), ("dropped_field_frames", ct.c_uint64)]


GEOMETRY_FRAME_FIELDS = ("body_position", "orientation", "linear_velocity", "omega_body_world", "left_root",
                         "left_chord", "left_span", "left_normal", "left_angular_velocity", "right_root",
                         "right_chord", "right_span", "right_normal", "right_angular_velocity")


class GeometryFrame(ct.Structure):
    _fields_ = [(name, ct.c_float * 4) for name in GEOMETRY_FRAME_FIELDS]


class FieldFrame(ct.Structure):
    _fields_ = [("lease", ct.c_uint64), ("snapshot", Snapshot), ("grid", ct.c_uint32 * 3), ("slot", ct.c_uint32),
                ("domain_origin", ct.c_float * 3), ("cell_size", ct.c_float), ("velocity_to_physical", ct.c_float),
                ("_pad", ct.c_float * 3), ("geometry", GeometryFrame), ("publication_uptime_seconds", ct.c_double),
                ("density", ct.c_void_p), ("velocity", ct.c_void_p)]


class AdjointObjective(ct.Structure):
    _fields_ = [("force_weight", ct.c_double * 3), ("power_weight", ct.c_double),
                ("window_first", ct.c_uint64), ("window_last", ct.c_uint64)]


class AdjointResult(ct.Structure):
    _fields_ = [("objective", ct.c_double), ("gradient", ct.c_double * 4), ("steps", ct.c_uint64),
                ("checkpoint_interval", ct.c_uint32), ("snapshots", ct.c_uint32), ("forward_ms", ct.c_double),
                ("reverse_ms", ct.c_double), ("max_links", ct.c_uint64), ("work_bytes", ct.c_uint64)]


LEDGER_VECTORS = ("fluid_momentum_before", "fluid_momentum_after", "fluid_momentum_change", "body_momentum_before",
                  "body_momentum_after", "wing_momentum_before", "wing_momentum_after", "aerodynamic_impulse",
                  "gravity_impulse", "far_field_impulse", "sponge_impulse", "link_exchange_impulse",
                  "topology_impulse", "fluid_boundary_impulse", "boundary_residual", "total_momentum_change",
                  "external_impulse", "system_residual")
LEDGER_COUNTS = ("far_field_links", "sponge_cells", "boundary_links", "topology_cells")


class LedgerSample(ct.Structure):
    _fields_ = ([("step", ct.c_uint64), ("time", ct.c_double)] + [(n, ct.c_double * 3) for n in LEDGER_VECTORS] +
                [(n, ct.c_uint64) for n in LEDGER_COUNTS])


EXPORTED = (
    "bfx_version", "bfx_abi_version", "bfx_device_count", "bfx_create", "bfx_destroy", "bfx_advance",
    "bfx_snapshot", "bfx_copy_fields", "bfx_copy_gauge_pressure", "bfx_runtime_safety", "bfx_last_loads",
    "bfx_copy_populations", "bfx_set_populations", "bfx_copy_mask", "bfx_copy_wall", "bfx_copy_links",
    "bfx_fluid_mass_momentum", "bfx_save_state", "bfx_restore_state", "bfx_get_body", "bfx_set_body",
    "bfx_step_index", "bfx_set_kernel_timing", "bfx_kernel_timing", "bfx_timer_begin", "bfx_timer_end",
    "bfx_launch_count", "bfx_device_bytes", "bfx_fluid_mass_momentum_noalloc", "bfx_adjoint", "bfx_advance_ledger",
    "bfx_last_error", "bfx_set_observation_buffers", "bfx_acquire_field_frame", "bfx_field_frame_copy",
    "bfx_release_field_frame", "bfx_release_field_frame_after", "bfx_capture_current_fields",
    "bfx_observation_counters", "bfx_flow_diagnostics", "bfx_create_flapping_wing", "bfx_test_stall_staged_kernel",
    "bfx_test_replay_topology",
)

_lib = None


class LibraryMissing(RuntimeError):
    pass


def load(path: str | None = None):
    """Loads libbfx.so (built by numi-gpu-physics_b200/build.py); raises if absent."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise LibraryMissing(f"libbfx.so not found at {p}; run numi-gpu-physics_b200/build.py")
    L = ct.CDLL(p)
    P = ct.POINTER
    vp = ct.c_void_p
    L.bfx_version.restype = ct.c_char_p
    L.bfx_abi_version.restype = ct.c_int
    L.bfx_device_count.argtypes = [P(ct.c_int)]
    L.bfx_create.argtypes = [P(Config), P(Bird), P(BodyState), P(Mesh), P(vp)]
    L.bfx_create_flapping_wing.argtypes = [P(Config), P(FlappingWing), P(vp)]
    L.bfx_test_stall_staged_kernel.argtypes = [vp, ct.c_int32, ct.c_uint32]
    L.bfx_test_replay_topology.argtypes = [vp, ct.c_int, ct.c_void_p, ct.c_uint64]
    L.bfx_destroy.argtypes = [vp]
    L.bfx_destroy.restype = None
    L.bfx_advance.argtypes = [vp, ct.c_uint64, ct.c_uint32, ct.c_uint32, P(RunSample), ct.c_size_t, P(AdvanceResult)]
    L.bfx_snapshot.argtypes = [vp, P(Snapshot)]
    L.bfx_copy_fields.argtypes = [vp, P(ct.c_float), P(ct.c_float), ct.c_size_t]
    L.bfx_copy_gauge_pressure.argtypes = [vp, ct.c_float, P(ct.c_float), ct.c_size_t]
    L.bfx_runtime_safety.argtypes = [vp, P(SafetyRecord)]
    L.bfx_last_loads.argtypes = [vp, P(Loads)]
    L.bfx_copy_populations.argtypes = [vp, P(ct.c_float), ct.c_size_t]
    L.bfx_set_populations.argtypes = [vp, P(ct.c_float), ct.c_size_t]
    L.bfx_copy_mask.argtypes = [vp, P(ct.c_uint8), ct.c_size_t]
    L.bfx_copy_wall.argtypes = [vp, P(ct.c_float), ct.c_size_t]
    L.bfx_copy_links.argtypes = [vp, P(ct.c_uint32), P(ct.c_uint8), P(ct.c_float), ct.c_size_t, P(ct.c_size_t)]
    L.bfx_fluid_mass_momentum.argtypes = [vp, P(ct.c_double)]
    L.bfx_save_state.argtypes = [vp, vp, ct.c_size_t, P(ct.c_size_t)]
    L.bfx_restore_state.argtypes = [vp, vp, ct.c_size_t]
    L.bfx_get_body.argtypes = [vp, P(BodyState)]
    L.bfx_set_body.argtypes = [vp, P(BodyState)]
    L.bfx_step_index.argtypes = [vp, P(ct.c_uint64), P(ct.c_double)]
    L.bfx_set_kernel_timing.argtypes = [vp, ct.c_int]
    L.bfx_kernel_timing.argtypes = [vp, P(ct.c_double), P(ct.c_uint64)]
    L.bfx_timer_begin.argtypes = [vp]
    L.bfx_timer_end.argtypes = [vp, P(ct.c_double)]
    L.bfx_launch_count.argtypes = [vp, P(ct.c_uint64)]
    L.bfx_device_bytes.argtypes = [vp, P(ct.c_uint64)]
    L.bfx_fluid_mass_momentum_noalloc.argtypes = [vp, vp, ct.c_uint32, ct.c_uint32, ct.c_uint32, vp]
    L.bfx_adjoint.argtypes = [vp, ct.c_uint64, P(AdjointObjective), ct.c_uint32, P(AdjointResult)]
    L.bfx_advance_ledger.argtypes = [vp, ct.c_uint64, P(LedgerSample), ct.c_size_t, P(ct.c_uint64)]
    L.bfx_last_error.argtypes = [vp, ct.c_char_p, ct.c_size_t]
    L.bfx_set_observation_buffers.argtypes = [vp, ct.c_uint32, ct.c_uint32]
    L.bfx_acquire_field_frame.argtypes = [vp, ct.c_int, ct.c_uint64, P(FieldFrame)]
    L.bfx_field_frame_copy.argtypes = [vp, ct.c_uint64, P(ct.c_float), P(ct.c_float), ct.c_size_t]
    L.bfx_release_field_frame.argtypes = [vp, ct.c_uint64]
    L.bfx_release_field_frame_after.argtypes = [vp, ct.c_uint64, vp]
    L.bfx_capture_current_fields.argtypes = [vp, ct.c_uint32, P(ct.c_uint32)]
    L.bfx_observation_counters.argtypes = [vp, P(ct.c_uint64), P(ct.c_uint64)]
    L.bfx_flow_diagnostics.argtypes = [vp, ct.c_uint64, vp, vp, vp, ct.c_size_t, ct.c_int]
    if path is None:
        _lib = L
    return L


def last_error(handle=None) -> str:
    buf = ct.create_string_buffer(1024)
    load().bfx_last_error(handle, buf, len(buf))
    return buf.value.decode(errors="replace")
