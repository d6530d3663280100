/*
 * bfx — B200-native D3Q19 lattice-Boltzmann step with moving articulated
 * boundaries.  Plain C ABI (no CUDA or torch types): opaque handle, plain
 * pointers and sizes, integer status codes.
 *
 * This library replaces the Metal execution path of BirdFlowMetal's
 * BirdFlowSimulation (Numi2/numi-gpu-physics,
 * Sources/BirdFlowMetal/BirdFlowSimulation.swift).  Each entry point below
 * names the reference interface it stands in for.  The reference has no plugin
 * protocol: its boundary is the concrete class, and its non-Metal branch
 * (BirdFlowSimulation.swift:2105-2182) is where a Linux backend calls this ABI.
 *
 * Threading: one handle owns one CUDA stream; calls on one handle must be
 * serialised by the caller (the reference class is @unchecked Sendable with
 * caller-serialised calls, BirdFlowSimulation.swift:410-478).  Independent
 * handles may be used from different threads.
 *
 * Errors: every function returns a bfx_status.  After a GPU failure the
 * handle is terminally invalid and later calls return BFX_ERR_INVALIDATED,
 * mirroring BirdFlowSimulation.invalidate (BirdFlowSimulation.swift:2059-2095).
 * bfx_last_error() returns the message of the last failure.
 */
#ifndef BFX_H
#define BFX_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* 2: bfx_mesh keyframe fields, bfx_advance_result.dropped_field_frames,
 * field observation and flow-diagnostics entry points.
 * 3: the prescribed flapping wing (BFX_GEOMETRY_FLAPPING_WING,
 * bfx_flapping_wing, bfx_create_flapping_wing). */
#define BFX_ABI_VERSION 3

#if defined(__GNUC__)
#define BFX_API __attribute__((visibility("default")))
#else
#define BFX_API
#endif

typedef struct bfx_sim bfx_sim;

/* Mirrors BirdFlowError (Sources/BirdFlowMetal/BirdFlowError.swift:3-55) and
 * BirdFlowConfigurationError (Sources/BirdFlowCore/SimulationConfiguration.swift:3-24). */
typedef enum bfx_status {
    BFX_OK = 0,
    BFX_ERR_DEVICE_UNAVAILABLE = 1, /* deviceUnavailable / metalUnavailable */
    BFX_ERR_ALLOCATION = 2,         /* allocationFailed */
    BFX_ERR_INVALID_ADVANCE = 3,    /* invalidAdvanceRequest */
    BFX_ERR_KERNEL = 4,             /* commandBufferFailed */
    BFX_ERR_SAFETY = 5,             /* runtimeSafetyViolation */
    BFX_ERR_INVALIDATED = 6,        /* simulationStateInvalidated */
    BFX_ERR_INVALID_CONFIG = 7,     /* BirdFlowConfigurationError */
    BFX_ERR_INVALID_ARGUMENT = 8,
    BFX_ERR_CAPACITY = 9,           /* caller buffer or link list too small */
    BFX_ERR_UNSUPPORTED = 10,       /* configuration outside the adjoint's scope */
    BFX_ERR_TIMEOUT = 11            /* a required field capture found no free observation slot in time */
} bfx_status;

/* Collision operator.  The reference selects these through caseParameters.w
 * thresholds inside stepFluidTRT (BF.metal:2544-2555, 2906-2912). */
typedef enum bfx_collision {
    BFX_COLLISION_TRT = 0,           /* BF.metal:3063-3093 */
    BFX_COLLISION_TRT_LIMITER = 1,   /* symmetric positivity limiter, BF.metal:3094-3174 */
    BFX_COLLISION_REGULARIZED = 2,   /* projected regularized BGK, BF.metal:2917-3062 */
    BFX_COLLISION_RR3 = 3            /* recursive regularized, third order, BF.metal:2917-3062 */
} bfx_collision;

/* Moving-wall bounce-back rule (BF.metal:2727-2806). */
typedef enum bfx_wall_rule {
    BFX_WALL_HALFWAY = 0,
    BFX_WALL_INTERPOLATED = 1
} bfx_wall_rule;

/* Population storage.  Collision arithmetic is FP32 for the first three and
 * FP64 for BFX_STORAGE_F64 (the reference run for error statements). */
typedef enum bfx_storage {
    BFX_STORAGE_F32 = 0,
    BFX_STORAGE_F16_DEVIATION = 1,   /* f - w_q in IEEE half, scaled by 2^12 */
    BFX_STORAGE_BF16_DEVIATION = 2,  /* f - w_q in bfloat16 */
    BFX_STORAGE_F64 = 3
} bfx_storage;

/* Domain face rule for populations pulled from outside the lattice.
 * FARFIELD is the reference rule (BF.metal:2696-2725); PERIODIC is per axis
 * (both faces of the axis must say so); VELOCITY and OUTFLOW are additions. */
typedef enum bfx_face_bc {
    BFX_BC_FARFIELD = 0,  /* equilibrium(far density, far velocity) */
    BFX_BC_PERIODIC = 1,
    BFX_BC_VELOCITY = 2,  /* equilibrium(far density, face_velocity[face]) */
    BFX_BC_OUTFLOW = 3    /* zero gradient: copy what the interior neighbour receives */
} bfx_face_bc;

typedef enum bfx_geometry_kind {
    BFX_GEOMETRY_NONE = 0,       /* all fluid */
    BFX_GEOMETRY_BIRD = 1,       /* analytic bird: ellipsoid body, tapered wings, tail (BF.metal:816-938) */
    BFX_GEOMETRY_ELLIPSOID = 2,  /* body ellipsoid alone, link fractions by bisection (BF.metal:1144-1175 rule) */
    BFX_GEOMETRY_MESH = 3,       /* articulated triangle mesh (BF.metal:1638-2076) */
    BFX_GEOMETRY_FLAPPING_WING = 4 /* prescribed Li-Nabawy beta-planform wing, link fractions by
                                      10-step bisection (BF.metal:940-1297); see bfx_create_flapping_wing */
} bfx_geometry_kind;

/* Link fraction rule for mesh geometry. */
typedef enum bfx_link_rule {
    BFX_LINK_LINEAR = 0,  /* q = d_f / (d_f - d_s) from signed distances (BF.metal:2044-2076) */
    BFX_LINK_RAY_ROOT = 1 /* bracketed root of the wall distance along the link */
} bfx_link_rule;

typedef enum bfx_init {
    BFX_INIT_EQUILIBRIUM = 0,   /* initializePopulations, BF.metal:2078-2103 */
    BFX_INIT_SHEAR_WAVE_Y = 1,  /* initializeShearWave, BF.metal:2132-2162: u_x = A sin(2 pi y / N_y) */
    BFX_INIT_SHEAR_WAVE_Z = 2   /* same wave along z */
} bfx_init;

/* Simulation parameters: the lattice-unit content of SimulationConfiguration
 * and LatticeScaling (SimulationConfiguration.swift:55-315) as packed into
 * GPUUniforms (Sources/BirdFlowMetal/GPUData.swift:4-80). */
typedef struct bfx_config {
    uint32_t nx, ny, nz;
    int32_t device;                 /* CUDA device ordinal */
    float origin[3];                /* domainOriginMeters */
    float cell_size;                /* cellSizeMeters (dx) */
    float time_step;                /* timeStepSeconds (dt) */
    float velocity_to_lattice;      /* dt/dx */
    float force_to_physical;        /* rho dx^4 / dt^2 */
    uint32_t fast_math;             /* SimulationConfiguration.fastMath: FP32 step with FMA contraction
                                       (not bit-identical to the reference order; 16-bit storage always is) */
    float omega_plus, omega_minus;  /* 1/tau+, 1/tau- */
    float sponge_strength;
    float sponge_width;             /* cells */
    float far_field[4];             /* lattice velocity xyz, density w */
    float gravity[3];               /* m/s^2 */
    uint32_t body_substeps;         /* 1...64 */
    int32_t face_bc[6];             /* bfx_face_bc for -x,+x,-y,+y,-z,+z */
    float face_velocity[6][3];      /* lattice velocity of BFX_BC_VELOCITY faces */
    int32_t collision;              /* bfx_collision */
    int32_t wall_rule;              /* bfx_wall_rule */
    int32_t storage;                /* bfx_storage */
    int32_t geometry;               /* bfx_geometry_kind */
    int32_t link_rule;              /* bfx_link_rule (mesh) */
    int32_t force_estimator;        /* 0..6; 6 = production conservative estimator */
    int32_t load_component;         /* 0 both, 1 link exchange only, 2 topology only */
    int32_t selected_part;          /* 0 = all parts */
    uint32_t free_flight;
    uint32_t accumulate_loads;
    uint32_t moving_wall_local_density; /* integration.y: pre-step local density in the wall term */
    uint32_t static_geometry;       /* geometry does not move: classify and build links once */
    int32_t init;                   /* bfx_init */
    uint32_t link_capacity;         /* 0 = automatic */
    float init_amplitude;           /* shear-wave amplitude (lattice velocity) */
    float mesh_half_thickness;      /* meters */
} bfx_config;

typedef struct bfx_float4 { float v[4]; } bfx_float4;

/* GPUBirdParameters (Sources/BirdFlowMetal/GPUData.swift:82-178), 13 float4. */
typedef struct bfx_bird {
    bfx_float4 body_radii_mass;     /* body radii xyz (m), mass (kg) */
    bfx_float4 inertia;             /* principal inertia xyz */
    bfx_float4 wing_geometry0;      /* span, root chord, tip chord, thickness */
    bfx_float4 wing_geometry1;      /* sweep, root offset xyz */
    bfx_float4 tail_geometry;       /* length, half width, thickness, - */
    bfx_float4 wing_kinematics0;    /* frequency Hz, stroke amplitude, stroke bias, pitch mean */
    bfx_float4 wing_kinematics1;    /* pitch amplitude, pitch phase, deviation amplitude, measured-keyframe flag
                                       (must be 0).  Deviation about the stroke-plane normal is
                                       amplitude * sin(2 * phase); the reference uses this slot for the
                                       keyframe count of measured kinematics, which bfx does not support. */
    bfx_float4 safety_geometry;     /* conservative local half extent xyz, bounding radius */
    bfx_float4 safety_limits;       /* max prescribed wing speed, Mach limit */
    bfx_float4 left_wing_mass_com;  /* mass, centre of mass from hinge (chord, span, normal) */
    bfx_float4 left_wing_inertia;   /* principal inertia xyz, w = 1 when present */
    bfx_float4 right_wing_mass_com;
    bfx_float4 right_wing_inertia;
} bfx_bird;

/* GPUFlappingWingParameters (Sources/BirdFlowMetal/GPUData.swift:383-388): the
 * analytic single wing of MetalFlappingWingValidation (Li and Nabawy's
 * beta-planform benchmark).  Lengths in metres, as the world coordinates; the
 * reference runs this wing with a 1 m cell, i.e. in lattice units
 * (MetalFlappingWingValidation.swift:3333-3367), and the wall velocity is the
 * wing's rotation rate (rad per step) times the distance from the root divided
 * by the cell size.  Angles in radians; the stroke rotates about the world z
 * axis through the root.
 *   root_and_chord  root position xyz (m), mean chord c
 *   geometry        radius R (span), thickness, beta shape - 1, beta normalisation
 *                   (local chord = c * geometry.w * (r (1 - r))^geometry.z at r = radial / R)
 *   kinematics0     cycle steps, stroke half amplitude, stroke acceleration duration,
 *                   pitch flip duration (the durations as cycle fractions, below 1/2)
 *   kinematics1     pitch angle low, pitch angle high, maximum stroke rate (rad per cycle),
 *                   reference speed (unused by the geometry) */
typedef struct bfx_flapping_wing {
    bfx_float4 root_and_chord;
    bfx_float4 geometry;
    bfx_float4 kinematics0;
    bfx_float4 kinematics1;
} bfx_flapping_wing;

/* BirdBodyState (Sources/BirdFlowCore/BirdModel.swift:53-68), FP64. */
typedef struct bfx_body_state {
    double position[3];
    double orientation[4];          /* body-to-world quaternion x, y, z, w */
    double velocity[3];
    double omega_body[3];
} bfx_body_state;

/* Hinge of an articulated wing segment: the child segment's frame is its
 * parent's frame rotated about `axis` by
 *   angle(t) = side * (bias + amplitude * sin(2 pi f t + phase))
 * and moved to `origin` (f the wing-beat frequency, side +1 left / -1 right).
 * Origin and axis are in the parent's (chord, span, normal) frame; the axis
 * must be a unit vector.  On the right wing the axis's normal component is
 * negated too (its normal is the mirror image of the left's, negated), so the
 * two wings stay mirror images. */
typedef struct bfx_joint {
    float origin[3];
    float axis[3];
    float bias, amplitude, phase;
    float _reserved;
} bfx_joint;

/* Articulated triangle mesh: vertex coordinates in the frame of their segment
 * (0 = body frame, relative to the body origin; 1 / 2 = left / right wing
 * frame, as (chord, span, normal) offsets from the wing root; with joints,
 * 3 / 4 = left / right middle segment after joints[0] (the elbow) and 5 / 6 =
 * left / right outer segment after joints[1] (the wrist), as offsets from the
 * joint in the segment's frame). */
typedef struct bfx_mesh {
    const float* local_vertices;    /* 3 * vertex_count */
    const uint8_t* vertex_segment;  /* vertex_count */
    uint32_t vertex_count;
    const uint32_t* triangles;      /* 3 * triangle_count vertex indices */
    const uint8_t* triangle_part;   /* part id 1..63 per triangle */
    uint32_t triangle_count;
    uint32_t joint_count;           /* 0, 1 (elbow) or 2 (elbow, wrist) */
    const bfx_joint* joints;
    /* Keyframe replay (MeasuredBirdSurfaceSequence; prepareIndexedBirdSurface,
     * BF.metal:1585-1622): keyframe_count >= 2 frames at strictly increasing
     * keyframe_times (s); keyframe_points holds keyframe_count * vertex_count * 3
     * body-frame offsets (m) that take the place of local_vertices.  Each step
     * interpolates linearly inside the interval holding its time (an exact
     * interior keyframe opens the following interval, times past the last
     * keyframe stay on the last interval) and adds the interval's slope to the
     * body's rigid motion.  Requires joint_count 0 and every vertex on segment 0;
     * 0 frames: no replay. */
    uint32_t keyframe_count;
    const float* keyframe_times;
    const float* keyframe_points;
} bfx_mesh;

/* ForceTorque (Sources/BirdFlowCore/Diagnostics.swift) plus step diagnostics. */
typedef struct bfx_loads {
    double force[3];                /* N, FP64 momentum-exchange sum */
    double torque[3];               /* N m about the body position */
    double force_lattice[3];
    double limiter_activations;     /* cells where the positivity limiter engaged */
    double max_restriction;
    int64_t link_count;
    int64_t covered_count;
    int64_t uncovered_count;
    double power;                   /* W: aerodynamic power -sum over cut links of F_link . u_wall */
} bfx_loads;

/* RunSample (Sources/BirdFlowMetal/GPUFieldObservation.swift; GPURunSample GPUData.swift:457-501). */
typedef struct bfx_run_sample {
    double time;
    double position[3];
    double orientation[4];
    double velocity[3];
    double omega_body[3];
    double force[3];
    double torque[3];
    float left_hinge_force[3];
    float left_hinge_torque[3];
    float right_hinge_force[3];
    float right_hinge_torque[3];
    uint64_t step;
} bfx_run_sample;

/* GPURuntimeSafetyRecord (BF.metal:80-83): metrics = max Mach, min clearance,
 * Mach and clearance at the first event; event = step (lo, hi), flags
 * (1 Mach, 2 clearance, 4 non-finite), reserved. */
typedef struct bfx_safety_record {
    float metrics[4];
    uint32_t event[4];
} bfx_safety_record;

typedef struct bfx_snapshot_data {  /* SimulationSnapshot (Diagnostics.swift) */
    uint64_t step;
    double time;
    bfx_body_state body;
    bfx_loads loads;
} bfx_snapshot_data;

/* FieldCaptureMode (GPUFieldObservation.swift:4-13): with neither capture
 * flag the advance runs with capture disabled. */
enum {
    BFX_ADVANCE_CAPTURE_FIELDS = 1,       /* .required: rho/u of the last step, waiting for a slot if need be */
    BFX_ADVANCE_RECORD_SAMPLES = 2,       /* recordRunSamples */
    BFX_ADVANCE_CAPTURE_BEST_EFFORT = 4   /* .bestEffort: publish only if a slot is free now, else drop */
};
enum { BFX_FIELD_CAPTURE_REQUIRED = 0, BFX_FIELD_CAPTURE_BEST_EFFORT = 1, BFX_FIELD_CAPTURE_DISABLED = 2 };

typedef struct bfx_advance_result { /* AdvanceResult (GPUFieldObservation.swift:90-108) */
    uint64_t steps_done;
    uint32_t field_frame_published;
    uint32_t safety_passed;
    bfx_safety_record safety;
    uint64_t dropped_field_frames;  /* droppedFieldFrameCount after the call */
} bfx_advance_result;

/* BirdGeometryFrame (GPUFieldObservation.swift:111-160): the prepared frame of
 * the step a field was captured on.  omega_body_world.w is the conservative
 * geometry radius. */
typedef struct bfx_geometry_frame {
    float body_position[4], orientation[4], linear_velocity[4], omega_body_world[4];
    float left_root[4], left_chord[4], left_span[4], left_normal[4], left_angular_velocity[4];
    float right_root[4], right_chord[4], right_span[4], right_normal[4], right_angular_velocity[4];
} bfx_geometry_frame;

/* GPUFieldFrameMetadata + GPUFieldFrameLease (GPUFieldObservation.swift:162-262).
 * density (n floats) and velocity (n float4: lattice velocity xyz, w = 0) are
 * device pointers into the leased slot, valid for reading until the lease is
 * released; nothing may write through them. */
typedef struct bfx_field_frame {
    uint64_t lease;                 /* 0: no frame was leased */
    bfx_snapshot_data snapshot;
    uint32_t grid[3];
    uint32_t slot;
    float domain_origin[3];
    float cell_size;                /* m */
    float velocity_to_physical;     /* m/s per lattice velocity unit */
    float _pad[3];
    bfx_geometry_frame geometry;
    double publication_uptime_seconds;  /* CLOCK_MONOTONIC at publication */
    const float* density;
    const float* velocity;
} bfx_field_frame;

BFX_API const char* bfx_version(void);
BFX_API int bfx_abi_version(void);
BFX_API int bfx_device_count(int* count);

/* BirdFlowSimulation.init(configuration:bird:initialBodyState:) (BirdFlowSimulation.swift:480-644).
 * bird/body may be NULL for BFX_GEOMETRY_NONE; mesh is required for BFX_GEOMETRY_MESH. */
BFX_API int bfx_create(const bfx_config* config, const bfx_bird* bird, const bfx_body_state* body,
               const bfx_mesh* mesh, bfx_sim** out);
BFX_API void bfx_destroy(bfx_sim* sim);
/* MetalFlappingWingValidator's prescribed-wing setup (MetalFlappingWingValidation.swift:3312-3600:
 * preparePrescribedFlappingWing + buildPrescribedFlappingWing around stepFluidTRT).  config->geometry
 * must be BFX_GEOMETRY_FLAPPING_WING and free_flight 0; the body sits at the wing root (loads and
 * torques about it).  Each step t (1, 2, ...) builds the wing at the phase of t / cycle steps. */
BFX_API int bfx_create_flapping_wing(const bfx_config* config, const bfx_flapping_wing* wing, bfx_sim** out);

/* advance(steps:batchSize:fieldCapture:recordRunSamples:) (BirdFlowSimulation.swift:688-799).
 * samples may be NULL unless BFX_ADVANCE_RECORD_SAMPLES is set (capacity >= steps). */
BFX_API int bfx_advance(bfx_sim* sim, uint64_t steps, uint32_t batch_size, uint32_t flags,
                bfx_run_sample* samples, size_t sample_capacity, bfx_advance_result* result);

/* snapshot() (BirdFlowSimulation.swift:1087) */
BFX_API int bfx_snapshot(bfx_sim* sim, bfx_snapshot_data* out);
/* copyMacroscopicFields() (BirdFlowSimulation.swift:1109): the newest published
 * field frame, else observation slot 0 (density[n], velocity[3n], lattice units). */
BFX_API int bfx_copy_fields(bfx_sim* sim, float* density, float* velocity_xyz, size_t cells);
/* copyGaugePressureFieldPascals() (BirdFlowSimulation.swift:1132) */
BFX_API int bfx_copy_gauge_pressure(bfx_sim* sim, float pressure_scale_pascals, float* out, size_t cells);
/* observationBufferCount (BirdFlowSimulation.swift:480-488, 540-600): the
 * number of field observation slots, 1...4 (default 1).  Allowed before the
 * first step only.  wait_limit_ms bounds how long a required capture waits for
 * a lease to be released (0: without limit, as the reference does); when it
 * runs out the call fails with BFX_ERR_TIMEOUT and the handle stays usable.
 * It replaces the slot set, so no acquire or release may run concurrently
 * with it (unlike with bfx_advance). */
BFX_API int bfx_set_observation_buffers(bfx_sim* sim, uint32_t count, uint32_t wait_limit_ms);
/* acquireLatestGPUFieldFrame(afterStep:) (BirdFlowSimulation.swift:1148-1171):
 * leases the newest published frame, if its step is above after_step when
 * has_after_step is set; out->lease == 0 when there is none.  Thread-safe with
 * respect to bfx_advance on the same handle. */
BFX_API int bfx_acquire_field_frame(bfx_sim* sim, int has_after_step, uint64_t after_step, bfx_field_frame* out);
/* Copies a leased frame to host memory (density[n], velocity[3n], lattice units). */
BFX_API int bfx_field_frame_copy(bfx_sim* sim, uint64_t lease, float* density, float* velocity_xyz, size_t cells);
/* GPUFieldFrameLease.releaseImmediately (GPUFieldObservation.swift:247-249).
 * Releasing twice is a no-op.  Thread-safe. */
BFX_API int bfx_release_field_frame(bfx_sim* sim, uint64_t lease);
/* GPUFieldFrameLease.releaseAfterCompletion(of:) (GPUFieldObservation.swift:241-245):
 * the release runs once the work queued so far on cuda_stream (a cudaStream_t;
 * NULL: the simulation's own stream) has completed. */
BFX_API int bfx_release_field_frame_after(bfx_sim* sim, uint64_t lease, void* cuda_stream);
/* captureCurrentMacroscopicField(mode:) (BirdFlowSimulation.swift:1176-1210):
 * publishes rho/u of the current populations without a step. */
BFX_API int bfx_capture_current_fields(bfx_sim* sim, uint32_t mode, uint32_t* published);
/* deriveFlowDiagnostics (Sources/BirdFlowVisualization/Metal/Visualization.metal:270-308)
 * of a leased frame: vorticity (curl xyz and |curl|, 1/s) as 4 floats per
 * cell, the Q criterion -tr(grad u . grad u) / 2 (1/s^2) and a validity byte;
 * boundary cells and cells whose 7-point stencil touches the body of the
 * captured step are invalid (zeros).  Outputs of `cells` >= n entries, in host
 * memory, or device memory of this simulation's GPU when device_outputs != 0. */
BFX_API int bfx_flow_diagnostics(bfx_sim* sim, uint64_t lease, float* vorticity4, float* q_criterion, uint8_t* valid,
                                 size_t cells, int device_outputs);
/* droppedFieldFrameCount, fieldCaptureWaitCount (BirdFlowSimulation.swift:466-478) */
BFX_API int bfx_observation_counters(bfx_sim* sim, uint64_t* dropped_frames, uint64_t* capture_waits);
/* runtimeSafetyReport() (BirdFlowSimulation.swift:1766) */
BFX_API int bfx_runtime_safety(bfx_sim* sim, bfx_safety_record* out);
BFX_API int bfx_last_loads(bfx_sim* sim, bfx_loads* out);
/* Canonical post-collision populations f*_q(x), direction-major [19][n] in FP32
 * (the reference's populationsIn layout, Docs/NUMERICS.md:33-37). */
BFX_API int bfx_copy_populations(bfx_sim* sim, float* out, size_t count);
BFX_API int bfx_set_populations(bfx_sim* sim, const float* in, size_t count);
/* Current occupancy (part id per cell) and wall field (xyz lattice velocity, w distance). */
BFX_API int bfx_copy_mask(bfx_sim* sim, uint8_t* out, size_t cells);
BFX_API int bfx_copy_wall(bfx_sim* sim, float* out4, size_t cells);
/* Cut links of the last step (fluid cell, direction, link fraction), in the
 * deterministic order of the compaction. */
BFX_API int bfx_copy_links(bfx_sim* sim, uint32_t* cell, uint8_t* direction, float* fraction, size_t capacity,
                   size_t* count);
/* Global mass and momentum of fluid cells in FP64 (measureFluidMassMomentum, BF.metal:4272-4297). */
BFX_API int bfx_fluid_mass_momentum(bfx_sim* sim, double out[4]);
/* Raw restart state (saveCheckpoint / init(checkpointURL:), BirdFlowSimulation.swift:1214-1298, 1920-2024):
 * bfx_save_state with buf == NULL reports the size. */
BFX_API int bfx_save_state(bfx_sim* sim, void* buf, size_t capacity, size_t* size);
BFX_API int bfx_restore_state(bfx_sim* sim, const void* buf, size_t size);
/* Body state (FP64) read/write between advances. */
BFX_API int bfx_get_body(bfx_sim* sim, bfx_body_state* out);
BFX_API int bfx_set_body(bfx_sim* sim, const bfx_body_state* in);
/* Step counter and time (stepIndex, timeSeconds). */
BFX_API int bfx_step_index(bfx_sim* sim, uint64_t* step, double* time);
/* Device timing of the fused stream-collide kernel: when enabled, CUDA events on
 * the simulation's stream bracket every launch; total milliseconds and launch
 * count since enabling. */
BFX_API int bfx_set_kernel_timing(bfx_sim* sim, int enabled);
BFX_API int bfx_kernel_timing(bfx_sim* sim, double* total_ms, uint64_t* launches);
/* Region timer on the simulation's stream: bfx_timer_begin records a CUDA event,
 * bfx_timer_end records a second one, waits for it and returns the elapsed
 * device time in milliseconds. */
BFX_API int bfx_timer_begin(bfx_sim* sim);
BFX_API int bfx_timer_end(bfx_sim* sim, double* elapsed_ms);
/* Test hook of the staged 16-bit fluid kernel's bounded pipeline waits; no
 * reference counterpart.  From the next step on, the kernel's producer
 * withholds the loads of tile `tile` (-1: none) and every pipeline wait gives
 * up after `wait_limit` polls (0: the default limit, about a second).  The
 * withheld tile's consumers then stop waiting, the kernel sets its error flag,
 * waits (bounded) for its own copies still in flight and returns, and the
 * advance fails with BFX_ERR_KERNEL, leaving the handle terminally invalid as
 * a failed command buffer does (BirdFlowSimulation.swift:2059-2095).  The GPU
 * and other handles stay usable.  BFX_ERR_UNSUPPORTED when the handle does not
 * run the staged kernel (FP32 / FP64 storage or the limiter operator). */
BFX_API int bfx_test_stall_staged_kernel(bfx_sim* sim, int32_t tile, uint32_t wait_limit);
/* Test hook for checking the discrete adjoint against finite differences of
 * the objective at a fixed topology; no reference counterpart.  mode 1 records
 * the occupancy (the mask bytes, n per step) of each following step into
 * device_masks, step k of the recording at k * nx*ny*nz; mode 2 replaces each
 * following step's freshly classified occupancy by the recorded one (the wall
 * field, link fractions and loads still follow this handle's geometry), so a
 * run with perturbed kinematic parameters keeps the recorded cut-link sets;
 * mode 0 turns it off.  The recording counts steps from the call; steps past
 * capacity_steps are neither recorded nor replaced.  While on, steps run
 * without CUDA graphs or the pipelined geometry build.  The buffer is the
 * caller's and must outlive the mode.  BFX_ERR_UNSUPPORTED without moving
 * geometry. */
BFX_API int bfx_test_replay_topology(bfx_sim* sim, int mode, uint8_t* device_masks, uint64_t capacity_steps);
/* Total kernel launches issued by the library on this handle. */
BFX_API int bfx_launch_count(bfx_sim* sim, uint64_t* launches);
/* Bytes of device memory held by the handle. */
BFX_API int bfx_device_bytes(bfx_sim* sim, uint64_t* bytes);
/* Allocation-free variant of bfx_fluid_mass_momentum.  It has no counterpart in
 * the reference.  It is for callers that cannot call cudaMalloc where they need
 * the sum: a host application whose device memory budget is already reserved
 * by its own allocator (a framework's caching pool), where a fresh allocation
 * fails or fragments that pool, and loops with a fixed time budget per
 * iteration, where cudaMalloc / cudaFree would synchronise the device.
 * The caller passes device pointers it already holds:
 *   populations  canonical, dense FP32 populations, direction-major
 *                [19][nx*ny*nz] (the layout of bfx_copy_populations).  This is
 *                not a handle's own population buffer, which carries a halo,
 *                a padded row pitch and possibly 16-bit storage: a caller that
 *                holds a bfx_sim copies the populations into such an array
 *                first;
 *   mask         part id per cell (0 = fluid), or NULL for an all-fluid lattice;
 *   out          4 doubles: fluid mass and momentum x, y, z (FP64).
 * Scratch is a fixed 1 MiB device array inside the library (kept by every GPU
 * that loads it until the process exits), so lattices above 8,388,608 cells
 * are rejected with BFX_ERR_CAPACITY.  The first call on a device looks up
 * that array's device address and keeps it, so make that first call before
 * any stream capture; the address belongs to the CUDA context current at that
 * call (a context recreated later, e.g. after cudaDeviceReset, is not
 * supported).  The work runs on the legacy default stream, not on any
 * handle's stream, and the call returns after it finishes.  Calls share the
 * scratch: calls that overlap on the GPU race and must be serialised. */
BFX_API int bfx_fluid_mass_momentum_noalloc(const float* populations, const uint8_t* mask, uint32_t nx, uint32_t ny,
                                            uint32_t nz, double* out);
/* ---- discrete adjoint ------------------------------------------------------
 * No reference counterpart (the reference has no adjoint).  Gradient of a
 * time-averaged load objective with respect to the four prescribed wing
 * kinematic parameters theta = (wing_kinematics0.y stroke amplitude,
 * wing_kinematics1.x pitch amplitude, wing_kinematics1.y pitch phase,
 * wing_kinematics1.z deviation amplitude), all in radians:
 *   J = mean over steps k in [window_first, window_last] of
 *       force_weight . F_k + power_weight * P_k,
 * F_k the momentum-exchange body force (N) of step k and
 * P_k = -sum over cut links of F_link . u_wall the aerodynamic power (W) the
 * wings deliver to the fluid.  Step indices count from 1 at the call.
 * The call advances the simulation by `steps` (the final state equals that of
 * bfx_advance(steps)), then runs the discrete adjoint backward with two-level
 * checkpointing: a population snapshot every `checkpoint_interval` steps
 * (0 = ceil(sqrt(steps))), each interval recomputed once with its adjoint
 * tape.  Scope: TRT collision, F32 or F64 storage, mesh geometry with moving
 * wings and no free flight, far-field / velocity / periodic faces, force
 * estimator 6, all parts, link and topology loads; anything else returns
 * BFX_ERR_UNSUPPORTED.  The topology of every step (solid cells, links,
 * bounce-back case) is held fixed, so the gradient is that of the smooth piece
 * of J the parameters lie on. */
typedef struct bfx_adjoint_objective {
    double force_weight[3];
    double power_weight;
    uint64_t window_first;          /* 0 and 0: every step of the call */
    uint64_t window_last;
} bfx_adjoint_objective;

typedef struct bfx_adjoint_result {
    double objective;               /* J */
    double gradient[4];             /* dJ/dtheta */
    uint64_t steps;
    uint32_t checkpoint_interval;
    uint32_t snapshots;
    double forward_ms;              /* device time of the forward pass with its snapshots */
    double reverse_ms;              /* device time of the recomputation and the reverse sweep, from its first
                                       launch (the allocation of its work memory is not included) */
    uint64_t max_links;             /* largest cut-link count of the run */
    uint64_t work_bytes;            /* device memory of snapshots, tape and adjoint fields */
} bfx_adjoint_result;

BFX_API int bfx_adjoint(bfx_sim* sim, uint64_t steps, const bfx_adjoint_objective* objective,
                        uint32_t checkpoint_interval, bfx_adjoint_result* result);

/* ---- coupled momentum ledger ------------------------------------------------
 * One linear-momentum balance per step of a free-flight run, all impulses in
 * SI (kg m / s): the fluid momentum reduced directly from the populations
 * before and after the step, the whole-bird and prescribed-wing momenta, and
 * the external sources the fluid receives (open far-field faces, sponge) with
 * the persistent cut-link exchange reconstructed from the pre-step
 * populations.  Replaces BirdFlowSimulation.advanceWithCoupledMomentumLedger
 * (BirdFlowSimulation.swift:806-1085, BF.metal:4322-4552); the report (RMS,
 * relative residuals, verdict) is assembled by the caller. */
typedef struct bfx_ledger_sample {
    uint64_t step;
    double time;
    double fluid_momentum_before[3], fluid_momentum_after[3], fluid_momentum_change[3];
    double body_momentum_before[3], body_momentum_after[3];
    double wing_momentum_before[3], wing_momentum_after[3];
    double aerodynamic_impulse[3], gravity_impulse[3];
    double far_field_impulse[3], sponge_impulse[3], link_exchange_impulse[3], topology_impulse[3];
    double fluid_boundary_impulse[3], boundary_residual[3];
    double total_momentum_change[3], external_impulse[3], system_residual[3];
    uint64_t far_field_links, sponge_cells, boundary_links, topology_cells;
} bfx_ledger_sample;

/* Advances `steps` steps one at a time and records a ledger sample per step
 * (capacity >= steps).  Free flight only, sponge strength below 1 - 1e-6 (the
 * pre-sponge populations are reconstructed from the post-sponge ones):
 * BFX_ERR_UNSUPPORTED otherwise.  *steps_done reports the samples written,
 * also when a safety violation (BFX_ERR_SAFETY) stops the run. */
BFX_API int bfx_advance_ledger(bfx_sim* sim, uint64_t steps, bfx_ledger_sample* samples, size_t capacity,
                               uint64_t* steps_done);

/* Message of the last failure on this handle (or of the last failed create when sim is NULL). */
BFX_API int bfx_last_error(bfx_sim* sim, char* buf, size_t capacity);

#ifdef __cplusplus
}
#endif
#endif /* BFX_H */
