/*
 * CPU oracle for the D3Q19 moving-boundary step — TEST INFRASTRUCTURE ONLY.
 *
 * This is a plain-C restatement of the BirdFlowMetal algorithm for the hot
 * path, written as the checker for the CUDA library.  It is never linked into,
 * loaded by, or called from the product; only tests/, the smoke check and
 * bench.py's CPU-baseline leg use it.
 *
 * It follows the reference literally: A/B ping-pong buffers with pull
 * streaming, interpolated link fractions stored in the dormant population
 * slots of solid cells, FP32 arithmetic in the reference's operation order
 * (compiled with -ffp-contract=off so a*b+c is never fused).
 *
 * Reference files (Numi2/numi-gpu-physics):
 *   Sources/BirdFlowMetal/Metal/BirdFlow.metal      (kernels; "BF.metal")
 *   Sources/BirdFlowCore/D3Q19.swift                (lattice, equilibrium, TRT)
 *   Sources/BirdFlowCore/RigidBody.swift            (6-DOF integrator)
 *   Sources/BirdFlowMetal/MetalShearWaveValidation.swift (CPU shear wave)
 *   Sources/BirdFlowMetal/InterpolatedBounceBackReference.swift
 * Parity is pinned by tests/golden (fixtures from Reference/shear_wave_reference.py
 * and the reference's known-answer tests).
 */
#ifndef BFX_ORACLE_H
#define BFX_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { OR_BC_FARFIELD = 0, OR_BC_PERIODIC = 1, OR_BC_VELOCITY = 2, OR_BC_OUTFLOW = 3 };
enum { OR_COLLISION_TRT = 0, OR_COLLISION_TRT_LIMITER = 1, OR_COLLISION_REGULARIZED = 2, OR_COLLISION_RR3 = 3 };

/* Per-step parameters: the typed form of the reference's GPUUniforms
 * (Sources/BirdFlowMetal/GPUData.swift:4-80). */
typedef struct or_params {
    int32_t nx, ny, nz, _pad0;
    float origin[3];
    float dx;
    float time, dt, v2l, f2p;
    float omega_p, omega_m, sponge_strength, sponge_width;
    float far[4];            /* far-field lattice velocity xyz, density w */
    float gravity[3];
    int32_t accumulate_loads;
    int32_t interpolated;    /* caseParameters.w < -0.5 */
    int32_t collision;       /* OR_COLLISION_* */
    int32_t load_component;  /* caseParameters.x when interpolated */
    int32_t force_mode;      /* caseParameters.y when interpolated, else 6 */
    int32_t selected_part;   /* caseParameters.z */
    int32_t free_flight, capture_fields, has_prev_geom;
    int32_t face_bc[6];      /* -x,+x,-y,+y,-z,+z */
    float face_velocity[6][3];
    int32_t substeps, local_density, _pad1, _pad2;
} or_params;

/* Body loads of one step.  f64_* follow the FP64 contribution sum used by the
 * CUDA library; f32_* follow the reference's FP32 group-of-256 partials plus
 * the sequential 256-way reduction (BF.metal:3199-3235, 5359-5387). */
typedef struct or_loads {
    double f64_force_lattice[3];
    double f64_force[3];     /* physical: lattice sum * force scale */
    double f64_torque[3];    /* physical */
    double activation;
    double max_restriction;
    float f32_force[4];      /* xyz force, w activation count */
    float f32_torque[4];     /* xyz torque, w max restriction */
    int64_t link_count;
    int64_t covered_count;
    int64_t uncovered_count;
} or_loads;

/* float4-packed structures identical to the reference's GPU ABI. */
typedef struct { float v[4]; } or_f4;
typedef struct or_bird {     /* GPUBirdParameters, GPUData.swift:82-178 */
    or_f4 body_radii_mass, inertia, wing_geometry0, wing_geometry1, tail_geometry,
          wing_kinematics0, wing_kinematics1, safety_geometry, safety_limits,
          left_wing_mass_com, left_wing_inertia, right_wing_mass_com, right_wing_inertia;
} or_bird;
typedef struct or_prepared { /* GPUPreparedBirdGeometry, BF.metal:112-127 */
    or_f4 body_position, orientation, linear_velocity, omega_body_world,
          left_root, left_chord, left_span, left_normal, left_angular_velocity,
          right_root, right_chord, right_span, right_normal, right_angular_velocity;
} or_prepared;
typedef struct or_body_f32 { float position[3], orientation[4], velocity[3], omega_body[3]; } or_body_f32;
typedef struct or_body_f64 { double position[3], orientation[4], velocity[3], omega_body[3]; } or_body_f64;

/* ---- lattice --------------------------------------------------------- */
void or_lattice(int32_t* c /*19x3*/, int32_t* opp /*19*/, float* w /*19*/);
float or_equilibrium(int q, float rho, const float u[3]);
/* One regularized (rr3 = 0) or RR3 (rr3 = 1) collision of the 19 populations
 * f (BF.metal:2917-3062).  order 0: the reference's literal per-direction
 * expressions; order 1: the opposite-direction pair order the stepping (and
 * the FP32 fluid kernel) uses.  activation / restriction report the
 * positivity admission. */
void or_collide_regularized(int order, const float* f, float omega_p, int rr3, float* post, float* activation,
                            float* restriction);
void or_trt_collision(const float* f, float rho, const float u[3], float omega_p, float omega_m, float* out);

/* ---- field initialisation (BF.metal:2078-2162) ----------------------- */
void or_init_equilibrium(const or_params* p, float* pops, const uint8_t* mask, const float* wall,
                         float* density, float* velocity);
/* axis = 1 reproduces initializeShearWave (u_x varies along y); axis = 2 varies along z */
void or_init_shear_wave(const or_params* p, float amplitude, int axis, float* pops, float* density, float* velocity);
void or_macroscopic(const or_params* p, const float* pops, float* density, float* velocity);

/* ---- fused fluid step (BF.metal:2507-3236) --------------------------- */
/* covered: float4 per cell preserved momentum xyz, density w (interpolated mode).
 * per_cell_loads: optional 8 floats per cell (reference per-thread values). */
void or_step(const or_params* p, const float* pin, float* pout,
             const uint8_t* mprev, const uint8_t* mcur, const float* wall, const float* covered,
             float* density, float* velocity, const float body_f[3], const double body_d[3],
             or_loads* loads, float* per_cell_loads);

/* Mass and momentum of fluid cells in FP64 (measureFluidMassMomentum, BF.metal:4272-4297). */
void or_fluid_mass_momentum(const or_params* p, const float* pops, const uint8_t* mask, double out[4]);

/* ---- analytic bird geometry ----------------------------------------- */
void or_prepare_bird(const or_bird* bird, const or_body_f32* body, float time, float dx, or_prepared* out);
void or_build_bird(const or_params* p, const or_bird* bird, const or_prepared* prep,
                   const uint8_t* mprev, uint8_t* mnext, float* wall);

/* ---- ellipsoid body with analytic link fractions --------------------- */
/* Classification of the body ellipsoid (part 1), wall velocity from rigid motion. */
void or_build_ellipsoid(const or_params* p, const or_bird* bird, const or_prepared* prep,
                        const uint8_t* mprev, uint8_t* mnext, float* wall);
float or_ellipsoid_link_fraction(const or_params* p, const or_bird* bird, const or_prepared* prep,
                                 int fx, int fy, int fz, int sx, int sy, int sz);

/* ---- coupled momentum ledger (BF.metal:4322-4552) ----------------------
 * Lattice-unit sums over one step from pin (before) to pout (after) with the
 * step's masks (mprev before, mcur after) and wall field: out[0..3] mass and
 * momentum of the cells that were fluid (pin), [4..7] of the cells that are
 * fluid (pout), [8..11] the open-face source (incoming - outgoing, momentum
 * (incoming + outgoing) c), [12..15] the persistent cut-link exchange on the
 * halfway moving-wall rule, [16..19] the sponge source recovered from
 * f_out = (1 - s) f_post + s f_far, [20] open-face links, [21] sponge cells,
 * [22] persistent links, [23] cells that changed occupancy. */
void or_ledger_sources(const or_params* p, const float* pin, const float* pout, const uint8_t* mprev,
                       const uint8_t* mcur, const float* wall, double out[24]);

/* ---- prescribed flapping wing (MetalFlappingWingValidation's analytic wing) */
typedef struct or_wing {     /* GPUFlappingWingParameters, GPUData.swift:383-388 */
    or_f4 root_and_chord, geometry, kinematics0, kinematics1;
} or_wing;
typedef struct or_wing_prepared { /* GPUPreparedFlappingWing, GPUData.swift:392-399 */
    or_f4 root, chord, span, normal, angular_velocity, state;
} or_wing_prepared;
/* preparePrescribedFlappingWing (BF.metal:1038-1078); time = absolute step index. */
void or_prepare_wing(const or_wing* w, float time, or_wing_prepared* out);
/* prescribedWingMaximumViolation of the boundary coordinates (BF.metal:1091-1142). */
float or_wing_violation(const or_params* p, const or_wing* w, const or_wing_prepared* pw, const float world[3]);
/* buildPrescribedFlappingWing classification (BF.metal:1179-1249). */
void or_build_wing(const or_params* p, const or_wing* w, const or_wing_prepared* pw, const uint8_t* mprev,
                   uint8_t* mnext, float* wall);
/* prescribedWingLinkFraction (BF.metal:1144-1175) of the link from solid s toward s + c_q. */
float or_wing_link_fraction(const or_params* p, const or_wing* w, const or_wing_prepared* pw, int q, int sx, int sy,
                            int sz);
void or_wing_link_fractions(const or_params* p, const or_wing* w, const or_wing_prepared* pw, const uint32_t* cell,
                            const uint8_t* dir, int64_t count, float* out);
float or_powf(float b, float e);

/* Writes link fractions into pops[q*N+s] for every solid s / fluid s+c_q pair and
 * preserves newly covered momentum (BF.metal:1251-1295 pattern).  kind 0 =
 * ellipsoid bisection, 1 = mesh linear signed-distance rule (BF.metal:2044-2076),
 * 2 = mesh ray root, 3 = prescribed-wing bisection (bird / prep then point to
 * the or_wing / or_wing_prepared). Returns the number of links written. */
int64_t or_write_links(const or_params* p, int kind, const or_bird* bird, const or_prepared* prep,
                       const float* mesh_pos /*4 per vertex*/, const uint32_t* tris, uint32_t ntris,
                       float half_thickness, const uint64_t* keys,
                       float* pops, const uint8_t* mprev, const uint8_t* mcur, const float* wall, float* covered);

/* Enumerates cut links (fluid x, direction q, solid source x-c_q) in cell-major,
 * direction-minor order; returns the count (arrays may be NULL to count). */
int64_t or_enumerate_links(const or_params* p, const uint8_t* mprev, const uint8_t* mcur,
                           uint32_t* cell, uint8_t* dir, int64_t capacity);

/* ---- triangle mesh -------------------------------------------------- */
/* Articulated rigid-segment vertices: local (chord, span, normal) coords per
 * vertex and segment 0 = body frame, 1 = left wing, 2 = right wing. */
/* Wing joints (bfx_joint) and the frames of the jointed segments 3..6:
 * the elbow / wrist hinge rotates its parent's frame about the hinge axis by
 * side * (bias + amplitude sin(phase_t + phase)) and moves it to the joint.
 * This is the library's extension for the multi-segment wings of the north
 * star's articulated bird; the reference drives its wings as one rigid frame
 * each (makeWingFrame, BF.metal:611-684). */
typedef struct or_joint { float origin[3], axis[3], bias, amplitude, phase, reserved; } or_joint;
typedef struct or_segment { float origin[4], chord[4], span[4], normal[4], omega[4], uvel[4]; } or_segment;
void or_prepare_segments(const or_bird* bird, const or_prepared* prep, const or_joint* joints, int njoints,
                         float time, or_segment* out /* 4: left / right middle, left / right outer */);
void or_mesh_prepare_segments(const or_prepared* prep, const or_segment* segs, const float* local,
                              const uint8_t* segment, uint32_t nverts, float v2l, float* pos, float* vel);
/* Keyframe replay of body-frame offsets (prepareIndexedBirdSurface,
 * BF.metal:1585-1622) on top of the body's rigid motion at `time`. */
void or_mesh_prepare_keyframes(const or_prepared* prep, const float* times, uint32_t nframes, const float* points,
                               uint32_t nverts, float time, float v2l, float* pos, float* vel);
void or_mesh_prepare_articulated(const or_prepared* prep, const float* local /*3 per vertex*/,
                                 const uint8_t* segment, uint32_t nverts, float v2l,
                                 float* pos /*4 per vertex*/, float* vel /*4 per vertex*/);
void or_mesh_rasterize(const or_params* p, const float* pos, const uint32_t* tris, uint32_t ntris,
                       float half_thickness, uint64_t* keys);
void or_mesh_resolve(const or_params* p, const float* pos, const float* vel, const uint32_t* tris,
                     const uint8_t* tri_part, uint32_t ntris, float half_thickness, const uint64_t* keys,
                     uint8_t* mask, float* wall);
float or_mesh_ray_root(const or_params* p, const float* pos, const uint32_t* tris, uint32_t ntris,
                       float half_thickness, const uint64_t* keys, int fx, int fy, int fz, int sx, int sy, int sz);

/* ---- rigid body, wing reaction, safety (BF.metal:6493-6707; RigidBody.swift:88-126) */
void or_integrate_body_f32(or_body_f32* body, const or_bird* bird, const float force[3], const float torque[3],
                           const float gravity[3], float dt, int substeps);
void or_integrate_body_f64(or_body_f64* body, const or_bird* bird, const double force[3], const double torque[3],
                           const double gravity[3], double dt, int substeps);
/* Reference CPU integrator RigidBodyIntegrator.integrate (RigidBody.swift:88-126), FP32. */
void or_rigid_body_swift_f32(or_body_f32* body, float mass, const float inertia[3], const float force[3],
                             const float torque[3], const float gravity[3], float dt, int substeps);
/* updateWingInertialReaction: previous[16] (left lin, left ang, right lin, right ang, float4 each),
 * reaction[16] output; returns 0 when the wings are massless. */
void or_wing_reaction(const or_prepared* prep, const or_bird* bird, float dt, int initialize_only,
                      float* previous, float* reaction);
/* monitorBirdRuntimeSafety; record = metrics float4 + event uint4 */
void or_safety(const or_body_f32* body, const or_bird* bird, const or_params* p, uint32_t step_lo,
               uint32_t step_hi, float* metrics, uint32_t* event);

/* ---- interpolated bounce-back algebra (InterpolatedBounceBackReference.swift:11-62), FP64 */
double or_link_fraction(double fluid_implicit, double solid_implicit);
double or_interpolated_population(double q, double reflected, double farther_outgoing, double previous_incoming,
                                  double moving_wall_correction);
void or_uncovered_impulse(const double refill_momentum[3], const double* directions /*3 per stencil*/,
                          const double* old_outgoing, const double* suppressed_incoming, int count, double out[3]);

#ifdef __cplusplus
}
#endif
#endif
