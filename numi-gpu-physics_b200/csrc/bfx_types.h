// Internal parameter blocks shared by the kernels and the host runtime.
#pragma once

#include <stdint.h>

#include "../../include/bfx.h"

namespace bfx {

struct Grid;
struct Spill;

// Per-run constants of the fluid step (the typed content of GPUUniforms,
// Sources/BirdFlowMetal/GPUData.swift:4-80).
struct FluidParams {
    float origin[3];
    float dx;
    float dt, v2l, f2p;
    float omega_p, omega_m, sponge_strength, sponge_width;
    float far[4];
    float face_u[6][3];
    int face_bc[6];
    int collision;
    int interpolated;
    int load_component;
    int force_mode;
    int selected_part;
    int local_density;
    int accumulate;
    int has_sponge;
    int any_outflow;
    int fast_math;
    int act_margin;          // cells around the mesh vertices' bounding box the geometry can touch
};

// Prepared articulated geometry (GPUPreparedBirdGeometry, BF.metal:112-127).
struct Prepared {
    float4 body_position, orientation, linear_velocity, omega_body_world;
    float4 left_root, left_chord, left_span, left_normal, left_angular_velocity;
    float4 right_root, right_chord, right_span, right_normal, right_angular_velocity;
};

// Frame of an articulated wing segment after the elbow / wrist joints:
// origin, axes, angular velocity relative to the body (world) and the velocity
// of the origin relative to the body.
struct SegmentFrame {
    float4 origin, chord, span, normal, omega, uvel;
};

// Device-resident per-simulation state updated by the single-thread kernels.
struct DeviceState {
    uint64_t step;                 // completed steps
    double body[13];               // position 3, orientation 4, velocity 3, omega 3
    Prepared prep;
    int32_t box_origin[3];         // geometry region origin (cells)
    float geom_time;               // time (s) of the step the geometry was built for
    // bounding box (cells, inclusive) of this step's mesh vertices; open
    // (+-2^30) for the analytic shapes, empty before the vertices are placed
    int32_t act_lo[3], act_hi[3];
    float wing_prev[16];           // GPUWingMomentumState
    float wing_reaction[16];       // GPUWingInertialReaction
    float safety_metrics[4];
    uint32_t safety_event[4];
    double loads_lattice[3];       // last step: lattice force sum
    double loads_torque[3];        // physical torque
    double limiter_count;          // bulk-kernel limiter activations
    uint32_t limiter_max_bits;     // bit pattern of max restriction (float, non-negative)
    uint32_t link_overflow;
    int64_t link_count;
    int64_t covered_count;
    int64_t uncovered_count;
    uint64_t launches_device;
    double power_lattice;          // last step: sum over cut links of F_link . u_wall (lattice units)
    uint32_t stream_error;         // nonzero: a staged-kernel pipeline wait timed out (1 producer, 2 consumer)
    // test hook of the staged kernel's bounded waits (bfx_test_stall_staged_kernel):
    // the producer skips the loads of tile test_stall_tile1 - 1 (0: none) and
    // every wait gives up after test_wait_limit polls (0: the default limit)
    uint32_t test_stall_tile1;
    uint32_t test_wait_limit;
    uint32_t apply_done;           // link-kernel blocks finished this launch (0 between launches)
    SegmentFrame seg[4];           // mesh segments 3..6: left / right middle, left / right outer
};

// Time-averaged load objective of the adjoint (one per simulation; disabled
// outside bfx_adjoint).  J = mean over the window of
// force_weight . F + power_weight * P, with F the body force (N) and
// P = -sum_links F_link . u_wall the aerodynamic power (W) the wings deliver.
struct Objective {
    int32_t enabled;
    int32_t _pad;
    uint64_t start;                // completed steps when the window count starts
    uint64_t first, last;          // window of relative step indices (1-based, inclusive)
    double force_weight[3];
    double power_weight;
    double value;                  // accumulated J
    double grad[4];                // accumulated dJ/dtheta
    int64_t max_links;             // largest cut-link count while enabled
};

// Number of kinematic parameters the adjoint differentiates: stroke
// amplitude, pitch amplitude, pitch phase, deviation amplitude (radians).
constexpr int kKinematicParams = 4;

// Forward-mode tangent of the wing frames with respect to the kinematic
// parameters, one step: value and the four partials of each component of
// chord, span, normal and the relative angular velocity, per side.
struct FrameTangent {
    float v[2][4][3];
    float d[2][4][3][kKinematicParams];
};

// Everything the adjoint of one cut link needs from its forward step.
template <class R>
struct LinkTape {
    uint32_t cell;                 // fluid cell (flat index)
    uint32_t dir;                  // direction q (the solid source is cell - c_q)
    uint32_t kase;                 // 0 halfway / fallback, 1 interpolated q <= 1/2, 2 interpolated q > 1/2
    uint32_t _pad;
    R value, reflected, other, q;  // other: f*_opp(q)(x + c_q) (kase 1) or f*_q(x) (kase 2)
    R wv[3];                       // wall velocity at the link (lattice)
    float dq[kKinematicParams];
    float dwv[kKinematicParams][3];
};

}  // namespace bfx
