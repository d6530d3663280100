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
};

// Prepared articulated geometry (GPUPreparedBirdGeometry, BF.metal:112-127).
struct Prepared {
    float4 body_position, orientation, linear_velocity, omega_body_world;
    float4 left_root, left_chord, left_span, left_normal, left_angular_velocity;
    float4 right_root, right_chord, right_span, right_normal, right_angular_velocity;
};

// Device-resident per-simulation state updated by the single-thread kernels.
struct DeviceState {
    uint64_t step;                 // completed steps
    double body[13];               // position 3, orientation 4, velocity 3, omega 3
    Prepared prep;
    int32_t box_origin[3];         // geometry region origin (cells)
    int32_t _pad0;
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
};

}  // namespace bfx
