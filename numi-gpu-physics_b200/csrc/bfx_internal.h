// Host-side launcher interface between the runtime (bfx_api.cu) and the
// kernel translation units.  Not part of the public ABI.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "bfx_types.h"

namespace bfx {

struct GridDesc {
    int nx, ny, nz;
    int per_x, per_y, per_z;
    int64_t n, nxy;
    int px;                 // padded row pitch: nx + 2 rounded up to 8 cells (16-byte rows for TMA)
    int64_t padded;         // px (ny+2)(nz+2): cells of the population array with its halo
};

struct FluidBuffers {
    void* pops;             // 19 * padded elements of the storage type
    uint8_t* mask;          // current occupancy (part id + topology flags); may be null
    const float4* wall;     // wall velocity / distance; may be null without geometry
    float* density;         // captured fields
    float4* velocity;
    DeviceState* state;
    void* tape;             // pre-collision (rho, u) per cell when the step is taped (capture == 2)
    const void* tmap;       // CUtensorMap of the population array for the staged kernel (null: k_bulk)
    int sm_count;
    const float* face_dev;  // host copy of the x-face values [2][19] for the staged kernel (null: the halo
                            // fill covers the x faces)
};

// Fused stream + collide of every cell: fluid cells collide, solid cells take
// the moving-wall equilibrium and newly uncovered cells refill and collide.
// box: extent of the geometry box (origin in DeviceState), null without
// geometry; the staged 16-bit kernel leaves the box's solid / uncovered cells
// to a second launch over the box.
void launch_bulk(int storage, int collision, int rep_s, const GridDesc& g, const FluidParams& fp,
                 const FluidBuffers& b, int capture, const int* box, cudaStream_t s);
// The step runs the TMA-staged kernel (16-bit storage, staged operator, a
// population tensor map, not taped).
bool bulk_staged(int storage, int collision, int capture, bool tma_ok);
// x-face values for the staged kernel when both x faces are far-field or
// velocity faces (BulkArgs::face_dev): out[2 * 19], computed as the halo fill
// computes and stores them, read back as stored deviations.
void launch_halo_values(int storage, const GridDesc& g, const FluidParams& fp, float* out, cudaStream_t s);
// Halo fill of the z and y faces only (the staged kernel takes the x faces'
// values from BulkArgs::face_dev).
void launch_halo_yz(int storage, int rep_s, const GridDesc& g, const FluidParams& fp, const FluidBuffers& b,
                    cudaStream_t s);
// The staged path's two launches (k_rare over the geometry box, then k_stream)
// for callers that queue work between them; only for a simulation whose
// population tensor map was encoded (16-bit storage, staged operator).
void launch_bulk_rare(int storage, int collision, int rep_s, const GridDesc& g, const FluidParams& fp,
                      const FluidBuffers& b, const int* box, cudaStream_t s);
void launch_bulk_stream(int storage, int collision, int rep_s, const GridDesc& g, const FluidParams& fp,
                        const FluidBuffers& b, const int* box, cudaStream_t s);
// Block counts per segment of the two-level link-offset scan (bfx_geometry.cu).
constexpr int kScanSegment = 8192;

// Vorticity (curl, |curl|), Q criterion and validity of a captured field
// (bfx_fields.cu); velocity in lattice units, scale = 0.5 * velocity_to_physical
// / cell_size; mask: occupancy of the captured step, or null.
void launch_flow_diagnostics(const float4* velocity, const uint8_t* mask, int nx, int ny, int nz, float scale,
                             float4* vorticity, float* q_criterion, uint8_t* valid, cudaStream_t s);
// Halo fill: the values boundary cells pull from outside the lattice (before the step).
void launch_halo(int storage, int rep_s, const GridDesc& g, const FluidParams& fp, const FluidBuffers& b,
                 cudaStream_t s);
// Equilibrium initialisation into representation E.
void launch_init(int storage, int init_kind, float amplitude, const GridDesc& g, const FluidParams& fp,
                 const FluidBuffers& b, cudaStream_t s);
// Canonical FP32 read-out / write-in of f*_q(x) ([19][n]).
void launch_readout(int storage, int rep_s, const GridDesc& g, const FluidBuffers& b, float* out, cudaStream_t s);
void launch_writein(int storage, int rep_s, const GridDesc& g, const FluidBuffers& b, const float* in,
                    cudaStream_t s);
// Macroscopic fields from the canonical populations.
void launch_macroscopic(int storage, int rep_s, const GridDesc& g, const FluidBuffers& b, cudaStream_t s);
// FP64 fluid mass / momentum (partials[blocks*4], result[4]).
void launch_mass_momentum(int storage, int rep_s, const GridDesc& g, const FluidBuffers& b, double* partials,
                          int blocks, double* result, cudaStream_t s);

// ---- geometry, links, loads, body -------------------------------------
struct BoxDesc {
    int sx, sy, sz;         // extent of the geometry region (cells)
    int64_t cells;
};

struct GeomBuffers {
    const bfx_bird* bird;           // device copy
    uint8_t* mask_prev;
    uint8_t* mask_next;
    float4* wall;
    // mesh
    const float* mesh_local;        // 3 per vertex
    const uint8_t* mesh_segment;
    const bfx_joint* joints;        // elbow, wrist (device copy)
    int joint_count;
    const uint32_t* mesh_tris;
    const uint8_t* mesh_tri_part;
    float4* mesh_pos;
    float4* mesh_vel;
    unsigned long long* keys;       // box-local
    uint32_t nverts, ntris;
    float half_thickness;
    // links
    uint32_t* link_cell;
    uint32_t* link_meta;            // direction | part << 8
    float* link_q;
    uint32_t link_capacity;
    uint32_t* block_counts;         // cut links per box block
    uint32_t* block_offsets;
    uint32_t* scan_sums;            // one per kScanSegment scan blocks (two-level scan)
    // topology events (cells newly covered / uncovered whose impulse enters the loads)
    uint32_t* event_counts;         // per box block
    uint32_t* event_offsets;
    uint32_t* event_sums;           // one per kScanSegment scan blocks
    uint32_t* event_cell;           // event list (flat cell index, box-cell order); capacity: box cells
    uint32_t* event_total;          // [1] events in the list
    const float* kf_times;          // keyframe replay: times, frames x vertices x 3 offsets (kf_count >= 2)
    const float* kf_points;
    int kf_count;
    uint32_t* live_list;            // box blocks with a key or an occupancy change (mesh resolve), or null
    uint32_t* live_count;           // [1] entries in live_list
    uint32_t* cell_bits;            // per box cell of a counted block: link sources (bits 1-18), event (bit 0)
    int box_blocks;                 // blocks of a one-slice-per-block box launch (allocations)
    int scan_blocks;                // blocks of the link count / scan / emission launch
    double* topo_partials;          // 8 per topology block
    int topo_blocks;                // blocks of the topology-impulse launch
    double* link_partials;          // 16 per apply block (link sums, topology sums)
    int apply_blocks;
    DeviceState* state;
    Objective* objective;           // load objective accumulated by the step end (may be null)
    void* link_tape;                // LinkTape<R> per link when the step is taped (else null)
    const float* link_tangent;      // per link: dq[4], du_fluid[4][3], du_solid[4][3]
    const FrameTangent* frames;     // wing-frame tangent of the taped step
};

void launch_prepare(int geometry, float dt, const GridDesc& g, const FluidParams& fp, const BoxDesc& box,
                    const GeomBuffers& gb, int init, cudaStream_t s);
void launch_classify(int geometry, int has_prev, const GridDesc& g, const FluidParams& fp, const BoxDesc& box,
                     const GeomBuffers& gb, cudaStream_t s, bool lean_raster = false);
// Cut-link and topology-event lists of the step's geometry (counts, offset
// scan, emission, link fractions).  Reads only geometry: masks, keys, wall
// field and mesh.
// lists_done (optional) is recorded once the lists are written, before the
// link fractions.
void launch_link_build(int geometry, int link_rule, const GridDesc& g, const FluidParams& fp, const BoxDesc& box,
                       const GeomBuffers& gb, cudaStream_t s, cudaEvent_t lists_done = nullptr);
// Topology impulses of the event list into topo_partials; reads the pre-step
// populations, so it runs before the link kernel writes any.
void launch_topology(int storage, int rep_s, const GridDesc& g, const FluidParams& fp, const BoxDesc& box,
                     const GeomBuffers& gb, const FluidBuffers& fb, cudaStream_t s);
// Coupled momentum ledger passes (bfx_ledger.cu): `blocks` rows of 16 (in) or
// 9 (out) FP64 partial sums.
constexpr int kLedgerInWidth = 16;
constexpr int kLedgerOutWidth = 9;
void launch_ledger_in(int storage, int rep_s, const GridDesc& g, const FluidParams& fp, const FluidBuffers& b,
                      const uint8_t* mprev, const uint8_t* mnext, double* partials, int blocks, cudaStream_t s);
void launch_ledger_out(int storage, int rep_s, const GridDesc& g, const FluidParams& fp, const FluidBuffers& b,
                       const uint8_t* mnext, double* partials, int blocks, cudaStream_t s);

// End-of-step body update parameters (k_finish).
struct FinishParams {
    float gravity[3];
    int substeps;
    int free_flight;
};
// Cut-link bounce-back and loads; the launch's last block also reduces the
// link and topology partials into the step's loads and, with `fin`, runs the
// end-of-step body update that launch_integrate would run.
void launch_links_apply(int storage, int rep_s, const GridDesc& g, const FluidParams& fp, const GeomBuffers& gb,
                        const FluidBuffers& fb, int with_topology, const FinishParams* fin, cudaStream_t s);
void launch_integrate(const GridDesc& g, const FluidParams& fp, const GeomBuffers& gb, float gravity_x,
                      float gravity_y, float gravity_z, int substeps, int free_flight, cudaStream_t s);
void launch_record_sample(const GeomBuffers& gb, const FluidParams& fp, bfx_run_sample* samples, uint64_t index,
                          float dt, cudaStream_t s);
void launch_step_counter(DeviceState* st, cudaStream_t s);

// ---- discrete adjoint (bfx_adjoint.cu) ----------------------------------
constexpr int kLinkTangentWords = 28;   // dq[4] + du_fluid[4][3] + du_solid[4][3]

// Wing-frame tangent of the step the state is about to take (init: of t = 0).
void launch_frame_tangent(const GeomBuffers& gb, float dt, int init, FrameTangent* out, cudaStream_t s);
// Per-link tangents dq/dtheta and du_wall/dtheta at both link ends (mesh geometry).
void launch_link_tangent(int link_rule, int interpolated, const GridDesc& g, const FluidParams& fp,
                         const BoxDesc& box, const GeomBuffers& gb, float* out, cudaStream_t s);

// Taped data of one forward step, as the adjoint step reads it.
struct StepTape {
    const void* moments;            // R4 per real cell: pre-collision rho, u
    const uint8_t* mask_next;       // occupancy after the step (with topology flags)
    const uint8_t* mask_prev;       // occupancy before the step
    const unsigned long long* keys; // box-local mesh keys of the step
    const DeviceState* state;       // box origin, link count, step index
    const FrameTangent* frames;
    const void* links;              // LinkTape<R>[link count]
};

struct AdjointWork {
    void* lam;                      // adjoint populations, same layout as the populations
    void* nu;                       // R per link: adjoint of the bounce-back value
    double* partials_rare;          // 4 per box block
    double* partials_links;         // 4 per apply block
    Objective* objective;
};

// One reverse step: the adjoint of the forward step that took the populations
// from representation rep_s (before) to the taped state.  weight is the
// objective weight of that step (0 outside the averaging window).
void launch_adjoint_step(int storage, int rep_s, const GridDesc& g, const FluidParams& fp, const BoxDesc& box,
                         const GeomBuffers& gb, const StepTape& tape, const AdjointWork& w, double weight,
                         cudaStream_t s);
// dJ/dtheta through the initial state (the wall equilibria k_init writes into
// cells solid at t = 0); init holds the t = 0 mask (mask_next), keys, state and
// frame tangent, rep_s the representation of the initial populations.
void launch_adjoint_init(int storage, int rep_s, const GridDesc& g, const FluidParams& fp, const BoxDesc& box,
                         const GeomBuffers& gb, const StepTape& init, const AdjointWork& w, cudaStream_t s);

}  // namespace bfx

namespace bfx {
struct Grid;
Grid device_grid(const GridDesc& gd);
int box_block_count(const BoxDesc& box);
int slab_block_count(const BoxDesc& box);
void launch_fill_wall(float4* wall, int64_t n, float w, cudaStream_t s);
// Tensor map (px, py, pz, 19) of a 16-bit population array for the staged
// fused kernel, with the box of the collision operator's tile shape; false when
// the driver entry point is missing or the format is not 16-bit.
bool encode_population_map(CUtensorMap* map, void* pops, int storage, int collision, int64_t px, int64_t py,
                           int64_t pz);
// Collision operators whose 16-bit fluid step runs the staged kernel.
bool staged_collision(int collision);
// Kernel launches of one launch_bulk call.
int launch_bulk_count(int storage, int collision, int capture, bool tma_ok, bool geometry);
// Raises the staged kernel's shared-memory limit for a 16-bit storage format
// and collision operator (call before any graph capture).
void prepare_stream(int storage, int collision);
}  // namespace bfx
