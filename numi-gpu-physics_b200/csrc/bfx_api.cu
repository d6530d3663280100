// C-ABI runtime of the bfx library: owns the device buffers of one
// simulation, encodes the per-step kernel sequence on one CUDA stream, and
// implements the BirdFlowSimulation surface (Sources/BirdFlowMetal/
// BirdFlowSimulation.swift) behind plain-C entry points (include/bfx.h).
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstdio>
#include <cstring>
#include <ctime>
#include <memory>
#include <string>
#include <vector>

#include "../../include/bfx.h"
#include "bfx_internal.h"
#include "bfx_observation.h"

using namespace bfx;

namespace {

thread_local std::string g_create_error;

size_t storage_bytes(int storage) {
    switch (storage) {
    case BFX_STORAGE_F16_DEVIATION:
    case BFX_STORAGE_BF16_DEVIATION: return 2;
    case BFX_STORAGE_F64: return 8;
    default: return 4;
    }
}

uint64_t fnv1a(const void* data, size_t n, uint64_t h = 1469598103934665603ull) {
    const unsigned char* p = (const unsigned char*)data;
    for (size_t i = 0; i < n; ++i) {
        h ^= p[i];
        h *= 1099511628211ull;
    }
    return h;
}

}  // namespace

namespace bfx {
// Message returned by bfx_last_error(NULL) (entry points without a handle).
void set_global_error(const std::string& message) { g_create_error = message; }
}  // namespace bfx

struct bfx_sim {
    bfx_config cfg{};
    bfx_bird bird{};
    bool has_bird = false;
    int device = 0;
    int sm_count = 148;
    cudaStream_t stream = nullptr;
    GridDesc g{};
    FluidParams fp{};
    BoxDesc box{};
    size_t elem = 4;
    void* pops = nullptr;
    alignas(64) CUtensorMap tmap;   // population array for the staged fused kernel
    bool tma_ok = false;
    uint8_t* mask[2] = {nullptr, nullptr};
    int cur = 0;
    float4* wall = nullptr;
    float* density = nullptr;      // observation slot 0
    float4* velocity = nullptr;
    // field observation slots: density / velocity volumes (slot 0 is the pair
    // above), the slot the next capture writes, and the publication protocol
    // (shared with pending stream-ordered releases)
    static constexpr int kMaxSlots = 4;
    float* slot_density[kMaxSlots] = {};
    float4* slot_velocity[kMaxSlots] = {};
    uint8_t* slot_mask[kMaxSlots] = {};   // occupancy of the captured step (with geometry)
    float* diag_scratch = nullptr;        // flow-diagnostics staging for host outputs (lazily)
    int capture_slot = 0;
    uint32_t slot_wait_ms = 0;
    std::shared_ptr<FieldSlots<bfx_field_frame>> slots;
    DeviceState* dstate = nullptr;
    Objective* dobjective = nullptr;
    bfx_bird* dbird = nullptr;
    // mesh
    float* mesh_local = nullptr;
    uint8_t* mesh_segment = nullptr;
    bfx_joint* joints = nullptr;
    int joint_count = 0;
    float* kf_times = nullptr;     // keyframe replay (kf_count >= 2)
    float* kf_points = nullptr;
    int kf_count = 0;
    uint32_t* mesh_tris = nullptr;
    uint8_t* mesh_tri_part = nullptr;
    float4* mesh_pos = nullptr;
    float4* mesh_vel = nullptr;
    unsigned long long* keys = nullptr;
    uint32_t nverts = 0, ntris = 0;
    // links and reductions
    uint32_t* link_cell = nullptr;
    uint32_t* link_meta = nullptr;
    float* link_q = nullptr;
    uint32_t link_capacity = 0;
    uint32_t* block_counts = nullptr;
    uint32_t* block_offsets = nullptr;
    uint32_t* scan_sums = nullptr;
    uint32_t* event_counts = nullptr;
    uint32_t* event_offsets = nullptr;
    uint32_t* event_sums = nullptr;
    uint32_t* event_cell = nullptr;
    uint32_t* event_total = nullptr;
    uint32_t* live_list = nullptr;
    uint32_t* live_count = nullptr;
    uint32_t* cell_bits = nullptr;
    int box_blocks = 0;
    int scan_blocks = 0;
    double* topo_partials = nullptr;
    int topo_blocks = 0;
    double* link_partials = nullptr;
    int apply_blocks = 0;
    double* mm_partials = nullptr;
    double* mm_result = nullptr;
    int mm_blocks = 0;
    float* scratch_f32 = nullptr;  // canonical read-out staging (lazily)
    bool face_ready = false;       // the staged kernel takes the x faces' values (face_dev) without their fill
    float face_dev[2 * 19] = {};   // those values (stored deviations, host copy)
    bfx_run_sample* dsamples = nullptr;
    size_t dsamples_cap = 0;
    // state
    int rep_s = 0;
    uint64_t step = 0;
    bool invalid = false;
    bool fields_valid = false;
    std::string err;
    uint64_t launches = 0;
    uint64_t device_bytes = 0;
    // kernel timing
    bool timing = false;
    std::vector<cudaEvent_t> ev_start, ev_stop;
    size_t ev_used = 0;
    double timing_ms = 0.0;
    uint64_t timing_launches = 0;
    std::vector<void*> allocations;
    cudaEvent_t region[2] = {nullptr, nullptr};
    // CUDA graphs of two consecutive steps, keyed by the representation the
    // pair starts from (the launch sequence repeats with period two).
    cudaGraphExec_t pair_graph[2] = {nullptr, nullptr};
    uint64_t pair_launches[2] = {0, 0};
    // single steps (an odd step count, one-step calls), same keying
    cudaGraphExec_t step_graph[2] = {nullptr, nullptr};
    uint64_t step_launches[2] = {0, 0};
    // pipelined pairs: each step's geometry was built during the previous
    // step's fluid kernel, and each step builds the next one's the same way
    cudaGraphExec_t pipe_graph[2] = {nullptr, nullptr};
    uint64_t pipe_launches[2] = {0, 0};
    // side stream of the next step's geometry build, with its fork / join events
    cudaStream_t side = nullptr;
    cudaEvent_t fork_ev = nullptr, join_ev = nullptr, lists_ev = nullptr;
    cudaEvent_t halo_fork_ev = nullptr, halo_join_ev = nullptr;
    // topology record / replay test hook (bfx_test_replay_topology): 0 off,
    // 1 record each step's occupancy into topo_buf, 2 replace it from there
    int topo_mode = 0;
    uint8_t* topo_buf = nullptr;
    uint64_t topo_cap = 0;
    uint64_t topo_next = 0;
    bool graphs_enabled = true;
    // pinned host staging of the device state: read-backs and body uploads
    // without a pageable-copy bounce
    DeviceState* hstate = nullptr;
    // coupled momentum ledger partial sums (allocated on first use)
    double* ledger_in = nullptr;
    double* ledger_out = nullptr;
    int ledger_blocks = 0;
    // hstate holds the device state as of now: no launch, copy or state
    // change since it was read (the read-only entry points reuse it)
    bool hstate_fresh = false;

    bool geometry() const { return cfg.geometry != BFX_GEOMETRY_NONE; }
    bool moving() const { return geometry() && !cfg.static_geometry; }
};

namespace {

int fail(bfx_sim* s, int code, const std::string& msg) {
    if (s) {
        s->err = msg;
        if (code == BFX_ERR_KERNEL || code == BFX_ERR_SAFETY) s->invalid = true;
    } else {
        g_create_error = msg;
    }
    return code;
}

int cuda_fail(bfx_sim* s, cudaError_t e, const char* what) {
    std::string m = std::string(what) + ": " + cudaGetErrorString(e);
    if (s) {
        s->err = m;
        s->invalid = true;
    } else {
        g_create_error = m;
    }
    return e == cudaErrorMemoryAllocation ? BFX_ERR_ALLOCATION : BFX_ERR_KERNEL;
}

template <class T>
cudaError_t dalloc(bfx_sim* s, T** p, size_t bytes) {
    if (bytes == 0) bytes = 16;
    cudaError_t e = cudaMalloc((void**)p, bytes);
    if (e == cudaSuccess) {
        s->allocations.push_back((void*)*p);
        s->device_bytes += bytes;
        cudaMemsetAsync(*p, 0, bytes, s->stream);
    }
    return e;
}

FluidBuffers fluid_buffers(bfx_sim* s, uint8_t* mask) {
    FluidBuffers b;
    b.pops = s->pops;
    b.mask = mask;
    b.wall = s->wall;
    b.density = s->slot_density[s->capture_slot];
    b.velocity = s->slot_velocity[s->capture_slot];
    b.state = s->dstate;
    b.tape = nullptr;
    b.tmap = s->tma_ok ? &s->tmap : nullptr;
    b.sm_count = s->sm_count;
    b.face_dev = s->face_ready ? s->face_dev : nullptr;
    return b;
}

GeomBuffers geom_buffers(bfx_sim* s, uint8_t* mprev, uint8_t* mnext) {
    GeomBuffers b;
    b.bird = s->dbird;
    b.mask_prev = mprev;
    b.mask_next = mnext;
    b.wall = s->wall;
    b.mesh_local = s->mesh_local;
    b.mesh_segment = s->mesh_segment;
    b.joints = s->joints;
    b.joint_count = s->joint_count;
    b.kf_times = s->kf_times;
    b.kf_points = s->kf_points;
    b.kf_count = s->kf_count;
    b.mesh_tris = s->mesh_tris;
    b.mesh_tri_part = s->mesh_tri_part;
    b.mesh_pos = s->mesh_pos;
    b.mesh_vel = s->mesh_vel;
    b.keys = s->keys;
    b.nverts = s->nverts;
    b.ntris = s->ntris;
    b.half_thickness = s->cfg.mesh_half_thickness;
    b.link_cell = s->link_cell;
    b.link_meta = s->link_meta;
    b.link_q = s->link_q;
    b.link_capacity = s->link_capacity;
    b.block_counts = s->block_counts;
    b.block_offsets = s->block_offsets;
    b.scan_sums = s->scan_sums;
    b.event_counts = s->event_counts;
    b.event_offsets = s->event_offsets;
    b.event_sums = s->event_sums;
    b.event_cell = s->event_cell;
    b.event_total = s->event_total;
    // the occupancy test hook's replayed masks are not what the resolve saw
    b.live_list = s->topo_mode ? nullptr : s->live_list;
    b.live_count = s->live_count;
    b.cell_bits = s->cell_bits;
    b.box_blocks = s->box_blocks;
    b.scan_blocks = s->scan_blocks;
    b.topo_partials = s->topo_partials;
    b.topo_blocks = s->topo_blocks;
    b.link_partials = s->link_partials;
    b.apply_blocks = s->apply_blocks;
    b.state = s->dstate;
    b.objective = s->dobjective;
    b.link_tape = nullptr;
    b.link_tangent = nullptr;
    b.frames = nullptr;
    return b;
}

// Device pointers of one taped step (discrete adjoint recomputation).
struct TapeSlot {
    void* moments;
    uint8_t* mask_next;
    uint8_t* mask_prev;
    unsigned long long* keys;
    DeviceState* state;
    FrameTangent* frames;
    void* links;
    float* link_tangent;    // per-link tangent scratch shared by all slots
};

// Classification for the geometry at the current state (pose and frames,
// occupancy, wall field, mesh keys), on the simulation's stream or another.
void encode_geometry_build(bfx_sim* s, int init, uint8_t* mprev, uint8_t* mnext, cudaStream_t st = nullptr) {
    GeomBuffers gb = geom_buffers(s, mprev, mnext);
    if (!st) st = s->stream;
    launch_prepare(s->cfg.geometry, s->cfg.time_step, s->g, s->fp, s->box, gb, init, st);
    // beside the TRT staged kernel (pipelined build): the register-lean raster
    const bool lean = st == s->side && s->cfg.collision == BFX_COLLISION_TRT;
    launch_classify(s->cfg.geometry, init ? 0 : 1, s->g, s->fp, s->box, gb, st, lean);
    s->launches += 1 + (s->cfg.geometry == BFX_GEOMETRY_MESH ? 4 : 1);
}

// The next step's geometry build can overlap this step's fluid kernel: with
// the staged 16-bit kernel the fluid cells read only the populations and this
// step's mask, while the build writes the other mask buffer, the wall field,
// the keys, the pose fields and link count of the device state, and the
// cut-link and event lists (this step's link kernel has read them before the
// fork); the body update it reads is done by the link kernel before the fluid
// kernel, and the box's solid cells (which read the wall field) are launched
// before the fork.
bool can_pipeline(const bfx_sim* s) { return s->moving() && s->tma_ok && s->side != nullptr; }

// Faces f0..f1 are far-field or velocity faces: the values the halo fill
// writes there depend only on the face and the direction.
bool faces_constant(const bfx_config& c, int f0 = 0, int f1 = 5) {
    for (int f = f0; f <= f1; ++f)
        if (c.face_bc[f] != BFX_BC_FARFIELD && c.face_bc[f] != BFX_BC_VELOCITY) return false;
    return true;
}
bool x_faces_constant(const bfx_config& c) { return faces_constant(c, 0, 1); }

// The halo fill can run beside the link build and the link kernel when every
// face is a far-field or velocity face: the fill then only writes constants
// into halo slots, which no link kernel reads or writes (an out-of-domain
// cell is never solid), and reads nothing they write.  A periodic face's fill
// copies real cells that a link may overwrite, an outflow face's copies its
// interior neighbour, and a link whose solid source is a periodic image writes
// a halo slot: those keep the fill first on the main stream.
bool halo_beside_links(const bfx_sim* s) {
    return s->moving() && s->side != nullptr && faces_constant(s->cfg);
}

// The cut-link and topology-event lists of a step's geometry, on the
// simulation's stream or (pipelined path) the side stream beside the previous
// step's fluid kernel.
void encode_link_build(bfx_sim* s, uint8_t* mprev, uint8_t* mnext, cudaStream_t st, cudaEvent_t lists_done = nullptr) {
    launch_link_build(s->cfg.geometry, s->cfg.link_rule, s->g, s->fp, s->box, geom_buffers(s, mprev, mnext), st,
                      lists_done);
    s->launches += 5;
}
// The topology impulses of the step's events: they read the pre-step
// populations, so they follow the previous step's fluid kernel and precede
// this step's link kernel on the simulation's stream.
void encode_topology(bfx_sim* s, uint8_t* mprev, uint8_t* mnext) {
    launch_topology(s->cfg.storage, s->rep_s, s->g, s->fp, s->box, geom_buffers(s, mprev, mnext),
                    fluid_buffers(s, mnext), s->stream);
    s->launches += 1;
}
void encode_links(bfx_sim* s, uint8_t* mprev, uint8_t* mnext) {
    encode_link_build(s, mprev, mnext, s->stream);
    if (s->moving()) encode_topology(s, mprev, mnext);
}

void timing_begin(bfx_sim* s) {
    if (!s->timing) return;
    if (s->ev_used >= s->ev_start.size()) {
        cudaEvent_t a, b;
        cudaEventCreate(&a);
        cudaEventCreate(&b);
        s->ev_start.push_back(a);
        s->ev_stop.push_back(b);
    }
    cudaEventRecord(s->ev_start[s->ev_used], s->stream);
}
void timing_end(bfx_sim* s) {
    if (!s->timing) return;
    cudaEventRecord(s->ev_stop[s->ev_used], s->stream);
    ++s->ev_used;
}
void timing_collect(bfx_sim* s) {
    for (size_t i = 0; i < s->ev_used; ++i) {
        float ms = 0.0f;
        if (cudaEventElapsedTime(&ms, s->ev_start[i], s->ev_stop[i]) == cudaSuccess) {
            s->timing_ms += ms;
            s->timing_launches += 1;
        }
    }
    s->ev_used = 0;
}

// One time step (BirdFlowSimulation.encodeBatch body, BirdFlowSimulation.swift:1374-1437).
// With a tape slot the step also records what its adjoint needs: the wing-frame
// and link tangents, the link values, masks, keys, state and pre-collision moments.
// geometry_ready: this step's geometry was built by the previous step's
// prefetch.  prefetch_next: build the next step's geometry on the side stream
// while this step's fluid kernel runs (can_pipeline; no capture, tape or ledger).
void encode_step(bfx_sim* s, int capture, bfx_run_sample* sample_slot_base, uint64_t sample_index,
                 const TapeSlot* tape = nullptr, double* ledger_in = nullptr, bool geometry_ready = false,
                 bool prefetch_next = false) {
    s->hstate_fresh = false;
    uint8_t* mprev = s->mask[s->cur];
    uint8_t* mnext = s->moving() ? s->mask[s->cur ^ 1] : s->mask[s->cur];
    FluidBuffers fb = fluid_buffers(s, s->geometry() ? mnext : nullptr);
    // The halo fill forks off here (after the previous step's fluid kernel)
    // and joins before this step's fluid kernel; without the x faces when
    // the staged kernel takes their values from its table
    const bool yz_only = s->face_ready && bulk_staged(s->cfg.storage, s->cfg.collision, tape ? 2 : capture, s->tma_ok);
    const bool halo_side = halo_beside_links(s) && !tape && !ledger_in;
    if (halo_side) {
        cudaEventRecord(s->halo_fork_ev, s->stream);
        cudaStreamWaitEvent(s->side, s->halo_fork_ev, 0);
        if (yz_only) launch_halo_yz(s->cfg.storage, s->rep_s, s->g, s->fp, fb, s->side);
        else launch_halo(s->cfg.storage, s->rep_s, s->g, s->fp, fb, s->side);
        cudaEventRecord(s->halo_join_ev, s->side);
        s->launches += 1;
    }
    if (s->moving() && !geometry_ready) {
        encode_geometry_build(s, 0, mprev, mnext);
    }
    if (s->topo_mode && s->moving() && !tape) {
        // the test hook's record / replay of the step's occupancy (direct steps only)
        const uint64_t i = s->topo_next++;
        if (i < s->topo_cap) {
            uint8_t* rec = s->topo_buf + i * (size_t)s->g.n;
            if (s->topo_mode == 1) cudaMemcpyAsync(rec, mnext, (size_t)s->g.n, cudaMemcpyDeviceToDevice, s->stream);
            else cudaMemcpyAsync(mnext, rec, (size_t)s->g.n, cudaMemcpyDeviceToDevice, s->stream);
        }
    }
    if (tape) {
        launch_frame_tangent(geom_buffers(s, mprev, mnext), s->cfg.time_step, 0, tape->frames, s->stream);
        s->launches += 1;
    }
    // geometry_ready: the previous step built this step's cut-link and event
    // lists with its geometry and ran its topology impulses
    if (s->geometry() && s->moving() && !geometry_ready) encode_links(s, mprev, mnext);
    if (tape) {
        GeomBuffers gb = geom_buffers(s, mprev, mnext);
        gb.frames = tape->frames;
        launch_link_tangent(s->cfg.link_rule, s->fp.interpolated, s->g, s->fp, s->box, gb, tape->link_tangent,
                            s->stream);
        s->launches += 1;
    }
    if (ledger_in) {
        // the ledger's pre-step pass: geometry built, no population written yet
        launch_ledger_in(s->cfg.storage, s->rep_s, s->g, s->fp, fb, s->geometry() ? mprev : nullptr,
                         s->geometry() ? mnext : nullptr, ledger_in, s->ledger_blocks, s->stream);
        s->launches += 1;
    }
    // halo fill before the link writes: a link whose solid source is a periodic
    // image writes into a halo slot and must win over the periodic copy
    if (!halo_side) {
        if (yz_only) launch_halo_yz(s->cfg.storage, s->rep_s, s->g, s->fp, fb, s->stream);
        else launch_halo(s->cfg.storage, s->rep_s, s->g, s->fp, fb, s->stream);
        s->launches += 1;
    }
    // The end-of-step body update needs only the reduced loads: it runs in the
    // link kernel's last block, except while taping (the tape records the
    // state between the loads and the body update).
    const FinishParams fin = {{s->cfg.gravity[0], s->cfg.gravity[1], s->cfg.gravity[2]}, (int)s->cfg.body_substeps,
                              s->cfg.free_flight && s->has_bird ? 1 : 0};
    const bool finish_fused = s->geometry() && !tape;
    if (s->geometry()) {
        GeomBuffers gb = geom_buffers(s, mprev, mnext);
        if (tape) {
            gb.link_tape = tape->links;
            gb.link_tangent = tape->link_tangent;
        }
        launch_links_apply(s->cfg.storage, s->rep_s, s->g, s->fp, gb, fb, s->moving() ? 1 : 0,
                           finish_fused ? &fin : nullptr, s->stream);
        s->launches += 1;
    }
    const bool pipelined = prefetch_next && capture == 0 && !tape && !ledger_in && can_pipeline(s);
    const int box[3] = {s->box.sx, s->box.sy, s->box.sz};
    if (pipelined) {
        // The solid / uncovered cells right after the link kernel, beside the
        // halo fill: they write only their own slots, which no fluid cell
        // reads or writes, and read the wall field, which the next step's
        // geometry rewrites after the fork below.
        launch_bulk_rare(s->cfg.storage, s->cfg.collision, s->rep_s, s->g, s->fp, fb, box, s->stream);
    }
    if (halo_side) cudaStreamWaitEvent(s->stream, s->halo_join_ev, 0);
    if (tape) {
        cudaMemcpyAsync(tape->state, s->dstate, sizeof(DeviceState), cudaMemcpyDeviceToDevice, s->stream);
        cudaMemcpyAsync(tape->mask_next, mnext, (size_t)s->g.n, cudaMemcpyDeviceToDevice, s->stream);
        cudaMemcpyAsync(tape->mask_prev, mprev, (size_t)s->g.n, cudaMemcpyDeviceToDevice, s->stream);
        cudaMemcpyAsync(tape->keys, s->keys, (size_t)s->box.cells * sizeof(unsigned long long),
                        cudaMemcpyDeviceToDevice, s->stream);
        fb.tape = tape->moments;
        capture = 2;
    }
    if (pipelined) {
        // Beside the fluid kernel, on the side stream: the next step's
        // geometry (masks swap roles) and its cut-link and event lists.
        cudaEventRecord(s->fork_ev, s->stream);
        cudaStreamWaitEvent(s->side, s->fork_ev, 0);
        encode_geometry_build(s, 0, mnext, mprev, s->side);
        if (s->geometry()) encode_link_build(s, mnext, mprev, s->side, s->lists_ev);
        else cudaEventRecord(s->lists_ev, s->side);
        cudaEventRecord(s->join_ev, s->side);
        launch_bulk_stream(s->cfg.storage, s->cfg.collision, s->rep_s, s->g, s->fp, fb, box, s->stream);
    } else {
        timing_begin(s);
        launch_bulk(s->cfg.storage, s->cfg.collision, s->rep_s, s->g, s->fp, fb, capture,
                    s->geometry() ? box : nullptr, s->stream);
        timing_end(s);
    }
    s->launches += launch_bulk_count(s->cfg.storage, s->cfg.collision, capture, s->tma_ok, s->geometry());
    GeomBuffers gb = geom_buffers(s, mprev, mnext);
    if (!finish_fused) {
        launch_integrate(s->g, s->fp, gb, fin.gravity[0], fin.gravity[1], fin.gravity[2], fin.substeps,
                         fin.free_flight, s->stream);
        s->launches += 1;
    }
    if (sample_slot_base) {
        launch_record_sample(gb, s->fp, sample_slot_base, sample_index, s->cfg.time_step, s->stream);
        s->launches += 1;
    }
    s->rep_s ^= 1;
    if (s->moving()) s->cur ^= 1;
    if (pipelined) {
        // The next step's topology impulses, as soon as its event list is
        // written (they read the populations after this step's fluid kernel,
        // before the next link kernel), beside its link fractions; then the
        // join.  Inside this step's encoding, so a captured graph holds both.
        cudaStreamWaitEvent(s->stream, s->lists_ev, 0);
        if (s->geometry()) encode_topology(s, s->mask[s->cur], s->mask[s->cur ^ 1]);
        cudaStreamWaitEvent(s->stream, s->join_ev, 0);
    }
}

// Replays (capturing on first use) the graph of `nsteps` (1 or 2) plain steps
// for the current parity.  Host-side state (representation, mask index)
// alternates with period two, so a pair graph leaves it where it started and
// the single-step graph of each parity hands over to the other's.  A pipelined
// pair takes its first step's geometry as built and builds the geometry of the
// step after the pair (so one more step of the same batch must follow).
int run_steps_graph(bfx_sim* s, int nsteps, bool pipelined = false) {
    s->hstate_fresh = false;
    const int key = s->rep_s;
    cudaGraphExec_t* slot = pipelined ? &s->pipe_graph[key] : nsteps == 2 ? &s->pair_graph[key] : &s->step_graph[key];
    uint64_t* count =
        pipelined ? &s->pipe_launches[key] : nsteps == 2 ? &s->pair_launches[key] : &s->step_launches[key];
    if (!*slot) {
        const int rep0 = s->rep_s, cur0 = s->cur;
        cudaGraph_t graph = nullptr;
        uint64_t before = s->launches;
        cudaError_t e = cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal);
        if (e != cudaSuccess) return cuda_fail(s, e, "graph capture begin");
        for (int i = 0; i < nsteps; ++i) encode_step(s, 0, nullptr, 0, nullptr, nullptr, pipelined, pipelined);
        e = cudaStreamEndCapture(s->stream, &graph);
        if (e != cudaSuccess) return cuda_fail(s, e, "graph capture end");
        // kernel nodes keep the priority of the stream they were captured on
        e = cudaGraphInstantiate(slot, graph, cudaGraphInstantiateFlagUseNodePriority);
        cudaGraphDestroy(graph);
        if (e != cudaSuccess) return cuda_fail(s, e, "graph instantiate");
        *count = s->launches - before;
        s->launches = before;
        // capture only recorded the steps: the host state advances at launch
        s->rep_s = rep0;
        s->cur = cur0;
    }
    cudaError_t e = cudaGraphLaunch(*slot, s->stream);
    if (e != cudaSuccess) return cuda_fail(s, e, "graph launch");
    s->launches += *count;
    for (int i = 0; i < nsteps; ++i) {
        s->rep_s ^= 1;
        if (s->moving()) s->cur ^= 1;
    }
    return BFX_OK;
}
int run_pair_graph(bfx_sim* s) { return run_steps_graph(s, 2); }

int sync_check(bfx_sim* s, const char* what) {
    cudaError_t e = cudaStreamSynchronize(s->stream);
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(s, e, what);
    timing_collect(s);
    return BFX_OK;
}

int validate_config(const bfx_config* c, const bfx_bird* bird, const bfx_mesh* mesh) {
    if (c->nx < 4 || c->ny < 4 || c->nz < 4) return fail(nullptr, BFX_ERR_INVALID_CONFIG, "each grid dimension must be at least 4 cells");
    uint64_t n = (uint64_t)c->nx * c->ny * c->nz;
    if (n > 0xFFFFFFFFull) return fail(nullptr, BFX_ERR_INVALID_CONFIG, "the total cell count must fit in 32 bits");
    for (int a = 0; a < 3; ++a) {
        int lo = c->face_bc[2 * a], hi = c->face_bc[2 * a + 1];
        if (lo < 0 || lo > 3 || hi < 0 || hi > 3)
            return fail(nullptr, BFX_ERR_INVALID_CONFIG, "face boundary rule out of range");
        if ((lo == BFX_BC_PERIODIC) != (hi == BFX_BC_PERIODIC))
            return fail(nullptr, BFX_ERR_INVALID_CONFIG, "a periodic axis needs both faces periodic");
    }
    if (c->collision < 0 || c->collision > 3) return fail(nullptr, BFX_ERR_INVALID_CONFIG, "unknown collision operator");
    if (c->storage < 0 || c->storage > 3) return fail(nullptr, BFX_ERR_INVALID_CONFIG, "unknown storage format");
    if (c->geometry < 0 || c->geometry > 4) return fail(nullptr, BFX_ERR_INVALID_CONFIG, "unknown geometry kind");
    if (c->wall_rule < 0 || c->wall_rule > 1) return fail(nullptr, BFX_ERR_INVALID_CONFIG, "unknown wall rule");
    if (c->force_estimator < 0 || c->force_estimator > 6)
        return fail(nullptr, BFX_ERR_INVALID_CONFIG, "force estimator must be 0...6");
    if (c->load_component < 0 || c->load_component > 2)
        return fail(nullptr, BFX_ERR_INVALID_CONFIG, "load component must be 0, 1 or 2");
    if (c->selected_part < 0 || c->selected_part > 63) return fail(nullptr, BFX_ERR_INVALID_CONFIG, "selected part out of range");
    if (!(c->omega_plus > 0.0f && c->omega_plus < 2.0f) || !(c->omega_minus > 0.0f && c->omega_minus < 2.0f))
        return fail(nullptr, BFX_ERR_INVALID_CONFIG, "relaxation rates must lie in (0, 2)");
    if (!(c->cell_size > 0.0f) || !(c->time_step > 0.0f))
        return fail(nullptr, BFX_ERR_INVALID_CONFIG, "cell size and time step must be positive");
    if (!(c->sponge_strength >= 0.0f && c->sponge_strength <= 1.0f))
        return fail(nullptr, BFX_ERR_INVALID_CONFIG, "sponge strength must be in [0, 1]");
    if (c->body_substeps < 1 || c->body_substeps > 64)
        return fail(nullptr, BFX_ERR_INVALID_CONFIG, "bodySubsteps must be in 1...64");
    float far2 = c->far_field[0] * c->far_field[0] + c->far_field[1] * c->far_field[1] + c->far_field[2] * c->far_field[2];
    if (std::sqrt(far2) / std::sqrt(1.0f / 3.0f) > 0.15f)
        return fail(nullptr, BFX_ERR_INVALID_CONFIG, "far-field lattice Mach number above 0.15");
    if (c->geometry != BFX_GEOMETRY_NONE && bird == nullptr)
        return fail(nullptr, BFX_ERR_INVALID_CONFIG, "a geometry needs bird parameters");
    if (c->geometry == BFX_GEOMETRY_MESH && (mesh == nullptr || mesh->triangle_count == 0 || mesh->vertex_count == 0))
        return fail(nullptr, BFX_ERR_INVALID_CONFIG, "mesh geometry needs a non-empty mesh");
    if (c->geometry == BFX_GEOMETRY_BIRD && c->wall_rule == BFX_WALL_INTERPOLATED)
        return fail(nullptr, BFX_ERR_INVALID_CONFIG, "the analytic bird provides halfway links only");
    if (c->geometry == BFX_GEOMETRY_MESH && !(c->mesh_half_thickness > 0.0f))
        return fail(nullptr, BFX_ERR_INVALID_CONFIG, "mesh half thickness must be positive");
    if (c->free_flight && bird == nullptr) return fail(nullptr, BFX_ERR_INVALID_CONFIG, "free flight needs bird parameters");
    if (bird && bird->wing_kinematics1.v[3] > 0.5f)
        return fail(nullptr, BFX_ERR_INVALID_CONFIG, "measured keyframe kinematics are not supported");
    if (c->free_flight && c->static_geometry)
        return fail(nullptr, BFX_ERR_INVALID_CONFIG, "a free-flying body cannot be static geometry");
    if (c->geometry == BFX_GEOMETRY_FLAPPING_WING && c->free_flight)
        return fail(nullptr, BFX_ERR_INVALID_CONFIG, "the prescribed flapping wing is held at its root (no free flight)");
    if (mesh && mesh->triangles) {
        for (uint32_t i = 0; i < 3 * mesh->triangle_count; ++i)
            if (mesh->triangles[i] >= mesh->vertex_count)
                return fail(nullptr, BFX_ERR_INVALID_CONFIG, "triangle index out of range");
        if (mesh->joint_count > 2 || (mesh->joint_count > 0 && mesh->joints == nullptr))
            return fail(nullptr, BFX_ERR_INVALID_CONFIG, "a mesh has at most two joints (elbow, wrist)");
        const uint32_t max_segment = 2 + 2 * mesh->joint_count;
        for (uint32_t i = 0; i < mesh->vertex_count; ++i)
            if (mesh->vertex_segment[i] > max_segment)
                return fail(nullptr, BFX_ERR_INVALID_CONFIG, "vertex segment exceeds the mesh's joint chain");
        for (uint32_t j = 0; j < mesh->joint_count; ++j) {
            const float* ax = mesh->joints[j].axis;
            const float n2 = ax[0] * ax[0] + ax[1] * ax[1] + ax[2] * ax[2];
            if (!(std::fabs(n2 - 1.0f) < 1.0e-4f))
                return fail(nullptr, BFX_ERR_INVALID_CONFIG, "joint axis must be a unit vector");
        }
        for (uint32_t i = 0; i < mesh->triangle_count; ++i)
            if (mesh->triangle_part[i] == 0 || mesh->triangle_part[i] > 63)
                return fail(nullptr, BFX_ERR_INVALID_CONFIG, "triangle part must be 1...63");
        if (mesh->keyframe_count > 0) {
            if (mesh->keyframe_count < 2 || !mesh->keyframe_times || !mesh->keyframe_points)
                return fail(nullptr, BFX_ERR_INVALID_CONFIG, "a keyframe replay needs at least two frames with times and points");
            if (mesh->joint_count != 0)
                return fail(nullptr, BFX_ERR_INVALID_CONFIG, "a keyframe replay takes no joints");
            for (uint32_t i = 0; i < mesh->vertex_count; ++i)
                if (mesh->vertex_segment[i] != 0)
                    return fail(nullptr, BFX_ERR_INVALID_CONFIG, "keyframed vertices belong to segment 0 (the body)");
            for (uint32_t f = 0; f < mesh->keyframe_count; ++f) {
                if (!std::isfinite(mesh->keyframe_times[f]) ||
                    (f > 0 && !(mesh->keyframe_times[f] > mesh->keyframe_times[f - 1])))
                    return fail(nullptr, BFX_ERR_INVALID_CONFIG, "keyframe times must be finite and strictly increasing");
            }
            const size_t np = (size_t)mesh->keyframe_count * mesh->vertex_count * 3;
            for (size_t k = 0; k < np; ++k)
                if (!std::isfinite(mesh->keyframe_points[k]))
                    return fail(nullptr, BFX_ERR_INVALID_CONFIG, "keyframe points must be finite");
        }
    }
    return BFX_OK;
}

// Conservative radius (m) of everything the geometry kernels may mark solid,
// measured from the body origin.
float geometry_radius(const bfx_config* c, const bfx_bird* b, const bfx_mesh* m) {
    const float* br = b->body_radii_mass.v;
    const float* tg = b->tail_geometry.v;
    const float* w0 = b->wing_geometry0.v;
    const float* w1 = b->wing_geometry1.v;
    float body = std::sqrt(br[0] * br[0] + br[1] * br[1] + br[2] * br[2]);
    if (c->geometry == BFX_GEOMETRY_ELLIPSOID) return std::max(br[0], std::max(br[1], br[2])) + 2.0f * c->cell_size;
    // the prescribed wing's bounding sphere about its root (buildPrescribedFlappingWing, BF.metal:1203-1206)
    if (c->geometry == BFX_GEOMETRY_FLAPPING_WING) return w1[0] + 1.5f * w0[3] + 2.0f * c->cell_size;
    float root = std::sqrt(w1[1] * w1[1] + w1[2] * w1[2] + w1[3] * w1[3]);
    if (c->geometry == BFX_GEOMETRY_BIRD) {
        float tx = br[0] + tg[0], ty = std::max(br[1], tg[1]), tz = br[2] + 0.5f * tg[2];
        float tail = std::sqrt(tx * tx + ty * ty + tz * tz);
        float wing = root + w0[0] + std::fabs(w1[0]) + 0.5f * std::max(w0[1], w0[2]) + 0.5f * w0[3];
        return std::max(body, std::max(tail, wing)) + 2.0f * c->cell_size;
    }
    // joint chain: a segment's vertices lie within the sum of the joint offsets
    // before it plus their own offset from the joint
    float chain[3] = {0.0f, 0.0f, 0.0f};
    for (uint32_t j = 0; j < m->joint_count && j < 2; ++j) {
        const float* o = m->joints[j].origin;
        chain[j + 1] = chain[j] + std::sqrt(o[0] * o[0] + o[1] * o[1] + o[2] * o[2]);
    }
    float r = 0.0f;
    if (m->keyframe_count >= 2) {
        // keyframe replay: every frame's offsets (the interpolation stays inside their hull)
        const size_t np = (size_t)m->keyframe_count * m->vertex_count;
        for (size_t i = 0; i < np; ++i) {
            const float* l = m->keyframe_points + 3 * i;
            r = std::max(r, std::sqrt(l[0] * l[0] + l[1] * l[1] + l[2] * l[2]));
        }
        return r + c->mesh_half_thickness + 2.0f * c->cell_size;
    }
    for (uint32_t i = 0; i < m->vertex_count; ++i) {
        const float* l = m->local_vertices + 3 * i;
        float d = std::sqrt(l[0] * l[0] + l[1] * l[1] + l[2] * l[2]);
        const int seg = m->vertex_segment[i];
        if (seg != 0) d += root + chain[(seg - 1) / 2];
        r = std::max(r, d);
    }
    return r + c->mesh_half_thickness + 2.0f * c->cell_size;
}

}  // namespace

extern "C" {

const char* bfx_version(void) { return "bfx 0.1.0 (sm_100a)"; }
int bfx_abi_version(void) { return BFX_ABI_VERSION; }

int bfx_device_count(int* count) {
    if (!count) return BFX_ERR_INVALID_ARGUMENT;
    int c = 0;
    cudaError_t e = cudaGetDeviceCount(&c);
    *count = e == cudaSuccess ? c : 0;
    return e == cudaSuccess ? BFX_OK : BFX_ERR_DEVICE_UNAVAILABLE;
}

static int read_state(bfx_sim* s, DeviceState* st);
static bfx_field_frame field_frame_meta(const bfx_sim* s, const DeviceState& st, int slot);
static int copy_slot(bfx_sim* s, int slot, float* density, float* velocity_xyz);
static int snapshot_slot_mask(bfx_sim* s, int slot);

void bfx_destroy(bfx_sim* s) {
    if (!s) return;
    if (s->stream) {
        cudaSetDevice(s->device);
        cudaStreamSynchronize(s->stream);
    }
    for (void* p : s->allocations) cudaFree(p);
    for (auto e : s->ev_start) cudaEventDestroy(e);
    for (auto e : s->ev_stop) cudaEventDestroy(e);
    for (auto e : s->region)
        if (e) cudaEventDestroy(e);
    for (auto g : s->pair_graph)
        if (g) cudaGraphExecDestroy(g);
    for (auto g : s->step_graph)
        if (g) cudaGraphExecDestroy(g);
    for (auto g : s->pipe_graph)
        if (g) cudaGraphExecDestroy(g);
    if (s->fork_ev) cudaEventDestroy(s->fork_ev);
    if (s->join_ev) cudaEventDestroy(s->join_ev);
    if (s->lists_ev) cudaEventDestroy(s->lists_ev);
    if (s->halo_fork_ev) cudaEventDestroy(s->halo_fork_ev);
    if (s->halo_join_ev) cudaEventDestroy(s->halo_join_ev);
    if (s->side) cudaStreamDestroy(s->side);
    if (s->hstate) cudaFreeHost(s->hstate);
    if (s->stream) cudaStreamDestroy(s->stream);
    delete s;
}

int bfx_create(const bfx_config* config, const bfx_bird* bird, const bfx_body_state* body, const bfx_mesh* mesh,
               bfx_sim** out) {
    if (!config || !out) return fail(nullptr, BFX_ERR_INVALID_ARGUMENT, "config and out must not be null");
    *out = nullptr;
    int rc = validate_config(config, bird, mesh);
    if (rc != BFX_OK) return rc;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
        return fail(nullptr, BFX_ERR_DEVICE_UNAVAILABLE, "no CUDA device is available");
    if (config->device < 0 || config->device >= ndev)
        return fail(nullptr, BFX_ERR_DEVICE_UNAVAILABLE, "CUDA device ordinal out of range");

    bfx_sim* s = new bfx_sim();
    s->cfg = *config;
    s->device = config->device;
    cudaSetDevice(s->device);
    cudaDeviceGetAttribute(&s->sm_count, cudaDevAttrMultiProcessorCount, s->device);
    // The main stream (fluid kernel, link build) has the device's greatest
    // priority and the side stream (the next step's geometry, the halo fill)
    // its least: when both have blocks waiting, the persistent fluid kernel's
    // CTAs are placed first and the side kernels fill the resources it leaves.
    int least_priority = 0, greatest_priority = 0;
    if (cudaDeviceGetStreamPriorityRange(&least_priority, &greatest_priority) != cudaSuccess) {
        (void)cudaGetLastError();
        least_priority = greatest_priority = 0;
    }
    cudaError_t e = cudaStreamCreateWithPriority(&s->stream, cudaStreamNonBlocking, greatest_priority);
    if (e != cudaSuccess) {
        bfx_destroy(s);
        return cuda_fail(nullptr, e, "stream creation");
    }
    // side stream for the pipelined geometry build (optional: without it the
    // steps run in order on the main stream)
    if (cudaStreamCreateWithPriority(&s->side, cudaStreamNonBlocking, least_priority) != cudaSuccess ||
        cudaEventCreateWithFlags(&s->fork_ev, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&s->join_ev, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&s->lists_ev, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&s->halo_fork_ev, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&s->halo_join_ev, cudaEventDisableTiming) != cudaSuccess) {
        (void)cudaGetLastError();
        if (s->side) cudaStreamDestroy(s->side);
        s->side = nullptr;
    }
    if (bird) {
        s->bird = *bird;
        s->has_bird = true;
    }
    const bfx_config& c = s->cfg;
    // grid
    GridDesc& g = s->g;
    g.nx = (int)c.nx;
    g.ny = (int)c.ny;
    g.nz = (int)c.nz;
    g.per_x = c.face_bc[0] == BFX_BC_PERIODIC;
    g.per_y = c.face_bc[2] == BFX_BC_PERIODIC;
    g.per_z = c.face_bc[4] == BFX_BC_PERIODIC;
    g.n = (int64_t)g.nx * g.ny * g.nz;
    g.nxy = (int64_t)g.nx * g.ny;
    g.px = ((g.nx + 2 + 7) / 8) * 8;
    g.padded = (int64_t)g.px * (g.ny + 2) * (g.nz + 2);
    // fluid parameters
    FluidParams& fp = s->fp;
    for (int k = 0; k < 3; ++k) fp.origin[k] = c.origin[k];
    fp.dx = c.cell_size;
    fp.dt = c.time_step;
    fp.v2l = c.velocity_to_lattice;
    fp.f2p = c.force_to_physical;
    fp.omega_p = c.omega_plus;
    fp.omega_m = c.omega_minus;
    fp.sponge_strength = c.sponge_strength;
    fp.sponge_width = c.sponge_width;
    for (int k = 0; k < 4; ++k) fp.far[k] = c.far_field[k];
    fp.any_outflow = 0;
    for (int f = 0; f < 6; ++f) {
        fp.face_bc[f] = c.face_bc[f];
        for (int k = 0; k < 3; ++k) fp.face_u[f][k] = c.face_velocity[f][k];
        if (c.face_bc[f] == BFX_BC_OUTFLOW) fp.any_outflow = 1;
    }
    fp.collision = c.collision;
    fp.interpolated = c.wall_rule == BFX_WALL_INTERPOLATED;
    fp.load_component = c.load_component;
    fp.force_mode = c.force_estimator;
    fp.selected_part = c.selected_part;
    fp.local_density = c.moving_wall_local_density ? 1 : 0;
    fp.accumulate = c.accumulate_loads ? 1 : 0;
    fp.has_sponge = c.sponge_strength > 0.0f ? 1 : 0;
    fp.fast_math = c.fast_math ? 1 : 0;
    // A mesh touches cells within the raster guard (half thickness + 2 cells)
    // of its vertices' bounding box; three more cells cover the cells solid or
    // flagged in the two previous steps (bounded motion, Mach <= 0.25).
    fp.act_margin = c.geometry == BFX_GEOMETRY_MESH
                        ? (int)std::ceil(c.mesh_half_thickness / c.cell_size) + 2 + 3
                        : 0;

    s->elem = storage_bytes(c.storage);
    size_t pop_bytes = (size_t)19 * (size_t)g.padded * s->elem;
#define BFX_ALLOC(ptr, bytes)                                   \
    do {                                                        \
        cudaError_t ee = dalloc(s, &(ptr), (bytes));            \
        if (ee != cudaSuccess) {                                \
            int code = cuda_fail(nullptr, ee, "device allocation"); \
            bfx_destroy(s);                                     \
            return code;                                        \
        }                                                       \
    } while (0)
    BFX_ALLOC(s->pops, pop_bytes);
    std::memset(&s->tmap, 0, sizeof(s->tmap));
    s->tma_ok = (c.storage == BFX_STORAGE_F16_DEVIATION || c.storage == BFX_STORAGE_BF16_DEVIATION) &&
                staged_collision(c.collision) &&
                encode_population_map(&s->tmap, s->pops, c.storage, c.collision, g.px, g.ny + 2, g.nz + 2);
    if (s->tma_ok) prepare_stream(c.storage, c.collision);
    // Both x faces far-field or velocity faces: what the halo fill writes
    // there depends on the face and the direction only, so the staged kernel
    // takes it from a table and its steps skip the x faces' fill (one
    // scattered store per lattice row and direction).
    if (s->tma_ok && x_faces_constant(c)) {
        float* dvals = nullptr;
        BFX_ALLOC(dvals, sizeof(s->face_dev));
        launch_halo_values(c.storage, s->g, s->fp, dvals, s->stream);
        cudaError_t fe = cudaMemcpyAsync(s->face_dev, dvals, sizeof(s->face_dev), cudaMemcpyDeviceToHost, s->stream);
        if (fe == cudaSuccess) fe = cudaStreamSynchronize(s->stream);
        if (fe != cudaSuccess) {
            int code = cuda_fail(nullptr, fe, "face values");
            bfx_destroy(s);
            return code;
        }
        s->face_ready = true;
    }
    BFX_ALLOC(s->density, (size_t)g.n * sizeof(float));
    BFX_ALLOC(s->velocity, (size_t)g.n * sizeof(float4));
    s->slot_density[0] = s->density;
    s->slot_velocity[0] = s->velocity;
    if (c.geometry != BFX_GEOMETRY_NONE) BFX_ALLOC(s->slot_mask[0], (size_t)g.n);
    s->slots = std::make_shared<FieldSlots<bfx_field_frame>>(1);
    BFX_ALLOC(s->dstate, sizeof(DeviceState));
    if (cudaMallocHost((void**)&s->hstate, sizeof(DeviceState)) != cudaSuccess) {
        (void)cudaGetLastError();
        s->hstate = nullptr;  // pageable copies instead
    }
    BFX_ALLOC(s->dobjective, sizeof(Objective));
    s->mm_blocks = 4 * s->sm_count;
    BFX_ALLOC(s->mm_partials, (size_t)s->mm_blocks * 4 * sizeof(double));
    BFX_ALLOC(s->mm_result, 4 * sizeof(double));

    // host-side initial device state
    DeviceState hs;
    std::memset(&hs, 0, sizeof(hs));
    hs.body[6] = 1.0;
    if (body) {
        for (int k = 0; k < 3; ++k) hs.body[k] = body->position[k];
        for (int k = 0; k < 4; ++k) hs.body[3 + k] = body->orientation[k];
        for (int k = 0; k < 3; ++k) hs.body[7 + k] = body->velocity[k];
        for (int k = 0; k < 3; ++k) hs.body[10 + k] = body->omega_body[k];
    }
    hs.safety_metrics[0] = 0.0f;
    hs.safety_metrics[1] = INFINITY;

    if (s->geometry()) {
        BFX_ALLOC(s->mask[0], (size_t)g.n);
        BFX_ALLOC(s->mask[1], (size_t)g.n);
        BFX_ALLOC(s->wall, (size_t)g.n * sizeof(float4));
        BFX_ALLOC(s->dbird, sizeof(bfx_bird));
        cudaMemcpyAsync(s->dbird, &s->bird, sizeof(bfx_bird), cudaMemcpyHostToDevice, s->stream);
        // geometry box
        float r = geometry_radius(&c, &s->bird, mesh);
        int half = (int)std::ceil(r / c.cell_size) + 4;
        int ext = 2 * half + 2;
        s->box.sx = std::min(ext, g.nx);
        s->box.sy = std::min(ext, g.ny);
        s->box.sz = std::min(ext, g.nz);
        s->box.cells = (int64_t)s->box.sx * s->box.sy * s->box.sz;
        s->box_blocks = box_block_count(s->box);
        s->scan_blocks = s->box_blocks;
        BFX_ALLOC(s->block_counts, (size_t)s->box_blocks * sizeof(uint32_t));
        BFX_ALLOC(s->block_offsets, (size_t)s->box_blocks * sizeof(uint32_t));
        const size_t nseg = (size_t)((s->box_blocks + kScanSegment - 1) / kScanSegment);
        BFX_ALLOC(s->scan_sums, nseg * sizeof(uint32_t));
        BFX_ALLOC(s->event_counts, (size_t)s->box_blocks * sizeof(uint32_t));
        BFX_ALLOC(s->event_offsets, (size_t)s->box_blocks * sizeof(uint32_t));
        BFX_ALLOC(s->event_sums, nseg * sizeof(uint32_t));
        BFX_ALLOC(s->event_cell, (size_t)s->box.cells * sizeof(uint32_t));
        BFX_ALLOC(s->event_total, sizeof(uint32_t));
        BFX_ALLOC(s->cell_bits, (size_t)s->box.cells * sizeof(uint32_t));
        if (c.geometry == BFX_GEOMETRY_MESH) {
            BFX_ALLOC(s->live_list, (size_t)s->box_blocks * sizeof(uint32_t));
            BFX_ALLOC(s->live_count, sizeof(uint32_t));
            cudaMemsetAsync(s->live_count, 0, sizeof(uint32_t), s->stream);
        }
        cudaMemsetAsync(s->event_total, 0, sizeof(uint32_t), s->stream);
        s->topo_blocks = s->sm_count;
        BFX_ALLOC(s->topo_partials, (size_t)s->topo_blocks * 8 * sizeof(double));
        cudaMemsetAsync(s->topo_partials, 0, (size_t)s->topo_blocks * 8 * sizeof(double), s->stream);
        s->apply_blocks = 4 * s->sm_count;
        BFX_ALLOC(s->link_partials, (size_t)s->apply_blocks * 16 * sizeof(double));
        uint64_t cap = c.link_capacity ? c.link_capacity
                                       : std::max<uint64_t>(1u << 18, std::min<uint64_t>((uint64_t)s->box.cells, 1u << 24));
        s->link_capacity = (uint32_t)cap;
        BFX_ALLOC(s->link_cell, cap * sizeof(uint32_t));
        BFX_ALLOC(s->link_meta, cap * sizeof(uint32_t));
        BFX_ALLOC(s->link_q, cap * sizeof(float));
        if (c.geometry == BFX_GEOMETRY_MESH) {
            s->nverts = mesh->vertex_count;
            s->ntris = mesh->triangle_count;
            BFX_ALLOC(s->mesh_local, (size_t)s->nverts * 3 * sizeof(float));
            BFX_ALLOC(s->mesh_segment, (size_t)s->nverts);
            BFX_ALLOC(s->mesh_tris, (size_t)s->ntris * 3 * sizeof(uint32_t));
            BFX_ALLOC(s->mesh_tri_part, (size_t)s->ntris);
            BFX_ALLOC(s->mesh_pos, (size_t)s->nverts * sizeof(float4));
            BFX_ALLOC(s->mesh_vel, (size_t)s->nverts * sizeof(float4));
            BFX_ALLOC(s->keys, (size_t)s->box.cells * sizeof(unsigned long long));
            cudaMemcpyAsync(s->mesh_local, mesh->local_vertices, (size_t)s->nverts * 3 * sizeof(float),
                            cudaMemcpyHostToDevice, s->stream);
            cudaMemcpyAsync(s->mesh_segment, mesh->vertex_segment, s->nverts, cudaMemcpyHostToDevice, s->stream);
            cudaMemcpyAsync(s->mesh_tris, mesh->triangles, (size_t)s->ntris * 3 * sizeof(uint32_t),
                            cudaMemcpyHostToDevice, s->stream);
            cudaMemcpyAsync(s->mesh_tri_part, mesh->triangle_part, s->ntris, cudaMemcpyHostToDevice, s->stream);
            if (mesh->keyframe_count >= 2) {
                s->kf_count = (int)mesh->keyframe_count;
                const size_t np = (size_t)s->kf_count * s->nverts * 3;
                BFX_ALLOC(s->kf_times, (size_t)s->kf_count * sizeof(float));
                BFX_ALLOC(s->kf_points, np * sizeof(float));
                cudaMemcpyAsync(s->kf_times, mesh->keyframe_times, (size_t)s->kf_count * sizeof(float),
                                cudaMemcpyHostToDevice, s->stream);
                cudaMemcpyAsync(s->kf_points, mesh->keyframe_points, np * sizeof(float), cudaMemcpyHostToDevice,
                                s->stream);
            }
            if (mesh->joint_count > 0) {
                s->joint_count = (int)mesh->joint_count;
                BFX_ALLOC(s->joints, (size_t)s->joint_count * sizeof(bfx_joint));
                cudaMemcpyAsync(s->joints, mesh->joints, (size_t)s->joint_count * sizeof(bfx_joint),
                                cudaMemcpyHostToDevice, s->stream);
            }
        }
    }
#undef BFX_ALLOC
    cudaMemcpyAsync(s->dstate, &hs, sizeof(hs), cudaMemcpyHostToDevice, s->stream);

    // initial geometry (BirdFlowSimulation.encodeInitialization, BirdFlowSimulation.swift:1300-1357)
    if (s->geometry()) {
        if (c.geometry == BFX_GEOMETRY_MESH) {
            launch_fill_wall(s->wall, g.n, 16.0f, s->stream);
            s->launches += 1;
        }
        encode_geometry_build(s, 1, s->mask[1], s->mask[0]);
    }
    launch_init(c.storage, c.init, c.init_amplitude, g, fp, fluid_buffers(s, s->geometry() ? s->mask[0] : nullptr),
                s->stream);
    s->launches += 1;
    if (s->geometry() && !s->moving()) encode_links(s, s->mask[0], s->mask[0]);
    s->rep_s = 0;
    s->cur = 0;
    s->fields_valid = true;
    int sc = sync_check(s, "initialisation");
    if (sc != BFX_OK) {
        g_create_error = s->err;
        bfx_destroy(s);
        return sc;
    }
    if (s->geometry() && !s->moving()) {
        DeviceState st;
        cudaError_t ce = cudaMemcpy(&st, s->dstate, sizeof(st), cudaMemcpyDeviceToHost);
        if (ce != cudaSuccess) {
            const int rc = cuda_fail(nullptr, ce, "static link build");
            bfx_destroy(s);
            return rc;
        }
        if (st.link_overflow) {
            g_create_error = "the cut-link list exceeds its capacity; raise link_capacity";
            bfx_destroy(s);
            return BFX_ERR_CAPACITY;
        }
    }
    // the initial fields are published in slot 0 (BirdFlowSimulation.swift:626-640)
    DeviceState st0;
    if (read_state(s, &st0) != BFX_OK) {
        g_create_error = s->err;
        bfx_destroy(s);
        return BFX_ERR_KERNEL;
    }
    if (snapshot_slot_mask(s, 0) != BFX_OK) {
        g_create_error = s->err;
        bfx_destroy(s);
        return BFX_ERR_KERNEL;
    }
    s->slots->reset(field_frame_meta(s, st0, 0));
    *out = s;
    return BFX_OK;
}

int bfx_create_flapping_wing(const bfx_config* config, const bfx_flapping_wing* wing, bfx_sim** out) {
    if (!config || !wing || !out) return fail(nullptr, BFX_ERR_INVALID_ARGUMENT, "config, wing and out must not be null");
    *out = nullptr;
    if (config->geometry != BFX_GEOMETRY_FLAPPING_WING)
        return fail(nullptr, BFX_ERR_INVALID_CONFIG, "a flapping-wing simulation needs geometry BFX_GEOMETRY_FLAPPING_WING");
    const float* rc = wing->root_and_chord.v;
    const float* ge = wing->geometry.v;
    const float* k0 = wing->kinematics0.v;
    const float* k1 = wing->kinematics1.v;
    for (int k = 0; k < 4; ++k)
        if (!std::isfinite(rc[k]) || !std::isfinite(ge[k]) || !std::isfinite(k0[k]) || !std::isfinite(k1[k]))
            return fail(nullptr, BFX_ERR_INVALID_CONFIG, "flapping-wing parameters must be finite");
    if (!(rc[3] > 0.0f) || !(ge[0] > 0.0f) || !(ge[1] >= 0.0f) || !(ge[3] > 0.0f) || !(ge[2] > -1.0f))
        return fail(nullptr, BFX_ERR_INVALID_CONFIG,
                    "flapping wing: chord, radius and beta normalisation must be positive, thickness non-negative");
    if (!(k0[0] >= 1.0f) || !(k0[2] > 0.0f && k0[2] < 0.5f) || !(k0[3] > 0.0f && k0[3] < 0.5f))
        return fail(nullptr, BFX_ERR_INVALID_CONFIG,
                    "flapping wing: cycle steps >= 1 and the stroke / pitch transition durations in (0, 1/2)");
    // the wing record travels in the bird record's wing rows (see bfx_geometry.cu)
    bfx_bird packed;
    std::memset(&packed, 0, sizeof(packed));
    packed.wing_geometry0 = wing->root_and_chord;
    packed.wing_geometry1 = wing->geometry;
    packed.wing_kinematics0 = wing->kinematics0;
    packed.wing_kinematics1 = wing->kinematics1;
    packed.wing_kinematics1.v[3] = 0.0f;  // reference speed: not part of the geometry
    bfx_body_state body;
    std::memset(&body, 0, sizeof(body));
    for (int k = 0; k < 3; ++k) body.position[k] = rc[k];
    body.orientation[3] = 1.0;
    return bfx_create(config, &packed, &body, nullptr, out);
}

#define BFX_GUARD_READ(s)                                        \
    do {                                                         \
        if (!(s)) return BFX_ERR_INVALID_ARGUMENT;               \
        if ((s)->invalid) return BFX_ERR_INVALIDATED;            \
        cudaSetDevice((s)->device);                              \
    } while (0)
// every entry point that may change the device state drops the host copy
#define BFX_GUARD(s)                                             \
    do {                                                         \
        BFX_GUARD_READ(s);                                       \
        (s)->hstate_fresh = false;                               \
    } while (0)

static int read_state(bfx_sim* s, DeviceState* st) {
    if (s->hstate && s->hstate_fresh) {
        *st = *s->hstate;
        return BFX_OK;
    }
    cudaError_t e;
    if (s->hstate) {
        // one synchronisation: the copy queues behind the pending work
        e = cudaMemcpyAsync(s->hstate, s->dstate, sizeof(*st), cudaMemcpyDeviceToHost, s->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
        if (e == cudaSuccess) e = cudaGetLastError();
        if (e == cudaSuccess) {
            *st = *s->hstate;
            s->hstate_fresh = true;
        }
    } else {
        int rc = sync_check(s, "read-back");
        if (rc != BFX_OK) return rc;
        e = cudaMemcpy(st, s->dstate, sizeof(*st), cudaMemcpyDeviceToHost);
    }
    if (e != cudaSuccess) return cuda_fail(s, e, "state read-back");
    return BFX_OK;
}

int bfx_advance(bfx_sim* s, uint64_t steps, uint32_t batch_size, uint32_t flags, bfx_run_sample* samples,
                size_t sample_capacity, bfx_advance_result* result) {
    BFX_GUARD(s);
    if (batch_size == 0) return fail(s, BFX_ERR_INVALID_ADVANCE, "batch size must be positive");
    const bool record = (flags & BFX_ADVANCE_RECORD_SAMPLES) != 0;
    const CaptureMode mode = (flags & BFX_ADVANCE_CAPTURE_FIELDS)        ? CaptureMode::Required
                             : (flags & BFX_ADVANCE_CAPTURE_BEST_EFFORT) ? CaptureMode::BestEffort
                                                                         : CaptureMode::Disabled;
    if (record && (samples == nullptr || sample_capacity < steps))
        return fail(s, BFX_ERR_CAPACITY, "run-sample buffer smaller than the step count");
    // selectCaptureSlot (BirdFlowSimulation.swift:711): a slot for the last
    // step's fields, given back if the advance fails
    const int slot = steps > 0 ? s->slots->select(mode, s->slot_wait_ms) : kNoSlot;
    if (slot == kSlotWaitTimeout)
        return fail(s, BFX_ERR_TIMEOUT, "no field observation slot was released within the wait limit");
    const bool capture = slot >= 0;
    struct SlotGuard {
        FieldSlots<bfx_field_frame>* slots;
        int index;
        ~SlotGuard() {
            if (index >= 0) slots->abandon(index);
        }
    } slot_guard{s->slots.get(), slot};
    if (record && steps > s->dsamples_cap) {
        void* p = nullptr;
        cudaError_t e = cudaMalloc(&p, steps * sizeof(bfx_run_sample));
        if (e != cudaSuccess) return cuda_fail(s, e, "run-sample allocation");
        if (s->dsamples) {
            cudaFree(s->dsamples);
            s->allocations.erase(std::find(s->allocations.begin(), s->allocations.end(), (void*)s->dsamples));
        }
        s->dsamples = (bfx_run_sample*)p;
        s->dsamples_cap = steps;
        s->allocations.push_back(p);
    }
    uint64_t done = 0;
    while (done < steps) {
        uint64_t count = std::min<uint64_t>(batch_size, steps - done);
        uint64_t k = 0;
        // Pairs of plain steps replay a captured graph; steps that capture
        // fields, record samples or are individually timed are encoded directly.
        const bool last_batch = done + count == steps;
        if (s->graphs_enabled && !record && !s->timing && !s->topo_mode && can_pipeline(s) && count > 1) {
            // Pipelined: every step but the batch's last builds the next
            // step's geometry beside its own fluid kernel.  The batch's first
            // step builds its own; pairs replay a graph while a step of the
            // batch remains after them; the last one or two run directly.
            encode_step(s, 0, nullptr, 0, nullptr, nullptr, false, true);
            k = 1;
            for (; k + 2 < count; k += 2) {
                int rc = run_steps_graph(s, 2, true);
                if (rc != BFX_OK) return rc;
            }
            for (; k < count; ++k) {
                const bool last = k + 1 == count;
                if (capture && last && last_batch) s->capture_slot = slot;
                encode_step(s, capture && last && last_batch ? 1 : 0, nullptr, 0, nullptr, nullptr, true, !last);
                s->capture_slot = 0;
            }
        } else if (s->graphs_enabled && !record && !s->timing && !s->topo_mode) {
            uint64_t plain = capture && done + count == steps ? count - 1 : count;
            for (; k + 1 < plain; k += 2) {
                int rc = run_pair_graph(s);
                if (rc != BFX_OK) return rc;
            }
            if (k < plain) {
                int rc = run_steps_graph(s, 1);
                if (rc != BFX_OK) return rc;
                ++k;
            }
        }
        for (; k < count; ++k) {
            bool last = done + k + 1 == steps;
            if (capture && last) s->capture_slot = slot;
            encode_step(s, capture && last ? 1 : 0, record ? s->dsamples : nullptr, done + k);
            s->capture_slot = 0;
        }
        cudaError_t le = cudaGetLastError();
        if (le != cudaSuccess) return cuda_fail(s, le, "kernel launch");
        done += count;
        if (s->cfg.free_flight || s->moving() || done == steps) {
            DeviceState st;
            int rc = read_state(s, &st);
            if (rc != BFX_OK) return rc;
            s->step = st.step;
            if (st.link_overflow) return fail(s, BFX_ERR_KERNEL, "the cut-link list exceeded its capacity; raise link_capacity");
            if (st.stream_error) return fail(s, BFX_ERR_KERNEL, "a fused-kernel pipeline wait timed out");
            if (s->cfg.free_flight && st.safety_event[2] != 0) {
                if (result) {
                    result->steps_done = done;
                    result->safety_passed = 0;
                    std::memcpy(result->safety.metrics, st.safety_metrics, sizeof(st.safety_metrics));
                    std::memcpy(result->safety.event, st.safety_event, sizeof(st.safety_event));
                }
                return fail(s, BFX_ERR_SAFETY, "runtime safety violation (Mach, clearance or non-finite state)");
            }
        }
    }
    if (capture) {
        // the state read after the last batch completed the captured step
        DeviceState st;
        int rc = read_state(s, &st);
        if (rc != BFX_OK) return rc;
        rc = snapshot_slot_mask(s, slot);
        if (rc != BFX_OK) return rc;
        s->slots->publish(slot, field_frame_meta(s, st, slot));
        slot_guard.index = -1;
        s->fields_valid = true;
    }
    if (record && steps > 0) {
        cudaError_t e = cudaMemcpy(samples, s->dsamples, steps * sizeof(bfx_run_sample), cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) return cuda_fail(s, e, "run-sample read-back");
    }
    if (result) {
        DeviceState st;
        int rc = read_state(s, &st);
        if (rc != BFX_OK) return rc;
        result->steps_done = steps;
        result->field_frame_published = capture ? 1 : 0;
        result->dropped_field_frames = s->slots->dropped();
        result->safety_passed = st.safety_event[2] == 0 ? 1 : 0;
        std::memcpy(result->safety.metrics, st.safety_metrics, sizeof(st.safety_metrics));
        std::memcpy(result->safety.event, st.safety_event, sizeof(st.safety_event));
    }
    return BFX_OK;
}


static void loads_from_state(const bfx_sim* s, const DeviceState& st, bfx_loads* out) {
    std::memset(out, 0, sizeof(*out));
    for (int k = 0; k < 3; ++k) {
        out->force_lattice[k] = st.loads_lattice[k];
        out->force[k] = st.loads_lattice[k] * (double)s->fp.f2p;
        out->torque[k] = st.loads_torque[k];
    }
    out->limiter_activations = st.limiter_count;
    float r;
    std::memcpy(&r, &st.limiter_max_bits, 4);
    out->max_restriction = r;
    out->link_count = st.link_count;
    out->covered_count = st.covered_count;
    out->uncovered_count = st.uncovered_count;
    out->power = -st.power_lattice * (double)s->fp.f2p / (double)s->fp.v2l;
}

int bfx_last_loads(bfx_sim* s, bfx_loads* out) {
    BFX_GUARD_READ(s);
    if (!out) return BFX_ERR_INVALID_ARGUMENT;
    DeviceState st;
    int rc = read_state(s, &st);
    if (rc != BFX_OK) return rc;
    loads_from_state(s, st, out);
    return BFX_OK;
}

static void snapshot_from_state(const bfx_sim* s, const DeviceState& st, bfx_snapshot_data* out) {
    out->step = st.step;
    out->time = (double)(float)((double)st.step * (double)s->cfg.time_step);
    for (int k = 0; k < 3; ++k) out->body.position[k] = st.body[k];
    for (int k = 0; k < 4; ++k) out->body.orientation[k] = st.body[3 + k];
    for (int k = 0; k < 3; ++k) out->body.velocity[k] = st.body[7 + k];
    for (int k = 0; k < 3; ++k) out->body.omega_body[k] = st.body[10 + k];
    loads_from_state(s, st, &out->loads);
}

int bfx_snapshot(bfx_sim* s, bfx_snapshot_data* out) {
    BFX_GUARD_READ(s);
    if (!out) return BFX_ERR_INVALID_ARGUMENT;
    DeviceState st;
    int rc = read_state(s, &st);
    if (rc != BFX_OK) return rc;
    snapshot_from_state(s, st, out);
    return BFX_OK;
}

static_assert(sizeof(bfx_geometry_frame) == sizeof(Prepared), "BirdGeometryFrame is the prepared frame");

// GPUFieldFrameMetadata of a capture (publishFieldSlot, BirdFlowSimulation.swift:1832-1880)
static bfx_field_frame field_frame_meta(const bfx_sim* s, const DeviceState& st, int slot) {
    bfx_field_frame m;
    std::memset(&m, 0, sizeof(m));
    snapshot_from_state(s, st, &m.snapshot);
    m.grid[0] = s->cfg.nx;
    m.grid[1] = s->cfg.ny;
    m.grid[2] = s->cfg.nz;
    m.slot = (uint32_t)slot;
    for (int k = 0; k < 3; ++k) m.domain_origin[k] = s->cfg.origin[k];
    m.cell_size = s->cfg.cell_size;
    m.velocity_to_physical = s->cfg.cell_size / s->cfg.time_step;
    std::memcpy(&m.geometry, &st.prep, sizeof(m.geometry));
    timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    m.publication_uptime_seconds = (double)ts.tv_sec + 1.0e-9 * (double)ts.tv_nsec;
    m.density = s->slot_density[slot];
    m.velocity = (const float*)s->slot_velocity[slot];
    return m;
}

int bfx_copy_fields(bfx_sim* s, float* density, float* velocity_xyz, size_t cells) {
    BFX_GUARD(s);
    if (cells < (size_t)s->g.n) return fail(s, BFX_ERR_CAPACITY, "field buffers smaller than the lattice");
    int rc = sync_check(s, "fields");
    if (rc != BFX_OK) return rc;
    // currentPublishedFieldSlot (BirdFlowSimulation.swift:1906-1918)
    return copy_slot(s, s->slots->current(), density, velocity_xyz);
}

// The occupancy of the step a slot's fields belong to, copied beside them so
// that its derived diagnostics exclude the body of that step; returns once the
// copy (and everything queued before it) is done.
static int snapshot_slot_mask(bfx_sim* s, int slot) {
    if (s->slot_mask[slot]) {
        cudaMemcpyAsync(s->slot_mask[slot], s->mask[s->cur], (size_t)s->g.n, cudaMemcpyDeviceToDevice, s->stream);
        cudaError_t e = cudaStreamSynchronize(s->stream);
        if (e != cudaSuccess) return cuda_fail(s, e, "occupancy snapshot");
    }
    return BFX_OK;
}

static int copy_slot(bfx_sim* s, int slot, float* density, float* velocity_xyz) {
    if (density) {
        cudaError_t e =
            cudaMemcpy(density, s->slot_density[slot], (size_t)s->g.n * sizeof(float), cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) return cuda_fail(s, e, "field read-back");
    }
    if (velocity_xyz) {
        std::vector<float> v4((size_t)s->g.n * 4);
        cudaError_t e =
            cudaMemcpy(v4.data(), s->slot_velocity[slot], v4.size() * sizeof(float), cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) return cuda_fail(s, e, "field read-back");
        for (int64_t i = 0; i < s->g.n; ++i) {
            velocity_xyz[3 * i] = v4[4 * i];
            velocity_xyz[3 * i + 1] = v4[4 * i + 1];
            velocity_xyz[3 * i + 2] = v4[4 * i + 2];
        }
    }
    return BFX_OK;
}

int bfx_copy_gauge_pressure(bfx_sim* s, float pressure_scale_pascals, float* out, size_t cells) {
    BFX_GUARD(s);
    if (!out || cells < (size_t)s->g.n) return fail(s, BFX_ERR_CAPACITY, "pressure buffer smaller than the lattice");
    int rc = bfx_copy_fields(s, out, nullptr, cells);
    if (rc != BFX_OK) return rc;
    // LatticeScaling.gaugePressurePascals (SimulationConfiguration.swift:189-196)
    for (int64_t i = 0; i < s->g.n; ++i) out[i] = (1.0f / 3.0f) * (out[i] - 1.0f) * pressure_scale_pascals;
    return BFX_OK;
}

int bfx_runtime_safety(bfx_sim* s, bfx_safety_record* out) {
    BFX_GUARD(s);
    if (!out) return BFX_ERR_INVALID_ARGUMENT;
    DeviceState st;
    int rc = read_state(s, &st);
    if (rc != BFX_OK) return rc;
    std::memcpy(out->metrics, st.safety_metrics, sizeof(out->metrics));
    std::memcpy(out->event, st.safety_event, sizeof(out->event));
    return BFX_OK;
}

static int ensure_scratch(bfx_sim* s) {
    if (s->scratch_f32) return BFX_OK;
    cudaError_t e = cudaMalloc(&s->scratch_f32, (size_t)19 * s->g.n * sizeof(float));
    if (e != cudaSuccess) return cuda_fail(s, e, "read-out staging allocation");
    s->allocations.push_back(s->scratch_f32);
    return BFX_OK;
}

int bfx_copy_populations(bfx_sim* s, float* out, size_t count) {
    BFX_GUARD(s);
    if (!out || count < (size_t)19 * s->g.n) return fail(s, BFX_ERR_CAPACITY, "population buffer smaller than 19 * cells");
    int rc = ensure_scratch(s);
    if (rc != BFX_OK) return rc;
    launch_readout(s->cfg.storage, s->rep_s, s->g, fluid_buffers(s, nullptr), s->scratch_f32, s->stream);
    s->launches += 1;
    rc = sync_check(s, "population read-out");
    if (rc != BFX_OK) return rc;
    cudaError_t e = cudaMemcpy(out, s->scratch_f32, (size_t)19 * s->g.n * sizeof(float), cudaMemcpyDeviceToHost);
    return e == cudaSuccess ? BFX_OK : cuda_fail(s, e, "population copy");
}

int bfx_set_populations(bfx_sim* s, const float* in, size_t count) {
    BFX_GUARD(s);
    if (!in || count < (size_t)19 * s->g.n) return fail(s, BFX_ERR_CAPACITY, "population buffer smaller than 19 * cells");
    int rc = ensure_scratch(s);
    if (rc != BFX_OK) return rc;
    cudaMemcpyAsync(s->scratch_f32, in, (size_t)19 * s->g.n * sizeof(float), cudaMemcpyHostToDevice, s->stream);
    launch_writein(s->cfg.storage, s->rep_s, s->g, fluid_buffers(s, nullptr), s->scratch_f32, s->stream);
    s->launches += 1;
    return sync_check(s, "population write-in");
}

int bfx_copy_mask(bfx_sim* s, uint8_t* out, size_t cells) {
    BFX_GUARD(s);
    if (!out || cells < (size_t)s->g.n) return fail(s, BFX_ERR_CAPACITY, "mask buffer smaller than the lattice");
    int rc = sync_check(s, "mask");
    if (rc != BFX_OK) return rc;
    if (!s->geometry()) {
        std::memset(out, 0, (size_t)s->g.n);
        return BFX_OK;
    }
    cudaError_t e = cudaMemcpy(out, s->mask[s->cur], (size_t)s->g.n, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_fail(s, e, "mask read-back");
    for (int64_t i = 0; i < s->g.n; ++i) out[i] &= 0x3F;  // part id bits
    return BFX_OK;
}

int bfx_copy_wall(bfx_sim* s, float* out4, size_t cells) {
    BFX_GUARD(s);
    if (!out4 || cells < (size_t)s->g.n) return fail(s, BFX_ERR_CAPACITY, "wall buffer smaller than the lattice");
    int rc = sync_check(s, "wall");
    if (rc != BFX_OK) return rc;
    if (!s->geometry()) {
        std::memset(out4, 0, (size_t)s->g.n * 16);
        return BFX_OK;
    }
    cudaError_t e = cudaMemcpy(out4, s->wall, (size_t)s->g.n * sizeof(float4), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_fail(s, e, "wall read-back");
    return BFX_OK;
}

int bfx_copy_links(bfx_sim* s, uint32_t* cell, uint8_t* direction, float* fraction, size_t capacity, size_t* count) {
    BFX_GUARD(s);
    if (!count) return BFX_ERR_INVALID_ARGUMENT;
    DeviceState st;
    int rc = read_state(s, &st);
    if (rc != BFX_OK) return rc;
    size_t n = s->geometry() ? (size_t)std::min<int64_t>(st.link_count, s->link_capacity) : 0;
    *count = n;
    if (!cell && !direction && !fraction) return BFX_OK;
    if (capacity < n) return fail(s, BFX_ERR_CAPACITY, "link buffers smaller than the link count");
    if (n == 0) return BFX_OK;
    std::vector<uint32_t> meta(n);
    cudaError_t e = cudaSuccess;
    if (cell) e = cudaMemcpy(cell, s->link_cell, n * sizeof(uint32_t), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(meta.data(), s->link_meta, n * sizeof(uint32_t), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && fraction) e = cudaMemcpy(fraction, s->link_q, n * sizeof(float), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_fail(s, e, "link read-back");
    if (direction)
        for (size_t i = 0; i < n; ++i) direction[i] = (uint8_t)(meta[i] & 0xFF);
    return BFX_OK;
}

int bfx_fluid_mass_momentum(bfx_sim* s, double out[4]) {
    BFX_GUARD(s);
    if (!out) return BFX_ERR_INVALID_ARGUMENT;
    launch_mass_momentum(s->cfg.storage, s->rep_s, s->g, fluid_buffers(s, s->geometry() ? s->mask[s->cur] : nullptr),
                         s->mm_partials, s->mm_blocks, s->mm_result, s->stream);
    s->launches += 2;
    int rc = sync_check(s, "mass/momentum");
    if (rc != BFX_OK) return rc;
    cudaError_t e = cudaMemcpy(out, s->mm_result, 4 * sizeof(double), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_fail(s, e, "mass/momentum read-back");
    return BFX_OK;
}

// Restart state: header, device state, populations (storage format, with halo),
// planes, both masks and the wall field, followed by an FNV-1a checksum.
struct StateHeader {
    char magic[8];
    uint32_t version;
    uint32_t storage;
    uint32_t nx, ny, nz;
    int32_t rep_s, cur;
    uint32_t geometry;
    uint64_t payload;
};

static size_t state_size(const bfx_sim* s) {
    size_t n = sizeof(StateHeader) + sizeof(DeviceState) + (size_t)19 * s->g.padded * s->elem;
    if (s->geometry()) n += 2 * (size_t)s->g.n + (size_t)s->g.n * sizeof(float4);
    return n + sizeof(uint64_t);
}

int bfx_save_state(bfx_sim* s, void* buf, size_t capacity, size_t* size) {
    BFX_GUARD(s);
    size_t need = state_size(s);
    if (size) *size = need;
    if (!buf) return BFX_OK;
    if (capacity < need) return fail(s, BFX_ERR_CAPACITY, "state buffer too small");
    int rc = sync_check(s, "save state");
    if (rc != BFX_OK) return rc;
    char* p = (char*)buf;
    StateHeader h;
    std::memset(&h, 0, sizeof(h));
    std::memcpy(h.magic, "BFXSTATE", 8);
    h.version = 1;
    h.storage = (uint32_t)s->cfg.storage;
    h.nx = s->cfg.nx;
    h.ny = s->cfg.ny;
    h.nz = s->cfg.nz;
    h.rep_s = s->rep_s;
    h.cur = s->cur;
    h.geometry = (uint32_t)s->cfg.geometry;
    h.payload = need - sizeof(StateHeader) - sizeof(uint64_t);
    std::memcpy(p, &h, sizeof(h));
    p += sizeof(h);
    cudaMemcpy(p, s->dstate, sizeof(DeviceState), cudaMemcpyDeviceToHost);
    p += sizeof(DeviceState);
    cudaMemcpy(p, s->pops, (size_t)19 * s->g.padded * s->elem, cudaMemcpyDeviceToHost);
    p += (size_t)19 * s->g.padded * s->elem;
    if (s->geometry()) {
        cudaMemcpy(p, s->mask[0], (size_t)s->g.n, cudaMemcpyDeviceToHost);
        p += s->g.n;
        cudaMemcpy(p, s->mask[1], (size_t)s->g.n, cudaMemcpyDeviceToHost);
        p += s->g.n;
        cudaMemcpy(p, s->wall, (size_t)s->g.n * sizeof(float4), cudaMemcpyDeviceToHost);
        p += (size_t)s->g.n * sizeof(float4);
    }
    uint64_t sum = fnv1a(buf, need - sizeof(uint64_t));
    std::memcpy(p, &sum, sizeof(sum));
    return sync_check(s, "save state");
}

int bfx_restore_state(bfx_sim* s, const void* buf, size_t size) {
    BFX_GUARD(s);
    if (!buf) return BFX_ERR_INVALID_ARGUMENT;
    size_t need = state_size(s);
    if (size != need) return fail(s, BFX_ERR_INVALID_ARGUMENT, "state size does not match this simulation");
    StateHeader h;
    std::memcpy(&h, buf, sizeof(h));
    if (std::memcmp(h.magic, "BFXSTATE", 8) != 0 || h.version != 1 || h.storage != (uint32_t)s->cfg.storage ||
        h.nx != s->cfg.nx || h.ny != s->cfg.ny || h.nz != s->cfg.nz || h.geometry != (uint32_t)s->cfg.geometry)
        return fail(s, BFX_ERR_INVALID_ARGUMENT, "state header does not match this simulation");
    // the representation and the mask index select device buffers: only 0 and 1 exist
    if ((h.rep_s != 0 && h.rep_s != 1) || (h.cur != 0 && h.cur != 1))
        return fail(s, BFX_ERR_INVALID_ARGUMENT, "state header holds an invalid representation or mask index");
    uint64_t sum;
    std::memcpy(&sum, (const char*)buf + need - sizeof(uint64_t), sizeof(sum));
    if (sum != fnv1a(buf, need - sizeof(uint64_t))) return fail(s, BFX_ERR_INVALID_ARGUMENT, "state checksum mismatch");
    // nothing queued (a body upload) may land after the restored state
    const int synced = sync_check(s, "restore state");
    if (synced != BFX_OK) return synced;
    const char* p = (const char*)buf + sizeof(h);
    cudaError_t e = cudaMemcpy(s->dstate, p, sizeof(DeviceState), cudaMemcpyHostToDevice);
    // a restored state never carries the staged kernel's test hook
    if (e == cudaSuccess)
        e = cudaMemset((char*)s->dstate + offsetof(DeviceState, test_stall_tile1), 0, 2 * sizeof(uint32_t));
    p += sizeof(DeviceState);
    if (e == cudaSuccess) e = cudaMemcpy(s->pops, p, (size_t)19 * s->g.padded * s->elem, cudaMemcpyHostToDevice);
    p += (size_t)19 * s->g.padded * s->elem;
    if (s->geometry()) {
        if (e == cudaSuccess) e = cudaMemcpy(s->mask[0], p, (size_t)s->g.n, cudaMemcpyHostToDevice);
        p += s->g.n;
        if (e == cudaSuccess) e = cudaMemcpy(s->mask[1], p, (size_t)s->g.n, cudaMemcpyHostToDevice);
        p += s->g.n;
        if (e == cudaSuccess) e = cudaMemcpy(s->wall, p, (size_t)s->g.n * sizeof(float4), cudaMemcpyHostToDevice);
    }
    // a partial restore leaves no usable state
    if (e != cudaSuccess) return cuda_fail(s, e, "restore state upload");
    s->rep_s = h.rep_s;
    s->cur = h.cur;
    if (s->geometry() && !s->moving()) {
        // rebuild the static link list for the restored representation
        encode_links(s, s->mask[s->cur], s->mask[s->cur]);
    }
    // every slot is freed and slot 0 republished from the restored
    // populations (restoreCheckpointState, BirdFlowSimulation.swift:1990-2023)
    s->capture_slot = 0;
    launch_macroscopic(s->cfg.storage, s->rep_s, s->g, fluid_buffers(s, nullptr), s->stream);
    s->launches += 1;
    DeviceState st;
    int rc = read_state(s, &st);
    if (rc != BFX_OK) return rc;
    s->step = st.step;
    rc = snapshot_slot_mask(s, 0);
    if (rc != BFX_OK) return rc;
    s->slots->reset(field_frame_meta(s, st, 0));
    return BFX_OK;
}

int bfx_get_body(bfx_sim* s, bfx_body_state* out) {
    BFX_GUARD(s);
    if (!out) return BFX_ERR_INVALID_ARGUMENT;
    DeviceState st;
    int rc = read_state(s, &st);
    if (rc != BFX_OK) return rc;
    for (int k = 0; k < 3; ++k) out->position[k] = st.body[k];
    for (int k = 0; k < 4; ++k) out->orientation[k] = st.body[3 + k];
    for (int k = 0; k < 3; ++k) out->velocity[k] = st.body[7 + k];
    for (int k = 0; k < 3; ++k) out->omega_body[k] = st.body[10 + k];
    return BFX_OK;
}

int bfx_set_body(bfx_sim* s, const bfx_body_state* in) {
    BFX_GUARD(s);
    if (!in) return BFX_ERR_INVALID_ARGUMENT;
    double b[13];
    for (int k = 0; k < 3; ++k) b[k] = in->position[k];
    for (int k = 0; k < 4; ++k) b[3 + k] = in->orientation[k];
    for (int k = 0; k < 3; ++k) b[7 + k] = in->velocity[k];
    for (int k = 0; k < 3; ++k) b[10 + k] = in->omega_body[k];
    int rc = sync_check(s, "set body");
    if (rc != BFX_OK) return rc;
    cudaError_t e;
    if (s->hstate) {
        // stream-ordered upload from pinned staging (the stream is idle, so no
        // earlier copy still reads the staging)
        std::memcpy(s->hstate->body, b, sizeof(b));
        e = cudaMemcpyAsync((char*)s->dstate + offsetof(DeviceState, body), s->hstate->body, sizeof(b),
                            cudaMemcpyHostToDevice, s->stream);
    } else {
        e = cudaMemcpy((char*)s->dstate + offsetof(DeviceState, body), b, sizeof(b), cudaMemcpyHostToDevice);
    }
    if (e != cudaSuccess) return cuda_fail(s, e, "body upload");
    return BFX_OK;
}

int bfx_step_index(bfx_sim* s, uint64_t* step, double* time) {
    BFX_GUARD_READ(s);
    DeviceState st;
    int rc = read_state(s, &st);
    if (rc != BFX_OK) return rc;
    if (step) *step = st.step;
    if (time) *time = (double)(float)((double)st.step * (double)s->cfg.time_step);
    return BFX_OK;
}

int bfx_test_stall_staged_kernel(bfx_sim* s, int32_t tile, uint32_t wait_limit) {
    BFX_GUARD(s);
    if (!s->tma_ok) return fail(s, BFX_ERR_UNSUPPORTED, "the simulation does not run the staged 16-bit fluid kernel");
    if (tile < -1) return fail(s, BFX_ERR_INVALID_ARGUMENT, "tile must be -1 (none) or a tile index");
    const int rc = sync_check(s, "stall hook");
    if (rc != BFX_OK) return rc;
    const uint32_t v[2] = {(uint32_t)(tile + 1), wait_limit};
    static_assert(offsetof(DeviceState, test_wait_limit) == offsetof(DeviceState, test_stall_tile1) + 4,
                  "the hook fields are adjacent");
    const cudaError_t e = cudaMemcpy((char*)s->dstate + offsetof(DeviceState, test_stall_tile1), v, sizeof(v),
                                     cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return cuda_fail(s, e, "stall hook");
    return BFX_OK;
}

int bfx_test_replay_topology(bfx_sim* s, int mode, uint8_t* device_masks, uint64_t capacity_steps) {
    BFX_GUARD(s);
    if (mode < 0 || mode > 2) return fail(s, BFX_ERR_INVALID_ARGUMENT, "mode must be 0 (off), 1 (record) or 2 (replay)");
    if (mode != 0 && !s->moving()) return fail(s, BFX_ERR_UNSUPPORTED, "topology replay needs moving geometry");
    if (mode != 0 && (!device_masks || capacity_steps == 0))
        return fail(s, BFX_ERR_INVALID_ARGUMENT, "record and replay need a device buffer of capacity_steps masks");
    const int rc = sync_check(s, "topology replay");
    if (rc != BFX_OK) return rc;
    s->topo_mode = mode;
    s->topo_buf = mode ? device_masks : nullptr;
    s->topo_cap = mode ? capacity_steps : 0;
    s->topo_next = 0;
    return BFX_OK;
}

int bfx_set_kernel_timing(bfx_sim* s, int enabled) {
    BFX_GUARD(s);
    int rc = sync_check(s, "timing");
    if (rc != BFX_OK) return rc;
    s->timing = enabled != 0;
    s->timing_ms = 0.0;
    s->timing_launches = 0;
    s->ev_used = 0;
    return BFX_OK;
}

int bfx_kernel_timing(bfx_sim* s, double* total_ms, uint64_t* launches) {
    BFX_GUARD(s);
    int rc = sync_check(s, "timing");
    if (rc != BFX_OK) return rc;
    if (total_ms) *total_ms = s->timing_ms;
    if (launches) *launches = s->timing_launches;
    return BFX_OK;
}

int bfx_timer_begin(bfx_sim* s) {
    BFX_GUARD(s);
    if (!s->region[0]) {
        cudaEventCreate(&s->region[0]);
        cudaEventCreate(&s->region[1]);
    }
    cudaError_t e = cudaEventRecord(s->region[0], s->stream);
    return e == cudaSuccess ? BFX_OK : cuda_fail(s, e, "timer begin");
}

int bfx_timer_end(bfx_sim* s, double* elapsed_ms) {
    BFX_GUARD(s);
    if (!elapsed_ms || !s->region[0]) return BFX_ERR_INVALID_ARGUMENT;
    cudaEventRecord(s->region[1], s->stream);
    cudaError_t e = cudaEventSynchronize(s->region[1]);
    if (e != cudaSuccess) return cuda_fail(s, e, "timer end");
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, s->region[0], s->region[1]);
    *elapsed_ms = ms;
    timing_collect(s);
    return BFX_OK;
}

int bfx_launch_count(bfx_sim* s, uint64_t* launches) {
    if (!s || !launches) return BFX_ERR_INVALID_ARGUMENT;
    *launches = s->launches;
    return BFX_OK;
}

int bfx_device_bytes(bfx_sim* s, uint64_t* bytes) {
    if (!s || !bytes) return BFX_ERR_INVALID_ARGUMENT;
    *bytes = s->device_bytes;
    return BFX_OK;
}

// ---------------------------------------------------------------------------
// Coupled momentum ledger (BirdFlowSimulation.advanceWithCoupledMomentumLedger,
// BirdFlowSimulation.swift:806-1085): steps one at a time with the ledger's
// pre- and post-step passes (bfx_ledger.cu) and forms the balance in SI.
// ---------------------------------------------------------------------------
int bfx_advance_ledger(bfx_sim* s, uint64_t steps, bfx_ledger_sample* samples, size_t capacity,
                       uint64_t* steps_done) {
    BFX_GUARD(s);
    if (steps_done) *steps_done = 0;
    if (!s->cfg.free_flight || !s->has_bird)
        return fail(s, BFX_ERR_UNSUPPORTED, "the total-system ledger requires free flight with a bird");
    if (!(s->cfg.sponge_strength < 1.0f - 1.0e-6f))
        return fail(s, BFX_ERR_UNSUPPORTED, "sponge strength must be below 0.999999 to reconstruct the pre-sponge populations");
    if (steps == 0) return BFX_OK;
    if (!samples || capacity < steps) return fail(s, BFX_ERR_CAPACITY, "ledger sample buffer smaller than the step count");
    if (!s->ledger_in) {
        s->ledger_blocks = 4 * s->sm_count;
        cudaError_t e = dalloc(s, &s->ledger_in, (size_t)s->ledger_blocks * kLedgerInWidth * sizeof(double));
        if (e == cudaSuccess) e = dalloc(s, &s->ledger_out, (size_t)s->ledger_blocks * kLedgerOutWidth * sizeof(double));
        if (e != cudaSuccess) return cuda_fail(s, e, "ledger allocation");
    }
    std::vector<double> pin((size_t)s->ledger_blocks * kLedgerInWidth), pout((size_t)s->ledger_blocks * kLedgerOutWidth);
    const double dt = (double)s->cfg.time_step;
    const double f2p = (double)s->fp.f2p;
    const double mscale = f2p * dt;  // lattice momentum -> kg m / s
    const double mass = (double)s->bird.body_radii_mass.v[3];
    for (uint64_t k = 0; k < steps; ++k) {
        DeviceState before, after;
        int rc = read_state(s, &before);
        if (rc != BFX_OK) return rc;
        encode_step(s, 0, nullptr, 0, nullptr, s->ledger_in);
        uint8_t* mcur = s->geometry() ? s->mask[s->cur] : nullptr;
        launch_ledger_out(s->cfg.storage, s->rep_s, s->g, s->fp, fluid_buffers(s, mcur), mcur, s->ledger_out,
                          s->ledger_blocks, s->stream);
        s->launches += 1;
        cudaError_t e = cudaMemcpyAsync(pin.data(), s->ledger_in, pin.size() * sizeof(double), cudaMemcpyDeviceToHost,
                                        s->stream);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(pout.data(), s->ledger_out, pout.size() * sizeof(double), cudaMemcpyDeviceToHost,
                                s->stream);
        if (e != cudaSuccess) return cuda_fail(s, e, "ledger read-back");
        rc = read_state(s, &after);
        if (rc != BFX_OK) return rc;
        s->step = after.step;
        double in[kLedgerInWidth] = {}, out[kLedgerOutWidth] = {};
        for (int b = 0; b < s->ledger_blocks; ++b) {
            for (int j = 0; j < kLedgerInWidth; ++j) in[j] += pin[(size_t)b * kLedgerInWidth + j];
            for (int j = 0; j < kLedgerOutWidth; ++j) out[j] += pout[(size_t)b * kLedgerOutWidth + j];
        }
        bfx_ledger_sample& r = samples[k];
        std::memset(&r, 0, sizeof(r));
        r.step = after.step;
        r.time = (double)(float)((double)after.step * dt);
        for (int c = 0; c < 3; ++c) {
            r.fluid_momentum_before[c] = in[1 + c] * mscale;
            r.fluid_momentum_after[c] = out[1 + c] * mscale;
            r.fluid_momentum_change[c] = r.fluid_momentum_after[c] - r.fluid_momentum_before[c];
            r.body_momentum_before[c] = before.body[7 + c] * mass;
            r.body_momentum_after[c] = after.body[7 + c] * mass;
            r.wing_momentum_before[c] = (double)before.wing_prev[c] + (double)before.wing_prev[8 + c];
            r.wing_momentum_after[c] = (double)after.wing_prev[c] + (double)after.wing_prev[8 + c];
            r.aerodynamic_impulse[c] = after.loads_lattice[c] * f2p * dt;
            r.gravity_impulse[c] = (double)s->cfg.gravity[c] * (mass * dt);
            r.far_field_impulse[c] = in[5 + c] * mscale;
            r.sponge_impulse[c] = out[5 + c] * mscale;
            r.link_exchange_impulse[c] = in[9 + c] * mscale;
            r.fluid_boundary_impulse[c] = r.fluid_momentum_change[c] - r.far_field_impulse[c] - r.sponge_impulse[c];
            r.topology_impulse[c] = r.fluid_boundary_impulse[c] - r.link_exchange_impulse[c];
            r.boundary_residual[c] = r.aerodynamic_impulse[c] + r.fluid_boundary_impulse[c];
            r.total_momentum_change[c] = r.fluid_momentum_change[c] + (r.body_momentum_after[c] - r.body_momentum_before[c]) +
                                         (r.wing_momentum_after[c] - r.wing_momentum_before[c]);
            r.external_impulse[c] = r.far_field_impulse[c] + r.sponge_impulse[c] + r.gravity_impulse[c];
            r.system_residual[c] = r.total_momentum_change[c] - r.external_impulse[c];
        }
        r.far_field_links = (uint64_t)in[12];
        r.boundary_links = (uint64_t)in[14];
        r.topology_cells = (uint64_t)in[15];
        r.sponge_cells = (uint64_t)out[8];
        if (steps_done) *steps_done = k + 1;
        if (after.link_overflow) return fail(s, BFX_ERR_KERNEL, "the cut-link list exceeded its capacity; raise link_capacity");
        if (after.safety_event[2] != 0)
            return fail(s, BFX_ERR_SAFETY, "runtime safety violation (Mach, clearance or non-finite state)");
    }
    return BFX_OK;
}

// ---------------------------------------------------------------------------
// Discrete adjoint driver (kernels in bfx_adjoint.cu).
//
// Pass 1 runs the steps forward with the load objective enabled and keeps a
// snapshot (populations, current mask, device state) at the start of every
// checkpoint interval plus one of the final state.  The reverse pass walks the
// intervals backward: it restores the interval's snapshot, recomputes the
// interval once while recording a tape per step (moments, masks, keys, state,
// frame and link tangents, link values), then runs the adjoint steps of the
// interval in reverse.  Every step is recomputed exactly once; memory is
// (steps / interval) snapshots plus interval tapes.
// ---------------------------------------------------------------------------
}  // extern "C"

namespace {

struct AdjointAllocs {
    std::vector<void*> ptrs;
    uint64_t bytes = 0;
    ~AdjointAllocs() {
        for (void* p : ptrs) cudaFree(p);
    }
    template <class T>
    cudaError_t get(T** p, size_t n) {
        if (n == 0) n = 16;
        cudaError_t e = cudaMalloc((void**)p, n);
        if (e == cudaSuccess) {
            ptrs.push_back((void*)*p);
            bytes += n;
        }
        return e;
    }
};

int adjoint_scope(bfx_sim* s) {
    const bfx_config& c = s->cfg;
    if (c.geometry != BFX_GEOMETRY_MESH || c.static_geometry)
        return fail(s, BFX_ERR_UNSUPPORTED, "the adjoint needs moving mesh geometry");
    if (c.free_flight) return fail(s, BFX_ERR_UNSUPPORTED, "the adjoint needs prescribed motion (no free flight)");
    if (s->joint_count > 0) return fail(s, BFX_ERR_UNSUPPORTED, "the adjoint supports unjointed wing meshes");
    if (c.collision != BFX_COLLISION_TRT) return fail(s, BFX_ERR_UNSUPPORTED, "the adjoint supports the TRT collision");
    if (c.storage != BFX_STORAGE_F32 && c.storage != BFX_STORAGE_F64)
        return fail(s, BFX_ERR_UNSUPPORTED, "the adjoint supports F32 and F64 storage");
    if (c.fast_math) return fail(s, BFX_ERR_UNSUPPORTED, "the adjoint differentiates the non-contracted step");
    if (s->kf_count >= 2)
        return fail(s, BFX_ERR_UNSUPPORTED, "a keyframe replay does not depend on the kinematic parameters");
    for (int f = 0; f < 6; ++f)
        if (c.face_bc[f] == BFX_BC_OUTFLOW)
            return fail(s, BFX_ERR_UNSUPPORTED, "the adjoint does not support zero-gradient outflow faces");
    if (c.force_estimator != 6 || c.load_component != 0 || c.selected_part != 0 || !c.accumulate_loads ||
        c.moving_wall_local_density)
        return fail(s, BFX_ERR_UNSUPPORTED,
                    "the adjoint needs estimator 6, all parts, both load components and the far-field wall density");
    return BFX_OK;
}

}  // namespace

extern "C" {

int bfx_adjoint(bfx_sim* s, uint64_t steps, const bfx_adjoint_objective* objective, uint32_t checkpoint_interval,
                bfx_adjoint_result* result) {
    BFX_GUARD(s);
    if (!objective || steps == 0) return fail(s, BFX_ERR_INVALID_ARGUMENT, "objective and a positive step count are required");
    int rc = adjoint_scope(s);
    if (rc != BFX_OK) return rc;
    uint64_t first = objective->window_first, last = objective->window_last;
    if (first == 0 && last == 0) {
        first = 1;
        last = steps;
    }
    if (first < 1 || last < first || last > steps)
        return fail(s, BFX_ERR_INVALID_ARGUMENT, "objective window must satisfy 1 <= first <= last <= steps");
    uint64_t K = checkpoint_interval ? checkpoint_interval : (uint64_t)std::ceil(std::sqrt((double)steps));
    K = std::max<uint64_t>(1, std::min<uint64_t>(K, steps));
    const uint64_t nseg = (steps + K - 1) / K;
    rc = sync_check(s, "adjoint start");
    if (rc != BFX_OK) return rc;

    const size_t pop_bytes = (size_t)19 * (size_t)s->g.padded * s->elem;
    const size_t n = (size_t)s->g.n;
    AdjointAllocs mem;
#define BFX_ADJ_ALLOC(ptr, bytes)                                                   \
    do {                                                                            \
        cudaError_t ee = mem.get(&(ptr), (bytes));                                  \
        if (ee != cudaSuccess) return fail(s, BFX_ERR_ALLOCATION, "adjoint work memory allocation failed"); \
    } while (0)
    // snapshots: nseg interval starts + the final state
    char* snap_pops = nullptr;
    uint8_t* snap_mask = nullptr;
    DeviceState* snap_state = nullptr;
    BFX_ADJ_ALLOC(snap_pops, (nseg + 1) * pop_bytes);
    // both mask buffers: the geometry rewrites only its active bounds, and the
    // cells outside them keep the zeros the other buffer holds
    BFX_ADJ_ALLOC(snap_mask, (nseg + 1) * 2 * n);
    BFX_ADJ_ALLOC(snap_state, (nseg + 1) * sizeof(DeviceState));
    std::vector<int> snap_rep(nseg + 1), snap_cur(nseg + 1);
    auto snapshot = [&](uint64_t i) {
        cudaMemcpyAsync(snap_pops + i * pop_bytes, s->pops, pop_bytes, cudaMemcpyDeviceToDevice, s->stream);
        cudaMemcpyAsync(snap_mask + i * 2 * n, s->mask[s->cur], n, cudaMemcpyDeviceToDevice, s->stream);
        cudaMemcpyAsync(snap_mask + i * 2 * n + n, s->mask[s->cur ^ 1], n, cudaMemcpyDeviceToDevice, s->stream);
        cudaMemcpyAsync(snap_state + i, s->dstate, sizeof(DeviceState), cudaMemcpyDeviceToDevice, s->stream);
        snap_rep[i] = s->rep_s;
        snap_cur[i] = s->cur;
    };
    auto restore = [&](uint64_t i) {
        s->hstate_fresh = false;
        cudaMemcpyAsync(s->pops, snap_pops + i * pop_bytes, pop_bytes, cudaMemcpyDeviceToDevice, s->stream);
        cudaMemcpyAsync(s->mask[snap_cur[i]], snap_mask + i * 2 * n, n, cudaMemcpyDeviceToDevice, s->stream);
        cudaMemcpyAsync(s->mask[snap_cur[i] ^ 1], snap_mask + i * 2 * n + n, n, cudaMemcpyDeviceToDevice, s->stream);
        cudaMemcpyAsync(s->dstate, snap_state + i, sizeof(DeviceState), cudaMemcpyDeviceToDevice, s->stream);
        s->rep_s = snap_rep[i];
        s->cur = snap_cur[i];
    };

    // objective on, accumulators cleared
    Objective ob;
    std::memset(&ob, 0, sizeof(ob));
    ob.enabled = 1;
    ob.start = s->step;
    ob.first = first;
    ob.last = last;
    for (int k = 0; k < 3; ++k) ob.force_weight[k] = objective->force_weight[k];
    ob.power_weight = objective->power_weight;
    cudaMemcpyAsync(s->dobjective, &ob, sizeof(ob), cudaMemcpyHostToDevice, s->stream);

    // From a fresh simulation the initial populations depend on theta (the
    // wall equilibria of the cells solid at t = 0): keep the t = 0 geometry.
    const bool from_start = s->step == 0;
    unsigned long long* init_keys = nullptr;
    DeviceState* init_state = nullptr;
    FrameTangent* init_frames = nullptr;
    if (from_start) {
        BFX_ADJ_ALLOC(init_keys, (size_t)s->box.cells * sizeof(unsigned long long));
        BFX_ADJ_ALLOC(init_state, sizeof(DeviceState));
        BFX_ADJ_ALLOC(init_frames, sizeof(FrameTangent));
        cudaMemcpyAsync(init_keys, s->keys, (size_t)s->box.cells * sizeof(unsigned long long),
                        cudaMemcpyDeviceToDevice, s->stream);
        cudaMemcpyAsync(init_state, s->dstate, sizeof(DeviceState), cudaMemcpyDeviceToDevice, s->stream);
        launch_frame_tangent(geom_buffers(s, s->mask[s->cur], s->mask[s->cur]), s->cfg.time_step, 1, init_frames,
                             s->stream);
    }

    // ev: forward start and end, reverse end, reverse start (after the
    // reverse pass's work memory is allocated: those host-side allocations
    // leave the device idle for a varying time that is not the pass's work)
    cudaEvent_t ev[4];
    for (auto& e : ev) cudaEventCreate(&e);
    cudaEventRecord(ev[0], s->stream);
    // pass 1: forward with snapshots
    for (uint64_t seg = 0; seg < nseg; ++seg) {
        snapshot(seg);
        const uint64_t len = std::min<uint64_t>(K, steps - seg * K);
        uint64_t k = 0;
        if (s->graphs_enabled && !s->timing)
            for (; k + 1 < len; k += 2) {
                rc = run_pair_graph(s);
                if (rc != BFX_OK) return rc;
            }
        for (; k < len; ++k) encode_step(s, 0, nullptr, 0);
    }
    snapshot(nseg);
    cudaEventRecord(ev[1], s->stream);
    rc = sync_check(s, "adjoint forward pass");
    if (rc != BFX_OK) return rc;
    DeviceState st_end;
    cudaError_t ce = cudaMemcpy(&st_end, s->dstate, sizeof(st_end), cudaMemcpyDeviceToHost);
    if (ce == cudaSuccess) ce = cudaMemcpy(&ob, s->dobjective, sizeof(ob), cudaMemcpyDeviceToHost);
    if (ce != cudaSuccess) return cuda_fail(s, ce, "adjoint forward read-back");
    if (st_end.link_overflow) return fail(s, BFX_ERR_KERNEL, "the cut-link list exceeded its capacity; raise link_capacity");
    const uint64_t link_slots = (uint64_t)std::max<int64_t>(1, std::min<int64_t>(ob.max_links, s->link_capacity));

    // tape of one interval and the adjoint work arrays
    const size_t R = s->elem;
    const size_t link_rec = R == 8 ? sizeof(LinkTape<double>) : sizeof(LinkTape<float>);
    char* t_moments = nullptr;
    uint8_t *t_mnext = nullptr, *t_mprev = nullptr;
    unsigned long long* t_keys = nullptr;
    DeviceState* t_state = nullptr;
    FrameTangent* t_frames = nullptr;
    char* t_links = nullptr;
    float* link_tangent = nullptr;
    void* lam = nullptr;
    void* nu = nullptr;
    double *p_rare = nullptr, *p_links = nullptr;
    BFX_ADJ_ALLOC(t_moments, K * n * 4 * R);
    BFX_ADJ_ALLOC(t_mnext, K * n);
    BFX_ADJ_ALLOC(t_mprev, K * n);
    BFX_ADJ_ALLOC(t_keys, K * (size_t)s->box.cells * sizeof(unsigned long long));
    BFX_ADJ_ALLOC(t_state, K * sizeof(DeviceState));
    BFX_ADJ_ALLOC(t_frames, K * sizeof(FrameTangent));
    BFX_ADJ_ALLOC(t_links, K * link_slots * link_rec);
    BFX_ADJ_ALLOC(link_tangent, (size_t)s->link_capacity * kLinkTangentWords * sizeof(float));
    BFX_ADJ_ALLOC(lam, pop_bytes);
    BFX_ADJ_ALLOC(nu, (size_t)s->link_capacity * R);
    BFX_ADJ_ALLOC(p_rare, (size_t)s->box_blocks * 4 * sizeof(double));
    BFX_ADJ_ALLOC(p_links, (size_t)s->apply_blocks * 4 * sizeof(double));
#undef BFX_ADJ_ALLOC
    cudaEventRecord(ev[3], s->stream);
    cudaMemsetAsync(lam, 0, pop_bytes, s->stream);
    const int32_t off = 0;
    cudaMemcpyAsync(&s->dobjective->enabled, &off, sizeof(off), cudaMemcpyHostToDevice, s->stream);
    auto slot = [&](uint64_t j) {
        TapeSlot t;
        t.moments = t_moments + j * n * 4 * R;
        t.mask_next = t_mnext + j * n;
        t.mask_prev = t_mprev + j * n;
        t.keys = t_keys + j * (size_t)s->box.cells;
        t.state = t_state + j;
        t.frames = t_frames + j;
        t.links = t_links + j * link_slots * link_rec;
        t.link_tangent = link_tangent;
        return t;
    };
    AdjointWork w;
    w.lam = lam;
    w.nu = nu;
    w.partials_rare = p_rare;
    w.partials_links = p_links;
    w.objective = s->dobjective;
    const uint32_t saved_capacity = s->link_capacity;
    std::vector<int> reps(K);
    const double inv_window = 1.0 / (double)(last - first + 1);
    for (uint64_t seg = nseg; seg-- > 0;) {
        restore(seg);
        const uint64_t len = std::min<uint64_t>(K, steps - seg * K);
        // the tape holds link_slots links per step: cap the link list there (the
        // recomputation reproduces the forward pass, whose largest count it is)
        s->link_capacity = (uint32_t)link_slots;
        for (uint64_t j = 0; j < len; ++j) {
            reps[j] = s->rep_s;
            TapeSlot t = slot(j);
            encode_step(s, 0, nullptr, 0, &t);
        }
        s->link_capacity = saved_capacity;
        for (uint64_t j = len; j-- > 0;) {
            const uint64_t rel = seg * K + j + 1;
            const double weight = rel >= first && rel <= last ? inv_window : 0.0;
            TapeSlot t = slot(j);
            StepTape tape;
            tape.moments = t.moments;
            tape.mask_next = t.mask_next;
            tape.mask_prev = t.mask_prev;
            tape.keys = t.keys;
            tape.state = t.state;
            tape.frames = t.frames;
            tape.links = t.links;
            GeomBuffers gb = geom_buffers(s, s->mask[0], s->mask[1]);
            gb.link_capacity = (uint32_t)link_slots;  // the tape slot's size
            launch_adjoint_step(s->cfg.storage, reps[j], s->g, s->fp, s->box, gb, tape, w, weight, s->stream);
            s->launches += 9;
        }
        cudaError_t le = cudaGetLastError();
        if (le != cudaSuccess) return cuda_fail(s, le, "adjoint launch");
    }
    if (from_start) {
        StepTape init;
        init.moments = nullptr;
        init.mask_next = snap_mask;   // the t = 0 occupancy
        init.mask_prev = snap_mask;
        init.keys = init_keys;
        init.state = init_state;
        init.frames = init_frames;
        init.links = nullptr;
        GeomBuffers gb = geom_buffers(s, s->mask[0], s->mask[1]);
        launch_adjoint_init(s->cfg.storage, snap_rep[0], s->g, s->fp, s->box, gb, init, w, s->stream);
    }
    cudaEventRecord(ev[2], s->stream);
    restore(nseg);
    rc = sync_check(s, "adjoint reverse pass");
    if (rc != BFX_OK) return rc;
    ce = cudaMemcpy(&ob, s->dobjective, sizeof(ob), cudaMemcpyDeviceToHost);
    if (ce != cudaSuccess) return cuda_fail(s, ce, "adjoint gradient read-back");
    s->step = st_end.step;
    float f_ms = 0.0f, r_ms = 0.0f;
    cudaEventElapsedTime(&f_ms, ev[0], ev[1]);
    cudaEventElapsedTime(&r_ms, ev[3], ev[2]);
    for (auto& e : ev) cudaEventDestroy(e);
    if (result) {
        std::memset(result, 0, sizeof(*result));
        result->objective = ob.value;
        for (int k = 0; k < 4; ++k) result->gradient[k] = ob.grad[k];
        result->steps = steps;
        result->checkpoint_interval = (uint32_t)K;
        result->snapshots = (uint32_t)(nseg + 1);
        result->forward_ms = f_ms;
        result->reverse_ms = r_ms;
        result->max_links = (uint64_t)ob.max_links;
        result->work_bytes = mem.bytes;
    }
    return BFX_OK;
}

// ---------------------------------------------------------------------------
// Field observation slots (BirdFlowSimulation.swift:1148-1210, 1806-1918)

int bfx_set_observation_buffers(bfx_sim* s, uint32_t count, uint32_t wait_limit_ms) {
    BFX_GUARD(s);
    if (count < 1 || count > (uint32_t)bfx_sim::kMaxSlots)
        return fail(s, BFX_ERR_INVALID_ARGUMENT, "observationBufferCount must be in 1...4");
    if (!s->slots->idle()) return fail(s, BFX_ERR_INVALID_ARGUMENT, "a field frame is leased or being written");
    int rc = sync_check(s, "observation buffers");
    if (rc != BFX_OK) return rc;
    for (uint32_t i = 1; i < count; ++i) {
        if (s->slot_density[i]) continue;
        cudaError_t e = dalloc(s, &s->slot_density[i], (size_t)s->g.n * sizeof(float));
        if (e == cudaSuccess) e = dalloc(s, &s->slot_velocity[i], (size_t)s->g.n * sizeof(float4));
        if (e == cudaSuccess && s->geometry()) e = dalloc(s, &s->slot_mask[i], (size_t)s->g.n);
        if (e != cudaSuccess) return cuda_fail(s, e, "observation slot allocation");
    }
    // The newest published frame carries over into slot 0 of the new set;
    // without one, slot 0 is extracted from the current populations.
    bfx_field_frame meta;
    int newest = 0;
    if (s->slots->acquire(false, 0, &meta, &newest) != 0) {
        if (newest != 0) {
            cudaMemcpyAsync(s->slot_density[0], s->slot_density[newest], (size_t)s->g.n * sizeof(float),
                            cudaMemcpyDeviceToDevice, s->stream);
            cudaMemcpyAsync(s->slot_velocity[0], s->slot_velocity[newest], (size_t)s->g.n * sizeof(float4),
                            cudaMemcpyDeviceToDevice, s->stream);
            if (s->slot_mask[0])
                cudaMemcpyAsync(s->slot_mask[0], s->slot_mask[newest], (size_t)s->g.n, cudaMemcpyDeviceToDevice,
                                s->stream);
        }
        meta.slot = 0;
        meta.density = s->slot_density[0];
        meta.velocity = (const float*)s->slot_velocity[0];
        rc = sync_check(s, "observation buffers");
        if (rc != BFX_OK) return rc;
    } else {
        s->capture_slot = 0;
        launch_macroscopic(s->cfg.storage, s->rep_s, s->g, fluid_buffers(s, nullptr), s->stream);
        s->launches += 1;
        DeviceState st;
        rc = read_state(s, &st);
        if (rc != BFX_OK) return rc;
        rc = snapshot_slot_mask(s, 0);
        if (rc != BFX_OK) return rc;
        meta = field_frame_meta(s, st, 0);
    }
    auto slots = std::make_shared<FieldSlots<bfx_field_frame>>((int)count);
    slots->reset(meta);
    slots->add_counters(s->slots->dropped(), s->slots->waits());
    s->slots = slots;
    s->slot_wait_ms = wait_limit_ms;
    return BFX_OK;
}

int bfx_acquire_field_frame(bfx_sim* s, int has_after_step, uint64_t after_step, bfx_field_frame* out) {
    if (!s || !out) return BFX_ERR_INVALID_ARGUMENT;
    std::memset(out, 0, sizeof(*out));
    bfx_field_frame meta;
    int slot = 0;
    const uint64_t lease = s->slots->acquire(has_after_step != 0, after_step, &meta, &slot);
    if (lease == 0) return BFX_OK;
    *out = meta;
    out->lease = lease;
    return BFX_OK;
}

int bfx_field_frame_copy(bfx_sim* s, uint64_t lease, float* density, float* velocity_xyz, size_t cells) {
    BFX_GUARD_READ(s);
    if (cells < (size_t)s->g.n) return fail(s, BFX_ERR_CAPACITY, "field buffers smaller than the lattice");
    const int slot = s->slots->leased_slot(lease);
    if (slot < 0) return fail(s, BFX_ERR_INVALID_ARGUMENT, "the field frame lease is not live");
    return copy_slot(s, slot, density, velocity_xyz);
}

int bfx_release_field_frame(bfx_sim* s, uint64_t lease) {
    if (!s) return BFX_ERR_INVALID_ARGUMENT;
    s->slots->release(lease);
    return BFX_OK;
}

namespace {
struct PendingRelease {
    std::shared_ptr<FieldSlots<bfx_field_frame>> slots;
    uint64_t lease;
};
void CUDART_CB release_when_done(void* p) {
    auto* r = static_cast<PendingRelease*>(p);
    r->slots->release(r->lease);
    delete r;
}
}  // namespace

int bfx_release_field_frame_after(bfx_sim* s, uint64_t lease, void* cuda_stream) {
    if (!s) return BFX_ERR_INVALID_ARGUMENT;
    if (s->slots->leased_slot(lease) < 0) return BFX_OK;  // released already
    cudaSetDevice(s->device);
    auto* r = new PendingRelease{s->slots, lease};
    cudaStream_t st = cuda_stream ? (cudaStream_t)cuda_stream : s->stream;
    cudaError_t e = cudaLaunchHostFunc(st, release_when_done, r);
    if (e != cudaSuccess) {
        delete r;
        (void)cudaGetLastError();
        return fail(s, BFX_ERR_INVALID_ARGUMENT, std::string("release after completion: ") + cudaGetErrorString(e));
    }
    return BFX_OK;
}

int bfx_capture_current_fields(bfx_sim* s, uint32_t mode, uint32_t* published) {
    BFX_GUARD(s);
    if (published) *published = 0;
    if (mode > BFX_FIELD_CAPTURE_DISABLED) return fail(s, BFX_ERR_INVALID_ARGUMENT, "unknown field capture mode");
    int rc = sync_check(s, "field capture");
    if (rc != BFX_OK) return rc;
    const int slot = s->slots->select((CaptureMode)mode, s->slot_wait_ms);
    if (slot == kSlotWaitTimeout)
        return fail(s, BFX_ERR_TIMEOUT, "no field observation slot was released within the wait limit");
    if (slot < 0) return BFX_OK;
    s->capture_slot = slot;
    launch_macroscopic(s->cfg.storage, s->rep_s, s->g, fluid_buffers(s, nullptr), s->stream);
    s->capture_slot = 0;
    s->launches += 1;
    DeviceState st;
    rc = read_state(s, &st);
    if (rc != BFX_OK) {
        s->slots->abandon(slot);
        return rc;
    }
    rc = snapshot_slot_mask(s, slot);
    if (rc != BFX_OK) {
        s->slots->abandon(slot);
        return rc;
    }
    s->slots->publish(slot, field_frame_meta(s, st, slot));
    s->fields_valid = true;
    if (published) *published = 1;
    return BFX_OK;
}

int bfx_flow_diagnostics(bfx_sim* s, uint64_t lease, float* vorticity4, float* q_criterion, uint8_t* valid,
                         size_t cells, int device_outputs) {
    BFX_GUARD_READ(s);
    if (!vorticity4 || !q_criterion || !valid) return BFX_ERR_INVALID_ARGUMENT;
    if (cells < (size_t)s->g.n) return fail(s, BFX_ERR_CAPACITY, "diagnostic buffers smaller than the lattice");
    const int slot = s->slots->leased_slot(lease);
    if (slot < 0) return fail(s, BFX_ERR_INVALID_ARGUMENT, "the field frame lease is not live");
    const size_t n = (size_t)s->g.n;
    float4* dv = (float4*)vorticity4;
    float* dq = q_criterion;
    uint8_t* dm = valid;
    if (!device_outputs) {
        if (!s->diag_scratch) {
            cudaError_t e = dalloc(s, &s->diag_scratch, n * (sizeof(float4) + sizeof(float) + 1));
            if (e != cudaSuccess) return cuda_fail(s, e, "diagnostics staging allocation");
        }
        dv = (float4*)s->diag_scratch;
        dq = (float*)(dv + n);
        dm = (uint8_t*)(dq + n);
    }
    // GPUFieldFrameMetadata.velocityToPhysical over the cell size
    const float v2p = s->cfg.cell_size / s->cfg.time_step;
    const float scale = 0.5f * v2p / s->cfg.cell_size;
    launch_flow_diagnostics(s->slot_velocity[slot], s->slot_mask[slot], (int)s->cfg.nx, (int)s->cfg.ny,
                            (int)s->cfg.nz, scale, dv, dq, dm, s->stream);
    s->launches += 1;
    if (!device_outputs) {
        cudaMemcpyAsync(vorticity4, dv, n * sizeof(float4), cudaMemcpyDeviceToHost, s->stream);
        cudaMemcpyAsync(q_criterion, dq, n * sizeof(float), cudaMemcpyDeviceToHost, s->stream);
        cudaMemcpyAsync(valid, dm, n, cudaMemcpyDeviceToHost, s->stream);
    }
    return sync_check(s, "flow diagnostics");
}

int bfx_observation_counters(bfx_sim* s, uint64_t* dropped_frames, uint64_t* capture_waits) {
    if (!s) return BFX_ERR_INVALID_ARGUMENT;
    if (dropped_frames) *dropped_frames = s->slots->dropped();
    if (capture_waits) *capture_waits = s->slots->waits();
    return BFX_OK;
}

int bfx_last_error(bfx_sim* s, char* buf, size_t capacity) {
    const std::string& m = s ? s->err : g_create_error;
    if (!buf || capacity == 0) return BFX_ERR_INVALID_ARGUMENT;
    size_t n = std::min(capacity - 1, m.size());
    std::memcpy(buf, m.data(), n);
    buf[n] = 0;
    return BFX_OK;
}

}  // extern "C"
