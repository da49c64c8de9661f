// Free-body ("scene") worlds: piles of spheres, capsules, boxes and
// cylinders on a ground plane.
// Device record, launch parameters and per-environment capacities of the
// free-body control-step kernel (scene_step.cu).
#pragma once

#include <cstdint>

#include <cuda_runtime.h>

#include "numi_b200.h"

namespace numi {

constexpr int kSceneMaxBodies = 64;
constexpr int kSceneMaxPairs = kSceneMaxBodies * (kSceneMaxBodies - 1) / 2 + kSceneMaxBodies;
constexpr int kSceneManifolds = MR_B200_SCENE_MANIFOLDS;  // persistent manifolds per environment
constexpr int kSceneContacts = 256;    // solver contacts per environment
constexpr int kSceneCandidates = 512;  // broadphase candidate pairs per environment
constexpr int kSceneMaxMaterials = 4;
constexpr int kSceneMaxHullVertices = 1024;  // hull vertices of all convex bodies of a world
// Words of one manifold slot of a scene (MRManifoldC layout) plus its pair key.
constexpr int kSceneSlotWords = MR_B200_SCENE_SLOT_WORDS;

struct alignas(16) SceneModel {
    std::int32_t nb;  // free bodies; the ground plane is collider nb
    std::int32_t np;  // compiled pairs
    float h;
    float slop;
    float gravity[4];
    float max_depenetration;
    float speculative_scale;
    float speed_envelope;
    float reserved0;
    float thresholds[4];  // breaking separation, drift, merge, normal cosine
    float4 plane_position;
    float4 plane_rotation;
    float4 plane_offsets;  // contact offset, rest offset
    float4 ground_position;  // pose of the plane's (static) body: manifold
    float4 ground_rotation;  // anchors on the plane live in this frame
    std::int32_t plane_material;
    std::int32_t support_mapped;  // some pair is MR_COLLISION_PAIR_CONVEX (GJK / EPA)
    std::uint32_t world_tag;  // identifies this record to launches that check SceneParams::world_tag (0: untagged)
    std::int32_t reserved1;
    // Bodies (one collider each, at the body's centre of mass).
    std::int32_t shape_type[kSceneMaxBodies];
    std::int32_t material[kSceneMaxBodies];
    float4 dims[kSceneMaxBodies];         // sphere radius; box half extents
    float4 mass[kSceneMaxBodies];         // mass, inverse mass, linear damping, angular damping
    float4 inv_inertia[kSceneMaxBodies];  // body-frame principal inverse inertia, max linear speed
    float4 offsets[kSceneMaxBodies];      // contact offset, rest offset, sweep radius, max angular speed
    float4 material_friction[kSceneMaxMaterials];
    float4 material_response[kSceneMaxMaterials];
    // Compiled pairs, ascending by key a * (kSceneMaxBodies + 1) + b (b = nb: plane).
    std::uint8_t pair_a[kSceneMaxPairs];
    std::uint8_t pair_b[kSceneMaxPairs];
    std::uint8_t pair_class[kSceneMaxPairs];
    // Convex bodies: their hull vertices, already scaled by the body's
    // dimensions (vertex x dimensions, rounded once to FP32 as the reference
    // rounds it per query), at [hull_first[b], hull_first[b] + hull_count[b]).
    std::int32_t hull_first[kSceneMaxBodies];
    std::int32_t hull_count[kSceneMaxBodies];
    float4 hull_vertices[kSceneMaxHullVertices];
};

// Environments ("slots") hold resident state; a launch processes work
// items, item i advancing slot env_index[i] (or slot i when env_index is
// null).  Per-item arrays: reset masks, observations, status codes, active
// contacts.  Per-slot arrays: everything else.
struct SceneParams {
    const SceneModel* model;
    float* q;                  // [slot][nb][7]: position, orientation xyzw
    float* v;                  // [slot][nb][6]: linear, angular velocity (world)
    float* manifolds;          // [slot][kSceneManifolds][kSceneSlotWords]
    std::uint32_t* manifold_count;  // [slot]
    const float* reset_q;      // [slot]
    const float* reset_v;
    const float* friction_scale;    // [slot]
    const std::int32_t* env_index;  // [item] -> slot, or null
    const std::uint32_t* reset_masks;  // [item] of this control step, or null
    float* observations;       // [item][nq + nv] of this control step, or null
    std::uint32_t* status_codes;     // [item]
    std::uint32_t* active_contacts;  // [item]
    std::uint32_t* stats;
    float* workspace;          // [slot][scene_workspace_words()]: substep tables, contacts, narrowphase scratch
    std::int32_t env_count;    // items in this launch
    std::int32_t substeps;
    std::int32_t velocity_iterations;
    std::int32_t final_velocity_iterations;
    float* q_comp;             // [slot][nb][7]: compensation of the position sums (entries 0-2), or null (FP32 sums)
    std::int32_t support_mapped;  // the model has support-mapped (cylinder) pairs: SceneModel::support_mapped
    // Non-zero: the launch was enqueued for the record with this tag.  A
    // launch that finds another record behind `model` (a shared record
    // replaced after the launch was recorded, e.g. in a replayed graph)
    // leaves every buffer of the item untouched and reports
    // MR_STEP_UNSUPPORTED in its status code and kStatWorldMismatch.
    std::uint32_t world_tag;
    // [slot][kSceneMaxBodies] island index of each body on the final
    // substep, islands numbered by ascending root (smallest) body as
    // buildConstraintIslands numbers them; 0xff: in no island.  Or null.
    std::uint8_t* island_labels;
    double* audit;             // [slot][kAuditWords] FP64 energy / momentum audit (audit.cuh), or null
};

size_t scene_step_smem_bytes(bool compensated = false);
size_t scene_workspace_words();
cudaError_t configure_scene_step_kernel();
cudaError_t launch_scene_step(const SceneParams& p, cudaStream_t stream);
// FP64 energy / momentum audit (audit.cuh) of the bodies the scene launch
// with the same parameters committed; p.audit must be set.
cudaError_t launch_scene_audit(const SceneParams& p, cudaStream_t stream);

}  // namespace numi
