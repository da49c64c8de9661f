// Packed, immutable world description read by the microstep kernels.  One
// record per rollout lives in device memory; every environment of the
// rollout shares it (the model is small enough to stay L1/L2 resident).
#pragma once

#include <cstdint>

#include "numi_b200.h"

namespace numi {

constexpr int kMaxBodies = MR_B200_MAX_BODIES;
constexpr int kMaxDofs = MR_B200_MAX_DOFS;
constexpr int kMaxQ = MR_B200_MAX_Q;
constexpr int kMaxShapes = MR_B200_MAX_SHAPES;
constexpr int kMaxPairs = MR_B200_MAX_PAIRS;
constexpr int kMaxContacts = MR_B200_MAX_CONTACTS;
constexpr int kManifoldPoints = MR_B200_MANIFOLD_POINTS;
constexpr int kMaxMaterials = 8;
// Words of one persistent manifold slot in device memory (MRManifoldC).
constexpr int kManifoldWords = 8 + kManifoldPoints * 12;

// Byte-sized topology tables copied into each CTA's shared memory at kernel
// start: every cross-lane index lookup of the sweeps reads shared memory,
// never global memory.  255 marks "none".
struct alignas(16) DeviceTables {
    std::uint8_t nb, nv, nq, n_levels;
    std::uint8_t floating, ns, np, max_anc;
    std::uint8_t n_dof_levels, reserved[7];
    std::uint8_t depth[kMaxBodies];          // tree depth of each body (root 0)
    std::uint8_t parent[kMaxBodies];
    std::uint8_t body_dof[kMaxBodies];
    std::uint8_t child_offsets[kMaxBodies + 1];
    std::uint8_t children[kMaxBodies];
    std::uint8_t anc_count[kMaxBodies];
    std::uint8_t dof_body[kMaxDofs];
    std::uint8_t dof_parent[kMaxDofs];
    std::uint8_t dof_depth[kMaxDofs];        // number of ancestor DoFs
    std::uint8_t anc[kMaxBodies][kMaxDofs];  // ancestor DoFs of a body, root first
    std::uint8_t pos[kMaxBodies][kMaxDofs];  // position of DoF d in anc[b], or 255
    std::uint8_t lcp[kMaxBodies][kMaxBodies];// common prefix length of anc[a], anc[b]
    std::uint8_t level_children[kMaxBodies]; // most children of a body at each depth
    std::uint8_t pad[7];
};

struct alignas(16) DeviceModel {
    DeviceTables tables;
    // World.
    std::int32_t nb;              // articulated bodies, DFS preorder, body 0 = root
    std::int32_t nv;
    std::int32_t nq;
    std::int32_t floating;        // 1 floating root, 0 fixed root
    std::int32_t n_levels;        // tree depth (levels 1..n_levels)
    std::int32_t action_count;
    std::int32_t implicit_drives; // MR_ACTUATION_IMPLICIT_POSITION
    std::int32_t apply_damping;
    std::int32_t ns;              // shapes
    std::int32_t np;              // compiled pairs
    std::int32_t contact_capacity;
    std::int32_t max_anc;         // stride of anc_dofs rows
    float gravity[4];
    float h;                      // physics substep
    float slop;
    float max_depenetration;
    float speculative_scale;
    float speed_envelope;
    float manifold_thresholds[4]; // breaking separation, drift, merge, normal cosine
    float reserved0[3];

    // Tree.
    std::int32_t level_offsets[kMaxBodies + 1];
    std::int32_t level_bodies[kMaxBodies];
    std::int32_t parent[kMaxBodies];
    std::int32_t subtree_end[kMaxBodies];
    std::int32_t body_dof[kMaxBodies];     // -1 fixed joint / root
    std::int32_t joint_type[kMaxBodies];
    std::int32_t child_offsets[kMaxBodies + 1];
    std::int32_t children[kMaxBodies];
    float4 axis[kMaxBodies];               // normalised joint-frame axis
    float4 parent_anchor[kMaxBodies];
    float4 child_anchor[kMaxBodies];
    float4 parent_rotation[kMaxBodies];    // normalised
    float4 child_rotation_conj[kMaxBodies];// conjugate of normalised child rotation
    float4 mass_damping[kMaxBodies];       // mass, linear damping, angular damping, 0
    float4 inertia_diag[kMaxBodies];       // body-frame Ixx, Iyy, Izz
    float4 inertia_off[kMaxBodies];        // body-frame Ixy, Ixz, Iyz
    std::int32_t anc_count[kMaxBodies];
    std::int32_t anc_dofs[kMaxBodies * kMaxDofs];

    // DoFs.
    std::int32_t dof_body[kMaxDofs];
    std::int32_t dof_parent[kMaxDofs];
    std::int32_t dof_anc_count[kMaxDofs];  // ancestors of a DoF = first entries of anc_dofs[dof_body]
    std::int32_t dof_q[kMaxDofs];          // -1 when no scalar coordinate
    std::uint32_t dof_flags[kMaxDofs];
    float armature_eff[kMaxDofs];          // armature (+ h kd + h^2 kp for implicit drives)
    float kp[kMaxDofs];
    float kd[kMaxDofs];
    float dry_friction[kMaxDofs];
    float effort_envelope[kMaxDofs];       // min(limit.w, default stall torque)
    float effort_limit[kMaxDofs];          // limits.w when EFFORT_LIMIT
    float q_lower[kMaxDofs];
    float q_upper[kMaxDofs];
    float v_max[kMaxDofs];
    std::int32_t action_dof[kMaxDofs];     // action a drives DoF action_dof[a]

    // Shapes.
    std::int32_t shape_body[kMaxShapes];   // articulated body index, or -1 for static
    std::int32_t shape_type[kMaxShapes];
    std::int32_t shape_material[kMaxShapes];
    std::int32_t reserved1;
    float4 shape_position[kMaxShapes];     // local position (articulated) or world (static)
    float4 shape_rotation[kMaxShapes];     // normalised local (articulated) or world (static)
    float4 shape_dims[kMaxShapes];
    float4 shape_offsets[kMaxShapes];      // contact offset, rest offset, sweep radius, 0
    float4 static_body_position[kMaxShapes];  // pose of a static shape's body
    float4 static_body_rotation[kMaxShapes];

    // Pairs (shape_a < shape_b; shape_a is never static for supported classes).
    std::int32_t pair_a[kMaxPairs];
    std::int32_t pair_b[kMaxPairs];
    std::int32_t pair_class[kMaxPairs];
    std::int32_t pair_max_points[kMaxPairs];

    float4 material_friction[kMaxMaterials];
    float4 material_response[kMaxMaterials];
};

// Settings of the converged (quality) contact solve, MRQualitySolverConfigC
// with its defaults applied (quality.cuh).
struct QualityConfig {
    std::int32_t max_newton;
    std::int32_t max_line_search;  // evaluations of the line search's phi' per Newton step
    double tolerance;              // on ||zeta - Y lambda||_inf / (1 + ||zeta||_inf + ||Y lambda||_inf)
    double line_search_tolerance;  // |phi'(t)| relative to |phi'(0)|
    double regularization_floor;
};

// Launch parameters of one control step of one rollout.
struct StepParams {
    const DeviceModel* model;
    float* q;                      // [env][nq] resident state (in/out)
    float* v;                      // [env][nv]
    float* manifolds;              // [env][np][kManifoldWords]
    const float* reset_q;          // [env][nq]
    const float* reset_v;          // [env][nv]
    const float* friction_scale;   // [env]
    const float* actions;          // [item][action_count] of this control step
    const float* const* action_rows;   // per item: its action row, or null (use `actions`)
    const std::int32_t* env_index;     // per item: resident environment slot, or null (item = slot)
    const std::uint32_t* reset_masks;  // [item] of this control step, or null
    float* observations;           // [item][nq+nv] of this control step, or null
    std::uint32_t* status_codes;   // [item] of this control step, or null
    std::uint32_t* active_contacts;// [item] of this control step, or null
    std::uint32_t* stats;          // per-launch counters (see kStat*)
    std::int32_t env_count;
    std::int32_t substeps;
    std::int32_t velocity_iterations;
    std::int32_t final_velocity_iterations;
    float* q_comp;                 // [env][nq] compensation terms of q's running sums (compensated precision), or null
    std::int32_t env_base;         // slot index of this launch's slot 0 (counters report absolute slots)
    double* audit;                 // [env][kAuditWords] FP64 energy / momentum audit (audit.cuh), or null
    QualityConfig quality;         // read by the quality-solver kernel instances only
};

enum StatIndex : int {
    kStatFailedEnvs = 0,
    kStatMaxContacts = 1,
    kStatMaxManifolds = 2,
    kStatMaxRawContacts = 3,
    kStatMaxCandidatePairs = 4,
    kStatMaxIslands = 5,
    kStatFirstFailEnv = 6,
    kStatFirstFailCode = 7,
    kStatResets = 8,
    kStatWorldMismatch = 9,  // scene items skipped: the world record was not the one the launch was enqueued for
    // Quality solver (largest over the launch's environment-substeps; the
    // FP32 bit patterns of non-negative values order like the values).
    kStatQualityNewton = 10,       // Newton steps of one solve
    kStatQualityLineSearch = 11,   // line-search evaluations, summed
    kStatQualityResidual = 12,     // scaled optimality (FP32 bits)
    kStatQualityCone = 13,         // cone violation (FP32 bits)
    kStatQualityComplementarity = 14,  // conic complementarity (FP32 bits)
    kStatCount = 16
};

}  // namespace numi
