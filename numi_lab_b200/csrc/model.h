// Host-side compiled world: immutable records of one articulated world plus
// the derived tables the device kernels need (tree levels, ancestor DoF
// lists, eligible collider pairs).  One compiled model is shared by every
// environment of a rollout, like one CompiledWorld per MetalWorldContext in
// numi-lab (include/metalrobo/MetalWorld.hpp:107-217).
#pragma once

#include "numi_b200.h"

#include <cstdint>
#include <string>
#include <vector>

namespace numi {

// Counter-based seeded stream: value = f(seed, stream, index).  Independent
// of call order, so every environment / field draws reproducibly.
std::uint64_t mix64(std::uint64_t x);
double uniform01(std::uint64_t seed, std::uint64_t stream, std::uint64_t index);
double uniform(std::uint64_t seed, std::uint64_t stream, std::uint64_t index, double lo, double hi);
double normal(std::uint64_t seed, std::uint64_t stream, std::uint64_t index);

struct CompiledModel {
    MRModelWorldC world{};
    std::vector<MRModelJointC> joints;
    std::vector<MRModelBodyC> bodies;
    std::vector<MRModelDofC> dofs;
    std::vector<MRModelShapeC> shapes;
    std::vector<MRModelMaterialC> materials;
    std::vector<MRModelPairC> pairs;
    std::vector<float> hull_vertices;  // [vertex][4] unit-scale local hull vertices (MR_SHAPE_CONVEX)
    std::string name;

    // Reset-state generation parameters.
    std::vector<float> nominal_q;     // nq
    float q_joint_uniform_half_range = 0.0f;  // q_j ~ nominal + U(-r, r)
    float qd_joint_normal_sigma = 0.0f;       // qd_j ~ N(0, sigma)
    float root_yaw_half_range = 0.0f;
    float friction_scale_lo = 1.0f;   // per-env contact friction scale ~ U(lo, hi)
    float friction_scale_hi = 1.0f;

    // Derived (filled by finalize()).
    std::uint32_t articulated_body_count = 0;  // bodies [0, n) form the tree, DFS preorder
    std::uint32_t level_count = 0;
    std::vector<std::uint32_t> level_offsets;  // level_count + 1
    std::vector<std::uint32_t> level_bodies;   // bodies grouped by depth (depth >= 1)
    std::vector<std::uint32_t> subtree_end;    // DFS: subtree of b is [b, subtree_end[b])
    std::vector<std::uint32_t> body_dof;       // DoF index of a body's inbound joint or MR_INVALID_INDEX
    std::vector<std::uint32_t> dof_body;       // body moved by DoF (root DoFs -> root body)
    std::vector<std::uint32_t> dof_parent;     // nearest ancestor DoF (tree DoF order), MR_INVALID_INDEX at root
    std::uint32_t max_ancestor_dofs = 0;       // longest ancestor-DoF list over bodies
    std::vector<std::uint32_t> body_ancestor_dofs;  // [body][max_ancestor_dofs], ascending, padded MR_INVALID_INDEX
    std::vector<std::uint32_t> body_ancestor_count;

    std::uint64_t fingerprint = 0;

    // Free-body scene (pile) instead of an articulation: bodies [0, scene_bodies)
    // are dynamic, each with one collider at its COM; the last body is the
    // static ground with the plane collider.  q = [body][position, orientation],
    // v = [body][linear, angular velocity]; pairs are all collider pairs.
    bool scene = false;
    std::uint32_t scene_bodies = 0;
    float scene_cell = 0.0f;  // reset grid spacing
    // Reset layout of a scene: a dropped pile, or a box stack on the plane.
    // pile: one body per cell of a square grid, dropped from U(0.1, 1) m;
    // stack: a yawed column of boxes; heap: the grid in three offset layers
    // one cell apart in height, so that falling bodies land on each other.
    enum class SceneLayout : std::uint32_t { pile = 0, stack = 1, heap = 2 };
    SceneLayout scene_layout = SceneLayout::pile;
    float stack_offset_sigma = 0.0f;  // horizontal offsets of stacked boxes ~ N(0, sigma)

    void finalize();  // validates and fills derived tables; throws on error
};

CompiledModel build_chain7(std::uint64_t seed);
CompiledModel build_tree29(std::uint64_t seed);
// Pile of 8-64 free boxes, spheres and capsules (size U(0.05, 0.3) m, density
// U(500, 2000) kg/m^3) dropped onto a ground plane; the body count is drawn
// from the seed unless `bodies` is non-zero.
// `cylinders`: one quarter each of boxes, spheres, capsules and cylinders.
// gjk_capsule_box: capsule-box pairs take the support-mapped (GJK / EPA)
// narrowphase instead of the analytic witness.
// `hulls`: one quarter each of boxes, spheres, capsules and convex hulls of
// 12 vertices (unit directions with radii U(0.75, 1), scaled per axis).
CompiledModel build_pile(std::uint64_t seed, std::uint32_t bodies = 0, bool cylinders = false, bool gjk_capsule_box = false,
                         bool hulls = false);
// Stack of `boxes` 0.1 m, 1 kg cubes (friction 0.6) resting on a ground
// plane, the stack yawed U(0, 2 pi) and each box offset horizontally by
// N(0, 2 mm) at reset.
CompiledModel build_stack(std::uint64_t seed, std::uint32_t boxes = 32);

// Reset state for environment `env` (q: nq, v: nv) and its friction scale.
void sample_reset_state(const CompiledModel& model, std::uint64_t seed, std::uint32_t env,
                        float* q, float* v, float* friction_scale);

}  // namespace numi
