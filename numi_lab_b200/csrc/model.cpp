// Seeded synthetic world compilers and reset-state sampling.
//
// Record meanings follow numi-lab's engine ABI (include/metalrobo/
// engine_types.h:284-434, 1349-1455): anchors are relative to each body's
// centre of mass, joint-frame rotations are xyzw quaternions, planes use the
// shape's local +Y as their normal, floating roots store q = (COM xyz,
// quaternion xyzw, joints) and v = (COM linear velocity, world angular
// velocity, joint rates).
#include "model.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <stdexcept>

namespace numi {

std::uint64_t mix64(std::uint64_t x) {
    // splitmix64 finaliser (Steele, Lea & Flood, OOPSLA 2014).
    x += 0x9e3779b97f4a7c15ull;
    x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
    x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
    return x ^ (x >> 31);
}

double uniform01(std::uint64_t seed, std::uint64_t stream, std::uint64_t index) {
    const std::uint64_t h = mix64(mix64(mix64(seed) ^ (stream * 0x632be59bd9b4e019ull)) ^ index);
    return (static_cast<double>(h >> 11) + 0.5) * (1.0 / 9007199254740992.0);
}

double uniform(std::uint64_t seed, std::uint64_t stream, std::uint64_t index, double lo, double hi) {
    return lo + (hi - lo) * uniform01(seed, stream, index);
}

double normal(std::uint64_t seed, std::uint64_t stream, std::uint64_t index) {
    // Box-Muller on two independent counter draws.
    const double u1 = uniform01(seed, stream, 2 * index);
    const double u2 = uniform01(seed, stream, 2 * index + 1);
    return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
}

namespace {

constexpr std::uint64_t kStreamModel = 1;
constexpr std::uint64_t kStreamResetQ = 2;
constexpr std::uint64_t kStreamResetV = 3;
constexpr std::uint64_t kStreamResetRoot = 4;
constexpr std::uint64_t kStreamFriction = 5;

void set4(float* d, double a, double b, double c, double w) {
    d[0] = static_cast<float>(a);
    d[1] = static_cast<float>(b);
    d[2] = static_cast<float>(c);
    d[3] = static_cast<float>(w);
}

MRModelBodyC box_body(std::uint32_t parent, std::uint32_t joint, double mass, double dx, double dy, double dz) {
    MRModelBodyC b{};
    b.parent_body = parent;
    b.inbound_joint = joint;
    b.motion_type = MR_MOTION_DYNAMIC;
    b.articulated = 1u;
    set4(b.mass_inverse_mass, mass, 1.0 / mass, 0.0, 0.0);
    const double ixx = mass * (dy * dy + dz * dz) / 12.0;
    const double iyy = mass * (dx * dx + dz * dz) / 12.0;
    const double izz = mass * (dx * dx + dy * dy) / 12.0;
    set4(b.inertia[0], ixx, 0.0, 0.0, 0.0);
    set4(b.inertia[1], 0.0, iyy, 0.0, 0.0);
    set4(b.inertia[2], 0.0, 0.0, izz, 0.0);
    set4(b.damping_speed, 0.0, 0.0, 0.0, 0.0);
    set4(b.static_pose, 0.0, 0.0, 0.0, 0.0);
    set4(b.static_pose + 4, 0.0, 0.0, 0.0, 1.0);
    return b;
}

MRModelJointC revolute(std::uint32_t parent, std::uint32_t child, int axis,
                       const double pa[3], const double child_com_from_joint[3]) {
    MRModelJointC j{};
    j.parent_body = parent;
    j.child_body = child;
    j.joint_type = MR_JOINT_REVOLUTE;
    set4(j.axis, axis == 0 ? 1.0 : 0.0, axis == 1 ? 1.0 : 0.0, axis == 2 ? 1.0 : 0.0, 0.0);
    set4(j.parent_anchor, pa[0], pa[1], pa[2], 0.0);
    set4(j.child_anchor, -child_com_from_joint[0], -child_com_from_joint[1], -child_com_from_joint[2], 0.0);
    set4(j.parent_rotation, 0.0, 0.0, 0.0, 1.0);
    set4(j.child_rotation, 0.0, 0.0, 0.0, 1.0);
    return j;
}

std::uint64_t hash_bytes(std::uint64_t h, const void* data, std::size_t n) {
    const unsigned char* p = static_cast<const unsigned char*>(data);
    for (std::size_t i = 0; i < n; ++i) {
        h = (h ^ p[i]) * 0x100000001b3ull;
    }
    return h;
}

}  // namespace

void CompiledModel::finalize() {
    const std::uint32_t nb = world.body_count;
    if (scene) {
        if (scene_bodies == 0 || scene_bodies > 64 || nb != scene_bodies + 1) throw std::runtime_error("scene body count outside capacity");
        if (world.nq != 7 * scene_bodies || world.nv != 6 * scene_bodies) throw std::runtime_error("scene nq/nv mismatch");
        articulated_body_count = 0;
        std::uint64_t h = 0x9e3779b97f4a7c15ull;
        auto mixin = [&](const void* data, std::size_t bytes) {
            const unsigned char* p = static_cast<const unsigned char*>(data);
            for (std::size_t i = 0; i < bytes; ++i) h = (h ^ p[i]) * 0x100000001b3ull;
        };
        mixin(&world, sizeof(world));
        mixin(bodies.data(), bodies.size() * sizeof(MRModelBodyC));
        mixin(shapes.data(), shapes.size() * sizeof(MRModelShapeC));
        if (!hull_vertices.empty()) mixin(hull_vertices.data(), hull_vertices.size() * sizeof(float));
        fingerprint = h;
        return;
    }
    if (nb == 0 || nb > MR_B200_MAX_BODIES + 1) throw std::runtime_error("body count outside capacity");
    if (world.nv == 0 || world.nv > MR_B200_MAX_DOFS || world.nq > MR_B200_MAX_Q)
        throw std::runtime_error("nq/nv outside capacity");
    if (world.shape_count > MR_B200_MAX_SHAPES || world.pair_count > MR_B200_MAX_PAIRS)
        throw std::runtime_error("shape/pair count outside capacity");
    // Articulated bodies occupy [0, n) in DFS preorder; statics follow.
    articulated_body_count = 0;
    while (articulated_body_count < nb && bodies[articulated_body_count].articulated) ++articulated_body_count;
    for (std::uint32_t b = articulated_body_count; b < nb; ++b) {
        if (bodies[b].articulated || bodies[b].motion_type != MR_MOTION_STATIC)
            throw std::runtime_error("non-articulated bodies must be static and follow the tree");
    }
    const std::uint32_t na = articulated_body_count;
    if (na == 0 || na > MR_B200_MAX_BODIES) throw std::runtime_error("articulation size outside capacity");
    if (bodies[0].parent_body != MR_INVALID_INDEX) throw std::runtime_error("body 0 must be the root");
    std::vector<std::uint32_t> depth(na, 0);
    subtree_end.assign(na, 0);
    for (std::uint32_t b = 1; b < na; ++b) {
        const std::uint32_t p = bodies[b].parent_body;
        if (p >= b) throw std::runtime_error("bodies must be in DFS preorder (parent before child)");
        depth[b] = depth[p] + 1;
        const MRModelJointC& j = joints[bodies[b].inbound_joint];
        if (j.child_body != b || j.parent_body != p) throw std::runtime_error("joint/body topology mismatch");
    }
    // DFS preorder check: subtree of b is contiguous.
    for (std::uint32_t b = 0; b < na; ++b) {
        std::uint32_t e = b + 1;
        while (e < na) {
            std::uint32_t a = bodies[e].parent_body;
            bool inside = false;
            while (a != MR_INVALID_INDEX) {
                if (a == b) { inside = true; break; }
                a = bodies[a].parent_body;
            }
            if (!inside) break;
            ++e;
        }
        subtree_end[b] = e;
    }
    for (std::uint32_t b = 0; b < na; ++b) {
        for (std::uint32_t c = subtree_end[b]; c < na; ++c) {
            std::uint32_t a = bodies[c].parent_body;
            while (a != MR_INVALID_INDEX) {
                if (a == b) throw std::runtime_error("bodies are not in DFS preorder");
                a = bodies[a].parent_body;
            }
        }
    }
    std::uint32_t max_depth = 0;
    for (std::uint32_t b = 0; b < na; ++b) max_depth = std::max(max_depth, depth[b]);
    level_count = max_depth;
    level_offsets.assign(level_count + 1, 0);
    level_bodies.clear();
    for (std::uint32_t l = 1; l <= max_depth; ++l) {
        level_offsets[l - 1] = static_cast<std::uint32_t>(level_bodies.size());
        for (std::uint32_t b = 1; b < na; ++b)
            if (depth[b] == l) level_bodies.push_back(b);
        if (level_bodies.size() - level_offsets[l - 1] > 32) throw std::runtime_error("more than 32 bodies in one tree level");
    }
    level_offsets[level_count] = static_cast<std::uint32_t>(level_bodies.size());

    // DoF tables.
    const std::uint32_t root_dofs = world.root_type == MR_ROOT_FLOATING ? 6u : 0u;
    body_dof.assign(na, MR_INVALID_INDEX);
    dof_body.assign(world.nv, 0);
    for (std::uint32_t d = 0; d < root_dofs; ++d) dof_body[d] = 0;
    for (std::uint32_t b = 1; b < na; ++b) {
        const MRModelJointC& j = joints[bodies[b].inbound_joint];
        if (j.joint_type == MR_JOINT_FIXED) continue;
        if (j.v_index >= world.nv) throw std::runtime_error("joint v_index out of range");
        body_dof[b] = j.v_index;
        dof_body[j.v_index] = b;
    }
    dof_parent.assign(world.nv, MR_INVALID_INDEX);
    for (std::uint32_t d = 1; d < root_dofs; ++d) dof_parent[d] = d - 1;
    max_ancestor_dofs = 0;
    std::vector<std::vector<std::uint32_t>> anc(na);
    for (std::uint32_t b = 0; b < na; ++b) {
        std::vector<std::uint32_t> list;
        for (std::uint32_t d = 0; d < root_dofs; ++d) list.push_back(d);
        std::vector<std::uint32_t> chain;
        std::uint32_t a = b;
        while (a != MR_INVALID_INDEX && a != 0) {
            if (body_dof[a] != MR_INVALID_INDEX) chain.push_back(body_dof[a]);
            a = bodies[a].parent_body;
        }
        std::reverse(chain.begin(), chain.end());
        list.insert(list.end(), chain.begin(), chain.end());
        for (std::size_t i = 1; i < list.size(); ++i) {
            if (list[i] <= list[i - 1]) throw std::runtime_error("DoFs must increase along every root-to-leaf path");
        }
        anc[b] = list;
        max_ancestor_dofs = std::max<std::uint32_t>(max_ancestor_dofs, static_cast<std::uint32_t>(list.size()));
    }
    for (std::uint32_t b = 1; b < na; ++b) {
        const std::uint32_t d = body_dof[b];
        if (d == MR_INVALID_INDEX) continue;
        const auto& list = anc[b];
        dof_parent[d] = list.size() >= 2 ? list[list.size() - 2] : MR_INVALID_INDEX;
    }
    if (max_ancestor_dofs == 0) max_ancestor_dofs = 1;
    body_ancestor_dofs.assign(static_cast<std::size_t>(na) * max_ancestor_dofs, MR_INVALID_INDEX);
    body_ancestor_count.assign(na, 0);
    for (std::uint32_t b = 0; b < na; ++b) {
        body_ancestor_count[b] = static_cast<std::uint32_t>(anc[b].size());
        for (std::size_t i = 0; i < anc[b].size(); ++i) body_ancestor_dofs[b * max_ancestor_dofs + i] = anc[b][i];
    }
    // Pair validation and contact capacity.
    std::uint32_t capacity = 0;
    for (const MRModelPairC& p : pairs) {
        if (p.shape_a >= p.shape_b || p.shape_b >= world.shape_count) throw std::runtime_error("invalid pair");
        capacity += p.max_points;
    }
    world.contact_capacity = std::min<std::uint32_t>(capacity, MR_B200_MAX_CONTACTS);

    std::uint64_t h = 0xcbf29ce484222325ull;
    h = hash_bytes(h, &world, sizeof(world));
    h = hash_bytes(h, joints.data(), joints.size() * sizeof(MRModelJointC));
    h = hash_bytes(h, bodies.data(), bodies.size() * sizeof(MRModelBodyC));
    h = hash_bytes(h, dofs.data(), dofs.size() * sizeof(MRModelDofC));
    h = hash_bytes(h, shapes.data(), shapes.size() * sizeof(MRModelShapeC));
    h = hash_bytes(h, materials.data(), materials.size() * sizeof(MRModelMaterialC));
    h = hash_bytes(h, pairs.data(), pairs.size() * sizeof(MRModelPairC));
    fingerprint = h == 0 ? 1 : h;
}

// Fixed-base 7-revolute serial chain: link lengths U(0.1, 0.3) m, masses
// U(0.5, 4) kg, solid-box inertias with dims U(0.04, 0.12) m, joint axes
// alternating z / y, effort actuation, no colliders.
CompiledModel build_chain7(std::uint64_t seed) {
    CompiledModel m;
    m.name = "synthetic_chain7";
    const std::uint32_t links = 7;
    std::uint64_t k = 0;
    auto draw = [&](double lo, double hi) { return uniform(seed, kStreamModel, k++, lo, hi); };
    MRModelBodyC base = box_body(MR_INVALID_INDEX, MR_INVALID_INDEX, 5.0, 0.2, 0.2, 0.1);
    m.bodies.push_back(base);
    double prev_half = 0.05;  // joint 1 sits 5 cm above the base origin
    for (std::uint32_t i = 1; i <= links; ++i) {
        const double length = draw(0.1, 0.3);
        const double mass = draw(0.5, 4.0);
        const double dx = draw(0.04, 0.12), dy = draw(0.04, 0.12), dz = draw(0.04, 0.12);
        const double pa[3] = {0.0, 0.0, prev_half};
        const double cc[3] = {0.0, 0.0, 0.5 * length};
        MRModelJointC j = revolute(i - 1, i, (i % 2 == 1) ? 2 : 1, pa, cc);
        j.q_index = i - 1;
        j.v_index = i - 1;
        m.joints.push_back(j);
        m.bodies.push_back(box_body(i - 1, i - 1, mass, dx, dy, dz));
        prev_half = 0.5 * length;
        MRModelDofC d{};
        d.joint_index = i - 1;
        d.q_index = i - 1;
        d.flags = MR_DOF_FLAG_ACTUATED | MR_DOF_FLAG_EFFORT_LIMIT;
        set4(d.limits, 0.0, 0.0, 0.0, 500.0);
        set4(d.drive, 0.0, 0.0, 0.0, 0.0);
        m.dofs.push_back(d);
    }
    m.world.body_count = static_cast<std::uint32_t>(m.bodies.size());
    m.world.joint_count = static_cast<std::uint32_t>(m.joints.size());
    m.world.nq = links;
    m.world.nv = links;
    m.world.root_type = MR_ROOT_FIXED;
    m.world.actuation_mode = MR_ACTUATION_EFFORT;
    m.world.action_count = links;
    m.world.apply_body_damping = 1u;
    set4(m.world.gravity, 0.0, 0.0, -9.81, 0.0);
    set4(m.world.solver_scales, 1.0e-7, 1.0e-9, 2.0, 1.0e-4);
    set4(m.world.manifold_thresholds, 0.02, 0.02, 0.002, 0.95);
    set4(m.world.speculative, 1.0, 1.0e4, 0.0, 0.0);
    m.nominal_q.assign(links, 0.0f);
    m.q_joint_uniform_half_range = static_cast<float>(1.5707963267948966);
    m.qd_joint_normal_sigma = 1.0f;
    m.finalize();
    return m;
}

// Floating 29-DoF humanoid tree with the Unitree G1 topology (pelvis root,
// 2 x 6-DoF legs, 3-DoF waist, 2 x 7-DoF arms; body order as in numi-lab's
// src/core/G1.cpp) and seeded synthetic dimensions: masses U(0.3, 8) kg,
// box feet 0.2 x 0.08 x 0.03 m, 12 sphere proxies r ~ U(0.03, 0.08) m,
// implicit PD drives, on a ground plane.
CompiledModel build_tree29(std::uint64_t seed) {
    CompiledModel m;
    m.name = "synthetic_tree29";
    std::uint64_t k = 0;
    auto draw = [&](double lo, double hi) { return uniform(seed, kStreamModel, k++, lo, hi); };
    struct LinkSpec {
        std::uint32_t parent;
        int axis;            // 0 x, 1 y, 2 z
        double pa[3];        // joint position from parent COM
        double cc[3];        // child COM from joint
        double dims[3];      // inertia box
    };
    std::vector<LinkSpec> links;  // index = body - 1
    const double thigh = draw(0.30, 0.40), shin = draw(0.30, 0.40);
    const double torso = draw(0.25, 0.35), upper_arm = draw(0.18, 0.25), forearm = draw(0.15, 0.22);
    auto leg = [&](double s) {
        const std::uint32_t b0 = static_cast<std::uint32_t>(links.size()) + 1;
        links.push_back({0, 1, {0.0, s * 0.09, -0.08}, {0.0, s * 0.02, -0.03}, {0.06, 0.06, 0.06}});
        links.push_back({b0, 0, {0.0, 0.0, -0.03}, {0.0, 0.0, -0.04}, {0.07, 0.07, 0.08}});
        links.push_back({b0 + 1, 2, {0.0, 0.0, -0.04}, {0.0, 0.0, -0.5 * thigh}, {0.08, 0.08, thigh}});
        links.push_back({b0 + 2, 1, {0.0, 0.0, -0.5 * thigh}, {0.0, 0.0, -0.5 * shin}, {0.07, 0.07, shin}});
        links.push_back({b0 + 3, 1, {0.0, 0.0, -0.5 * shin}, {0.0, 0.0, -0.01}, {0.04, 0.04, 0.04}});
        links.push_back({b0 + 4, 0, {0.0, 0.0, -0.01}, {0.03, 0.0, -0.03}, {0.2, 0.08, 0.03}});
    };
    leg(+1.0);  // bodies 1..6, left
    leg(-1.0);  // bodies 7..12, right
    links.push_back({0, 2, {0.0, 0.0, 0.06}, {0.0, 0.0, 0.02}, {0.06, 0.06, 0.04}});        // 13 waist yaw
    links.push_back({13, 0, {0.0, 0.0, 0.02}, {0.0, 0.0, 0.02}, {0.06, 0.06, 0.04}});       // 14 waist roll
    links.push_back({14, 1, {0.0, 0.0, 0.02}, {0.0, 0.0, 0.5 * torso}, {0.2, 0.3, torso}}); // 15 torso
    auto arm = [&](double s) {
        const std::uint32_t b0 = static_cast<std::uint32_t>(links.size()) + 1;
        links.push_back({15, 1, {0.0, s * 0.15, 0.5 * torso - 0.05}, {0.0, s * 0.04, 0.0}, {0.05, 0.05, 0.05}});
        links.push_back({b0, 0, {0.0, s * 0.02, 0.0}, {0.0, 0.0, -0.03}, {0.05, 0.05, 0.06}});
        links.push_back({b0 + 1, 2, {0.0, 0.0, -0.03}, {0.0, 0.0, -0.5 * upper_arm}, {0.06, 0.06, upper_arm}});
        links.push_back({b0 + 2, 1, {0.0, 0.0, -0.5 * upper_arm}, {0.0, 0.0, -0.5 * forearm}, {0.05, 0.05, forearm}});
        links.push_back({b0 + 3, 0, {0.0, 0.0, -0.5 * forearm}, {0.0, 0.0, -0.02}, {0.04, 0.04, 0.04}});
        links.push_back({b0 + 4, 1, {0.0, 0.0, -0.02}, {0.0, 0.0, -0.02}, {0.04, 0.04, 0.04}});
        links.push_back({b0 + 5, 2, {0.0, 0.0, -0.02}, {0.0, 0.0, -0.05}, {0.06, 0.04, 0.08}});
    };
    arm(+1.0);  // bodies 16..22, left
    arm(-1.0);  // bodies 23..29, right

    m.bodies.push_back(box_body(MR_INVALID_INDEX, MR_INVALID_INDEX, draw(0.3, 8.0), 0.2, 0.25, 0.12));
    for (std::size_t i = 0; i < links.size(); ++i) {
        const LinkSpec& s = links[i];
        const std::uint32_t body = static_cast<std::uint32_t>(i) + 1;
        MRModelJointC j = revolute(s.parent, body, s.axis, s.pa, s.cc);
        j.q_index = 7 + static_cast<std::uint32_t>(i);
        j.v_index = 6 + static_cast<std::uint32_t>(i);
        m.joints.push_back(j);
        m.bodies.push_back(box_body(s.parent, static_cast<std::uint32_t>(i), draw(0.3, 8.0), s.dims[0], s.dims[1], s.dims[2]));
    }
    // Static ground body (plane collider), after the tree.
    MRModelBodyC ground{};
    ground.parent_body = MR_INVALID_INDEX;
    ground.inbound_joint = MR_INVALID_INDEX;
    ground.motion_type = MR_MOTION_STATIC;
    ground.articulated = 0u;
    set4(ground.mass_inverse_mass, 0.0, 0.0, 0.0, 0.0);
    set4(ground.static_pose, 0.0, 0.0, 0.0, 0.0);
    set4(ground.static_pose + 4, 0.0, 0.0, 0.0, 1.0);
    m.bodies.push_back(ground);
    const std::uint32_t ground_body = static_cast<std::uint32_t>(m.bodies.size()) - 1;

    // Root DoFs (reference: src/core/G1.cpp, root records carry only the ROOT flag).
    for (std::uint32_t d = 0; d < 6; ++d) {
        MRModelDofC dof{};
        dof.joint_index = MR_INVALID_INDEX;
        dof.q_index = d < 3 ? d : MR_INVALID_INDEX;
        dof.flags = MR_DOF_FLAG_ROOT;
        m.dofs.push_back(dof);
    }
    for (std::uint32_t i = 0; i < links.size(); ++i) {
        MRModelDofC dof{};
        dof.joint_index = i;
        dof.q_index = 7 + i;
        dof.flags = MR_DOF_FLAG_ACTUATED | MR_DOF_FLAG_POSITION_LIMIT | MR_DOF_FLAG_VELOCITY_LIMIT |
                    MR_DOF_FLAG_EFFORT_LIMIT | MR_DOF_FLAG_DRIVE;
        set4(dof.limits, -2.5, 2.5, 30.0, draw(60.0, 150.0));
        set4(dof.drive, draw(40.0, 120.0), draw(1.0, 4.0), draw(0.01, 0.05), 0.0);
        m.dofs.push_back(dof);
    }

    // Materials: robot and ground; per-environment friction scale multiplies
    // the geometric-mean coefficient.
    MRModelMaterialC mat{};
    set4(mat.friction, 1.0, 1.0, 0.0, 0.0);
    set4(mat.response, 0.0, 0.5, 0.0, 0.0);
    m.materials.push_back(mat);
    m.materials.push_back(mat);

    auto shape = [&](std::uint32_t body, std::uint32_t type, std::uint32_t material, const double lp[3],
                     const double dims[3], double bound) {
        MRModelShapeC s{};
        s.body = body;
        s.shape_type = type;
        s.material = material;
        s.collision_group = type == MR_SHAPE_PLANE ? 2u : 1u;
        s.collision_mask = type == MR_SHAPE_PLANE ? 1u : 2u;
        set4(s.local_position, lp[0], lp[1], lp[2], 0.0);
        set4(s.local_rotation, 0.0, 0.0, 0.0, 1.0);
        set4(s.dimensions, dims[0], dims[1], dims[2], 0.0);
        set4(s.contact_rest_bound, 0.002, 0.0, bound, 0.0);
        return s;
    };
    const double foot_local[3] = {0.01, 0.0, -0.015};
    const double foot_half[3] = {0.1, 0.04, 0.015};
    const double foot_bound = std::sqrt(0.1 * 0.1 + 0.04 * 0.04 + 0.015 * 0.015);
    m.shapes.push_back(shape(6, MR_SHAPE_BOX, 0, foot_local, foot_half, foot_bound));
    m.shapes.push_back(shape(12, MR_SHAPE_BOX, 0, foot_local, foot_half, foot_bound));
    const std::uint32_t sphere_bodies[12] = {0, 15, 3, 9, 4, 10, 17, 24, 19, 26, 22, 29};
    for (std::uint32_t b : sphere_bodies) {
        const double r = draw(0.03, 0.08);
        const double zero[3] = {0.0, 0.0, 0.0};
        const double dims[3] = {r, 0.0, 0.0};
        m.shapes.push_back(shape(b, MR_SHAPE_SPHERE, 0, zero, dims, r));
    }
    {
        const double zero[3] = {0.0, 0.0, 0.0};
        MRModelShapeC plane = shape(ground_body, MR_SHAPE_PLANE, 1, zero, zero, 0.0);
        // local +Y -> world +Z: rotation of +90 degrees about x.
        const double h = std::sqrt(0.5);
        set4(plane.local_rotation, h, 0.0, 0.0, h);
        set4(plane.contact_rest_bound, 0.0, 0.0, 0.0, 0.0);
        m.shapes.push_back(plane);
    }
    const std::uint32_t plane_index = static_cast<std::uint32_t>(m.shapes.size()) - 1;
    for (std::uint32_t s = 0; s < plane_index; ++s) {
        MRModelPairC p{};
        p.shape_a = s;
        p.shape_b = plane_index;
        p.pair_class = m.shapes[s].shape_type == MR_SHAPE_BOX ? MR_COLLISION_PAIR_BOX_PLANE : MR_COLLISION_PAIR_SPHERE_PLANE;
        p.max_points = m.shapes[s].shape_type == MR_SHAPE_BOX ? 4u : 1u;
        m.pairs.push_back(p);
    }

    m.world.body_count = static_cast<std::uint32_t>(m.bodies.size());
    m.world.joint_count = static_cast<std::uint32_t>(m.joints.size());
    m.world.nq = 36;
    m.world.nv = 35;
    m.world.shape_count = static_cast<std::uint32_t>(m.shapes.size());
    m.world.material_count = static_cast<std::uint32_t>(m.materials.size());
    m.world.pair_count = static_cast<std::uint32_t>(m.pairs.size());
    m.world.root_type = MR_ROOT_FLOATING;
    m.world.actuation_mode = MR_ACTUATION_IMPLICIT_POSITION;
    m.world.action_count = 29;
    m.world.apply_body_damping = 1u;
    set4(m.world.gravity, 0.0, 0.0, -9.81, 0.0);
    set4(m.world.solver_scales, 1.0e-7, 1.0e-9, 2.0, 1.0e-4);
    set4(m.world.manifold_thresholds, 0.02, 0.02, 0.002, 0.95);
    set4(m.world.speculative, 1.0, 1.0e4, 0.0, 0.0);

    // Nominal standing pose: all joints zero; root height puts the lowest
    // foot-box vertex 0.5 mm above the plane (identity link rotations at
    // zero joint angles, so offsets add directly).
    std::vector<double> com_z(m.bodies.size(), 0.0);
    for (std::size_t i = 0; i < links.size(); ++i) {
        const LinkSpec& s = links[i];
        com_z[i + 1] = com_z[s.parent] + s.pa[2] + s.cc[2];
    }
    double lowest = 1e9;
    for (std::uint32_t f = 0; f < 2; ++f) {
        const MRModelShapeC& foot = m.shapes[f];
        lowest = std::min(lowest, com_z[foot.body] + foot.local_position[2] - foot.dimensions[2]);
    }
    m.nominal_q.assign(m.world.nq, 0.0f);
    m.nominal_q[2] = static_cast<float>(-lowest + 0.0005);
    m.nominal_q[6] = 1.0f;
    m.q_joint_uniform_half_range = 0.1f;
    m.qd_joint_normal_sigma = 0.0f;
    m.root_yaw_half_range = static_cast<float>(3.141592653589793);
    m.friction_scale_lo = 0.4f;
    m.friction_scale_hi = 1.0f;
    (void)ground_body;
    m.finalize();
    return m;
}

// Ground body with the plane collider, materials, the all-pairs list in key
// order (a, b), b = n for the plane, and the world record of a scene with
// `n` free bodies already in m.bodies / m.shapes.
static void finish_scene(CompiledModel& m, std::uint32_t n, double friction, bool gjk_capsule_box = false) {
    MRModelBodyC ground{};
    ground.parent_body = MR_INVALID_INDEX;
    ground.inbound_joint = MR_INVALID_INDEX;
    ground.motion_type = MR_MOTION_STATIC;
    set4(ground.static_pose + 4, 0.0, 0.0, 0.0, 1.0);
    m.bodies.push_back(ground);
    {
        MRModelShapeC plane{};
        plane.body = n;
        plane.shape_type = MR_SHAPE_PLANE;
        plane.material = 1;
        plane.collision_group = 2u;
        plane.collision_mask = 1u;
        const double h = std::sqrt(0.5);
        set4(plane.local_rotation, h, 0.0, 0.0, h);  // local +Y -> world +Z
        m.shapes.push_back(plane);
    }
    MRModelMaterialC mat{};
    set4(mat.friction, friction, friction, 0.0, 0.0);
    set4(mat.response, 0.0, 0.5, 0.0, 0.0);
    m.materials.push_back(mat);
    m.materials.push_back(mat);
    // Pair classes as the reference compiles them (MetalWorld.mm:1413-1500):
    // a cylinder against the plane is analytic, against any finite shape
    // support-mapped (GJK / EPA); a hull against anything, the plane
    // included, takes the hull path of the support-mapped query
    // (Collision.metal:8026-8045, 3623-3720).
    auto cls = [&](std::uint32_t a, std::uint32_t b) {
        const std::uint32_t ta = m.shapes[a].shape_type, tb = m.shapes[b].shape_type;
        if (ta == MR_SHAPE_CONVEX || tb == MR_SHAPE_CONVEX) return MR_COLLISION_PAIR_CONVEX;
        if (tb == MR_SHAPE_PLANE)
            return ta == MR_SHAPE_BOX ? MR_COLLISION_PAIR_BOX_PLANE
                   : (ta == MR_SHAPE_CAPSULE ? MR_COLLISION_PAIR_CAPSULE_PLANE
                   : (ta == MR_SHAPE_CYLINDER ? MR_COLLISION_PAIR_CYLINDER_PLANE : MR_COLLISION_PAIR_SPHERE_PLANE));
        if (ta == MR_SHAPE_CYLINDER || tb == MR_SHAPE_CYLINDER) return MR_COLLISION_PAIR_CONVEX;
        const bool sphere = ta == MR_SHAPE_SPHERE || tb == MR_SHAPE_SPHERE;
        const bool capsule = ta == MR_SHAPE_CAPSULE || tb == MR_SHAPE_CAPSULE;
        const bool box = ta == MR_SHAPE_BOX || tb == MR_SHAPE_BOX;
        if (ta == tb)
            return ta == MR_SHAPE_SPHERE ? MR_COLLISION_PAIR_SPHERE_SPHERE
                   : (ta == MR_SHAPE_BOX ? MR_COLLISION_PAIR_BOX_BOX : MR_COLLISION_PAIR_CAPSULE_CAPSULE);
        if (sphere && box) return MR_COLLISION_PAIR_SPHERE_BOX;
        if (sphere && capsule) return MR_COLLISION_PAIR_SPHERE_CAPSULE;
        return gjk_capsule_box ? MR_COLLISION_PAIR_CONVEX : MR_COLLISION_PAIR_CAPSULE_BOX;
    };
    // Compiled pairs in key order (a, b), b = n for the plane.
    for (std::uint32_t a = 0; a < n; ++a) {
        for (std::uint32_t b = a + 1; b < n; ++b) {
            MRModelPairC pr{a, b, static_cast<std::uint32_t>(cls(a, b)), 4u};
            m.pairs.push_back(pr);
        }
        MRModelPairC pr{a, n, static_cast<std::uint32_t>(cls(a, n)), 4u};
        m.pairs.push_back(pr);
    }
    m.world.body_count = n + 1;
    m.world.joint_count = 0;
    m.world.nq = 7 * n;
    m.world.nv = 6 * n;
    m.world.shape_count = n + 1;
    m.world.material_count = 2;
    m.world.pair_count = static_cast<std::uint32_t>(m.pairs.size());
    m.world.root_type = MR_ROOT_FIXED;
    m.world.actuation_mode = MR_ACTUATION_EFFORT;
    m.world.action_count = 0;
    m.world.contact_capacity = 256;
    m.world.apply_body_damping = 1u;
    set4(m.world.gravity, 0.0, 0.0, -9.81, 0.0);
    set4(m.world.solver_scales, 1.0e-7, 1.0e-9, 2.0, 1.0e-4);
    set4(m.world.manifold_thresholds, 0.02, 0.02, 0.002, 0.95);
    set4(m.world.speculative, 1.0, 1.0e4, 0.0, 0.0);
    m.nominal_q.assign(m.world.nq, 0.0f);
    m.friction_scale_lo = 1.0f;
    m.friction_scale_hi = 1.0f;
    m.finalize();
}


constexpr int kHullVertices = 12;  // vertices of each synthetic hull

CompiledModel build_pile(std::uint64_t seed, std::uint32_t count, bool cylinders, bool gjk_capsule_box, bool hulls) {
    CompiledModel m;
    m.name = hulls ? "synthetic_hull_pile"
                   : (cylinders ? "synthetic_cylinder_pile" : (gjk_capsule_box ? "synthetic_pile_gjk" : "synthetic_pile"));
    m.scene = true;
    std::uint64_t k = 0;
    auto draw = [&](double lo, double hi) { return uniform(seed, kStreamModel, k++, lo, hi); };
    const std::uint32_t n = count ? count : 8u + static_cast<std::uint32_t>(mix64(seed ^ 0x5ca1ab1eull) % 57u);
    if (n < 1 || n > 64) throw std::invalid_argument("pile body count must be in [1, 64]");
    m.scene_bodies = n;
    double largest = 0.0;
    for (std::uint32_t b = 0; b < n; ++b) {
        // One third each of boxes, spheres and capsules; with cylinders,
        // one quarter each of boxes, spheres, capsules and cylinders.
        const double kind = draw(0.0, 1.0);
        const bool quarters = cylinders || hulls;
        const bool box = quarters ? kind < 0.25 : kind < 1.0 / 3.0;
        const bool capsule = quarters ? (kind >= 0.5 && kind < 0.75) : kind >= 2.0 / 3.0;
        const bool cylinder = cylinders && kind >= 0.75;
        const bool hull = hulls && kind >= 0.75;
        const double size = draw(0.05, 0.3);
        const double density = draw(500.0, 2000.0);
        double hx = 0.5 * size, hy = 0.5 * size, hz = 0.5 * size;
        if (box) {
            hx *= draw(0.7, 1.0);
            hy *= draw(0.7, 1.0);
            hz *= draw(0.7, 1.0);
        }
        // Capsule: overall length `size` along local +Y, radius size x U(0.15, 0.3).
        const double cap_r = capsule ? size * draw(0.15, 0.3) : 0.0;
        const double cap_hl = capsule ? 0.5 * size - cap_r : 0.0;
        // Cylinder: radius and half length each 0.5 size x U(0.5, 1) (local +Y axis).
        const double cyl_r = cylinder ? 0.5 * size * draw(0.5, 1.0) : 0.0;
        const double cyl_hl = cylinder ? 0.5 * size * draw(0.5, 1.0) : 0.0;
        // Hull: 12 unit vertices -- seeded directions with radii U(0.75, 1)
        // -- scaled by per-axis half sizes 0.5 size x U(0.7, 1).
        std::uint32_t hull_first = 0;
        double hull_bound = 0.0;
        if (hull) {
            hx *= draw(0.7, 1.0);
            hy *= draw(0.7, 1.0);
            hz *= draw(0.7, 1.0);
            hull_first = static_cast<std::uint32_t>(m.hull_vertices.size() / 4);
            for (int i = 0; i < kHullVertices; ++i) {
                double d[3];
                double len = 0.0;
                do {
                    for (double& c : d) c = draw(-1.0, 1.0);
                    len = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
                } while (len < 0.2 || len > 1.0);
                const double r = draw(0.75, 1.0) / len;
                const double p[3] = {d[0] * r, d[1] * r, d[2] * r};
                for (double c : p) m.hull_vertices.push_back(static_cast<float>(c));
                m.hull_vertices.push_back(0.0f);
                hull_bound = std::max(hull_bound, std::sqrt(p[0] * p[0] * hx * hx + p[1] * p[1] * hy * hy + p[2] * p[2] * hz * hz));
            }
        }
        MRModelBodyC body{};
        body.parent_body = MR_INVALID_INDEX;
        body.inbound_joint = MR_INVALID_INDEX;
        body.motion_type = MR_MOTION_DYNAMIC;
        body.articulated = 0u;
        double mass, ixx, iyy, izz, bound;
        if (box) {
            mass = density * 8.0 * hx * hy * hz;
            ixx = mass / 3.0 * (hy * hy + hz * hz);
            iyy = mass / 3.0 * (hx * hx + hz * hz);
            izz = mass / 3.0 * (hx * hx + hy * hy);
            bound = std::sqrt(hx * hx + hy * hy + hz * hz);
        } else if (capsule) {
            // Cylinder of height 2 hl plus two hemispherical caps.
            const double pi = 3.141592653589793, r = cap_r, hgt = 2.0 * cap_hl;
            const double m_cyl = density * pi * r * r * hgt;
            const double m_cap = density * 2.0 / 3.0 * pi * r * r * r;  // one hemisphere
            mass = m_cyl + 2.0 * m_cap;
            iyy = 0.5 * m_cyl * r * r + 2.0 * m_cap * 0.4 * r * r;
            ixx = izz = m_cyl * (hgt * hgt / 12.0 + 0.25 * r * r) +
                        2.0 * m_cap * (0.4 * r * r + 0.25 * hgt * hgt + 0.375 * hgt * r);
            bound = cap_hl + r;
        } else if (cylinder) {
            const double r = cyl_r, hgt = 2.0 * cyl_hl;
            mass = density * 3.141592653589793 * r * r * hgt;
            iyy = 0.5 * mass * r * r;
            ixx = izz = mass * (3.0 * r * r + hgt * hgt) / 12.0;
            bound = std::sqrt(r * r + cyl_hl * cyl_hl);  // Collision.metal:5731-5734
        } else if (hull) {
            // Mass properties of the ellipsoid with semi-axes 0.875 x the
            // half sizes (the mean vertex radius), a stand-in for the hull's.
            const double a = 0.875 * hx, bb = 0.875 * hy, c = 0.875 * hz;
            mass = density * 4.0 / 3.0 * 3.141592653589793 * a * bb * c;
            ixx = 0.2 * mass * (bb * bb + c * c);
            iyy = 0.2 * mass * (a * a + c * c);
            izz = 0.2 * mass * (a * a + bb * bb);
            bound = hull_bound;
        } else {
            const double r = hx;
            mass = density * 4.0 / 3.0 * 3.141592653589793 * r * r * r;
            ixx = iyy = izz = 0.4 * mass * r * r;
            bound = r;
        }
        largest = std::max(largest, bound);
        set4(body.mass_inverse_mass, mass, 1.0 / mass, 0.0, 0.0);
        set4(body.inertia[0], ixx, 0.0, 0.0, 0.0);
        set4(body.inertia[1], 0.0, iyy, 0.0, 0.0);
        set4(body.inertia[2], 0.0, 0.0, izz, 0.0);
        set4(body.damping_speed, 0.0, 0.0, 100.0, 100.0);
        set4(body.static_pose, 0.0, 0.0, 0.0, 0.0);
        set4(body.static_pose + 4, 0.0, 0.0, 0.0, 1.0);
        m.bodies.push_back(body);
        MRModelShapeC s{};
        s.body = b;
        s.shape_type = box ? MR_SHAPE_BOX
                           : (capsule ? MR_SHAPE_CAPSULE
                                      : (cylinder ? MR_SHAPE_CYLINDER : (hull ? MR_SHAPE_CONVEX : MR_SHAPE_SPHERE)));
        if (hull) {
            s.hull_first = hull_first;
            s.hull_count = kHullVertices;
        }
        s.material = 0;
        s.collision_group = 1u;
        s.collision_mask = 3u;
        set4(s.local_position, 0.0, 0.0, 0.0, 0.0);
        set4(s.local_rotation, 0.0, 0.0, 0.0, 1.0);
        if (capsule) set4(s.dimensions, cap_r, cap_hl, 0.0, 0.0);
        else if (cylinder) set4(s.dimensions, cyl_r, cyl_hl, 0.0, 0.0);
        else set4(s.dimensions, hx, box || hull ? hy : 0.0, box || hull ? hz : 0.0, 0.0);
        set4(s.contact_rest_bound, 0.002, 0.0, bound, 0.0);
        m.shapes.push_back(s);
    }
    m.scene_cell = static_cast<float>(2.0 * largest + 0.05);
    if (gjk_capsule_box) m.scene_layout = CompiledModel::SceneLayout::heap;
    finish_scene(m, n, 0.6, gjk_capsule_box);
    return m;
}

CompiledModel build_stack(std::uint64_t seed, std::uint32_t boxes) {
    CompiledModel m;
    m.name = "synthetic_stack";
    m.scene = true;
    m.scene_layout = CompiledModel::SceneLayout::stack;
    m.stack_offset_sigma = 0.002f;
    (void)seed;  // every box is the same; the seed drives the reset layout
    if (boxes < 1 || boxes > 64) throw std::invalid_argument("stack box count must be in [1, 64]");
    m.scene_bodies = boxes;
    const double he = 0.05, mass = 1.0;
    const double inertia = mass / 3.0 * (2.0 * he * he);
    for (std::uint32_t b = 0; b < boxes; ++b) {
        MRModelBodyC body{};
        body.parent_body = MR_INVALID_INDEX;
        body.inbound_joint = MR_INVALID_INDEX;
        body.motion_type = MR_MOTION_DYNAMIC;
        body.articulated = 0u;
        set4(body.mass_inverse_mass, mass, 1.0 / mass, 0.0, 0.0);
        set4(body.inertia[0], inertia, 0.0, 0.0, 0.0);
        set4(body.inertia[1], 0.0, inertia, 0.0, 0.0);
        set4(body.inertia[2], 0.0, 0.0, inertia, 0.0);
        set4(body.damping_speed, 0.0, 0.0, 100.0, 100.0);
        set4(body.static_pose, 0.0, 0.0, 0.0, 0.0);
        set4(body.static_pose + 4, 0.0, 0.0, 0.0, 1.0);
        m.bodies.push_back(body);
        MRModelShapeC s{};
        s.body = b;
        s.shape_type = MR_SHAPE_BOX;
        s.material = 0;
        s.collision_group = 1u;
        s.collision_mask = 3u;
        set4(s.local_position, 0.0, 0.0, 0.0, 0.0);
        set4(s.local_rotation, 0.0, 0.0, 0.0, 1.0);
        set4(s.dimensions, he, he, he, 0.0);
        set4(s.contact_rest_bound, 0.002, 0.0, std::sqrt(3.0) * he, 0.0);
        m.shapes.push_back(s);
    }
    m.scene_cell = static_cast<float>(2.0 * he);  // stack pitch
    finish_scene(m, boxes, 0.6);
    return m;
}

void sample_reset_state(const CompiledModel& model, std::uint64_t seed, std::uint32_t env,
                        float* q, float* v, float* friction_scale) {
    const std::uint32_t nq = model.world.nq, nv = model.world.nv;
    if (model.scene && model.scene_layout == CompiledModel::SceneLayout::stack) {
        // Boxes resting on each other (box k's centre at (k + 1/2) pitch),
        // the stack yawed U(0, 2 pi) as a whole and each box offset
        // horizontally by N(0, sigma).
        const std::uint32_t n = model.scene_bodies;
        const std::uint64_t base = static_cast<std::uint64_t>(env) * 1024u;
        const double pitch = model.scene_cell;
        const double yaw = uniform(seed, kStreamResetRoot, base, 0.0, 6.283185307179586);
        for (std::uint32_t b = 0; b < n; ++b) {
            float* qb = q + 7 * b;
            qb[0] = static_cast<float>(model.stack_offset_sigma * normal(seed, kStreamResetQ, base + 8 * b));
            qb[1] = static_cast<float>(model.stack_offset_sigma * normal(seed, kStreamResetQ, base + 8 * b + 1));
            qb[2] = static_cast<float>((b + 0.5) * pitch);
            qb[3] = 0.0f;
            qb[4] = 0.0f;
            qb[5] = static_cast<float>(std::sin(0.5 * yaw));
            qb[6] = static_cast<float>(std::cos(0.5 * yaw));
        }
        for (std::uint32_t i = 0; i < nv; ++i) v[i] = 0.0f;
        *friction_scale = 1.0f;
        return;
    }
    if (model.scene) {
        // Bodies on a jittered square grid, dropped from U(0.1, 1) m above
        // the plane with a uniformly random orientation, at rest.  A heap
        // puts the grid in three layers one cell apart in height, each layer
        // shifted by half a cell: no two bodies overlap at the start, and
        // the upper layers fall onto the lower ones.
        const std::uint32_t n = model.scene_bodies;
        const bool heap = model.scene_layout == CompiledModel::SceneLayout::heap;
        const std::uint32_t per_layer = heap ? (n + 2) / 3 : n;
        const std::uint32_t side = static_cast<std::uint32_t>(std::ceil(std::sqrt(static_cast<double>(per_layer))));
        const std::uint64_t base = static_cast<std::uint64_t>(env) * 1024u;
        for (std::uint32_t b = 0; b < n; ++b) {
            const double cell = model.scene_cell;
            const std::uint32_t layer = b / per_layer, i = b % per_layer;
            const double shift = heap ? 0.5 * cell * static_cast<double>(layer % 2) : 0.0;
            const double x = (static_cast<double>(i % side) - 0.5 * (side - 1)) * cell + shift +
                             uniform(seed, kStreamResetQ, base + 8 * b, -0.02, 0.02);
            const double y = (static_cast<double>(i / side) - 0.5 * (side - 1)) * cell + shift +
                             uniform(seed, kStreamResetQ, base + 8 * b + 1, -0.02, 0.02);
            const double bound = model.shapes[b].contact_rest_bound[2];
            const double z = heap ? 0.5 * cell + layer * cell + uniform(seed, kStreamResetQ, base + 8 * b + 2, 0.0, 0.05)
                                  : bound + uniform(seed, kStreamResetQ, base + 8 * b + 2, 0.1, 1.0);
            // Uniform rotation (Shoemake): three uniforms -> unit quaternion.
            const double u1 = uniform01(seed, kStreamResetRoot, base + 8 * b);
            const double u2 = uniform01(seed, kStreamResetRoot, base + 8 * b + 1);
            const double u3 = uniform01(seed, kStreamResetRoot, base + 8 * b + 2);
            const double a = std::sqrt(1.0 - u1), c = std::sqrt(u1), tp = 6.283185307179586;
            float* qb = q + 7 * b;
            qb[0] = static_cast<float>(x);
            qb[1] = static_cast<float>(y);
            qb[2] = static_cast<float>(z);
            qb[3] = static_cast<float>(a * std::sin(tp * u2));
            qb[4] = static_cast<float>(a * std::cos(tp * u2));
            qb[5] = static_cast<float>(c * std::sin(tp * u3));
            qb[6] = static_cast<float>(c * std::cos(tp * u3));
        }
        for (std::uint32_t i = 0; i < nv; ++i) v[i] = 0.0f;
        *friction_scale = static_cast<float>(
            uniform(seed, kStreamFriction, env, model.friction_scale_lo, model.friction_scale_hi));
        return;
    }
    for (std::uint32_t i = 0; i < nq; ++i) q[i] = model.nominal_q[i];
    for (std::uint32_t i = 0; i < nv; ++i) v[i] = 0.0f;
    const std::uint64_t base = static_cast<std::uint64_t>(env) * 64u;
    const std::uint32_t root_q = model.world.root_type == MR_ROOT_FLOATING ? 7u : 0u;
    const std::uint32_t root_v = model.world.root_type == MR_ROOT_FLOATING ? 6u : 0u;
    for (std::uint32_t i = root_q; i < nq; ++i) {
        const double r = model.q_joint_uniform_half_range;
        q[i] = static_cast<float>(q[i] + uniform(seed, kStreamResetQ, base + i, -r, r));
    }
    if (model.qd_joint_normal_sigma > 0.0f) {
        for (std::uint32_t i = root_v; i < nv; ++i)
            v[i] = static_cast<float>(model.qd_joint_normal_sigma * normal(seed, kStreamResetV, base + i));
    }
    if (model.world.root_type == MR_ROOT_FLOATING && model.root_yaw_half_range > 0.0f) {
        const double r = model.root_yaw_half_range;
        const double yaw = uniform(seed, kStreamResetRoot, env, -r, r);
        q[3] = 0.0f;
        q[4] = 0.0f;
        q[5] = static_cast<float>(std::sin(0.5 * yaw));
        q[6] = static_cast<float>(std::cos(0.5 * yaw));
    }
    *friction_scale = static_cast<float>(
        uniform(seed, kStreamFriction, env, model.friction_scale_lo, model.friction_scale_hi));
}

}  // namespace numi
