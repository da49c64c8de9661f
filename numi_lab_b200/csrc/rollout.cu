// Host runtime behind the task-rollout C ABI (include/numi_b200.h).
//
// Mirrors numi-lab's mr_* rollout boundary (src/c_api.cpp:3370-3990):
// validation with exceptions translated into a thread-local last-error
// string, handle-owned results that alias until the next advance / reset /
// destroy, synchronous host advance.  Underneath, a rollout owns its
// compiled model, the device-resident state of every environment and a
// cache of CUDA graphs, one per horizon length, each holding the horizon's
// control-step launches (no contact-count readback inside a horizon).
#include "device_model.h"
#include "layout.h"
#include "audit.cuh"
#include "mix.h"
#include "model.h"
#include "numi_b200.h"
#include "packs.h"
#include "policy.h"
#include "quality.cuh"
#include "runtime.h"
#include "scene.h"
#include "task.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <chrono>
#include <cmath>
#include <cstring>
#include <limits>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace {

using numi::rt::check;
using numi::rt::DeviceBuffer;
using numi::rt::PinnedBuffer;
using numi::rt::guarded;

thread_local std::string g_last_error;

}  // namespace

void numi::rt::set_last_error(const std::string& message) { g_last_error = message; }
const char* numi::rt::last_error() { return g_last_error.c_str(); }

numi::DeviceModel numi::rt::pack_model(const numi::CompiledModel& m, float h) {
    using namespace numi;
    DeviceModel d{};
    std::memset(&d, 0, sizeof(d));
    const MRModelWorldC& w = m.world;
    d.nb = static_cast<int>(m.articulated_body_count);
    d.nv = static_cast<int>(w.nv);
    d.nq = static_cast<int>(w.nq);
    d.floating = w.root_type == MR_ROOT_FLOATING ? 1 : 0;
    d.n_levels = static_cast<int>(m.level_count);
    d.action_count = static_cast<int>(w.action_count);
    d.implicit_drives = w.actuation_mode == MR_ACTUATION_IMPLICIT_POSITION ? 1 : 0;
    d.apply_damping = w.apply_body_damping ? 1 : 0;
    d.ns = static_cast<int>(w.shape_count);
    d.np = static_cast<int>(w.pair_count);
    d.contact_capacity = static_cast<int>(w.contact_capacity);
    d.max_anc = static_cast<int>(m.max_ancestor_dofs);
    for (int i = 0; i < 3; ++i) d.gravity[i] = w.gravity[i];
    d.h = h;
    d.slop = w.solver_scales[3];
    d.max_depenetration = w.solver_scales[2];
    d.speculative_scale = w.speculative[0];
    d.speed_envelope = w.speculative[1];
    for (int i = 0; i < 4; ++i) d.manifold_thresholds[i] = w.manifold_thresholds[i];
    for (std::uint32_t l = 0; l <= m.level_count; ++l) d.level_offsets[l] = static_cast<int>(m.level_offsets[l]);
    for (size_t i = 0; i < m.level_bodies.size(); ++i) d.level_bodies[i] = static_cast<int>(m.level_bodies[i]);
    const int nb = d.nb;
    // children lists in body order
    std::vector<std::vector<int>> kids(nb);
    for (int b = 1; b < nb; ++b) kids[m.bodies[b].parent_body].push_back(b);
    int co = 0;
    for (int b = 0; b < nb; ++b) {
        d.child_offsets[b] = co;
        for (int c : kids[b]) d.children[co++] = c;
    }
    d.child_offsets[nb] = co;
    auto norm4 = [](const float* q) {
        const double n = std::sqrt(double(q[0]) * q[0] + double(q[1]) * q[1] + double(q[2]) * q[2] + double(q[3]) * q[3]);
        return make_float4(float(q[0] / n), float(q[1] / n), float(q[2] / n), float(q[3] / n));
    };
    for (int b = 0; b < nb; ++b) {
        const MRModelBodyC& body = m.bodies[b];
        d.parent[b] = b == 0 ? -1 : static_cast<int>(body.parent_body);
        d.subtree_end[b] = static_cast<int>(m.subtree_end[b]);
        d.body_dof[b] = m.body_dof[b] == MR_INVALID_INDEX ? -1 : static_cast<int>(m.body_dof[b]);
        d.mass_damping[b] = make_float4(body.mass_inverse_mass[0], body.damping_speed[0], body.damping_speed[1], 0.0f);
        d.inertia_diag[b] = make_float4(body.inertia[0][0], body.inertia[1][1], body.inertia[2][2], 0.0f);
        d.inertia_off[b] = make_float4(body.inertia[0][1], body.inertia[0][2], body.inertia[1][2], 0.0f);
        d.anc_count[b] = static_cast<int>(m.body_ancestor_count[b]);
        for (std::uint32_t k = 0; k < m.max_ancestor_dofs; ++k)
            d.anc_dofs[b * kMaxDofs + k] = static_cast<int>(m.body_ancestor_dofs[b * m.max_ancestor_dofs + k]);
        if (b > 0) {
            const MRModelJointC& j = m.joints[body.inbound_joint];
            d.joint_type[b] = static_cast<int>(j.joint_type);
            const double an = std::sqrt(double(j.axis[0]) * j.axis[0] + double(j.axis[1]) * j.axis[1] + double(j.axis[2]) * j.axis[2]);
            d.axis[b] = make_float4(float(j.axis[0] / an), float(j.axis[1] / an), float(j.axis[2] / an), 0.0f);
            d.parent_anchor[b] = make_float4(j.parent_anchor[0], j.parent_anchor[1], j.parent_anchor[2], 0.0f);
            d.child_anchor[b] = make_float4(j.child_anchor[0], j.child_anchor[1], j.child_anchor[2], 0.0f);
            d.parent_rotation[b] = norm4(j.parent_rotation);
            const float4 cr = norm4(j.child_rotation);
            d.child_rotation_conj[b] = make_float4(-cr.x, -cr.y, -cr.z, cr.w);
        } else {
            d.joint_type[b] = MR_JOINT_FIXED;
            d.parent_rotation[b] = make_float4(0, 0, 0, 1);
            d.child_rotation_conj[b] = make_float4(0, 0, 0, 1);
        }
    }
    for (std::uint32_t k = 0; k < w.nv; ++k) {
        const MRModelDofC& dof = m.dofs[k];
        d.dof_body[k] = static_cast<int>(m.dof_body[k]);
        d.dof_parent[k] = m.dof_parent[k] == MR_INVALID_INDEX ? -1 : static_cast<int>(m.dof_parent[k]);
        // position of k in its body's ancestor list = number of ancestors
        const std::uint32_t b = m.dof_body[k];
        int count = 0;
        for (std::uint32_t t = 0; t < m.body_ancestor_count[b]; ++t) {
            if (m.body_ancestor_dofs[b * m.max_ancestor_dofs + t] == k) { count = static_cast<int>(t); break; }
        }
        d.dof_anc_count[k] = count;
        d.dof_q[k] = dof.q_index == MR_INVALID_INDEX ? -1 : static_cast<int>(dof.q_index);
        d.dof_flags[k] = dof.flags;
        float arm = dof.drive[2];
        if (d.implicit_drives && (dof.flags & MR_DOF_FLAG_DRIVE)) arm += h * dof.drive[1] + h * h * dof.drive[0];
        d.armature_eff[k] = arm;
        d.kp[k] = dof.drive[0];
        d.kd[k] = dof.drive[1];
        d.dry_friction[k] = dof.drive[3];
        const float stall = ((dof.flags & MR_DOF_FLAG_EFFORT_LIMIT) && dof.limits[3] > 0.0f)
                                ? dof.limits[3] : std::numeric_limits<float>::max();
        d.effort_envelope[k] = std::min(dof.limits[3], stall);
        d.effort_limit[k] = dof.limits[3];
        d.q_lower[k] = dof.limits[0];
        d.q_upper[k] = dof.limits[1];
        d.v_max[k] = dof.limits[2];
    }
    // Actions drive the actuated DoFs in v order.
    int a = 0;
    for (std::uint32_t k = 0; k < w.nv && a < d.action_count; ++k)
        if (m.dofs[k].flags & MR_DOF_FLAG_ACTUATED) d.action_dof[a++] = static_cast<int>(k);
    if (a != d.action_count) throw std::runtime_error("action count does not match actuated DoFs");
    for (std::uint32_t s = 0; s < w.shape_count; ++s) {
        const MRModelShapeC& sh = m.shapes[s];
        const MRModelBodyC& body = m.bodies[sh.body];
        d.shape_type[s] = static_cast<int>(sh.shape_type);
        d.shape_material[s] = static_cast<int>(sh.material);
        d.shape_dims[s] = make_float4(sh.dimensions[0], sh.dimensions[1], sh.dimensions[2], 0.0f);
        float sweep = sh.contact_rest_bound[2];
        if (!(sweep > 0.0f) || !std::isfinite(sweep)) {
            if (sh.shape_type == MR_SHAPE_SPHERE) sweep = sh.dimensions[0];
            else if (sh.shape_type == MR_SHAPE_CAPSULE) sweep = sh.dimensions[0] + sh.dimensions[1];
            else sweep = std::sqrt(sh.dimensions[0] * sh.dimensions[0] + sh.dimensions[1] * sh.dimensions[1] + sh.dimensions[2] * sh.dimensions[2]);
        }
        d.shape_offsets[s] = make_float4(sh.contact_rest_bound[0], sh.contact_rest_bound[1], sweep, 0.0f);
        const float4 lr = norm4(sh.local_rotation);
        if (body.articulated) {
            d.shape_body[s] = static_cast<int>(sh.body);
            d.shape_position[s] = make_float4(sh.local_position[0], sh.local_position[1], sh.local_position[2], 0.0f);
            d.shape_rotation[s] = lr;
        } else {
            // World pose of a static shape (reference: body pose composed with local pose).
            d.shape_body[s] = -1;
            const float4 br = norm4(body.static_pose + 4);
            const double bx = br.x, by = br.y, bz = br.z, bw = br.w;
            const double lx = sh.local_position[0], ly = sh.local_position[1], lz = sh.local_position[2];
            // rotate local position by body rotation
            const double tx = 2 * (by * lz - bz * ly), ty = 2 * (bz * lx - bx * lz), tz = 2 * (bx * ly - by * lx);
            const double rx = lx + bw * tx + (by * tz - bz * ty);
            const double ry = ly + bw * ty + (bz * tx - bx * tz);
            const double rz = lz + bw * tz + (bx * ty - by * tx);
            d.shape_position[s] = make_float4(float(body.static_pose[0] + rx), float(body.static_pose[1] + ry),
                                              float(body.static_pose[2] + rz), 0.0f);
            const float4 q = make_float4(
                float(bw * lr.x + bx * lr.w + by * lr.z - bz * lr.y), float(bw * lr.y - bx * lr.z + by * lr.w + bz * lr.x),
                float(bw * lr.z + bx * lr.y - by * lr.x + bz * lr.w), float(bw * lr.w - bx * lr.x - by * lr.y - bz * lr.z));
            d.shape_rotation[s] = q;
            d.static_body_position[s] = make_float4(body.static_pose[0], body.static_pose[1], body.static_pose[2], 0.0f);
            d.static_body_rotation[s] = br;
        }
    }
    for (std::uint32_t p = 0; p < w.pair_count; ++p) {
        const MRModelPairC& pr = m.pairs[p];
        const bool a_art = m.bodies[m.shapes[pr.shape_a].body].articulated != 0;
        const bool b_art = m.bodies[m.shapes[pr.shape_b].body].articulated != 0;
        if (a_art == b_art) throw std::runtime_error("pairs must join one articulated and one static collider");
        if (pr.pair_class != MR_COLLISION_PAIR_SPHERE_PLANE && pr.pair_class != MR_COLLISION_PAIR_BOX_PLANE &&
            pr.pair_class != MR_COLLISION_PAIR_CAPSULE_PLANE)
            throw std::runtime_error("unsupported collision pair class");
        d.pair_a[p] = static_cast<int>(pr.shape_a);
        d.pair_b[p] = static_cast<int>(pr.shape_b);
        d.pair_class[p] = static_cast<int>(pr.pair_class);
        d.pair_max_points[p] = static_cast<int>(pr.max_points);
    }
    // Byte tables for the kernels' shared-memory copy.
    {
        DeviceTables& t = d.tables;
        std::memset(&t, 0xff, sizeof(t));
        t.nb = static_cast<std::uint8_t>(nb);
        t.nv = static_cast<std::uint8_t>(w.nv);
        t.nq = static_cast<std::uint8_t>(w.nq);
        t.n_levels = static_cast<std::uint8_t>(m.level_count);
        t.floating = static_cast<std::uint8_t>(d.floating);
        t.ns = static_cast<std::uint8_t>(w.shape_count);
        t.np = static_cast<std::uint8_t>(w.pair_count);
        t.max_anc = static_cast<std::uint8_t>(m.max_ancestor_dofs);
        std::vector<int> depth(nb, 0);
        for (int b = 1; b < nb; ++b) depth[b] = depth[m.bodies[b].parent_body] + 1;
        for (int b = 0; b < nb; ++b) {
            t.depth[b] = static_cast<std::uint8_t>(depth[b]);
            t.parent[b] = b == 0 ? 255 : static_cast<std::uint8_t>(m.bodies[b].parent_body);
            t.body_dof[b] = m.body_dof[b] == MR_INVALID_INDEX ? 255 : static_cast<std::uint8_t>(m.body_dof[b]);
            t.child_offsets[b] = static_cast<std::uint8_t>(d.child_offsets[b]);
            t.children[b] = static_cast<std::uint8_t>(d.children[b]);
            t.anc_count[b] = static_cast<std::uint8_t>(m.body_ancestor_count[b]);
            for (std::uint32_t k = 0; k < m.body_ancestor_count[b]; ++k)
                t.anc[b][k] = static_cast<std::uint8_t>(m.body_ancestor_dofs[b * m.max_ancestor_dofs + k]);
            for (std::uint32_t dof = 0; dof < w.nv; ++dof) {
                t.pos[b][dof] = 255;
                for (std::uint32_t k = 0; k < m.body_ancestor_count[b]; ++k)
                    if (m.body_ancestor_dofs[b * m.max_ancestor_dofs + k] == dof) t.pos[b][dof] = static_cast<std::uint8_t>(k);
            }
        }
        t.child_offsets[nb] = static_cast<std::uint8_t>(d.child_offsets[nb]);
        std::memset(t.level_children, 0, sizeof(t.level_children));
        for (int b = 0; b < nb; ++b) {
            const int children = d.child_offsets[b + 1] - d.child_offsets[b];
            t.level_children[depth[b]] = static_cast<std::uint8_t>(std::max<int>(t.level_children[depth[b]], children));
        }
        for (int a = 0; a < nb; ++a)
            for (int b = 0; b < nb; ++b) {
                std::uint32_t n = 0;
                while (n < m.body_ancestor_count[a] && n < m.body_ancestor_count[b] &&
                       m.body_ancestor_dofs[a * m.max_ancestor_dofs + n] == m.body_ancestor_dofs[b * m.max_ancestor_dofs + n])
                    ++n;
                t.lcp[a][b] = static_cast<std::uint8_t>(n);
            }
        int levels = 0;
        for (std::uint32_t k = 0; k < w.nv; ++k) {
            t.dof_body[k] = static_cast<std::uint8_t>(m.dof_body[k]);
            t.dof_parent[k] = m.dof_parent[k] == MR_INVALID_INDEX ? 255 : static_cast<std::uint8_t>(m.dof_parent[k]);
            t.dof_depth[k] = static_cast<std::uint8_t>(d.dof_anc_count[k]);
            levels = std::max(levels, d.dof_anc_count[k] + 1);
        }
        t.n_dof_levels = static_cast<std::uint8_t>(levels);
    }
    if (w.material_count > kMaxMaterials) throw std::runtime_error("too many materials");
    for (std::uint32_t i = 0; i < w.material_count; ++i) {
        const MRModelMaterialC& mt = m.materials[i];
        d.material_friction[i] = make_float4(mt.friction[0], mt.friction[1], mt.friction[2], mt.friction[3]);
        d.material_response[i] = make_float4(mt.response[0], mt.response[1], mt.response[2], mt.response[3]);
    }
    return d;
}

void numi::rt::make_plan(const numi::CompiledModel& m, float h, KernelPlan& plan) {
    plan.contact = m.world.pair_count > 0;
    plan.dmodel = pack_model(m, h);
    int narrow_words = 0;
    for (const MRModelPairC& pr : m.pairs) narrow_words += numi::pair_scratch_words(numi::pair_max_raw(static_cast<int>(pr.pair_class)));
    const int nv = static_cast<int>(m.world.nv), ncap = static_cast<int>(m.world.contact_capacity);
    const int solvers = plan.contact ? kSolverModes : 1;
    for (int quality = 0; quality < solvers; ++quality)
        for (const bool compensated : {false, true})
            (compensated ? plan.layout_comp : plan.layout)[quality] =
                numi::make_layout(static_cast<int>(m.articulated_body_count), nv, static_cast<int>(m.world.nq),
                                  static_cast<int>(m.world.pair_count), ncap, static_cast<int>(m.max_ancestor_dofs), narrow_words,
                                  plan.contact, compensated, quality ? numi::quality_workspace_doubles(nv, ncap) : 0);
    int device = 0;
    check(cudaGetDevice(&device), "cudaGetDevice");
    cudaDeviceProp prop{};
    check(cudaGetDeviceProperties(&prop, device), "cudaGetDeviceProperties");
    const size_t tables = numi::control_step_table_bytes();
    const size_t limit = prop.sharedMemPerBlockOptin;
    if (tables + static_cast<size_t>(plan.layout[0].total) * sizeof(float) > limit)
        throw std::runtime_error("per-environment shared memory exceeds the device limit");
    check(numi::configure_control_step_kernels(limit), "kernel attributes");
    // Environments per CTA: the choice that keeps the most warps resident
    // per SM under the kernel's register and shared-memory footprint (each
    // CTA carries one copy of the topology tables).
    for (int quality = 0; quality < solvers; ++quality)
        for (std::uint32_t prec = 0; prec < static_cast<std::uint32_t>(numi::rt::kPrecisionModes); ++prec) {
            const size_t per_warp = static_cast<size_t>(plan.layout_for(prec, quality != 0).total) * sizeof(float);
            int best = 1, best_warps = 0;
            // NUMI_B200_STEP_WARPS_PER_BLOCK fixes the CTA size (clamped to
            // what the instance is built for) instead of the search.
            const int max_wpb = numi::control_step_max_warps_per_block(prec, quality != 0);
            int lo = 1, hi = max_wpb;
            if (const char* env = std::getenv("NUMI_B200_STEP_WARPS_PER_BLOCK")) lo = hi = std::max(1, std::min(max_wpb, std::atoi(env)));
            for (int wpb = lo; wpb <= hi; ++wpb) {
                const size_t smem = tables + wpb * per_warp;
                if (smem > limit) break;
                int blocks = 0;
                check(numi::control_step_occupancy(plan.contact, prec, quality != 0, wpb, smem, &blocks), "occupancy query");
                if (blocks * wpb > best_warps) { best_warps = blocks * wpb; best = wpb; }
            }
            if (best_warps == 0) {
                if (quality) continue;  // the quality solver stays unavailable for this model
                throw std::runtime_error("the control-step kernel cannot be resident with this model");
            }
            plan.warps_per_block[quality][prec] = best;
            plan.resident_warps_per_sm[quality][prec] = best_warps;
        }
}

numi::SceneModel numi::rt::pack_scene(const numi::CompiledModel& m, float h) {
    numi::SceneModel d{};
    const std::uint32_t n = m.scene_bodies;
    if (m.pairs.size() > static_cast<size_t>(numi::kSceneMaxPairs)) throw std::runtime_error("scene pair count outside capacity");
    if (m.materials.size() > static_cast<size_t>(numi::kSceneMaxMaterials)) throw std::runtime_error("too many scene materials");
    d.nb = static_cast<int>(n);
    d.np = static_cast<int>(m.pairs.size());
    d.h = h;
    d.slop = m.world.solver_scales[3];
    for (int i = 0; i < 3; ++i) d.gravity[i] = m.world.gravity[i];
    d.max_depenetration = m.world.solver_scales[2];
    d.speculative_scale = m.world.speculative[0];
    d.speed_envelope = m.world.speculative[1];
    for (int i = 0; i < 4; ++i) d.thresholds[i] = m.world.manifold_thresholds[i];
    const MRModelShapeC& plane = m.shapes[n];
    const MRModelBodyC& ground = m.bodies[n];
    d.plane_position = make_float4(ground.static_pose[0] + plane.local_position[0], ground.static_pose[1] + plane.local_position[1],
                                   ground.static_pose[2] + plane.local_position[2], 0.0f);
    {
        const double qw[4] = {plane.local_rotation[0], plane.local_rotation[1], plane.local_rotation[2], plane.local_rotation[3]};
        const double nrm = std::sqrt(qw[0] * qw[0] + qw[1] * qw[1] + qw[2] * qw[2] + qw[3] * qw[3]);
        d.plane_rotation = make_float4(static_cast<float>(qw[0] / nrm), static_cast<float>(qw[1] / nrm), static_cast<float>(qw[2] / nrm),
                                       static_cast<float>(qw[3] / nrm));
    }
    d.plane_offsets = make_float4(plane.contact_rest_bound[0], plane.contact_rest_bound[1], 0.0f, 0.0f);
    d.ground_position = make_float4(ground.static_pose[0], ground.static_pose[1], ground.static_pose[2], 0.0f);
    {
        const double qw[4] = {ground.static_pose[4], ground.static_pose[5], ground.static_pose[6], ground.static_pose[7]};
        const double nrm = std::sqrt(qw[0] * qw[0] + qw[1] * qw[1] + qw[2] * qw[2] + qw[3] * qw[3]);
        d.ground_rotation = make_float4(static_cast<float>(qw[0] / nrm), static_cast<float>(qw[1] / nrm), static_cast<float>(qw[2] / nrm),
                                        static_cast<float>(qw[3] / nrm));
    }
    d.plane_material = static_cast<int>(plane.material);
    d.support_mapped = 0;
    for (const MRModelPairC& pr : m.pairs)
        if (pr.pair_class == MR_COLLISION_PAIR_CONVEX) d.support_mapped = 1;
    for (std::uint32_t b = 0; b < n; ++b) {
        const MRModelShapeC& sh = m.shapes[b];
        const MRModelBodyC& body = m.bodies[b];
        d.shape_type[b] = static_cast<int>(sh.shape_type);
        d.material[b] = static_cast<int>(sh.material);
        d.dims[b] = make_float4(sh.dimensions[0], sh.dimensions[1], sh.dimensions[2], 0.0f);
        const float damp_lin = m.world.apply_body_damping ? body.damping_speed[0] : 0.0f;
        const float damp_ang = m.world.apply_body_damping ? body.damping_speed[1] : 0.0f;
        d.mass[b] = make_float4(body.mass_inverse_mass[0], body.mass_inverse_mass[1], damp_lin, damp_ang);
        d.inv_inertia[b] = make_float4(1.0f / body.inertia[0][0], 1.0f / body.inertia[1][1], 1.0f / body.inertia[2][2],
                                       body.damping_speed[2]);
        d.offsets[b] = make_float4(sh.contact_rest_bound[0], sh.contact_rest_bound[1], sh.contact_rest_bound[2], body.damping_speed[3]);
    }
    for (std::size_t i = 0; i < m.materials.size(); ++i) {
        const MRModelMaterialC& mt = m.materials[i];
        d.material_friction[i] = make_float4(mt.friction[0], mt.friction[1], mt.friction[2], mt.friction[3]);
        d.material_response[i] = make_float4(mt.response[0], mt.response[1], mt.response[2], mt.response[3]);
    }
    for (std::size_t p = 0; p < m.pairs.size(); ++p) {
        d.pair_a[p] = static_cast<std::uint8_t>(m.pairs[p].shape_a);
        d.pair_b[p] = static_cast<std::uint8_t>(m.pairs[p].shape_b);
        d.pair_class[p] = static_cast<std::uint8_t>(m.pairs[p].pair_class);
    }
    int used = 0;
    for (std::uint32_t b = 0; b < n; ++b) {
        const MRModelShapeC& sh = m.shapes[b];
        if (sh.shape_type != MR_SHAPE_CONVEX) continue;
        if (sh.hull_count == 0 || used + static_cast<int>(sh.hull_count) > numi::kSceneMaxHullVertices ||
            (static_cast<size_t>(sh.hull_first) + sh.hull_count) * 4 > m.hull_vertices.size())
            throw std::runtime_error("convex hull vertices outside the scene capacity");
        d.hull_first[b] = used;
        d.hull_count[b] = static_cast<int>(sh.hull_count);
        for (std::uint32_t i = 0; i < sh.hull_count; ++i) {
            const float* v = m.hull_vertices.data() + (static_cast<size_t>(sh.hull_first) + i) * 4;
            d.hull_vertices[used++] = make_float4(v[0] * sh.dimensions[0], v[1] * sh.dimensions[1], v[2] * sh.dimensions[2], 0.0f);
        }
    }
    return d;
}

// A policy installed on a rollout (mr_task_rollout_set_policy): every span
// copied into one device arena, the launch parameters pointing into it.
struct InstalledPolicy {
    std::uint64_t revision = 0;
    std::uint64_t fingerprint = 0;  // FNV-1a 64 of the policy's PolicyPack payload (version 4 encoding)
    std::string id;
    DeviceBuffer<float> arena;
    numi::PolicyParams params{};  // arena pointers; state and output pointers are set per launch
    bool has_critic = false;
};

// A task program installed on a rollout (mr_task_rollout_set_task): its
// tables in one device arena, the launch constants pointing into it.
struct InstalledTask {
    DeviceBuffer<unsigned char> arena;
    numi::TaskProgramDevice prog{};
    std::uint64_t fingerprint = 0;
};

struct MRTaskRolloutHandle {
    numi::CompiledModel model;
    numi::DeviceModel dmodel{};
    numi::WarpLayout layout{};
    numi::WarpLayout layout_comp{};     // with the q compensation section
    // Converged contact solve (MR_SOLVER_QUALITY_NEWTON) in place of the
    // temporalCone sweeps: its kernel instances, layouts (with the solver
    // workspace) and launch shapes.
    bool quality = false;
    numi::QualityConfig quality_cfg{};
    numi::WarpLayout layout_q{};
    numi::WarpLayout layout_q_comp{};
    int warps_per_block_q[numi::rt::kPrecisionModes] = {1, 1, 1};
    int resident_warps_per_sm_q[numi::rt::kPrecisionModes] = {0, 0, 0};
    MRQualityDiagnosticsC last_quality{};  // of the last advance (zeros under temporalCone)
    bool contact = false;
    bool scene = false;                 // free-body pile world (scene_step kernel)
    numi::SceneModel smodel{};
    DeviceBuffer<numi::SceneModel> d_smodel;
    DeviceBuffer<std::uint32_t> d_mcount;
    DeviceBuffer<float> d_workspace;    // scene substep tables, contacts, narrowphase scratch
    // Scene worlds: island index per body on each control step's final
    // substep ([env][kSceneMaxBodies]), written while enabled.
    DeviceBuffer<std::uint8_t> d_island_labels;
    bool island_labels = false;
    // FP64 energy / momentum audit records ([env][kAuditWords]) while enabled.
    DeviceBuffer<double> d_audit;
    bool audit = false;
    std::uint32_t precision = MR_PRECISION_FP32;  // MRPrecisionModeC
    int warps_per_block[numi::rt::kPrecisionModes] = {1, 1, 1};  // per precision mode
    int resident_warps_per_sm[numi::rt::kPrecisionModes] = {0, 0, 0};
    MRTaskRolloutConfigC config{};
    std::uint32_t envs = 0;
    float h = 0.0f;
    std::uint64_t seed = 0;
    bool readback = false;
    int device = 0;
    std::string device_name;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev_start = nullptr, ev_stop = nullptr;
    cudaEvent_t ev_in = nullptr, ev_out = nullptr;  // caller-stream handoff
    // Observation read-back of the host-buffer advance: each control step's
    // slice is copied on copy_stream while the next step computes.
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t ev_step = nullptr, ev_copies = nullptr;
    // Environment chains: an articulated advance runs its environments as
    // `chains` contiguous blocks, each a chain of per-step launches on its
    // own stream inside the captured graph, so one chain's partial last wave
    // overlaps the others' launches (environments are independent).
    static constexpr int kMaxChains = 4;
    int chains = 1;
    cudaStream_t chain_stream[kMaxChains] = {};
    cudaEvent_t ev_fork = nullptr, ev_chain[kMaxChains] = {};
    // Chain c > 0 reads its observations back on its own copy stream (chain 0
    // uses copy_stream), so no chain's copies queue behind another chain's.
    cudaStream_t chain_copy_stream[kMaxChains] = {};
    cudaEvent_t ev_chain_copies[kMaxChains] = {};

    DeviceBuffer<numi::DeviceModel> d_model;
    DeviceBuffer<float> d_q, d_v, d_manifolds, d_reset_q, d_reset_v, d_friction;
    DeviceBuffer<float> d_qcomp;        // [env][nq] compensation of q's running sums (compensated precision)
    // Native policy: outputs of the last policy-driven advance and the
    // control-step counter that keys its draws.
    std::unique_ptr<InstalledPolicy> policy;
    DeviceBuffer<float> d_latents, d_log_prob, d_values;
    PinnedBuffer<float> h_latents, h_log_prob, h_values;
    DeviceBuffer<unsigned long long> d_policy_steps;
    bool have_policy_outputs = false;
    std::uint32_t last_policy_steps = 0;
    // Task layer: the installed program, per-environment task records, the
    // drive targets of the step in flight, the steps' reset masks and
    // transitions ([step][env]) of the last advance.
    std::unique_ptr<InstalledTask> task;
    DeviceBuffer<numi::TaskEnvState> d_task_state;
    DeviceBuffer<float> d_task_history, d_task_previous, d_task_frame, d_task_critic, d_task_targets, d_task_air;
    DeviceBuffer<std::uint32_t> d_task_masks;
    DeviceBuffer<MRTaskTransitionC> d_transitions;
    PinnedBuffer<MRTaskTransitionC> h_transitions;
    std::uint32_t transition_steps = 0;   // steps of d_transitions written by the last advance
    bool have_host_transitions = false;
    DeviceBuffer<float> d_actions, d_obs;
    DeviceBuffer<std::uint32_t> d_masks, d_status, d_contacts, d_stats;
    PinnedBuffer<float> h_obs, h_final_q;
    PinnedBuffer<std::uint32_t> h_status, h_contacts, h_stats;
    std::vector<float> reset_q, reset_v, friction;

    // graph cache keyed by (steps, has masks, obs/status targets)
    struct GraphKey {
        std::uint32_t steps;
        const void* actions;
        const void* masks;
        const void* obs;
        const void* status;
        const void* contacts;
        std::uint32_t precision;
        const void* host_obs;
        const void* policy;  // installed policy's arena, or null
        bool evaluate_final;
        const void* latents;  // policy outputs (reallocated when an advance needs more room)
        const void* log_prob;
        const void* values;
        const void* task;         // installed task's arena, or null
        const void* task_masks;   // task-layer buffers (reallocated when an advance needs more room)
        const void* transitions;
        bool operator<(const GraphKey& o) const {
            return std::tie(steps, actions, masks, obs, status, contacts, precision, host_obs, policy, evaluate_final, latents,
                            log_prob, values, task, task_masks, transitions) <
                   std::tie(o.steps, o.actions, o.masks, o.obs, o.status, o.contacts, o.precision, o.host_obs, o.policy,
                            o.evaluate_final, o.latents, o.log_prob, o.values, o.task, o.task_masks, o.transitions);
        }
    };
    std::map<GraphKey, cudaGraphExec_t> graphs;

    // Last-advance publication.
    std::uint32_t last_steps = 0;
    bool have_final_q = false;
    MRTaskRolloutLayoutC stats_layout{};

    ~MRTaskRolloutHandle() {
        for (auto& kv : graphs) cudaGraphExecDestroy(kv.second);
        if (ev_start) cudaEventDestroy(ev_start);
        if (ev_stop) cudaEventDestroy(ev_stop);
        if (ev_in) cudaEventDestroy(ev_in);
        if (ev_out) cudaEventDestroy(ev_out);
        for (int c = 0; c < kMaxChains; ++c) {
            if (ev_chain[c]) cudaEventDestroy(ev_chain[c]);
            if (chain_stream[c]) cudaStreamDestroy(chain_stream[c]);
            if (ev_chain_copies[c]) cudaEventDestroy(ev_chain_copies[c]);
            if (chain_copy_stream[c]) cudaStreamDestroy(chain_copy_stream[c]);
        }
        if (ev_fork) cudaEventDestroy(ev_fork);
        if (ev_step) cudaEventDestroy(ev_step);
        if (ev_copies) cudaEventDestroy(ev_copies);
        if (copy_stream) cudaStreamDestroy(copy_stream);
        if (stream) cudaStreamDestroy(stream);
    }

    // This world's work at control step k of a heterogeneous batch: the
    // parameters its own kernel would get (FP32, all environments, items
    // indexed by slot).  actions [steps][env][action], masks [steps][env]
    // and status [steps][env] are device buffers or null.
    numi::MixWorld mix_world(std::uint32_t k, const float* actions, const std::uint32_t* masks, std::uint32_t* status) const {
        numi::MixWorld w{};
        w.envs = static_cast<std::int32_t>(envs);
        const size_t item0 = static_cast<size_t>(k) * envs;
        if (scene) {
            w.kind = numi::kMixScene;
            numi::SceneParams& p = w.scene;
            p.model = d_smodel.ptr;
            p.q = d_q.ptr;
            p.v = d_v.ptr;
            p.manifolds = d_manifolds.ptr;
            p.manifold_count = d_mcount.ptr;
            p.reset_q = d_reset_q.ptr;
            p.reset_v = d_reset_v.ptr;
            p.friction_scale = d_friction.ptr;
            p.reset_masks = masks ? masks + item0 : nullptr;
            p.status_codes = status ? status + item0 : nullptr;
            p.stats = d_stats.ptr;
            p.workspace = d_workspace.ptr;
            p.env_count = static_cast<int>(envs);
            p.substeps = static_cast<int>(config.physics_substeps);
            p.velocity_iterations = static_cast<int>(config.velocity_iterations);
            p.final_velocity_iterations = static_cast<int>(config.final_velocity_iterations);
            p.support_mapped = smodel.support_mapped;
            p.island_labels = island_labels ? d_island_labels.ptr : nullptr;
            return w;
        }
        w.kind = contact ? numi::kMixContact : numi::kMixFreeMotion;
        w.layout = layout;
        numi::StepParams& p = w.step;
        p.model = d_model.ptr;
        p.q = d_q.ptr;
        p.v = d_v.ptr;
        p.manifolds = d_manifolds.ptr;
        p.reset_q = d_reset_q.ptr;
        p.reset_v = d_reset_v.ptr;
        p.friction_scale = d_friction.ptr;
        p.actions = actions ? actions + item0 * model.world.action_count : nullptr;
        p.reset_masks = masks ? masks + item0 : nullptr;
        p.status_codes = status ? status + item0 : nullptr;
        p.stats = d_stats.ptr;
        p.env_count = static_cast<int>(envs);
        p.substeps = static_cast<int>(config.physics_substeps);
        p.velocity_iterations = static_cast<int>(config.velocity_iterations);
        p.final_velocity_iterations = static_cast<int>(config.final_velocity_iterations);
        return w;
    }

    void sample_resets() {
        const std::uint32_t nq = model.world.nq, nv = model.world.nv;
        reset_q.assign(static_cast<size_t>(envs) * nq, 0.0f);
        reset_v.assign(static_cast<size_t>(envs) * nv, 0.0f);
        friction.assign(envs, 1.0f);
        for (std::uint32_t e = 0; e < envs; ++e)
            numi::sample_reset_state(model, seed, e, &reset_q[static_cast<size_t>(e) * nq], &reset_v[static_cast<size_t>(e) * nv], &friction[e]);
        check(cudaMemcpyAsync(d_reset_q.ptr, reset_q.data(), reset_q.size() * sizeof(float), cudaMemcpyHostToDevice, stream), "upload reset q");
        check(cudaMemcpyAsync(d_reset_v.ptr, reset_v.data(), reset_v.size() * sizeof(float), cudaMemcpyHostToDevice, stream), "upload reset v");
        check(cudaMemcpyAsync(d_friction.ptr, friction.data(), friction.size() * sizeof(float), cudaMemcpyHostToDevice, stream), "upload friction");
        check(cudaMemcpyAsync(d_q.ptr, d_reset_q.ptr, reset_q.size() * sizeof(float), cudaMemcpyDeviceToDevice, stream), "init q");
        check(cudaMemcpyAsync(d_v.ptr, d_reset_v.ptr, reset_v.size() * sizeof(float), cudaMemcpyDeviceToDevice, stream), "init v");
        if (d_manifolds.count) check(cudaMemsetAsync(d_manifolds.ptr, 0, d_manifolds.count * sizeof(float), stream), "clear manifolds");
        if (d_mcount.count) check(cudaMemsetAsync(d_mcount.ptr, 0, d_mcount.count * sizeof(std::uint32_t), stream), "clear manifold counts");
        clear_compensation();
        check(cudaStreamSynchronize(stream), "reset");
    }

    // The compensation terms belong to the state they were accumulated on:
    // any new state starts without them; the audit takes a new reference.
    void clear_compensation() {
        if (d_qcomp.count) check(cudaMemsetAsync(d_qcomp.ptr, 0, d_qcomp.count * sizeof(float), stream), "clear compensation");
        if (audit) check(cudaMemsetAsync(d_audit.ptr, 0, d_audit.count * sizeof(double), stream), "clear audit");
    }

    // Layout and environments per CTA of the current (solver, precision).
    const numi::WarpLayout& step_layout() const {
        if (quality) return precision == MR_PRECISION_COMPENSATED ? layout_q_comp : layout_q;
        return precision == MR_PRECISION_COMPENSATED ? layout_comp : layout;
    }
    int step_warps_per_block() const { return quality ? warps_per_block_q[precision] : warps_per_block[precision]; }
    int step_resident_warps_per_sm() const { return quality ? resident_warps_per_sm_q[precision] : resident_warps_per_sm[precision]; }

    size_t manifold_words() const {
        return scene ? static_cast<size_t>(numi::kSceneManifolds) * numi::kSceneSlotWords
                     : static_cast<size_t>(model.world.pair_count) * numi::kManifoldWords;
    }

    // Enqueue `steps` control steps reading actions/masks from device memory.
    // With `host_obs` (pinned), step k's observation slice is copied there on
    // copy_stream once step k is done, overlapping step k + 1; `s` waits for
    // the last copy.
    void enqueue(std::uint32_t steps, const float* actions, const std::uint32_t* masks, float* obs,
                 std::uint32_t* status, std::uint32_t* contacts, cudaStream_t s, float* host_obs = nullptr) {
        const std::uint32_t na = model.world.action_count;
        const std::uint32_t nobs = model.world.nq + model.world.nv;
        check(cudaMemsetAsync(d_stats.ptr, 0, numi::kStatCount * sizeof(std::uint32_t), s), "clear stats");
        check(cudaMemsetAsync(d_stats.ptr + numi::kStatFirstFailEnv, 0xff, sizeof(std::uint32_t), s), "clear stats");
        if (scene) {
            for (std::uint32_t k = 0; k < steps; ++k) {
                numi::SceneParams p{};
                p.model = d_smodel.ptr;
                p.q = d_q.ptr;
                p.v = d_v.ptr;
                p.manifolds = d_manifolds.ptr;
                p.manifold_count = d_mcount.ptr;
                p.reset_q = d_reset_q.ptr;
                p.reset_v = d_reset_v.ptr;
                p.friction_scale = d_friction.ptr;
                p.reset_masks = masks ? masks + static_cast<size_t>(k) * envs : nullptr;
                p.observations = obs ? obs + static_cast<size_t>(k) * envs * nobs : nullptr;
                p.status_codes = status ? status + static_cast<size_t>(k) * envs : nullptr;
                p.active_contacts = contacts ? contacts + static_cast<size_t>(k) * envs : nullptr;
                p.stats = d_stats.ptr;
                p.workspace = d_workspace.ptr;
                p.env_count = static_cast<int>(envs);
                p.substeps = static_cast<int>(config.physics_substeps);
                p.velocity_iterations = static_cast<int>(config.velocity_iterations);
                p.final_velocity_iterations = static_cast<int>(config.final_velocity_iterations);
                p.q_comp = precision == MR_PRECISION_COMPENSATED ? d_qcomp.ptr : nullptr;
                p.support_mapped = smodel.support_mapped;
                p.island_labels = island_labels ? d_island_labels.ptr : nullptr;
                p.audit = audit ? d_audit.ptr : nullptr;
                check(numi::launch_scene_step(p, s), "scene step launch");
                if (audit) check(numi::launch_scene_audit(p, s), "audit launch");
                if (host_obs && obs) copy_observations(k, obs, host_obs, s);
            }
            if (host_obs && obs) join_copies(s);
            (void)actions;
            (void)na;
            return;
        }
        const bool driven = policy != nullptr;
        const bool tasked = task != nullptr;
        // With a policy each chain evaluates it on its own block before each
        // of its steps; with a task, observe runs before the policy, apply
        // after it and complete after the physics step.
        const int nchains = static_cast<int>(std::min<std::uint32_t>(static_cast<std::uint32_t>(chains), envs));
        if (nchains > 1) {
            check(cudaEventRecord(ev_fork, s), "event");
            for (int c = 0; c < nchains; ++c) check(cudaStreamWaitEvent(chain_stream[c], ev_fork, 0), "stream wait");
        }
        for (int c = 0; c < nchains; ++c) {
            const std::uint32_t o = static_cast<std::uint32_t>(static_cast<std::uint64_t>(envs) * c / nchains);
            const std::uint32_t n = static_cast<std::uint32_t>(static_cast<std::uint64_t>(envs) * (c + 1) / nchains) - o;
            cudaStream_t cs = nchains > 1 ? chain_stream[c] : s;
            for (std::uint32_t k = 0; k < steps; ++k) {
                if (tasked) check(numi::launch_task_observe(task_params(k, o, n, actions, masks, obs, status), cs), "task observe launch");
                if (driven) enqueue_policy(k, o, n, const_cast<float*>(actions) + static_cast<size_t>(k) * envs * na, true, cs);
                if (tasked) check(numi::launch_task_apply(task_params(k, o, n, actions, masks, obs, status), cs), "task apply launch");
                const size_t item0 = static_cast<size_t>(k) * envs + o;  // this chain's first item of step k
                numi::StepParams p{};
                p.model = d_model.ptr;
                p.q = d_q.ptr + static_cast<size_t>(o) * model.world.nq;
                p.v = d_v.ptr + static_cast<size_t>(o) * model.world.nv;
                p.manifolds = d_manifolds.ptr + static_cast<size_t>(o) * manifold_words();
                p.reset_q = d_reset_q.ptr + static_cast<size_t>(o) * model.world.nq;
                p.reset_v = d_reset_v.ptr + static_cast<size_t>(o) * model.world.nv;
                p.friction_scale = d_friction.ptr + o;
                p.actions = tasked ? d_task_targets.ptr + static_cast<size_t>(o) * na : actions + item0 * na;
                p.reset_masks = tasked ? d_task_masks.ptr + item0 : (masks ? masks + item0 : nullptr);
                p.observations = obs && !tasked ? obs + item0 * nobs : nullptr;
                p.status_codes = status ? status + item0 : nullptr;
                p.active_contacts = contacts ? contacts + item0 : nullptr;
                p.stats = d_stats.ptr;
                p.env_count = static_cast<int>(n);
                p.env_base = static_cast<int>(o);
                p.substeps = static_cast<int>(config.physics_substeps);
                p.velocity_iterations = static_cast<int>(config.velocity_iterations);
                p.final_velocity_iterations = static_cast<int>(config.final_velocity_iterations);
                p.q_comp = precision == MR_PRECISION_COMPENSATED ? d_qcomp.ptr + static_cast<size_t>(o) * model.world.nq : nullptr;
                p.audit = audit ? d_audit.ptr + static_cast<size_t>(o) * numi::kAuditWords : nullptr;
                p.quality = quality_cfg;
                check(numi::launch_control_step(p, step_layout(), contact, precision, quality, step_warps_per_block(), cs),
                      "control step launch");
                if (audit)
                    check(numi::launch_audit_step(p, step_layout(), precision != MR_PRECISION_FP32, step_warps_per_block(), cs),
                          "audit launch");
                if (tasked)
                    check(numi::launch_task_complete(task_params(k, o, n, actions, masks, obs, status), cs), "task complete launch");
                if (host_obs && obs) copy_observation_rows(k, o, n, obs, host_obs, cs, c);
            }
            if (driven && evaluate_final) enqueue_policy(steps, o, n, nullptr, false, cs);
        }
        if (nchains > 1) {
            for (int c = 0; c < nchains; ++c) {
                check(cudaEventRecord(ev_chain[c], chain_stream[c]), "event");
                check(cudaStreamWaitEvent(s, ev_chain[c], 0), "stream wait");
            }
        }
        if (driven) check(numi::launch_policy_counter(d_policy_steps.ptr, steps, s), "policy counter");
        if (host_obs && obs) join_copies(s, nchains);
    }

    // Checks an advance's policy arguments and sizes the policy outputs.
    void prepare_policy(std::uint32_t steps, std::uint64_t revision, std::uint32_t evaluate_final_policy) {
        have_policy_outputs = false;
        if (!policy) {
            if (revision != 0 || evaluate_final_policy != 0)
                throw std::invalid_argument("no native policy is installed on this rollout (mr_task_rollout_set_policy)");
            evaluate_final = false;
            return;
        }
        if (revision != 0 && revision != policy->revision)
            throw std::invalid_argument("policy_revision " + std::to_string(revision) + " differs from the installed revision " +
                                        std::to_string(policy->revision));
        evaluate_final = evaluate_final_policy != 0;
        const size_t cells = static_cast<size_t>(steps) * envs;
        const size_t na = model.world.action_count;
        d_actions.resize(cells * na);
        d_latents.resize(cells * na);
        d_log_prob.resize(cells);
        d_values.resize(cells + envs);
        if (!d_policy_steps.ptr) {
            d_policy_steps.resize(1);
            check(cudaMemsetAsync(d_policy_steps.ptr, 0, sizeof(unsigned long long), stream), "policy counter");
        }
    }
    void read_policy_outputs(std::uint32_t steps, cudaStream_t s) {
        if (!policy) return;
        const size_t cells = static_cast<size_t>(steps) * envs;
        const size_t na = model.world.action_count;
        h_latents.resize(cells * na);
        h_log_prob.resize(cells);
        h_values.resize(cells + envs);
        check(cudaMemcpyAsync(h_latents.ptr, d_latents.ptr, cells * na * sizeof(float), cudaMemcpyDeviceToHost, s), "latents D2H");
        check(cudaMemcpyAsync(h_log_prob.ptr, d_log_prob.ptr, cells * sizeof(float), cudaMemcpyDeviceToHost, s), "log-probabilities D2H");
        if (!evaluate_final) check(cudaMemsetAsync(d_values.ptr + cells, 0, envs * sizeof(float), s), "bootstrap values");
        check(cudaMemcpyAsync(h_values.ptr, d_values.ptr, (cells + envs) * sizeof(float), cudaMemcpyDeviceToHost, s), "values D2H");
        have_policy_outputs = true;
        last_policy_steps = steps;
    }

    // Values per environment in an observation row: the task's actor frame,
    // else [q, v].
    std::uint32_t observation_count() const {
        return task ? static_cast<std::uint32_t>(task->prog.frames * task->prog.nobs) : model.world.nq + model.world.nv;
    }

    // Task-layer launch over environments [o, o + n) of control step k.
    numi::TaskParams task_params(std::uint32_t k, std::uint32_t o, std::uint32_t n, const float* actions, const std::uint32_t* masks,
                                 float* obs, const std::uint32_t* status) {
        const numi::TaskProgramDevice& P = task->prog;
        const size_t item0 = static_cast<size_t>(k) * envs + o;
        numi::TaskParams t{};
        t.prog = P;
        t.state = d_task_state.ptr + o;
        t.action_history = d_task_history.ptr + static_cast<size_t>(o) * P.history * P.na;
        t.previous_joint = d_task_previous.ptr + static_cast<size_t>(o) * 2 * P.na;
        t.frame = d_task_frame.ptr + static_cast<size_t>(o) * P.frames * P.nobs;
        t.critic_frame = P.ncritic ? d_task_critic.ptr + static_cast<size_t>(o) * P.ncritic : nullptr;
        t.reset_q = d_reset_q.ptr + static_cast<size_t>(o) * P.nq;
        t.reset_v = d_reset_v.ptr + static_cast<size_t>(o) * P.nv;
        t.q = d_q.ptr + static_cast<size_t>(o) * P.nq;
        t.v = d_v.ptr + static_cast<size_t>(o) * P.nv;
        t.masks_in = masks ? masks + item0 : nullptr;
        t.masks_out = d_task_masks.ptr + item0;
        t.observations = obs ? obs + item0 * P.frames * P.nobs : nullptr;
        t.actions = actions ? actions + item0 * P.na : nullptr;
        t.targets = d_task_targets.ptr + static_cast<size_t>(o) * P.na;
        t.status = status + item0;
        t.manifolds = d_manifolds.ptr + static_cast<size_t>(o) * manifold_words();
        t.air_time = d_task_air.ptr + static_cast<size_t>(o) * numi::kTaskMaxGroups;
        t.transitions = d_transitions.ptr + item0;
        t.policy_revision = policy ? policy->revision : 0u;
        t.env_count = static_cast<int>(n);
        t.env_base = static_cast<int>(o);
        return t;
    }

    // Every environment starts a new episode at the next advance.
    void clear_task_state() {
        check(cudaMemsetAsync(d_task_state.ptr, 0, d_task_state.count * sizeof(numi::TaskEnvState), stream), "clear task state");
        check(cudaStreamSynchronize(stream), "clear task state");
        transition_steps = 0;
        have_host_transitions = false;
    }

    void drop_all_graphs() {
        check(cudaStreamSynchronize(stream), "sync");
        for (auto& kv : graphs) cudaGraphExecDestroy(kv.second);
        graphs.clear();
    }

    // Sizes the task layer's per-advance buffers (reset masks, transitions).
    void prepare_task(std::uint32_t steps) {
        transition_steps = 0;
        have_host_transitions = false;
        if (!task) return;
        const size_t cells = static_cast<size_t>(steps) * envs;
        d_task_masks.resize(cells);
        d_transitions.resize(cells);
        transition_steps = steps;
    }

    // Policy evaluation before control step k (k == steps: the final state,
    // values into the bootstrap slot) writing step k's actions.
    bool evaluate_final = false;
    // Environments [o, o + n) only (one chain's block).
    void enqueue_policy(std::uint32_t k, std::uint32_t o, std::uint32_t n, float* actions_k, bool step, cudaStream_t s) {
        numi::PolicyParams pp = policy->params;
        pp.nq = static_cast<int>(model.world.nq);
        pp.nv = static_cast<int>(model.world.nv);
        pp.q = d_q.ptr + static_cast<size_t>(o) * pp.nq;
        pp.v = d_v.ptr + static_cast<size_t>(o) * pp.nv;
        pp.frame = task ? d_task_frame.ptr + static_cast<size_t>(o) * task->prog.frames * task->prog.nobs : nullptr;
        pp.frame_count = task ? task->prog.frames * task->prog.nobs : 0;
        pp.critic_frame = task && task->prog.ncritic ? d_task_critic.ptr + static_cast<size_t>(o) * task->prog.ncritic : nullptr;
        pp.critic_frame_count = task ? task->prog.ncritic : 0;
        pp.envs = static_cast<int>(n);
        pp.env_base = static_cast<int>(o);
        pp.na = static_cast<int>(model.world.action_count);
        const size_t cells = static_cast<size_t>(k) * envs + o;
        pp.actions = step ? actions_k + static_cast<size_t>(o) * pp.na : nullptr;
        pp.latents = step ? d_latents.ptr + cells * pp.na : nullptr;
        pp.log_prob = step ? d_log_prob.ptr + cells : nullptr;
        pp.values = d_values.ptr + cells;  // step `steps` holds the bootstrap values
        pp.step_base = d_policy_steps.ptr;
        pp.step_offset = static_cast<int>(k);
        check(numi::launch_policy(pp, s), "policy launch");
    }

    void copy_observations(std::uint32_t k, const float* obs, float* host_obs, cudaStream_t s) {
        copy_observation_rows(k, 0, envs, obs, host_obs, s);
    }
    // Rows [o, o + n) of step k's observations, once the work enqueued on
    // `s` so far is done.
    // Chain `chain` copies on its own copy stream.
    void copy_observation_rows(std::uint32_t k, std::uint32_t o, std::uint32_t n, const float* obs, float* host_obs, cudaStream_t s,
                               int chain = 0) {
        const size_t nobs = observation_count();
        const size_t at = (static_cast<size_t>(k) * envs + o) * nobs;
        cudaStream_t cs = chain == 0 ? copy_stream : chain_copy_stream[chain];
        check(cudaEventRecord(ev_step, s), "event");
        check(cudaStreamWaitEvent(cs, ev_step, 0), "stream wait");
        check(cudaMemcpyAsync(host_obs + at, obs + at, static_cast<size_t>(n) * nobs * sizeof(float), cudaMemcpyDeviceToHost, cs),
              "observations D2H");
    }
    // `s` waits for the copies of chains [0, chains).
    void join_copies(cudaStream_t s, int chains_used = 1) {
        check(cudaEventRecord(ev_copies, copy_stream), "event");
        check(cudaStreamWaitEvent(s, ev_copies, 0), "stream wait");
        for (int c = 1; c < chains_used; ++c) {
            check(cudaEventRecord(ev_chain_copies[c], chain_copy_stream[c]), "event");
            check(cudaStreamWaitEvent(s, ev_chain_copies[c], 0), "stream wait");
        }
    }

    void run(std::uint32_t steps, const float* actions, const std::uint32_t* masks, float* obs, std::uint32_t* status,
             std::uint32_t* contacts, cudaStream_t s, float* host_obs = nullptr) {
        const bool driven = policy != nullptr;
        const bool tasked = task != nullptr;
        const GraphKey key{steps, actions, masks, obs, status, contacts, precision, host_obs,
                           driven ? static_cast<const void*>(policy->arena.ptr) : nullptr, driven && evaluate_final,
                           driven ? d_latents.ptr : nullptr, driven ? d_log_prob.ptr : nullptr, driven ? d_values.ptr : nullptr,
                           tasked ? static_cast<const void*>(task->arena.ptr) : nullptr, tasked ? d_task_masks.ptr : nullptr,
                           tasked ? d_transitions.ptr : nullptr};
        auto it = graphs.find(key);
        if (it == graphs.end()) {
            cudaGraph_t graph = nullptr;
            check(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal), "begin capture");
            try {
                enqueue(steps, actions, masks, obs, status, contacts, s, host_obs);
            } catch (...) {
                cudaStreamEndCapture(s, &graph);
                if (graph) cudaGraphDestroy(graph);
                throw;
            }
            check(cudaStreamEndCapture(s, &graph), "end capture");
            cudaGraphExec_t exec = nullptr;
            const cudaError_t e = cudaGraphInstantiate(&exec, graph, 0);
            cudaGraphDestroy(graph);
            check(e, "graph instantiate");
            if (graphs.size() > 64) {
                for (auto& kv : graphs) cudaGraphExecDestroy(kv.second);
                graphs.clear();
            }
            it = graphs.emplace(key, exec).first;
        }
        check(cudaGraphLaunch(it->second, s), "graph launch");
    }

    void fill_advance(std::uint32_t steps, const std::uint32_t* host_status, const std::uint32_t* host_stats,
                      MRTaskRolloutAdvanceC* out, double gpu_ms, double wall_ms) {
        MRTaskRolloutAdvanceC a{};
        a.control_step_count = steps;
        a.first_failing_environment = MR_INVALID_INDEX;
        a.first_failing_control_step = MR_INVALID_INDEX;
        a.first_gpu_status_code = MR_STEP_SUCCESS;
        std::uint64_t failed = 0;
        if (host_status) {
            for (std::uint32_t k = 0; k < steps; ++k)
                for (std::uint32_t e = 0; e < envs; ++e) {
                    const std::uint32_t c = host_status[static_cast<size_t>(k) * envs + e];
                    if (c != MR_STEP_SUCCESS) {
                        ++failed;
                        if (a.first_failing_environment == MR_INVALID_INDEX) {
                            a.first_failing_environment = e;
                            a.first_failing_control_step = k;
                            a.first_gpu_status_code = c;
                        }
                    }
                }
        } else {
            // Device path: the kernels' counters (the lowest failing slot).
            failed = host_stats[numi::kStatFailedEnvs];
            if (failed != 0) a.first_failing_environment = host_stats[numi::kStatFirstFailEnv];
        }
        a.failed_environment_steps = static_cast<std::uint32_t>(failed);
        a.successful_environment_steps = static_cast<std::uint32_t>(static_cast<std::uint64_t>(steps) * envs - failed);
        a.host_requested_resets = host_stats[numi::kStatResets];
        a.maximum_active_contacts = host_stats[numi::kStatMaxContacts];
        a.maximum_manifolds = host_stats[numi::kStatMaxManifolds];
        a.high_water.candidate_pairs = host_stats[numi::kStatMaxCandidatePairs];
        a.high_water.raw_contacts = host_stats[numi::kStatMaxRawContacts];
        a.high_water.manifolds = host_stats[numi::kStatMaxManifolds];
        a.high_water.constraint_blocks = host_stats[numi::kStatMaxContacts];
        a.high_water.constraint_rows = 3u * host_stats[numi::kStatMaxContacts];
        a.high_water.islands = host_stats[numi::kStatMaxIslands];
        a.high_water.articulation_point_queries = 2u * host_stats[numi::kStatMaxContacts];
        a.high_water.dynamic_nodes = 1u;
        last_quality = MRQualityDiagnosticsC{};
        if (quality) {
            a.high_water.quality_generalized_velocities = model.world.nv;
            a.high_water.quality_rows = 3u * host_stats[numi::kStatMaxContacts];
            a.high_water.quality_direct_tiles = host_stats[numi::kStatMaxContacts] > 0 ? 1u : 0u;
            last_quality.maximum_newton_iterations = host_stats[numi::kStatQualityNewton];
            last_quality.line_search_iterations = host_stats[numi::kStatQualityLineSearch];
            std::memcpy(&last_quality.maximum_scaled_optimality, &host_stats[numi::kStatQualityResidual], sizeof(float));
            std::memcpy(&last_quality.maximum_cone_violation, &host_stats[numi::kStatQualityCone], sizeof(float));
            std::memcpy(&last_quality.maximum_complementarity, &host_stats[numi::kStatQualityComplementarity], sizeof(float));
        }
        a.high_water.operator_velocity_elements = model.world.nv;
        a.gpu_milliseconds = gpu_ms;
        a.submission_milliseconds = wall_ms;
        stats_layout.submitted_control_steps += steps;
        stats_layout.completed_environment_steps += a.successful_environment_steps;
        stats_layout.submission_count += 1;
        stats_layout.total_gpu_milliseconds += gpu_ms;
        stats_layout.total_submission_milliseconds += wall_ms;
        if (out) *out = a;
    }
};


extern "C" {

MR_API const char* mr_version(void) { return "numi-b200 0.1.0 (sm_100a)"; }

MR_API uint64_t mr_runtime_abi_fingerprint(void) {
    std::uint64_t h = 0xcbf29ce484222325ull;
    const std::size_t sizes[] = {sizeof(MRTaskRolloutConfigC), sizeof(MRRunManifestC), sizeof(MRTaskRolloutLayoutC),
                                 sizeof(MRTaskRolloutStageHighWaterC), sizeof(MRTaskRolloutAdvanceC), sizeof(MRModelWorldC),
                                 sizeof(MRModelJointC), sizeof(MRModelBodyC), sizeof(MRModelDofC), sizeof(MRModelShapeC),
                                 sizeof(MRModelMaterialC), sizeof(MRModelPairC), sizeof(MRManifoldC)};
    for (std::size_t s : sizes) h = (h ^ s) * 0x100000001b3ull;
    return h;
}

MR_API const char* mr_last_error(void) { return numi::rt::last_error(); }

MR_API MRTaskRolloutHandle* mr_create_task_rollout(const MRRunManifestC* manifest) {
    std::unique_ptr<MRTaskRolloutHandle> handle;
    const int rc = guarded([&] {
        if (manifest == nullptr) throw std::invalid_argument("manifest is null");
        const MRTaskRolloutConfigC& cfg = manifest->profile;
        if (cfg.environment_count == 0) throw std::invalid_argument("environment_count must be positive");
        if (cfg.physics_substeps == 0 || cfg.physics_substeps > MR_B200_MAX_SUBSTEPS)
            throw std::invalid_argument("physics_substeps must be in [1, 64]");
        if (!(cfg.control_timestep_seconds > 0.0f) || !std::isfinite(cfg.control_timestep_seconds))
            throw std::invalid_argument("control_timestep_seconds must be positive and finite");
        if (cfg.dynamic_sphere_count != 0 || cfg.dynamic_spheres != nullptr)
            throw std::invalid_argument("dynamic spheres are not supported by the synthetic worlds");
        if (manifest->visual_sensor_program != nullptr || manifest->inspection_visual_program != nullptr)
            throw std::invalid_argument("visual programs are not part of the physics path");
        handle = std::make_unique<MRTaskRolloutHandle>();
        MRTaskRolloutHandle& h = *handle;
        switch (manifest->source) {
            case MR_RUN_SOURCE_SYNTHETIC_CHAIN7: h.model = numi::build_chain7(cfg.seed); break;
            case MR_RUN_SOURCE_SYNTHETIC_TREE29: h.model = numi::build_tree29(cfg.seed); break;
            case MR_RUN_SOURCE_SYNTHETIC_PILE: h.model = numi::build_pile(cfg.seed); break;
            case MR_RUN_SOURCE_SYNTHETIC_CYLINDER_PILE: h.model = numi::build_pile(cfg.seed, 0, true); break;
            case MR_RUN_SOURCE_SYNTHETIC_PILE_GJK: h.model = numi::build_pile(cfg.seed, 0, false, true); break;
            case MR_RUN_SOURCE_SYNTHETIC_HULL_PILE: h.model = numi::build_pile(cfg.seed, 0, false, false, true); break;
            case MR_RUN_SOURCE_SYNTHETIC_STACK: h.model = numi::build_stack(cfg.seed); break;
            default:
                throw std::invalid_argument("unsupported run source " + std::to_string(manifest->source) +
                                            " (robot assets, URDF and world packs are not compiled by this library; "
                                            "use MR_RUN_SOURCE_SYNTHETIC_CHAIN7, _TREE29, _PILE or _STACK)");
        }
        if (h.model.world.pair_count > 0 && cfg.velocity_iterations == 0 && cfg.final_velocity_iterations == 0)
            throw std::invalid_argument("contact worlds need at least one velocity iteration");
        h.config = cfg;
        h.envs = cfg.environment_count;
        h.seed = cfg.seed;
        h.h = cfg.control_timestep_seconds / static_cast<float>(cfg.physics_substeps);
        const numi::CompiledModel& m = h.model;
        if (m.scene) {
            h.scene = true;
            h.contact = true;
            h.smodel = numi::rt::pack_scene(m, h.h);
            check(numi::configure_scene_step_kernel(), "scene kernel attributes");
        } else {
            numi::rt::KernelPlan plan;
            numi::rt::make_plan(h.model, h.h, plan);
            h.contact = plan.contact;
            h.dmodel = plan.dmodel;
            h.layout = plan.layout[0];
            h.layout_comp = plan.layout_comp[0];
            h.layout_q = plan.layout[1];
            h.layout_q_comp = plan.layout_comp[1];
            for (int prec = 0; prec < numi::rt::kPrecisionModes; ++prec) {
                h.warps_per_block[prec] = plan.warps_per_block[0][prec];
                h.resident_warps_per_sm[prec] = plan.resident_warps_per_sm[0][prec];
                h.warps_per_block_q[prec] = plan.warps_per_block[1][prec];
                h.resident_warps_per_sm_q[prec] = plan.resident_warps_per_sm[1][prec];
            }
        }
        check(cudaGetDevice(&h.device), "cudaGetDevice");
        cudaDeviceProp prop{};
        check(cudaGetDeviceProperties(&prop, h.device), "cudaGetDeviceProperties");
        h.device_name = prop.name;
        check(cudaStreamCreateWithFlags(&h.stream, cudaStreamNonBlocking), "stream");
        check(cudaStreamCreateWithFlags(&h.copy_stream, cudaStreamNonBlocking), "copy stream");
        check(cudaEventCreateWithFlags(&h.ev_step, cudaEventDisableTiming), "event");
        check(cudaEventCreateWithFlags(&h.ev_copies, cudaEventDisableTiming), "event");
        check(cudaEventCreateWithFlags(&h.ev_fork, cudaEventDisableTiming), "event");
        for (int c = 0; c < MRTaskRolloutHandle::kMaxChains; ++c) {
            check(cudaStreamCreateWithFlags(&h.chain_stream[c], cudaStreamNonBlocking), "chain stream");
            check(cudaEventCreateWithFlags(&h.ev_chain[c], cudaEventDisableTiming), "event");
            if (c > 0) {
                check(cudaStreamCreateWithFlags(&h.chain_copy_stream[c], cudaStreamNonBlocking), "chain copy stream");
                check(cudaEventCreateWithFlags(&h.ev_chain_copies[c], cudaEventDisableTiming), "event");
            }
        }
        // Two chains once the batch exceeds one resident wave of the FP32
        // kernel (at 4096 tree29 envs: 2.3 waves; measured +18 % over one
        // chain, three and four chains slower); NUMI_B200_CHAINS overrides.
        if (!h.scene) {
            const long resident = static_cast<long>(h.resident_warps_per_sm[0]) * prop.multiProcessorCount;
            h.chains = static_cast<long>(h.envs) > resident ? 2 : 1;
        }
        if (const char* env = std::getenv("NUMI_B200_CHAINS")) h.chains = std::max(1, std::min(MRTaskRolloutHandle::kMaxChains, std::atoi(env)));
        check(cudaEventCreate(&h.ev_start), "event");
        check(cudaEventCreate(&h.ev_stop), "event");
        check(cudaEventCreateWithFlags(&h.ev_in, cudaEventDisableTiming), "event");
        check(cudaEventCreateWithFlags(&h.ev_out, cudaEventDisableTiming), "event");
        if (h.scene) {
            h.d_smodel.resize(1);
            check(cudaMemcpy(h.d_smodel.ptr, &h.smodel, sizeof(numi::SceneModel), cudaMemcpyHostToDevice), "upload scene model");
            h.d_mcount.resize(h.envs);
            h.d_workspace.resize(h.envs * numi::scene_workspace_words());
        } else {
            h.d_model.resize(1);
            check(cudaMemcpy(h.d_model.ptr, &h.dmodel, sizeof(numi::DeviceModel), cudaMemcpyHostToDevice), "upload model");
        }
        const size_t nq = m.world.nq, nv = m.world.nv;
        h.d_q.resize(h.envs * nq);
        h.d_v.resize(h.envs * nv);
        h.d_reset_q.resize(h.envs * nq);
        h.d_reset_v.resize(h.envs * nv);
        h.d_friction.resize(h.envs);
        h.d_qcomp.resize(h.envs * nq);
        if (h.contact) h.d_manifolds.resize(h.envs * h.manifold_words());
        h.d_stats.resize(numi::kStatCount);
        h.h_stats.resize(numi::kStatCount);
        h.sample_resets();
        h.stats_layout.environment_count = h.envs;
        h.stats_layout.nq = m.world.nq;
        h.stats_layout.nv = m.world.nv;
        h.stats_layout.action_count = m.world.action_count;
        h.stats_layout.actor_observation_count = m.world.nq + m.world.nv;
        h.stats_layout.critic_observation_count = m.world.nq + m.world.nv;
        h.stats_layout.scene_body_count = m.scene ? m.scene_bodies : 0u;
        h.stats_layout.world_fingerprint = m.fingerprint;
        h.stats_layout.run_fingerprint = m.fingerprint ^ (cfg.seed * 0x9e3779b97f4a7c15ull);
        h.stats_layout.robot_fingerprint = m.fingerprint;
        h.stats_layout.immutable_private_bytes = sizeof(numi::DeviceModel);
        h.stats_layout.persistent_state_private_bytes =
            (h.d_q.count + h.d_v.count + h.d_manifolds.count + h.d_reset_q.count + h.d_reset_v.count + h.d_friction.count) * sizeof(float);
    });
    if (rc != 0) return nullptr;
    return handle.release();
}

MR_API void mr_task_rollout_destroy(MRTaskRolloutHandle* handle) {
    if (handle) {
        if (handle->stream) cudaStreamSynchronize(handle->stream);
        delete handle;
    }
}

MR_API int mr_task_rollout_reset(MRTaskRolloutHandle* handle, uint64_t seed) {
    return guarded([&] {
        if (!handle) throw std::invalid_argument("handle is null");
        handle->seed = seed;
        handle->sample_resets();
        handle->last_steps = 0;
        handle->have_final_q = false;
        if (handle->task) {
            // Every environment starts a new episode under the new seed's draws.
            handle->task->prog.seed = seed;
            handle->clear_task_state();
            handle->drop_all_graphs();
        }
    });
}

MR_API int mr_task_rollout_set_state_readback(MRTaskRolloutHandle* handle, uint32_t enabled) {
    return guarded([&] {
        if (!handle) throw std::invalid_argument("handle is null");
        handle->readback = enabled != 0;
        if (!handle->readback) handle->have_final_q = false;
    });
}

namespace {

// Validates a policy pack against the rollout's world and uploads it
// (transposed weights, vectors with their defaults) as one device arena.
std::unique_ptr<InstalledPolicy> compile_policy(const MRTaskRolloutHandle& h, const MRPolicyPackC& pk) {
    using numi::kPolicyMaxLayers;
    using numi::kPolicyMaxWidth;
    const std::uint32_t nobs = h.observation_count(), na = h.model.world.action_count;
    if (!pk.id || !pk.id[0] || !pk.layers || pk.layer_count == 0)
        throw std::invalid_argument("policy identity and dense layers are required");
    if (pk.revision == 0) throw std::invalid_argument("policy revision must be non-zero (zero means no policy)");
    if (na == 0) throw std::invalid_argument("this world takes no actions; a policy cannot drive it");
    if (pk.layer_count > static_cast<size_t>(kPolicyMaxLayers) || pk.critic_layer_count > static_cast<size_t>(kPolicyMaxLayers))
        throw std::invalid_argument("at most " + std::to_string(kPolicyMaxLayers) + " dense layers per network");
    if (pk.critic_layer_count != 0 && !pk.critic_layers) throw std::invalid_argument("critic layers are null");
    if (nobs > static_cast<std::uint32_t>(kPolicyMaxWidth))
        throw std::invalid_argument("the observation is wider than " + std::to_string(kPolicyMaxWidth));
    if (!(pk.action_clip > 0.0f)) throw std::invalid_argument("action_clip must be positive");
    auto optional = [](const float* v, size_t n, size_t want, const char* what) {
        if (n != 0 && (n != want || !v))
            throw std::invalid_argument(std::string(what) + " must have " + std::to_string(want) + " values (or none)");
        return n != 0;
    };
    const bool norm = optional(pk.observation_mean, pk.observation_mean_count, nobs, "observation_mean");
    if (optional(pk.observation_inverse_standard_deviation, pk.observation_inverse_standard_deviation_count, nobs,
                 "observation_inverse_standard_deviation") != norm)
        throw std::invalid_argument("observation mean and inverse standard deviation go together");
    // The critic reads the task's critic frame when the task has critic operators.
    const std::uint32_t ncrit = h.task && h.task->prog.ncritic ? static_cast<std::uint32_t>(h.task->prog.ncritic) : nobs;
    const bool cnorm = optional(pk.critic_observation_mean, pk.critic_observation_mean_count, ncrit, "critic_observation_mean");
    if (optional(pk.critic_observation_inverse_standard_deviation, pk.critic_observation_inverse_standard_deviation_count, ncrit,
                 "critic_observation_inverse_standard_deviation") != cnorm)
        throw std::invalid_argument("critic observation mean and inverse standard deviation go together");
    if ((norm || cnorm) && !(pk.observation_clip > 0.0f)) throw std::invalid_argument("observation_clip must be positive");
    const bool stochastic = optional(pk.action_log_standard_deviation, pk.action_log_standard_deviation_count, na,
                                     "action_log_standard_deviation");
    const bool has_bias = optional(pk.action_bias, pk.action_bias_count, na, "action_bias");
    const bool has_scale = optional(pk.action_scale, pk.action_scale_count, na, "action_scale");
    auto check_chain = [&](const MRPolicyDenseLayerC* L, size_t n, std::uint32_t out, const char* net, std::uint32_t inputs) {
        std::uint32_t in = inputs;
        for (size_t l = 0; l < n; ++l) {
            const MRPolicyDenseLayerC& d = L[l];
            const std::string where = std::string(net) + " layer " + std::to_string(l);
            if (d.input_count != in) throw std::invalid_argument(where + " takes " + std::to_string(d.input_count) + " inputs, expected " + std::to_string(in));
            if (d.output_count == 0 || d.output_count > static_cast<std::uint32_t>(kPolicyMaxWidth))
                throw std::invalid_argument(where + " must have 1-" + std::to_string(kPolicyMaxWidth) + " outputs");
            if (d.activation > MR_POLICY_ACTIVATION_C_SILU) throw std::invalid_argument(where + " has an unknown activation");
            if (!d.weights || d.weight_count != static_cast<size_t>(d.input_count) * d.output_count)
                throw std::invalid_argument(where + " needs input_count x output_count weights");
            if (d.bias_count != 0 && (d.bias_count != d.output_count || !d.bias))
                throw std::invalid_argument(where + " bias must have output_count values (or none)");
            in = d.output_count;
        }
        if (in != out) throw std::invalid_argument(std::string(net) + " must end in " + std::to_string(out) + " outputs");
    };
    check_chain(pk.layers, pk.layer_count, na, "actor", nobs);
    if (pk.critic_layer_count) check_chain(pk.critic_layers, pk.critic_layer_count, 1u, "critic", ncrit);

    // Arena: per layer [in][out] weights then bias; then the vectors.
    std::vector<float> arena;
    auto put = [&](const float* v, size_t n, float fill) {
        const size_t at = arena.size();
        for (size_t i = 0; i < n; ++i) arena.push_back(v ? v[i] : fill);
        while (arena.size() % 4) arena.push_back(0.0f);  // 16-byte aligned spans
        return at;
    };
    std::vector<size_t> w_at, b_at, cw_at, cb_at;
    auto put_layers = [&](const MRPolicyDenseLayerC* L, size_t n, std::vector<size_t>& wa, std::vector<size_t>& ba) {
        for (size_t l = 0; l < n; ++l) {
            const MRPolicyDenseLayerC& d = L[l];
            std::vector<float> t(static_cast<size_t>(d.input_count) * d.output_count);
            for (std::uint32_t o = 0; o < d.output_count; ++o)
                for (std::uint32_t i = 0; i < d.input_count; ++i) t[static_cast<size_t>(i) * d.output_count + o] = d.weights[static_cast<size_t>(o) * d.input_count + i];
            wa.push_back(put(t.data(), t.size(), 0.0f));
            ba.push_back(put(d.bias_count ? d.bias : nullptr, d.output_count, 0.0f));
        }
    };
    put_layers(pk.layers, pk.layer_count, w_at, b_at);
    put_layers(pk.critic_layers, pk.critic_layer_count, cw_at, cb_at);
    const size_t mean_at = norm ? put(pk.observation_mean, nobs, 0.0f) : 0, inv_at = norm ? put(pk.observation_inverse_standard_deviation, nobs, 0.0f) : 0;
    const size_t cmean_at = cnorm ? put(pk.critic_observation_mean, ncrit, 0.0f) : 0,
                 cinv_at = cnorm ? put(pk.critic_observation_inverse_standard_deviation, ncrit, 0.0f) : 0;
    const size_t ls_at = stochastic ? put(pk.action_log_standard_deviation, na, 0.0f) : 0;
    const size_t ab_at = put(has_bias ? pk.action_bias : nullptr, na, 0.0f);
    const size_t as_at = put(has_scale ? pk.action_scale : nullptr, na, 1.0f);

    auto out = std::make_unique<InstalledPolicy>();
    out->revision = pk.revision;
    out->id = pk.id;
    out->has_critic = pk.critic_layer_count != 0;
    out->arena.resize(arena.size());
    check(cudaMemcpy(out->arena.ptr, arena.data(), arena.size() * sizeof(float), cudaMemcpyHostToDevice), "policy upload");
    const float* base = out->arena.ptr;
    numi::PolicyParams& pp = out->params;
    pp.actor_layers = static_cast<int>(pk.layer_count);
    pp.critic_layers = static_cast<int>(pk.critic_layer_count);
    for (size_t l = 0; l < pk.layer_count; ++l)
        pp.actor[l] = numi::PolicyLayer{static_cast<int>(pk.layers[l].input_count), static_cast<int>(pk.layers[l].output_count),
                                        static_cast<int>(pk.layers[l].activation), 0, base + w_at[l], base + b_at[l]};
    for (size_t l = 0; l < pk.critic_layer_count; ++l)
        pp.critic[l] = numi::PolicyLayer{static_cast<int>(pk.critic_layers[l].input_count),
                                         static_cast<int>(pk.critic_layers[l].output_count),
                                         static_cast<int>(pk.critic_layers[l].activation), 0, base + cw_at[l], base + cb_at[l]};
    pp.obs_mean = norm ? base + mean_at : nullptr;
    pp.obs_inv_std = norm ? base + inv_at : nullptr;
    pp.critic_mean = cnorm ? base + cmean_at : nullptr;
    pp.critic_inv_std = cnorm ? base + cinv_at : nullptr;
    pp.obs_clip = pk.observation_clip;
    pp.action_clip = pk.action_clip;
    pp.log_std = stochastic ? base + ls_at : nullptr;
    pp.action_bias = base + ab_at;
    pp.action_scale = base + as_at;
    // Draw key: the rollout seed and the policy revision, mixed (SplitMix64).
    auto mix = [](std::uint64_t x) {
        x += 0x9e3779b97f4a7c15ull;
        x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
        x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
        return x ^ (x >> 31);
    };
    pp.key = mix(h.seed) ^ mix(pk.revision ^ 0x5bd1e995ull);
    return out;
}

void drop_graphs(MRTaskRolloutHandle& h) { h.drop_all_graphs(); }

bool finite_value(float x) { return std::isfinite(x); }

// Validates a task program against the rollout's world (the operator subset
// of include/numi_b200.h, every index in range) and uploads its tables as one
// device arena.
std::unique_ptr<InstalledTask> compile_task(const MRTaskRolloutHandle& h, const MRTaskProgramC& t) {
    using std::to_string;
    const numi::DeviceModel& M = h.dmodel;
    const std::uint32_t nq = h.model.world.nq, nv = h.model.world.nv, na = h.model.world.action_count;
    auto need = [](bool ok, const std::string& what) {
        if (!ok) throw std::invalid_argument("task program: " + what);
    };
    need(na > 0 && na <= static_cast<std::uint32_t>(numi::kTaskMaxActions), "the world must take 1-64 actions");
    need(t.actions != nullptr && t.action_count == na, "action_count must equal the world's " + to_string(na) + " actions");
    need(t.actor != nullptr && t.actor_count > 0 && t.actor_count <= static_cast<std::uint32_t>(numi::kTaskMaxObservations),
         "1-256 actor observation operators are required");
    need(t.default_q != nullptr && t.default_q_count == nq, "default_q must hold nq = " + to_string(nq) + " values");
    for (std::uint32_t i = 0; i < nq; ++i) need(finite_value(t.default_q[i]), "default_q must be finite");
    need(t.action_history >= 3 && t.action_history <= static_cast<std::uint32_t>(numi::kTaskMaxHistory), "action_history must be 3-8");
    need(t.observation_history >= 1 && t.observation_history <= 8u, "observation_history must be 1-8");
    need(static_cast<std::uint64_t>(t.observation_history) * t.actor_count <= static_cast<std::uint64_t>(numi::kTaskMaxObservations),
         "observation_history x actor_count must be at most 256 (the policy's widest input)");
    need(t.maximum_episode_steps >= 1, "maximum_episode_steps must be positive");
    need(finite_value(t.gait_period_seconds) && t.gait_period_seconds > 0.0f, "gait_period_seconds must be positive");
    need(finite_value(t.command_duration_seconds[0]) && finite_value(t.command_duration_seconds[1]) &&
             t.command_duration_seconds[0] > 0.0f && t.command_duration_seconds[0] <= t.command_duration_seconds[1],
         "command durations must satisfy 0 < minimum <= maximum");
    need(finite_value(t.standing_probability) && t.standing_probability >= 0.0f && t.standing_probability <= 1.0f,
         "standing_probability must lie in [0, 1]");
    need(finite_value(t.base_height_target), "base_height_target must be finite");
    // One band at least, as the reference's pack validation asks
    // (TaskProgram.cpp:855); the band range widens each command bound by
    // its step per band, within limits that contain the band-0 range.
    need(t.difficulty_band_count >= 1 && t.difficulty_band_count <= 1024u, "difficulty_band_count must be 1-1024");
    need(finite_value(t.band_sampling_exponent) && t.band_sampling_exponent > 0.0f, "band_sampling_exponent must be positive");
    for (int k = 0; k < 3; ++k) {
        need(finite_value(t.command_lower[k]) && finite_value(t.command_upper[k]) && t.command_lower[k] <= t.command_upper[k],
             "command bounds must be finite with lower <= upper");
        need(finite_value(t.command_limit_lower[k]) && finite_value(t.command_limit_upper[k]) &&
                 t.command_limit_lower[k] <= t.command_lower[k] && t.command_upper[k] <= t.command_limit_upper[k],
             "command limits must be finite and contain the command bounds");
        need(finite_value(t.command_band_step[k]) && t.command_band_step[k] >= 0.0f, "command_band_step must be finite and >= 0");
        need(finite_value(t.root_reference[k]), "root_reference must be finite");
    }
    if (h.config.override_difficulty_band_range != 0u)
        need(h.config.minimum_difficulty_band <= h.config.maximum_difficulty_band,
             "minimum_difficulty_band must not exceed maximum_difficulty_band");
    for (std::uint32_t a = 0; a < na; ++a) {
        const MRTaskActionBindingC& b = t.actions[a];
        const std::string where = "action " + to_string(a);
        need(b.dof_index == static_cast<std::uint32_t>(M.action_dof[a]), where + " must bind DoF " + to_string(M.action_dof[a]) +
                                                                             ", the DoF the world drives from it");
        need(b.v_index == b.dof_index && M.dof_q[b.dof_index] >= 0 && b.q_index == static_cast<std::uint32_t>(M.dof_q[b.dof_index]),
             where + ": q_index and v_index must be the DoF's coordinate and velocity");
        need(finite_value(b.scale) && finite_value(b.lower_target) && finite_value(b.upper_target) && b.lower_target <= b.upper_target,
             where + ": scale and target bounds must be finite with lower <= upper");
        need(finite_value(b.response_time_seconds) && b.response_time_seconds >= 0.0f, where + ": response time must be >= 0");
    }
    need(t.critic_count == 0 || t.critic != nullptr, "critic is null");
    need(t.critic_count <= static_cast<std::uint32_t>(numi::kTaskMaxObservations), "at most 256 critic operators");
    for (std::uint32_t i = 0; i < t.actor_count + t.critic_count; ++i) {
        const bool actor_op = i < t.actor_count;
        const MRTaskObservationOperatorC& o = actor_op ? t.actor[i] : t.critic[i - t.actor_count];
        const std::string where = (actor_op ? "actor operator " : "critic operator ") + to_string(actor_op ? i : i - t.actor_count);
        need(finite_value(o.transform_scale) && finite_value(o.transform_offset) && finite_value(o.noise_amplitude) &&
                 o.noise_amplitude >= 0.0f, where + ": transform and noise must be finite");
        need((o.flags & ~static_cast<std::uint32_t>(MR_TASK_OBSERVATION_NORMALIZE_VECTOR3)) == 0u &&
                 (o.flags == 0u || o.opcode == MR_TASK_OBSERVE_PROJECTED_GRAVITY), where + ": only projected gravity may be normalised");
        switch (o.opcode) {
        case MR_TASK_OBSERVE_ROOT_ANGULAR_VELOCITY_LOCAL:
        case MR_TASK_OBSERVE_PROJECTED_GRAVITY:
        case MR_TASK_OBSERVE_ROOT_LINEAR_VELOCITY_LOCAL:
            need(o.component < 3u, where + ": component must be 0-2");
            break;
        case MR_TASK_OBSERVE_COMMAND:
            need(o.component < 4u, where + ": component must be 0-3");
            break;
        case MR_TASK_OBSERVE_GAIT_PHASE:
            need(o.component < 2u, where + ": component must be 0-1");
            break;
        case MR_TASK_OBSERVE_SUPPORT_SENSE:
            need(o.component < 3u, where + ": component must be 0-2");
            break;
        case MR_TASK_OBSERVE_ROOT_HEIGHT:
            break;
        case MR_TASK_OBSERVE_CONTACT_METRIC:
        case MR_TASK_OBSERVE_CONTACT_WRENCH_LOCAL:
            need(o.source < t.contact_group_count && o.component < 6u, where + ": source must be a contact group and component 0-5");
            break;
        case MR_TASK_OBSERVE_JOINT_POSITION_ERROR:
        case MR_TASK_OBSERVE_JOINT_VELOCITY:
        case MR_TASK_OBSERVE_PREVIOUS_ACTION:
        case MR_TASK_OBSERVE_JOINT_FINITE_DIFFERENCE_VELOCITY:
            need(o.source < na, where + ": source must be an action index");
            break;
        case MR_TASK_OBSERVE_DELAYED_ACTION:
            need(o.source < na && o.component <= t.action_history - 2, where + ": source must be an action index and component at most "
                                                                               "action_history - 2");
            break;
        default:
            need(false, where + ": opcode " + to_string(o.opcode) + " is outside the evaluated subset");
        }
    }
    need(t.joint_group_count == 0 || t.joint_groups != nullptr, "joint_groups is null");
    need(t.joint_member_count == 0 || t.joint_members != nullptr, "joint_members is null");
    for (std::uint32_t g = 0; g < t.joint_group_count; ++g) {
        const MRTaskIndexGroupC& G = t.joint_groups[g];
        need(static_cast<std::uint64_t>(G.first) + G.count <= t.joint_member_count, "joint group " + to_string(g) + " overruns joint_members");
    }
    for (std::uint32_t m = 0; m < t.joint_member_count; ++m) need(t.joint_members[m] < na, "joint members must be action indices");
    need(t.contact_group_count <= static_cast<std::uint32_t>(numi::kTaskMaxGroups), "at most 8 contact groups");
    need(t.contact_group_count == 0 || t.contact_groups != nullptr, "contact_groups is null");
    need(t.contact_member_count == 0 || t.contact_members != nullptr, "contact_members is null");
    need(finite_value(t.support_force_threshold) && t.support_force_threshold >= 0.0f && finite_value(t.clearance_target),
         "support_force_threshold and clearance_target must be finite");
    for (std::uint32_t g = 0; g < t.contact_group_count; ++g) {
        const MRTaskContactGroupC& G = t.contact_groups[g];
        const std::string where = "contact group " + to_string(g);
        need(static_cast<std::uint64_t>(G.first) + G.count <= t.contact_member_count, where + " overruns contact_members");
        need(G.reference_body < static_cast<std::uint32_t>(M.nb), where + ": reference_body must be an articulated body");
        need((G.flags & ~3u) == 0u, where + ": flags are SUPPORT and FORBIDDEN");
        bool finite_all = finite_value(G.gait_phase_offset) && finite_value(G.stance_fraction);
        for (int k = 0; k < 4; ++k) finite_all = finite_all && finite_value(G.local_reference[k]) && finite_value(G.kinematic_reference[k]);
        need(finite_all, where + ": references and gait must be finite");
    }
    for (std::uint32_t m = 0; m < t.contact_member_count; ++m)
        need(t.contact_members[m] < static_cast<std::uint32_t>(M.nb), "contact members must be articulated bodies");
    need(t.reward_count == 0 || t.rewards != nullptr, "rewards is null");
    for (std::uint32_t i = 0; i < t.reward_count; ++i) {
        const MRTaskRewardOperatorC& r = t.rewards[i];
        const std::string where = "reward operator " + to_string(i);
        need(finite_value(r.weight) && finite_value(r.parameters[0]) && finite_value(r.parameters[1]) && finite_value(r.parameters[2]),
             where + ": weight and parameters must be finite");
        switch (r.opcode) {
        case MR_TASK_REWARD_JOINT_GROUP_POSTURE_SQUARED:
        case MR_TASK_REWARD_JOINT_GROUP_POSTURE_ABSOLUTE:
            need(r.group < t.joint_group_count, where + ": group must be a joint group index");
            break;
        case MR_TASK_REWARD_GAIT_CONTACT_MATCH:
        case MR_TASK_REWARD_SWING_CLEARANCE:
        case MR_TASK_REWARD_FOOT_CLEARANCE:
        case MR_TASK_REWARD_SUPPORT_SLIP:
        case MR_TASK_REWARD_FORBIDDEN_CONTACT:
            need(r.group == MR_INVALID_INDEX || r.group < t.contact_group_count,
                 where + ": group must be a contact group index or MR_INVALID_INDEX");
            break;
        case MR_TASK_REWARD_LINEAR_VELOCITY_TRACKING:
        case MR_TASK_REWARD_YAW_VELOCITY_TRACKING:
        case MR_TASK_REWARD_CONSTANT:
        case MR_TASK_REWARD_ROOT_VERTICAL_VELOCITY_SQUARED:
        case MR_TASK_REWARD_ROOT_ROLL_PITCH_VELOCITY_SQUARED:
        case MR_TASK_REWARD_TILT_SQUARED:
        case MR_TASK_REWARD_ROOT_HEIGHT_ERROR_SQUARED:
        case MR_TASK_REWARD_JOINT_VELOCITY_SQUARED:
        case MR_TASK_REWARD_JOINT_ACCELERATION_SQUARED:
        case MR_TASK_REWARD_ACTION_RATE_SQUARED:
        case MR_TASK_REWARD_JOINT_LIMIT_VIOLATION_SQUARED:
        case MR_TASK_REWARD_PROJECTED_GRAVITY_HORIZONTAL_SQUARED:
        case MR_TASK_REWARD_JOINT_LIMIT_VIOLATION_ABSOLUTE:
        case MR_TASK_REWARD_ROOT_HEIGHT_NORMALIZED:
        case MR_TASK_REWARD_ROOT_HEIGHT_PROGRESS:
        case MR_TASK_REWARD_UPRIGHTNESS:
            break;
        default:
            need(false, where + ": opcode " + to_string(r.opcode) + " is outside the evaluated subset");
        }
    }
    const bool terminations = h.config.disable_task_terminations == 0u;  // the reference clears them (c_api.cpp:1415-1417)
    need(t.termination_count == 0 || t.terminations != nullptr, "terminations is null");
    for (std::uint32_t i = 0; i < t.termination_count; ++i) {
        const MRTaskTerminationOperatorC& o = t.terminations[i];
        need(o.opcode == MR_TASK_TERMINATE_MINIMUM_ROOT_HEIGHT || o.opcode == MR_TASK_TERMINATE_MAXIMUM_TILT ||
                 o.opcode == MR_TASK_TERMINATE_CONTACT_GROUP,
             "termination operator " + to_string(i) + ": opcode " + to_string(o.opcode) + " is outside the evaluated subset");
        need(o.opcode != MR_TASK_TERMINATE_CONTACT_GROUP || o.group < t.contact_group_count,
             "termination operator " + to_string(i) + ": group must be a contact group index");
        need(finite_value(o.threshold) && finite_value(o.failure_penalty), "termination operator " + to_string(i) + " must be finite");
        need(o.maximum_band == MR_INVALID_INDEX || o.minimum_band <= o.maximum_band,
             "termination operator " + to_string(i) + ": minimum_band must not exceed maximum_band");
    }
    need(t.randomization_count == 0 || t.randomization != nullptr, "randomization is null");
    for (std::uint32_t i = 0; i < t.randomization_count; ++i) {
        const MRTaskRandomizationOperatorC& o = t.randomization[i];
        const std::string where = "randomization operator " + to_string(i);
        for (int k = 0; k < 4; ++k) need(finite_value(o.parameters[k]), where + ": parameters must be finite");
        switch (o.opcode) {
        case MR_TASK_RANDOMIZE_ROOT_POSITION:
        case MR_TASK_RANDOMIZE_ROOT_YAW:
        case MR_TASK_RANDOMIZE_ROOT_HEIGHT:
            need(M.floating != 0, where + ": root operators need a floating root");
            break;
        case MR_TASK_RANDOMIZE_JOINT_POSITION:
            need(o.target < nq, where + ": target must be a q index");
            break;
        case MR_TASK_RANDOMIZE_ACTION_POSITION:
        case MR_TASK_RANDOMIZE_VELOCITY:
        case MR_TASK_RANDOMIZE_ACTION_VELOCITY:
        case MR_TASK_RANDOMIZE_ACTION_DELAY:
        case MR_TASK_RANDOMIZE_OBSERVATION_DELAY:
            break;
        default:
            need(false, where + ": opcode " + to_string(o.opcode) + " is outside the evaluated subset");
        }
    }

    // One arena, every table 16-byte aligned.
    std::vector<unsigned char> arena;
    auto put = [&arena](const void* src, size_t bytes) {
        const size_t at = (arena.size() + 15) & ~static_cast<size_t>(15);
        arena.resize(at + bytes);
        if (bytes) std::memcpy(arena.data() + at, src, bytes);
        return at;
    };
    std::vector<float> lower(na), upper(na);
    for (std::uint32_t a = 0; a < na; ++a) {
        lower[a] = M.q_lower[t.actions[a].dof_index];
        upper[a] = M.q_upper[t.actions[a].dof_index];
    }
    const std::uint32_t nterm = terminations ? t.termination_count : 0u;
    const size_t at_actions = put(t.actions, na * sizeof(MRTaskActionBindingC));
    const size_t at_actor = put(t.actor, t.actor_count * sizeof(MRTaskObservationOperatorC));
    const size_t at_critic = put(t.critic, t.critic_count * sizeof(MRTaskObservationOperatorC));
    const size_t at_rewards = put(t.rewards, t.reward_count * sizeof(MRTaskRewardOperatorC));
    const size_t at_terms = put(t.terminations, nterm * sizeof(MRTaskTerminationOperatorC));
    const size_t at_random = put(t.randomization, t.randomization_count * sizeof(MRTaskRandomizationOperatorC));
    const size_t at_groups = put(t.joint_groups, t.joint_group_count * sizeof(MRTaskIndexGroupC));
    const size_t at_members = put(t.joint_members, t.joint_member_count * sizeof(std::uint32_t));
    const size_t at_cgroups = put(t.contact_groups, t.contact_group_count * sizeof(MRTaskContactGroupC));
    const size_t at_cmembers = put(t.contact_members, t.contact_member_count * sizeof(std::uint32_t));
    const size_t at_default = put(t.default_q, nq * sizeof(float));
    const size_t at_lower = put(lower.data(), na * sizeof(float));
    const size_t at_upper = put(upper.data(), na * sizeof(float));
    auto out = std::make_unique<InstalledTask>();
    out->arena.resize(arena.size());
    check(cudaMemcpy(out->arena.ptr, arena.data(), arena.size(), cudaMemcpyHostToDevice), "task upload");
    const unsigned char* base = out->arena.ptr;
    numi::TaskProgramDevice& P = out->prog;
    P.actions = reinterpret_cast<const MRTaskActionBindingC*>(base + at_actions);
    P.actor = reinterpret_cast<const MRTaskObservationOperatorC*>(base + at_actor);
    P.critic = reinterpret_cast<const MRTaskObservationOperatorC*>(base + at_critic);
    P.ncritic = static_cast<int>(t.critic_count);
    P.rewards = reinterpret_cast<const MRTaskRewardOperatorC*>(base + at_rewards);
    P.terminations = reinterpret_cast<const MRTaskTerminationOperatorC*>(base + at_terms);
    P.randomization = reinterpret_cast<const MRTaskRandomizationOperatorC*>(base + at_random);
    P.groups = reinterpret_cast<const MRTaskIndexGroupC*>(base + at_groups);
    P.members = reinterpret_cast<const std::uint32_t*>(base + at_members);
    P.contact_groups = reinterpret_cast<const MRTaskContactGroupC*>(base + at_cgroups);
    P.contact_members = reinterpret_cast<const std::uint32_t*>(base + at_cmembers);
    P.ncontact_groups = static_cast<int>(t.contact_group_count);
    P.model = h.d_model.ptr;
    P.support_force_threshold = t.support_force_threshold;
    P.clearance_target = t.clearance_target;
    P.physics_dt = h.config.control_timestep_seconds / static_cast<float>(std::max<std::uint32_t>(h.config.physics_substeps, 1u));
    P.ground_height = 0.0f;  // the world's static plane (normal +z): its height
    for (int sh = 0; sh < M.ns; ++sh)
        if (M.shape_body[sh] < 0 && M.shape_type[sh] == MR_SHAPE_PLANE) {
            P.ground_height = M.shape_position[sh].z;  // a static shape's position is in world coordinates
            break;
        }
    P.default_q = reinterpret_cast<const float*>(base + at_default);
    P.limit_lower = reinterpret_cast<const float*>(base + at_lower);
    P.limit_upper = reinterpret_cast<const float*>(base + at_upper);
    P.na = static_cast<int>(na);
    P.nobs = static_cast<int>(t.actor_count);
    P.nrewards = static_cast<int>(t.reward_count);
    P.nterminations = static_cast<int>(nterm);
    P.nrandom = static_cast<int>(t.randomization_count);
    P.ngroups = static_cast<int>(t.joint_group_count);
    P.history = static_cast<int>(t.action_history);
    P.frames = static_cast<int>(t.observation_history);
    P.max_observation_delay = static_cast<int>(std::min<std::uint32_t>(t.maximum_observation_delay, 8u));
    P.delay = static_cast<int>(std::min<std::uint32_t>(t.action_delay_steps, t.action_history - 2));
    P.max_episode_steps = static_cast<int>(t.maximum_episode_steps);
    P.nq = static_cast<int>(nq);
    P.nv = static_cast<int>(nv);
    P.fixed_root = M.floating ? 0 : 1;
    P.dt = h.config.control_timestep_seconds;
    P.base_height = t.base_height_target;
    P.gait_period = t.gait_period_seconds;
    P.standing_probability = t.standing_probability;
    P.duration_min = t.command_duration_seconds[0];
    P.duration_max = t.command_duration_seconds[1];
    for (int k = 0; k < 3; ++k) {
        P.root_reference[k] = t.root_reference[k];
        P.command_lower[k] = t.command_lower[k];
        P.command_upper[k] = t.command_upper[k];
        P.command_limit_lower[k] = t.command_limit_lower[k];
        P.command_limit_upper[k] = t.command_limit_upper[k];
        P.command_step[k] = t.command_band_step[k];
    }
    // The sampled band range: the configuration's override, else every band
    // (the dispatch's sampling lanes).
    P.bands = static_cast<int>(t.difficulty_band_count);
    P.band_exponent = t.band_sampling_exponent;
    P.band_min = h.config.override_difficulty_band_range ? static_cast<int>(std::min<std::uint32_t>(h.config.minimum_difficulty_band, 1023u)) : 0;
    P.band_max = h.config.override_difficulty_band_range && h.config.maximum_difficulty_band != MR_INVALID_INDEX
                     ? static_cast<int>(std::min<std::uint32_t>(h.config.maximum_difficulty_band, 1023u))
                     : -1;
    P.seed = h.seed;
    out->fingerprint = t.task_fingerprint;
    return out;
}

}  // namespace

MR_API int mr_task_rollout_load_policy_pack(MRTaskRolloutHandle* handle, const char* policy_pack_path) {
    return guarded([&] {
        if (!handle) throw std::invalid_argument("handle is null");
        if (!policy_pack_path || !policy_pack_path[0]) throw std::invalid_argument("PolicyPack path is empty");
        if (handle->scene) throw std::invalid_argument("pile and stack worlds take no actions; a policy cannot drive them");
        const numi::PolicyPackData pack = numi::read_policy_pack(policy_pack_path);
        // The artifact rules of the reference's compile step: an exact
        // semantic contract (so version-3 packs, which carry none, need the
        // reference's explicit migration first), shapes and values.
        numi::validate_policy_pack(pack);
        std::vector<MRPolicyDenseLayerC> layers;
        const MRPolicyPackC view = numi::policy_pack_view(pack, layers);
        check(numi::configure_policy_kernel(), "policy kernel attributes");
        std::unique_ptr<InstalledPolicy> compiled = compile_policy(*handle, view);
        compiled->fingerprint = numi::policy_pack_payload_hash(pack);
        // A failed load returns above and leaves the installed policy in place.
        drop_graphs(*handle);
        handle->policy = std::move(compiled);
        handle->have_policy_outputs = false;
    });
}

MR_API int mr_task_rollout_set_policy(MRTaskRolloutHandle* handle, const MRPolicyPackC* policy) {
    return guarded([&] {
        if (!handle) throw std::invalid_argument("handle is null");
        if (!policy) throw std::invalid_argument("task-rollout policy is null");
        if (handle->scene) throw std::invalid_argument("pile and stack worlds take no actions; a policy cannot drive them");
        check(numi::configure_policy_kernel(), "policy kernel attributes");
        std::unique_ptr<InstalledPolicy> compiled = compile_policy(*handle, *policy);
        compiled->fingerprint = numi::policy_pack_payload_hash(numi::policy_pack_from_c(*policy));
        // Captured graphs hold the previous policy's arena: drop them.
        drop_graphs(*handle);
        handle->policy = std::move(compiled);
        handle->have_policy_outputs = false;
    });
}

MR_API uint64_t mr_task_rollout_policy_revision(const MRTaskRolloutHandle* handle) {
    return handle && handle->policy ? handle->policy->revision : 0u;
}

MR_API int mr_task_rollout_clear_policy(MRTaskRolloutHandle* handle) {
    return guarded([&] {
        if (!handle) throw std::invalid_argument("handle is null");
        drop_graphs(*handle);
        handle->policy.reset();
        handle->have_policy_outputs = false;
    });
}

MR_API int mr_task_rollout_set_task(MRTaskRolloutHandle* handle, const MRTaskProgramC* program) {
    return guarded([&] {
        if (!handle) throw std::invalid_argument("handle is null");
        if (!program) throw std::invalid_argument("task program is null");
        MRTaskRolloutHandle& h = *handle;
        if (h.scene) throw std::invalid_argument("pile and stack worlds take no actions; a task cannot drive them");
        std::unique_ptr<InstalledTask> compiled = compile_task(h, *program);
        if (h.policy) {
            const int in = h.policy->params.actor[0].in;
            const int cin = h.policy->params.critic_layers ? h.policy->params.critic[0].in : 0;
            const int cwant = compiled->prog.ncritic ? compiled->prog.ncritic : compiled->prog.frames * compiled->prog.nobs;
            if (cin != 0 && cin != cwant)
                throw std::invalid_argument("the installed policy's critic takes " + std::to_string(cin) + " observations; the task's critic frame has " +
                                            std::to_string(cwant) + " (clear the policy first)");
            if (in != compiled->prog.frames * compiled->prog.nobs)
                throw std::invalid_argument("the installed policy takes " + std::to_string(in) + " observations; the task's actor history has " +
                                            std::to_string(compiled->prog.frames * compiled->prog.nobs) + " (clear the policy first)");
        }
        drop_graphs(h);
        const numi::TaskProgramDevice& P = compiled->prog;
        h.d_task_state.resize(h.envs);
        h.d_task_history.resize(static_cast<size_t>(h.envs) * P.history * P.na);
        h.d_task_previous.resize(static_cast<size_t>(h.envs) * 2 * P.na);
        h.d_task_frame.resize(static_cast<size_t>(h.envs) * P.frames * P.nobs);
        if (P.ncritic) h.d_task_critic.resize(static_cast<size_t>(h.envs) * P.ncritic);
        h.d_task_targets.resize(static_cast<size_t>(h.envs) * P.na);
        h.d_task_air.resize(static_cast<size_t>(h.envs) * numi::kTaskMaxGroups);
        check(cudaMemsetAsync(h.d_task_history.ptr, 0, h.d_task_history.count * sizeof(float), h.stream), "clear task history");
        check(cudaMemsetAsync(h.d_task_previous.ptr, 0, h.d_task_previous.count * sizeof(float), h.stream), "clear task history");
        h.task = std::move(compiled);
        h.clear_task_state();
        h.stats_layout.actor_observation_count = static_cast<std::uint32_t>(P.frames * P.nobs);
        h.stats_layout.critic_observation_count = static_cast<std::uint32_t>(P.ncritic ? P.ncritic : P.frames * P.nobs);
        h.stats_layout.maximum_episode_steps = static_cast<std::uint32_t>(P.max_episode_steps);
        h.stats_layout.task_fingerprint = h.task->fingerprint;
        h.last_steps = 0;
        h.have_final_q = false;
    });
}

MR_API int mr_task_rollout_clear_task(MRTaskRolloutHandle* handle) {
    return guarded([&] {
        if (!handle) throw std::invalid_argument("handle is null");
        MRTaskRolloutHandle& h = *handle;
        if (!h.task) return;
        if (h.policy && h.policy->params.actor[0].in != static_cast<int>(h.model.world.nq + h.model.world.nv))
            throw std::invalid_argument("the installed policy reads the task's actor frame; clear the policy first");
        drop_graphs(h);
        h.task.reset();
        h.transition_steps = 0;
        h.have_host_transitions = false;
        // The sampled reset states come back (the task wrote its own).
        check(cudaMemcpyAsync(h.d_reset_q.ptr, h.reset_q.data(), h.reset_q.size() * sizeof(float), cudaMemcpyHostToDevice, h.stream),
              "upload reset q");
        check(cudaMemcpyAsync(h.d_reset_v.ptr, h.reset_v.data(), h.reset_v.size() * sizeof(float), cudaMemcpyHostToDevice, h.stream),
              "upload reset v");
        check(cudaStreamSynchronize(h.stream), "clear task");
        h.stats_layout.actor_observation_count = h.model.world.nq + h.model.world.nv;
        h.stats_layout.critic_observation_count = h.model.world.nq + h.model.world.nv;
        h.stats_layout.maximum_episode_steps = 0;
        h.stats_layout.task_fingerprint = 0;
        h.last_steps = 0;
        h.have_final_q = false;
    });
}

MR_API const MRTaskTransitionC* mr_task_rollout_transitions(const MRTaskRolloutHandle* handle) {
    return handle && handle->have_host_transitions ? handle->h_transitions.ptr : nullptr;
}

MR_API uint64_t mr_task_rollout_device_transitions(const MRTaskRolloutHandle* handle) {
    return handle && handle->task && handle->transition_steps ? reinterpret_cast<uint64_t>(handle->d_transitions.ptr) : 0u;
}

MR_API int mr_task_rollout_write_policy_rollout_pack(const MRTaskRolloutHandle* handle, const MRPolicyRolloutBatchC* batch,
                                                     const char* batch_id, const char* output_path) {
    return guarded([&] {
        if (!handle) throw std::invalid_argument("handle is null");
        if (!batch || !batch_id || !batch_id[0] || !output_path || !output_path[0])
            throw std::invalid_argument("policy rollout batch, identity, and output path are required.");
        const MRTaskRolloutHandle& h = *handle;
        if (!h.policy) throw std::invalid_argument("a compiled policy must be installed before publishing a rollout pack");
        MRPolicyRolloutPackC c{};
        c.id = batch_id;
        // Without a task program the world's fingerprint names what was rolled out.
        c.task_fingerprint = h.task && h.task->fingerprint ? h.task->fingerprint : h.stats_layout.world_fingerprint;
        c.policy_fingerprint = h.policy->fingerprint;
        c.policy_revision = h.policy->revision;
        c.environment_count = h.envs;
        c.actor_observation_count = h.observation_count();
        c.critic_observation_count = h.observation_count();
        c.action_count = h.model.world.action_count;
        c.motion_feature_count = 0;
        c.batch = batch;
        numi::write_policy_rollout_pack(numi::policy_rollout_pack_from_c(c), output_path);
    });
}

MR_API int mr_task_rollout_copy_transitions(const MRTaskRolloutHandle* handle, MRTaskTransitionC* output, size_t count) {
    return guarded([&] {
        if (!handle) throw std::invalid_argument("handle is null");
        const MRTaskRolloutHandle& h = *handle;
        if (!h.task || h.transition_steps == 0) throw std::invalid_argument("no transitions: install a task and advance first");
        if (count > static_cast<size_t>(h.transition_steps) * h.envs)
            throw std::invalid_argument("count exceeds the last advance's steps x environments");
        if (count != 0 && !output) throw std::invalid_argument("output is null");
        check(cudaStreamSynchronize(h.stream), "transitions");
        if (count) check(cudaMemcpy(output, h.d_transitions.ptr, count * sizeof(MRTaskTransitionC), cudaMemcpyDeviceToHost), "transitions D2H");
    });
}

MR_API const float* mr_task_rollout_policy_latents(const MRTaskRolloutHandle* handle) {
    return handle && handle->have_policy_outputs ? handle->h_latents.ptr : nullptr;
}
MR_API const float* mr_task_rollout_policy_log_probabilities(const MRTaskRolloutHandle* handle) {
    return handle && handle->have_policy_outputs ? handle->h_log_prob.ptr : nullptr;
}
MR_API const float* mr_task_rollout_policy_values(const MRTaskRolloutHandle* handle) {
    return handle && handle->have_policy_outputs ? handle->h_values.ptr : nullptr;
}
MR_API const float* mr_task_rollout_bootstrap_policy_values(const MRTaskRolloutHandle* handle) {
    return handle && handle->have_policy_outputs ? handle->h_values.ptr + static_cast<size_t>(handle->last_policy_steps) * handle->envs
                                                 : nullptr;
}

MR_API int mr_task_rollout_set_precision(MRTaskRolloutHandle* handle, uint32_t mode) {
    return guarded([&] {
        if (!handle) throw std::invalid_argument("handle is null");
        if (mode != MR_PRECISION_FP32 && mode != MR_PRECISION_FP64_ARTICULATED_INERTIA && mode != MR_PRECISION_COMPENSATED)
            throw std::invalid_argument("unknown precision mode " + std::to_string(mode));
        // Compensation terms accumulated before a change of mode do not
        // describe the state the new mode starts from.
        if (mode != handle->precision) handle->clear_compensation();
        handle->precision = mode;
    });
}

MR_API int mr_task_rollout_set_solver(MRTaskRolloutHandle* handle, uint32_t solver, const MRQualitySolverConfigC* quality) {
    return guarded([&] {
        if (!handle) throw std::invalid_argument("handle is null");
        if (solver != MR_SOLVER_TEMPORAL_CONE && solver != MR_SOLVER_QUALITY_NEWTON)
            throw std::invalid_argument("solver " + std::to_string(solver) +
                                        " is not available: MR_SOLVER_TEMPORAL_CONE or MR_SOLVER_QUALITY_NEWTON");
        const bool q = solver == MR_SOLVER_QUALITY_NEWTON;
        if (q && handle->scene)
            throw std::invalid_argument("MR_SOLVER_QUALITY_NEWTON runs articulated contact worlds; pile and stack worlds take temporalCone");
        if (q && !handle->contact) throw std::invalid_argument("MR_SOLVER_QUALITY_NEWTON needs a contact world");
        if (q && handle->resident_warps_per_sm_q[0] == 0)
            throw std::invalid_argument("the quality solver's workspace does not fit this model's shared-memory budget");
        const numi::QualityConfig cfg = q ? numi::rt::quality_config(quality) : numi::QualityConfig{};
        // Captured graphs hold the previous solver's kernel and settings.
        drop_graphs(*handle);
        handle->quality = q;
        handle->quality_cfg = cfg;
    });
}

MR_API int mr_task_rollout_quality_diagnostics(const MRTaskRolloutHandle* handle, MRQualityDiagnosticsC* out) {
    return guarded([&] {
        if (!handle || !out) throw std::invalid_argument("handle or output is null");
        *out = handle->last_quality;
    });
}

MR_API int mr_task_rollout_advance(MRTaskRolloutHandle* handle, const float* normalized_actions, size_t normalized_action_count,
                                   const uint32_t* reset_masks, size_t reset_mask_count, uint32_t control_step_count,
                                   uint64_t policy_revision, uint32_t evaluate_final_policy, MRTaskRolloutAdvanceC* advance) {
    return guarded([&] {
        if (!handle) throw std::invalid_argument("handle is null");
        if (!advance) throw std::invalid_argument("advance output is null");
        MRTaskRolloutHandle& h = *handle;
        if (control_step_count == 0) throw std::invalid_argument("control_step_count must be positive");
        h.prepare_policy(control_step_count, policy_revision, evaluate_final_policy);
        const bool driven = h.policy != nullptr;
        const size_t na = h.model.world.action_count;
        const size_t expected = static_cast<size_t>(control_step_count) * h.envs * na;
        // With a native policy the advance takes no action stream (c_api.cpp:3783-3795).
        const size_t action_span = driven ? 0 : expected;
        if (normalized_action_count != action_span || (action_span > 0 && normalized_actions == nullptr))
            throw std::invalid_argument("normalized_action_count must equal " +
                                        std::string(driven ? "0 with a native policy installed" :
                                                             "control_step_count * environment_count * action_count (" +
                                                                 std::to_string(expected) + ")"));
        const size_t mask_expected = static_cast<size_t>(control_step_count) * h.envs;
        if (reset_mask_count != 0 && (reset_mask_count != mask_expected || reset_masks == nullptr))
            throw std::invalid_argument("reset_mask_count must be 0 or control_step_count * environment_count");
        const auto wall0 = std::chrono::steady_clock::now();
        // Caller spans are copied to the device straight from the caller's
        // memory; the call returns only after the copies have finished, so
        // nothing of them is kept past return.
        h.d_actions.resize(expected);
        const bool masks = reset_mask_count != 0;
        if (masks) h.d_masks.resize(mask_expected);
        const size_t nobs = h.observation_count();
        h.prepare_task(control_step_count);
        h.d_status.resize(mask_expected);
        h.d_contacts.resize(mask_expected);
        h.h_status.resize(mask_expected);
        h.h_contacts.resize(mask_expected);
        if (h.readback) {
            h.d_obs.resize(mask_expected * nobs);
            h.h_obs.resize(mask_expected * nobs);
            h.h_final_q.resize(static_cast<size_t>(h.envs) * h.model.world.nq);
        }
        cudaStream_t s = h.stream;
        check(cudaEventRecord(h.ev_start, s), "event");
        if (action_span > 0)
            check(cudaMemcpyAsync(h.d_actions.ptr, normalized_actions, expected * sizeof(float), cudaMemcpyHostToDevice, s),
                  "actions H2D");
        if (masks) check(cudaMemcpyAsync(h.d_masks.ptr, reset_masks, mask_expected * sizeof(uint32_t), cudaMemcpyHostToDevice, s), "masks H2D");
        h.run(control_step_count, h.d_actions.ptr, masks ? h.d_masks.ptr : nullptr, h.readback ? h.d_obs.ptr : nullptr,
              h.d_status.ptr, h.d_contacts.ptr, s, h.readback ? h.h_obs.ptr : nullptr);
        check(cudaMemcpyAsync(h.h_status.ptr, h.d_status.ptr, mask_expected * sizeof(uint32_t), cudaMemcpyDeviceToHost, s), "status D2H");
        check(cudaMemcpyAsync(h.h_contacts.ptr, h.d_contacts.ptr, mask_expected * sizeof(uint32_t), cudaMemcpyDeviceToHost, s), "contacts D2H");
        check(cudaMemcpyAsync(h.h_stats.ptr, h.d_stats.ptr, numi::kStatCount * sizeof(uint32_t), cudaMemcpyDeviceToHost, s), "stats D2H");
        h.read_policy_outputs(control_step_count, s);
        if (h.task) {
            h.h_transitions.resize(mask_expected);
            check(cudaMemcpyAsync(h.h_transitions.ptr, h.d_transitions.ptr, mask_expected * sizeof(MRTaskTransitionC),
                                  cudaMemcpyDeviceToHost, s), "transitions D2H");
        }
        if (h.readback) {
            check(cudaMemcpyAsync(h.h_final_q.ptr, h.d_q.ptr, static_cast<size_t>(h.envs) * h.model.world.nq * sizeof(float),
                                  cudaMemcpyDeviceToHost, s), "final q D2H");
        }
        check(cudaEventRecord(h.ev_stop, s), "event");
        check(cudaStreamSynchronize(s), "advance");
        float gpu_ms = 0.0f;
        check(cudaEventElapsedTime(&gpu_ms, h.ev_start, h.ev_stop), "elapsed");
        const double wall_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - wall0).count();
        h.last_steps = control_step_count;
        h.have_final_q = h.readback;
        h.have_host_transitions = h.task != nullptr;
        h.fill_advance(control_step_count, h.h_status.ptr, h.h_stats.ptr, advance, gpu_ms, wall_ms);
        // The reference reports failed environments in the counters and also
        // as an error return (src/c_api.cpp:3983-3988).
        if (advance->failed_environment_steps != 0)
            throw std::runtime_error("environment " + std::to_string(advance->first_failing_environment) + " failed at control step " +
                                     std::to_string(advance->first_failing_control_step) + " with status " +
                                     std::to_string(advance->first_gpu_status_code));
    });
}

MR_API int mr_task_rollout_advance_device(MRTaskRolloutHandle* handle, const float* device_actions, const uint32_t* device_reset_masks,
                                          uint32_t control_step_count, float* device_observations, uint32_t* device_status_codes,
                                          uint64_t cuda_stream, MRTaskRolloutAdvanceC* advance) {
    return guarded([&] {
        if (!handle) throw std::invalid_argument("handle is null");
        if (control_step_count == 0) throw std::invalid_argument("control_step_count must be positive");
        MRTaskRolloutHandle& h = *handle;
        h.prepare_policy(control_step_count, 0, 0);
        if (h.policy) {
            // The policy writes the actions; device_actions is not read.
            h.d_actions.resize(static_cast<size_t>(control_step_count) * h.envs * h.model.world.action_count);
            device_actions = h.d_actions.ptr;
        }
        if (!device_actions && handle->model.world.action_count > 0) throw std::invalid_argument("device_actions is null");
        // The horizon runs (and is graph-captured) on the rollout's own
        // stream; events order it after the caller's prior work and the
        // caller's later work after it.  cuda_stream 0 is the legacy default
        // stream, which a non-blocking stream does not otherwise wait for.
        cudaStream_t caller = reinterpret_cast<cudaStream_t>(cuda_stream);
        cudaStream_t s = h.stream;
        check(cudaEventRecord(h.ev_in, caller), "event");
        check(cudaStreamWaitEvent(s, h.ev_in, 0), "stream wait");
        const size_t cells = static_cast<size_t>(control_step_count) * h.envs;
        h.prepare_task(control_step_count);
        std::uint32_t* status = device_status_codes;
        if (!status) {
            h.d_status.resize(cells);
            status = h.d_status.ptr;
        }
        h.d_contacts.resize(cells);
        const auto wall0 = std::chrono::steady_clock::now();
        if (advance) check(cudaEventRecord(h.ev_start, s), "event");
        h.run(control_step_count, device_actions, device_reset_masks, device_observations, status, h.d_contacts.ptr, s);
        h.read_policy_outputs(control_step_count, s);
        check(cudaEventRecord(h.ev_out, s), "event");
        check(cudaStreamWaitEvent(caller, h.ev_out, 0), "stream wait");
        if (advance) {
            check(cudaMemcpyAsync(h.h_stats.ptr, h.d_stats.ptr, numi::kStatCount * sizeof(uint32_t), cudaMemcpyDeviceToHost, s), "stats D2H");
            check(cudaEventRecord(h.ev_stop, s), "event");
            check(cudaStreamSynchronize(s), "advance");
            float gpu_ms = 0.0f;
            check(cudaEventElapsedTime(&gpu_ms, h.ev_start, h.ev_stop), "elapsed");
            const double wall_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - wall0).count();
            h.fill_advance(control_step_count, nullptr, h.h_stats.ptr, advance, gpu_ms, wall_ms);
        }
        h.have_final_q = false;
        h.last_steps = 0;
    });
}

MR_API MRTaskRolloutLayoutC mr_task_rollout_layout(const MRTaskRolloutHandle* handle) {
    if (!handle) {
        numi::rt::set_last_error("handle is null");
        return MRTaskRolloutLayoutC{};
    }
    return handle->stats_layout;
}

MR_API const char* mr_task_rollout_device_name(const MRTaskRolloutHandle* handle) {
    return handle ? handle->device_name.c_str() : nullptr;
}

MR_API const uint32_t* mr_task_rollout_status_codes(const MRTaskRolloutHandle* handle) {
    return handle && handle->last_steps ? handle->h_status.ptr : nullptr;
}

MR_API const uint32_t* mr_task_rollout_active_contacts(const MRTaskRolloutHandle* handle) {
    return handle && handle->last_steps ? handle->h_contacts.ptr : nullptr;
}

MR_API const float* mr_task_rollout_actor_observations(const MRTaskRolloutHandle* handle) {
    return handle && handle->have_final_q ? handle->h_obs.ptr : nullptr;
}

MR_API const float* mr_task_rollout_final_q(const MRTaskRolloutHandle* handle) {
    return handle && handle->have_final_q ? handle->h_final_q.ptr : nullptr;
}

MR_API int mr_task_rollout_copy_final_scene_states(const MRTaskRolloutHandle* handle, float* output, size_t output_count) {
    return guarded([&] {
        if (!handle) throw std::invalid_argument("handle is null");
        if (output_count != 0 && output == nullptr) throw std::invalid_argument("output is null");
        const MRTaskRolloutHandle& h = *handle;
        if (!h.scene) {
            if (output_count != 0) throw std::invalid_argument("this world has no scene bodies; output_count must be 0");
            return;
        }
        const size_t n = h.model.scene_bodies;
        const size_t need = static_cast<size_t>(h.envs) * n * 13;
        if (output_count != need) throw std::invalid_argument("output_count must be envs x scene bodies x 13 = " + std::to_string(need));
        check(cudaStreamSynchronize(h.stream), "sync");
        std::vector<float> q(static_cast<size_t>(h.envs) * n * 7), v(static_cast<size_t>(h.envs) * n * 6);
        check(cudaMemcpy(q.data(), h.d_q.ptr, q.size() * sizeof(float), cudaMemcpyDeviceToHost), "q D2H");
        check(cudaMemcpy(v.data(), h.d_v.ptr, v.size() * sizeof(float), cudaMemcpyDeviceToHost), "v D2H");
        // Packed [env][body][position xyz, orientation xyzw, linear xyz, angular xyz].
        for (size_t i = 0; i < static_cast<size_t>(h.envs) * n; ++i) {
            std::memcpy(output + i * 13, q.data() + i * 7, 7 * sizeof(float));
            std::memcpy(output + i * 13 + 7, v.data() + i * 6, 6 * sizeof(float));
        }
    });
}

// The hull vertex table of a model view (MRModelViewC::hull_vertices).
static void copy_hull_vertices(const numi::CompiledModel& m, MRModelViewC* view) {
    const std::uint32_t count = static_cast<std::uint32_t>(m.hull_vertices.size() / 4);
    view->hull_vertex_count = count;
    if (view->hull_vertices && count > 0) {
        if (view->hull_vertex_capacity < count)
            throw std::invalid_argument("hull_vertices holds " + std::to_string(view->hull_vertex_capacity) + " vertices; the model has " +
                                        std::to_string(count));
        std::memcpy(view->hull_vertices, m.hull_vertices.data(), m.hull_vertices.size() * sizeof(float));
    }
}

MR_API int mr_task_rollout_copy_model(const MRTaskRolloutHandle* handle, MRModelViewC* view) {
    return guarded([&] {
        if (!handle || !view) throw std::invalid_argument("handle or view is null");
        const numi::CompiledModel& m = handle->model;
        view->world = m.world;
        if (view->joints) std::memcpy(view->joints, m.joints.data(), m.joints.size() * sizeof(MRModelJointC));
        if (view->bodies) std::memcpy(view->bodies, m.bodies.data(), m.bodies.size() * sizeof(MRModelBodyC));
        if (view->dofs) std::memcpy(view->dofs, m.dofs.data(), m.dofs.size() * sizeof(MRModelDofC));
        if (view->shapes) std::memcpy(view->shapes, m.shapes.data(), m.shapes.size() * sizeof(MRModelShapeC));
        if (view->materials) std::memcpy(view->materials, m.materials.data(), m.materials.size() * sizeof(MRModelMaterialC));
        if (view->pairs) std::memcpy(view->pairs, m.pairs.data(), m.pairs.size() * sizeof(MRModelPairC));
        copy_hull_vertices(m, view);
    });
}

static numi::CompiledModel compile_source(uint32_t source, uint64_t seed) {
    switch (source) {
        case MR_RUN_SOURCE_SYNTHETIC_CHAIN7: return numi::build_chain7(seed);
        case MR_RUN_SOURCE_SYNTHETIC_TREE29: return numi::build_tree29(seed);
        case MR_RUN_SOURCE_SYNTHETIC_PILE: return numi::build_pile(seed);
        case MR_RUN_SOURCE_SYNTHETIC_CYLINDER_PILE: return numi::build_pile(seed, 0, true);
        case MR_RUN_SOURCE_SYNTHETIC_PILE_GJK: return numi::build_pile(seed, 0, false, true);
        case MR_RUN_SOURCE_SYNTHETIC_HULL_PILE: return numi::build_pile(seed, 0, false, false, true);
        case MR_RUN_SOURCE_SYNTHETIC_STACK: return numi::build_stack(seed);
        default: throw std::invalid_argument("unsupported synthetic source " + std::to_string(source));
    }
}

MR_API int mr_compile_synthetic_model(uint32_t source, uint64_t seed, MRModelViewC* view) {
    return guarded([&] {
        if (!view) throw std::invalid_argument("view is null");
        const numi::CompiledModel m = compile_source(source, seed);
        view->world = m.world;
        if (view->joints) std::memcpy(view->joints, m.joints.data(), m.joints.size() * sizeof(MRModelJointC));
        if (view->bodies) std::memcpy(view->bodies, m.bodies.data(), m.bodies.size() * sizeof(MRModelBodyC));
        if (view->dofs) std::memcpy(view->dofs, m.dofs.data(), m.dofs.size() * sizeof(MRModelDofC));
        if (view->shapes) std::memcpy(view->shapes, m.shapes.data(), m.shapes.size() * sizeof(MRModelShapeC));
        if (view->materials) std::memcpy(view->materials, m.materials.data(), m.materials.size() * sizeof(MRModelMaterialC));
        if (view->pairs) std::memcpy(view->pairs, m.pairs.data(), m.pairs.size() * sizeof(MRModelPairC));
        copy_hull_vertices(m, view);
    });
}

MR_API int mr_sample_synthetic_reset(uint32_t source, uint64_t model_seed, uint64_t reset_seed, uint32_t env_begin,
                                     uint32_t env_count, float* q, float* v, float* friction_scale) {
    return guarded([&] {
        if (!q || !v || !friction_scale) throw std::invalid_argument("outputs must be non-null");
        const numi::CompiledModel m = compile_source(source, model_seed);
        for (uint32_t i = 0; i < env_count; ++i)
            numi::sample_reset_state(m, reset_seed, env_begin + i, q + static_cast<size_t>(i) * m.world.nq,
                                     v + static_cast<size_t>(i) * m.world.nv, friction_scale + i);
    });
}

MR_API int mr_task_rollout_copy_environment_parameters(const MRTaskRolloutHandle* handle, float* friction_scale) {
    return guarded([&] {
        if (!handle || !friction_scale) throw std::invalid_argument("handle or output is null");
        std::memcpy(friction_scale, handle->friction.data(), handle->friction.size() * sizeof(float));
    });
}

MR_API uint32_t mr_task_rollout_environment_chains(const MRTaskRolloutHandle* handle) {
    if (!handle) return 0u;
    if (handle->scene) return 1u;
    return static_cast<uint32_t>(std::min<std::uint32_t>(static_cast<std::uint32_t>(handle->chains), handle->envs));
}

MR_API int mr_task_rollout_launch_shape(const MRTaskRolloutHandle* handle, uint32_t* warps_per_block,
                                        uint32_t* resident_warps_per_sm) {
    return guarded([&] {
        if (!handle) throw std::invalid_argument("handle is null");
        if (warps_per_block) *warps_per_block = handle->scene ? 1u : static_cast<uint32_t>(handle->step_warps_per_block());
        if (resident_warps_per_sm) *resident_warps_per_sm = handle->scene ? 0u : static_cast<uint32_t>(handle->step_resident_warps_per_sm());
    });
}

MR_API int mr_task_rollout_copy_state(const MRTaskRolloutHandle* handle, float* q, float* v, MRManifoldC* manifolds) {
    return guarded([&] {
        if (!handle) throw std::invalid_argument("handle is null");
        const MRTaskRolloutHandle& h = *handle;
        check(cudaStreamSynchronize(h.stream), "sync");
        if (q) check(cudaMemcpy(q, h.d_q.ptr, static_cast<size_t>(h.envs) * h.model.world.nq * sizeof(float), cudaMemcpyDeviceToHost), "q D2H");
        if (v) check(cudaMemcpy(v, h.d_v.ptr, static_cast<size_t>(h.envs) * h.model.world.nv * sizeof(float), cudaMemcpyDeviceToHost), "v D2H");
        if (manifolds && h.contact)
            check(cudaMemcpy(manifolds, h.d_manifolds.ptr, static_cast<size_t>(h.envs) * h.manifold_words() * sizeof(float),
                             cudaMemcpyDeviceToHost), "manifolds D2H");
    });
}

MR_API int mr_task_rollout_set_audit(MRTaskRolloutHandle* handle, uint32_t enabled) {
    return guarded([&] {
        if (!handle) throw std::invalid_argument("handle is null");
        MRTaskRolloutHandle& h = *handle;
        const bool on = enabled != 0;
        check(cudaStreamSynchronize(h.stream), "sync");
        if (on) {
            h.d_audit.resize(static_cast<size_t>(h.envs) * numi::kAuditWords);
            check(cudaMemset(h.d_audit.ptr, 0, h.d_audit.count * sizeof(double)), "clear audit");
        }
        if (on != h.audit) drop_graphs(h);  // captured launches hold the previous setting
        h.audit = on;
    });
}

MR_API int mr_task_rollout_copy_audit(const MRTaskRolloutHandle* handle, double* records, size_t count) {
    return guarded([&] {
        if (!handle || !records) throw std::invalid_argument("handle and records must be non-null");
        const MRTaskRolloutHandle& h = *handle;
        if (!h.audit) throw std::invalid_argument("the audit is not enabled (mr_task_rollout_set_audit)");
        const size_t need = static_cast<size_t>(h.envs) * numi::kAuditWords;
        if (count != need) throw std::invalid_argument("records must hold environments x 12 = " + std::to_string(need) + " doubles");
        check(cudaStreamSynchronize(h.stream), "sync");
        check(cudaMemcpy(records, h.d_audit.ptr, need * sizeof(double), cudaMemcpyDeviceToHost), "audit D2H");
    });
}

MR_API int mr_task_rollout_set_island_labels(MRTaskRolloutHandle* handle, uint32_t enabled) {
    return guarded([&] {
        if (!handle) throw std::invalid_argument("handle is null");
        MRTaskRolloutHandle& h = *handle;
        if (!h.scene) throw std::invalid_argument("island labels are recorded for free-body (scene) worlds only");
        const bool on = enabled != 0;
        if (on == h.island_labels) return;
        check(cudaStreamSynchronize(h.stream), "sync");
        if (on) {
            h.d_island_labels.resize(static_cast<size_t>(h.envs) * numi::kSceneMaxBodies);
            check(cudaMemset(h.d_island_labels.ptr, 0xff, h.d_island_labels.count), "clear island labels");
        }
        h.island_labels = on;
        drop_graphs(h);  // captured launches hold the previous setting
    });
}

MR_API int mr_task_rollout_copy_island_labels(const MRTaskRolloutHandle* handle, uint8_t* labels, size_t count) {
    return guarded([&] {
        if (!handle || !labels) throw std::invalid_argument("handle and labels must be non-null");
        const MRTaskRolloutHandle& h = *handle;
        if (!h.island_labels) throw std::invalid_argument("island labels are not enabled (mr_task_rollout_set_island_labels)");
        const size_t need = static_cast<size_t>(h.envs) * numi::kSceneMaxBodies;
        if (count != need) throw std::invalid_argument("labels must hold environments x " + std::to_string(numi::kSceneMaxBodies) +
                                                       " = " + std::to_string(need) + " entries");
        check(cudaStreamSynchronize(h.stream), "sync");
        check(cudaMemcpy(labels, h.d_island_labels.ptr, need, cudaMemcpyDeviceToHost), "island labels D2H");
    });
}

MR_API int mr_task_rollout_set_state(MRTaskRolloutHandle* handle, const float* q, const float* v, const MRManifoldC* manifolds,
                                     uint32_t as_reset_state) {
    return guarded([&] {
        if (!handle || !q || !v) throw std::invalid_argument("handle, q and v must be non-null");
        MRTaskRolloutHandle& h = *handle;
        const size_t nq = static_cast<size_t>(h.envs) * h.model.world.nq;
        const size_t nv = static_cast<size_t>(h.envs) * h.model.world.nv;
        check(cudaStreamSynchronize(h.stream), "sync");
        check(cudaMemcpy(h.d_q.ptr, q, nq * sizeof(float), cudaMemcpyHostToDevice), "q H2D");
        check(cudaMemcpy(h.d_v.ptr, v, nv * sizeof(float), cudaMemcpyHostToDevice), "v H2D");
        h.clear_compensation();
        if (h.contact) {
            if (manifolds)
                check(cudaMemcpy(h.d_manifolds.ptr, manifolds, static_cast<size_t>(h.envs) * h.manifold_words() * sizeof(float),
                                 cudaMemcpyHostToDevice), "manifolds H2D");
            else
                check(cudaMemset(h.d_manifolds.ptr, 0, h.d_manifolds.count * sizeof(float)), "clear manifolds");
        }
        if (h.scene) {
            // Scene tables: leading slots with a non-zero point count are live.
            std::vector<std::uint32_t> counts(h.envs, 0u);
            if (manifolds) {
                const float* words = reinterpret_cast<const float*>(manifolds);
                for (std::uint32_t e = 0; e < h.envs; ++e) {
                    const float* t = words + static_cast<size_t>(e) * h.manifold_words();
                    std::uint32_t c = 0;
                    while (c < static_cast<std::uint32_t>(numi::kSceneManifolds)) {
                        std::uint32_t pts;
                        std::memcpy(&pts, t + c * numi::kSceneSlotWords + 7, sizeof(pts));
                        if (pts == 0u) break;
                        ++c;
                    }
                    counts[e] = c;
                }
            }
            check(cudaMemcpy(h.d_mcount.ptr, counts.data(), counts.size() * sizeof(std::uint32_t), cudaMemcpyHostToDevice),
                  "manifold counts H2D");
        }
        if (as_reset_state) {
            h.reset_q.assign(q, q + nq);
            h.reset_v.assign(v, v + nv);
            check(cudaMemcpy(h.d_reset_q.ptr, q, nq * sizeof(float), cudaMemcpyHostToDevice), "reset q H2D");
            check(cudaMemcpy(h.d_reset_v.ptr, v, nv * sizeof(float), cudaMemcpyHostToDevice), "reset v H2D");
        }
    });
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Heterogeneous batch: several rollouts advanced by one persistent launch per
// control step (mix.h, mix_step.cu).
// ---------------------------------------------------------------------------

struct MRBatchHandle {
    std::vector<MRTaskRolloutHandle*> worlds;
    int device = 0;
    int sms = 0;
    cudaStream_t stream = nullptr, side = nullptr;
    cudaEvent_t ev_in = nullptr, ev_out = nullptr, ev_fork = nullptr, ev_join = nullptr, ev_a = nullptr, ev_b = nullptr;
    // Shared memory per warp (floats) and resident CTAs per SM of each
    // kernel family (numi::MixFamily: fused, articulated, scene).
    int smem_floats[3] = {0, 0, 0};
    int blocks_per_sm[3] = {0, 0, 0};
    int warps_per_block = 2;            // fused and articulated kernels; the scene kernel runs one warp per CTA
    std::uint32_t mode = MR_BATCH_LAUNCH_FUSED;
    std::uint32_t order = MR_BATCH_ORDER_LONGEST_FIRST;
    bool tuned = false;
    float tuned_step_ms = 0.0f;
    std::vector<float> cost;            // per world: latency of one item (ms), the claim-order key
    // Claim orders: every item (fused) and each family's items.
    std::vector<std::uint32_t> items[3];
    DeviceBuffer<std::uint32_t> d_items[3];
    DeviceBuffer<numi::MixWorld> d_worlds;  // [steps][worlds] of the cached advance
    DeviceBuffer<unsigned> d_next;          // one queue counter per family
    PinnedBuffer<numi::MixWorld> h_worlds;
    std::vector<numi::MixWorld> cached;     // descriptors behind d_worlds and the graph
    cudaGraphExec_t graph = nullptr;
    std::uint32_t graph_steps = 0;

    ~MRBatchHandle() {
        if (graph) cudaGraphExecDestroy(graph);
        for (cudaEvent_t e : {ev_in, ev_out, ev_fork, ev_join, ev_a, ev_b})
            if (e) cudaEventDestroy(e);
        for (cudaStream_t st : {stream, side})
            if (st) cudaStreamDestroy(st);
    }

    // Some free-body world has support-mapped (GJK / EPA) pairs: its family
    // runs the kernel instance with that narrowphase, and only per family.
    bool convex = false;
    int kernel_of(int family) const { return family == numi::kMixFamilyScene && convex ? numi::kMixFamilySceneConvex : family; }
    int wpb(int family) const { return family == numi::kMixFamilyScene ? 1 : warps_per_block; }
    int grid(int family) const { return std::max(1, blocks_per_sm[family]) * sms; }
    std::uint32_t item_count() const { return static_cast<std::uint32_t>(items[numi::kMixFamilyFused].size()); }
    bool is_scene(std::uint32_t w) const { return worlds[w]->scene; }

    void plan_launch() {
        for (int f = 0; f < 3; ++f) {
            blocks_per_sm[f] = 0;
            if (!smem_floats[f]) continue;
            const size_t smem = static_cast<size_t>(smem_floats[f]) * sizeof(float) * wpb(f);
            check(numi::mix_occupancy(kernel_of(f), wpb(f), smem, &blocks_per_sm[f]), "batch occupancy");
            if (blocks_per_sm[f] < 1) throw std::runtime_error("the batch's per-warp shared memory does not fit one CTA on this device");
        }
    }

    // Claim orders: the longest item first (cost, then world, then slot) or
    // round robin over the worlds; the family lists keep the same order.
    void order_items() {
        for (auto& l : items) l.clear();
        std::vector<std::uint32_t> world_order(worlds.size());
        for (std::uint32_t w = 0; w < worlds.size(); ++w) world_order[w] = w;
        std::stable_sort(world_order.begin(), world_order.end(), [&](std::uint32_t a, std::uint32_t b) { return cost[a] > cost[b]; });
        auto push = [&](std::uint32_t w, std::uint32_t e) {
            const std::uint32_t code = (w << numi::kMixWorldShift) | e;
            items[numi::kMixFamilyFused].push_back(code);
            items[is_scene(w) ? numi::kMixFamilyScene : numi::kMixFamilyArticulated].push_back(code);
        };
        if (order == MR_BATCH_ORDER_LONGEST_FIRST) {
            for (std::uint32_t w : world_order)
                for (std::uint32_t e = 0; e < worlds[w]->envs; ++e) push(w, e);
        } else {
            std::uint32_t most = 0;
            for (auto* h : worlds) most = std::max(most, h->envs);
            for (std::uint32_t e = 0; e < most; ++e)
                for (std::uint32_t w : world_order)
                    if (e < worlds[w]->envs) push(w, e);
        }
        for (int f = 0; f < 3; ++f) {
            d_items[f].resize(items[f].size());
            if (!items[f].empty())
                check(cudaMemcpy(d_items[f].ptr, items[f].data(), items[f].size() * sizeof(std::uint32_t), cudaMemcpyHostToDevice),
                      "batch items H2D");
        }
    }

    void drop_graph() {
        if (graph) cudaGraphExecDestroy(graph);
        graph = nullptr;
        cached.clear();
    }

    void launch(int family, std::uint32_t steps, const std::uint32_t* item_list, int n, cudaStream_t s) {
        check(numi::launch_mix_horizon(kernel_of(family), d_worlds.ptr, static_cast<int>(worlds.size()), static_cast<int>(steps), item_list, n,
                                       d_next.ptr + family, wpb(family), smem_floats[family], grid(family), s),
              "batch horizon launch");
    }

    // Enqueues `steps` control steps of every item on `s`: one fused launch,
    // or one launch per family (the scene family on the side stream).
    void enqueue(std::uint32_t steps, cudaStream_t s) {
        check(cudaMemsetAsync(d_next.ptr, 0, 3 * sizeof(unsigned), s), "batch queue reset");
        if (mode == MR_BATCH_LAUNCH_FUSED) {
            launch(numi::kMixFamilyFused, steps, d_items[0].ptr, static_cast<int>(items[0].size()), s);
            return;
        }
        const bool art = !items[numi::kMixFamilyArticulated].empty(), scn = !items[numi::kMixFamilyScene].empty();
        if (art && scn) {
            check(cudaEventRecord(ev_fork, s), "event");
            check(cudaStreamWaitEvent(side, ev_fork, 0), "stream wait");
        }
        if (art)
            launch(numi::kMixFamilyArticulated, steps, d_items[1].ptr, static_cast<int>(items[1].size()), s);
        if (scn)
            launch(numi::kMixFamilyScene, steps, d_items[2].ptr, static_cast<int>(items[2].size()), art ? side : s);
        if (art && scn) {
            check(cudaEventRecord(ev_join, side), "event");
            check(cudaStreamWaitEvent(s, ev_join, 0), "stream wait");
        }
    }

    void clear_stats(cudaStream_t s) {
        for (auto* h : worlds) {
            check(cudaMemsetAsync(h->d_stats.ptr, 0, numi::kStatCount * sizeof(std::uint32_t), s), "clear stats");
            check(cudaMemsetAsync(h->d_stats.ptr + numi::kStatFirstFailEnv, 0xff, sizeof(std::uint32_t), s), "clear stats");
        }
    }

    // Uploads the descriptors of an advance (when they differ from the
    // cached ones, which also drops the captured graph).
    void upload(std::uint32_t steps, const float* const* actions, const std::uint32_t* const* masks, std::uint32_t* const* status) {
        std::vector<numi::MixWorld> desc(static_cast<size_t>(steps) * worlds.size());
        for (std::uint32_t k = 0; k < steps; ++k)
            for (size_t w = 0; w < worlds.size(); ++w)
                desc[k * worlds.size() + w] = worlds[w]->mix_world(k, actions ? actions[w] : nullptr, masks ? masks[w] : nullptr,
                                                                   status ? status[w] : nullptr);
        if (desc.size() == cached.size() && std::memcmp(desc.data(), cached.data(), desc.size() * sizeof(numi::MixWorld)) == 0) return;
        drop_graph();
        d_worlds.resize(desc.size());
        d_next.resize(3);
        h_worlds.resize(desc.size());
        std::memcpy(h_worlds.ptr, desc.data(), desc.size() * sizeof(numi::MixWorld));
        check(cudaMemcpyAsync(d_worlds.ptr, h_worlds.ptr, desc.size() * sizeof(numi::MixWorld), cudaMemcpyHostToDevice, stream),
              "batch descriptors H2D");
        check(cudaStreamSynchronize(stream), "batch descriptors H2D");
        cached = std::move(desc);
    }

    void run(std::uint32_t steps, cudaStream_t caller) {
        check(cudaEventRecord(ev_in, caller), "event");
        check(cudaStreamWaitEvent(stream, ev_in, 0), "stream wait");
        if (!graph || graph_steps != steps) {
            if (graph) cudaGraphExecDestroy(graph);
            graph = nullptr;
            cudaGraph_t g = nullptr;
            check(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal), "begin capture");
            try {
                clear_stats(stream);
                enqueue(steps, stream);
            } catch (...) {
                cudaStreamEndCapture(stream, &g);
                if (g) cudaGraphDestroy(g);
                throw;
            }
            check(cudaStreamEndCapture(stream, &g), "end capture");
            cudaGraphExec_t exec = nullptr;
            const cudaError_t e = cudaGraphInstantiate(&exec, g, 0);
            cudaGraphDestroy(g);
            check(e, "graph instantiate");
            graph = exec;
            graph_steps = steps;
        }
        check(cudaGraphLaunch(graph, stream), "graph launch");
        check(cudaEventRecord(ev_out, stream), "event");
        check(cudaStreamWaitEvent(caller, ev_out, 0), "stream wait");
    }

    // Device state of every world (q, v, manifolds, manifold counts): the
    // tuner steps the worlds and puts them back.
    struct Snapshot {
        std::vector<std::unique_ptr<DeviceBuffer<float>>> f;
        std::vector<std::unique_ptr<DeviceBuffer<std::uint32_t>>> u;
    };
    void snapshot(Snapshot& snap, bool take) {
        check(cudaStreamSynchronize(stream), "sync");
        size_t fi = 0, ui = 0;
        for (auto* h : worlds) {
            for (DeviceBuffer<float>* b : {&h->d_q, &h->d_v, &h->d_manifolds}) {
                if (take) {
                    snap.f.push_back(std::make_unique<DeviceBuffer<float>>());
                    if (b->count) snap.f.back()->resize(b->count);
                }
                DeviceBuffer<float>& d = *snap.f[fi++];
                if (b->count)
                    check(cudaMemcpy(take ? d.ptr : b->ptr, take ? b->ptr : d.ptr, b->count * sizeof(float), cudaMemcpyDeviceToDevice),
                          "batch snapshot");
            }
            if (h->d_mcount.count) {
                if (take) {
                    snap.u.push_back(std::make_unique<DeviceBuffer<std::uint32_t>>());
                    snap.u.back()->resize(h->d_mcount.count);
                }
                DeviceBuffer<std::uint32_t>& d = *snap.u[ui++];
                check(cudaMemcpy(take ? d.ptr : h->d_mcount.ptr, take ? h->d_mcount.ptr : d.ptr,
                                 h->d_mcount.count * sizeof(std::uint32_t), cudaMemcpyDeviceToDevice), "batch snapshot");
            }
        }
    }

    template <typename F>
    float best_ms(int repeats, F&& body) {
        float best = 1e30f;
        for (int r = 0; r < repeats + 1; ++r) {
            check(cudaEventRecord(ev_a, stream), "event");
            body();
            check(cudaEventRecord(ev_b, stream), "event");
            check(cudaEventSynchronize(ev_b), "sync");
            float ms = 0.0f;
            check(cudaEventElapsedTime(&ms, ev_a, ev_b), "elapsed");
            if (r > 0) best = std::min(best, ms);  // the first run warms up
        }
        return best;
    }

    // Autotuner: calibrates each world's item latency (its environments
    // alone, one control step, in its family's kernel), orders the queues by
    // it, then times the whole batch for every (launch mode, warps per CTA,
    // claim order) candidate and keeps the fastest.  The worlds' state is
    // put back afterwards.
    void tune(std::uint32_t steps, const float* const* actions) {
        Snapshot snap;
        snapshot(snap, true);
        upload(steps, actions, nullptr, nullptr);
        plan_launch();
        for (std::uint32_t w = 0; w < worlds.size(); ++w) {
            std::vector<std::uint32_t> own;
            for (std::uint32_t e = 0; e < worlds[w]->envs; ++e) own.push_back((w << numi::kMixWorldShift) | e);
            DeviceBuffer<std::uint32_t> d_own;
            d_own.resize(own.size());
            check(cudaMemcpy(d_own.ptr, own.data(), own.size() * sizeof(std::uint32_t), cudaMemcpyHostToDevice), "tuner items");
            const int family = is_scene(w) ? numi::kMixFamilyScene : numi::kMixFamilyArticulated;
            const float ms = best_ms(2, [&] {
                check(cudaMemsetAsync(d_next.ptr, 0, 3 * sizeof(unsigned), stream), "batch queue reset");
                launch(family, 1, d_own.ptr, static_cast<int>(own.size()), stream);
            });
            const double slots = static_cast<double>(grid(family)) * wpb(family);
            cost[w] = static_cast<float>(ms / std::max(1.0, std::ceil(static_cast<double>(own.size()) / slots)));
        }
        float best = 1e30f;
        int best_wpb = warps_per_block;
        std::uint32_t best_order = order, best_mode = mode;
        for (const std::uint32_t md : {std::uint32_t(MR_BATCH_LAUNCH_FUSED), std::uint32_t(MR_BATCH_LAUNCH_PER_FAMILY)})
            for (const std::uint32_t ord : {std::uint32_t(MR_BATCH_ORDER_LONGEST_FIRST), std::uint32_t(MR_BATCH_ORDER_ROUND_ROBIN)})
                for (const int wp : {1, 2, 4}) {
                    if (convex && md == MR_BATCH_LAUNCH_FUSED) continue;
                    mode = md;
                    order = ord;
                    warps_per_block = wp;
                    try {
                        plan_launch();
                    } catch (const std::exception&) {
                        continue;
                    }
                    order_items();
                    const float ms = best_ms(2, [&] { enqueue(steps, stream); }) / static_cast<float>(steps);
                    if (ms < best) {
                        best = ms;
                        best_wpb = wp;
                        best_order = ord;
                        best_mode = md;
                    }
                }
        warps_per_block = best_wpb;
        order = best_order;
        mode = best_mode;
        plan_launch();
        order_items();
        tuned = true;
        tuned_step_ms = best;
        drop_graph();
        snapshot(snap, false);
    }
};

extern "C" {

MR_API MRBatchHandle* mr_create_batch(MRTaskRolloutHandle* const* rollouts, size_t count) {
    std::unique_ptr<MRBatchHandle> b;
    const int rc = guarded([&] {
        if (!rollouts || count == 0) throw std::invalid_argument("rollouts must hold at least one handle");
        if (count > static_cast<size_t>(numi::kMixMaxWorlds))
            throw std::invalid_argument("a batch holds at most " + std::to_string(numi::kMixMaxWorlds) + " rollouts");
        b = std::make_unique<MRBatchHandle>();
        check(cudaGetDevice(&b->device), "cudaGetDevice");
        cudaDeviceProp prop{};
        check(cudaGetDeviceProperties(&prop, b->device), "cudaGetDeviceProperties");
        b->sms = prop.multiProcessorCount;
        int floats_art = 0, floats_scene = 0;
        for (size_t i = 0; i < count; ++i) {
            MRTaskRolloutHandle* h = rollouts[i];
            if (!h) throw std::invalid_argument("rollout " + std::to_string(i) + " is null");
            if (h->device != b->device) throw std::invalid_argument("every rollout of a batch must live on the current device");
            if (h->precision != MR_PRECISION_FP32) throw std::invalid_argument("batched rollouts run in FP32 precision only");
            if (h->quality) throw std::invalid_argument("batched rollouts run the temporalCone solver only");
            if (h->policy) throw std::invalid_argument("batched rollouts take their actions from the caller (no native policy)");
            if (h->task) throw std::invalid_argument("batched rollouts step raw drive targets (no task program)");
            if (h->scene && h->smodel.support_mapped) b->convex = true;
            if (h->envs > numi::kMixEnvMask) throw std::invalid_argument("a batched rollout holds at most 2^24 - 1 environments");
            for (size_t j = 0; j < i; ++j)
                if (rollouts[j] == h) throw std::invalid_argument("a rollout appears twice in the batch");
            if (h->scene) floats_scene = numi::mix_scene_warp_floats();
            else floats_art = std::max(floats_art, numi::mix_articulated_warp_floats(h->layout));
            b->worlds.push_back(h);
            // First estimate of an item's latency (ms), replaced by the tuner.
            const double bodies = h->scene ? h->smodel.nb : h->dmodel.nb;
            b->cost.push_back(static_cast<float>(h->scene ? 0.02 * std::pow(bodies, 1.2) : (h->contact ? 0.4 : 0.02 * bodies)));
        }
        auto round4 = [](int x) { return (x + 3) & ~3; };
        b->smem_floats[numi::kMixFamilyArticulated] = floats_art ? round4(floats_art) : 0;
        b->smem_floats[numi::kMixFamilyScene] = floats_scene ? round4(floats_scene) : 0;
        b->smem_floats[numi::kMixFamilyFused] = round4(std::max(floats_art, floats_scene));
        for (int f = 0; f < 3; ++f) {
            if (!b->smem_floats[f]) continue;
            const size_t bytes = std::min(static_cast<size_t>(b->smem_floats[f]) * sizeof(float) * 4,
                                          static_cast<size_t>(prop.sharedMemPerBlockOptin));
            check(numi::configure_mix_kernel(b->kernel_of(f), bytes), "batch kernel attributes");
        }
        if (b->convex) b->mode = MR_BATCH_LAUNCH_PER_FAMILY;
        for (cudaStream_t* st : {&b->stream, &b->side}) check(cudaStreamCreateWithFlags(st, cudaStreamNonBlocking), "stream");
        for (cudaEvent_t* e : {&b->ev_in, &b->ev_out, &b->ev_fork, &b->ev_join}) check(cudaEventCreateWithFlags(e, cudaEventDisableTiming), "event");
        for (cudaEvent_t* e : {&b->ev_a, &b->ev_b}) check(cudaEventCreate(e), "event");
        b->plan_launch();
        b->order_items();
    });
    return rc == 0 ? b.release() : nullptr;
}

MR_API void mr_batch_destroy(MRBatchHandle* batch) {
    if (!batch) return;
    cudaStreamSynchronize(batch->stream);
    delete batch;
}

MR_API int mr_batch_advance(MRBatchHandle* batch, uint32_t control_step_count, const float* const* actions,
                            const uint32_t* const* reset_masks, uint32_t* const* status_codes, uint64_t cuda_stream) {
    return guarded([&] {
        if (!batch) throw std::invalid_argument("batch is null");
        if (control_step_count == 0) throw std::invalid_argument("control_step_count must be positive");
        for (size_t w = 0; w < batch->worlds.size(); ++w)
            if (batch->worlds[w]->model.world.action_count > 0 && (!actions || !actions[w]))
                throw std::invalid_argument("rollout " + std::to_string(w) + " takes actions: actions[" + std::to_string(w) +
                                            "] must be a device buffer [steps][envs][actions]");
        batch->upload(control_step_count, actions, reset_masks, status_codes);
        batch->run(control_step_count, reinterpret_cast<cudaStream_t>(cuda_stream));
    });
}

MR_API int mr_batch_tune(MRBatchHandle* batch, uint32_t control_step_count, const float* const* actions) {
    return guarded([&] {
        if (!batch) throw std::invalid_argument("batch is null");
        if (control_step_count == 0) throw std::invalid_argument("control_step_count must be positive");
        for (size_t w = 0; w < batch->worlds.size(); ++w)
            if (batch->worlds[w]->model.world.action_count > 0 && (!actions || !actions[w]))
                throw std::invalid_argument("the tuner steps every rollout: actions[" + std::to_string(w) + "] is required");
        batch->tune(control_step_count, actions);
    });
}

MR_API int mr_batch_launch_shape(const MRBatchHandle* batch, MRBatchLaunchShapeC* out) {
    return guarded([&] {
        if (!batch || !out) throw std::invalid_argument("batch and out must be non-null");
        *out = MRBatchLaunchShapeC{};
        out->worlds = static_cast<uint32_t>(batch->worlds.size());
        out->items = batch->item_count();
        const int main_family = batch->mode == MR_BATCH_LAUNCH_FUSED ? numi::kMixFamilyFused : numi::kMixFamilyArticulated;
        out->warps_per_block = static_cast<uint32_t>(batch->warps_per_block);
        out->blocks = static_cast<uint32_t>(batch->grid(main_family));
        out->resident_warps_per_sm = static_cast<uint32_t>(batch->blocks_per_sm[main_family] * batch->warps_per_block);
        out->shared_bytes_per_warp = static_cast<uint32_t>(batch->smem_floats[main_family] * sizeof(float));
        out->scene_blocks = batch->mode == MR_BATCH_LAUNCH_PER_FAMILY ? static_cast<uint32_t>(batch->grid(numi::kMixFamilyScene)) : 0u;
        out->scene_resident_warps_per_sm =
            batch->mode == MR_BATCH_LAUNCH_PER_FAMILY ? static_cast<uint32_t>(batch->blocks_per_sm[numi::kMixFamilyScene]) : 0u;
        out->mode = batch->mode;
        out->order = batch->order;
        out->tuned = batch->tuned ? 1u : 0u;
        out->tuned_step_milliseconds = batch->tuned_step_ms;
    });
}

MR_API int mr_batch_world_costs(const MRBatchHandle* batch, float* milliseconds, size_t count) {
    return guarded([&] {
        if (!batch || !milliseconds) throw std::invalid_argument("batch and milliseconds must be non-null");
        if (count != batch->worlds.size()) throw std::invalid_argument("milliseconds must hold one entry per rollout of the batch");
        for (size_t w = 0; w < count; ++w) milliseconds[w] = batch->cost[w];
    });
}

}  // extern "C"
