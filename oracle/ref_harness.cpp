// ORACLE (reference side) — test infrastructure only.
//
// A C-ABI harness, written for this project, over numi-lab's own FP64 CPU
// core (compiled out of tree from its sources by oracle/Makefile into
// oracle/_ref/).  It rebuilds a reference EngineModel from the records this
// library exports (MRModel*C, include/numi_b200.h) and exposes:
//   - computeArticulatedForwardDynamics / MassMatrix / PointJacobians
//     (src/core/ArticulatedDynamics.cpp:2010, 2241, and friends),
//   - integrateArticulatedState (ArticulatedDynamics.cpp:2333),
//   - solveReferenceConicProblem (src/core/ReferenceConicSolver.cpp:182),
//   - stepControlledArticulatedWorldCpu (src/core/ArticulatedWorld.cpp:1232)
//     and a multi-threaded timing loop over it (the CPU baseline),
//   - collideCpuReference (src/core/Collision.cpp:2959) over a free-body
//     pile: raw contacts and persistent manifolds of every touching pair,
//   - writePolicyPack / readPolicyPack (src/core/LearningPacks.cpp:2428-2470).
// Implicit PD drives are expressed for the reference the way its own GPU
// ABA does: armature raised by h kd + h^2 kp and the PD law evaluated as an
// effort (ArticulatedABA.metal:301-326, MetalWorld.metal:280-370).
#include "metalrobo/ArticulatedDynamics.hpp"
#include "metalrobo/ArticulatedWorld.hpp"
#include "metalrobo/Collision.hpp"
#include "metalrobo/ConstraintIR.hpp"
#include "metalrobo/ConstraintSolver.hpp"
#include "metalrobo/RigidBodyWorld.hpp"
#include "metalrobo/EngineModel.hpp"
#include "metalrobo/LearningPacks.hpp"
#include "metalrobo/MetalWorldCapacity.hpp"
#include "metalrobo/TaskProgram.hpp"
#include "metalrobo/PolicyProgram.hpp"
#include "metalrobo/QualityContactSolver.hpp"
#include "metalrobo/ReferenceConicSolver.hpp"

#define NUMI_B200_OMIT_SHARED_ENUMS
#include "numi_b200.h"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <string>
#include <thread>
#include <vector>

using namespace metalrobo;

namespace {

mr_float4 f4(const float* p) { return mr_float4{p[0], p[1], p[2], p[3]}; }
mr_float4 f4(double x, double y, double z, double w) {
    return mr_float4{static_cast<float>(x), static_cast<float>(y), static_cast<float>(z), static_cast<float>(w)};
}

void write_error(char* err, size_t len, const std::string& msg) {
    if (err && len) {
        std::strncpy(err, msg.c_str(), len - 1);
        err[len - 1] = 0;
    }
}

}  // namespace

struct RefModel {
    EngineModel model;
    std::vector<MRBodyStateGPU> env_bodies;
    std::vector<MRShapeGPU> env_shapes;
    MRModelWorldC world{};
    std::vector<MRModelDofC> dofs;
    std::vector<std::uint32_t> action_dof;
    double h = 0.0;
    bool implicit = false;
    // Record shape index -> collider index of the reference's combined
    // shape list (articulated shapes first, then the environment's).
    std::vector<std::uint32_t> collider_of_shape;
    std::vector<std::uint32_t> shape_of_collider;
};

extern "C" {

__attribute__((visibility("default"))) RefModel* ref_model_create(
    const MRModelWorldC* world, const MRModelJointC* joints, const MRModelBodyC* bodies, const MRModelDofC* dofs,
    const MRModelShapeC* shapes, const MRModelMaterialC* materials, double h, double friction, char* err, size_t err_len) {
    try {
        auto r = std::make_unique<RefModel>();
        r->world = *world;
        r->h = h;
        r->implicit = world->actuation_mode == MR_ACTUATION_IMPLICIT_POSITION;
        r->dofs.assign(dofs, dofs + world->nv);
        std::uint32_t na = 0;
        while (na < world->body_count && bodies[na].articulated) ++na;
        EngineModel& m = r->model;
        m.name = "numi_b200_export";
        m.world.abiVersion = MR_ENGINE_ABI_VERSION;
        m.world.bodyCount = na;
        m.world.articulationCount = 1;
        m.world.jointCount = world->joint_count;
        m.world.nq = world->nq;
        m.world.nv = world->nv;
        m.world.pairCapacity = 2048;
        m.world.contactCapacity = 1024;
        m.world.constraintCapacity = 2048;
        m.world.islandCapacity = 32;
        m.world.solverType = MR_SOLVER_QUALITY_NEWTON;
        m.world.frictionConeType = MR_FRICTION_CONE_ELLIPTIC;
        m.world.gravityAndTimestep = f4(world->gravity[0], world->gravity[1], world->gravity[2], h);
        m.world.solverScales = f4(world->solver_scales);
        MRArticulationGPU art{};
        art.rootBody = 0;
        art.rootType = world->root_type;
        art.firstBody = 0;
        art.bodyCount = na;
        art.firstJoint = 0;
        art.jointCount = world->joint_count;
        art.qOffset = 0;
        art.nq = world->nq;
        art.vOffset = 0;
        art.nv = world->nv;
        m.articulations.push_back(art);
        for (std::uint32_t b = 0; b < na; ++b) {
            const MRModelBodyC& s = bodies[b];
            MRBodyPropertiesGPU p{};
            p.articulationIndex = 0;
            p.parentBody = s.parent_body;
            p.inboundJoint = s.inbound_joint;
            p.motionType = MR_MOTION_DYNAMIC;
            p.massAndInverseMass = f4(s.mass_inverse_mass[0], 1.0 / s.mass_inverse_mass[0], 0.0, 0.0);
            p.centerOfMass = f4(0, 0, 0, 0);
            p.inertiaRow0 = f4(s.inertia[0][0], s.inertia[0][1], s.inertia[0][2], 0.0);
            p.inertiaRow1 = f4(s.inertia[1][0], s.inertia[1][1], s.inertia[1][2], 0.0);
            p.inertiaRow2 = f4(s.inertia[2][0], s.inertia[2][1], s.inertia[2][2], 0.0);
            // Inverse of the (diagonal-dominant) body inertia by cofactors.
            const double a = s.inertia[0][0], bq = s.inertia[0][1], c = s.inertia[0][2];
            const double d = s.inertia[1][1], e = s.inertia[1][2], f = s.inertia[2][2];
            const double c00 = d * f - e * e, c01 = c * e - bq * f, c02 = bq * e - c * d;
            const double det = a * c00 + bq * c01 + c * c02;
            const double c11 = a * f - c * c, c12 = bq * c - a * e, c22 = a * d - bq * bq;
            p.inverseInertiaRow0 = f4(c00 / det, c01 / det, c02 / det, 0.0);
            p.inverseInertiaRow1 = f4(c01 / det, c11 / det, c12 / det, 0.0);
            p.inverseInertiaRow2 = f4(c02 / det, c12 / det, c22 / det, 0.0);
            p.dampingAndSpeedLimits = f4(s.damping_speed);
            m.bodies.push_back(p);
        }
        for (std::uint32_t j = 0; j < world->joint_count; ++j) {
            const MRModelJointC& s = joints[j];
            MRJointDescriptorGPU d{};
            d.parentBody = s.parent_body;
            d.childBody = s.child_body;
            d.jointType = s.joint_type;
            d.flags = 0;
            const bool scalar = s.joint_type != MR_JOINT_FIXED;
            d.qOffset = scalar ? s.q_index : 0;
            d.nq = scalar ? 1 : 0;
            d.vOffset = scalar ? s.v_index : 0;
            d.nv = scalar ? 1 : 0;
            d.axis0 = f4(s.axis);
            d.parentAnchor = f4(s.parent_anchor);
            d.childAnchor = f4(s.child_anchor);
            d.parentRotation = f4(s.parent_rotation);
            d.childRotation = f4(s.child_rotation);
            m.joints.push_back(d);
        }
        for (std::uint32_t k = 0; k < world->nv; ++k) {
            const MRModelDofC& s = dofs[k];
            MRDofPropertiesGPU d{};
            d.articulationIndex = 0;
            d.jointIndex = s.joint_index;
            d.qIndex = s.q_index;
            d.vIndex = k;
            d.localDof = s.joint_index == MR_INVALID_INDEX ? k : 0;
            d.flags = s.flags;
            d.limits = f4(s.limits);
            double arm = s.drive[2];
            if (r->implicit && (s.flags & MR_DOF_FLAG_DRIVE)) arm += h * s.drive[1] + h * h * s.drive[0];
            d.drive = f4(s.drive[0], s.drive[1], arm, s.drive[3]);
            m.dofs.push_back(d);
            if ((s.flags & MR_DOF_FLAG_ACTUATED) && r->action_dof.size() < world->action_count) r->action_dof.push_back(k);
        }
        for (std::uint32_t i = 0; i < world->material_count; ++i) {
            MRMaterialGPU mt{};
            mt.friction = f4(materials[i].friction[0] * friction, materials[i].friction[1] * friction, materials[i].friction[2],
                             materials[i].friction[3]);
            mt.response = f4(materials[i].response);
            m.materials.push_back(mt);
        }
        m.world.materialCount = static_cast<mr_u32>(m.materials.size());
        for (std::uint32_t s = 0; s < world->shape_count; ++s) {
            const MRModelShapeC& src = shapes[s];
            MRShapeGPU sh{};
            sh.shapeType = src.shape_type;
            sh.materialIndex = src.material;
            sh.collisionGroup = src.collision_group;
            sh.collisionMask = src.collision_mask;
            sh.slotGeneration = 1;
            sh.localPosition = f4(src.local_position[0], src.local_position[1], src.local_position[2], 1.0);
            sh.localRotation = f4(src.local_rotation);
            sh.dimensions = f4(src.dimensions);
            sh.contactRestAndBoundingRadius = f4(src.contact_rest_bound);
            if (bodies[src.body].articulated) {
                sh.bodyIndex = src.body;
                m.shapes.push_back(sh);
            } else {
                const MRModelBodyC& gb = bodies[src.body];
                MRBodyStateGPU st{};
                st.position = f4(gb.static_pose[0], gb.static_pose[1], gb.static_pose[2], 0.0);
                st.orientation = f4(gb.static_pose + 4);
                st.linearVelocityAndInverseMass = f4(0, 0, 0, 0);
                st.flagsAndIndices[0] = MR_MOTION_STATIC;
                st.flagsAndIndices[1] = MR_INVALID_INDEX;
                st.flagsAndIndices[2] = MR_INVALID_INDEX;
                st.flagsAndIndices[3] = 0;
                sh.bodyIndex = static_cast<mr_u32>(r->env_bodies.size());
                r->env_bodies.push_back(st);
                r->env_shapes.push_back(sh);
            }
        }
        m.world.shapeCount = static_cast<mr_u32>(m.shapes.size());
        {
            std::uint32_t art = 0, env = 0;
            const std::uint32_t nart = static_cast<std::uint32_t>(m.shapes.size());
            r->collider_of_shape.resize(world->shape_count);
            r->shape_of_collider.resize(world->shape_count);
            for (std::uint32_t s2 = 0; s2 < world->shape_count; ++s2) {
                const std::uint32_t c = bodies[shapes[s2].body].articulated ? art++ : nart + env++;
                r->collider_of_shape[s2] = c;
                r->shape_of_collider[c] = s2;
            }
        }
        m.defaultQ.assign(world->nq, 0.0f);
        m.defaultV.assign(world->nv, 0.0f);
        if (world->root_type == MR_ROOT_FLOATING) m.defaultQ[6] = 1.0f;
        std::string reason;
        if (!m.valid(&reason)) {
            write_error(err, err_len, "reference EngineModel rejected: " + reason);
            return nullptr;
        }
        return r.release();
    } catch (const std::exception& e) {
        write_error(err, err_len, e.what());
        return nullptr;
    }
}

__attribute__((visibility("default"))) void ref_model_destroy(RefModel* r) { delete r; }

static ArticulatedDynamicsConfig dyn_config(const RefModel* r) {
    ArticulatedDynamicsConfig c{};
    c.gravity = {r->world.gravity[0], r->world.gravity[1], r->world.gravity[2]};
    c.timestep = r->h;
    c.applyBodyDamping = r->world.apply_body_damping != 0;
    return c;
}

__attribute__((visibility("default"))) int ref_forward_dynamics(RefModel* r, const double* q, const double* v, const double* tau,
                                                                double* qdd) {
    const std::uint32_t nq = r->world.nq, nv = r->world.nv;
    auto d = computeArticulatedForwardDynamics(r->model, 0, std::span<const double>(q, nq), std::span<const double>(v, nv),
                                               std::span<const double>(tau, nv), {}, std::span<double>(qdd, nv), dyn_config(r));
    return static_cast<int>(d.status);
}

__attribute__((visibility("default"))) int ref_mass_matrix(RefModel* r, const double* q, double* mass) {
    const std::uint32_t nq = r->world.nq, nv = r->world.nv;
    auto d = computeArticulatedMassMatrix(r->model, 0, std::span<const double>(q, nq), std::span<double>(mass, nv * nv), dyn_config(r));
    return static_cast<int>(d.status);
}

__attribute__((visibility("default"))) int ref_point_jacobian(RefModel* r, const double* q, uint32_t body, const double* local,
                                                              double* world_point, double* jacobian) {
    const std::uint32_t nq = r->world.nq, nv = r->world.nv;
    std::vector<double> v0(nv, 0.0);
    ArticulatedPointQuery query{};
    query.bodyIndex = body;
    query.localPoint = {local[0], local[1], local[2]};
    ArticulatedPointKinematics pk{};
    auto d = computeArticulatedPointJacobians(r->model, 0, std::span<const double>(q, nq), v0, std::span<const ArticulatedPointQuery>(&query, 1),
                                              std::span<ArticulatedPointKinematics>(&pk, 1), std::span<double>(jacobian, 3 * nv), dyn_config(r));
    world_point[0] = pk.position[0];
    world_point[1] = pk.position[1];
    world_point[2] = pk.position[2];
    return static_cast<int>(d.status);
}

__attribute__((visibility("default"))) int ref_integrate(RefModel* r, double* q, double* v, const double* tau) {
    const std::uint32_t nq = r->world.nq, nv = r->world.nv;
    auto d = integrateArticulatedState(r->model, 0, std::span<double>(q, nq), std::span<double>(v, nv), std::span<const double>(tau, nv),
                                       {}, dyn_config(r));
    return static_cast<int>(d.status);
}

// Converged FP64 conic contact solve on an explicit dense problem.
// inverse_mass nv x nv, free_velocity nv, jac (3n x nv: n, t, b rows per
// contact), mu n, target 3n; impulses 3n out, velocity nv out.
__attribute__((visibility("default"))) int ref_conic_solve(uint32_t nv, const double* inverse_mass, const double* free_velocity, uint32_t n,
                                                           const double* jac, const double* mu, const double* target, const double* reg,
                                                           double* impulses, double* velocity, double* cone_violation) {
    DenseConicProblem p{};
    p.nv = nv;
    p.inverseMass.assign(inverse_mass, inverse_mass + nv * nv);
    p.freeVelocity.assign(free_velocity, free_velocity + nv);
    for (uint32_t i = 0; i < n; ++i) {
        DenseContactBlock b{};
        b.normalJacobian.assign(jac + (3 * i + 0) * nv, jac + (3 * i + 1) * nv);
        b.tangentUJacobian.assign(jac + (3 * i + 1) * nv, jac + (3 * i + 2) * nv);
        b.tangentVJacobian.assign(jac + (3 * i + 2) * nv, jac + (3 * i + 3) * nv);
        b.targetVelocity = {target[3 * i], target[3 * i + 1], target[3 * i + 2]};
        b.regularization = {reg[3 * i], reg[3 * i + 1], reg[3 * i + 2]};
        b.warmImpulse = {0.0, 0.0, 0.0};
        b.friction = mu[i];
        p.contacts.push_back(b);
    }
    ReferenceConicSolverConfig cfg{};
    auto s = solveReferenceConicProblem(p, cfg);
    for (uint32_t i = 0; i < 3 * n && i < s.impulses.size(); ++i) impulses[i] = s.impulses[i];
    for (uint32_t i = 0; i < nv && i < s.velocity.size(); ++i) velocity[i] = s.velocity[i];
    if (cone_violation) *cone_violation = s.maximumConeViolation;
    return static_cast<int>(s.code);
}

// Converged quality solve of the same dense problem: the reference's
// globalized semismooth Newton (solveQualityContactProblem,
// src/core/QualityContactSolver.cpp:1480) with its default configuration.
// certificates[8]: scaled KKT certificate, scaled natural residual, primal
// and dual cone violation, conic complementarity, complementarity gap,
// objective, normal-impulse violation.  Returns the status code.
__attribute__((visibility("default"))) int ref_quality_solve(uint32_t nv, const double* inverse_mass, const double* free_velocity, uint32_t n,
                                                             const double* jac, const double* mu, const double* target, const double* reg,
                                                             double* impulses, double* velocity, double* certificates,
                                                             uint32_t* iterations) {
    DenseConicProblem p{};
    p.nv = nv;
    p.inverseMass.assign(inverse_mass, inverse_mass + nv * nv);
    p.freeVelocity.assign(free_velocity, free_velocity + nv);
    for (uint32_t i = 0; i < n; ++i) {
        DenseContactBlock b{};
        b.normalJacobian.assign(jac + (3 * i + 0) * nv, jac + (3 * i + 1) * nv);
        b.tangentUJacobian.assign(jac + (3 * i + 1) * nv, jac + (3 * i + 2) * nv);
        b.tangentVJacobian.assign(jac + (3 * i + 2) * nv, jac + (3 * i + 3) * nv);
        b.targetVelocity = {target[3 * i], target[3 * i + 1], target[3 * i + 2]};
        b.regularization = {reg[3 * i], reg[3 * i + 1], reg[3 * i + 2]};
        b.warmImpulse = {0.0, 0.0, 0.0};
        b.friction = mu[i];
        p.contacts.push_back(b);
    }
    QualityContactSolverConfig cfg{};
    const QualityContactSolution s = solveQualityContactProblem(p, cfg);
    for (uint32_t i = 0; i < 3 * n && i < s.impulses.size(); ++i) impulses[i] = s.impulses[i];
    for (uint32_t i = 0; i < nv && i < s.velocity.size(); ++i) velocity[i] = s.velocity[i];
    if (certificates) {
        certificates[0] = s.scaledKktCertificate;
        certificates[1] = s.scaledNaturalResidual;
        certificates[2] = s.maximumPrimalConeViolation;
        certificates[3] = s.maximumDualConeViolation;
        certificates[4] = s.maximumConicComplementarityResidual;
        certificates[5] = s.complementarityGap;
        certificates[6] = s.objective;
        certificates[7] = s.maximumNormalImpulseViolation;
    }
    if (iterations) *iterations = s.iterations;
    return static_cast<int>(s.code);
}

// Implicit-drive efforts as the reference GPU prepares them (the CPU world
// receives them as effort commands together with the raised armature).
static void drive_efforts(const RefModel* r, const double* q, const double* v, const float* actions, double* tau) {
    const std::uint32_t nv = r->world.nv;
    std::vector<double> tgt(nv, 0.0);
    for (size_t a = 0; a < r->action_dof.size(); ++a) tgt[r->action_dof[a]] = actions[a];
    for (std::uint32_t k = 0; k < nv; ++k) {
        const MRModelDofC& d = r->dofs[k];
        double command = tgt[k];
        if (r->implicit) {
            command = 0.0;
            if ((d.flags & MR_DOF_FLAG_DRIVE) && d.q_index != MR_INVALID_INDEX) {
                double target = tgt[k];
                if (d.flags & MR_DOF_FLAG_POSITION_LIMIT) target = std::min<double>(std::max<double>(target, d.limits[0]), d.limits[1]);
                command = d.drive[0] * (target - q[d.q_index] - r->h * v[k]) - d.drive[1] * v[k];
                if ((d.flags & MR_DOF_FLAG_EFFORT_LIMIT) && d.limits[3] > 0.0f)
                    command = std::min<double>(std::max<double>(command, -d.limits[3]), d.limits[3]);
            }
        }
        const double stall = ((d.flags & MR_DOF_FLAG_EFFORT_LIMIT) && d.limits[3] > 0.0f) ? d.limits[3] : std::numeric_limits<float>::max();
        const double env = std::min<double>(d.limits[3], stall);
        tau[k] = std::min(std::max(command, -env), env);
    }
}

// World-step configuration: one timestep shared by dynamics, constraint
// evaluation and joint limits (ArticulatedWorld.cpp:480-520 rejects a
// mismatch), the evaluation slop / depenetration speed of the world.
static ArticulatedWorldConfig world_config(const RefModel* r, int solver) {
    ArticulatedWorldConfig cfg{};
    cfg.dynamics = dyn_config(r);
    cfg.constraintEvaluation.timestep = r->h;
    cfg.jointLimits.timestep = r->h;
    cfg.constraintEvaluation.penetrationSlop = r->world.solver_scales[3];
    cfg.constraintEvaluation.maximumDepenetrationVelocity = r->world.solver_scales[2];
    cfg.solverType = solver == 0 ? MR_SOLVER_REFERENCE_FP64 : MR_SOLVER_QUALITY_NEWTON;
    return cfg;
}

// One transactional world step with diagnostics: returns the step status
// code and writes the failing stage (ArticulatedWorldFailure) and contact
// count.
__attribute__((visibility("default"))) int ref_world_step_once(RefModel* r, double* q, double* v, const float* actions, int solver,
                                                               uint32_t* failure, uint32_t* contacts) {
    const std::uint32_t nq = r->world.nq, nv = r->world.nv;
    const ArticulatedWorldConfig cfg = world_config(r, solver);
    std::vector<double> tau(nv);
    std::vector<ArticulatedDofCommand> commands(nv);
    drive_efforts(r, q, v, actions, tau.data());
    for (std::uint32_t k = 0; k < nv; ++k) {
        if (r->dofs[k].flags & MR_DOF_FLAG_ACTUATED) {
            commands[k].mode = ArticulatedActuationMode::effort;
            commands[k].feedForward = tau[k];
        }
    }
    static thread_local ArticulatedWorldCache cache{};
    auto d = stepControlledArticulatedWorldCpu(r->model, 0, std::span<double>(q, nq), std::span<double>(v, nv), commands, {},
                                               r->env_bodies, r->env_shapes, cfg, cache);
    if (failure) *failure = static_cast<uint32_t>(d.failure);
    if (contacts) *contacts = d.contactCount;
    return static_cast<int>(d.code);
}

// Runs `steps` control steps x `substeps` physics steps for `envs`
// environments with `threads` std::threads (static env partition) and
// returns elapsed wall seconds.  Contact worlds use the reference's
// transactional CPU world step with its quality (default) or FP64
// reference-conic solver; free-motion worlds use integrateArticulatedState.
// q/v are updated in place; failed steps are counted.
// `models` holds one model per environment (they differ only in their
// material friction: each environment's friction scale), all of one world.
__attribute__((visibility("default"))) double ref_run_envs(RefModel* const* models, uint32_t envs, double* q, double* v,
                                                           const float* actions, uint32_t steps, uint32_t substeps, uint32_t threads,
                                                           int solver, uint64_t* failed_steps) {
    const RefModel* r0 = models[0];
    const std::uint32_t nq = r0->world.nq, nv = r0->world.nv, na = r0->world.action_count;
    const bool contact = !r0->env_shapes.empty();
    std::atomic<std::uint64_t> failed{0};
    auto worker = [&](std::uint32_t begin, std::uint32_t end) {
        std::vector<double> tau(nv);
        std::vector<ArticulatedDofCommand> commands(nv);
        for (std::uint32_t e = begin; e < end; ++e) {
            RefModel* r = models[e];
            const ArticulatedWorldConfig cfg = world_config(r, solver);
            ArticulatedWorldCache cache{};
            double* qe = q + static_cast<size_t>(e) * nq;
            double* ve = v + static_cast<size_t>(e) * nv;
            for (std::uint32_t s = 0; s < steps; ++s) {
                const float* act = actions + (static_cast<size_t>(s) * envs + e) * na;
                for (std::uint32_t sub = 0; sub < substeps; ++sub) {
                    drive_efforts(r, qe, ve, act, tau.data());
                    bool ok = true;
                    if (contact) {
                        for (std::uint32_t k = 0; k < nv; ++k) {
                            commands[k] = ArticulatedDofCommand{};
                            if (r->dofs[k].flags & MR_DOF_FLAG_ACTUATED) {
                                commands[k].mode = ArticulatedActuationMode::effort;
                                commands[k].feedForward = tau[k];
                            }
                        }
                        auto d = stepControlledArticulatedWorldCpu(r->model, 0, std::span<double>(qe, nq), std::span<double>(ve, nv), commands, {},
                                                                   r->env_bodies, r->env_shapes, cfg, cache);
                        ok = d.succeeded();
                    } else {
                        auto d = integrateArticulatedState(r->model, 0, std::span<double>(qe, nq), std::span<double>(ve, nv), tau, {}, cfg.dynamics);
                        ok = d.succeeded();
                    }
                    if (!ok) {
                        failed.fetch_add(1);
                        break;
                    }
                }
            }
        }
    };
    const auto t0 = std::chrono::steady_clock::now();
    threads = std::max<std::uint32_t>(1, std::min(threads, envs));
    std::vector<std::thread> pool;
    for (std::uint32_t t = 0; t < threads; ++t) {
        const std::uint32_t b = static_cast<std::uint32_t>(static_cast<std::uint64_t>(envs) * t / threads);
        const std::uint32_t e = static_cast<std::uint32_t>(static_cast<std::uint64_t>(envs) * (t + 1) / threads);
        pool.emplace_back(worker, b, e);
    }
    for (auto& th : pool) th.join();
    const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (failed_steps) *failed_steps = failed.load();
    return secs;
}

// All environments share model `r` (one friction scale).
__attribute__((visibility("default"))) double ref_run(RefModel* r, uint32_t envs, double* q, double* v, const float* actions,
                                                      uint32_t steps, uint32_t substeps, uint32_t threads, int solver,
                                                      uint64_t* failed_steps) {
    std::vector<RefModel*> models(envs, r);
    return ref_run_envs(models.data(), envs, q, v, actions, steps, substeps, threads, solver, failed_steps);
}

// Persistent manifolds of one articulated environment across calls.
struct RefContactCache {
    PersistentManifoldCache manifolds;
};

__attribute__((visibility("default"))) RefContactCache* ref_contact_cache_create() { return new RefContactCache(); }
__attribute__((visibility("default"))) void ref_contact_cache_destroy(RefContactCache* c) { delete c; }

// The reference CPU world step's contact front end, up to the evaluated
// ConstraintIR, at configuration q with free velocity vf
// (ArticulatedWorld.cpp:573-800): link kinematics, projected body states,
// collideCpuReference with the parent/child-link exclusions, contact
// assembly, the v1 -> ConstraintIR adapter, world-point relative velocities
// and evaluateConstraintIR.  The evaluation uses the substep h, the world's
// slop and depenetration cap and no regularisation floor (the GPU world's
// semantics; the CPU world step adds a 1e-6 floor for its Newton solver).
// Raw contacts and manifolds as ref_scene_collide writes them, colliders
// translated to record shape indices.  Contact rows (24 doubles): shape a,
// shape b, feature A, feature B, separation, normal xyz, point xyz, target
// velocity n/t/u, regularisation n/t/u, effective mu, relative velocity
// n/t/u, new impact, pre-solve normal velocity.  Returns a status code.
__attribute__((visibility("default"))) int ref_articulated_contacts(RefModel* r, RefContactCache* cache, const double* q,
                                                                   const double* vf, std::uint32_t raw_cap, double* raw,
                                                                   std::uint32_t* raw_count, std::uint32_t manifold_cap,
                                                                   double* manifolds, std::uint32_t* manifold_count,
                                                                   std::uint32_t row_cap, double* rows, std::uint32_t* row_count) {
    *raw_count = *manifold_count = *row_count = 0;
    const EngineModel& model = r->model;
    const std::uint32_t nq = r->world.nq, nv = r->world.nv;
    const MRArticulationGPU& art = model.articulations[0];
    std::vector<ArticulatedBodyKinematics> bk(art.bodyCount);
    auto kd = computeArticulatedBodyKinematics(model, 0, std::span<const double>(q, nq), std::span<const double>(vf, nv), bk,
                                               dyn_config(r));
    if (!kd.succeeded()) return MR_STEP_NONFINITE_INPUT;
    std::vector<MRBodyStateGPU> states(model.bodies.size() + r->env_bodies.size());
    for (const ArticulatedBodyKinematics& b : bk) {
        const MRBodyPropertiesGPU& pr = model.bodies[b.bodyIndex];
        MRBodyStateGPU st{};
        st.position = f4(b.centerOfMassPosition[0], b.centerOfMassPosition[1], b.centerOfMassPosition[2], 1.0);
        st.orientation = f4(b.orientation[0], b.orientation[1], b.orientation[2], b.orientation[3]);
        st.linearVelocityAndInverseMass = f4(b.linearVelocity[0], b.linearVelocity[1], b.linearVelocity[2], pr.massAndInverseMass.y);
        st.angularVelocity = f4(b.angularVelocity[0], b.angularVelocity[1], b.angularVelocity[2], 0.0);
        st.flagsAndIndices[0] = MR_MOTION_DYNAMIC;
        states[b.bodyIndex] = st;
    }
    std::copy(r->env_bodies.begin(), r->env_bodies.end(), states.begin() + model.bodies.size());
    std::vector<MRShapeGPU> shapes = model.shapes;
    for (MRShapeGPU sh : r->env_shapes) {
        sh.bodyIndex += static_cast<std::uint32_t>(model.bodies.size());
        shapes.push_back(sh);
    }
    std::vector<CollisionPairExclusion> exclusions;
    for (std::uint32_t j = 0; j < art.jointCount; ++j) {
        const MRJointDescriptorGPU& jd = model.joints[art.firstJoint + j];
        for (std::uint32_t a = 0; a < model.shapes.size(); ++a) {
            if (model.shapes[a].bodyIndex != jd.parentBody) continue;
            for (std::uint32_t b = 0; b < model.shapes.size(); ++b)
                if (model.shapes[b].bodyIndex == jd.childBody) exclusions.push_back({a, b});
        }
    }
    CollisionConfig ccfg{};
    ccfg.capacities = CollisionCapacities{4096u, 8192u, 2048u};
    ccfg.manifoldBreakingSeparation = r->world.manifold_thresholds[0];
    ccfg.manifoldBreakingTangential = r->world.manifold_thresholds[1];
    ccfg.manifoldMergeDistance = r->world.manifold_thresholds[2];
    ccfg.manifoldNormalCosine = r->world.manifold_thresholds[3];
    const CollisionFrame f = collideCpuReference(shapes, states, ccfg, cache->manifolds, exclusions);
    if (!f.succeeded()) return static_cast<int>(f.diagnostics.code);
    auto shape_of = [&](std::uint32_t collider) -> double { return r->shape_of_collider[collider]; };
    for (std::size_t i = 0; i < f.rawContacts.size() && i < raw_cap; ++i) {
        const MRRawContactGPU& c = f.rawContacts[i];
        const MRCandidatePairGPU& p = f.pairs[f.rawContactPairIndices[i]];
        double* o = raw + 16 * i;
        o[0] = shape_of(p.colliderA);
        o[1] = shape_of(p.colliderB);
        o[2] = c.normalAndSeparation.x;
        o[3] = c.normalAndSeparation.y;
        o[4] = c.normalAndSeparation.z;
        o[5] = c.normalAndSeparation.w;
        o[6] = c.pointAWorld.x;
        o[7] = c.pointAWorld.y;
        o[8] = c.pointAWorld.z;
        o[9] = c.pointBWorld.x;
        o[10] = c.pointBWorld.y;
        o[11] = c.pointBWorld.z;
        o[12] = c.featureAndFlags[0];
        o[13] = c.featureAndFlags[1];
        o[14] = o[15] = 0.0;
        *raw_count = static_cast<std::uint32_t>(i + 1);
    }
    for (std::size_t m = 0; m < f.manifoldHeaders.size() && m < manifold_cap; ++m) {
        const MRManifoldHeaderGPU& hd = f.manifoldHeaders[m];
        double* o = manifolds + 58 * m;
        o[0] = shape_of(hd.pairAndCount[1]);
        o[1] = shape_of(hd.pairAndCount[2]);
        o[2] = hd.pairAndCount[3];
        o[3] = hd.normalAndAge.x;
        o[4] = hd.normalAndAge.y;
        o[5] = hd.normalAndAge.z;
        o[6] = hd.normalAndAge.w;
        o[7] = hd.tangentAndMetric.x;
        o[8] = hd.tangentAndMetric.y;
        o[9] = hd.tangentAndMetric.z;
        for (int k = 0; k < 4; ++k) {
            const MRManifoldPointGPU& pt = f.manifoldPoints[4 * m + k];
            double* po = o + 10 + 12 * k;
            po[0] = pt.localAnchorA.x;
            po[1] = pt.localAnchorA.y;
            po[2] = pt.localAnchorA.z;
            po[3] = pt.localAnchorB.x;
            po[4] = pt.localAnchorB.y;
            po[5] = pt.localAnchorB.z;
            po[6] = pt.impulses.x;
            po[7] = pt.impulses.y;
            po[8] = pt.impulses.z;
            po[9] = pt.featureAndLife[0];
            po[10] = pt.featureAndLife[1];
            po[11] = pt.featureAndLife[2];
        }
        *manifold_count = static_cast<std::uint32_t>(m + 1);
    }
    ContactAssemblyResult assembly = assembleContactConstraints(f, shapes, model.materials, states, 4096u);
    if (!assembly.diagnostics.succeeded()) return static_cast<int>(assembly.diagnostics.code);
    if (assembly.constraints.empty()) return 0;
    const ConstraintIRV1AdapterResult compiled = adaptV1ContactsToConstraintIR(assembly.constraints, ConstraintIRV1AdapterConfig{});
    if (!compiled.succeeded()) return MR_STEP_NONFINITE_RESULT;
    const ConstraintIRVelocityResult vel = computeConstraintIRWorldPointVelocities(compiled.ir, states);
    if (!vel.succeeded()) return MR_STEP_NONFINITE_RESULT;
    ConstraintIREvaluationConfig ecfg{};
    ecfg.timestep = r->h;
    ecfg.penetrationSlop = r->world.solver_scales[3];
    ecfg.maximumDepenetrationVelocity = r->world.solver_scales[2];
    ecfg.minimumRegularization = 0.0;
    const ConstraintIREvaluationResult ev =
        evaluateConstraintIR(compiled.ir, {vel.relativeVelocities, compiled.preSolveVelocities}, ecfg);
    if (!ev.succeeded()) return MR_STEP_NONFINITE_RESULT;
    for (std::size_t b = 0; b < ev.evaluated.blocks.size() && *row_count < row_cap; ++b) {
        const ConstraintIRBlock& blk = ev.evaluated.blocks[b];
        if (blk.type != MR_CONSTRAINT_CONTACT) continue;
        const MRContactConstraintGPU& c = assembly.constraints[compiled.sourceConstraintIndices[b]];
        double* o = rows + 24 * (*row_count)++;
        o[0] = shape_of(static_cast<std::uint32_t>(c.pairKey >> 32u));
        o[1] = shape_of(static_cast<std::uint32_t>(c.pairKey & 0xffffffffu));
        o[2] = static_cast<double>(static_cast<std::uint32_t>(c.featureKey >> 32u));
        o[3] = static_cast<double>(static_cast<std::uint32_t>(c.featureKey & 0xffffffffu));
        o[4] = c.pointAndSeparation.w;
        o[5] = c.normal.x;
        o[6] = c.normal.y;
        o[7] = c.normal.z;
        o[8] = c.pointAndSeparation.x;
        o[9] = c.pointAndSeparation.y;
        o[10] = c.pointAndSeparation.z;
        for (std::uint32_t k = 0; k < 3; ++k) {
            const EvaluatedConstraintIRRow& row = ev.evaluated.rows[blk.rowOffset + k];
            o[11 + k] = row.targetVelocity;
            o[14 + k] = row.regularization;
            o[18 + k] = row.relativeVelocity;
        }
        o[17] = ev.evaluated.cones[blk.coneIndex].effectiveFrictionU;
        o[21] = (c.flags & MR_CONSTRAINT_FLAG_NEW_IMPACT) ? 1.0 : 0.0;
        o[22] = c.targetVelocityAndPreSolveNormal.w;
        o[23] = 0.0;
    }
    return 0;
}

// Island partition of a contact set by the reference (buildConstraintIslands,
// ConstraintSolver.cpp:848): `dynamic[b]` != 0 marks dynamic bodies, contacts
// are (bodyA, bodyB) pairs (MR_INVALID_INDEX-free).  Writes each body's
// island index (MR_INVALID_INDEX: in no island) and returns the island count.
__attribute__((visibility("default"))) std::uint32_t ref_build_islands(std::uint32_t bodies, const std::uint8_t* dynamic,
                                                                      std::uint32_t contacts, const std::uint32_t* pairs,
                                                                      std::uint32_t* body_island) {
    std::vector<MRBodyStateGPU> states(bodies);
    for (std::uint32_t b = 0; b < bodies; ++b) {
        states[b] = MRBodyStateGPU{};
        states[b].orientation = f4(0.0, 0.0, 0.0, 1.0);
        states[b].linearVelocityAndInverseMass = f4(0.0, 0.0, 0.0, dynamic[b] ? 1.0 : 0.0);
        states[b].flagsAndIndices[0] = dynamic[b] ? MR_MOTION_DYNAMIC : MR_MOTION_STATIC;
    }
    std::vector<MRContactConstraintGPU> cs(contacts);
    for (std::uint32_t i = 0; i < contacts; ++i) {
        cs[i] = MRContactConstraintGPU{};
        cs[i].bodyA = pairs[2 * i];
        cs[i].bodyB = pairs[2 * i + 1];
    }
    const std::vector<ConstraintIsland> islands = buildConstraintIslands(states, cs);
    for (std::uint32_t b = 0; b < bodies; ++b) body_island[b] = MR_INVALID_INDEX;
    for (std::size_t i = 0; i < islands.size(); ++i)
        for (std::uint32_t b : islands[i].dynamicBodies) body_island[b] = static_cast<std::uint32_t>(i);
    return static_cast<std::uint32_t>(islands.size());
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Free-body piles: the reference's FP64 collision oracle over one pile.
// ---------------------------------------------------------------------------

struct RefScene {
    std::vector<MRShapeGPU> shapes;
    std::vector<MRBodyStateGPU> bodies;
    CollisionConfig config;
    PersistentManifoldCache cache;
    std::uint32_t nb = 0;
};

extern "C" {

__attribute__((visibility("default"))) RefScene* ref_scene_create(const MRModelWorldC* world, const MRModelBodyC* bodies,
                                                                  const MRModelShapeC* shapes, char* err, size_t err_len) {
    try {
        auto r = std::make_unique<RefScene>();
        r->nb = world->body_count - 1;
        for (std::uint32_t b = 0; b < world->body_count; ++b) {
            MRBodyStateGPU st{};
            const bool ground = b == r->nb;
            st.position = ground ? f4(bodies[b].static_pose[0], bodies[b].static_pose[1], bodies[b].static_pose[2], 0.0)
                                 : f4(0.0, 0.0, 0.0, 0.0);
            st.orientation = ground ? f4(bodies[b].static_pose + 4) : f4(0.0, 0.0, 0.0, 1.0);
            st.flagsAndIndices[0] = ground ? MR_MOTION_STATIC : MR_MOTION_DYNAMIC;
            st.flagsAndIndices[1] = MR_INVALID_INDEX;
            st.flagsAndIndices[2] = MR_INVALID_INDEX;
            r->bodies.push_back(st);
        }
        for (std::uint32_t s = 0; s < world->shape_count; ++s) {
            const MRModelShapeC& src = shapes[s];
            MRShapeGPU sh{};
            sh.bodyIndex = src.body;
            sh.shapeType = src.shape_type;
            sh.materialIndex = src.material;
            sh.collisionGroup = src.collision_group;
            sh.collisionMask = src.collision_mask;
            sh.slotGeneration = 1;
            sh.localPosition = f4(src.local_position[0], src.local_position[1], src.local_position[2], 1.0);
            sh.localRotation = f4(src.local_rotation);
            sh.dimensions = f4(src.dimensions);
            sh.contactRestAndBoundingRadius = f4(src.contact_rest_bound);
            r->shapes.push_back(sh);
        }
        r->config.capacities = CollisionCapacities{4096u, 8192u, 2048u};
        r->config.manifoldBreakingSeparation = world->manifold_thresholds[0];
        r->config.manifoldBreakingTangential = world->manifold_thresholds[1];
        r->config.manifoldMergeDistance = world->manifold_thresholds[2];
        r->config.manifoldNormalCosine = world->manifold_thresholds[3];
        return r.release();
    } catch (const std::exception& e) {
        write_error(err, err_len, e.what());
        return nullptr;
    }
}

__attribute__((visibility("default"))) void ref_scene_destroy(RefScene* r) { delete r; }

// One collision pass at body poses q ([nb][7], xyzw).  Raw contacts: 16
// doubles each (collider a, b, normal xyz, separation, point A xyz, point B
// xyz, feature A, feature B, 0, 0).  Manifolds: 58 doubles each (a, b,
// count, normal xyz, age, tangent xyz, then four points of anchor A xyz,
// anchor B xyz, impulses xyz, feature A, feature B, life).  Returns the
// reference's status code; the cache carries manifolds to the next call.
__attribute__((visibility("default"))) int ref_scene_collide(RefScene* r, const double* q, std::uint32_t raw_cap, double* raw,
                                                             std::uint32_t* raw_count, std::uint32_t manifold_cap, double* manifolds,
                                                             std::uint32_t* manifold_count) {
    for (std::uint32_t b = 0; b < r->nb; ++b) {
        r->bodies[b].position = f4(q[7 * b], q[7 * b + 1], q[7 * b + 2], 0.0);
        r->bodies[b].orientation = f4(q[7 * b + 3], q[7 * b + 4], q[7 * b + 5], q[7 * b + 6]);
    }
    const CollisionFrame f = collideCpuReference(r->shapes, r->bodies, r->config, r->cache);
    *raw_count = 0;
    *manifold_count = 0;
    if (!f.succeeded()) return static_cast<int>(f.diagnostics.code);
    for (std::size_t i = 0; i < f.rawContacts.size() && i < raw_cap; ++i) {
        const MRRawContactGPU& c = f.rawContacts[i];
        const MRCandidatePairGPU& p = f.pairs[f.rawContactPairIndices[i]];
        double* o = raw + 16 * i;
        o[0] = p.colliderA;
        o[1] = p.colliderB;
        o[2] = c.normalAndSeparation.x;
        o[3] = c.normalAndSeparation.y;
        o[4] = c.normalAndSeparation.z;
        o[5] = c.normalAndSeparation.w;
        o[6] = c.pointAWorld.x;
        o[7] = c.pointAWorld.y;
        o[8] = c.pointAWorld.z;
        o[9] = c.pointBWorld.x;
        o[10] = c.pointBWorld.y;
        o[11] = c.pointBWorld.z;
        o[12] = c.featureAndFlags[0];
        o[13] = c.featureAndFlags[1];
        o[14] = o[15] = 0.0;
        *raw_count = static_cast<std::uint32_t>(i + 1);
    }
    for (std::size_t m = 0; m < f.manifoldHeaders.size() && m < manifold_cap; ++m) {
        const MRManifoldHeaderGPU& hd = f.manifoldHeaders[m];
        double* o = manifolds + 58 * m;
        o[0] = hd.pairAndCount[1];
        o[1] = hd.pairAndCount[2];
        o[2] = hd.pairAndCount[3];
        o[3] = hd.normalAndAge.x;
        o[4] = hd.normalAndAge.y;
        o[5] = hd.normalAndAge.z;
        o[6] = hd.normalAndAge.w;
        o[7] = hd.tangentAndMetric.x;
        o[8] = hd.tangentAndMetric.y;
        o[9] = hd.tangentAndMetric.z;
        for (int k = 0; k < 4; ++k) {
            const MRManifoldPointGPU& pt = f.manifoldPoints[4 * m + k];
            double* po = o + 10 + 12 * k;
            po[0] = pt.localAnchorA.x;
            po[1] = pt.localAnchorA.y;
            po[2] = pt.localAnchorA.z;
            po[3] = pt.localAnchorB.x;
            po[4] = pt.localAnchorB.y;
            po[5] = pt.localAnchorB.z;
            po[6] = pt.impulses.x;
            po[7] = pt.impulses.y;
            po[8] = pt.impulses.z;
            po[9] = pt.featureAndLife[0];
            po[10] = pt.featureAndLife[1];
            po[11] = pt.featureAndLife[2];
        }
        *manifold_count = static_cast<std::uint32_t>(m + 1);
    }
    return 0;
}

}  // extern "C"

// PolicyPack files through the reference's own writer and reader.  The pack
// is given in this library's MRPolicyPackC (the field set of the
// reference's c_api.h:344-372).  Errors go to `err`.
static void ref_copy_layers(std::vector<PolicyDenseLayer>& out, const MRPolicyDenseLayerC* ls, size_t n) {
    out.resize(n);
    for (size_t i = 0; i < n; ++i) {
        out[i].inputCount = ls[i].input_count;
        out[i].outputCount = ls[i].output_count;
        out[i].activation = static_cast<PolicyActivation>(ls[i].activation);
        out[i].weights.assign(ls[i].weights, ls[i].weights + ls[i].weight_count);
        out[i].bias.assign(ls[i].bias, ls[i].bias + ls[i].bias_count);
    }
}

extern "C" {

__attribute__((visibility("default"))) int ref_write_policy_pack(const MRPolicyPackC* c, const char* path, char* err, size_t err_len) {
    PolicyPack p;
    p.id = c->id;
    p.revision = c->revision;
    p.contract.version = c->contract_version;
    p.contract.worldFingerprint = c->world_fingerprint;
    p.contract.taskFingerprint = c->task_fingerprint;
    p.contract.observationFingerprint = c->observation_fingerprint;
    p.contract.actionFingerprint = c->action_fingerprint;
    auto vec = [](const float* v, size_t n) { return std::vector<float>(v, v + n); };
    p.observationMean = vec(c->observation_mean, c->observation_mean_count);
    p.observationInverseStandardDeviation = vec(c->observation_inverse_standard_deviation, c->observation_inverse_standard_deviation_count);
    ref_copy_layers(p.layers, c->layers, c->layer_count);
    p.criticObservationMean = vec(c->critic_observation_mean, c->critic_observation_mean_count);
    p.criticObservationInverseStandardDeviation =
        vec(c->critic_observation_inverse_standard_deviation, c->critic_observation_inverse_standard_deviation_count);
    ref_copy_layers(p.criticLayers, c->critic_layers, c->critic_layer_count);
    p.actionLogStandardDeviation = vec(c->action_log_standard_deviation, c->action_log_standard_deviation_count);
    p.actionBias = vec(c->action_bias, c->action_bias_count);
    p.actionScale = vec(c->action_scale, c->action_scale_count);
    p.observationClip = c->observation_clip;
    p.actionClip = c->action_clip;
    const LearningPackResult r = writePolicyPack(p, path);
    if (!r.succeeded() && err && err_len) std::snprintf(err, err_len, "%s", r.message.c_str());
    return r.succeeded() ? 0 : static_cast<int>(r.status);
}

// A TaskPack filled field by field (variant 0: every table and program used,
// a support patch, projectile ballistics, a threat program, terrain samples;
// variant 1: the smallest valid pack), written by the reference's writer
// (writeTaskPack).  The reference's own task builders live beside its world
// compiler, which needs sources absent here.
__attribute__((visibility("default"))) int ref_write_task_pack(int variant, const char* path, char* err, size_t err_len) {
    TaskPack p;
    p.id = variant == 0 ? "full_task_pack" : "minimal";
    p.actions = {{"hip_pitch"}};
    if (variant == 0) {
        p.capacities.candidatePairs = 96u;
        p.capacities.rawContacts = 384u;
        p.capacities.manifolds = 48u;
        p.actions = {{"left_hip"}, {"right_hip"}, {"left_knee"}, {"right_knee"}, {"waist"}};
        p.outcomes = {{"tracking", "score", TaskOutcomeSource::trackingScore, TaskOutcomeDirection::higherIsBetter,
                       TaskRewardOperator::constant},
                      {"slip", "m/s", TaskOutcomeSource::rewardContribution, TaskOutcomeDirection::lowerIsBetter,
                       TaskRewardOperator::supportSlip}};
        TaskContactGroup foot;
        foot.id = "left_foot";
        foot.bodies = {"left_ankle", "left_toe"};
        foot.support = true;
        foot.referenceBody = "left_ankle";
        foot.localReference = {0.02f, 0.0f, -0.03f, 0.01f};
        foot.gaitPhaseOffsetRadians = 3.14159f;
        foot.stanceFraction = 0.6f;
        foot.supportPatchBounds = {-0.1f, -0.04f, 0.1f, 0.04f};
        foot.supportPatchWidth = 4u;
        foot.supportPatchHeight = 2u;
        TaskContactGroup torso;
        torso.id = "undesired";
        torso.bodies = {"pelvis", "torso", "head"};
        torso.forbidden = true;
        torso.referenceBody = "torso";
        p.contactGroups = {foot, torso};
        p.jointGroups = {{"legs", {"left_hip", "right_hip", "left_knee", "right_knee"}}, {"waist", {"waist"}}};
        TaskRewardOperatorSpec r0;
        r0.operation = TaskRewardOperator::linearVelocityTracking;
        r0.weight = 1.0f;
        r0.parameters = {0.25f, 0.0f, 0.0f, 0.0f};
        TaskRewardOperatorSpec r1;
        r1.operation = TaskRewardOperator::jointGroupPostureAbsolute;
        r1.sourceGroup = "waist";
        r1.weight = -1.0f;
        TaskRewardOperatorSpec r2;
        r2.operation = TaskRewardOperator::objectLift;
        r2.target = "box";
        r2.weight = 2.0f;
        r2.parameters = {0.1f, 0.4f, 0.0f, 0.0f};
        p.rewards = {r0, r1, r2};
        TaskTerminationOperatorSpec t0;
        t0.operation = TaskTerminationOperator::minimumRootHeight;
        t0.reason = MR_TASK_TERMINATION_HEIGHT;
        t0.priority = 1u;
        t0.threshold = 0.3f;
        t0.failurePenalty = -2.0f;
        TaskTerminationOperatorSpec t1;
        t1.operation = TaskTerminationOperator::contactGroup;
        t1.sourceGroup = "undesired";
        t1.reason = MR_TASK_TERMINATION_CONTACT;
        t1.priority = 3u;
        t1.threshold = 0.5f;
        t1.minimumDifficultyBand = 1u;
        t1.maximumDifficultyBand = 4u;
        p.terminations = {t0, t1};
        p.commands.lower = {-0.5f, -0.3f, -0.5f, 0.0f};
        p.commands.upper = {1.0f, 0.3f, 0.5f, 0.0f};
        p.commands.limitLower = {-1.0f, -0.6f, -1.0f, 0.0f};
        p.commands.limitUpper = {2.0f, 0.6f, 1.0f, 0.0f};
        p.commands.difficultyStep = {0.1f, 0.05f, 0.1f, 0.0f};
        p.commands.standingProbability = 0.1f;
        p.commands.minimumDurationSeconds = 2.0f;
        p.commands.maximumDurationSeconds = 4.0f;
        p.pushes.maximumVelocity = 1.5f;
        p.pushes.projectileTargetHorizontalRadius = 0.2f;
        p.pushes.projectileHorizontalSpeedLower = 2.0f;
        p.pushes.projectileHorizontalSpeedUpper = 4.0f;
        p.pushes.projectileTargetHeightLower = 0.3f;
        p.pushes.projectileTargetHeightUpper = 1.2f;
        p.terrain.body = "terrain";
        p.terrain.sampleOffsets = {{0.1f, 0.0f, 0.0f, 0.0f}, {-0.1f, 0.0f, 0.0f, 0.0f}, {0.0f, 0.1f, 0.0f, 0.0f}};
        p.terrain.resetTranslations = {{0.0f, 0.0f, 0.05f, 0.0f}};
        p.threat.protectedGroup = "undesired";
        p.motion.anchorBody = "pelvis";
        p.motion.trackedBodies = {"left_ankle", "torso"};
        p.maximumEpisodeSteps = 750u;
        p.difficultyBandCount = 5u;
        p.interactionStudentAuthority = 0.25f;
        p.interactionResetPhaseFraction = 0.1f;
        p.initialActionPositions = {0.1f, -0.1f, 0.3f, 0.3f, 0.0f};
        p.interactionAlignReferenceYaw = true;
        p.baseHeightTarget = 0.74f;
        p.gaitPeriodSeconds = 0.7f;
        p.clearanceTarget = 0.08f;
        p.successTrackingThreshold = 0.75f;
        p.supportForceThreshold = 2.0f;
    }
    const LearningPackResult r = writeTaskPack(p, path);
    if (!r.succeeded() && err && err_len) std::snprintf(err, err_len, "%s", r.message.c_str());
    return r.succeeded() ? 0 : static_cast<int>(r.status);
}

// The reference's reader (readTaskPack) into this library's info record.
__attribute__((visibility("default"))) int ref_task_pack_inspect(const char* path, MRTaskPackInfoC* info, char* err, size_t err_len) {
    TaskPack p;
    const LearningPackResult r = readTaskPack(path, p);
    if (!r.succeeded()) {
        if (err && err_len) std::snprintf(err, err_len, "%s", r.message.c_str());
        return static_cast<int>(r.status);
    }
    MRTaskPackInfoC o{};
    o.content_hash = r.contentHash;
    o.action_count = static_cast<uint32_t>(p.actions.size());
    o.outcome_count = static_cast<uint32_t>(p.outcomes.size());
    o.contact_group_count = static_cast<uint32_t>(p.contactGroups.size());
    o.joint_group_count = static_cast<uint32_t>(p.jointGroups.size());
    o.reward_count = static_cast<uint32_t>(p.rewards.size());
    o.termination_count = static_cast<uint32_t>(p.terminations.size());
    o.maximum_episode_steps = p.maximumEpisodeSteps;
    o.difficulty_band_count = p.difficultyBandCount;
    o.terrain_sample_count = static_cast<uint32_t>(p.terrain.sampleOffsets.size());
    o.motion_tracked_body_count = static_cast<uint32_t>(p.motion.trackedBodies.size());
    o.base_height_target = p.baseHeightTarget;
    o.gait_period_seconds = p.gaitPeriodSeconds;
    o.clearance_target = p.clearanceTarget;
    o.support_force_threshold = p.supportForceThreshold;
    std::snprintf(o.id, sizeof(o.id), "%s", p.id.c_str());
    *info = o;
    return 0;
}

// readTaskPack then writeTaskPack (the reference's artifact rules apply).
__attribute__((visibility("default"))) int ref_task_pack_rewrite(const char* in, const char* out, char* err, size_t err_len) {
    TaskPack p;
    LearningPackResult r = readTaskPack(in, p);
    if (r.succeeded()) r = writeTaskPack(p, out);
    if (!r.succeeded() && err && err_len) std::snprintf(err, err_len, "%s", r.message.c_str());
    return r.succeeded() ? 0 : static_cast<int>(r.status);
}

__attribute__((visibility("default"))) size_t ref_capacity_profile_bytes() { return sizeof(MetalWorldCapacityProfile); }

// The reference's PolicyRolloutPack writer (writePolicyRolloutPack) over the
// same record this library's mr_write_policy_rollout_pack takes; task
// transitions become learner transitions the way c_api.cpp:4410-4445 does.
__attribute__((visibility("default"))) int ref_write_policy_rollout_pack(const MRPolicyRolloutPackC* c, const char* path, char* err,
                                                                         size_t err_len) {
    const MRPolicyRolloutBatchC& b = *c->batch;
    std::vector<MRLearningTransitionGPU> transitions(b.transition_count);
    for (size_t i = 0; i < b.transition_count; ++i) {
        const MRTaskTransitionC& t = b.transitions[i];
        MRLearningTransitionGPU& d = transitions[i];
        d = MRLearningTransitionGPU{};
        d.rewardAndBootstrap = {t.reward, t.timeout_bootstrap_value, 0.0f, 0.0f};
        d.termination = {t.done, t.timeout, t.physics_error, t.termination_reason};
        d.context = {t.difficulty_band, t.terrain_level, t.impact_sequence_index, t.impact_event_flags};
        d.policyRevision = t.policy_revision;
    }
    auto span = [](const float* v, size_t n) { return std::span<const float>(v, n); };
    const PolicyRolloutPackView view{
        .id = c->id,
        .taskFingerprint = c->task_fingerprint,
        .policyFingerprint = c->policy_fingerprint,
        .policyRevision = c->policy_revision,
        .environmentCount = c->environment_count,
        .controlStepCount = b.control_step_count,
        .actorObservationCount = c->actor_observation_count,
        .criticObservationCount = c->critic_observation_count,
        .actionCount = c->action_count,
        .motionFeatureCount = c->motion_feature_count,
        .actorObservations = span(b.actor_observations, b.actor_observation_count),
        .criticObservations = span(b.critic_observations, b.critic_observation_count),
        .motionFeatures = span(b.motion_features, b.motion_feature_count),
        .teacherActions = span(b.teacher_actions, b.teacher_action_count),
        .latents = span(b.latents, b.latent_count),
        .logProbabilities = span(b.log_probabilities, b.log_probability_count),
        .values = span(b.values, b.value_count),
        .bootstrapValues = span(b.bootstrap_values, b.bootstrap_value_count),
        .outcomes = {},
        .outcomeValues = {},
        .transitions = transitions,
    };
    const LearningPackResult r = writePolicyRolloutPack(view, path);
    if (!r.succeeded() && err && err_len) std::snprintf(err, err_len, "%s", r.message.c_str());
    return r.succeeded() ? 0 : static_cast<int>(r.status);
}

// The reference's reader (readPolicyRolloutPack) into this library's info record.
__attribute__((visibility("default"))) int ref_policy_rollout_pack_inspect(const char* path, MRPolicyRolloutPackInfoC* info,
                                                                           float* params, size_t cap, char* err, size_t err_len) {
    PolicyRolloutPack p;
    const LearningPackResult r = readPolicyRolloutPack(path, p);
    if (!r.succeeded()) {
        if (err && err_len) std::snprintf(err, err_len, "%s", r.message.c_str());
        return static_cast<int>(r.status);
    }
    MRPolicyRolloutPackInfoC o{};
    o.task_fingerprint = p.taskFingerprint;
    o.policy_fingerprint = p.policyFingerprint;
    o.policy_revision = p.policyRevision;
    o.content_hash = r.contentHash;
    o.environment_count = p.environmentCount;
    o.control_step_count = p.controlStepCount;
    o.actor_observation_count = p.actorObservationCount;
    o.critic_observation_count = p.criticObservationCount;
    o.action_count = p.actionCount;
    o.motion_feature_count = p.motionFeatureCount;
    o.outcome_count = static_cast<uint32_t>(p.outcomes.size());
    o.has_teacher_actions = p.teacherActions.empty() ? 0u : 1u;
    o.transition_count = p.transitions.size();
    for (const MRLearningTransitionGPU& t : p.transitions) {
        o.reward_sum += t.rewardAndBootstrap.x;
        o.done_count += t.termination.x;
    }
    std::snprintf(o.id, sizeof(o.id), "%s", p.id.c_str());
    if (params) {
        size_t at = 0;
        for (const std::vector<float>* v : {&p.actorObservations, &p.latents, &p.logProbabilities, &p.values, &p.bootstrapValues}) {
            if (v->size() > cap - at) {
                if (err && err_len) std::snprintf(err, err_len, "parameters capacity is too small");
                return -1;
            }
            std::memcpy(params + at, v->data(), v->size() * sizeof(float));
            at += v->size();
        }
    }
    *info = o;
    return 0;
}

__attribute__((visibility("default"))) int ref_policy_pack_inspect(const char* path, MRPolicyPackInfoC* info, float* params, size_t cap,
                                                                   char* err, size_t err_len) {
    PolicyPack p;
    const LearningPackResult r = readPolicyPack(path, p);
    if (!r.succeeded()) {
        if (err && err_len) std::snprintf(err, err_len, "%s", r.message.c_str());
        return static_cast<int>(r.status);
    }
    MRPolicyPackInfoC o{};
    o.layer_count = static_cast<uint32_t>(p.layers.size());
    o.critic_layer_count = static_cast<uint32_t>(p.criticLayers.size());
    o.observation_count = p.layers.empty() ? 0u : p.layers.front().inputCount;
    o.action_count = p.layers.empty() ? 0u : p.layers.back().outputCount;
    o.stochastic = p.actionLogStandardDeviation.empty() ? 0u : 1u;
    o.revision = p.revision;
    o.content_hash = r.contentHash;
    o.contract_version = p.contract.version;
    o.world_fingerprint = p.contract.worldFingerprint;
    o.task_fingerprint = p.contract.taskFingerprint;
    o.observation_fingerprint = p.contract.observationFingerprint;
    o.action_fingerprint = p.contract.actionFingerprint;
    o.observation_clip = p.observationClip;
    o.action_clip = p.actionClip;
    std::snprintf(o.id, sizeof(o.id), "%s", p.id.c_str());
    std::vector<const std::vector<float>*> t{&p.observationMean, &p.observationInverseStandardDeviation};
    for (const PolicyDenseLayer& l : p.layers) { t.push_back(&l.weights); t.push_back(&l.bias); }
    t.push_back(&p.criticObservationMean);
    t.push_back(&p.criticObservationInverseStandardDeviation);
    for (const PolicyDenseLayer& l : p.criticLayers) { t.push_back(&l.weights); t.push_back(&l.bias); }
    t.push_back(&p.actionLogStandardDeviation);
    t.push_back(&p.actionBias);
    t.push_back(&p.actionScale);
    size_t total = 0;
    for (const auto* v : t) total += v->size();
    o.parameter_count = total;
    if (params && cap >= total) {
        size_t at = 0;
        for (const auto* v : t) { std::copy(v->begin(), v->end(), params + at); at += v->size(); }
    }
    *info = o;
    return 0;
}

}  // extern "C"
