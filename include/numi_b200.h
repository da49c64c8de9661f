/*
 * numi_b200 — B200 (sm_100a) batched articulated-physics microstep behind
 * numi-lab's task-rollout C ABI.
 *
 * Every declaration below that carries a "reference:" note replaces the
 * numi-lab (MetalRobo) interface at that file:line with the same name,
 * argument meaning and error behaviour:
 *   - ints return 0 on success and -1 on error;
 *   - errors are stored in a thread-local string read by mr_last_error();
 *   - caller spans are copied before return;
 *   - returned pointers alias handle-owned memory until the next advance,
 *     reset or destroy of that handle;
 *   - a handle is not internally locked: one caller thread per handle.
 *
 * Entry points marked "no counterpart in the reference" are additions of
 * this library (device-pointer advance for zero-copy torch tensors, model
 * and state export for checking and serving).
 */
#ifndef NUMI_B200_H
#define NUMI_B200_H

#include <stddef.h>
#include <stdint.h>

#define MR_API __attribute__((visibility("default")))

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------------- */
/* Capacities and enumerations                                             */
/* ---------------------------------------------------------------------- */

#define MR_INVALID_INDEX 0xffffffffu
#define MR_B200_MAX_BODIES 32u     /* bodies per articulated world           */
#define MR_B200_MAX_DOFS 40u       /* generalized velocities per world       */
#define MR_B200_MAX_Q 41u          /* generalized coordinates per world      */
#define MR_B200_MAX_SHAPES 32u     /* colliders per world                    */
#define MR_B200_MAX_PAIRS 32u      /* compiled eligible collider pairs       */
#define MR_B200_SCENE_MANIFOLDS 128u  /* persistent manifold slots per pile   */
#define MR_B200_SCENE_SLOT_WORDS 57u  /* MRManifoldC + pair key               */
#define MR_B200_MAX_CONTACTS 32u   /* solver contacts per environment        */
#define MR_B200_MANIFOLD_POINTS 4u /* persistent points per manifold         */
#define MR_B200_MAX_SUBSTEPS 64u   /* physics substeps per control step      */

/* The enumerations below carry the reference's own names and values; a
 * translation unit that already includes the reference's engine_types.h
 * defines NUMI_B200_OMIT_SHARED_ENUMS before including this header. */
#ifndef NUMI_B200_OMIT_SHARED_ENUMS
/* reference: include/metalrobo/engine_types.h:171-188 (same values). */
enum MRStepStatusCode {
    MR_STEP_SUCCESS = 0u,
    MR_STEP_FIXED_BUDGET_COMPLETE = 1u,
    MR_STEP_NONFINITE_INPUT = 2u,
    MR_STEP_NONFINITE_RESULT = 3u,
    MR_STEP_PAIR_CAPACITY_OVERFLOW = 4u,
    MR_STEP_CONTACT_CAPACITY_OVERFLOW = 5u,
    MR_STEP_MANIFOLD_CAPACITY_OVERFLOW = 6u,
    MR_STEP_CONSTRAINT_CAPACITY_OVERFLOW = 7u,
    MR_STEP_ISLAND_CAPACITY_OVERFLOW = 8u,
    MR_STEP_CCD_EVENT_BUDGET_EXHAUSTED = 9u,
    MR_STEP_FACTORIZATION_FAILED = 10u,
    MR_STEP_DID_NOT_CONVERGE = 11u,
    MR_STEP_UNSUPPORTED = 12u,
    MR_STEP_CCD_CAPACITY_OVERFLOW = 13u
};

/* reference: include/metalrobo/engine_types.h:159-164 (same values). */
enum MRSolverType {
    MR_SOLVER_REFERENCE_FP64 = 0u,
    MR_SOLVER_QUALITY_NEWTON = 1u,
    MR_SOLVER_TEMPORAL_CONE = 2u,
    MR_SOLVER_THROUGHPUT_PGS = 3u
};

/* reference: include/metalrobo/gpu_types.h:41-49 (same values). */
enum MRShapeType {
    MR_SHAPE_SPHERE = 0u,
    MR_SHAPE_CAPSULE = 1u,
    MR_SHAPE_BOX = 2u,
    MR_SHAPE_PLANE = 3u,
    MR_SHAPE_CYLINDER = 4u,  /* radius dimensions.x, half length dimensions.y along local +Y */
    MR_SHAPE_CONVEX = 5u     /* hull vertices (MRModelViewC.hull_vertices) scaled by dimensions.xyz */
};

/* reference: include/metalrobo/engine_types.h:114-134 (same values). */
enum MRJointTypeExt {
    MR_JOINT_REVOLUTE = 0u,
    MR_JOINT_PRISMATIC = 1u,
    MR_JOINT_CONTINUOUS = 2u,
    MR_JOINT_FIXED = 5u
};

enum MRRootType { MR_ROOT_FIXED = 0u, MR_ROOT_FLOATING = 1u };
enum MRMotionType { MR_MOTION_STATIC = 0u, MR_MOTION_KINEMATIC = 1u, MR_MOTION_DYNAMIC = 2u };

/* reference: include/metalrobo/engine_types.h:262-272 (same bits). */
enum MRDofFlags {
    MR_DOF_FLAG_ROOT = 1u << 0u,
    MR_DOF_FLAG_ACTUATED = 1u << 1u,
    MR_DOF_FLAG_POSITION_LIMIT = 1u << 2u,
    MR_DOF_FLAG_VELOCITY_LIMIT = 1u << 3u,
    MR_DOF_FLAG_EFFORT_LIMIT = 1u << 4u,
    MR_DOF_FLAG_DRIVE = 1u << 5u
};

/* reference: include/metalrobo/engine_types.h:149-163 (same values). */
enum MRCollisionPairClass {
    MR_COLLISION_PAIR_UNSUPPORTED = 0u,
    MR_COLLISION_PAIR_SPHERE_SPHERE = 1u,
    MR_COLLISION_PAIR_SPHERE_PLANE = 2u,
    MR_COLLISION_PAIR_CAPSULE_PLANE = 3u,
    MR_COLLISION_PAIR_BOX_PLANE = 4u,
    MR_COLLISION_PAIR_CYLINDER_PLANE = 5u,
    MR_COLLISION_PAIR_SPHERE_CAPSULE = 6u,
    MR_COLLISION_PAIR_CAPSULE_CAPSULE = 7u,
    MR_COLLISION_PAIR_SPHERE_BOX = 8u,
    MR_COLLISION_PAIR_CAPSULE_BOX = 9u,
    MR_COLLISION_PAIR_BOX_BOX = 10u,
    MR_COLLISION_PAIR_CONVEX = 11u   /* support-mapped (GJK / EPA): here, a cylinder against a finite shape */
};
#endif /* NUMI_B200_OMIT_SHARED_ENUMS */

/* Actuation law of a world: efforts are generalized forces, or position
 * targets of implicit PD drives (reference: MetalWorld.hpp:388-391). */
enum MRActuationMode { MR_ACTUATION_EFFORT = 0u, MR_ACTUATION_IMPLICIT_POSITION = 1u };

/* ---------------------------------------------------------------------- */
/* Rollout configuration (reference: include/metalrobo/c_api.h:54-88)     */
/* ---------------------------------------------------------------------- */

typedef struct MRTaskRolloutHandle MRTaskRolloutHandle;

typedef struct MRTaskRolloutDynamicSphereC {
    float position[3];
    float linear_velocity[3];
    float radius;
    float mass;
    uint32_t launch_step;
} MRTaskRolloutDynamicSphereC;

typedef struct MRTaskRolloutConfigC {
    uint32_t environment_count;
    uint32_t physics_substeps;
    uint32_t velocity_iterations;
    uint32_t final_velocity_iterations;
    float control_timestep_seconds;
    uint64_t seed;
    const MRTaskRolloutDynamicSphereC* dynamic_spheres;
    uint32_t dynamic_sphere_count;
    uint32_t disable_task_terminations;
    uint32_t interaction_reference_mode;
    float interaction_student_authority;
    uint32_t override_interaction_student_authority;
    float interaction_reset_phase_fraction;
    uint32_t override_interaction_reset_phase_fraction;
    uint32_t materialize_articulated_contact_responses;
    uint32_t override_difficulty_band_range;
    uint32_t minimum_difficulty_band;
    uint32_t maximum_difficulty_band;
    float interaction_reset_phase_probability;
    uint32_t override_interaction_reset_phase_probability;
    float interaction_reset_maximum_phase;
    uint32_t override_interaction_reset_maximum_phase;
} MRTaskRolloutConfigC;

/* Visual programs are not part of the physics path; the type stays opaque
 * and a non-null pointer is rejected. */
typedef struct MRTaskVisualObservationConfigC MRTaskVisualObservationConfigC;

/* reference: include/metalrobo/c_api.h:160-166.  The reference sources
 * 0..4 load robot assets; this library compiles seeded synthetic worlds. */
enum MRRunManifestSourceC {
    MR_RUN_SOURCE_UNITREE_G1 = 0u,
    MR_RUN_SOURCE_FRANKA_PICK_PLACE = 1u,
    MR_RUN_SOURCE_IMPORTED_URDF = 2u,
    MR_RUN_SOURCE_WORLD_PACK = 3u,
    MR_RUN_SOURCE_PX4_X500 = 4u,
    /* Fixed-base 7-revolute serial chain, effort actuation, no contact. */
    MR_RUN_SOURCE_SYNTHETIC_CHAIN7 = 100u,
    /* Floating 29-DoF humanoid tree (pelvis, 2x6 legs, 3 waist, 2x7 arms),
     * implicit PD position drives, box feet and 12 sphere proxies on a
     * ground plane. */
    MR_RUN_SOURCE_SYNTHETIC_TREE29 = 101u,
    /* Pile of 8-64 free boxes, spheres and capsules dropped onto a ground plane (body
     * count drawn from the seed); scene bodies, no actuation. */
    MR_RUN_SOURCE_SYNTHETIC_PILE = 102u,
    /* Stack of 32 0.1 m, 1 kg boxes (friction 0.6) resting on a ground
     * plane, the stack yawed U(0, 2 pi) and each box offset N(0, 2 mm) at
     * reset; scene bodies, no actuation. */
    MR_RUN_SOURCE_SYNTHETIC_STACK = 103u,
    /* Pile of 8-64 free boxes, spheres, capsules and cylinders (one quarter
     * each) dropped onto a ground plane; cylinder pairs take the
     * support-mapped (GJK / EPA) narrowphase. */
    MR_RUN_SOURCE_SYNTHETIC_CYLINDER_PILE = 104u,
    /* The pile of MR_RUN_SOURCE_SYNTHETIC_PILE (same bodies for the same
     * seed) with every capsule-box pair taking the support-mapped (GJK /
     * EPA, MPR fallback) narrowphase instead of the analytic witness. */
    MR_RUN_SOURCE_SYNTHETIC_PILE_GJK = 105,
    /* Pile of 8-64 free boxes, spheres, capsules and convex hulls (one
     * quarter each; each hull 12 vertices) dropped onto a ground plane;
     * pairs with a hull take the hull path of the support-mapped
     * narrowphase (GJK distance, support-axis penetration witness, sampled
     * patch; a hull on the plane: its deepest vertex). */
    MR_RUN_SOURCE_SYNTHETIC_HULL_PILE = 106u
};

/* reference: include/metalrobo/c_api.h:171-190 (same shape). */
typedef struct MRRunManifestC {
    MRTaskRolloutConfigC profile;
    uint32_t source;
    uint32_t surface;
    uint32_t task;
    const char* urdf_path;
    const char* srdf_path;
    const char* world_pack_path;
    const char* task_pack_path;
    const char* robot_actuator_pack_path;
    const char* sensor_program_pack_path;
    const char* reality_program_pack_path;
    const char* teacher_pack_path;
    const char* teacher_clip_id;
    const MRTaskVisualObservationConfigC* visual_sensor_program;
    const MRTaskVisualObservationConfigC* inspection_visual_program;
    const char* metallib_path;
} MRRunManifestC;

/* reference: include/metalrobo/c_api.h:128-158 (same shape). */
typedef struct MRTaskRolloutLayoutC {
    uint32_t environment_count;
    uint32_t nq;
    uint32_t nv;
    uint32_t action_count;
    uint32_t actor_observation_count;
    uint32_t critic_observation_count;
    uint32_t scene_body_count;
    uint32_t motion_feature_count;
    uint32_t maximum_episode_steps;
    uint64_t world_fingerprint;
    uint64_t task_fingerprint;
    uint64_t observation_fingerprint;
    uint64_t action_fingerprint;
    uint64_t run_fingerprint;
    uint64_t robot_fingerprint;
    uint64_t sensor_fingerprint;
    uint64_t reality_fingerprint;
    uint64_t teacher_fingerprint;
    uint64_t submitted_control_steps;
    uint64_t completed_environment_steps;
    uint64_t submission_count;
    size_t retained_buffer_bytes;
    size_t immutable_private_bytes;
    size_t persistent_state_private_bytes;
    size_t transient_private_bytes;
    size_t shared_boundary_bytes;
    size_t peak_aliased_bytes;
    double total_gpu_milliseconds;
    double total_submission_milliseconds;
} MRTaskRolloutLayoutC;

/* reference: include/metalrobo/c_api.h:192-220 (same shape). */
typedef struct MRTaskRolloutStageHighWaterC {
    uint32_t candidate_pairs;
    uint32_t raw_contacts;
    uint32_t manifolds;
    uint32_t constraint_blocks;
    uint32_t constraint_rows;
    uint32_t islands;
    uint32_t hard_convex_pairs;
    uint32_t mesh_triangle_candidates;
    uint32_t solver_tiles;
    uint32_t spill_rows;
    uint32_t ccd_candidates;
    uint32_t ccd_events;
    uint32_t endpoint_runtime_records;
    uint32_t articulation_point_queries;
    uint32_t rod_candidate_pairs;
    uint32_t rod_raw_contacts;
    uint32_t rod_manifolds;
    uint32_t rod_ccd_events;
    uint32_t quality_generalized_velocities;
    uint32_t quality_rows;
    uint32_t quality_krylov_vectors;
    uint32_t quality_direct_tiles;
    uint32_t dynamic_nodes;
    uint32_t island_node_references;
    uint32_t island_constraint_references;
    uint32_t rod_factor_blocks;
    uint32_t operator_velocity_elements;
} MRTaskRolloutStageHighWaterC;

/* reference: include/metalrobo/c_api.h:222-235 (same shape). */
typedef struct MRTaskRolloutAdvanceC {
    uint32_t control_step_count;
    uint32_t successful_environment_steps;
    uint32_t failed_environment_steps;
    uint32_t first_failing_environment;
    uint32_t first_failing_control_step;
    uint32_t first_gpu_status_code;
    uint32_t host_requested_resets;
    uint32_t maximum_active_contacts;
    uint32_t maximum_manifolds;
    MRTaskRolloutStageHighWaterC high_water;
    double gpu_milliseconds;
    double submission_milliseconds;
} MRTaskRolloutAdvanceC;

/* ---------------------------------------------------------------------- */
/* Compiled model records (no counterpart in the reference's C ABI; they   */
/* carry the fields of engine_types.h MRWorldGPU, MRJointDescriptorGPU,    */
/* MRBodyPropertiesGPU, MRDofPropertiesGPU, MRShapeGPU and MRMaterialGPU   */
/* that the microstep reads, so a checker can rebuild the same world).     */
/* ---------------------------------------------------------------------- */

typedef struct MRModelWorldC {
    uint32_t body_count;
    uint32_t joint_count;
    uint32_t nq;
    uint32_t nv;
    uint32_t shape_count;
    uint32_t material_count;
    uint32_t pair_count;
    uint32_t root_type;            /* MRRootType                              */
    uint32_t actuation_mode;       /* MRActuationMode                         */
    uint32_t action_count;         /* actions per env per control step        */
    uint32_t contact_capacity;     /* solver contacts per env                 */
    uint32_t apply_body_damping;
    float gravity[4];              /* xyz gravity, w unused                   */
    /* tolerance, minimum compliance, maximum depenetration speed, slop      */
    float solver_scales[4];
    /* breaking separation, breaking tangential drift, merge distance,
     * normal cosine (reference: MetalWorld.hpp:441-444)                     */
    float manifold_thresholds[4];
    /* speculative margin scale, speed envelope, reserved, reserved          */
    float speculative[4];
} MRModelWorldC;

typedef struct MRModelJointC {
    uint32_t parent_body;
    uint32_t child_body;
    uint32_t joint_type;           /* MRJointTypeExt                          */
    uint32_t q_index;              /* MR_INVALID_INDEX for fixed joints       */
    uint32_t v_index;
    uint32_t reserved[3];
    float axis[4];                 /* joint-frame axis                        */
    float parent_anchor[4];        /* relative to parent COM, parent axes     */
    float child_anchor[4];         /* relative to child COM, child axes       */
    float parent_rotation[4];      /* joint frame in parent, xyzw             */
    float child_rotation[4];       /* joint frame in child, xyzw              */
} MRModelJointC;

typedef struct MRModelBodyC {
    uint32_t parent_body;          /* MR_INVALID_INDEX for the root / statics */
    uint32_t inbound_joint;
    uint32_t motion_type;          /* MRMotionType                            */
    uint32_t articulated;          /* 1 when part of the articulation         */
    float mass_inverse_mass[4];
    float inertia[3][4];           /* symmetric inertia about COM, body axes  */
    /* linear damping, angular damping, max linear speed, max angular speed  */
    float damping_speed[4];
    float static_pose[8];          /* static bodies: position xyz_, quat xyzw */
} MRModelBodyC;

typedef struct MRModelDofC {
    uint32_t joint_index;          /* MR_INVALID_INDEX for root coordinates   */
    uint32_t q_index;              /* MR_INVALID_INDEX for root angular rates */
    uint32_t flags;                /* MRDofFlags                              */
    uint32_t reserved;
    float limits[4];               /* lower, upper, max velocity, max effort  */
    float drive[4];                /* stiffness, damping, armature, friction  */
} MRModelDofC;

typedef struct MRModelShapeC {
    uint32_t body;
    uint32_t shape_type;           /* MRShapeType                             */
    uint32_t material;
    uint32_t flags;
    uint32_t collision_group;
    uint32_t collision_mask;
    /* MR_SHAPE_CONVEX: first vertex and vertex count of its hull in the
     * model's hull vertex table; 0 otherwise.                              */
    uint32_t hull_first;
    uint32_t hull_count;
    float local_position[4];
    float local_rotation[4];
    float dimensions[4];           /* sphere r; capsule r, half length; box half extents */
    float contact_rest_bound[4];   /* contact offset, rest offset, bounding radius */
} MRModelShapeC;

typedef struct MRModelMaterialC {
    float friction[4];             /* static, dynamic, rolling, torsional     */
    float response[4];             /* restitution, threshold, compliance, dissipation */
} MRModelMaterialC;

typedef struct MRModelPairC {
    uint32_t shape_a;              /* shape_a < shape_b                       */
    uint32_t shape_b;
    uint32_t pair_class;           /* MRCollisionPairClass                    */
    uint32_t max_points;           /* manifold points this pair can hold      */
} MRModelPairC;

/* Caller-owned destination for mr_task_rollout_copy_model.  Each pointer
 * must hold the count reported in `world`; pass null to skip a table. */
typedef struct MRModelViewC {
    MRModelWorldC world;
    MRModelJointC* joints;
    MRModelBodyC* bodies;
    MRModelDofC* dofs;
    MRModelShapeC* shapes;
    MRModelMaterialC* materials;
    MRModelPairC* pairs;
    /* Unit-scale local hull vertices of every MR_SHAPE_CONVEX shape, xyz
     * plus one unused float each ([hull_vertex_count][4]); written when
     * non-null and hull_vertex_capacity (vertices) suffices.  The count is
     * always reported. */
    float* hull_vertices;
    uint32_t hull_vertex_capacity;
    uint32_t hull_vertex_count;
} MRModelViewC;

/* Persistent contact state of one environment: one slot per compiled pair.
 * Anchors are relative to each shape's body COM in body axes. */
typedef struct MRManifoldPointC {
    float anchor_a[3];
    float anchor_b[3];
    uint32_t feature_a;
    uint32_t feature_b;
    uint32_t life;
    float impulses[3];             /* normal, tangent, bitangent              */
} MRManifoldPointC;

typedef struct MRManifoldC {
    float normal_local[3];         /* in shape A's body frame                 */
    float age;
    float tangent_local[3];
    uint32_t count;
    MRManifoldPointC points[MR_B200_MANIFOLD_POINTS];
} MRManifoldC;

/* ---------------------------------------------------------------------- */
/* Reference-shaped entry points                                           */
/* ---------------------------------------------------------------------- */

/* reference: include/metalrobo/c_api.h:553 */
MR_API const char* mr_version(void);
/* reference: include/metalrobo/c_api.h:556 */
MR_API uint64_t mr_runtime_abi_fingerprint(void);
/* reference: include/metalrobo/c_api.h:557 */
MR_API const char* mr_last_error(void);

/* reference: include/metalrobo/c_api.h:583-585 */
MR_API MRTaskRolloutHandle* mr_create_task_rollout(const MRRunManifestC* manifest);
/* reference: include/metalrobo/c_api.h:586 */
MR_API void mr_task_rollout_destroy(MRTaskRolloutHandle* handle);
/* reference: include/metalrobo/c_api.h:587-590.  Re-seeds and re-samples
 * every environment's reset state, clears contact state and statistics. */
MR_API int mr_task_rollout_reset(MRTaskRolloutHandle* handle, uint64_t seed);
/* reference: include/metalrobo/c_api.h:631-634 */
MR_API int mr_task_rollout_set_state_readback(MRTaskRolloutHandle* handle, uint32_t enabled);
/* reference: include/metalrobo/c_api.h:635-645.  Host actions packed
 * [step][env][action]; reset masks 0 or [step][env]; synchronous. */
MR_API int mr_task_rollout_advance(
    MRTaskRolloutHandle* handle,
    const float* normalized_actions,
    size_t normalized_action_count,
    const uint32_t* reset_masks,
    size_t reset_mask_count,
    uint32_t control_step_count,
    uint64_t policy_revision,
    uint32_t evaluate_final_policy,
    MRTaskRolloutAdvanceC* advance);
/* reference: include/metalrobo/c_api.h:646-648 */
MR_API MRTaskRolloutLayoutC mr_task_rollout_layout(const MRTaskRolloutHandle* handle);
/* reference: include/metalrobo/c_api.h:658-660 */
MR_API const char* mr_task_rollout_device_name(const MRTaskRolloutHandle* handle);
/* reference: include/metalrobo/c_api.h:682-684.  [step][env] of the last advance. */
MR_API const uint32_t* mr_task_rollout_status_codes(const MRTaskRolloutHandle* handle);
/* reference: include/metalrobo/c_api.h:685-687.  [step][env] of the last advance. */
MR_API const uint32_t* mr_task_rollout_active_contacts(const MRTaskRolloutHandle* handle);
/* reference: include/metalrobo/c_api.h:688-690.  [step][env][nq + nv] of the
 * last advance; null unless state readback is enabled. */
MR_API const float* mr_task_rollout_actor_observations(const MRTaskRolloutHandle* handle);
/* reference: include/metalrobo/c_api.h:736-738.  [env][nq]; null unless
 * state readback is enabled. */
MR_API const float* mr_task_rollout_final_q(const MRTaskRolloutHandle* handle);

/* ---------------------------------------------------------------------- */
/* Native policy (reference: include/metalrobo/c_api.h:326-372, 597-616,   */
/* 722-735; src/metal/PolicyInference.metal)                               */
/* ---------------------------------------------------------------------- */

/* reference: c_api.h:326-332 (same values). */
typedef enum MRPolicyActivationC {
    MR_POLICY_ACTIVATION_C_IDENTITY = 0,
    MR_POLICY_ACTIVATION_C_RELU = 1,
    MR_POLICY_ACTIVATION_C_TANH = 2,
    MR_POLICY_ACTIVATION_C_ELU = 3,
    MR_POLICY_ACTIVATION_C_SILU = 4
} MRPolicyActivationC;

/* reference: c_api.h:334-342 (same shape).  weights [output][input]. */
typedef struct MRPolicyDenseLayerC {
    uint32_t input_count;
    uint32_t output_count;
    uint32_t activation;
    const float* weights;
    size_t weight_count;
    const float* bias;
    size_t bias_count;
} MRPolicyDenseLayerC;

/* reference: c_api.h:344-372 (same shape).  The actor maps the actor
 * observation ([q, v], nq + nv values; normalised and clipped to
 * +-observation_clip when a mean is given) to the action mean; actions are
 * clamp(action_scale * latent + action_bias, +-action_clip), the latent
 * being the mean, plus exp(log sigma) times a standard normal draw when
 * action_log_standard_deviation is given.  The optional critic (one output)
 * gives the value.  Layers are at most 256 wide, at most 8 deep.  The
 * fingerprints and contract version are kept and not checked: this
 * library's worlds are synthetic. */
typedef struct MRPolicyPackC {
    const char* id;
    uint64_t revision;
    uint64_t contract_version;
    uint64_t world_fingerprint;
    uint64_t task_fingerprint;
    uint64_t observation_fingerprint;
    uint64_t action_fingerprint;
    const float* observation_mean;
    size_t observation_mean_count;
    const float* observation_inverse_standard_deviation;
    size_t observation_inverse_standard_deviation_count;
    const MRPolicyDenseLayerC* layers;
    size_t layer_count;
    const float* critic_observation_mean;
    size_t critic_observation_mean_count;
    const float* critic_observation_inverse_standard_deviation;
    size_t critic_observation_inverse_standard_deviation_count;
    const MRPolicyDenseLayerC* critic_layers;
    size_t critic_layer_count;
    const float* action_log_standard_deviation;
    size_t action_log_standard_deviation_count;
    const float* action_bias;
    size_t action_bias_count;
    const float* action_scale;
    size_t action_scale_count;
    float observation_clip;
    float action_clip;
} MRPolicyPackC;

/* Persisted PolicyPacks (reference: c_api.h:562-573, 604-608; the file is
 * numi-lab's learning-pack container, src/core/LearningPacks.cpp: a 32-byte
 * header -- "MRLEARN\0", format version, kind 2, payload bytes, FNV-1a 64
 * payload hash -- and the policy fields in MRPolicyPackC order).
 * mr_write_policy_pack validates the pack (identity, non-zero revision, an
 * exact contract: version 1 and non-zero fingerprints, positive finite
 * clips, layer shapes, finite values, a critic for a stochastic actor) and
 * writes a version-4 file atomically.  mr_learning_pack_content_hash is the
 * payload hash.  mr_task_rollout_load_policy_pack reads a version 3 or 4
 * file, applies the same rules and installs the policy as
 * mr_task_rollout_set_policy does; a failed load leaves the installed
 * policy unchanged.  Version-3 packs carry no contract and are refused, as
 * the reference refuses them outside its migration path.  The contract's
 * fingerprints are kept, not compared: this library's worlds are synthetic
 * and carry no task program. */
MR_API int mr_write_policy_pack(const MRPolicyPackC* policy, const char* policy_pack_path);
MR_API uint64_t mr_learning_pack_content_hash(const void* payload, size_t byte_count);
MR_API int mr_task_rollout_load_policy_pack(MRTaskRolloutHandle* handle, const char* policy_pack_path);

/* No counterpart in the reference: reads a PolicyPack file without a
 * device (header and payload checks as above, without the artifact rules)
 * and reports its fields; with `parameters` non-null also copies every FP32
 * table in file order (actor normalisation, actor layers' weights and bias,
 * critic normalisation, critic layers, action log sigma, bias, scale). */
typedef struct MRPolicyPackInfoC {
    uint32_t format_version;
    uint32_t layer_count;
    uint32_t critic_layer_count;
    uint32_t observation_count;     /* inputs of the first actor layer  */
    uint32_t action_count;          /* outputs of the last actor layer  */
    uint32_t stochastic;            /* action log sigma present         */
    uint64_t revision;
    uint64_t content_hash;
    uint64_t contract_version;
    uint64_t world_fingerprint;
    uint64_t task_fingerprint;
    uint64_t observation_fingerprint;
    uint64_t action_fingerprint;
    uint64_t parameter_count;       /* FP32 values in all tables        */
    float observation_clip;
    float action_clip;
    char id[64];                    /* truncated, NUL-terminated        */
} MRPolicyPackInfoC;
MR_API int mr_policy_pack_inspect(const char* policy_pack_path, MRPolicyPackInfoC* info, float* parameters,
                                  size_t parameter_capacity);

/* reference: c_api.h:597-603.  Copies every span; later advances take no
 * action stream (action count 0) and evaluate the policy on the device
 * before each control step, from the resident state. */
MR_API int mr_task_rollout_set_policy(MRTaskRolloutHandle* handle, const MRPolicyPackC* policy);
/* reference: c_api.h:610-614.  0 when no policy is installed. */
MR_API uint64_t mr_task_rollout_policy_revision(const MRTaskRolloutHandle* handle);
/* reference: c_api.h:615-616. */
MR_API int mr_task_rollout_clear_policy(MRTaskRolloutHandle* handle);
/* reference: c_api.h:722-735.  Outputs of the last policy-driven advance:
 * latents [step][env][action], log-probabilities and values [step][env],
 * bootstrap values [env] (the critic on the final state when the advance
 * asked for evaluate_final_policy; zeros without a critic).  Null when the
 * last advance ran no policy. */
MR_API const float* mr_task_rollout_policy_latents(const MRTaskRolloutHandle* handle);
MR_API const float* mr_task_rollout_policy_log_probabilities(const MRTaskRolloutHandle* handle);
MR_API const float* mr_task_rollout_policy_values(const MRTaskRolloutHandle* handle);
MR_API const float* mr_task_rollout_bootstrap_policy_values(const MRTaskRolloutHandle* handle);
/* reference: include/metalrobo/c_api.h:742-746.  Packed [env][scene body]
 * [position xyz, orientation xyzw, linear xyz, angular xyz]; scene bodies
 * are the free bodies of the pile and stack worlds. */
MR_API int mr_task_rollout_copy_final_scene_states(
    const MRTaskRolloutHandle* handle, float* output, size_t output_count);

/* ---------------------------------------------------------------------- */
/* PolicyRolloutPack files (reference: c_api.h:374-394, 750-755;           */
/* include/metalrobo/LearningPacks.hpp:54-105, src/core/LearningPacks.cpp) */
/* ---------------------------------------------------------------------- */

typedef struct MRTaskTransitionC MRTaskTransitionC;

/* reference: c_api.h:374-394 (same shape).  Tables [control step][env]
 * (x features); teacher actions and motion features may be empty. */
typedef struct MRPolicyRolloutBatchC {
    uint32_t control_step_count;
    const float* actor_observations;
    size_t actor_observation_count;
    const float* critic_observations;
    size_t critic_observation_count;
    const float* motion_features;
    size_t motion_feature_count;
    const float* teacher_actions;
    size_t teacher_action_count;
    const float* latents;
    size_t latent_count;
    const float* log_probabilities;
    size_t log_probability_count;
    const float* values;
    size_t value_count;
    const float* bootstrap_values;
    size_t bootstrap_value_count;
    const MRTaskTransitionC* transitions;
    size_t transition_count;
} MRPolicyRolloutBatchC;

/* No counterpart in the reference's C ABI (its PolicyRolloutPackView,
 * LearningPacks.hpp:83-105, without the outcome schema): a rollout pack
 * written without a rollout. */
typedef struct MRPolicyRolloutPackC {
    const char* id;
    uint64_t task_fingerprint;
    uint64_t policy_fingerprint;
    uint64_t policy_revision;
    uint32_t environment_count;
    uint32_t actor_observation_count;
    uint32_t critic_observation_count;
    uint32_t action_count;
    uint32_t motion_feature_count;
    uint32_t reserved;
    const MRPolicyRolloutBatchC* batch;
} MRPolicyRolloutPackC;

typedef struct MRPolicyRolloutPackInfoC {
    uint64_t task_fingerprint;
    uint64_t policy_fingerprint;
    uint64_t policy_revision;
    uint64_t content_hash;
    uint32_t environment_count;
    uint32_t control_step_count;
    uint32_t actor_observation_count;
    uint32_t critic_observation_count;
    uint32_t action_count;
    uint32_t motion_feature_count;
    uint32_t outcome_count;
    uint32_t has_teacher_actions;
    uint64_t transition_count;
    double reward_sum;              /* over every transition */
    uint64_t done_count;
    char id[64];                    /* truncated, NUL-terminated */
} MRPolicyRolloutPackInfoC;

/* reference: c_api.h:750-755.  Publishes a batch collected from this
 * rollout: fingerprints, revision and dimensions come from the installed
 * task and policy (a policy is required; the task's actor frame is both
 * the actor and the critic observation; no outcome schema).  Task
 * transitions become learner transitions (reward and timeout bootstrap,
 * termination, context, revision) as c_api.cpp:4410-4445 does. */
MR_API int mr_task_rollout_write_policy_rollout_pack(const MRTaskRolloutHandle* handle, const MRPolicyRolloutBatchC* batch,
                                                     const char* batch_id, const char* output_path);
/* No counterpart in the reference: the same file from explicit identity,
 * fingerprints and dimensions; the artifact rules of the reference's
 * writer (LearningPacks.cpp:726-918) apply. */
MR_API int mr_write_policy_rollout_pack(const MRPolicyRolloutPackC* pack, const char* output_path);
/* No counterpart in the reference: reads and checks a PolicyRolloutPack;
 * `parameters` (optional, `capacity` floats) receives the actor
 * observations, latents, log-probabilities, values and bootstrap values in
 * that order. */
MR_API int mr_policy_rollout_pack_inspect(const char* path, MRPolicyRolloutPackInfoC* info, float* parameters, size_t capacity);

/* ---------------------------------------------------------------------- */
/* TaskPack files (reference: include/metalrobo/TaskProgram.hpp:442-500,   */
/* src/core/LearningPacks.cpp:81-258, 1127-1412, 2300-2345)                */
/* ---------------------------------------------------------------------- */

/* No counterpart in the reference's C ABI: the authored task's tables and
 * the episode constants of a TaskPack file. */
typedef struct MRTaskPackInfoC {
    uint64_t content_hash;
    uint32_t action_count;
    uint32_t outcome_count;
    uint32_t contact_group_count;
    uint32_t joint_group_count;
    uint32_t reward_count;
    uint32_t termination_count;
    uint32_t maximum_episode_steps;
    uint32_t difficulty_band_count;
    uint32_t terrain_sample_count;
    uint32_t motion_tracked_body_count;
    float base_height_target;
    float gait_period_seconds;
    float clearance_target;
    float support_force_threshold;
    char id[64];                    /* truncated, NUL-terminated */
} MRTaskPackInfoC;

/* No counterpart in the reference: reads a TaskPack (kind 1, version 17). */
MR_API int mr_task_pack_inspect(const char* path, MRTaskPackInfoC* info);
/* No counterpart in the reference: reads a TaskPack, checks the artifact
 * rules of the reference's writer and writes it to output_path (atomic:
 * temporary, fsync, rename); the bytes equal the reference writer's. */
MR_API int mr_task_pack_rewrite(const char* input_path, const char* output_path);

/* ---------------------------------------------------------------------- */
/* Task layer (reference: include/metalrobo/task_program_types.h,         */
/* src/metal/LocomotionTask.metal observe / apply_actions / complete)      */
/* ---------------------------------------------------------------------- */

/* Operator codes: the reference's MRTaskObservationOpcode,
 * MRTaskRewardOpcode, MRTaskTerminationOpcode, MRTaskTerminationReason and
 * MRTaskRandomizationOpcode (task_program_types.h:68-300), same values.
 * The task layer evaluates the subset listed here; mr_task_rollout_set_task
 * refuses any other code.  A translation unit that already included the
 * reference's task_program_types.h (which defines
 * MR_TASK_PROGRAM_ABI_VERSION) keeps its identical definitions. */
#ifndef MR_TASK_PROGRAM_ABI_VERSION
enum {
    MR_TASK_OBSERVE_ROOT_ANGULAR_VELOCITY_LOCAL = 0u,
    MR_TASK_OBSERVE_PROJECTED_GRAVITY = 1u,
    MR_TASK_OBSERVE_COMMAND = 2u,
    MR_TASK_OBSERVE_JOINT_POSITION_ERROR = 3u,
    MR_TASK_OBSERVE_JOINT_VELOCITY = 4u,
    MR_TASK_OBSERVE_PREVIOUS_ACTION = 5u,
    MR_TASK_OBSERVE_ROOT_LINEAR_VELOCITY_LOCAL = 6u,
    MR_TASK_OBSERVE_ROOT_HEIGHT = 7u,
    MR_TASK_OBSERVE_CONTACT_METRIC = 8u,
    MR_TASK_OBSERVE_CONTACT_WRENCH_LOCAL = 13u,
    MR_TASK_OBSERVE_GAIT_PHASE = 14u,
    MR_TASK_OBSERVE_SUPPORT_SENSE = 18u,
    MR_TASK_OBSERVE_DELAYED_ACTION = 26u,
    MR_TASK_OBSERVE_JOINT_FINITE_DIFFERENCE_VELOCITY = 27u
};
enum { MR_TASK_OBSERVATION_NORMALIZE_VECTOR3 = 1u };
enum { MR_TASK_CONTACT_SUPPORT = 1u, MR_TASK_CONTACT_FORBIDDEN = 2u };
enum {
    MR_TASK_REWARD_LINEAR_VELOCITY_TRACKING = 0u,
    MR_TASK_REWARD_YAW_VELOCITY_TRACKING = 1u,
    MR_TASK_REWARD_CONSTANT = 2u,
    MR_TASK_REWARD_ROOT_VERTICAL_VELOCITY_SQUARED = 3u,
    MR_TASK_REWARD_ROOT_ROLL_PITCH_VELOCITY_SQUARED = 4u,
    MR_TASK_REWARD_TILT_SQUARED = 5u,
    MR_TASK_REWARD_ROOT_HEIGHT_ERROR_SQUARED = 6u,
    MR_TASK_REWARD_JOINT_VELOCITY_SQUARED = 7u,
    MR_TASK_REWARD_JOINT_ACCELERATION_SQUARED = 8u,
    MR_TASK_REWARD_ACTION_RATE_SQUARED = 9u,
    MR_TASK_REWARD_JOINT_LIMIT_VIOLATION_SQUARED = 10u,
    MR_TASK_REWARD_JOINT_GROUP_POSTURE_SQUARED = 12u,
    MR_TASK_REWARD_GAIT_CONTACT_MATCH = 13u,
    MR_TASK_REWARD_SWING_CLEARANCE = 14u,
    MR_TASK_REWARD_SUPPORT_SLIP = 15u,
    MR_TASK_REWARD_FORBIDDEN_CONTACT = 16u,
    MR_TASK_REWARD_JOINT_GROUP_POSTURE_ABSOLUTE = 17u,
    MR_TASK_REWARD_PROJECTED_GRAVITY_HORIZONTAL_SQUARED = 18u,
    MR_TASK_REWARD_FOOT_CLEARANCE = 19u,
    MR_TASK_REWARD_JOINT_LIMIT_VIOLATION_ABSOLUTE = 20u,
    MR_TASK_REWARD_ROOT_HEIGHT_NORMALIZED = 21u,
    MR_TASK_REWARD_ROOT_HEIGHT_PROGRESS = 22u,
    MR_TASK_REWARD_UPRIGHTNESS = 23u
};
enum {
    MR_TASK_TERMINATE_MINIMUM_ROOT_HEIGHT = 0u,
    MR_TASK_TERMINATE_MAXIMUM_TILT = 1u,
    MR_TASK_TERMINATE_CONTACT_GROUP = 2u
};
enum {
    MR_TASK_TERMINATION_CONTINUING = 0u,
    MR_TASK_TERMINATION_HEIGHT = 1u,
    MR_TASK_TERMINATION_TILT = 2u,
    MR_TASK_TERMINATION_CONTACT = 3u,
    MR_TASK_TERMINATION_TIMEOUT = 4u,
    MR_TASK_TERMINATION_PHYSICS_ERROR = 5u
};
enum {
    MR_TASK_RANDOMIZE_ROOT_POSITION = 0u,
    MR_TASK_RANDOMIZE_ROOT_YAW = 1u,
    MR_TASK_RANDOMIZE_ACTION_POSITION = 2u,
    MR_TASK_RANDOMIZE_VELOCITY = 3u,
    MR_TASK_RANDOMIZE_ACTION_DELAY = 7u,
    MR_TASK_RANDOMIZE_OBSERVATION_DELAY = 8u,
    MR_TASK_RANDOMIZE_ACTION_VELOCITY = 9u,
    MR_TASK_RANDOMIZE_ROOT_HEIGHT = 10u,
    MR_TASK_RANDOMIZE_JOINT_POSITION = 12u
};
#endif /* MR_TASK_PROGRAM_ABI_VERSION */

/* reference: MRTaskActionBindingGPU (task_program_types.h:443-458), the
 * joint-position actuator.  Action `index` of the policy sets the drive
 * target of DoF `dof_index` (its coordinate q_index, velocity v_index):
 * clamp(default_q[q_index] + scale x filtered action, lower_target,
 * upper_target), the filtered action following the delayed raw action with
 * a first-order response of `response_time_seconds` (0: none). */
typedef struct MRTaskActionBindingC {
    uint32_t dof_index;
    uint32_t q_index;
    uint32_t v_index;
    uint32_t reserved;
    float scale;
    float lower_target;
    float upper_target;
    float response_time_seconds;
} MRTaskActionBindingC;

/* reference: MRTaskObservationOperatorGPU (:460-467).  One actor
 * observation: transform_scale x source + transform_offset, plus
 * noise_amplitude x a uniform draw in [-1, 1] on noise_channel.  `source`
 * is the action index for joint sources; `component` the vector lane (for
 * DELAYED_ACTION: how many raw actions back). */
typedef struct MRTaskObservationOperatorC {
    uint32_t opcode;
    uint32_t source;
    uint32_t component;
    uint32_t flags;
    float transform_scale;
    float transform_offset;
    float noise_amplitude;
    uint32_t noise_channel;
} MRTaskObservationOperatorC;

/* reference: MRTaskRewardOperatorGPU (:496-504).  The step's reward is
 * control_dt x sum(weight x value). */
typedef struct MRTaskRewardOperatorC {
    uint32_t opcode;
    uint32_t group;      /* joint group of the posture rewards; contact group of
                            the contact rewards (MR_INVALID_INDEX: every group) */
    float weight;
    float parameters[3]; /* the reference's parameters.yzw */
} MRTaskRewardOperatorC;

/* reference: MRTaskTerminationOperatorGPU (:506-513). */
typedef struct MRTaskTerminationOperatorC {
    uint32_t opcode;
    uint32_t reason;
    uint32_t priority;
    uint32_t group;      /* contact group of CONTACT_GROUP */
    float threshold;
    float failure_penalty;
    uint32_t minimum_band;   /* active in episodes of bands [minimum_band, maximum_band] */
    uint32_t maximum_band;   /* MR_INVALID_INDEX: the last band */
} MRTaskTerminationOperatorC;

/* reference: MRTaskRandomizationOperatorGPU (:515-520); `target` is the q
 * index of JOINT_POSITION. */
typedef struct MRTaskRandomizationOperatorC {
    uint32_t opcode;
    uint32_t target;
    uint32_t minimum_band;   /* inactive in episodes of a lower difficulty band */
    uint32_t reserved;
    float parameters[4];
} MRTaskRandomizationOperatorC;

/* reference: MRTaskIndexGroupGPU (:491-494): action indices
 * joint_members[first, first + count). */
typedef struct MRTaskIndexGroupC {
    uint32_t first;
    uint32_t count;
} MRTaskIndexGroupC;

/* reference: MRTaskContactGroupGPU (:469-489), without support patches.
 * Bodies contact_members[first, first + count) (articulated body indices).
 * Per step the group publishes, from the final microstep's contacts of its
 * bodies with the ground: support groups the normal force (sum of normal
 * impulses / physics dt), the slip (planar speed of the kinematic
 * reference point while in contact), the air time, the clearance of the
 * reference point above the ground less its radius and the centre of
 * pressure in the reference body's frame; forbidden groups 1 when a contact
 * pushes harder than the support force threshold; every group the contact
 * wrench (force and torque about the reference point) in the reference
 * body's frame. */
typedef struct MRTaskContactGroupC {
    uint32_t first;
    uint32_t count;
    uint32_t flags;                 /* MR_TASK_CONTACT_SUPPORT / _FORBIDDEN */
    uint32_t reference_body;
    float local_reference[4];       /* point from the reference body's COM, its axes; w clearance radius */
    float kinematic_reference[4];   /* link-frame origin from the COM, its axes */
    float gait_phase_offset;        /* radians */
    float stance_fraction;
    float reserved[2];
} MRTaskContactGroupC;

/* A compiled task program: the tables and constants of the reference's
 * MRTaskProgramHeaderGPU (:358-441) that the evaluated subset reads.  A
 * stacked actor history without observation delay, one difficulty band, a
 * flat ground; no terrain, pushes, support patches or sensor biases. */
typedef struct MRTaskProgramC {
    const MRTaskActionBindingC* actions;
    uint32_t action_count;          /* equals the world's action count */
    const MRTaskObservationOperatorC* actor;
    uint32_t actor_count;
    const MRTaskObservationOperatorC* critic;  /* the critic's frame (program.counts0.z): clean values, no
                                                  noise; 0 operators: the critic reads the actor history */
    uint32_t critic_count;
    const MRTaskRewardOperatorC* rewards;
    uint32_t reward_count;
    const MRTaskTerminationOperatorC* terminations;
    uint32_t termination_count;
    const MRTaskRandomizationOperatorC* randomization;
    uint32_t randomization_count;
    const MRTaskIndexGroupC* joint_groups;
    uint32_t joint_group_count;
    const uint32_t* joint_members;
    uint32_t joint_member_count;
    const MRTaskContactGroupC* contact_groups;  /* at most 8 */
    uint32_t contact_group_count;
    const uint32_t* contact_members;
    uint32_t contact_member_count;
    float support_force_threshold;  /* program.dynamics.y, newtons */
    float clearance_target;         /* program.locomotion.z, metres */
    const float* default_q;         /* [nq]: the reset pose and posture reference */
    uint32_t default_q_count;
    uint32_t maximum_episode_steps; /* timeout */
    uint32_t action_history;        /* delay-line slots including the filter slot, 3..8 */
    uint32_t action_delay_steps;    /* an episode's action delay without an ACTION_DELAY operator;
                                       at most action_history - 2 take effect */
    uint32_t observation_history;   /* actor frames stacked, oldest first (program.layout.y), 1..8 */
    uint32_t maximum_observation_delay; /* program.schedule.y: the OBSERVATION_DELAY draw's ceiling */
    float base_height_target;       /* program.locomotion.x */
    float gait_period_seconds;      /* program.locomotion.y */
    float root_reference[3];        /* root link origin from the root's q position, root axes */
    float command_lower[3];         /* x, y velocity and yaw rate, band 0 */
    float command_upper[3];
    float standing_probability;     /* a drawn command is zeroed with it */
    float command_duration_seconds[2];
    uint32_t difficulty_band_count; /* program.schedule.z; an episode draws its band (0 for one band) */
    float band_sampling_exponent;   /* band = floor(u^exponent x bands) over the configuration's band range */
    float command_limit_lower[3];   /* each band widens the command range by command_band_step, within these limits */
    float command_limit_upper[3];
    float command_band_step[3];
    uint64_t task_fingerprint;
} MRTaskProgramC;

/* reference: include/metalrobo/c_api.h:261-295 (same layout, 128 bytes). */
struct MRTaskTransitionC {
    float reward;
    float tracking_score;
    float root_height;
    float tilt;
    uint32_t done;
    uint32_t timeout;
    uint32_t physics_error;
    uint32_t termination_reason;
    float task_reward;
    float base_reward;
    float joint_velocity_reward;
    float joint_acceleration_reward;
    float control_reward;
    float posture_reward;
    float energy_reward;
    float contact_reward;
    float task_outcome_channel_0;
    float task_outcome_channel_1;
    float task_outcome_channel_2;
    float task_outcome_channel_3;
    float task_outcome_channel_4;
    float task_outcome_channel_5;
    float task_outcome_channel_6;
    float task_outcome_channel_7;
    uint64_t policy_revision;
    float timeout_bootstrap_value;
    float episode_tracking_score;
    uint32_t difficulty_band;
    uint32_t terrain_level;
    uint32_t impact_sequence_index;
    uint32_t impact_event_flags;
};

/* No counterpart in the reference's C ABI, which compiles its task from the
 * run manifest's TaskPack; this installs a compiled task program on an
 * articulated rollout (the synthetic sources).  From the next advance each
 * control step runs, per environment: observe (a pending reset draws the
 * reset state from default_q and the randomization operators, starts an
 * episode and a command, and writes the actor frame of the reset state);
 * the policy, when one is installed, on that frame; apply (actions through
 * the bindings to drive targets); the physics step; complete (rewards,
 * terminations, timeout, the next command and the next actor frame).
 * Observations become the actor frames the step's actions were taken on
 * (observation_history x actor_count values, the oldest frame first),
 * actions the policy's normalised outputs.  Every
 * environment starts a new episode at the next advance.  Refused: an
 * operator outside the subset above, an index out of range, a pile or
 * stack world. */
MR_API int mr_task_rollout_set_task(MRTaskRolloutHandle* handle, const MRTaskProgramC* task);
/* No counterpart in the reference: removes the task (raw PD targets and
 * [q, v] observations again). */
MR_API int mr_task_rollout_clear_task(MRTaskRolloutHandle* handle);
/* reference: c_api.h:700-702.  [step][env] of the last advance; null
 * without a task or before the first advance. */
MR_API const MRTaskTransitionC* mr_task_rollout_transitions(const MRTaskRolloutHandle* handle);
/* No counterpart in the reference: device address of the last advance's
 * transitions ([step][env], valid until the next advance), 0 without a
 * task. */
MR_API uint64_t mr_task_rollout_device_transitions(const MRTaskRolloutHandle* handle);
/* No counterpart in the reference: copies the first `count` transitions of
 * the last advance ([step][env]) into host memory after its work finished;
 * count must not exceed its steps x environments. */
MR_API int mr_task_rollout_copy_transitions(const MRTaskRolloutHandle* handle, MRTaskTransitionC* output, size_t count);

/* ---------------------------------------------------------------------- */
/* Additions of this library                                               */
/* ---------------------------------------------------------------------- */

/* No counterpart in the reference: arithmetic precision of the microstep.
 * MR_PRECISION_FP32 (default) keeps the whole microstep in FP32 like the
 * reference; MR_PRECISION_FP64_ARTICULATED_INERTIA carries the articulated
 * inertias, their joint pivots and the floating root's 6x6 factorisation in
 * FP64 (state, contacts and the cone solve stay FP32);
 * MR_PRECISION_COMPENSATED adds to that compensated (Kahan) FP32 sums for the
 * position integration -- joint coordinates, the floating root's and free
 * bodies' positions, whose compensation terms persist across control steps
 * beside the resident state -- and for the impulse accumulation of the cone
 * solve's sweeps.  Piles and stacks have no articulated inertia: there the
 * FP64 mode equals FP32 and the compensated mode adds only the sums.
 * Applies to the next advance; a change of mode, a reset and set_state
 * clear the compensation terms. */
enum MRPrecisionModeC {
    MR_PRECISION_FP32 = 0u,
    MR_PRECISION_FP64_ARTICULATED_INERTIA = 1u,
    MR_PRECISION_COMPENSATED = 2u
};
MR_API int mr_task_rollout_set_precision(MRTaskRolloutHandle* handle, uint32_t mode);

/* Contact solver of a rollout (reference: MetalWorldSolverMode,
 * include/metalrobo/MetalWorld.hpp:31-39, and MetalWorldQualityConfig,
 * :41-52).  MR_SOLVER_TEMPORAL_CONE (default) runs the fixed-budget
 * temporalCone sweeps; MR_SOLVER_QUALITY_NEWTON solves every substep's
 * contact problem to convergence instead:
 *
 *   min 0.5 l' (G H^-1 G' + R) l + (G v_free - v_target)' l
 *   s.t. l_n >= 0, ||l_t|| <= mu l_n
 *
 * with R = max(the ConstraintIR regularisation, regularization_floor) per
 * row (the reference's CPU world uses minimumRegularization 1e-6,
 * ArticulatedWorld.hpp:58), in FP64, by a semismooth Newton iteration with
 * a direct (Cholesky) solve of its nv x nv system and an exact line search.
 * The optimality measure is ||zeta - Y l|| / (1 + ||zeta|| + ||Y l||)
 * (inf-norms) for the factor rows Y of G H^-1 G' = Y'Y and zeta the
 * iterate (zeta = Y l at the solution).  A solve
 * that does not reach `optimality_tolerance` within the budgets latches
 * MR_STEP_DID_NOT_CONVERGE and the environment keeps its checkpoint, like
 * any failed step.  Articulated contact worlds only (tree29); pile and
 * stack worlds and batched rollouts keep temporalCone.  Zero / non-positive
 * fields take the defaults in brackets.  Applies from the next advance. */
typedef struct MRQualitySolverConfigC {
    uint32_t maximum_newton_iterations;        /* [100]                                       */
    uint32_t maximum_line_search_iterations;   /* [50] line-search evaluations per Newton step */
    double optimality_tolerance;               /* [1e-9] on the optimality measure above       */
    double line_search_tolerance;              /* [0.1] |phi'(t)| relative to |phi'(0)|        */
    double regularization_floor;               /* [1e-6] per-row minimum of R                  */
    double reserved;
} MRQualitySolverConfigC;
MR_API int mr_task_rollout_set_solver(MRTaskRolloutHandle* handle, uint32_t solver, const MRQualitySolverConfigC* quality);

/* Certificates of the last advance's quality solves (all zero under
 * temporalCone): the most Newton steps of one solve, the line-search
 * evaluations summed, and the largest scaled optimality residual, cone
 * violation max(-l_n, ||l_t|| - mu l_n) and conic complementarity
 * |l' (G v - v_target + R l)| over every environment-substep (reference:
 * MRUnifiedQualityStatusGPU certificates, unified_quality_shared.h:124-146). */
typedef struct MRQualityDiagnosticsC {
    uint32_t maximum_newton_iterations;
    uint32_t line_search_iterations;
    float maximum_scaled_optimality;
    float maximum_cone_violation;
    float maximum_complementarity;
    uint32_t reserved[3];
} MRQualityDiagnosticsC;
MR_API int mr_task_rollout_quality_diagnostics(const MRTaskRolloutHandle* handle, MRQualityDiagnosticsC* out);

/* Batched converged contact solve of independent dense problems (reference:
 * solveMetalUnifiedQuality, include/metalrobo/MetalUnifiedQualitySolver.hpp:
 * 85-90, whose problems also carry the dynamics operator and the Jacobian
 * rather than the Delassus matrix).  Problem p has `nv` generalized
 * velocities and contact_counts[p] (or, with null, `contact_capacity`)
 * contacts; arrays are problem-major with the capacity as stride:
 *   mass            [p][nv][nv]   symmetric positive definite H
 *   jacobian        [p][3 cap][nv] rows normal, tangent, bitangent per contact
 *   free_velocity   [p][nv]
 *   target_velocity, regularization, warm_impulses (may be null): [p][3 cap]
 *   friction        [p][cap]      mu >= 0 (0: frictionless)
 * The two tangent regularisations of a frictional contact must be equal.
 * Solves on the current device in FP64 (one warp per problem; 1 <= nv <= 64,
 * cap <= 32) with the settings of `config` (null: defaults) and writes the
 * impulses [p][3 cap], the post-impulse velocity v_free + H^-1 G' l [p][nv]
 * and one result per problem (host arrays; the call is synchronous). */
typedef struct MRQualityResultC {
    uint32_t code;                 /* MRStepStatusCode: SUCCESS, DID_NOT_CONVERGE, FACTORIZATION_FAILED, NONFINITE_RESULT */
    uint32_t newton_iterations;
    uint32_t line_search_iterations;
    uint32_t reserved;
    double scaled_optimality;
    double cone_violation;
    double complementarity;
    double objective;              /* dual objective of the returned impulses */
} MRQualityResultC;
MR_API int mr_quality_solve_batch(
    uint32_t problem_count,
    uint32_t nv,
    uint32_t contact_capacity,
    const uint32_t* contact_counts,
    const double* mass,
    const double* jacobian,
    const double* free_velocity,
    const double* target_velocity,
    const double* regularization,
    const double* friction,
    const double* warm_impulses,
    const MRQualitySolverConfigC* config,
    double* impulses,
    double* velocity,
    MRQualityResultC* results);

/* No counterpart in the reference: zero-copy advance for device buffers
 * (e.g. torch CUDA tensors).  `device_actions` [step][env][action] and the
 * optional `device_reset_masks` [step][env] live on the rollout's device;
 * `device_observations` [step][env][nq+nv] and `device_status_codes`
 * [step][env] may be null.  The control steps run after all work already
 * enqueued on `cuda_stream` (a cudaStream_t; 0 = the legacy default
 * stream), and work enqueued on it afterwards runs after them.  With
 * `advance` non-null the call waits and fills the same counters as
 * mr_task_rollout_advance; with null it returns after enqueueing. */
MR_API int mr_task_rollout_advance_device(
    MRTaskRolloutHandle* handle,
    const float* device_actions,
    const uint32_t* device_reset_masks,
    uint32_t control_step_count,
    float* device_observations,
    uint32_t* device_status_codes,
    uint64_t cuda_stream,
    MRTaskRolloutAdvanceC* advance);

/* No counterpart in the reference: copies the compiled world records. */
MR_API int mr_task_rollout_copy_model(const MRTaskRolloutHandle* handle, MRModelViewC* view);

/* No counterpart in the reference: compiles a synthetic world on the host
 * (no device work) and copies its records into `view` (null tables are
 * skipped; `view->world` always receives the counts). */
MR_API int mr_compile_synthetic_model(uint32_t source, uint64_t seed, MRModelViewC* view);

/* No counterpart in the reference: samples the reset state the rollout
 * would use for environments [env_begin, env_begin + env_count) (host only).
 * q [env][nq], v [env][nv], friction_scale [env]. */
MR_API int mr_sample_synthetic_reset(uint32_t source, uint64_t model_seed, uint64_t reset_seed,
                                     uint32_t env_begin, uint32_t env_count, float* q, float* v,
                                     float* friction_scale);

/* No counterpart in the reference: per-environment contact friction scale
 * [env] (the synthetic worlds draw one coefficient per environment). */
MR_API int mr_task_rollout_copy_environment_parameters(
    const MRTaskRolloutHandle* handle, float* friction_scale);

/* No counterpart in the reference: the control-step kernel's launch shape
 * for the current precision mode (environments per CTA and resident
 * environments per SM, from the occupancy query at creation; 1 and 0 for
 * pile and stack worlds, whose kernel runs one environment per CTA). */
MR_API int mr_task_rollout_launch_shape(const MRTaskRolloutHandle* handle, uint32_t* warps_per_block,
                                        uint32_t* resident_warps_per_sm);
/* No counterpart in the reference: how many environment chains an
 * articulated advance runs as (contiguous blocks of
 * environments, each a chain of per-step launches on its own stream inside
 * the advance's graph; launches per control step = chains). */
MR_API uint32_t mr_task_rollout_environment_chains(const MRTaskRolloutHandle* handle);

/* No counterpart in the reference: copies the resident state of every
 * environment, q [env][nq], v [env][nv] and manifolds [env][pair_count];
 * any pointer may be null.  Pile worlds (scene bodies) store instead a
 * table of MR_B200_SCENE_MANIFOLDS slots per environment, each one
 * MRManifoldC followed by its pair key (a * 65 + b; b = body count for the
 * ground plane) as a uint32 word, live slots first in ascending key order
 * (MR_B200_SCENE_SLOT_WORDS floats per slot). */
MR_API int mr_task_rollout_copy_state(
    const MRTaskRolloutHandle* handle, float* q, float* v, MRManifoldC* manifolds);

/* No counterpart in the reference: a per-environment FP64 energy and
 * momentum audit.  While enabled, a kernel after every control step adds
 * each body's kinetic energy, potential energy (-m g . c), linear momentum
 * and angular momentum about the world origin in FP64 from the committed
 * FP32 state (a failed step's checkpoint), reduced per environment in
 * FP64, into a resident record of 12
 * doubles: kinetic, potential, total, reference total (taken on the first
 * audited step after enabling, a reset, mr_task_rollout_reset or a new
 * state), largest |total - reference| so far, linear momentum xyz, angular
 * momentum xyz, audited steps since the reference.  Enabling allocates
 * [env][12] doubles.  Batch advances (mr_batch_advance) do not audit. */
MR_API int mr_task_rollout_set_audit(MRTaskRolloutHandle* handle, uint32_t enabled);
/* No counterpart in the reference: copies the audit records ([env][12]). */
MR_API int mr_task_rollout_copy_audit(const MRTaskRolloutHandle* handle, double* records, size_t count);

/* No counterpart in the reference (its islands, ConstraintSolver.cpp:848
 * and MetalWorldContact.metal:4002, are internal): while enabled, every
 * control step of a free-body (scene) world records the island partition
 * of its final substep's contacts, per environment and body: the island
 * index, islands numbered by ascending smallest body as
 * buildConstraintIslands numbers them, or 0xff for a body in no island.
 * Enabling allocates [env][64] bytes; only scene worlds accept it. */
MR_API int mr_task_rollout_set_island_labels(MRTaskRolloutHandle* handle, uint32_t enabled);
/* No counterpart in the reference: copies the labels of the last control
 * step ([env][64] bytes; entries beyond the body count are undefined;
 * meaningful for environments whose step succeeded). */
MR_API int mr_task_rollout_copy_island_labels(const MRTaskRolloutHandle* handle, uint8_t* labels, size_t count);

/* No counterpart in the reference: replaces the resident state (same
 * layouts as mr_task_rollout_copy_state; null manifolds clears them).
 * The new state also becomes every environment's reset state when
 * `as_reset_state` is non-zero. */
MR_API int mr_task_rollout_set_state(
    MRTaskRolloutHandle* handle, const float* q, const float* v,
    const MRManifoldC* manifolds, uint32_t as_reset_state);

/* ---------------------------------------------------------------------- */
/* Continuous-batching rollout server (no counterpart in the reference)   */
/* ---------------------------------------------------------------------- */

/* Requests of differing worlds, env counts and horizons are admitted into
 * resident environment slots as slots and the HBM budget allow, packed with
 * the requests already running into one control-step launch per world per
 * tick, and retired when their horizon completes.  An environment's result
 * depends only on its request (world, seed, env index, actions).  Worlds:
 * MR_RUN_SOURCE_SYNTHETIC_CHAIN7, _TREE29 and _PILE (no actions). */
typedef struct MRServerHandle MRServerHandle;

typedef struct MRServerConfigC {
    uint64_t hbm_budget_bytes;         /* slots + request actions              */
    uint64_t model_seed;               /* seed of the synthetic worlds         */
    uint32_t physics_substeps;
    uint32_t velocity_iterations;
    uint32_t final_velocity_iterations;
    float control_timestep_seconds;
    uint32_t max_envs_per_source;      /* slot pool size per world source      */
    uint32_t control_steps_per_tick;   /* control steps one tick advances (0: 1) */
} MRServerConfigC;

typedef struct MRServerRequestC {
    uint32_t source;                   /* MR_RUN_SOURCE_SYNTHETIC_*            */
    uint32_t env_count;
    uint32_t horizon;                  /* control steps                        */
    uint32_t reserved;
    uint64_t seed;                     /* reset sampling of the request's envs */
    const float* actions;              /* host [horizon][env][action], copied  */
} MRServerRequestC;

typedef struct MRServerCompletionC {
    uint64_t request_id;
    uint32_t source;
    uint32_t env_count;
    uint32_t horizon;
    uint32_t failed_env_steps;
    uint32_t first_failure_status;
    uint32_t reserved;
    double queue_seconds;              /* submit -> admission                  */
    double latency_seconds;            /* submit -> final state on the host    */
} MRServerCompletionC;

typedef struct MRServerStatsC {
    uint32_t pending_requests;
    uint32_t running_requests;
    uint32_t free_slots;
    uint32_t reserved;
    uint64_t completed_env_steps;
    uint64_t hbm_bytes_in_use;
} MRServerStatsC;

MR_API MRServerHandle* mr_create_server(const MRServerConfigC* config);
MR_API void mr_server_destroy(MRServerHandle* server);
/* Slot-pool size and action width of a world source. */
MR_API int mr_server_capacity(const MRServerHandle* server, uint32_t source, uint32_t* slots, uint32_t* action_count);
MR_API int mr_server_submit(MRServerHandle* server, const MRServerRequestC* request, uint64_t* request_id);
/* Admits waiting requests (slots and a range of the pool's preallocated
 * action arena: no device allocation), advances every admitted request by
 * control_steps_per_tick control steps (fewer when its horizon ends first;
 * one launch per pool and step, the pools on their own streams), retires
 * the finished ones, and synchronises once.  active_envs receives the
 * environment-steps this tick advanced. */
MR_API int mr_server_tick(MRServerHandle* server, uint32_t* active_requests, uint32_t* active_envs);
/* Completions not reported yet, oldest first. */
MR_API int mr_server_poll(MRServerHandle* server, MRServerCompletionC* out, uint32_t capacity, uint32_t* count);
/* Final q [env][nq] and v [env][nv] of a completed request (kept until released). */
MR_API int mr_server_copy_result(const MRServerHandle* server, uint64_t request_id, float* q, size_t q_count, float* v,
                                 size_t v_count);
MR_API int mr_server_release(MRServerHandle* server, uint64_t request_id);
MR_API int mr_server_stats(const MRServerHandle* server, MRServerStatsC* stats);

/* No counterpart in the reference.  Measures the current device's FP32 FMA
 * peak (TFLOP/s) and its warp-instruction issue rate (warp instructions per
 * second of FMA issue) with CUDA events: the denominators of the issue
 * roofline of the control-step kernels.  Synchronous; allocates 1 KB. */
MR_API int mr_measure_issue_peak(double* fma_tflops, double* warp_instructions_per_second);

/* ---------------------------------------------------------------------- */
/* Heterogeneous batch (no counterpart in the reference)                  */
/* ---------------------------------------------------------------------- */
/* The reference compiles one topology per context and dispatches each
 * world on its own.  A batch groups existing rollouts -- any mix of
 * articulated chains and trees and free-body piles of any body count, each
 * with its own substeps and iterations -- and advances all their
 * environments with ONE persistent launch per horizon of control steps
 * (or one per device-code family, MRBatchLaunchModeC): resident warps claim
 * (world, environment) items from a device queue in a claim order (longest
 * item first, or round robin over the worlds) and run that environment's
 * control steps back to back with its world's own device code;
 * environments never wait for each other.  The queue reset and the launches
 * are captured as one CUDA graph.  The rollouts keep owning their state; a batch stores
 * pointers to them (destroy the batch before its rollouts).  Rollouts must
 * be FP32 and without a native policy; a batch with support-mapped (GJK /
 * EPA) pairs runs per family. */
typedef struct MRBatchHandle MRBatchHandle;

enum MRBatchOrderC {
    MR_BATCH_ORDER_LONGEST_FIRST = 0u,
    MR_BATCH_ORDER_ROUND_ROBIN = 1u
};

/* FUSED: one kernel runs every item (register budget of the most demanding
 * world).  PER_FAMILY: one persistent launch per device-code family --
 * articulated and free-body -- running concurrently, each at its own
 * kernel's register budget and occupancy. */
enum MRBatchLaunchModeC {
    MR_BATCH_LAUNCH_FUSED = 0u,
    MR_BATCH_LAUNCH_PER_FAMILY = 1u
};

typedef struct MRBatchLaunchShapeC {
    uint32_t worlds;
    uint32_t items;                  /* environments over all rollouts */
    uint32_t warps_per_block;        /* fused / articulated launch */
    uint32_t blocks;                 /* persistent grid: SMs x resident CTAs */
    uint32_t resident_warps_per_sm;
    uint32_t shared_bytes_per_warp;
    uint32_t order;                  /* MRBatchOrderC */
    uint32_t tuned;                  /* 1 after mr_batch_tune */
    float tuned_step_milliseconds;   /* the tuner's best time of one control step */
    uint32_t mode;                   /* MRBatchLaunchModeC */
    uint32_t scene_blocks;           /* PER_FAMILY: the free-body launch's grid (one warp per CTA) */
    uint32_t scene_resident_warps_per_sm;
} MRBatchLaunchShapeC;

/* No counterpart in the reference.  Null with mr_last_error on failure. */
MR_API MRBatchHandle* mr_create_batch(MRTaskRolloutHandle* const* rollouts, size_t count);
MR_API void mr_batch_destroy(MRBatchHandle* batch);
/* No counterpart in the reference.  Advances every environment of every
 * rollout by control_step_count steps.  Per rollout w (arrays of `count`
 * device pointers, as in mr_create_batch): actions[w] [steps][envs][action
 * count] (required when the world takes actions), reset_masks[w]
 * [steps][envs] and status_codes[w] [steps][envs] (arrays or entries may
 * be null).  Stream-ordered on cuda_stream; returns without waiting.  Each
 * rollout's launch counters describe the advance. */
MR_API int mr_batch_advance(MRBatchHandle* batch, uint32_t control_step_count, const float* const* actions,
                            const uint32_t* const* reset_masks, uint32_t* const* status_codes, uint64_t cuda_stream);
/* No counterpart in the reference.  Autotuner: measures each rollout's item
 * latency (a launch of its environments alone), orders the queue by it,
 * then times control_step_count steps of the whole batch for both launch
 * modes, 1, 2 and 4 warps per CTA and both claim orders and keeps the
 * fastest.  Steps the
 * rollouts with `actions` (as in mr_batch_advance) and restores their
 * state afterwards; synchronous. */
MR_API int mr_batch_tune(MRBatchHandle* batch, uint32_t control_step_count, const float* const* actions);
MR_API int mr_batch_launch_shape(const MRBatchHandle* batch, MRBatchLaunchShapeC* out);
/* Item latency per rollout (ms per control step of one environment), the
 * key of the longest-first claim order. */
MR_API int mr_batch_world_costs(const MRBatchHandle* batch, float* milliseconds, size_t count);

/* ---------------------------------------------------------------------- */
/* Stepping without device allocation (no counterpart in the reference)   */
/* ---------------------------------------------------------------------- */

/* Most environments one mr_pile_step_no_alloc call may step. */
#define MR_B200_NO_ALLOC_MAX_ENVS 64u

/* No counterpart in the reference.  Advances `environment_count` pile or
 * stack environments by `control_step_count` control steps on buffers the
 * caller owns, without allocating any device memory: for hosts that manage
 * all GPU memory themselves (a framework's own allocator, a fixed memory
 * budget) or cannot afford cudaMalloc's device-wide synchronisation inside
 * their loop, and so cannot use the rollout handle, which allocates its
 * state and workspace.  The kernel is the rollout's pile kernel; its
 * workspace (at most MR_B200_NO_ALLOC_MAX_ENVS environments), launch
 * counters and packed world record live in fixed device arrays of the
 * library, about 8 MB that every GPU loading the library holds until exit.
 *
 * Device buffers (in/out unless noted): q [env][bodies * 7] (position,
 * orientation xyzw), v [env][bodies * 6], manifolds [env]
 * [MR_B200_SCENE_MANIFOLDS][MR_B200_SCENE_SLOT_WORDS] and manifold_counts
 * [env] (all zero for fresh environments), friction_scale [env] (in),
 * status_codes [control step][env] (out; may be null).  The body count
 * comes from mr_compile_synthetic_model(source, model_seed).  Work is
 * enqueued on `cuda_stream` and the call returns without waiting.
 *
 * The first call on a device resolves the device addresses of those arrays
 * (with that device current); make that first call before any stream
 * capture.  The first call for a new (source, model_seed, substep length)
 * also compiles that world on the host and uploads its record.  Every call
 * shares the arrays, so calls whose work overlaps on the GPU (other streams,
 * other host threads) race with each other; nothing in the workspace needs
 * to start at zero, since the kernel writes every word before reading it.
 * environment_count above MR_B200_NO_ALLOC_MAX_ENVS is rejected with a
 * message (-1).
 *
 * The world record is shared too: only one world is resident per device.
 * Each upload gets a new tag and each launch carries the tag current when it
 * was enqueued, so work that runs after another world was uploaded (work
 * the caller recorded into a graph and replays later, say) steps nothing:
 * such an environment
 * keeps q, v and manifolds untouched and reports MR_STEP_UNSUPPORTED in
 * status_codes and in counter 9 of mr_pile_step_no_alloc_counters.  Work
 * enqueued by this call therefore depends on the world record current when
 * it runs, not only on the arguments. */
MR_API int mr_pile_step_no_alloc(
    uint32_t source, uint64_t model_seed, uint32_t environment_count,
    float* q, float* v, float* manifolds, uint32_t* manifold_counts,
    const float* friction_scale, uint32_t* status_codes,
    uint32_t control_step_count, float control_timestep_seconds,
    uint32_t physics_substeps, uint32_t velocity_iterations,
    uint32_t final_velocity_iterations, uint64_t cuda_stream);

/* No counterpart in the reference.  Copies the first `count` (<= 16) launch
 * counters of the last mr_pile_step_no_alloc call on the current device into
 * host memory, after the work on `cuda_stream` has finished (the call waits
 * for that stream).  Counters: 0 failed environment-steps, 1 most active
 * contacts, 2 most manifolds, 3 most raw contacts, 4 most candidate pairs,
 * 5 most islands, 6 lowest failing environment (0xffffffff: none), 8 resets,
 * 9 environment-steps skipped because the world record had been replaced.
 * Allocates nothing. */
MR_API int mr_pile_step_no_alloc_counters(uint32_t* counters, uint32_t count, uint64_t cuda_stream);

#ifdef __cplusplus
}
#endif

#endif /* NUMI_B200_H */
