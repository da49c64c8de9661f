"""Thin ctypes binding for the numi_b200 task-rollout C ABI.

Conventions follow numi-lab's own binding (python/metalrobo/native.py):
``ctypes.CDLL`` over the shared library, a ``MetalRoboError`` exception
carrying ``mr_last_error()``, and an environment override
(``METALROBO_LIBRARY``) for the library path.  The product path is the CUDA
library only; importing this module on a machine without the built library
raises instead of falling back to anything else.
"""

from __future__ import annotations

import ctypes as ct
import os
from pathlib import Path
from typing import Final

_LIBRARY_ENV: Final = "METALROBO_LIBRARY"
_PACKAGE_DIR: Final = Path(__file__).resolve().parent
DEFAULT_LIBRARY: Final = _PACKAGE_DIR / "libnumi_b200.so"

MR_INVALID_INDEX: Final = 0xFFFFFFFF
MR_RUN_SOURCE_SYNTHETIC_CHAIN7: Final = 100
MR_RUN_SOURCE_SYNTHETIC_TREE29: Final = 101
MR_RUN_SOURCE_SYNTHETIC_PILE: Final = 102
MR_RUN_SOURCE_SYNTHETIC_STACK: Final = 103
MR_RUN_SOURCE_SYNTHETIC_CYLINDER_PILE: Final = 104
MR_RUN_SOURCE_SYNTHETIC_PILE_GJK: Final = 105
MR_RUN_SOURCE_SYNTHETIC_HULL_PILE: Final = 106
MR_SHAPE_CONVEX: Final = 5
MR_DOF_FLAG_ACTUATED: Final = 1 << 1
MANIFOLD_POINTS: Final = 4
MR_PRECISION_FP32: Final = 0
MR_PRECISION_FP64_ARTICULATED_INERTIA: Final = 1
MR_PRECISION_COMPENSATED: Final = 2
PRECISION_MODES: Final = {
    "fp32": MR_PRECISION_FP32,
    "fp64-inertia": MR_PRECISION_FP64_ARTICULATED_INERTIA,
    "compensated": MR_PRECISION_COMPENSATED,
}

STATUS_NAMES: Final = {
    0: "success",
    1: "fixed_budget_complete",
    2: "nonfinite_input",
    3: "nonfinite_result",
    4: "pair_capacity_overflow",
    5: "contact_capacity_overflow",
    6: "manifold_capacity_overflow",
    7: "constraint_capacity_overflow",
    8: "island_capacity_overflow",
    9: "ccd_event_budget_exhausted",
    10: "factorization_failed",
    11: "did_not_converge",
    12: "unsupported",
    13: "ccd_capacity_overflow",
}


class MetalRoboError(RuntimeError):
    """Raised when the native runtime reports an error."""


class DynamicSphereC(ct.Structure):
    _fields_ = [
        ("position", ct.c_float * 3),
        ("linear_velocity", ct.c_float * 3),
        ("radius", ct.c_float),
        ("mass", ct.c_float),
        ("launch_step", ct.c_uint32),
    ]


class TaskRolloutConfigC(ct.Structure):
    _fields_ = [
        ("environment_count", ct.c_uint32),
        ("physics_substeps", ct.c_uint32),
        ("velocity_iterations", ct.c_uint32),
        ("final_velocity_iterations", ct.c_uint32),
        ("control_timestep_seconds", ct.c_float),
        ("seed", ct.c_uint64),
        ("dynamic_spheres", ct.POINTER(DynamicSphereC)),
        ("dynamic_sphere_count", ct.c_uint32),
        ("disable_task_terminations", ct.c_uint32),
        ("interaction_reference_mode", ct.c_uint32),
        ("interaction_student_authority", ct.c_float),
        ("override_interaction_student_authority", ct.c_uint32),
        ("interaction_reset_phase_fraction", ct.c_float),
        ("override_interaction_reset_phase_fraction", ct.c_uint32),
        ("materialize_articulated_contact_responses", ct.c_uint32),
        ("override_difficulty_band_range", ct.c_uint32),
        ("minimum_difficulty_band", ct.c_uint32),
        ("maximum_difficulty_band", ct.c_uint32),
        ("interaction_reset_phase_probability", ct.c_float),
        ("override_interaction_reset_phase_probability", ct.c_uint32),
        ("interaction_reset_maximum_phase", ct.c_float),
        ("override_interaction_reset_maximum_phase", ct.c_uint32),
    ]


class RunManifestC(ct.Structure):
    _fields_ = [
        ("profile", TaskRolloutConfigC),
        ("source", ct.c_uint32),
        ("surface", ct.c_uint32),
        ("task", ct.c_uint32),
        ("urdf_path", ct.c_char_p),
        ("srdf_path", ct.c_char_p),
        ("world_pack_path", ct.c_char_p),
        ("task_pack_path", ct.c_char_p),
        ("robot_actuator_pack_path", ct.c_char_p),
        ("sensor_program_pack_path", ct.c_char_p),
        ("reality_program_pack_path", ct.c_char_p),
        ("teacher_pack_path", ct.c_char_p),
        ("teacher_clip_id", ct.c_char_p),
        ("visual_sensor_program", ct.c_void_p),
        ("inspection_visual_program", ct.c_void_p),
        ("metallib_path", ct.c_char_p),
    ]


class BatchLaunchShapeC(ct.Structure):
    _fields_ = [
        ("worlds", ct.c_uint32),
        ("items", ct.c_uint32),
        ("warps_per_block", ct.c_uint32),
        ("blocks", ct.c_uint32),
        ("resident_warps_per_sm", ct.c_uint32),
        ("shared_bytes_per_warp", ct.c_uint32),
        ("order", ct.c_uint32),
        ("tuned", ct.c_uint32),
        ("tuned_step_milliseconds", ct.c_float),
        ("mode", ct.c_uint32),
        ("scene_blocks", ct.c_uint32),
        ("scene_resident_warps_per_sm", ct.c_uint32),
    ]


MR_SOLVER_QUALITY_NEWTON: Final = 1
MR_SOLVER_TEMPORAL_CONE: Final = 2
SOLVERS: Final = {"temporal_cone": MR_SOLVER_TEMPORAL_CONE, "quality_newton": MR_SOLVER_QUALITY_NEWTON}


class QualitySolverConfigC(ct.Structure):
    """MRQualitySolverConfigC (zero / non-positive fields take the defaults)."""

    _fields_ = [
        ("maximum_newton_iterations", ct.c_uint32),
        ("maximum_line_search_iterations", ct.c_uint32),
        ("optimality_tolerance", ct.c_double),
        ("line_search_tolerance", ct.c_double),
        ("regularization_floor", ct.c_double),
        ("reserved", ct.c_double),
    ]


class QualityDiagnosticsC(ct.Structure):
    _fields_ = [
        ("maximum_newton_iterations", ct.c_uint32),
        ("line_search_iterations", ct.c_uint32),
        ("maximum_scaled_optimality", ct.c_float),
        ("maximum_cone_violation", ct.c_float),
        ("maximum_complementarity", ct.c_float),
        ("reserved", ct.c_uint32 * 3),
    ]


class PolicyPackInfoC(ct.Structure):
    _fields_ = [
        ("format_version", ct.c_uint32),
        ("layer_count", ct.c_uint32),
        ("critic_layer_count", ct.c_uint32),
        ("observation_count", ct.c_uint32),
        ("action_count", ct.c_uint32),
        ("stochastic", ct.c_uint32),
        ("revision", ct.c_uint64),
        ("content_hash", ct.c_uint64),
        ("contract_version", ct.c_uint64),
        ("world_fingerprint", ct.c_uint64),
        ("task_fingerprint", ct.c_uint64),
        ("observation_fingerprint", ct.c_uint64),
        ("action_fingerprint", ct.c_uint64),
        ("parameter_count", ct.c_uint64),
        ("observation_clip", ct.c_float),
        ("action_clip", ct.c_float),
        ("id", ct.c_char * 64),
    ]


class QualityResultC(ct.Structure):
    _fields_ = [
        ("code", ct.c_uint32),
        ("newton_iterations", ct.c_uint32),
        ("line_search_iterations", ct.c_uint32),
        ("reserved", ct.c_uint32),
        ("scaled_optimality", ct.c_double),
        ("cone_violation", ct.c_double),
        ("complementarity", ct.c_double),
        ("objective", ct.c_double),
    ]


MR_BATCH_ORDER_LONGEST_FIRST: Final = 0
MR_BATCH_ORDER_ROUND_ROBIN: Final = 1
MR_BATCH_LAUNCH_FUSED: Final = 0
MR_BATCH_LAUNCH_PER_FAMILY: Final = 1


class TaskRolloutLayoutC(ct.Structure):
    _fields_ = [
        ("environment_count", ct.c_uint32),
        ("nq", ct.c_uint32),
        ("nv", ct.c_uint32),
        ("action_count", ct.c_uint32),
        ("actor_observation_count", ct.c_uint32),
        ("critic_observation_count", ct.c_uint32),
        ("scene_body_count", ct.c_uint32),
        ("motion_feature_count", ct.c_uint32),
        ("maximum_episode_steps", ct.c_uint32),
        ("world_fingerprint", ct.c_uint64),
        ("task_fingerprint", ct.c_uint64),
        ("observation_fingerprint", ct.c_uint64),
        ("action_fingerprint", ct.c_uint64),
        ("run_fingerprint", ct.c_uint64),
        ("robot_fingerprint", ct.c_uint64),
        ("sensor_fingerprint", ct.c_uint64),
        ("reality_fingerprint", ct.c_uint64),
        ("teacher_fingerprint", ct.c_uint64),
        ("submitted_control_steps", ct.c_uint64),
        ("completed_environment_steps", ct.c_uint64),
        ("submission_count", ct.c_uint64),
        ("retained_buffer_bytes", ct.c_size_t),
        ("immutable_private_bytes", ct.c_size_t),
        ("persistent_state_private_bytes", ct.c_size_t),
        ("transient_private_bytes", ct.c_size_t),
        ("shared_boundary_bytes", ct.c_size_t),
        ("peak_aliased_bytes", ct.c_size_t),
        ("total_gpu_milliseconds", ct.c_double),
        ("total_submission_milliseconds", ct.c_double),
    ]


class StageHighWaterC(ct.Structure):
    _fields_ = [
        (name, ct.c_uint32)
        for name in (
            "candidate_pairs raw_contacts manifolds constraint_blocks constraint_rows islands "
            "hard_convex_pairs mesh_triangle_candidates solver_tiles spill_rows ccd_candidates ccd_events "
            "endpoint_runtime_records articulation_point_queries rod_candidate_pairs rod_raw_contacts "
            "rod_manifolds rod_ccd_events quality_generalized_velocities quality_rows quality_krylov_vectors "
            "quality_direct_tiles dynamic_nodes island_node_references island_constraint_references "
            "rod_factor_blocks operator_velocity_elements"
        ).split()
    ]


class PolicyDenseLayerC(ct.Structure):
    """MRPolicyDenseLayerC (reference c_api.h:334-342); weights [output][input]."""

    _fields_ = [
        ("input_count", ct.c_uint32),
        ("output_count", ct.c_uint32),
        ("activation", ct.c_uint32),
        ("weights", ct.POINTER(ct.c_float)),
        ("weight_count", ct.c_size_t),
        ("bias", ct.POINTER(ct.c_float)),
        ("bias_count", ct.c_size_t),
    ]


class PolicyPackC(ct.Structure):
    """MRPolicyPackC (reference c_api.h:344-372)."""

    _fields_ = [
        ("id", ct.c_char_p),
        ("revision", ct.c_uint64),
        ("contract_version", ct.c_uint64),
        ("world_fingerprint", ct.c_uint64),
        ("task_fingerprint", ct.c_uint64),
        ("observation_fingerprint", ct.c_uint64),
        ("action_fingerprint", ct.c_uint64),
        ("observation_mean", ct.POINTER(ct.c_float)),
        ("observation_mean_count", ct.c_size_t),
        ("observation_inverse_standard_deviation", ct.POINTER(ct.c_float)),
        ("observation_inverse_standard_deviation_count", ct.c_size_t),
        ("layers", ct.POINTER(PolicyDenseLayerC)),
        ("layer_count", ct.c_size_t),
        ("critic_observation_mean", ct.POINTER(ct.c_float)),
        ("critic_observation_mean_count", ct.c_size_t),
        ("critic_observation_inverse_standard_deviation", ct.POINTER(ct.c_float)),
        ("critic_observation_inverse_standard_deviation_count", ct.c_size_t),
        ("critic_layers", ct.POINTER(PolicyDenseLayerC)),
        ("critic_layer_count", ct.c_size_t),
        ("action_log_standard_deviation", ct.POINTER(ct.c_float)),
        ("action_log_standard_deviation_count", ct.c_size_t),
        ("action_bias", ct.POINTER(ct.c_float)),
        ("action_bias_count", ct.c_size_t),
        ("action_scale", ct.POINTER(ct.c_float)),
        ("action_scale_count", ct.c_size_t),
        ("observation_clip", ct.c_float),
        ("action_clip", ct.c_float),
    ]


POLICY_ACTIVATIONS: Final = {"identity": 0, "relu": 1, "tanh": 2, "elu": 3, "silu": 4}


class TaskRolloutAdvanceC(ct.Structure):
    _fields_ = [
        ("control_step_count", ct.c_uint32),
        ("successful_environment_steps", ct.c_uint32),
        ("failed_environment_steps", ct.c_uint32),
        ("first_failing_environment", ct.c_uint32),
        ("first_failing_control_step", ct.c_uint32),
        ("first_gpu_status_code", ct.c_uint32),
        ("host_requested_resets", ct.c_uint32),
        ("maximum_active_contacts", ct.c_uint32),
        ("maximum_manifolds", ct.c_uint32),
        ("high_water", StageHighWaterC),
        ("gpu_milliseconds", ct.c_double),
        ("submission_milliseconds", ct.c_double),
    ]


class TaskActionBindingC(ct.Structure):
    _fields_ = [
        ("dof_index", ct.c_uint32),
        ("q_index", ct.c_uint32),
        ("v_index", ct.c_uint32),
        ("reserved", ct.c_uint32),
        ("scale", ct.c_float),
        ("lower_target", ct.c_float),
        ("upper_target", ct.c_float),
        ("response_time_seconds", ct.c_float),
    ]


class TaskObservationOperatorC(ct.Structure):
    _fields_ = [
        ("opcode", ct.c_uint32),
        ("source", ct.c_uint32),
        ("component", ct.c_uint32),
        ("flags", ct.c_uint32),
        ("transform_scale", ct.c_float),
        ("transform_offset", ct.c_float),
        ("noise_amplitude", ct.c_float),
        ("noise_channel", ct.c_uint32),
    ]


class TaskRewardOperatorC(ct.Structure):
    _fields_ = [
        ("opcode", ct.c_uint32),
        ("group", ct.c_uint32),
        ("weight", ct.c_float),
        ("parameters", ct.c_float * 3),
    ]


class TaskTerminationOperatorC(ct.Structure):
    _fields_ = [
        ("opcode", ct.c_uint32),
        ("reason", ct.c_uint32),
        ("priority", ct.c_uint32),
        ("group", ct.c_uint32),
        ("threshold", ct.c_float),
        ("failure_penalty", ct.c_float),
        ("minimum_band", ct.c_uint32),
        ("maximum_band", ct.c_uint32),
    ]


class TaskRandomizationOperatorC(ct.Structure):
    _fields_ = [
        ("opcode", ct.c_uint32),
        ("target", ct.c_uint32),
        ("minimum_band", ct.c_uint32),
        ("reserved", ct.c_uint32),
        ("parameters", ct.c_float * 4),
    ]


class TaskIndexGroupC(ct.Structure):
    _fields_ = [("first", ct.c_uint32), ("count", ct.c_uint32)]


class TaskContactGroupC(ct.Structure):
    _fields_ = [
        ("first", ct.c_uint32),
        ("count", ct.c_uint32),
        ("flags", ct.c_uint32),
        ("reference_body", ct.c_uint32),
        ("local_reference", ct.c_float * 4),
        ("kinematic_reference", ct.c_float * 4),
        ("gait_phase_offset", ct.c_float),
        ("stance_fraction", ct.c_float),
        ("reserved", ct.c_float * 2),
    ]


class TaskProgramC(ct.Structure):
    _fields_ = [
        ("actions", ct.POINTER(TaskActionBindingC)),
        ("action_count", ct.c_uint32),
        ("actor", ct.POINTER(TaskObservationOperatorC)),
        ("actor_count", ct.c_uint32),
        ("critic", ct.POINTER(TaskObservationOperatorC)),
        ("critic_count", ct.c_uint32),
        ("rewards", ct.POINTER(TaskRewardOperatorC)),
        ("reward_count", ct.c_uint32),
        ("terminations", ct.POINTER(TaskTerminationOperatorC)),
        ("termination_count", ct.c_uint32),
        ("randomization", ct.POINTER(TaskRandomizationOperatorC)),
        ("randomization_count", ct.c_uint32),
        ("joint_groups", ct.POINTER(TaskIndexGroupC)),
        ("joint_group_count", ct.c_uint32),
        ("joint_members", ct.POINTER(ct.c_uint32)),
        ("joint_member_count", ct.c_uint32),
        ("contact_groups", ct.POINTER(TaskContactGroupC)),
        ("contact_group_count", ct.c_uint32),
        ("contact_members", ct.POINTER(ct.c_uint32)),
        ("contact_member_count", ct.c_uint32),
        ("support_force_threshold", ct.c_float),
        ("clearance_target", ct.c_float),
        ("default_q", ct.POINTER(ct.c_float)),
        ("default_q_count", ct.c_uint32),
        ("maximum_episode_steps", ct.c_uint32),
        ("action_history", ct.c_uint32),
        ("action_delay_steps", ct.c_uint32),
        ("observation_history", ct.c_uint32),
        ("maximum_observation_delay", ct.c_uint32),
        ("base_height_target", ct.c_float),
        ("gait_period_seconds", ct.c_float),
        ("root_reference", ct.c_float * 3),
        ("command_lower", ct.c_float * 3),
        ("command_upper", ct.c_float * 3),
        ("standing_probability", ct.c_float),
        ("command_duration_seconds", ct.c_float * 2),
        ("difficulty_band_count", ct.c_uint32),
        ("band_sampling_exponent", ct.c_float),
        ("command_limit_lower", ct.c_float * 3),
        ("command_limit_upper", ct.c_float * 3),
        ("command_band_step", ct.c_float * 3),
        ("task_fingerprint", ct.c_uint64),
    ]


class TaskTransitionC(ct.Structure):
    _fields_ = [
        ("reward", ct.c_float),
        ("tracking_score", ct.c_float),
        ("root_height", ct.c_float),
        ("tilt", ct.c_float),
        ("done", ct.c_uint32),
        ("timeout", ct.c_uint32),
        ("physics_error", ct.c_uint32),
        ("termination_reason", ct.c_uint32),
        ("task_reward", ct.c_float),
        ("base_reward", ct.c_float),
        ("joint_velocity_reward", ct.c_float),
        ("joint_acceleration_reward", ct.c_float),
        ("control_reward", ct.c_float),
        ("posture_reward", ct.c_float),
        ("energy_reward", ct.c_float),
        ("contact_reward", ct.c_float),
        ("task_outcome_channels", ct.c_float * 8),
        ("policy_revision", ct.c_uint64),
        ("timeout_bootstrap_value", ct.c_float),
        ("episode_tracking_score", ct.c_float),
        ("difficulty_band", ct.c_uint32),
        ("terrain_level", ct.c_uint32),
        ("impact_sequence_index", ct.c_uint32),
        ("impact_event_flags", ct.c_uint32),
    ]


class PolicyRolloutBatchC(ct.Structure):
    _fields_ = [
        ("control_step_count", ct.c_uint32),
        ("actor_observations", ct.POINTER(ct.c_float)),
        ("actor_observation_count", ct.c_size_t),
        ("critic_observations", ct.POINTER(ct.c_float)),
        ("critic_observation_count", ct.c_size_t),
        ("motion_features", ct.POINTER(ct.c_float)),
        ("motion_feature_count", ct.c_size_t),
        ("teacher_actions", ct.POINTER(ct.c_float)),
        ("teacher_action_count", ct.c_size_t),
        ("latents", ct.POINTER(ct.c_float)),
        ("latent_count", ct.c_size_t),
        ("log_probabilities", ct.POINTER(ct.c_float)),
        ("log_probability_count", ct.c_size_t),
        ("values", ct.POINTER(ct.c_float)),
        ("value_count", ct.c_size_t),
        ("bootstrap_values", ct.POINTER(ct.c_float)),
        ("bootstrap_value_count", ct.c_size_t),
        ("transitions", ct.POINTER(TaskTransitionC)),
        ("transition_count", ct.c_size_t),
    ]


class PolicyRolloutPackC(ct.Structure):
    _fields_ = [
        ("id", ct.c_char_p),
        ("task_fingerprint", ct.c_uint64),
        ("policy_fingerprint", ct.c_uint64),
        ("policy_revision", ct.c_uint64),
        ("environment_count", ct.c_uint32),
        ("actor_observation_count", ct.c_uint32),
        ("critic_observation_count", ct.c_uint32),
        ("action_count", ct.c_uint32),
        ("motion_feature_count", ct.c_uint32),
        ("reserved", ct.c_uint32),
        ("batch", ct.POINTER(PolicyRolloutBatchC)),
    ]


class PolicyRolloutPackInfoC(ct.Structure):
    _fields_ = [
        ("task_fingerprint", ct.c_uint64),
        ("policy_fingerprint", ct.c_uint64),
        ("policy_revision", ct.c_uint64),
        ("content_hash", ct.c_uint64),
        ("environment_count", ct.c_uint32),
        ("control_step_count", ct.c_uint32),
        ("actor_observation_count", ct.c_uint32),
        ("critic_observation_count", ct.c_uint32),
        ("action_count", ct.c_uint32),
        ("motion_feature_count", ct.c_uint32),
        ("outcome_count", ct.c_uint32),
        ("has_teacher_actions", ct.c_uint32),
        ("transition_count", ct.c_uint64),
        ("reward_sum", ct.c_double),
        ("done_count", ct.c_uint64),
        ("id", ct.c_char * 64),
    ]


class TaskPackInfoC(ct.Structure):
    _fields_ = [
        ("content_hash", ct.c_uint64),
        ("action_count", ct.c_uint32),
        ("outcome_count", ct.c_uint32),
        ("contact_group_count", ct.c_uint32),
        ("joint_group_count", ct.c_uint32),
        ("reward_count", ct.c_uint32),
        ("termination_count", ct.c_uint32),
        ("maximum_episode_steps", ct.c_uint32),
        ("difficulty_band_count", ct.c_uint32),
        ("terrain_sample_count", ct.c_uint32),
        ("motion_tracked_body_count", ct.c_uint32),
        ("base_height_target", ct.c_float),
        ("gait_period_seconds", ct.c_float),
        ("clearance_target", ct.c_float),
        ("support_force_threshold", ct.c_float),
        ("id", ct.c_char * 64),
    ]


class ModelWorldC(ct.Structure):
    _fields_ = [
        ("body_count", ct.c_uint32),
        ("joint_count", ct.c_uint32),
        ("nq", ct.c_uint32),
        ("nv", ct.c_uint32),
        ("shape_count", ct.c_uint32),
        ("material_count", ct.c_uint32),
        ("pair_count", ct.c_uint32),
        ("root_type", ct.c_uint32),
        ("actuation_mode", ct.c_uint32),
        ("action_count", ct.c_uint32),
        ("contact_capacity", ct.c_uint32),
        ("apply_body_damping", ct.c_uint32),
        ("gravity", ct.c_float * 4),
        ("solver_scales", ct.c_float * 4),
        ("manifold_thresholds", ct.c_float * 4),
        ("speculative", ct.c_float * 4),
    ]


class ModelJointC(ct.Structure):
    _fields_ = [
        ("parent_body", ct.c_uint32),
        ("child_body", ct.c_uint32),
        ("joint_type", ct.c_uint32),
        ("q_index", ct.c_uint32),
        ("v_index", ct.c_uint32),
        ("reserved", ct.c_uint32 * 3),
        ("axis", ct.c_float * 4),
        ("parent_anchor", ct.c_float * 4),
        ("child_anchor", ct.c_float * 4),
        ("parent_rotation", ct.c_float * 4),
        ("child_rotation", ct.c_float * 4),
    ]


class ModelBodyC(ct.Structure):
    _fields_ = [
        ("parent_body", ct.c_uint32),
        ("inbound_joint", ct.c_uint32),
        ("motion_type", ct.c_uint32),
        ("articulated", ct.c_uint32),
        ("mass_inverse_mass", ct.c_float * 4),
        ("inertia", (ct.c_float * 4) * 3),
        ("damping_speed", ct.c_float * 4),
        ("static_pose", ct.c_float * 8),
    ]


class ModelDofC(ct.Structure):
    _fields_ = [
        ("joint_index", ct.c_uint32),
        ("q_index", ct.c_uint32),
        ("flags", ct.c_uint32),
        ("reserved", ct.c_uint32),
        ("limits", ct.c_float * 4),
        ("drive", ct.c_float * 4),
    ]


class ModelShapeC(ct.Structure):
    _fields_ = [
        ("body", ct.c_uint32),
        ("shape_type", ct.c_uint32),
        ("material", ct.c_uint32),
        ("flags", ct.c_uint32),
        ("collision_group", ct.c_uint32),
        ("collision_mask", ct.c_uint32),
        ("hull_first", ct.c_uint32),
        ("hull_count", ct.c_uint32),
        ("local_position", ct.c_float * 4),
        ("local_rotation", ct.c_float * 4),
        ("dimensions", ct.c_float * 4),
        ("contact_rest_bound", ct.c_float * 4),
    ]


class ModelMaterialC(ct.Structure):
    _fields_ = [("friction", ct.c_float * 4), ("response", ct.c_float * 4)]


class ModelPairC(ct.Structure):
    _fields_ = [
        ("shape_a", ct.c_uint32),
        ("shape_b", ct.c_uint32),
        ("pair_class", ct.c_uint32),
        ("max_points", ct.c_uint32),
    ]


class ModelViewC(ct.Structure):
    _fields_ = [
        ("world", ModelWorldC),
        ("joints", ct.POINTER(ModelJointC)),
        ("bodies", ct.POINTER(ModelBodyC)),
        ("dofs", ct.POINTER(ModelDofC)),
        ("shapes", ct.POINTER(ModelShapeC)),
        ("materials", ct.POINTER(ModelMaterialC)),
        ("pairs", ct.POINTER(ModelPairC)),
        ("hull_vertices", ct.POINTER(ct.c_float)),
        ("hull_vertex_capacity", ct.c_uint32),
        ("hull_vertex_count", ct.c_uint32),
    ]


class ManifoldPointC(ct.Structure):
    _fields_ = [
        ("anchor_a", ct.c_float * 3),
        ("anchor_b", ct.c_float * 3),
        ("feature_a", ct.c_uint32),
        ("feature_b", ct.c_uint32),
        ("life", ct.c_uint32),
        ("impulses", ct.c_float * 3),
    ]


class ManifoldC(ct.Structure):
    _fields_ = [
        ("normal_local", ct.c_float * 3),
        ("age", ct.c_float),
        ("tangent_local", ct.c_float * 3),
        ("count", ct.c_uint32),
        ("points", ManifoldPointC * MANIFOLD_POINTS),
    ]


# Every C-ABI entry point this binding configures, by name.  Tests check the
# loaded library exports each of them.
class ServerConfigC(ct.Structure):
    _fields_ = [
        ("hbm_budget_bytes", ct.c_uint64),
        ("model_seed", ct.c_uint64),
        ("physics_substeps", ct.c_uint32),
        ("velocity_iterations", ct.c_uint32),
        ("final_velocity_iterations", ct.c_uint32),
        ("control_timestep_seconds", ct.c_float),
        ("max_envs_per_source", ct.c_uint32),
        ("control_steps_per_tick", ct.c_uint32),
    ]


class ServerRequestC(ct.Structure):
    _fields_ = [
        ("source", ct.c_uint32),
        ("env_count", ct.c_uint32),
        ("horizon", ct.c_uint32),
        ("reserved", ct.c_uint32),
        ("seed", ct.c_uint64),
        ("actions", ct.POINTER(ct.c_float)),
    ]


class ServerCompletionC(ct.Structure):
    _fields_ = [
        ("request_id", ct.c_uint64),
        ("source", ct.c_uint32),
        ("env_count", ct.c_uint32),
        ("horizon", ct.c_uint32),
        ("failed_env_steps", ct.c_uint32),
        ("first_failure_status", ct.c_uint32),
        ("reserved", ct.c_uint32),
        ("queue_seconds", ct.c_double),
        ("latency_seconds", ct.c_double),
    ]


class ServerStatsC(ct.Structure):
    _fields_ = [
        ("pending_requests", ct.c_uint32),
        ("running_requests", ct.c_uint32),
        ("free_slots", ct.c_uint32),
        ("reserved", ct.c_uint32),
        ("completed_env_steps", ct.c_uint64),
        ("hbm_bytes_in_use", ct.c_uint64),
    ]


EXPORTED_SYMBOLS: Final = (
    "mr_version",
    "mr_runtime_abi_fingerprint",
    "mr_last_error",
    "mr_create_task_rollout",
    "mr_task_rollout_destroy",
    "mr_task_rollout_reset",
    "mr_task_rollout_set_state_readback",
    "mr_task_rollout_advance",
    "mr_task_rollout_layout",
    "mr_task_rollout_device_name",
    "mr_task_rollout_status_codes",
    "mr_task_rollout_active_contacts",
    "mr_task_rollout_actor_observations",
    "mr_task_rollout_final_q",
    "mr_task_rollout_copy_final_scene_states",
    "mr_task_rollout_advance_device",
    "mr_task_rollout_copy_model",
    "mr_task_rollout_copy_environment_parameters",
    "mr_task_rollout_copy_state",
    "mr_task_rollout_launch_shape",
    "mr_task_rollout_set_state",
    "mr_task_rollout_set_precision",
    "mr_create_server",
    "mr_server_destroy",
    "mr_server_capacity",
    "mr_server_submit",
    "mr_server_tick",
    "mr_server_poll",
    "mr_server_copy_result",
    "mr_server_release",
    "mr_server_stats",
    "mr_pile_step_no_alloc",
    "mr_pile_step_no_alloc_counters",
    "mr_task_rollout_set_island_labels",
    "mr_task_rollout_copy_island_labels",
    "mr_task_rollout_set_audit",
    "mr_task_rollout_copy_audit",
    "mr_measure_issue_peak",
    "mr_create_batch",
    "mr_batch_destroy",
    "mr_batch_advance",
    "mr_batch_tune",
    "mr_batch_launch_shape",
    "mr_batch_world_costs",
    "mr_task_rollout_set_policy",
    "mr_task_rollout_environment_chains",
    "mr_task_rollout_policy_revision",
    "mr_task_rollout_clear_policy",
    "mr_task_rollout_set_task",
    "mr_task_rollout_clear_task",
    "mr_task_rollout_transitions",
    "mr_task_rollout_device_transitions",
    "mr_task_rollout_copy_transitions",
    "mr_task_rollout_write_policy_rollout_pack",
    "mr_write_policy_rollout_pack",
    "mr_policy_rollout_pack_inspect",
    "mr_task_pack_inspect",
    "mr_task_pack_rewrite",
    "mr_task_rollout_policy_latents",
    "mr_task_rollout_policy_log_probabilities",
    "mr_task_rollout_policy_values",
    "mr_task_rollout_bootstrap_policy_values",
    "mr_task_rollout_set_solver",
    "mr_task_rollout_quality_diagnostics",
    "mr_quality_solve_batch",
    "mr_write_policy_pack",
    "mr_learning_pack_content_hash",
    "mr_task_rollout_load_policy_pack",
    "mr_policy_pack_inspect",
)


def resolve_library_path(path: str | os.PathLike[str] | None = None) -> Path:
    """Resolves the native library, preferring explicit and environment paths."""

    if path is not None:
        explicit = Path(path).expanduser()
        if not explicit.is_file():
            raise FileNotFoundError(f"numi_b200 library does not exist: {explicit}")
        return explicit.resolve()
    configured = os.environ.get(_LIBRARY_ENV)
    if configured:
        configured_path = Path(configured).expanduser()
        if not configured_path.is_file():
            raise FileNotFoundError(f"{_LIBRARY_ENV} points to a missing file: {configured_path}")
        return configured_path.resolve()
    if DEFAULT_LIBRARY.is_file():
        return DEFAULT_LIBRARY
    raise FileNotFoundError(
        f"Could not find {DEFAULT_LIBRARY.name}. Build it with `python -m numi_lab_b200.build` "
        f"or set {_LIBRARY_ENV}."
    )


class Bindings:
    """Configured ctypes function table for one loaded library."""

    def __init__(self, path: str | os.PathLike[str] | None = None) -> None:
        self.path = resolve_library_path(path)
        self.lib = ct.CDLL(str(self.path))
        L = self.lib
        P = ct.POINTER
        L.mr_version.argtypes = []
        L.mr_version.restype = ct.c_char_p
        L.mr_runtime_abi_fingerprint.argtypes = []
        L.mr_runtime_abi_fingerprint.restype = ct.c_uint64
        L.mr_last_error.argtypes = []
        L.mr_last_error.restype = ct.c_char_p
        L.mr_create_task_rollout.argtypes = [P(RunManifestC)]
        L.mr_create_task_rollout.restype = ct.c_void_p
        L.mr_task_rollout_destroy.argtypes = [ct.c_void_p]
        L.mr_task_rollout_destroy.restype = None
        L.mr_task_rollout_reset.argtypes = [ct.c_void_p, ct.c_uint64]
        L.mr_task_rollout_reset.restype = ct.c_int
        L.mr_task_rollout_set_state_readback.argtypes = [ct.c_void_p, ct.c_uint32]
        L.mr_task_rollout_set_state_readback.restype = ct.c_int
        L.mr_task_rollout_set_precision.argtypes = [ct.c_void_p, ct.c_uint32]
        L.mr_task_rollout_set_precision.restype = ct.c_int
        L.mr_task_rollout_environment_chains.argtypes = [ct.c_void_p]
        L.mr_task_rollout_environment_chains.restype = ct.c_uint32
        L.mr_task_rollout_set_policy.argtypes = [ct.c_void_p, ct.POINTER(PolicyPackC)]
        L.mr_task_rollout_set_policy.restype = ct.c_int
        L.mr_task_rollout_policy_revision.argtypes = [ct.c_void_p]
        L.mr_task_rollout_policy_revision.restype = ct.c_uint64
        L.mr_task_rollout_clear_policy.argtypes = [ct.c_void_p]
        L.mr_task_rollout_clear_policy.restype = ct.c_int
        for name in ("latents", "log_probabilities", "values"):
            fn = getattr(L, f"mr_task_rollout_policy_{name}")
            fn.argtypes = [ct.c_void_p]
            fn.restype = ct.POINTER(ct.c_float)
        L.mr_task_rollout_bootstrap_policy_values.argtypes = [ct.c_void_p]
        L.mr_task_rollout_bootstrap_policy_values.restype = ct.POINTER(ct.c_float)
        L.mr_task_rollout_advance.argtypes = [
            ct.c_void_p,
            P(ct.c_float),
            ct.c_size_t,
            P(ct.c_uint32),
            ct.c_size_t,
            ct.c_uint32,
            ct.c_uint64,
            ct.c_uint32,
            P(TaskRolloutAdvanceC),
        ]
        L.mr_task_rollout_advance.restype = ct.c_int
        L.mr_task_rollout_layout.argtypes = [ct.c_void_p]
        L.mr_task_rollout_layout.restype = TaskRolloutLayoutC
        L.mr_task_rollout_device_name.argtypes = [ct.c_void_p]
        L.mr_task_rollout_device_name.restype = ct.c_char_p
        for name in ("mr_task_rollout_status_codes", "mr_task_rollout_active_contacts"):
            getattr(L, name).argtypes = [ct.c_void_p]
            getattr(L, name).restype = P(ct.c_uint32)
        for name in ("mr_task_rollout_actor_observations", "mr_task_rollout_final_q"):
            getattr(L, name).argtypes = [ct.c_void_p]
            getattr(L, name).restype = P(ct.c_float)
        L.mr_task_rollout_copy_final_scene_states.argtypes = [ct.c_void_p, P(ct.c_float), ct.c_size_t]
        L.mr_task_rollout_copy_final_scene_states.restype = ct.c_int
        L.mr_task_rollout_advance_device.argtypes = [
            ct.c_void_p,
            ct.c_void_p,
            ct.c_void_p,
            ct.c_uint32,
            ct.c_void_p,
            ct.c_void_p,
            ct.c_uint64,
            P(TaskRolloutAdvanceC),
        ]
        L.mr_task_rollout_advance_device.restype = ct.c_int
        L.mr_task_rollout_copy_model.argtypes = [ct.c_void_p, P(ModelViewC)]
        L.mr_task_rollout_copy_model.restype = ct.c_int
        L.mr_task_rollout_copy_environment_parameters.argtypes = [ct.c_void_p, P(ct.c_float)]
        L.mr_task_rollout_copy_environment_parameters.restype = ct.c_int
        L.mr_task_rollout_copy_state.argtypes = [ct.c_void_p, P(ct.c_float), P(ct.c_float), ct.c_void_p]
        L.mr_task_rollout_copy_state.restype = ct.c_int
        L.mr_task_rollout_launch_shape.argtypes = [ct.c_void_p, P(ct.c_uint32), P(ct.c_uint32)]
        L.mr_task_rollout_launch_shape.restype = ct.c_int
        L.mr_task_rollout_set_state.argtypes = [ct.c_void_p, P(ct.c_float), P(ct.c_float), ct.c_void_p, ct.c_uint32]
        L.mr_task_rollout_set_state.restype = ct.c_int
        L.mr_create_server.argtypes = [P(ServerConfigC)]
        L.mr_create_server.restype = ct.c_void_p
        L.mr_server_destroy.argtypes = [ct.c_void_p]
        L.mr_server_destroy.restype = None
        L.mr_server_capacity.argtypes = [ct.c_void_p, ct.c_uint32, P(ct.c_uint32), P(ct.c_uint32)]
        L.mr_server_capacity.restype = ct.c_int
        L.mr_server_submit.argtypes = [ct.c_void_p, P(ServerRequestC), P(ct.c_uint64)]
        L.mr_server_submit.restype = ct.c_int
        L.mr_server_tick.argtypes = [ct.c_void_p, P(ct.c_uint32), P(ct.c_uint32)]
        L.mr_server_tick.restype = ct.c_int
        L.mr_server_poll.argtypes = [ct.c_void_p, P(ServerCompletionC), ct.c_uint32, P(ct.c_uint32)]
        L.mr_server_poll.restype = ct.c_int
        L.mr_server_copy_result.argtypes = [ct.c_void_p, ct.c_uint64, P(ct.c_float), ct.c_size_t, P(ct.c_float), ct.c_size_t]
        L.mr_server_copy_result.restype = ct.c_int
        L.mr_server_release.argtypes = [ct.c_void_p, ct.c_uint64]
        L.mr_server_release.restype = ct.c_int
        L.mr_server_stats.argtypes = [ct.c_void_p, P(ServerStatsC)]
        L.mr_server_stats.restype = ct.c_int
        L.mr_pile_step_no_alloc.argtypes = [ct.c_uint32, ct.c_uint64, ct.c_uint32] + [ct.c_void_p] * 6 + [
            ct.c_uint32, ct.c_float, ct.c_uint32, ct.c_uint32, ct.c_uint32, ct.c_uint64]
        L.mr_pile_step_no_alloc.restype = ct.c_int
        L.mr_pile_step_no_alloc_counters.argtypes = [P(ct.c_uint32), ct.c_uint32, ct.c_uint64]
        L.mr_pile_step_no_alloc_counters.restype = ct.c_int
        L.mr_task_rollout_set_island_labels.argtypes = [ct.c_void_p, ct.c_uint32]
        L.mr_task_rollout_set_island_labels.restype = ct.c_int
        L.mr_task_rollout_copy_island_labels.argtypes = [ct.c_void_p, P(ct.c_uint8), ct.c_size_t]
        L.mr_task_rollout_copy_island_labels.restype = ct.c_int
        L.mr_task_rollout_set_audit.argtypes = [ct.c_void_p, ct.c_uint32]
        L.mr_task_rollout_set_audit.restype = ct.c_int
        L.mr_task_rollout_copy_audit.argtypes = [ct.c_void_p, P(ct.c_double), ct.c_size_t]
        L.mr_task_rollout_copy_audit.restype = ct.c_int
        L.mr_measure_issue_peak.argtypes = [P(ct.c_double), P(ct.c_double)]
        L.mr_measure_issue_peak.restype = ct.c_int
        PP = ct.POINTER(ct.c_void_p)
        L.mr_create_batch.argtypes = [PP, ct.c_size_t]
        L.mr_create_batch.restype = ct.c_void_p
        L.mr_batch_destroy.argtypes = [ct.c_void_p]
        L.mr_batch_destroy.restype = None
        L.mr_batch_advance.argtypes = [ct.c_void_p, ct.c_uint32, PP, PP, PP, ct.c_uint64]
        L.mr_batch_advance.restype = ct.c_int
        L.mr_batch_tune.argtypes = [ct.c_void_p, ct.c_uint32, PP]
        L.mr_batch_tune.restype = ct.c_int
        L.mr_batch_launch_shape.argtypes = [ct.c_void_p, P(BatchLaunchShapeC)]
        L.mr_batch_launch_shape.restype = ct.c_int
        L.mr_batch_world_costs.argtypes = [ct.c_void_p, P(ct.c_float), ct.c_size_t]
        L.mr_batch_world_costs.restype = ct.c_int
        L.mr_task_rollout_set_solver.argtypes = [ct.c_void_p, ct.c_uint32, P(QualitySolverConfigC)]
        L.mr_task_rollout_set_solver.restype = ct.c_int
        L.mr_task_rollout_quality_diagnostics.argtypes = [ct.c_void_p, P(QualityDiagnosticsC)]
        L.mr_task_rollout_quality_diagnostics.restype = ct.c_int
        PD = P(ct.c_double)
        L.mr_quality_solve_batch.argtypes = [ct.c_uint32, ct.c_uint32, ct.c_uint32, P(ct.c_uint32), PD, PD, PD, PD, PD, PD, PD,
                                             P(QualitySolverConfigC), PD, PD, P(QualityResultC)]
        L.mr_quality_solve_batch.restype = ct.c_int
        L.mr_write_policy_pack.argtypes = [P(PolicyPackC), ct.c_char_p]
        L.mr_write_policy_pack.restype = ct.c_int
        L.mr_learning_pack_content_hash.argtypes = [ct.c_void_p, ct.c_size_t]
        L.mr_learning_pack_content_hash.restype = ct.c_uint64
        L.mr_task_rollout_load_policy_pack.argtypes = [ct.c_void_p, ct.c_char_p]
        L.mr_task_rollout_load_policy_pack.restype = ct.c_int
        L.mr_policy_pack_inspect.argtypes = [ct.c_char_p, P(PolicyPackInfoC), P(ct.c_float), ct.c_size_t]
        L.mr_policy_pack_inspect.restype = ct.c_int
        L.mr_task_rollout_set_task.argtypes = [ct.c_void_p, P(TaskProgramC)]
        L.mr_task_rollout_set_task.restype = ct.c_int
        L.mr_task_rollout_clear_task.argtypes = [ct.c_void_p]
        L.mr_task_rollout_clear_task.restype = ct.c_int
        L.mr_task_rollout_transitions.argtypes = [ct.c_void_p]
        L.mr_task_rollout_transitions.restype = P(TaskTransitionC)
        L.mr_task_rollout_device_transitions.argtypes = [ct.c_void_p]
        L.mr_task_rollout_device_transitions.restype = ct.c_uint64
        L.mr_task_rollout_copy_transitions.argtypes = [ct.c_void_p, P(TaskTransitionC), ct.c_size_t]
        L.mr_task_rollout_copy_transitions.restype = ct.c_int
        L.mr_task_rollout_write_policy_rollout_pack.argtypes = [ct.c_void_p, P(PolicyRolloutBatchC), ct.c_char_p, ct.c_char_p]
        L.mr_task_rollout_write_policy_rollout_pack.restype = ct.c_int
        L.mr_write_policy_rollout_pack.argtypes = [P(PolicyRolloutPackC), ct.c_char_p]
        L.mr_write_policy_rollout_pack.restype = ct.c_int
        L.mr_policy_rollout_pack_inspect.argtypes = [ct.c_char_p, P(PolicyRolloutPackInfoC), P(ct.c_float), ct.c_size_t]
        L.mr_policy_rollout_pack_inspect.restype = ct.c_int
        L.mr_task_pack_inspect.argtypes = [ct.c_char_p, P(TaskPackInfoC)]
        L.mr_task_pack_inspect.restype = ct.c_int
        L.mr_task_pack_rewrite.argtypes = [ct.c_char_p, ct.c_char_p]
        L.mr_task_pack_rewrite.restype = ct.c_int

    def last_error(self) -> str:
        value = self.lib.mr_last_error()
        return value.decode("utf-8", "replace") if value else ""

    def check(self, rc: int, what: str) -> None:
        if rc != 0:
            raise MetalRoboError(f"{what}: {self.last_error()}")


_BINDINGS: Bindings | None = None


def bindings(path: str | os.PathLike[str] | None = None) -> Bindings:
    """Returns the process-wide bindings (loading the library on first use)."""

    global _BINDINGS
    if path is not None:
        return Bindings(path)
    if _BINDINGS is None:
        _BINDINGS = Bindings()
    return _BINDINGS


def default_manifest(
    source: int,
    environment_count: int,
    *,
    physics_substeps: int = 1,
    velocity_iterations: int = 8,
    final_velocity_iterations: int = 0,
    control_timestep_seconds: float = 0.005,
    seed: int = 0,
) -> RunManifestC:
    manifest = RunManifestC()
    profile = manifest.profile
    profile.environment_count = environment_count
    profile.physics_substeps = physics_substeps
    profile.velocity_iterations = velocity_iterations
    profile.final_velocity_iterations = final_velocity_iterations
    profile.control_timestep_seconds = control_timestep_seconds
    profile.seed = seed
    manifest.source = source
    return manifest
