"""PolicyRolloutPack files (mr_write_policy_rollout_pack,
mr_policy_rollout_pack_inspect) against the reference's own writer and
reader (writePolicyRolloutPack / readPolicyRolloutPack,
src/core/LearningPacks.cpp, compiled into oracle/_ref): identical bytes,
each side reads the other's files, the artifact rules refuse the same
packs, corrupt files are refused.  No device work."""

from __future__ import annotations

import struct

import numpy as np
import pytest

import numi_lab_b200 as nb
from numi_lab_b200 import native
from numi_lab_b200.native import MetalRoboError

pytestmark = pytest.mark.reference


def _transitions(rng, steps, envs, revision):
    raw = (native.TaskTransitionC * (steps * envs))()
    for i, t in enumerate(raw):
        t.reward = float(rng.normal())
        t.tracking_score = float(rng.uniform())
        t.done = int(rng.uniform() < 0.2)
        t.timeout = int(t.done and rng.uniform() < 0.5)
        t.termination_reason = 4 if t.timeout else (1 if t.done else 0)
        t.timeout_bootstrap_value = float(rng.normal()) if t.timeout else 0.0
        t.policy_revision = revision
        t.difficulty_band = 0
    return raw


def _fields(seed=1, steps=5, envs=3, nobs=11, na=4, revision=9, **over):
    rng = np.random.default_rng(seed)
    f = dict(id="batch-" + str(seed), task_fingerprint=0x1234, policy_fingerprint=0xABCDEF, policy_revision=revision,
             environment_count=envs, control_step_count=steps,
             actor_observations=rng.normal(size=(steps, envs, nobs)).astype(np.float32),
             latents=rng.normal(size=(steps, envs, na)).astype(np.float32),
             log_probabilities=rng.normal(size=(steps, envs)).astype(np.float32),
             values=rng.normal(size=(steps, envs)).astype(np.float32),
             bootstrap_values=rng.normal(size=envs).astype(np.float32),
             transitions=_transitions(rng, steps, envs, revision))
    f.update(over)
    return f


def test_writers_produce_identical_files(tmp_path, reference_available):
    from oracle import reference_write_policy_rollout_pack

    for seed, extra in ((1, {}), (2, {"teacher_actions": np.ones((5, 3, 4), np.float32)}),
                        (3, {"critic_observations": np.zeros((5, 3, 6), np.float32)})):
        f = _fields(seed, **extra)
        ours, theirs = tmp_path / f"ours{seed}.mrrollout", tmp_path / f"ref{seed}.mrrollout"
        nb.write_policy_rollout_pack(ours, **f)
        c, keep = nb.world.policy_rollout_pack_c(**f)
        reference_write_policy_rollout_pack(c, theirs)
        assert ours.read_bytes() == theirs.read_bytes(), seed
        head = ours.read_bytes()[:32]
        assert head[:8] == b"MRLEARN\0" and struct.unpack_from("<II", head, 8) == (7, 3)
        del keep


def test_each_side_reads_the_others_files(tmp_path, reference_available):
    from oracle import reference_inspect_policy_rollout_pack, reference_write_policy_rollout_pack

    f = _fields(4, steps=6, envs=5)
    ours, theirs = tmp_path / "ours.mrrollout", tmp_path / "ref.mrrollout"
    nb.write_policy_rollout_pack(ours, **f)
    c, keep = nb.world.policy_rollout_pack_c(**f)
    reference_write_policy_rollout_pack(c, theirs)
    mine, mine_params = nb.inspect_policy_rollout_pack(theirs)
    ref, ref_params = reference_inspect_policy_rollout_pack(ours, mine_params.size)
    # The reference's reader returns its validation result, whose content
    # hash is zero (LearningPacks.cpp:2540-2550); ours reports the header's.
    assert ref.pop("content_hash") == 0
    payload = theirs.read_bytes()[32:]
    assert mine.pop("content_hash") == native.bindings().lib.mr_learning_pack_content_hash(payload, len(payload))
    assert mine == ref
    want = np.concatenate([f[k].reshape(-1) for k in ("actor_observations", "latents", "log_probabilities", "values", "bootstrap_values")])
    np.testing.assert_array_equal(mine_params, want)
    np.testing.assert_array_equal(ref_params, want)
    assert mine["transition_count"] == 30 and mine["done_count"] == sum(t.done for t in f["transitions"])
    assert mine["reward_sum"] == pytest.approx(sum(t.reward for t in f["transitions"]))
    assert (mine["task_fingerprint"], mine["policy_fingerprint"], mine["policy_revision"]) == (0x1234, 0xABCDEF, 9)
    del keep


def test_artifact_rules_refuse_the_same_packs(tmp_path, reference_available):
    from oracle import reference_write_policy_rollout_pack

    rng = np.random.default_rng(0)
    bad_tr = _transitions(rng, 5, 3, 9)
    bad_tr[4].policy_revision = 8
    nan_obs = _fields()["actor_observations"].copy()
    nan_obs[0, 0, 0] = np.nan
    cases = {
        "revision": dict(policy_revision=0),
        "fingerprint": dict(task_fingerprint=0),
        "latent shape": dict(latents=np.zeros((5, 3, 3), np.float32), action_count=4),
        "bootstrap": dict(bootstrap_values=np.zeros(2, np.float32)),
        "transition revision": dict(transitions=bad_tr),
        "non-finite": dict(actor_observations=nan_obs),
        "teacher shape": dict(teacher_actions=np.zeros(7, np.float32)),
    }
    for name, over in cases.items():
        f = _fields(**over)
        with pytest.raises(MetalRoboError):
            nb.write_policy_rollout_pack(tmp_path / f"{name}.mine", **f)
        c, keep = nb.world.policy_rollout_pack_c(**f)
        with pytest.raises(ValueError):
            reference_write_policy_rollout_pack(c, tmp_path / f"{name}.ref")
        del keep


def test_corrupt_and_foreign_files_are_refused(tmp_path):
    good = tmp_path / "good.mrrollout"
    nb.write_policy_rollout_pack(good, **_fields())
    data = good.read_bytes()
    cases = {
        "bit": (data[:-9] + bytes([data[-9] ^ 1]) + data[-8:], "hash"),
        "version": (data[:8] + struct.pack("<I", 6) + data[12:], "version"),
        "kind": (data[:12] + struct.pack("<I", 2) + data[16:], "kind"),
        "truncated": (data[:-3], "length"),
    }
    for name, (blob, message) in cases.items():
        p = tmp_path / f"{name}.mrrollout"
        p.write_bytes(blob)
        with pytest.raises(MetalRoboError, match=message):
            nb.inspect_policy_rollout_pack(p)
    # A PolicyPack is not a rollout pack.
    pack = tmp_path / "policy.mrpolicy"
    rng = np.random.default_rng(1)
    nb.write_policy_pack(pack, layers=[(rng.normal(size=(4, 11)).astype(np.float32), np.zeros(4, np.float32), "tanh")], revision=1,
                         action_clip=1.0, observation_clip=10.0, policy_id="p", contract=(1, 2, 3, 4, 5))
    with pytest.raises(MetalRoboError, match="kind"):
        nb.inspect_policy_rollout_pack(pack)
