"""PolicyPack files (mr_write_policy_pack, mr_policy_pack_inspect,
mr_learning_pack_content_hash) against the reference's own writer and
reader (writePolicyPack / readPolicyPack, src/core/LearningPacks.cpp,
compiled into oracle/_ref): the two writers produce the same bytes, each
side reads the other's files field for field, and malformed or legacy
files are refused.  No device work.
"""

from __future__ import annotations

import struct

import numpy as np
import pytest

import numi_lab_b200 as nb
from numi_lab_b200 import native

pytestmark = pytest.mark.reference

CONTRACT = (1, 0x1111, 0x2222, 0x3333, 0x4444)


def _dense(rng, sizes, acts):
    return [(rng.normal(0.0, 1.0 / np.sqrt(a), (b, a)).astype(np.float32), rng.normal(0.0, 0.1, b).astype(np.float32), f)
            for (a, b), f in zip(zip(sizes[:-1], sizes[1:]), acts)]


def _packs(seed: int = 3):
    """Three packs: deterministic actor; normalised stochastic actor with a
    critic; action scale and bias with a deep actor."""

    rng = np.random.default_rng(seed)
    nobs, na = 71, 29
    yield dict(layers=_dense(rng, [nobs, 64, na], ["tanh", "identity"]), revision=7, action_clip=2.0, policy_id="actor",
               observation_clip=100.0, contract=CONTRACT)
    yield dict(layers=_dense(rng, [nobs, 128, 64, na], ["elu", "silu", "tanh"]), revision=12, action_clip=3.5,
               policy_id="stochastic", observation_mean=rng.normal(size=nobs), observation_inverse_std=rng.uniform(0.5, 2.0, nobs),
               observation_clip=10.0, critic_layers=_dense(rng, [nobs, 32, 1], ["relu", "identity"]),
               critic_observation_mean=rng.normal(size=nobs), critic_observation_inverse_std=rng.uniform(0.5, 2.0, nobs),
               action_log_std=rng.uniform(-2.0, -0.5, na), contract=CONTRACT)
    yield dict(layers=_dense(rng, [nobs, 32, 32, 32, na], ["relu", "relu", "silu", "identity"]), revision=1, action_clip=1.0,
               policy_id="scaled-" + "x" * 40, action_bias=rng.normal(size=na), action_scale=rng.uniform(0.1, 1.0, na),
               observation_clip=50.0, contract=(1, 2**64 - 1, 5, 6, 7))


def _tables(p: dict) -> np.ndarray:
    out = []
    f32 = lambda a: [] if a is None else list(np.asarray(a, np.float32).reshape(-1))  # noqa: E731
    out += f32(p.get("observation_mean")) + f32(p.get("observation_inverse_std"))
    for w, b, _ in p["layers"]:
        out += f32(w) + f32(b)
    out += f32(p.get("critic_observation_mean")) + f32(p.get("critic_observation_inverse_std"))
    for w, b, _ in p.get("critic_layers", ()):
        out += f32(w) + f32(b)
    out += f32(p.get("action_log_std")) + f32(p.get("action_bias")) + f32(p.get("action_scale"))
    return np.array(out, np.float32)


def test_writers_produce_identical_files(tmp_path, reference_available):
    from oracle import reference_write_policy_pack

    for i, p in enumerate(_packs()):
        ours, theirs = tmp_path / f"ours{i}.mrpolicy", tmp_path / f"ref{i}.mrpolicy"
        nb.write_policy_pack(ours, **{k: v for k, v in p.items() if k != "layers"}, layers=p["layers"])
        pk, keep = nb.world.policy_pack_c(**p)
        reference_write_policy_pack(pk, theirs)
        assert ours.read_bytes() == theirs.read_bytes(), i
        del keep


def test_each_side_reads_the_others_files(tmp_path, reference_available):
    from oracle import reference_inspect_policy_pack, reference_write_policy_pack

    for i, p in enumerate(_packs(11)):
        ours, theirs = tmp_path / f"ours{i}.mrpolicy", tmp_path / f"ref{i}.mrpolicy"
        nb.write_policy_pack(ours, **p)
        pk, keep = nb.world.policy_pack_c(**p)
        reference_write_policy_pack(pk, theirs)
        mine, mine_params = nb.inspect_policy_pack(theirs)
        ref, ref_params = reference_inspect_policy_pack(ours)
        ref.pop("format_version")  # the reference's reader does not report it
        for key, value in ref.items():
            assert mine[key] == value, (i, key)
        assert mine["format_version"] == 4
        assert mine["id"] == p["policy_id"][:63] and mine["revision"] == p["revision"]
        assert (mine["contract_version"], mine["world_fingerprint"], mine["task_fingerprint"], mine["observation_fingerprint"],
                mine["action_fingerprint"]) == p["contract"]
        np.testing.assert_array_equal(mine_params, _tables(p))
        np.testing.assert_array_equal(ref_params, _tables(p))
        del keep


def test_content_hash_is_the_headers():
    lib = native.bindings()
    for payload in (b"", b"abc", bytes(range(256)) * 7):
        h = lib.lib.mr_learning_pack_content_hash(payload, len(payload))
        ref = 14695981039346656037
        for byte in payload:
            ref = ((ref ^ byte) * 1099511628211) & (2**64 - 1)
        assert h == (ref or 1)


def _rewrite(path, mutate) -> None:
    data = bytearray(path.read_bytes())
    mutate(data)
    path.write_bytes(bytes(data))


def _rehash(data: bytearray) -> None:
    lib = native.bindings()
    payload = bytes(data[32:])
    struct.pack_into("<QQ", data, 16, len(payload), lib.lib.mr_learning_pack_content_hash(payload, len(payload)))


def test_malformed_files_are_refused(tmp_path):
    p = next(_packs())
    good = tmp_path / "good.mrpolicy"
    nb.write_policy_pack(good, **p)
    cases = {
        "magic": (lambda d: d.__setitem__(0, ord("X")), "magic"),
        "kind": (lambda d: struct.pack_into("<I", d, 12, 1), "kind"),
        "version": (lambda d: struct.pack_into("<I", d, 8, 5), "version"),
        "payload bit": (lambda d: d.__setitem__(len(d) - 50, d[len(d) - 50] ^ 1), "hash"),
        "truncated": (lambda d: d.__delitem__(slice(len(d) - 4, len(d))), "length"),
        "layer count": (lambda d: (struct.pack_into("<Q", d, 32 + 8 + len(p["policy_id"]) + 8 + 16, 2**40), _rehash(d)), "malformed"),
    }
    for name, (mutate, message) in cases.items():
        bad = tmp_path / f"{name}.mrpolicy"
        bad.write_bytes(good.read_bytes())
        _rewrite(bad, mutate)
        with pytest.raises(nb.MetalRoboError, match=message):
            nb.inspect_policy_pack(bad)


def test_legacy_version_3_pack_reads_without_a_contract(tmp_path, reference_available):
    """A version-3 pack ends after the clips; both readers accept it and
    report an empty contract (installing one needs the reference's
    migration; mr_task_rollout_load_policy_pack refuses it)."""

    from oracle import reference_inspect_policy_pack

    p = next(_packs())
    path = tmp_path / "legacy.mrpolicy"
    nb.write_policy_pack(path, **p)

    def to_v3(d: bytearray) -> None:
        del d[len(d) - 40:]
        struct.pack_into("<I", d, 8, 3)
        _rehash(d)

    _rewrite(path, to_v3)
    mine, mine_params = nb.inspect_policy_pack(path)
    ref, ref_params = reference_inspect_policy_pack(path)
    assert mine["format_version"] == 3 and mine["contract_version"] == 0 and ref["contract_version"] == 0
    np.testing.assert_array_equal(mine_params, ref_params)


def test_writer_applies_the_artifact_rules(tmp_path, reference_available):
    from oracle import reference_write_policy_pack

    base = next(_packs())
    rng = np.random.default_rng(0)
    bad_layers = [(np.full((29, 71), np.nan, np.float32), np.zeros(29, np.float32), "tanh")]
    cases = {
        "contract": dict(base, contract=(1, 0, 2, 3, 4)),
        "revision": dict(base, revision=0),
        "stochastic": dict(base, action_log_std=np.zeros(29)),
        "values": dict(base, layers=bad_layers),
        "clip": dict(base, action_clip=0.0),
        "shape": dict(base, layers=[(rng.normal(size=(29, 71)).astype(np.float32), np.zeros(28, np.float32), "tanh")]),
    }
    for name, p in cases.items():
        with pytest.raises(nb.MetalRoboError):
            nb.write_policy_pack(tmp_path / f"{name}.mrpolicy", **p)
        pk, keep = nb.world.policy_pack_c(**p)
        with pytest.raises(ValueError):
            reference_write_policy_pack(pk, tmp_path / f"{name}.ref.mrpolicy")
        del keep
