"""TaskPack files (mr_task_pack_inspect, mr_task_pack_rewrite) against the
reference's own writer and reader (writeTaskPack / readTaskPack,
src/core/LearningPacks.cpp, compiled into oracle/_ref): the capacity
profile's size, each side reads the other's files field for field, a file
read and written again keeps its bytes, the artifact rules refuse the same
packs, corrupt files are refused.  No device work."""

from __future__ import annotations

import struct

import pytest

import numi_lab_b200 as nb
from numi_lab_b200 import native
from numi_lab_b200.native import MetalRoboError

pytestmark = pytest.mark.reference


def _rehash(data: bytearray) -> bytes:
    payload = bytes(data[32:])
    struct.pack_into("<QQ", data, 16, len(payload), native.bindings().lib.mr_learning_pack_content_hash(payload, len(payload)))
    return bytes(data)


def test_capacity_profile_is_27_words(reference_available):
    from oracle import reference_capacity_profile_bytes

    assert reference_capacity_profile_bytes() == 27 * 4


def test_reference_packs_read_and_rewrite_byte_for_byte(tmp_path, reference_available):
    from oracle import reference_inspect_task_pack, reference_write_task_pack

    for variant in (0, 1):
        ref = tmp_path / f"ref{variant}.mrtask"
        reference_write_task_pack(variant, ref)
        head = ref.read_bytes()[:32]
        assert head[:8] == b"MRLEARN\0" and struct.unpack_from("<II", head, 8) == (17, 1)
        mine = nb.world.inspect_task_pack(ref)
        theirs = reference_inspect_task_pack(ref)
        assert mine == theirs, variant
        again = tmp_path / f"again{variant}.mrtask"
        nb.world.rewrite_task_pack(ref, again)
        assert again.read_bytes() == ref.read_bytes(), variant
    full = nb.world.inspect_task_pack(tmp_path / "ref0.mrtask")
    assert (full["action_count"], full["outcome_count"], full["contact_group_count"], full["joint_group_count"],
            full["reward_count"], full["termination_count"], full["terrain_sample_count"], full["motion_tracked_body_count"],
            full["maximum_episode_steps"], full["difficulty_band_count"]) == (5, 2, 2, 2, 3, 2, 3, 2, 750, 5)
    assert full["id"] == "full_task_pack" and full["support_force_threshold"] == 2.0


def test_artifact_rules_refuse_the_same_packs(tmp_path, reference_available):
    from oracle import reference_rewrite_task_pack, reference_write_task_pack

    ref = tmp_path / "ref.mrtask"
    reference_write_task_pack(0, ref)
    data = bytearray(ref.read_bytes())
    # The tail: ..., u32 episode steps, u32 bands, f32 authority, f32 reset
    # fraction, 5 initial positions (u64 + 20 B), 3 u8 flags, 5 f32.
    at = len(data) - (20 + 3 + 28 + 4 + 4 + 4 + 4)
    assert struct.unpack_from("<I", data, at)[0] == 750
    cases = {"episode steps": (at, "<I", 0), "authority": (at + 8, "<f", 1.5)}
    for name, (offset, fmt, value) in cases.items():
        bad = bytearray(data)
        struct.pack_into(fmt, bad, offset, value)
        src = tmp_path / f"{name}.mrtask"
        src.write_bytes(_rehash(bad))
        nb.world.inspect_task_pack(src)  # readers do not apply the writer's rules
        with pytest.raises(MetalRoboError, match="TaskPack"):
            nb.world.rewrite_task_pack(src, tmp_path / f"{name}.mine")
        with pytest.raises(ValueError):
            reference_rewrite_task_pack(src, tmp_path / f"{name}.ref")


def test_corrupt_and_foreign_files_are_refused(tmp_path, reference_available):
    from oracle import reference_write_task_pack

    ref = tmp_path / "ref.mrtask"
    reference_write_task_pack(1, ref)
    data = ref.read_bytes()
    cases = {
        "bit": (data[:-5] + bytes([data[-5] ^ 1]) + data[-4:], "hash"),
        "version": (data[:8] + struct.pack("<I", 16) + data[12:], "version"),
        "kind": (data[:12] + struct.pack("<I", 3) + data[16:], "kind"),
        "truncated": (data[:-3], "length"),
    }
    for name, (blob, message) in cases.items():
        p = tmp_path / f"{name}.mrtask"
        p.write_bytes(blob)
        with pytest.raises(MetalRoboError, match=message):
            nb.world.inspect_task_pack(p)
