"""bench.py's rank set-up (no GPU): `--gpus N` without a launcher starts N
ranks through torch.distributed.run, a launcher's ranks are used as they
are, and a request that cannot be met exits non-zero instead of measuring on
fewer GPUs than asked."""
import sys

import pytest

import bench


def test_two_gpus_without_a_launcher_start_two_ranks():
    cmd = bench.spawn_command(2, {}, ["--gpus", "2", "--steps", "3"], device_count=8)
    assert cmd[:3] == [sys.executable, "-m", "torch.distributed.run"]
    assert "--nproc-per-node=2" in cmd
    assert cmd[cmd.index("--master-addr") + 1] == "127.0.0.1"
    assert cmd[-4:] == ["--gpus", "2", "--steps", "3"]
    assert cmd[-5].endswith("bench.py")


def test_a_rank_of_a_launcher_runs_itself():
    assert bench.spawn_command(2, {"WORLD_SIZE": "2"}, [], device_count=0) is None
    assert bench.spawn_command(1, {}, [], device_count=0) is None
    assert bench.spawn_command(1, {"WORLD_SIZE": "1"}, [], device_count=1) is None


def test_requests_that_cannot_be_met_exit_non_zero():
    with pytest.raises(SystemExit) as e:
        bench.spawn_command(4, {}, [], device_count=2)
    assert e.value.code != 0
    with pytest.raises(SystemExit):
        bench.spawn_command(2, {"WORLD_SIZE": "4"}, [], device_count=8)
    with pytest.raises(SystemExit):
        bench.spawn_command(0, {}, [], device_count=8)


def test_reference_arm_needs_no_gpus_to_start_ranks():
    cmd = bench.spawn_command(2, {}, ["--impl", "reference"], device_count=0,
                              needs_gpus=False)
    assert "--nproc-per-node=2" in cmd
