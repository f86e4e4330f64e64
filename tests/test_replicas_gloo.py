"""The multi-GPU path is replicas only (one process per GPU, no collective on the data path): two
gloo ranks on CPU, launched the way the benchmark is launched (torch.distributed.run, 127.0.0.1),
split the campaign's instances between them without overlap or loss, and reduce the timed region
to its maximum over ranks (the whole-job time)."""
import json
import os
import socket
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_ranks_split_instances_and_take_the_slowest_time(tmp_path):
    env = dict(os.environ, PYTHONPATH=str(ROOT) + os.pathsep + os.environ.get("PYTHONPATH", ""),
               CUDA_VISIBLE_DEVICES="")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()),
           str(ROOT / "tests" / "replicas_worker.py"), str(tmp_path)]
    r = subprocess.run(cmd, cwd=ROOT, env=env, capture_output=True, text=True, timeout=240)
    assert r.returncode == 0, r.stderr[-2000:]
    outs = [json.loads((tmp_path / f"rank{k}.json").read_text()) for k in range(2)]
    assert [o["rank"] for o in outs] == [0, 1] and all(o["world"] == 2 for o in outs)
    assert [o["local"] for o in outs] == [0, 1]
    a, b = outs[0]["share"], outs[1]["share"]
    assert not set(a) & set(b) and sorted(a + b) == list(range(24)) and len(a) == len(b) == 12
    assert all(o["max"] == pytest.approx(13.5) for o in outs)          # max(10.0, 13.5) on every rank
    assert all(o["total"] == 24 for o in outs)
    assert [o["seed"] for o in outs] == [7, 8]


def test_single_process_helpers_need_no_process_group(monkeypatch):
    from bug_defense_b200 import replicas
    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    assert replicas.dist_env() == (0, 1, 0)
    assert replicas.max_over_ranks(2.5) == 2.5 and replicas.sum_over_ranks(3) == 3.0
    assert replicas.rank_share(list("abcde"), 1, 2) == ["b", "d"]
    monkeypatch.setenv("RANK", "2")
    monkeypatch.setenv("WORLD_SIZE", "2")
    with pytest.raises(ValueError):
        replicas.dist_env()
