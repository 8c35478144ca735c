"""The multi-rank plumbing of ``bench.py`` on CPU: two ``gloo`` ranks on 127.0.0.1.

``bench.py --gpus N`` runs N independent replicas of the pass (no data-path collective); its only collective is the
max over ranks of each device time (timed passes, plain form, end to end), so that the slowest replica sets the
job's time.  These tests check that reduction with world size 2 and that one rank makes no collective call, and
that the reference arm does its work on rank 0 only; and that the bench's FFT roofline geometry matches the
library source.
"""

from __future__ import annotations

import os
import socket

import pytest


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, values, out_dir: str) -> None:
    import datetime

    import torch.distributed as dist

    import bench

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        got = [bench.max_over_ranks(v, world, device="cpu") for v in values[rank]]
        with open(os.path.join(out_dir, f"rank{rank}.txt"), "w") as fh:
            fh.write(" ".join(repr(x) for x in got))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_two_gloo_ranks(tmp_path):
    import torch.multiprocessing as mp

    # three reductions in the same order on both ranks (timed passes, plain form, end to end)
    values = [[0.61, 9.7, 0.64], [0.58, 9.9, 0.66]]
    mp.spawn(_rank_main, args=(2, _free_port(), values, str(tmp_path)), nprocs=2, join=True)
    for rank in range(2):
        got = [float(x) for x in (tmp_path / f"rank{rank}.txt").read_text().split()]
        assert got == [0.61, 9.9, 0.66]


def test_max_over_ranks_single_rank_makes_no_collective_call():
    import torch.distributed as dist

    import bench

    assert not dist.is_initialized()
    assert bench.max_over_ranks(0.5, 1) == 0.5  # would raise if it called a collective without a process group


@pytest.mark.parametrize("rank", ["1", "3"])
def test_reference_arm_runs_on_rank_zero_only(monkeypatch, capsys, rank):
    import bench

    monkeypatch.setenv("RANK", rank)

    class Args:
        config = 5
        cpu_nodes = 8

    bench.run_reference(Args())  # returns before any work on ranks other than 0
    assert capsys.readouterr().out == ""


def test_roofline_fft_geometry_matches_the_library_source():
    """The FFT byte counts of the bench's roofline assume the library's in-register box lengths and pass-3 block
    height (map planes per CTA); both are read here from the CUDA sources so that the two cannot drift apart."""
    import re

    import bench

    csrc = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "pyaldvc_b200", "csrc")
    reg = open(os.path.join(csrc, "fft_reg.cuh")).read()
    sizes = re.search(r"FFTR_SIZES\[FFTR_NSIZES\]\s*=\s*\{([^}]*)\}", reg).group(1)
    assert tuple(int(v) for v in sizes.split(",")) == bench.FFT_REG_SIZES
    ncc = open(os.path.join(csrc, "ncc.cu")).read()
    body = ncc[ncc.index("constexpr int fftr_planes3()"):][:400]
    assert "70000 / (N * (NH | 1) * 8)" in body and "256 / NH" in body


def test_reference_arm_uses_neither_the_device_nor_the_cuda_library():
    """bench.py --impl reference runs the oracle pass on host-rendered volumes: in a fresh process it loads no
    library of this package, imports neither torch nor the device modules, and prints one JSON line."""
    import json
    import subprocess
    import sys

    repo = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    probe = (
        "import sys, runpy, io, contextlib\n"
        "sys.argv = ['bench.py', '--impl', 'reference', '--config', '1', '--cpu-nodes', '2', '--steps', '1', '--warmup', '0']\n"
        "buf = io.StringIO()\n"
        "with contextlib.redirect_stdout(buf):\n"
        "    runpy.run_path('bench.py', run_name='__main__')\n"
        "maps = open('/proc/self/maps').read()\n"
        "print(buf.getvalue().strip())\n"
        "print('LOADED', 'libaldvc_b200' in maps, 'torch' in sys.modules, 'pyaldvc_b200.kernels' in sys.modules)\n"
    )
    r = subprocess.run([sys.executable, "-c", probe], cwd=repo, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = r.stdout.strip().splitlines()
    assert lines[-1] == "LOADED False False False"
    line = json.loads(lines[-2])
    assert line["impl"] == "reference" and line["value"] > 0 and line["cpu_baseline"]["kind"] == "port"
    assert line["e2e"]["h2d_bytes_per_step"] == 0
