"""CPU: the N > 1 path of bench.py, with world_size-2 gloo process groups.

Every rank runs its own replica (the timestep path needs no collective), the
job's time is the slowest rank's (max over ranks), and the whole-job value
counts every rank's cells. The reference arm under torchrun runs on rank 0
alone and prints one line; the other ranks exit 0 without work.
"""
import argparse
import json
import datetime
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=120))
    try:
        t = bench.max_over_ranks(dist, 1.5 + rank, device="cpu")  # rank r "took" 1.5 + r
        with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
            json.dump({"max": t, "value": bench.whole_job_value(world, 1000, 10, t)}, f)
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_whole_job_value_gloo(tmp_path):
    import torch.multiprocessing as mp
    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world,
                       start_method="spawn", join=True)
    got = [json.load(open(tmp_path / f"rank{r}.json")) for r in range(world)]
    for g in got:
        assert g["max"] == 2.5  # every rank sees the slowest rank's time
        assert g["value"] == pytest.approx(world * 1000 * 10 / 2.5 / 1e6)


def test_whole_job_value_single_rank():
    assert bench.max_over_ranks(None, 3.25) == 3.25
    assert bench.whole_job_value(1, 512 ** 3, 1000, 1.5) == pytest.approx(512 ** 3 * 1000 / 1.5 / 1e6)


def test_reference_arm_under_torchrun_prints_once():
    env = dict(os.environ, WF_REF_SECONDS="5")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()), "bench.py",
           "--impl", "reference", "--grid", "64", "--steps", "2", "--warmup", "3"]
    r = subprocess.run(cmd, cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["steps"] == 2 and d["warmup"] == 3
    assert d["e2e"]["value"] == d["value"] and d["cpu_baseline"]["kind"] == "port"


def test_reference_arm_maps_only_the_oracle():
    """bench.py --impl reference builds the workload with the oracle's own
    voxelizer and tables: after a run in a fresh process, the CUDA library was
    never loaded there, and the oracle's shared object was."""
    code = (
        "import sys, json; sys.argv=['bench.py','--impl','reference','--grid','64','--steps','2',"
        "'--warmup','3']; import bench; bench.main();"
        "import wavefront_b200._lib as L;"
        "maps=open('/proc/self/maps').read();"
        "print(json.dumps({'lib': L._lib is None, 'gpu_so': 'libwavefront_gpu.so' in maps,"
        "'oracle_so': 'libwforacle.so' in maps}))")
    env = dict(os.environ, WF_REF_SECONDS="5")
    r = subprocess.run([sys.executable, "-c", code], cwd=ROOT, env=env, capture_output=True,
                       text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [json.loads(l) for l in r.stdout.splitlines() if l.startswith("{")]
    assert lines[0]["impl"] == "reference"
    assert lines[-1] == {"lib": True, "gpu_so": False, "oracle_so": True}


@pytest.mark.parametrize("which", ["two_spheres", "demo_sphere", "random_spheres"])
def test_oracle_description_tables_equal_the_products(which):
    """The oracle's tables built from a workload description (ids, Q16.16
    table, graded depth per axis) equal those of the Scenario the CUDA path
    runs, built from the same description by the library's host code."""
    import numpy as np
    from oracle import oracle as O
    from wavefront_b200 import configs
    desc = {"two_spheres": lambda: configs.two_spheres_desc(n=64, steps=4),
            "demo_sphere": lambda: configs.demo_sphere_cube_desc(n=64, steps=4),
            "random_spheres": lambda: configs.random_spheres_desc(n=64, steps=4)}[which]()
    sc = configs.from_desc(desc)
    ids, table = O.tables_from_description(desc)
    assert np.array_equal(ids, sc.grid.ids)
    assert np.array_equal(table, sc.table.q16)
    assert O.pml_thickness_from_description(desc) == tuple(sc.pml.thickness_voxels)


def _slab_bench_main(rank, world, port, out_dir):
    """One rank of bench.py's slab leg (the path `--gpus N` takes under
    torchrun), with the oracle stepping each slab and gloo moving the ghost
    blocks; rank 0's JSON line goes to a file."""
    import contextlib
    import io
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from test_slabs import OracleSlabState
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK="0")
    bench.GRID = 64
    bench.N_CELLS = 64 ** 3
    args = argparse.Namespace(workload="two_spheres", steps=12, warmup=3, tiling="",
                              backend="gloo")
    buf = io.StringIO()
    with contextlib.redirect_stdout(buf):
        bench.run_slab_ranks(args, rank, world, 0, make_state=OracleSlabState)
    with open(os.path.join(out_dir, f"slab{rank}.txt"), "w") as f:
        f.write(buf.getvalue())


def test_bench_slab_leg_two_gloo_ranks(tmp_path):
    """bench.py's z-slab leg (`--gpus N` under torchrun) with world_size 2:
    both ranks step their slab, exchange ghost blocks, agree on the slowest
    rank's time, and rank 0 alone prints one strong-scaling line whose value
    counts the whole grid's cells once, with an end-to-end figure."""
    import torch.multiprocessing as mp
    world = 2
    mp.start_processes(_slab_bench_main, args=(world, _free_port(), str(tmp_path)), nprocs=world,
                       start_method="spawn", join=True)
    lines = [l for l in (tmp_path / "slab0.txt").read_text().splitlines() if l.startswith("{")]
    assert len(lines) == 1
    assert not (tmp_path / "slab1.txt").read_text().strip()
    d = json.loads(lines[0])
    assert d["scaling"] == "strong" and d["ranks"] == 2 and d["config"]["slabs"] == 2
    assert d["steps"] == 12 and d["value"] > 0
    # value is printed to 0.1 and ms_per_step to 1e-4: allow both roundings
    assert d["value"] == pytest.approx(64 ** 3 * 12 / (d["ms_per_step"] * 12 / 1e3) / 1e6, rel=1e-3,
                                       abs=0.06)
    assert d["e2e"]["value"] > 0 and d["e2e"]["h2d_bytes_per_step"] > 0
    assert d["config"]["rank0_planes_stepped_per_step"] == 32 + 8


def test_e2e_leg_sends_the_scene_text(monkeypatch):
    """The e2e leg's workload leaves a text scene to the device voxelizer
    (only the text crosses the host link); the device-resident leg keeps the
    host-voxelized ids; a scene without text (demo sphere) keeps its ids."""
    import argparse
    from wavefront_b200 import configs
    monkeypatch.setattr(bench, "GRID", 64)
    args = argparse.Namespace(workload="two_spheres")
    dev = bench.scenario(args, 10, device_voxelize=True)
    host = bench.scenario(args, 10)
    assert dev.grid is None and dev.scene_text == configs.two_spheres_text(64)
    assert host.grid is not None and host.scene_text is None
    assert host.grid.ids.any()
    demo = bench.scenario(argparse.Namespace(workload="demo_sphere"), 10, device_voxelize=True)
    assert demo.grid is not None and demo.scene_text is None
