"""Multi-GPU path (replicas of independent scans) on CPU: world-size-2 gloo
process groups exercise the scan assignment, the max-over-ranks timing and a
rank that fails between steps."""
import datetime
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from ctbb_icd_b200 import replicas as R


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, mode, out):
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=10))
    try:
        specs = R.batch_specs(32, seed=0)
        costs = [R.scan_cost(s) for s in specs]
        mine = R.my_scans(costs, world, rank)
        if mode == "fail" and rank == 1:
            os._exit(3)  # leaves between steps, with nothing in flight
        gathered = [None] * world
        dist.all_gather_object(gathered, mine)
        t = R.max_over_ranks(10.0 * (rank + 1), dist)
        out[rank] = (gathered, t)
    except Exception as e:  # noqa: BLE001
        out[rank] = ("error", type(e).__name__)
    finally:
        if dist.is_initialized():
            try:
                dist.destroy_process_group()
            except Exception:  # noqa: BLE001
                pass


def _run(world, mode):
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, mode, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    for p in procs:
        if p.is_alive():
            p.kill()
    return dict(out), [p.exitcode for p in procs]


def test_batch_specs_are_seeded_and_uneven():
    a, b = R.batch_specs(32, seed=0), R.batch_specs(32, seed=0)
    assert a == b
    sizes = {s["prm"]["nx"] for s in a}
    rows = {s["prm"]["Nrows"] for s in a}
    assert len(a) == 32 and len(sizes) >= 3 and len(rows) >= 3
    assert {s["prm"]["Phiffs"] for s in a} == {0, 1}


def test_batch_specs_configure_and_fit_the_scan(tmp_path):
    import ctbb_icd_b200 as C
    from ctbb_icd_b200 import workloads as W

    for s in R.batch_specs(32, seed=0):
        prm = dict(s["prm"], sinogram_path=str(tmp_path / "r.bin"), output_dir=str(tmp_path), output_file="o.img")
        rp = C.configure_recon_params(W.write_prm(str(tmp_path / f"{s['name']}.prm"), prm))
        tables = C.slice_tables(rp)  # raises CTBB_ERR_RANGE if the slab is outside the scan
        # the slice thickness is snapped to whole table steps (setup.cpp:207)
        assert len(tables.slice_indices) == rp.geom.num_voxels_z >= 7


def test_assignment_is_a_balanced_partition():
    costs = [R.scan_cost(s) for s in R.batch_specs(32, seed=0)]
    for world in (1, 2, 3, 8):
        plan = R.assign(costs, world)
        flat = sorted(i for p in plan for i in p)
        assert flat == list(range(32))
        loads = [sum(costs[i] for i in p) for p in plan]
        assert max(loads) <= sum(costs) / world + max(costs)


def test_two_gloo_ranks_split_scans_and_time_by_max():
    out, codes = _run(2, "ok")
    assert codes == [0, 0]
    (g0, t0), (g1, t1) = out[0], out[1]
    assert g0 == g1
    assert sorted(g0[0] + g0[1]) == list(range(32)) and not set(g0[0]) & set(g0[1])
    assert t0 == t1 == 20.0


@pytest.mark.timeout(120)
def test_rank_leaving_between_steps_is_detected_on_the_host():
    out, codes = _run(2, "fail")
    assert codes[1] == 3
    # The surviving rank's next collective ends with an error instead of hanging.
    assert out[0][0] == "error"
