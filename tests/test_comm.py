"""The library's communicator (msf_comm_*): the TCP bootstrap through rank 0
and the host all-gather that a sharded raster uses for its exchange when
ranks share a GPU.  No GPU: ranks are CPU processes (spawned), and the
failure cases are made on the host (a rank that never joins, a rank that
exits before the exchange); each must end the other rank's call with
MSF_ERR_TIMEOUT or an I/O error within the communicator's timeout, never a
hang."""
import multiprocessing as mpp
import os
import socket
import tempfile
import time

import numpy as np
import pytest

import msf

MSF_ERR_ARG, MSF_ERR_TIMEOUT = 1, 7


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _gather_rank(rank, world, port, out_dir):
    c = msf.Comm(rank, world, "127.0.0.1:%d" % port, msf.COMM_HOST, timeout_s=30)
    mine = np.arange(5, dtype=np.float64) + 100.0 * rank
    got = c.allgather(mine)
    # a second exchange of another size on the same connections
    got2 = c.allgather(np.full((2, 3), rank, dtype=np.int32))
    np.savez(os.path.join(out_dir, "rank%d.npz" % rank), got=got, got2=got2)
    c.close()


def _spawn(target, world, *args, timeout=120):
    ctx = mpp.get_context("spawn")
    procs = [ctx.Process(target=target, args=(r, world) + args) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=timeout)
    alive = [p for p in procs if p.is_alive()]
    for p in alive:
        p.kill()
    assert not alive, "a rank hung"
    return procs


@pytest.mark.parametrize("world", [2, 3])
def test_host_allgather_over_ranks(world):
    with tempfile.TemporaryDirectory() as out:
        procs = _spawn(_gather_rank, world, free_port(), out)
        assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
        want = np.stack([np.arange(5, dtype=np.float64) + 100.0 * r for r in range(world)])
        want2 = np.stack([np.full((2, 3), r, dtype=np.int32) for r in range(world)])
        for r in range(world):
            d = np.load(os.path.join(out, "rank%d.npz" % r))
            assert np.array_equal(d["got"], want)
            assert np.array_equal(d["got2"], want2)


def test_single_rank_needs_no_rendezvous():
    c = msf.Comm(0, 1)
    a = np.array([1.5, 2.5])
    assert np.array_equal(c.allgather(a), a[None])
    c.close()


def test_argument_checks():
    with pytest.raises(msf.MsfError) as e:
        msf.Comm(2, 2, "127.0.0.1:1")
    assert e.value.status == MSF_ERR_ARG
    with pytest.raises(msf.MsfError) as e:
        msf.Comm(0, 2, "")
    assert e.value.status == MSF_ERR_ARG
    with pytest.raises(msf.MsfError) as e:
        msf.Comm(0, 2, "no-port-here")
    assert e.value.status == MSF_ERR_ARG


def test_missing_rank_times_out():
    """Rank 0 of a world of two whose other rank never joins."""
    t0 = time.time()
    with pytest.raises(msf.MsfError) as e:
        msf.Comm(0, 2, "127.0.0.1:%d" % free_port(), msf.COMM_HOST, timeout_s=1.5)
    assert e.value.status == MSF_ERR_TIMEOUT
    assert "more rank" in str(e.value)
    assert time.time() - t0 < 20


def _dies_before_exchange(rank, world, port, out_dir):
    c = msf.Comm(rank, world, "127.0.0.1:%d" % port, msf.COMM_HOST, timeout_s=5)
    if rank == 1:
        os._exit(3)  # between steps: joined, then gone before the exchange
    t0 = time.time()
    try:
        c.allgather(np.zeros(4))
        outcome = "no-error"
    except msf.MsfError as ex:
        outcome = "error:%d" % ex.status
    with open(os.path.join(out_dir, "rank0.txt"), "w") as f:
        f.write("%s %.1f\n" % (outcome, time.time() - t0))


def test_rank_that_exits_surfaces_as_error_not_hang():
    with tempfile.TemporaryDirectory() as out:
        procs = _spawn(_dies_before_exchange, 2, free_port(), out)
        assert procs[1].exitcode == 3
        outcome, seconds = open(os.path.join(out, "rank0.txt")).read().split()
        assert outcome.startswith("error:"), outcome
        assert float(seconds) < 30.0
