"""Time-step pipeline (hipace2_b200/pipeline.py, the reference's MultiBuffer): rank r runs steps
r, r+N, ... and hands each finished beam slice to rank r+1. The reference's own tests of this
mode run the same deck on 1 and 2 ranks and compare (tests/*.2Rank.sh). Here:

* CPU: 2 and 3 gloo ranks, each driving the FP64 oracle, reproduce the fields of the last step
  and the beam after it of a 1-rank run bit for bit (the oracle's sums do not depend on the
  thread count, and the hand-off moves the very particles the 1-rank run keeps);
* GPU: 2 processes on one GPU (host-staged gloo transport), each driving the library in
  deterministic mode, reproduce a 1-process run bit for bit.
"""
import datetime
import os
import socket

import numpy as np
import pytest

from cases import EXPLICIT_MOVING

# moving beam with momentum spread (particles slip between slices), 5 steps of dt = 20
DECK = EXPLICIT_MOVING.replace("max_step = 2", "max_step = 4")
N_STEPS = 5
DT = 20.0
COMPS = ["Ez", "Bx", "By", "Psi", "jz_beam", "rhomjz"]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


class OracleEngine:
    def __init__(self, o):
        self.o, self.step = o, None

    def begin_step(self, step):
        self.step = step
        self.o.begin_step(step)

    def solve_slice(self, islice):
        assert self.o.solve_slice(islice, self.step) == 0

    def end_step(self):
        self.o.end_step()

    def get_beam_slice(self, b, islice):
        return self.o.get_beam_slice(b, islice)

    def put_beam_slice(self, b, islice, beam):
        self.o.put_beam_slice(b, islice, beam)

    def set_time(self, t):
        self.o.set_time(t)


def _sorted_beam(b):
    o = np.argsort(b["id"], kind="stable")
    return {k: v[o] for k, v in b.items()}


def _worker(kind, rank, world, port, q):
    # a few OpenMP threads per rank: the ranks share the host's cores (the oracle's results do
    # not depend on the thread count)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), OMP_NUM_THREADS="2")
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    from hipace2_b200.pipeline import HipaceEngine, TorchTransport, run_pipeline
    if kind == "oracle":
        from oracle_lib import Oracle
        o = Oracle(DECK)
        o.init_beams()
        o.set_diag(COMPS)
        eng, nz = OracleEngine(o), o.nz
    else:
        import hipace2_b200 as hp
        o = hp.Hipace(DECK, graphs=True, deterministic=True)
        o.init_data()
        o.set_diag(COMPS)
        eng, nz = HipaceEngine(o), o.n_cell[2]
    ran = run_pipeline(eng, N_STEPS, nz, 1, DT, TorchTransport("cpu"), rank, world)
    out = None
    if N_STEPS - 1 in ran:
        out = ({k: o.get_diag(k) for k in COMPS}, _sorted_beam(o.get_beam(0)))
    q.put((rank, ran, out))
    dist.barrier()
    dist.destroy_process_group()


def _run_ranks(kind, world):
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(kind, r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=600) for _ in procs]
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    steps = sorted(s for _, ran, _ in res for s in ran)
    assert steps == list(range(N_STEPS))
    return next(out for _, _, out in res if out is not None)


def _compare(ref_fields, ref_beam, got):
    fields, beam = got
    for k in COMPS:
        assert np.array_equal(fields[k], ref_fields[k]), k
    assert np.array_equal(beam["id"], ref_beam["id"])
    for k in ("x", "y", "z", "w", "ux", "uy", "uz"):
        assert np.array_equal(beam[k], ref_beam[k]), k


@pytest.mark.parametrize("world", [2, 3])
def test_oracle_pipeline_reproduces_one_rank_bit_for_bit(world):
    from oracle_lib import Oracle
    o = Oracle(DECK)
    o.init_beams()
    o.set_diag(COMPS)
    for s in range(N_STEPS):
        assert o.step(s) == 0
    ref = ({k: o.get_diag(k) for k in COMPS}, _sorted_beam(o.get_beam(0)))
    _compare(ref[0], ref[1], _run_ranks("oracle", world))


def test_pipeline_single_rank_is_the_plain_step_loop():
    """world == 1: the driver is the per-slice step loop, with no transport."""
    from oracle_lib import Oracle
    from hipace2_b200.pipeline import run_pipeline
    a, b = Oracle(DECK), Oracle(DECK)
    for o in (a, b):
        o.init_beams()
        o.set_diag(COMPS)
    for s in range(N_STEPS):
        assert a.step(s) == 0
    assert run_pipeline(OracleEngine(b), N_STEPS, b.nz, 1, DT, None, 0, 1) == list(range(N_STEPS))
    for k in COMPS:
        assert np.array_equal(a.get_diag(k), b.get_diag(k)), k


@pytest.mark.gpu
def test_library_pipeline_two_processes_reproduce_one_process():
    import hipace2_b200 as hp
    o = hp.Hipace(DECK, graphs=True, deterministic=True)
    o.init_data()
    o.set_diag(COMPS)
    for s in range(N_STEPS):
        o.step(s)
    ref = ({k: o.get_diag(k) for k in COMPS}, _sorted_beam(o.get_beam(0)))
    o.close()
    _compare(ref[0], ref[1], _run_ranks("gpu", 2))
