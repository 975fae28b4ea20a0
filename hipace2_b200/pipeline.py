"""Time-step pipeline across processes: the reference's MultiBuffer (src/utils/MultiBuffer.cpp).

The quasi-static slice march is serial within a time step, but consecutive steps only couple
through the beam: step s+1 needs, for slice i, the particles that slice i of step s handed on after
its beam push. The reference therefore runs step r, r+N, r+2N, ... on rank r and passes each
finished beam slice from rank r to rank r+1 while both march (Hipace.cpp:401, get_data/put_data
around SolveOneSlice, MultiBuffer.cpp:181-430). Rank r+1 can start a slice as soon as the two
slices it reads (this one, and the next one for the jx/jy beam deposit) have arrived, so the N
ranks march N consecutive steps a few slices apart.

Here each rank drives one simulation through the per-slice surface of the C ABI
(hpq_begin_step / hpq_solve_slice / hpq_end_step) and moves slices with hpq_get_beam_slice and
hpq_put_beam_slice; the transport is torch.distributed point-to-point: NCCL with device tensors
between GPUs, gloo with host tensors otherwise. The plasma is created anew every step and the
fields of one step do not feed the next, so nothing else crosses ranks. Every rank sets the
physical time of the step it runs (hpq_set_time).

An `engine` is any object with begin_step(step), solve_slice(islice), end_step(),
get_beam_slice(b, islice), put_beam_slice(b, islice, beam) and set_time(t): `Hipace` through
`HipaceEngine`, or a CPU restatement with the same methods.
"""
import collections

import numpy as np

BEAM_KEYS = ("x", "y", "z", "w", "ux", "uy", "uz")


class HipaceEngine:
    """The pipeline's view of a `hipace2_b200.Hipace` simulation."""

    def __init__(self, sim):
        self.sim = sim

    def begin_step(self, step):
        self.sim.begin_step(step)

    def solve_slice(self, islice):
        self.sim.solve_one_slice(islice)

    def end_step(self):
        self.sim.end_step()

    def get_beam_slice(self, b, islice):
        return self.sim.get_beam_slice(b, islice)

    def put_beam_slice(self, b, islice, beam):
        self.sim.put_beam_slice(b, islice, beam)

    def set_time(self, t):
        self.sim.set_time(t)


class TorchTransport:
    """Beam slices between ranks over torch.distributed. A slice is two messages: its particle
    count (int64), then, if it is not empty, an 8 x n float64 array (x y z w ux uy uz and the ids,
    whose int64 bits travel unchanged). `device` is "cpu" for gloo, a CUDA device for NCCL."""

    def __init__(self, device="cpu"):
        import torch
        import torch.distributed as dist
        self.torch, self.dist, self.device = torch, dist, device

    def send(self, beam, dst):
        """Non-blocking; returns (work handles, tensors to keep alive until they complete)."""
        torch, dist = self.torch, self.dist
        n = int(beam["x"].size)
        head = torch.tensor([n], dtype=torch.int64, device=self.device)
        works, keep = [dist.isend(head, dst)], [head]
        if n:
            a = np.empty((8, n))
            for r, k in enumerate(BEAM_KEYS):
                a[r] = beam[k]
            a[7] = np.ascontiguousarray(beam["id"], dtype=np.int64).view(np.float64)
            t = torch.from_numpy(a).to(self.device)
            works.append(dist.isend(t, dst))
            keep.append(t)
        return works, keep

    def recv(self, src):
        torch, dist = self.torch, self.dist
        head = torch.zeros(1, dtype=torch.int64, device=self.device)
        dist.recv(head, src)
        n = int(head.item())
        out = {k: np.zeros(0) for k in BEAM_KEYS}
        out["id"] = np.zeros(0, dtype=np.int64)
        if n:
            t = torch.empty((8, n), dtype=torch.float64, device=self.device)
            dist.recv(t, src)
            a = t.cpu().numpy()
            for r, k in enumerate(BEAM_KEYS):
                out[k] = a[r].copy()
            out["id"] = a[7].copy().view(np.int64)
        return out


def run_pipeline(engine, n_steps, nz, n_beams, dt, transport, rank, world, t0=0.0, on_step=None):
    """March steps rank, rank + world, ... < n_steps of the time-step pipeline.

    Before slice i is solved, the slices down to i - 1 of this step have been received from
    rank - 1 (slice i - 1 is read by slice i's jx/jy beam deposit); after slice i is solved,
    slice i + 1 is final and goes to rank + 1 (slice 0 after the step ends). Sends do not block:
    they complete while the next rank consumes them. Step 0 uses the engine's own beam; with
    world == 1 every step does. `on_step(step)` runs after each step of this rank (diagnostics).
    Returns the steps this rank ran."""
    prev, nxt = (rank - 1) % world, (rank + 1) % world
    pending = collections.deque()
    ran = []
    for step in range(rank, n_steps, world):
        recv = world > 1 and step > 0
        send = world > 1 and step + 1 < n_steps
        engine.set_time(t0 + step * dt)
        engine.begin_step(step)
        state = {"got": nz, "sent": nz}

        def need(lo):
            while recv and state["got"] > lo:
                state["got"] -= 1
                for b in range(n_beams):
                    engine.put_beam_slice(b, state["got"], transport.recv(prev))

        def flush(lo):
            while send and state["sent"] > lo:
                state["sent"] -= 1
                for b in range(n_beams):
                    pending.append(transport.send(engine.get_beam_slice(b, state["sent"]), nxt))

        for i in range(nz - 1, -1, -1):
            need(max(i - 1, 0))
            engine.solve_slice(i)
            flush(i + 1)
        engine.end_step()
        flush(0)
        # release the sends the next rank has already taken
        while pending and all(w.is_completed() for w in pending[0][0]):
            pending.popleft()
        ran.append(step)
        if on_step:
            on_step(step)
    while pending:
        works, _ = pending.popleft()
        for w in works:
            w.wait()
    return ran
