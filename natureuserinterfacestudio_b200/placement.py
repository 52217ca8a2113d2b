"""Placement of RGB-D streams on the GPUs of one node (sessions -> GPUs at admission).

Sessions are independent: a stream lives on one GPU for its whole life, and the data path
has no collective.  What the GPUs share is the admission decision.  Rank 0 keeps every
GPU's HBM budget; an arriving stream goes to the GPU with the most free budget that can
hold its session (the bytes `nui_session_device_bytes` reports plus its frame buffers), and
waits when none can; a released stream returns its bytes to its GPU.  The decisions reach
every rank through one object broadcast per admission round (gloo on CPU, NCCL on GPUs),
so that each rank admits exactly the streams placed on it into its own serving loop
(`nui_server_*`).  The reference serves one stream on one device and has no counterpart.
"""


class Placement:
    """Most-free-budget placement over n GPUs (host state of rank 0)."""

    def __init__(self, budgets):
        self.budget = [int(b) for b in budgets]
        self.used = [0] * len(self.budget)
        self.where = {}  # stream id -> (gpu, bytes)

    def free(self, gpu):
        return self.budget[gpu] - self.used[gpu]

    def place(self, stream, need):
        """GPU index for the stream (its bytes charged there), or -1 if no GPU can hold it."""
        if stream in self.where:
            raise ValueError("stream %r is already placed" % (stream,))
        best = -1
        for g in range(len(self.budget)):
            if self.free(g) >= need and (best < 0 or self.free(g) > self.free(best)):
                best = g
        if best >= 0:
            self.used[best] += int(need)
            self.where[stream] = (best, int(need))
        return best

    def release(self, stream):
        gpu, need = self.where.pop(stream)
        self.used[gpu] -= need
        return gpu


def place_round(placement, arrivals, releases, rank, world):
    """One admission round on every rank: rank 0 releases the finished streams and places the
    arrivals (a list of (stream id, bytes)), then broadcasts the decisions.  Returns, on every
    rank, (admitted: stream ids placed on this rank, waiting: stream ids no GPU could hold)."""
    import torch.distributed as dist
    decisions = [None]
    if rank == 0:
        for s in releases:
            placement.release(s)
        decisions[0] = [(s, placement.place(s, need)) for s, need in arrivals]
    if world > 1:
        dist.broadcast_object_list(decisions, src=0)
    mine = [s for s, g in decisions[0] if g == rank]
    waiting = [s for s, g in decisions[0] if g < 0]
    return mine, waiting
