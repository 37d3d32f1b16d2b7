"""Placement of independent problems on the GPUs of one node.

The batched ensemble and the serving loop advance independent problems, so
they shard across GPUs with no exchange on the data path: one process per
GPU serves the problems placed on it, and only the host-side placement and
the final statistics are shared.  The reference has no counterpart (it runs
one problem per MPI job); the units are the problems of a parameter study or
the requests of a service.

Every rank computes the same placement from the same inputs (the problem
list or the request trace and the footprint estimates), so placement needs
no communication.
"""
import heapq


def partition_by_cost(costs, world):
    """Longest-processing-time placement: problems in decreasing cost, each
    onto the rank with the least cost so far (ties to the lower rank).
    Returns the rank of every problem."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda k: (-costs[k], k))
    heap = [(0.0, r) for r in range(world)]
    rank_of = [0] * len(costs)
    for k in order:
        load, r = heapq.heappop(heap)
        rank_of[k] = r
        heapq.heappush(heap, (load + float(costs[k]), r))
    return rank_of


def route_requests(arrivals, costs, world):
    """Online routing of a request stream: in arrival order, each request
    goes to the rank whose routed work still outstanding at its arrival is
    least.  A rank's outstanding work drains at one unit per second, an
    estimate only used for routing; ties go to the lower rank.  Returns the
    rank of every request."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(arrivals)), key=lambda k: (arrivals[k], k))
    backlog = [0.0] * world
    last = 0.0
    rank_of = [0] * len(arrivals)
    for k in order:
        t = float(arrivals[k])
        drained = max(0.0, t - last)
        backlog = [max(0.0, b - drained) for b in backlog]
        last = max(last, t)
        r = min(range(world), key=lambda q: (backlog[q], q))
        rank_of[k] = r
        backlog[r] += float(costs[k])
    return rank_of


def local_items(rank_of, rank):
    """Indices of the items placed on `rank`, in their original order."""
    return [k for k, r in enumerate(rank_of) if r == rank]
