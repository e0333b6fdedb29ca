"""Planet-to-GPU sharding for multi-GPU runs (one process per GPU).

Planets are independent, so the only multi-GPU work is host-side planning:
every rank computes the same assignment of planets to ranks (longest
processing time first by an estimated per-step cost), advances its own
planets with no collective on the data path, and the job time is the maximum
over ranks.
"""


def planet_cost(N, particles, R, cg_iters=8):
    """Estimated bytes moved per step: fluid (one read of every input and one write of every
    output per pass of the upstream step, K_it CG iterations), particles and faces."""
    n = 6 * N * N
    return n * (344 + 253 + cg_iters * (76 + 253)) + 76 * particles + 32 * 6 * R * R


def assign(costs, world):
    """Greedy LPT: planets sorted by cost (descending, ties by index) go to the
    least-loaded rank (ties to the lower rank).  Returns a list per rank of
    planet indices (ascending) and the per-rank loads."""
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    loads = [0.0] * world
    owned = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (loads[k], k))
        owned[r].append(i)
        loads[r] += costs[i]
    return [sorted(o) for o in owned], loads


def max_over_ranks(value, dist=None, device=None):
    """Maximum of a float over all ranks (identity without a process group)."""
    if dist is None or not dist.is_initialized():
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device or "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
