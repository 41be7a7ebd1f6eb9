"""Multi-GPU placement of ensemble instances (independent pours).

A single pour does not shard (a domain split would exchange halos after P2G and after
every red-black half-sweep), so the multi-GPU path runs replicas: an ensemble's
instances are partitioned across ranks, each rank steps its share as one batched
ensemble on its own GPU, and the only collective is the final gather of per-instance
statistics.  Partitioning is particle-count balanced (greedy, largest first), because
a substep's cost grows with the instance's particle count.
"""
import heapq


def partition_instances(particle_counts, world):
    """Split instance indices over `world` ranks, balancing the particle totals.

    Greedy longest-processing-time packing: instances in decreasing particle count,
    each to the currently lightest rank (ties to the lower rank).  Returns one sorted
    index list per rank; every instance appears exactly once."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(particle_counts)), key=lambda i: (-particle_counts[i], i))
    heap = [(0, r) for r in range(world)]
    parts = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        parts[r].append(i)
        heapq.heappush(heap, (load + particle_counts[i], r))
    return [sorted(p) for p in parts]


def local_instances(particle_counts, rank, world):
    return partition_instances(particle_counts, world)[rank]


def gather_statistics(local_stats, group=None):
    """All ranks receive every instance's statistics: `local_stats` maps instance index
    to a list of floats; the result maps every index of every rank to its list.  Uses
    torch.distributed (NCCL on GPUs, gloo on CPUs); without an initialised process
    group it returns the local statistics."""
    import torch.distributed as dist

    if not dist.is_available() or not dist.is_initialized():
        return dict(local_stats)
    world = dist.get_world_size(group)
    gathered = [None] * world
    dist.all_gather_object(gathered, dict(local_stats), group=group)
    out = {}
    for part in gathered:
        for k, v in part.items():
            if k in out:
                raise RuntimeError(f"instance {k} reported by two ranks")
            out[k] = v
    return out
