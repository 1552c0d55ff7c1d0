"""Several GPUs, one process each (torch.distributed; NCCL on GPUs, gloo for
the CPU tests).

* The plain step path runs one simulation per GPU (replicas; bench.py
  --gpus N): no data-path collective.
* The batched form splits its independent networks over the ranks
  (``shard_instances``): each rank advances its own batch, no collective.
* The differentiable form is data-parallel over trials: each rank runs its
  share of the trials (``shard_trials``) through the adjoint kernel and one
  all-reduce sums the weight gradients (``dp_grad``), scaled so that the
  result is the gradient of the loss averaged over all trials.
"""

import numpy as np


def shard_trials(total, rank, world):
    """The contiguous range of trials rank `rank` runs: sizes differ by at
    most one, lower ranks take the extra ones."""
    q, r = divmod(int(total), int(world))
    start = rank * q + min(rank, r)
    return start, start + q + (1 if rank < r else 0)


def shard_instances(sizes, world):
    """Assign networks (by their synapse counts or sizes) to ranks: largest
    first to the least loaded rank (ties: the lowest rank). Returns one list
    of instance indices per rank, each in increasing order."""
    sizes = np.asarray(sizes, np.int64)
    load = np.zeros(int(world), np.int64)
    owner = np.empty(sizes.size, np.int64)
    for j in np.argsort(-sizes, kind="stable"):
        r = int(np.argmin(load))
        owner[j] = r
        load[r] += sizes[j]
    return [sorted(np.nonzero(owner == r)[0].tolist()) for r in range(int(world))]


def dp_grad(local_grad, local_trials, total_trials, group=None):
    """Sum of the ranks' gradients, each computed for the mean loss over the
    rank's own trials, weighted by its share of the trials: the gradient of
    the mean loss over all trials. One all-reduce (in place; returned)."""
    import torch.distributed as dist
    local_grad.mul_(float(local_trials) / float(total_trials))
    if dist.is_available() and dist.is_initialized():
        dist.all_reduce(local_grad, op=dist.ReduceOp.SUM, group=group)
    return local_grad
