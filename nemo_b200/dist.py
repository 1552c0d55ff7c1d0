"""Several GPUs, one process each (torch.distributed; NCCL on GPUs, gloo for
the CPU tests).

* The plain step path either runs one simulation per GPU (replicas; bench.py
  --gpus N, no data-path collective) or one network over all GPUs as shards
  (``ShardedSimulation``; bench.py --sharded): each shard owns a contiguous
  range of neuron warps and the synapses to them, and the shards' fired
  words are all-gathered once per cycle: through host memory
  (``exchange_fired_words``; gloo and NCCL), or as CUDA tensors that never
  leave the GPUs (``exchange_fired_words_device``; NCCL, queued without
  waiting on the host).
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


def shard_warps(total, rank, world):
    """The warps [first, first + count) shard `rank` of `world` owns out of
    `total` (the library's nemo_b200_shard_warps): sizes differ by at most
    one, lower ranks take the extra ones."""
    q, r = divmod(int(total), int(world))
    first = rank * q + min(rank, r)
    return first, q + (1 if rank < r else 0)


def exchange_fired_words(local_words, first_word, total_words, group=None):
    """One cycle's fired words of all shards: every rank contributes the
    words of its own warps (shard_warps of the group's size); one all-gather
    of equal-length tensors (padded to the largest share). On NCCL the
    tensors travel through the current CUDA device. Returns total_words
    uint32 words."""
    import torch
    import torch.distributed as dist
    local = np.ascontiguousarray(local_words, dtype=np.uint32)
    if not (dist.is_available() and dist.is_initialized()):
        if first_word != 0 or local.size != total_words:
            raise ValueError("without a process group the shard must own every warp")
        return local
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    if (first_word, local.size) != shard_warps(total_words, rank, world):
        raise ValueError("rank %d does not own warps [%d, %d)" % (rank, first_word, first_word + local.size))
    width = -(-int(total_words) // world)
    dev = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend(group) == "nccl" \
        else torch.device("cpu")
    send = torch.zeros(width, dtype=torch.int32, device=dev)
    send[:local.size] = torch.from_numpy(local.view(np.int32)).to(dev)
    parts = [torch.empty(width, dtype=torch.int32, device=dev) for _ in range(world)]
    dist.all_gather(parts, send, group=group)
    full = np.empty(int(total_words), dtype=np.uint32)
    for r, part in enumerate(parts):
        f, c = shard_warps(total_words, r, world)
        full[f:f + c] = part[:c].cpu().numpy().view(np.uint32)
    return full


def exchange_fired_words_device(local_words, first_word, total_words, group=None):
    """exchange_fired_words for CUDA tensors: `local_words` (int32, this
    rank's words) -> a new int32 CUDA tensor of all total_words words, by one
    all_gather_into_tensor of padded shares and one index gather, both queued
    on the current stream. Without a process group the shard must own every
    warp and the tensor is returned as it is."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        if first_word != 0 or local_words.numel() != total_words:
            raise ValueError("without a process group the shard must own every warp")
        return local_words
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    if (first_word, local_words.numel()) != shard_warps(total_words, rank, world):
        raise ValueError("rank %d does not own warps [%d, %d)" % (rank, first_word, first_word + local_words.numel()))
    width = -(-int(total_words) // world)
    dev = local_words.device
    send = torch.zeros(width, dtype=torch.int32, device=dev)
    send[:local_words.numel()] = local_words
    gathered = torch.empty(world * width, dtype=torch.int32, device=dev)
    dist.all_gather_into_tensor(gathered, send, group=group)
    key = (int(total_words), world, dev)
    index = _gather_index.get(key)
    if index is None:
        parts = [r * width + np.arange(shard_warps(total_words, r, world)[1]) for r in range(world)]
        index = torch.as_tensor(np.concatenate(parts), dtype=torch.int64, device=dev)
        _gather_index[key] = index
    return gathered.index_select(0, index)


_gather_index = {}
