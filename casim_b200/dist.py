"""Multi-GPU plumbing of the release-site batch: one process per GPU.

Sites are independent once every site owns its jSR pool and RNG stream, so a
batch shards by sites with no collective inside the time loop (weak scaling:
each rank steps its own sites). The only exchanges are after a run: the
maximum of the ranks' device times and the per-site outputs gathered on
rank 0. torch.distributed is the transport (NCCL between GPUs, gloo on CPU).
"""
import numpy as np


def site_cost(sites, cyto_nodes=0):
    """Node-steps of one time step per site: cleft nodes plus cytosol nodes."""
    nx, ny = np.asarray(sites["nx"], np.int64), np.asarray(sites["ny"], np.int64)
    nz = np.asarray(sites.get("nz", np.ones_like(nx)), np.int64)
    return nx * ny * nz + int(cyto_nodes)


def partition(costs, world):
    """Longest-processing-time split of sites over `world` ranks: sites by
    decreasing cost, each to the least-loaded rank (ties to the lower rank).
    Deterministic; returns one sorted index array per rank."""
    costs = np.asarray(costs, np.int64)
    order = np.argsort(-costs, kind="stable")
    load = np.zeros(world, np.int64)
    parts = [[] for _ in range(world)]
    for i in order:
        r = int(np.argmin(load))
        parts[r].append(int(i))
        load[r] += costs[i]
    return [np.array(sorted(p), dtype=np.int64) for p in parts]


def shard(sites, idx):
    """The site table restricted to the sites `idx` (channel rows follow their site)."""
    idx = np.asarray(idx, np.int64)
    S = len(sites["nx"])
    off = np.concatenate([[0], np.cumsum(sites["n_ch"])]).astype(np.int64)
    out = {}
    for k, v in sites.items():
        if isinstance(v, np.ndarray) and v.shape[:1] == (S,):
            out[k] = v[idx]
        else:
            out[k] = v
    for k in ("ch_x", "ch_y"):
        out[k] = np.concatenate([sites[k][off[i]:off[i + 1]] for i in idx]) if len(idx) else sites[k][:0]
    return out


def shard_of_rank(sites, cyto_nodes, world, rank):
    """This rank's sites of a global table: the cost-balanced partition's part
    `rank` (indices into the global table) and the table restricted to them."""
    parts = partition(site_cost(sites, cyto_nodes), world)
    idx = parts[rank]
    return idx, shard(sites, idx)


SITE_OUTPUT_COLUMNS = ("released_ca", "open_ryrs", "draws", "jsr_ca")


def site_outputs(sim, n_sites):
    """Per-site result rows of a batch (library handle or oracle, same getters):
    released Ca, open RyRs, draws consumed, jSR Ca; [n_sites, 4] float64."""
    out = np.zeros((n_sites, len(SITE_OUTPUT_COLUMNS)))
    for k in range(n_sites):
        out[k, 0] = sim.release(k)
        out[k, 1] = float(np.sum(sim.states(k)))
        out[k, 2] = float(sim.draws(k))
        out[k, 3] = float(sim.jsr(k)[0])
    return out


def max_over_ranks(value, device=None):
    """Maximum of a float over all ranks (the device-time reduction of a timed region)."""
    import torch
    import torch.distributed as dist
    if not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_sites(local, idx, n_total):
    """Assemble per-site rows from every rank on rank 0: `local` [n_local, ...]
    rows of the sites `idx`; returns the [n_total, ...] array on rank 0, None elsewhere."""
    import torch.distributed as dist
    local = np.asarray(local)
    if not dist.is_initialized() or dist.get_world_size() == 1:
        out = np.zeros((n_total,) + local.shape[1:], local.dtype)
        out[np.asarray(idx)] = local
        return out
    objs = [None] * dist.get_world_size() if dist.get_rank() == 0 else None
    dist.gather_object((np.asarray(idx), local), objs, dst=0)
    if dist.get_rank() != 0:
        return None
    out = np.zeros((n_total,) + local.shape[1:], local.dtype)
    for ix, rows in objs:
        out[ix] = rows
    return out
