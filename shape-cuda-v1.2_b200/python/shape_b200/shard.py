"""Frame sharding across GPUs (one rank per GPU).

Delay-Doppler frames are independent once the model is realized, so a
multi-GPU evaluation gives each rank a contiguous block of frames and the
only exchange is the sum of the per-rank chi-square totals (one all-reduce
of a few doubles per objective evaluation). Blocks are balanced by the
frames' work estimate: POS pixels plus delay-Doppler pixels.
"""
import numpy as np

from . import synth


def frame_cost(fr):
    return (2 * fr.pos_n + 1) ** 2 + fr.ndel * fr.ndop


def shard_bounds(costs, world):
    """Contiguous [start, end) blocks of `costs` for `world` ranks with
    near-equal total cost; every rank gets at least one item when possible."""
    n = len(costs)
    cum = np.concatenate([[0.0], np.cumsum(np.asarray(costs, dtype=np.float64))])
    total = cum[-1]
    bounds = [0]
    for r in range(1, world):
        target = total * r / world
        k = int(np.searchsorted(cum, target, side="left"))
        k = max(k, bounds[-1] + (1 if bounds[-1] < n else 0))
        k = min(k, n - (world - r) if n >= world else n)
        bounds.append(max(k, bounds[-1]))
    bounds.append(n)
    return [(bounds[r], bounds[r + 1]) for r in range(world)]


def shard_dataset(ds, rank, world):
    """The frames of `ds` that rank `rank` of `world` evaluates."""
    lo, hi = shard_bounds([frame_cost(f) for f in ds.frames], world)[rank]
    frames = ds.frames[lo:hi]
    obs = ds.obs[ds.offsets[lo]:ds.offsets[hi]].copy()
    oov = ds.oneovervar[ds.offsets[lo]:ds.offsets[hi]].copy()
    offsets = ds.offsets[lo:hi + 1] - ds.offsets[lo]
    return synth.DeldopDataset(ds.set, list(frames), obs, oov, offsets), (lo, hi)


def allreduce_summary(summary, dist, device=None):
    """Sum the additive fields of per-rank evaluation summaries (chi2 and the
    dof-weighted flag log-factors) over the process group."""
    import torch
    keys = ["chi2", "chi2_deldop", "chi2_lghtcrv"]
    t = torch.tensor([summary[k] for k in keys] + [float(summary["posbnd"]), float(summary["badradar"])],
                     dtype=torch.float64, device=device)
    dist.all_reduce(t)
    out = dict(summary)
    for i, k in enumerate(keys):
        out[k] = t[i].item()
    out["posbnd"] = int(t[3].item() > 0)
    out["badradar"] = int(t[4].item() > 0)
    return out
