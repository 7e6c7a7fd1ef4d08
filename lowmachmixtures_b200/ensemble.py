"""Ensembles of independent Stokes problems (uneven grid sizes, different
seeds and viscosity fields): the units of work that shard across GPUs.

Instances are independent, so a multi-GPU run gives every rank a disjoint
set of whole instances -- no collective on the data path, only a final
gather of per-instance statistics.  `shard` balances the ranks by the
expected cost of an instance (`instance_cost`: its cell count times the
FGMRES iterations its viscosity contrast is expected to take).
"""
from __future__ import annotations

import numpy as np

SIZES_2D = (64, 96, 128, 192, 256)


def instance_sizes(count: int, seed: int = 0, sizes=SIZES_2D):
    """grid size of each instance, drawn per seed from `sizes`"""
    rng = np.random.Generator(np.random.PCG64(424242 + seed))
    return [int(v) for v in rng.choice(np.asarray(sizes), size=count)]


def instance_contrast(i: int, seed: int = 0) -> float:
    """viscosity contrast of instance i: log-uniform in [10, 1000]"""
    u = np.random.Generator(np.random.PCG64(777 + 1000003 * seed + i)).uniform()
    return float(10.0 ** (1.0 + 2.0 * u))


def expected_iterations(contrast: float) -> float:
    """FGMRES + V-cycle iterations to 1e-8 expected at a viscosity contrast:
    12.7 + 10.6 log10(contrast / 10), fitted to oracle solves of 2D 64^2 and
    128^2 problems of this family (precon_type 2, visc_type -2; three seeds
    each at contrasts 10, 30, 100, 300 and 1000: 12.7, 16.5, 21, 26 and 34
    iterations on average, the same at both sizes)."""
    return 12.7 + 10.6 * float(np.log10(max(contrast, 1.0) / 10.0))


def instance_cost(n: int, contrast: float, dm: int = 2) -> float:
    """expected work of one instance: cells times expected iterations"""
    return float(n) ** dm * max(1.0, expected_iterations(contrast))


def shard(costs, world: int):
    """Partition instance indices over `world` ranks, largest first onto the
    least-loaded rank (longest-processing-time rule).  Returns one sorted
    index list per rank; every index appears exactly once."""
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    load = [0.0] * world
    parts = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda q: (load[q], q))
        parts[r].append(i)
        load[r] += costs[i]
    return [sorted(p) for p in parts]


def make_instances(count: int, seed: int = 0, dm: int = 2, sizes=SIZES_2D, theta_alpha: float = 0.0):
    """The 512-problem 2D ensemble (by default): instance i has grid size instance_sizes()[i],
    its own seeded log-viscosity field with contrast instance_contrast(i)
    and an N(0,1) mean-removed face rhs."""
    from . import synth
    ns = instance_sizes(count, seed, sizes)
    return [synth.make_problem(dm, n, instance_contrast(i, seed), 100000 * (seed + 1) + i, theta_alpha=theta_alpha)
            for i, n in enumerate(ns)]


def _items(problems, device):
    """device copies of the problems' arrays and the lmm_ensemble_item array"""
    import torch

    from . import abi
    dev = lambda x: torch.from_numpy(np.ascontiguousarray(x)).cuda(device)  # noqa: E731
    keep, sols = [], []
    items = (abi.EnsembleItem * len(problems))()
    for it, p in zip(items, problems):
        dm = p.dm
        arrs = dict(b_u=[dev(a) for a in p.b_u], b_p=dev(p.b_p), al=[dev(a) for a in p.alpha_fc], be=dev(p.beta),
                    bed=[dev(a) for a in p.beta_ed], ga=dev(p.gamma))
        xu = [torch.zeros_like(arrs["b_p"]) for _ in range(dm)]
        xp = torch.zeros_like(arrs["b_p"])
        keep.append(arrs)
        sols.append((xu, xp))
        for d in range(3):
            it.n[d] = p.n[d]
        it.dx = p.dx
        it.theta_alpha = p.theta_alpha
        for d in range(dm):
            it.b_u[d] = abi.ptr(arrs["b_u"][d])
            it.alpha_fc[d] = abi.ptr(arrs["al"][d])
            it.x_u[d] = abi.ptr(xu[d])
        for d, b in enumerate(arrs["bed"]):
            it.beta_ed[d] = abi.ptr(b)
        it.b_p, it.beta, it.gamma, it.x_p = abi.ptr(arrs["b_p"]), abi.ptr(arrs["be"]), abi.ptr(arrs["ga"]), abi.ptr(xp)
    return items, keep, sols


class Ensemble:
    """A worker pool with a solver handle per (worker, grid shape), kept
    between runs (lmm_ensemble_create / _run / _destroy)."""

    def __init__(self, problems, knobs, workers: int = 4, device: int = 0):
        import ctypes as C

        from . import _native
        self.lib = _native.load()
        self.device = device
        self.knobs = knobs
        self.h = C.c_void_p()
        items, _, _ = _items(problems, device)
        rc = self.lib.lmm_ensemble_create(problems[0].dm, C.byref(knobs), device, items, len(problems), workers,
                                          C.byref(self.h))
        if rc != 0:
            raise RuntimeError(f"lmm_ensemble_create: {self.lib.lmm_strerror(rc).decode()}")

    def run(self, problems):
        """solve every problem; returns (statuses, stats, solutions, seconds)"""
        import time

        import torch
        items, keep, sols = _items(problems, self.device)
        torch.cuda.synchronize(self.device)
        t0 = time.perf_counter()
        self.lib.lmm_ensemble_run(self.h, items, len(problems))
        secs = time.perf_counter() - t0
        return [it.status for it in items], [it.stats.as_dict() for it in items], sols, secs

    def close(self):
        if self.h:
            self.lib.lmm_ensemble_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def solve(problems, knobs, workers: int = 4, device: int = 0):
    """One-shot: create the pool, solve the list, release.  Returns
    (statuses, stats dicts, solutions as (x_u, x_p) torch tensors, seconds
    of the solves)."""
    with Ensemble(problems, knobs, workers, device) as e:
        return e.run(problems)


def main():
    import argparse
    import json
    import os

    from . import abi
    ap = argparse.ArgumentParser(description="ensemble of independent 2D periodic Stokes problems of uneven sizes")
    ap.add_argument("--count", type=int, default=512)
    ap.add_argument("--workers", type=int, default=4)
    ap.add_argument("--rel-tol", type=float, default=1e-8)
    ap.add_argument("--repeats", type=int, default=3)
    ap.add_argument("--host-wait", type=int, default=0, help="0: worker threads spin on their streams (1: block)")
    ap.add_argument("--mode", choices=("batch", "pool"), default="batch",
                    help="batch: one batch handle per grid size; pool: worker threads with one-problem handles")
    ap.add_argument("--orthogonalization", type=int, default=None,
                    help="0 modified, 1 classical Gram-Schmidt (default: 1 in batches, 0 in the pool, the faster of each)")
    ap.add_argument("--knob", action="append", default=[], metavar="NAME=VALUE", help="any other lmm_knobs field")
    ap.add_argument("--sizes", default=",".join(str(n) for n in SIZES_2D),
                    help="comma-separated grid sizes the instances are drawn from")
    a = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        # whole instances per rank (no collective on the data path); only the
        # per-rank results are gathered at the end
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600), device_id=torch.device("cuda", local))
    pool_sizes = tuple(int(v) for v in a.sizes.split(","))
    sizes = instance_sizes(a.count, sizes=pool_sizes)
    mine = shard([instance_cost(n, instance_contrast(i)) for i, n in enumerate(sizes)], world)[rank]
    allp = make_instances(a.count, sizes=pool_sizes)
    probs = [allp[i] for i in mine]
    pool = a.mode == "pool"
    kn = abi.make_knobs(precon_type=2, visc_type=-2, method=abi.LMM_METHOD_FGMRES, precision=abi.LMM_PRECISION_FP32,
                        orthogonalization=(0 if pool else 1) if a.orthogonalization is None else a.orthogonalization,
                        gmres_rel_tol=a.rel_tol, host_wait=a.host_wait,
                        ensemble_batch=-1 if pool else 0)
    for kv in a.knob:
        name, val = kv.split("=", 1)
        setattr(kn, name, type(getattr(kn, name))(float(val)))
    from . import _native
    lib = _native.load()
    import time
    t0 = time.perf_counter()
    ens = Ensemble(probs, kn, a.workers, local)
    create_s = time.perf_counter() - t0
    best = None
    each = []  # seconds of every repeat
    for _ in range(a.repeats):
        if dist is not None:
            dist.barrier()
        st, stats, _, secs = ens.run(probs)
        bad = sorted({p.n[0] for c, p in zip(st, probs) if c < 0})
        if bad:
            raise RuntimeError(f"instances of sizes {bad} failed: " + lib.lmm_strerror(min(st)).decode())
        best = secs if best is None else min(best, secs)
        each.append(secs)
    ens.close()
    ok = [s for s, c in zip(stats, st) if c >= 0]
    errors = {}
    for c, p in zip(st, probs):
        if c < 0:
            errors.setdefault(lib.lmm_strerror(c).decode(), []).append(p.n[0])
    out = dict(rank=rank, mode=a.mode, workers=a.workers if pool else None, instances=len(probs), seconds=best,
               seconds_each=each,
               instances_per_s=len(probs) / best,
               pool_creation_seconds=create_s,
               failed=int(sum(1 for c in st if c < 0)), unconverged=int(sum(1 for c in st if c > 0)), errors=errors,
               iterations_mean=float(np.mean([s["total_iter"] for s in ok])) if ok else None,
               max_true_rel_residual=float(max(s["norm_resid_true"] / s["norm_b"] for s in ok)) if ok else None,
               sizes={int(n): int(sum(1 for p in probs if p.n[0] == n)) for n in sorted(set(p.n[0] for p in probs))})
    if dist is None:
        print(json.dumps(out), flush=True)
        return
    outs = [None] * world
    dist.all_gather_object(outs, out)
    if rank == 0:
        slowest = max(o["seconds"] for o in outs)
        print(json.dumps(dict(ranks=world, instances=sum(o["instances"] for o in outs), seconds=slowest,
                              instances_per_s=sum(o["instances"] for o in outs) / slowest,
                              failed=sum(o["failed"] for o in outs), per_rank=outs)), flush=True)
    dist.destroy_process_group()


if __name__ == "__main__":
    main()
