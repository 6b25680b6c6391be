"""Many mock catalogues through the estimators, over one or several GPUs.

The covariance workload of the reference (hundreds to thousands of independent mocks,
src/hitomi_measurement/main.cpp:64-76 loops realizations over MPI ranks) shards by mock:
one process per GPU, each with its own context, no data exchanged on the GPU.  This
module holds the host side of that: a deterministic split of mocks of uneven particle
counts over ranks, the per-rank loop, and the gather of the small per-mock results.
"""
from __future__ import annotations

from typing import Callable, Dict, List, Sequence


def shard(sizes: Sequence[int], world: int) -> List[List[int]]:
    """Split mock indices over `world` ranks: largest mock first onto the rank with the
    least total particles so far (ties to the lower rank).  Deterministic, so every rank
    computes the same split without communicating.  Each rank's list is in index order."""
    if world < 1:
        raise ValueError("world must be >= 1")
    load = [0] * world
    out: List[List[int]] = [[] for _ in range(world)]
    for i in sorted(range(len(sizes)), key=lambda j: (-int(sizes[j]), j)):
        r = min(range(world), key=lambda q: (load[q], q))
        out[r].append(i)
        load[r] += int(sizes[i])
    return [sorted(v) for v in out]


def run_rank(sizes: Sequence[int], rank: int, world: int, measure: Callable[[int], dict]) -> Dict[int, dict]:
    """Run `measure(mock_index)` for this rank's share of the mocks."""
    return {i: measure(i) for i in shard(sizes, world)[rank]}


def gather(local: Dict[int, dict], world: int, group=None) -> Dict[int, dict]:
    """All ranks' results keyed by mock index (host objects through torch.distributed;
    the per-mock results are a few KB)."""
    if world == 1:
        return dict(local)
    import torch.distributed as dist
    parts: list = [None] * world
    dist.all_gather_object(parts, local, group=group)
    out: Dict[int, dict] = {}
    for p in parts:
        out.update(p)
    return out


def covariance_measure(ctx, catalogue: Callable[[int], "object"], pk_ells=(0, 2, 4), zeta_multipoles=()):
    """A `measure` for run_rank: P_l and 3PCF multipoles of one mock on an open context.
    `catalogue(i)` returns the (n, 3) positions of mock i."""
    def measure(i: int) -> dict:
        ctx.set_particles(0, catalogue(i))
        out = {}
        for ell in pk_ells:
            pk, nm, norm = ctx.pk_box(ell)
            out[f"pk{ell}"] = norm * pk
        if zeta_multipoles:
            z, sn, norm = ctx.zeta_box_multi(zeta_multipoles)
            for q, mp in enumerate(zeta_multipoles):
                out["zeta" + "".join(map(str, mp))] = norm * (z[q] - sn[q]).real
        return out
    return measure


def run_pipelined(indices: Sequence[int], contexts: Sequence[object],
                  measure_on: Callable[[object, int], dict]) -> Dict[int, dict]:
    """Measure mocks on one GPU with several contexts, one host thread each: context c takes
    mocks c, c + n, c + 2n, ... of `indices`.  Each context has its own CUDA stream and the
    C ABI calls release the GIL, so one context's upload of its next catalogue
    (hg_set_particles from pinned host memory) runs while another context computes; with
    two contexts the host-to-device copy leaves the critical path once the compute per mock
    is the longer of the two.  `measure_on(ctx, i)` does the whole mock (upload, statistics,
    read-back) and returns its results.  Results are keyed by mock index; the first
    exception of any thread is raised after all threads have stopped."""
    import threading

    out: Dict[int, dict] = {}
    errors: List[BaseException] = []
    lock = threading.Lock()
    n = len(contexts)
    if n < 1:
        raise ValueError("need at least one context")

    def worker(c: int) -> None:
        try:
            for k in range(c, len(indices), n):
                if errors:
                    return
                r = measure_on(contexts[c], indices[k])
                with lock:
                    out[indices[k]] = r
        except BaseException as e:  # noqa: BLE001 - re-raised in the caller's thread
            with lock:
                errors.append(e)

    threads = [threading.Thread(target=worker, args=(c,), daemon=True) for c in range(n)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    if errors:
        raise errors[0]
    return out
