"""Instance sharding of the batched and served workloads across GPUs.

The reference solves one instance at a time (``PlasticitySolver::solve``,
src/PlasticitySolver.cu:469-512) and instances share nothing, so N processes,
one per GPU, split a request list with no data-path collective: each rank
solves its share through the solve service on its own GPU, and only the
per-request records (status, latency, iteration counts, a checksum of the
result) meet on the host, through one object all-gather over the process
group (gloo or NCCL).

The split is longest-processing-time first on an a-priori cost (degrees of
freedom times load increments): requests in decreasing cost go to the rank
with the least cost so far, ties to the lower rank. It is deterministic, so
every rank computes the same split from the same list without exchanging it.
"""
import time


def request_cost(dof, levels=1):
    """A-priori cost of one request: DOF x load increments (the CG work of a
    linear solve grows with the DOF, and every increment repeats the secant
    iteration)."""
    return float(dof) * max(1, int(levels))


def partition(costs, world):
    """Splits request indices 0..len(costs)-1 over ``world`` ranks (LPT).

    Returns one list per rank, each in increasing index (submission) order;
    together they hold every index exactly once."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    load = [0.0] * world
    parts = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        parts[r].append(i)
        load[r] += float(costs[i])
    return [sorted(p) for p in parts]


def run_share(indices, build, submit, wait, clock=time.perf_counter):
    """Solves this rank's requests through one solve service.

    build(i) -> request (whatever ``submit`` takes); submit(request) -> id;
    wait(id) -> record dict (status, outer, cg, checksum, latency, ...).
    All requests are submitted at once (a burst), then waited for in
    submission order. Returns {index: record}, each record with ``done_at``:
    seconds from the first submission to the moment its result was taken."""
    reqs = [(i, build(i)) for i in indices]
    t0 = clock()
    ids = [(i, submit(r)) for i, r in reqs]
    out = {}
    for i, rid in ids:
        rec = dict(wait(rid))
        rec["done_at"] = clock() - t0
        out[i] = rec
    return out


def gather_objects(obj, dist=None):
    """[obj of rank 0, obj of rank 1, ...] on every rank (an object
    all-gather; [obj] when ``dist`` is None)."""
    if dist is None:
        return [obj]
    parts = [None] * dist.get_world_size()
    dist.all_gather_object(parts, obj)
    return parts


def merge_records(parts):
    """One {index: record} from the ranks' record dicts; an index on two
    ranks is an error."""
    merged = {}
    for p in parts:
        for k, v in p.items():
            if k in merged:
                raise RuntimeError(f"request {k} was solved on two ranks")
            merged[k] = v
    return merged


def gather_records(records, dist=None):
    """Merges every rank's {index: record} into one dict, on every rank."""
    return merge_records(gather_objects(dict(records), dist))


def summarize(merged, n_requests, world):
    """Whole-job figures of a sharded run: completed requests over the
    slowest rank's span (the last ``done_at``), statuses, latency p50/p99."""
    done = sorted(merged)
    if len(done) != n_requests:
        raise RuntimeError(f"{len(done)} of {n_requests} requests have a record")
    span = max(r["done_at"] for r in merged.values()) if merged else 0.0
    lat = sorted(r["latency"] for r in merged.values())

    def pct(q):
        if not lat:
            return 0.0
        k = min(len(lat) - 1, max(0, int(round(q / 100.0 * (len(lat) - 1)))))
        return float(lat[k])

    return {"ranks": world, "requests": n_requests, "seconds": span,
            "solves_per_s": n_requests / span if span > 0 else 0.0,
            "statuses": sorted({r["status"] for r in merged.values()}),
            "p50_s": pct(50), "p99_s": pct(99)}
