"""Serve benchmark: roots arrive as a Poisson stream into one running
persistent kernel; p50/p99 latency and throughput per arrival rate.

Workload: half the roots are asynchronous BFS from the highest-degree vertex
of an R-MAT graph (scale 16..20, edge factor 16, a/b/c/d = .57/.19/.19/.05,
CSR int32), half are sums over random unbalanced binary trees of 2^18..2^20
nodes (48 % of each subtree's descendants go left); kinds, graphs and trees
are drawn with a seeded generator.  Arrivals are open-loop: the host publishes
every root whose arrival time has passed (gtap_serve_enqueue), polls the
completion ring between arrivals, and records

  latency          host clock, scheduled arrival -> completion seen by the host
                   (includes the wait for admission when the GPU is saturated)
  device service   the kernel's own stamps, admission -> last task finished

The capacity of the GPU for this workload is measured first, with every root
of a session enqueued at once; then sessions run at fixed fractions of that
capacity (where latency means something) and at the requested absolute rates
(above capacity they measure queueing).

All device buffers (graphs, trees, one BFS depth array per BFS root) exist
before the session starts: while the persistent kernel holds the SMs no other
kernel may be launched.

    python -m gtap_b200.serve_bench --loads 0.25,0.5,0.75,0.9 --rates 2000,50000
"""
import argparse
import json
import sys
import time

import numpy as np

INF = 0x3f3f3f3f


class ServeWorkload:
    def __init__(self, gt, scales=(16, 17, 18, 19, 20), tree_sizes=(1 << 18, 1 << 19, 1 << 20), seed=7):
        import torch
        self.gt = gt
        self.graphs = []
        for s in scales:
            row, col = gt.gen_rmat(s, 16, 1000 + s)
            self.graphs.append({"scale": s, "nv": len(row) - 1, "src": gt.max_degree_vertex(row),
                                "row": torch.from_numpy(row).cuda(), "col": torch.from_numpy(col).cuda()})
        self.trees = []
        for n in tree_sizes:
            left, right, value, size = gt.gen_tree(n, 2000 + n)
            self.trees.append({"n": n, "arrays": [torch.from_numpy(a).cuda() for a in (left, right, value, size)],
                               "sum": int(value.astype(np.int64).sum())})
        self.rng = np.random.default_rng(seed)
        self.ref_depth = {}   # graph index -> a validated depth array

    def draw(self, count):
        """(kind, index) per root: kind 0 = BFS on graph index, 1 = tree sum."""
        kinds = self.rng.integers(0, 2, count)
        return [(int(k), int(self.rng.integers(0, len(self.graphs) if k == 0 else len(self.trees)))) for k in kinds]

    def roots(self, plan):
        """Root descriptors and the depth arrays their BFS roots write."""
        import torch
        gt = self.gt
        roots, depths = [], []
        for kind, i in plan:
            if kind == 0:
                g = self.graphs[i]
                d = torch.full((g["nv"],), INF, dtype=torch.int32, device="cuda")
                depths.append(d)
                roots.append(gt.bfs_root(g["row"].data_ptr(), g["col"].data_ptr(), d.data_ptr(), g["nv"], g["src"], 32))
            else:
                t = self.trees[i]
                depths.append(None)
                roots.append(gt.treesum_root(*[a.data_ptr() for a in t["arrays"]], t["n"], 0, 32))
        torch.cuda.synchronize()
        return roots, depths


def bfs_depths_valid(row, col, src, depth):
    """Whether depth is the BFS distance labelling from src (Graph500-style
    validation): the source at 0, no edge out of a reached vertex skips a
    level, and every other reached vertex has a predecessor one level up."""
    d = depth.astype(np.int64)
    nv = len(row) - 1
    if d[src] != 0:
        return False
    reached = d < INF
    u = np.repeat(np.arange(nv), np.diff(row))
    v = col.astype(np.int64)
    from_reached = reached[u]
    if np.any(~reached[v[from_reached]]) or np.any(d[v[from_reached]] > d[u[from_reached]] + 1):
        return False
    best = np.full(nv, np.iinfo(np.int64).max)
    np.minimum.at(best, v[from_reached], d[u[from_reached]])
    others = reached.copy()
    others[src] = False
    return bool(np.all(best[others] == d[others] - 1))


def pct(x, q):
    return float(np.percentile(np.asarray(x), q)) if len(x) else None


def run_rate(gt, wl, rate, count, seed=11, limit_s=120.0):
    """One serve session of `count` roots at `rate` roots/s (None: all at once)."""
    plan = wl.draw(count)
    roots, depths = wl.roots(plan)
    if rate is None:
        arrivals = np.zeros(count)
    else:
        rng = np.random.default_rng(seed + int(rate))
        arrivals = np.cumsum(rng.exponential(1.0 / rate, count))
    gt.serve_start(ring_capacity=max(64, count))
    slot_of = {}
    done_t = {}
    t0 = time.perf_counter()
    nxt = 0
    try:
        while len(done_t) < count:
            now = time.perf_counter() - t0
            if nxt < count and arrivals[nxt] <= now:
                end = int(np.searchsorted(arrivals, now, side="right"))
                first = gt.serve_enqueue(roots[nxt:end])
                for j in range(nxt, end):
                    slot_of[(first + j - nxt) % max(64, count)] = j
                nxt = end
            for s in gt.serve_poll(4096):
                done_t[slot_of[s]] = time.perf_counter() - t0
            if now > limit_s:
                raise RuntimeError("serve run at %s roots/s did not finish in %.0f s" % (rate, limit_s))
        wall = time.perf_counter() - t0
    finally:
        st = gt.serve_shutdown()
    slots = sorted(slot_of)
    res = gt.serve_results(slots)
    by_root = {slot_of[s]: r for s, r in zip(slots, res)}
    lat = [(done_t[j] - arrivals[j]) * 1e3 for j in range(count)]
    svc = [(by_root[j].t_done_ns - by_root[j].t_admit_ns) / 1e6 for j in range(count)]
    tasks = sum(r.tasks for r in res)
    ok = all(r.status == gt.ROOT_DONE for r in res)
    for j, (kind, i) in enumerate(plan):
        if kind == 1:
            ok &= by_root[j].value == wl.trees[i]["sum"]
    return {"rate_roots_per_s": rate, "roots": count, "wall_s": wall, "ok": bool(ok) and st.status == 0,
            "tasks": tasks,
            "throughput_roots_per_s": count / wall, "tasks_per_s": tasks / wall,
            "latency_ms": {"p50": pct(lat, 50), "p99": pct(lat, 99), "max": max(lat)},
            "device_service_ms": {"p50": pct(svc, 50), "p99": pct(svc, 99)}, "depth_arrays": depths}


def _check_depths(wl, r):
    """Every BFS root's depths: BFS distances are unique, so the first array
    seen for a graph is validated as a distance labelling and the others
    must equal it."""
    import torch
    for d in r.pop("depth_arrays"):
        if d is None:
            continue
        gi = next(i for i, g in enumerate(wl.graphs) if g["nv"] == d.numel())
        ref = wl.ref_depth.get(gi)
        if ref is None:
            g = wl.graphs[gi]
            if bfs_depths_valid(g["row"].cpu().numpy(), g["col"].cpu().numpy(), g["src"], d.cpu().numpy()):
                wl.ref_depth[gi] = d.clone()
            else:
                r["ok"] = False
        elif not torch.equal(d, ref):
            r["ok"] = False
    return r


def run(loads=(0.25, 0.5, 0.75, 0.9), rates=(), count=300, config=None, workload=None):
    """Capacity session, then one session per load fraction and per absolute
    rate.  Returns {"capacity": {...}, "sessions": [...]}."""
    import torch
    import gtap_b200 as gt
    torch.cuda.init()
    wl = workload or ServeWorkload(gt)
    gt.gtap_initialize(gt.default_config(**(config or {})))
    out = {"sessions": []}
    try:
        cap = _check_depths(wl, run_rate(gt, wl, None, count))
        cap["load"] = None
        out["capacity"] = cap
        capacity = cap["throughput_roots_per_s"]
        for f in loads:
            r = _check_depths(wl, run_rate(gt, wl, f * capacity, count))
            r["load"] = f
            out["sessions"].append(r)
        for rate in rates:
            r = _check_depths(wl, run_rate(gt, wl, rate, count))
            r["load"] = rate / capacity
            out["sessions"].append(r)
    finally:
        gt.gtap_finalize()
    return out


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--loads", default="0.25,0.5,0.75,0.9", help="fractions of the measured capacity")
    ap.add_argument("--rates", default="2000,50000", help="absolute arrival rates, roots/s")
    ap.add_argument("--roots", type=int, default=300, help="roots per session")
    a = ap.parse_args(argv)
    loads = [float(x) for x in a.loads.split(",") if x]
    rates = [int(x) for x in a.rates.split(",") if x]
    out = run(loads, rates, a.roots)
    print(json.dumps(out["capacity"]), flush=True)
    for r in out["sessions"]:
        print(json.dumps(r), flush=True)
    return 0 if out["capacity"]["ok"] and all(r["ok"] for r in out["sessions"]) else 1


if __name__ == "__main__":
    sys.exit(main())
