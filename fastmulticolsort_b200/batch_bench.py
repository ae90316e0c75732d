"""Many-instances and wide-table workloads (seeded, generated on the device).

Instances: 4,096 independent sort instances with n_i = floor(2^U(10, 20)) rows
(mean about 151k, about 619M rows in all), three columns of 8 / 24 / 40 bits
(u16 / u32 / u64 storage); col0 draws from 16 distinct values in [0, 2^8),
col1 and col2 are uniform.  Compared:
  batched      ONE fmcs_run_batch call for all instances (the cost model's plan);
  per_instance the same plan, one fmcs_run_plan call per instance;
  plain        one full LSD sort per original column per instance
               (fmcs_sort_round_plain, no massaging, no size binning).

Wide: N = 60,000,000 rows, six columns of 2 / 1 / 12 / 12 / 32 / 7 bits with
3 / 2 / 2,526 / 2,526 / uniform 32-bit / 100 distinct values (66 bits: at least
two banks).  ORDER BY runs the cost model's ordered plan; GROUP BY runs its
column order and plan through the hash-grouping rounds; plain sorts column by
column.  The reference's TPC-H-derived inputs are not available here; these
seeded shapes stand in for them.
"""
from __future__ import annotations

import math
import time

import numpy as np

from . import capi
from . import workloads as W

INSTANCE_COUNT = 4096
WIDE_ROWS = 60_000_000
WIDE_BITS = [2, 1, 12, 12, 32, 7]
WIDE_CARD = [3, 2, 2526, 2526, 1 << 32, 100]


def _store_dtype(torch, w):
    return torch.int16 if w <= 16 else (torch.int32 if w <= 32 else torch.int64)


def _gen(torch, rng):
    g = torch.Generator(device="cuda")
    g.manual_seed(int(rng.integers(1 << 62)))
    return g


def _pool_column(torch, rng, n, w, count):
    """n codes drawn uniformly from `count` distinct w-bit values, stored in the
    reference's width (u16 / u32 / u64 as int16 / int32 / int64 bits)."""
    pool = W.distinct_pool(rng, count, w).astype(np.int64)
    idx = torch.randint(0, count, (n,), device="cuda", generator=_gen(torch, rng))
    v = torch.from_numpy(pool).cuda()[idx]
    return _narrow(torch, v, w)


def _uniform_column(torch, rng, n, w):
    g = _gen(torch, rng)
    if w >= 63:
        v = torch.randint(-(1 << 63), (1 << 63) - 1, (n,), dtype=torch.int64, device="cuda", generator=g)
    else:
        v = torch.randint(0, 1 << w, (n,), dtype=torch.int64, device="cuda", generator=g)
    return _narrow(torch, v, w)


def _narrow(torch, v, w):
    if w > 32:
        return v.contiguous()
    bits = 16 if w <= 16 else 32
    v = torch.where(v >= (1 << (bits - 1)), v - (1 << bits), v)
    return v.to(_store_dtype(torch, w)).contiguous()


def _time_ms(torch, stream, fn, reps):
    """Mean ms of fn() over reps, CUDA events on the context's stream."""
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    a.record(stream)
    for _ in range(reps):
        fn()
    b.record(stream)
    torch.cuda.synchronize()
    return a.elapsed_time(b) / reps


def instance_workload(torch, count=INSTANCE_COUNT):
    """The many-instances shape on the device: (cols, sizes, bw, split, est_ms).
    est_ms is the cost model's estimate for ONE instance of the mean size
    (the plan is chosen for that instance)."""
    rng = W.rng_for(4)
    sizes = np.floor(2.0 ** rng.uniform(10, 20, size=count)).astype(np.int64)
    total = int(sizes.sum())
    bw = [8, 24, 40]
    cols = [_pool_column(torch, rng, total, 8, 16), _uniform_column(torch, rng, total, 24),
            _uniform_column(torch, rng, total, 40)]
    col_bytes = [c.element_size() for c in cols]
    mean_n = int(sizes.mean())
    split, _, est = capi.optimize_plan(bw, [16, min(mean_n, 1 << 24), mean_n], col_bytes, mean_n)
    return cols, sizes, bw, split, est


def wide_workload(torch, n=WIDE_ROWS):
    """The wide table on the device (n rows, 60,000,000 by default): (cols,
    card, ORDER BY split, GROUP BY (split, column order)).  The plans are the
    cost model's for the 60,000,000-row table."""
    rng = W.rng_for(4, salt=1)
    cols = []
    for w, k in zip(WIDE_BITS, WIDE_CARD):
        cols.append(_uniform_column(torch, rng, n, w) if k >= (1 << w) else _pool_column(torch, rng, n, w, k))
    col_bytes = [c.element_size() for c in cols]
    card = [min(k, WIDE_ROWS) for k in WIDE_CARD]
    split, _, _ = capi.optimize_plan(WIDE_BITS, card, col_bytes, WIDE_ROWS, ordered=True)
    gsplit, gorder, _ = capi.optimize_plan(WIDE_BITS, card, col_bytes, WIDE_ROWS, ordered=False)
    return cols, card, split, (gsplit, gorder)


def sample_instances(sizes, count=20, seed=7):
    """Indices of `count` instances spread over the size range (smallest,
    largest and a seeded sample between), for the oracle check."""
    rng = np.random.default_rng(seed)
    k = len(sizes)
    pick = {int(np.argmin(sizes)), int(np.argmax(sizes))}
    pick.update(int(i) for i in rng.choice(k, size=min(k, count) - len(pick), replace=False))
    return sorted(pick)[:count]


def check_instances_vs_oracle(cols, sizes, bw, split, order, group, counts, picks):
    """Each picked instance's instance-local order and group ids, and its group
    count, against the oracle on that instance's rows (host copies)."""
    from oracle import oracle as O
    offs = np.concatenate([[0], np.cumsum(sizes)])
    for i in picks:
        a, b = int(offs[i]), int(offs[i + 1])
        sub = [c[a:b].cpu().numpy() for c in cols]
        sub = [x.view(np.uint16 if x.dtype == np.int16 else (np.uint32 if x.dtype == np.int32 else np.uint64))
               for x in sub]
        o, g, ng = O.run_plan_sort(sub, bw, split)
        if not (np.array_equal(order[a:b].cpu().numpy().view(np.uint32), o)
                and np.array_equal(group[a:b].cpu().numpy().view(np.uint32), g) and int(counts[i]) == ng):
            return False, i
    return True, None


def instances(torch, ctx, stream, reps=3, plain=True):
    cols, sizes, bw, split, est = instance_workload(torch)
    total = int(sizes.sum())
    col_bytes = [c.element_size() for c in cols]
    order = torch.empty(total, dtype=torch.int32, device="cuda")
    group = torch.empty(total, dtype=torch.int32, device="cuda")
    offs = np.concatenate([[0], np.cumsum(sizes)])

    def batched():
        ctx.run_batch(cols, bw, split, sizes, order, group)

    def per_instance():
        for i in range(INSTANCE_COUNT):
            a, b = int(offs[i]), int(offs[i + 1])
            ctx.run_plan([c[a:b] for c in cols], bw, split, order[a:b], group[a:b])

    g2 = torch.empty_like(group)

    def plain_path():
        for i in range(INSTANCE_COUNT):
            a, b = int(offs[i]), int(offs[i + 1])
            o, g, h = order[a:b], group[a:b], g2[a:b]
            ctx.sort_round_plain(cols[0][a:b], 8, o, out_group=g)
            ctx.sort_round_plain(cols[1][a:b], 24, o, in_group=g, out_group=h)
            ctx.sort_round_plain(cols[2][a:b], 40, o, in_group=h, out_group=g)

    out = {"instances": INSTANCE_COUNT, "rows": total, "rows_min": int(sizes.min()), "rows_max": int(sizes.max()),
           "rows_mean": round(float(sizes.mean()), 1), "columns": "8-bit (16 distinct values, u16), 24-bit (u32), "
           "40-bit (u64)", "plan": split, "plan_est_ms_mean_instance": round(est, 3),
           "column_bytes": int(total * sum(col_bytes))}
    counts = ctx.run_batch(cols, bw, split, sizes, order, group)
    out["batched_ms"] = round(_time_ms(torch, stream, batched, reps), 3)
    torch.cuda.synchronize()
    b_order, b_group = order.clone(), group.clone()
    per_instance()
    out["per_instance_ms"] = round(_time_ms(torch, stream, per_instance, 1), 3)
    torch.cuda.synchronize()
    same_pi = bool(torch.equal(order, b_order) and torch.equal(group, b_group))
    if plain:
        plain_path()
        out["plain_ms"] = round(_time_ms(torch, stream, plain_path, 1), 3)
        torch.cuda.synchronize()
        same_plain = bool(torch.equal(order, b_order) and torch.equal(group, b_group))
    else:
        same_plain = True
    picks = sample_instances(sizes)
    ok, bad = check_instances_vs_oracle(cols, sizes, bw, split, b_order, b_group, counts, picks)
    out["check"] = {"batched_equals_per_instance": same_pi, "batched_equals_plain": same_plain,
                    "oracle_instances": len(picks), "oracle_equal": ok, "first_mismatch": bad,
                    "digest_order_group": _digest(torch, b_order, b_group)}
    out["checked"] = bool(same_pi and same_plain and ok)
    del b_order, b_group
    for k in ("batched", "per_instance", "plain"):
        if f"{k}_ms" in out:
            out[f"{k}_mrows_s"] = round(total / (out[f"{k}_ms"] / 1e3) / 1e6, 1)
    out["speedup_batched_vs_per_instance"] = round(out["per_instance_ms"] / out["batched_ms"], 2)
    if plain:
        out["speedup_batched_vs_plain"] = round(out["plain_ms"] / out["batched_ms"], 2)
    del cols, order, group, g2
    torch.cuda.empty_cache()
    return out


def wide(torch, ctx, stream, reps=3, n=WIDE_ROWS):
    cols, card, split, (gsplit, gorder) = wide_workload(torch, n)
    order = torch.empty(n, dtype=torch.int32, device="cuda")
    group = torch.empty(n, dtype=torch.int32, device="cuda")
    g2 = torch.empty_like(group)

    def order_by():
        ctx.run_plan(cols, WIDE_BITS, split, order, group)

    def group_by():
        ctx.run_plan(cols, WIDE_BITS, gsplit, order, group, col_order=gorder, hash=True)

    def plain_path():
        ig, og = None, group
        for c, w in zip(cols, WIDE_BITS):
            ctx.sort_round_plain(c, w, order, in_group=ig, out_group=og)
            ig, og = og, (g2 if og is group else group)

    out = {"rows": n, "bits": WIDE_BITS, "distinct": WIDE_CARD, "order_by_plan": split,
           "group_by_plan": gsplit, "group_by_column_order": gorder}
    results = {}
    for name, fn in (("order_by", order_by), ("group_by", group_by), ("plain", plain_path)):
        fn()
        ms = _time_ms(torch, stream, fn, reps)
        out[f"{name}_ms"] = round(ms, 3)
        out[f"{name}_mrows_s"] = round(n / (ms / 1e3) / 1e6, 1)
        torch.cuda.synchronize()
        # the plain path's last round leaves its group ids in `group` or `g2`
        fin = group if name != "plain" or len(WIDE_BITS) % 2 == 1 else g2
        results[name] = (order.clone(), fin.clone())
        if name != "plain":
            # where the time goes: one more run with per-launch CUDA events
            ctx.profile(True)
            ctx.profile_report()
            fn()
            rep = ctx.profile_report()
            ctx.profile(False)
            out[f"{name}_kernels_ms"] = {k: round(v["ms"], 3) for k, v in
                                         sorted(((k, v) for k, v in rep.items() if not k.startswith("_")),
                                                key=lambda kv: -kv[1]["ms"])}
    out["speedup_order_by_vs_plain"] = round(out["plain_ms"] / out["order_by_ms"], 2)
    same = bool(torch.equal(results["order_by"][0], results["plain"][0])
                and torch.equal(results["order_by"][1], results["plain"][1]))
    props = sorted_properties(torch, cols, results["order_by"][0], results["order_by"][1])
    same_groups = same_grouping(torch, results["order_by"], results["group_by"], n)
    out["check"] = {"order_by_equals_plain": same, "order_by_properties": props,
                    "group_by_same_groups_as_order_by": same_groups,
                    "digest_order_by": _digest(torch, *results["order_by"]),
                    "digest_group_by": _digest(torch, *results["group_by"])}
    out["checked"] = bool(same and all(props.values()) and same_groups)
    del results
    del cols, order, group, g2
    torch.cuda.empty_cache()
    return out


def _digest(torch, *arrays) -> str:
    """sha256 of the arrays' bytes (host copies), a fingerprint of a result."""
    import hashlib
    h = hashlib.sha256()
    for a in arrays:
        h.update(a.cpu().numpy().tobytes())
    return h.hexdigest()[:16]


def _as_u64(torch, c):
    """A column's codes as non-negative int64 (u16 / u32 bits stored signed)."""
    if c.dtype == torch.int16:
        return c.to(torch.int64) & 0xFFFF
    if c.dtype == torch.int32:
        return c.to(torch.int64) & 0xFFFFFFFF
    return c


def sorted_properties(torch, cols, order, group):
    """Size-independent checks of an ORDER BY result on the device: order is a
    permutation, the key tuples read through it do not decrease, the group id
    goes up by one exactly where the tuple changes, and equal tuples keep
    ascending row ids (the canonical tie order)."""
    n = order.shape[0]
    o = order.to(torch.int64)
    perm = bool(torch.equal(torch.sort(o).values, torch.arange(n, device=o.device)))
    gt = torch.zeros(n - 1, dtype=torch.bool, device=o.device)   # tuple[i+1] > tuple[i] decided
    eq = torch.ones(n - 1, dtype=torch.bool, device=o.device)    # equal so far
    lt = torch.zeros(n - 1, dtype=torch.bool, device=o.device)
    for c in cols:
        v = _as_u64(torch, c)[o]
        a, b = v[:-1], v[1:]
        if v.dtype == torch.int64 and c.dtype == torch.int64:
            # full 64-bit codes: compare as unsigned
            a, b = a ^ (-(1 << 63)), b ^ (-(1 << 63))
        gt |= eq & (b > a)
        lt |= eq & (b < a)
        eq &= (b == a)
    nondecreasing = not bool(lt.any())
    g = group.to(torch.int64)
    dense = bool(int(g[0]) == 0 and torch.equal(g[1:] - g[:-1], (~eq).to(torch.int64)))
    ties = bool((o[1:][eq] > o[:-1][eq]).all())
    return {"permutation": perm, "tuples_nondecreasing": nondecreasing, "dense_group_ids": dense,
            "canonical_ties": ties}


def same_grouping(torch, sort_res, hash_res, n):
    """The hash plan groups rows exactly as the sort plan does: per row id,
    (sort group, hash group) pairs form a one-to-one map."""
    so, sg = sort_res
    ho, hg = hash_res
    a = torch.empty(n, dtype=torch.int64, device=so.device)
    b = torch.empty(n, dtype=torch.int64, device=so.device)
    a[so.to(torch.int64)] = sg.to(torch.int64)
    b[ho.to(torch.int64)] = hg.to(torch.int64)
    na = int(a.max()) + 1
    nb = int(b.max()) + 1
    pairs = torch.unique(a * nb + b).numel()
    return bool(na == nb == pairs)


def benchmark(reps=3, plain=True, with_instances=True, wide_rows=WIDE_ROWS):
    import torch
    out = {}
    with capi.Context(0) as ctx:
        stream = torch.cuda.ExternalStream(ctx.stream)
        if with_instances:
            out["instances"] = instances(torch, ctx, stream, reps=reps, plain=plain)
        out["wide"] = wide(torch, ctx, stream, reps=reps, n=wide_rows)
    return out
