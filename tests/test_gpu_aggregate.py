"""fmcs_group_aggregate: per-group count / sum / min / max of a payload column
over (order, group) from a sort plan (groups are runs of positions) and from
a hash plan (groups are not), against numpy; and its bad-input check."""
import numpy as np
import pytest

from fastmulticolsort_b200 import capi
from fastmulticolsort_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _expect(payload, order, group, ng, signed):
    v = payload[order].astype(np.int64 if signed else np.uint64)
    cnt = np.bincount(group, minlength=ng).astype(np.uint64)
    s = np.zeros(ng, np.uint64)
    np.add.at(s, group, v.astype(np.uint64))
    mn = np.full(ng, np.iinfo(v.dtype).max, v.dtype)
    np.minimum.at(mn, group, v)
    mx = np.full(ng, np.iinfo(v.dtype).min, v.dtype)
    np.maximum.at(mx, group, v)
    return cnt, s, mn, mx


@pytest.mark.parametrize("hash_plan", [False, True])
@pytest.mark.parametrize("ptype,signed", [(np.uint32, False), (np.int32, True), (np.uint64, False), (np.int64, True)])
def test_group_aggregate_matches_numpy(ctx, hash_plan, ptype, signed):
    torch = pytest.importorskip("torch")
    n = 200000
    cols, bw = W.cols_uniform(n, [12, 20], seed_index=71, distinct=[300, 50])
    order = np.zeros(n, np.uint32)
    group = np.zeros(n, np.uint32)
    ng = ctx.run_plan(cols, bw, [32], order, group, hash=hash_plan)
    rng = np.random.default_rng(5)
    info = np.iinfo(ptype)
    payload = rng.integers(max(info.min, -(1 << 40)), min(info.max, 1 << 40), size=n, dtype=np.int64).astype(ptype)
    d_payload = torch.from_numpy(payload.view({4: np.int32, 8: np.int64}[payload.itemsize])).cuda()
    d_order = torch.from_numpy(order.view(np.int32)).cuda()
    d_group = torch.from_numpy(group.view(np.int32)).cuda()
    outs = [torch.empty(ng, dtype=torch.int64, device="cuda") for _ in range(4)]
    for _ in range(2):   # twice: the outputs are reset by every call
        ctx.group_aggregate(d_payload, d_order, d_group, ng, *outs, signed=signed)
    cnt, s, mn, mx = _expect(payload, order, group, ng, signed)
    got = [o.cpu().numpy() for o in outs]
    assert np.array_equal(got[0].view(np.uint64), cnt)
    assert np.array_equal(got[1].view(np.uint64), s)
    vt = np.int64 if signed else np.uint64
    assert np.array_equal(got[2].view(vt), mn)
    assert np.array_equal(got[3].view(vt), mx)


def test_group_aggregate_rejects_ids_out_of_range(ctx):
    torch = pytest.importorskip("torch")
    n = 1000
    payload = torch.arange(n, dtype=torch.int32, device="cuda")
    order = torch.arange(n, dtype=torch.int32, device="cuda")
    group = torch.arange(n, dtype=torch.int32, device="cuda") // 10   # 100 groups
    cnt = torch.empty(50, dtype=torch.int64, device="cuda")
    with pytest.raises(capi.FmcsError):
        ctx.group_aggregate(payload, order, group, 50, count=cnt)   # ids 50..99 beyond ngroups
    # the context keeps working
    cnt = torch.empty(100, dtype=torch.int64, device="cuda")
    ctx.group_aggregate(payload, order, group, 100, count=cnt)
    assert (cnt.cpu().numpy() == 10).all()
