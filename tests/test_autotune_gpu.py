"""The launch-shape autotuner on the GPU: every candidate shape (and RHS packing) gives
bit-identical results -- the Dslash of each link format and RHS count, and a whole mixed-precision
multi-shift solve whose fused reductions are block-size independent -- and the first launch of an
instantiation records its timed choice, which the JSON cache file receives."""
import json

import numpy as np
import pytest

import rhmc_b200 as rb
from rhmc_b200 import fields as F

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def _restore():
    yield
    rb.autotune_override(-1)


@pytest.mark.parametrize("fmt", [rb.LINKS_F64_18, rb.LINKS_F64_12, rb.LINKS_F32_12, rb.LINKS_F16_12])
@pytest.mark.parametrize("n", [1, 4, 5, 8])
def test_dslash_shapes_bit_identical(fmt, n):
    from gpu_util import new_ctx, to_internal, from_internal, internal_buffer
    dims = (8, 8, 8, 8)
    ctx = new_ctx(dims)
    ctx.set_gauge(F.random_links(dims, seed=61))
    xin = to_internal(ctx, fmt, F.random_spinor(dims, seed=62, n=n))
    outs = []
    for cand in (0, 1, 2):
        rb.autotune_override(cand)
        out = internal_buffer(ctx, fmt, n)
        ctx.dslash(fmt, 1, out, xin, n)
        outs.append(from_internal(ctx, fmt, out, n))
    assert np.array_equal(outs[0], outs[1]) and np.array_equal(outs[0], outs[2])


def test_mixed_solve_bit_identical_across_shapes():
    from gpu_util import new_ctx
    dims = (6, 4, 4, 8)
    ctx = new_ctx(dims, mass=0.05)
    ctx.set_gauge(F.random_links(dims, seed=63))
    b = F.random_spinor(dims, seed=64, n=4)
    shifts = np.geomspace(1e-3, 10.0, 6)
    res = []
    for cand in (0, 1, 2):
        rb.autotune_override(cand)
        x, info = ctx.msolve_host(b, shifts, 1e-10, mode=rb.MSOLVE_MIXED, fmt=rb.LINKS_F32_12)
        assert info["status"] == 0
        res.append((x, info["iters_total"], info["refine_iters"]))
    for x, it, rit in res[1:]:
        assert np.array_equal(x, res[0][0]) and it == res[0][1] and rit == res[0][2]


def test_first_launch_records_choice(tmp_path):
    from gpu_util import new_ctx, to_internal, internal_buffer
    rb.tune_clear()
    cache = tmp_path / "tune.json"
    rb.tune_cache_load(str(cache))
    dims = (8, 8, 8, 16)
    ctx = new_ctx(dims)
    ctx.set_gauge(F.random_links(dims, seed=65))
    fmt = rb.LINKS_F32_12
    xin = to_internal(ctx, fmt, F.random_spinor(dims, seed=66, n=4))
    out = internal_buffer(ctx, fmt, 4)
    ctx.dslash(fmt, 1, out, xin, 4)
    ents = {e["key"]: e for e in rb.tune_report()["entries"]}
    key = [k for k in ents if k.endswith("|vh=%d|dslash f32_12 nr=4 y=0 red=0" % ctx.Vh)]
    assert len(key) == 1, list(ents)
    e = ents[key[0]]
    assert 0 <= e["choice"] <= 2 and len(e["us"]) == 3 and min(e["us"]) > 0
    assert e["us"][e["choice"]] == min(e["us"])
    on_disk = {x["key"] for x in json.loads(cache.read_text())["entries"]}
    assert key[0] in on_disk
