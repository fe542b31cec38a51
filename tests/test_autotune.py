"""The single-table autotuner: tile size of the build and section size of the sectioned
sampler, timed on the device and recorded per (GPU, ceil(log2 n)), with the JSON cache written
and read back. CPU: the cache file format is checked on load."""
import numpy as np
import pytest
import torch

import py_oracle as po
import wrs


def test_cache_load_checks_the_format(tmp_path):
    good = tmp_path / "good.json"
    good.write_text('{"entries": [\n  {"gpu": "Some GPU", "log2n": 20, "tile_items": 2048, "section_items": 4096}\n]}\n')
    assert wrs.autotune_cache_load(str(good)) == wrs.WRS_SUCCESS
    bad = tmp_path / "bad.json"
    bad.write_text('{"entries": [{"gpu": "x", "log2n": 3}]}')
    assert wrs.autotune_cache_load(str(bad)) == wrs.WRS_ERR_INVALID_ARGUMENT
    assert wrs.autotune_cache_load(str(tmp_path / "missing.json")) == wrs.WRS_ERR_INVALID_ARGUMENT


@pytest.mark.gpu
def test_autotune_records_choices_and_round_trips_the_cache(cuda, tmp_path):
    n = (1 << 20) + 11
    w_np = np.random.default_rng(9).random(n, dtype=np.float32)
    w = torch.from_numpy(w_np).cuda()
    table = torch.empty(n, dtype=torch.int64, device="cuda")
    need = max(wrs.alias_build_scratch_bytes(n, wrs.build_opts(tile_items=t)) for t in (1024, 2048, 4096))
    scratch = torch.empty(need, dtype=torch.uint8, device="cuda")
    st, opts = wrs.autotune_build(w, table, scratch)
    assert st == wrs.WRS_SUCCESS and opts.tile_items in (1024, 2048, 4096)
    # the table it left is the build's (the tile size does not change the table)
    W = po.exact_sum(w_np)
    np.testing.assert_array_equal(table.cpu().numpy().view(np.uint32).reshape(-1, 2), po.exact_build(w_np, W))
    out = torch.empty(1 << 24, dtype=torch.int32, device="cuda")
    st, S = wrs.autotune_sections(table, n, out.numel(), out)
    assert st == wrs.WRS_SUCCESS and S in [512 << k for k in range(8)]
    st, t_rec, S_rec = wrs.autotune_lookup(n)
    assert (st, t_rec, S_rec) == (wrs.WRS_SUCCESS, opts.tile_items, S)
    path = str(tmp_path / "tune.json")
    assert wrs.autotune_cache_save(path) == wrs.WRS_SUCCESS
    assert '"log2n": 21' in open(path).read()
    assert wrs.autotune_cache_load(path) == wrs.WRS_SUCCESS
    assert wrs.autotune_lookup(n)[1:] == (opts.tile_items, S)
