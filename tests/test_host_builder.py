"""The product's host level builder (lg_hgraph, lg_host.cpp) must produce the
reference's level layout byte for byte, and reject malformed levels."""
import numpy as np
import pytest

import llama_b200 as lb
from llama_b200 import HostGraph, LgError


def test_levels_match_reference(golden):
    hg = HostGraph(int(golden["V"]))
    for lv in golden["levels"]:
        hg.add_level(*lv)
    for l in range(len(golden["levels"])):
        for dr in (0, 1):
            vt, sl = hg.level_arrays(l, dr)
            assert np.array_equal(vt.view(np.uint8), golden[f"vt{l}_{dr}"]), (l, dr)
            assert np.array_equal(sl, golden[f"slots{l}_{dr}"]), (l, dr)


def test_level_desc_deletions_point_at_marked_slots(golden):
    hg = HostGraph(int(golden["V"]))
    for lv in golden["levels"]:
        hg.add_level(*lv)
    import ctypes as C
    for l in range(1, len(golden["levels"])):
        d = hg.level_desc(l)
        n = d.n_out_deletions
        assert n == len(golden["levels"][l][2])
        if n == 0:
            continue
        dels = np.ctypeslib.as_array(C.cast(d.out_deletions, C.POINTER(C.c_uint8)),
                                     (n * 16,)).view([("edge", "<i8"), ("ml", "<u4"), ("r", "<u4")])
        for e, ml in zip(dels["edge"], dels["ml"]):
            lev, idx = int(e) >> 38, int(e) & ((1 << 38) - 1)
            slot = golden[f"slots{lev}_0"][idx]
            assert int(slot) >> 38 <= ml == l


def test_generator_is_deterministic_and_simple():
    spec = lb.workloads.rmat_multiversion(scale=9, seed=5, levels=3, level0=0.8, delete=0.1)
    a = HostGraph.from_spec(spec)
    b = HostGraph.from_spec(spec)
    for l in range(3):
        for x, y in zip(a.level_input(l)[:4], b.level_input(l)[:4]):
            assert np.array_equal(x, y)
    s, d = a.level_input(0)[:2]
    keys = s.astype(np.uint64) << 32 | d
    assert np.all(np.diff(keys.astype(np.int64)) > 0)      # sorted, no duplicates
    assert not np.any(s == d)                               # no self-loops


@pytest.mark.parametrize("bad", ["dup", "range", "not_live", "delete_at_level0"])
def test_rejects_malformed_levels(bad):
    hg = HostGraph(4)
    if bad == "dup":
        with pytest.raises(LgError):
            hg.add_level([0, 0], [1, 1])
    elif bad == "range":
        with pytest.raises(LgError):
            hg.add_level([0], [4])
    elif bad == "not_live":
        hg.add_level([0], [1])
        with pytest.raises(LgError):
            hg.add_level([], [], [1], [0])
    else:
        with pytest.raises(LgError):
            hg.add_level([0], [1], [0], [1])
