"""ActivateSpace (V:2766-2856) through the C-ABI against the oracle's
restatement of the reference's host tree walk: the result of every position,
then the node pools and child lists bit for bit, and the atlas map that
UpdateAtlas assigns to the activated leaves.  Positions go one call per
batch of `split`, so batching cannot change what the walk does."""
import numpy as np
import pytest

from _helpers import assert_nodes_equal, make_oracle, shell_points
from test_gpu_topology import gpu_volume
from test_oracle import activation_positions

pytestmark = pytest.mark.gpu


def compare_pools(v, o):
    inf = v.info()
    for lev in range(5):
        assert inf.pool_count[lev] == o.pool_count(lev), f"pool count level {lev}"
        assert_nodes_equal(v.nodes(lev), o.nodes(lev), lev)
        if lev >= 1:
            assert np.array_equal(v.childlists(lev), o.childlists(lev)), f"child lists level {lev}"


def activate_both(v, o, pos, split):
    want = [o.activate_space(*p) for p in pos]
    got = np.concatenate([v.ActivateSpace(pos[i:i + split]) for i in range(0, len(pos), split)])
    assert [int(x) for x in got] == want


@pytest.mark.parametrize("split", [1, 7, 1000])
def test_activate_space_from_empty(gvdb2_mod, oracle_mod, split):
    pos = activation_positions()
    o = make_oracle(oracle_mod)
    v = gpu_volume(gvdb2_mod, pos)
    activate_both(v, o, pos, split)
    compare_pools(v, o)
    o.update_atlas()
    v.UpdateAtlas()
    assert v.info().atlas_slots == o.atlas_slots()
    assert np.array_equal(v.atlas_map(), o.atlas_map())


def test_activate_space_after_rebuild(gvdb2_mod, oracle_mod):
    pts = shell_points(50_000, seed=0)
    o = make_oracle(oracle_mod)
    assert o.rebuild_topology(pts, 1.0) == 0
    v = gpu_volume(gvdb2_mod, pts)
    v.RebuildTopology(len(pts), 1.0)
    # existing leaves (the points themselves), new ones, and one past the root
    pos = np.concatenate([pts[:8], activation_positions(11)]).astype(np.float32)
    activate_both(v, o, pos, 16)
    compare_pools(v, o)
    o.update_atlas()
    v.UpdateAtlas()
    assert np.array_equal(v.atlas_map(), o.atlas_map())
