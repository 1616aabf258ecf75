"""A BFS level loop driven through the C ABI one level at a time
(gsw_traversal_begin, gsw_level_begin, gsw_select, gsw_level_end,
gsw_traversal_end), as a host framework that cannot instantiate the
templates would drive it: levels bit-exact with the oracle, the rule and
learned selectors taking the built-in loop's decisions level for level, every
fixed variant, and the misuse cases rejected."""
import numpy as np
import pytest

import gswitch_b200 as gs
import oracle
from conftest import golden_names, load_golden

pytestmark = pytest.mark.gpu

VARIANTS = [(d, f, lb) for d in ("Push", "Pull") for f in ("Queue", "Bitmap") for lb in ("TM", "WM", "CM", "STRICT",
                                                                                           "TWC")]


def drive(ctx, g, root, selector="rules", fixed=None):
    t = g.traversal(root)
    chosen = []
    while True:
        stats, done = t.level_begin()
        if done:
            break
        choice = fixed if fixed is not None else ctx.select(stats, selector)[0]
        chosen.append(tuple(choice))
        t.level_end(choice)
    lv, st = t.end()
    return lv, st, chosen


@pytest.mark.parametrize("name", golden_names())
def test_traversal_goldens_rules_and_every_variant(ctx, name):
    d = load_golden(name)
    g = ctx.upload(d["off"], d["col"])
    root = int(d["root"])
    lv, st, _ = drive(ctx, g, root)
    assert np.array_equal(lv, d["lvl"])
    assert st.device_error == 0
    for v in VARIANTS:
        lv, _, chosen = drive(ctx, g, root, fixed=v)
        assert np.array_equal(lv, d["lvl"]), (name, v)
        assert all(c == v for c in chosen)


@pytest.fixture(scope="module")
def rmat14():
    h = oracle.rmat(14, 16, seed=1)
    return h, oracle.bfs(h, 0)


@pytest.mark.parametrize("selector", ["rules", "mlp"])
def test_traversal_takes_the_built_in_loop_decisions(ctx, rmat14, selector):
    """The caller's loop (gsw_select on the counters gsw_level_begin returns)
    runs the same variant and frontier at every level as gsw_bfs with the same
    selector and standalone levels (no fusion, no persistent launches)."""
    from gswitch_b200.selector_train import load_model

    h, ref = rmat14
    if selector == "mlp":
        model, conf = load_model()
        ctx.mlp_load(model, conf)
    try:
        g = ctx.upload(h.off, h.col)
        for root in [0] + [int(r) for r in oracle.roots(h, 5, 3)]:
            lv, st, chosen = drive(ctx, g, root, selector)
            assert np.array_equal(lv, oracle.bfs(h, root)), root
            _, host = g.bfs(root, gs.RunOpts(selector=selector, fusion=gs.STANDALONE, persistent=False))
            assert [t[:3] for t in host.trace] == chosen, root
            assert st.trace == host.trace, root
            assert st.edges == host.edges
    finally:
        ctx.mlp_load(None)


def test_traversal_misuse_is_rejected(ctx, rmat14):
    h, _ = rmat14
    g = ctx.upload(h.off, h.col)
    t = g.traversal(0)
    with pytest.raises(gs.GswError) as e:  # no gsw_level_begin for this level yet
        t.level_end(("Push", "Queue", "WM"))
    assert gs.STATUS[e.value.code] == "INVALID_ARG"
    t.level_begin()
    with pytest.raises(gs.GswError):  # 2D partition is not a level variant here
        t.level_end(("Push", "Queue", "TWOD"))
    while True:
        stats, done = t.level_begin()
        if done:
            break
        t.level_end(("Push", "Queue", "STRICT"))
    with pytest.raises(gs.GswError):  # the loop is over
        t.level_end(("Push", "Queue", "STRICT"))
    lv, _ = t.end()
    assert np.array_equal(lv, oracle.bfs(h, 0))
    with pytest.raises(gs.GswError):  # BFS from a vertex of the graph only
        g.traversal(h.n)
