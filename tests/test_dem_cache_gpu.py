"""The graph step's clearance cache (config key contact_cache, default on) against the same step without
it: a pair settled on a cached clearance has no segment, and a pair narrowed to its cached near pairs has
the segments of those alone, as the full triangle stage finds, so state, forces and the step log's
counters agree bit for bit.  Covers pairs that close in, touch and part; poses moved by set_state between
steps (translations and rotations larger than any clearance); and the cache emptied by a capacity
growth."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

COUNTERS = ("contacts", "tri_checks", "segments", "comps", "loops", "pairs", "wall_contacts", "history",
            "wall_history")


def _pair(tmp_path, n, seed, cache, name):
    from zdemx.workloads import pour_scene

    cfg = pour_scene(str(tmp_path / name), n=n, seed=seed, steps=1000, vel_sigma=0.3)
    text = open(cfg).read().replace("split_contacts = 1", f"split_contacts = 1\ncontact_cache = {cache}")
    open(cfg, "w").write(text)
    return cfg


def _same(a, b, what):
    sa, fa, ta, ca = a.state()
    sb, fb, tb, cb = b.state()
    for x, y, name in ((sa, sb, "state"), (fa, fb, "force"), (ta, tb, "torque"), (ca, cb, "contact_count")):
        assert np.array_equal(x, y), f"{what}: {name} differs (max {np.max(np.abs(x - y))})"
    ia, ib = a.info(), b.info()
    for k in COUNTERS:
        assert ia[k] == ib[k], f"{what}: {k} without cache {ia[k]}, with {ib[k]}"


def _scenes(tmp_path, n=1500, seed=3):
    from zdemx.dem import Scene

    off = Scene(_pair(tmp_path, n, seed, 0, "off"))
    on = Scene(_pair(tmp_path, n, seed, 1, "on"))
    return off, on


def test_cache_matches_no_cache(tmp_path):
    off, on = _scenes(tmp_path)
    skipped = 0
    for chunk in (1, 1, 2, 5, 20, 40, 60, 80):
        off.step_graph(chunk)
        on.step_graph(chunk)
        _same(off, on, f"after {off.info()['steps']} steps")
        skipped += on.graph_cache()["skipped"]
        assert off.graph_cache()["entries"] == 0
    assert on.graph_cache()["entries"] > 0
    assert skipped > 0, "no pair was skipped on the cache"
    assert off.info()["contacts"] > 0


def test_cache_after_moves_and_growth(tmp_path):
    """Poses set from the host between graph steps: the cached poses, not the step count, decide."""
    off, on = _scenes(tmp_path, n=800, seed=5)
    rng = np.random.default_rng(11)
    for k in range(4):
        off.step_graph(30)
        on.step_graph(30)
        _same(off, on, f"round {k}")
        st, _, _, _ = off.state()
        # some particles translated by 0 .. 40 um (clearances are a few to tens of um), others rotated by
        # up to 0.05 rad, the rest untouched
        n = st.shape[0]
        mv = rng.random(n) < 0.3
        st[mv, 0:3] += rng.normal(size=(mv.sum(), 3)) * 2e-5
        rot = rng.random(n) < 0.3
        ang = rng.uniform(0, 0.05, rot.sum())
        ax = rng.normal(size=(rot.sum(), 3))
        ax /= np.linalg.norm(ax, axis=1, keepdims=True)
        dq = np.concatenate([np.cos(ang / 2)[:, None], np.sin(ang / 2)[:, None] * ax], 1)
        q = st[rot, 3:7]
        w1, x1, y1, z1 = dq.T
        w2, x2, y2, z2 = q.T
        st[rot, 3:7] = np.stack([w1 * w2 - x1 * x2 - y1 * y2 - z1 * z2, w1 * x2 + x1 * w2 + y1 * z2 - z1 * y2,
                                 w1 * y2 - x1 * z2 + y1 * w2 + z1 * x2, w1 * z2 + x1 * y2 - y1 * x2 + z1 * w2], 1)
        off.set_state(st)
        on.set_state(st)
    for chunk in (1, 3, 10):
        off.step_graph(chunk)
        on.step_graph(chunk)
        _same(off, on, "after the last move")


def test_cache_with_tiny_capacities(tmp_path):
    """Capacities that overflow: the step reruns after growth with an empty cache."""
    off, on = _scenes(tmp_path, n=600, seed=8)
    on.graph_reserve(64, 16, 4096, 8)
    off.graph_reserve(64, 16, 4096, 8)
    for chunk in (1, 2, 7, 20):
        off.step_graph(chunk)
        on.step_graph(chunk)
        _same(off, on, f"after {off.info()['steps']} steps")


def test_state_into_caller_buffers(tmp_path):
    """Scene.state(out=...) fills the caller's arrays with what a fresh call returns."""
    off, on = _scenes(tmp_path, n=300, seed=4)
    on.step_graph(5)
    fresh = on.state()
    buf = tuple(np.full_like(a, 7) for a in fresh)
    got = on.state(out=buf)
    assert all(g is b for g, b in zip(got, buf))
    assert all(np.array_equal(g, f) for g, f in zip(got, fresh))
    with pytest.raises(ValueError):
        on.state(out=(np.zeros((on.n, 15)),) + buf[1:])
