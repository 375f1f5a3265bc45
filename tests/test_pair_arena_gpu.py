"""The arena form of the rebuild (zdx_tuning.rebuild_arena 1-3) against the oracle and against the
warp-per-pair form, bit for bit: a mixed batch with large pairs (up to 5,120 triangles a mesh), with and
without split_contacts, each form and the fallback path (form 3 sends every pair back to form 0)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _batch(seed):
    from zdemx import synth
    from zdemx.contact import MeshLibrary

    rng = np.random.default_rng(seed)
    meshes = [synth.noised_icosphere(s, 1e-3, 0.15, rng) for s in (1, 2, 3, 3, 4, 4)]
    lib = MeshLibrary.build(meshes)
    npairs = 48
    pm = rng.integers(0, lib.n_mesh, size=(npairs, 2)).astype(np.int32)
    pm[:6] = [[4, 5], [5, 4], [4, 4], [3, 4], [2, 5], [0, 5]]  # pairs of hundreds of segments
    pp = synth.pair_poses(rng, npairs, 1e-3, 0.0, 0.12)
    return lib, pm, pp


@pytest.mark.parametrize("split", [True, False])
def test_arena_forms_match_oracle_and_each_other(ctx, oracle, split):
    from zdemx import contact

    lib, pm, pp = _batch(77 + split)
    results = {}
    before = ctx.tuning()
    try:
        for form in (0, 1, 2, 3):
            ctx.set_tuning(rebuild_arena=form, arena_min_seg=64, arena_warps=8)
            results[form] = contact.pair_contacts_batch(ctx, lib, pm, pp, k=1e7, want_points=False, split=split)
    finally:
        ctx.set_tuning(**before)
    ref = results[0]
    for form in (1, 2, 3):
        r = results[form]
        for key in ("contact_off", "stats"):
            assert np.array_equal(r[key], ref[key]), (form, key)
        assert np.array_equal(r["geom"], ref["geom"]), form
        assert np.array_equal(r["info"], ref["info"]), form
    total = 0
    for p in range(len(pm)):
        a, b = pm[p]
        o = oracle.pair(lib.mesh(a), lib.mean_edge[a], lib.bbox_diag[a], lib.mesh(b), pp[p, :7], pp[p, 7:], split=split)
        acc = [l for l in range(o["nloop"]) if o["loop_status"][l] == 3]
        c0, c1 = ref["contact_off"][p], ref["contact_off"][p + 1]
        assert c1 - c0 == len(acc), p
        assert ref["stats"][p, 0] == o["nseg"] and ref["stats"][p, 1] == o["ncomp"] and ref["stats"][p, 2] == o["nloop"], p
        for c, l in zip(range(c0, c1), acc):
            assert np.array_equal(ref["geom"][c, :13], o["loop_geom"][l]), (p, c - c0)
        total += len(acc)
    assert total > 0
    assert max(int(x) for x in ref["stats"][:, 0]) > 200  # the arena took pairs of hundreds of segments
