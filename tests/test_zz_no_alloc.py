"""zdx_pair_contacts_noalloc: the pair call for callers that may not allocate GPU memory (a host program
whose own pool allocator owns the device, a real-time loop that cannot take cudaMalloc's device-wide
synchronisation).  Its scratch is a fixed __device__ array inside libzdemx.so; the caller owns inputs
and outputs.  Checked here against zdx_pair_contacts on the same inputs, bit-exact, on two calls in a
row (the second call reuses the array the first one left behind), with the device's free memory the
same before and after the second call.  Kept in its own file, collected last."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _setup(levels=(1, 2, 2, 3, 3), npairs=200, depth=0.1):
    import torch

    from zdemx import synth
    from zdemx.contact import MeshLibrary

    rng = np.random.default_rng(77)
    lib = MeshLibrary.build([synth.noised_icosphere(s, 1e-3, 0.15, rng) for s in levels])
    pm = rng.integers(0, lib.n_mesh, size=(npairs, 2)).astype(np.int32)
    pp = synth.pair_poses(rng, npairs, 1e-3, 0.0, depth)
    dev = torch.device("cuda", 0)
    meshes = {"tris": torch.from_numpy(lib.tris).to(dev), "tri_off": torch.from_numpy(lib.tri_off).to(dev),
              "mean_edge": torch.from_numpy(lib.mean_edge).to(dev),
              "bbox_diag": torch.from_numpy(lib.bbox_diag).to(dev)}
    pairs = {"mesh": torch.from_numpy(pm).to(dev), "pose": torch.from_numpy(pp).to(dev)}
    return meshes, pairs, npairs


def _outputs(npairs, cap):
    import torch

    dev = torch.device("cuda", 0)
    return {"ncontact": torch.full((npairs,), -1, dtype=torch.int32, device=dev),
            "contact_off": torch.full((npairs + 1,), -1, dtype=torch.int64, device=dev),
            "stats": torch.full((npairs, 4), -1, dtype=torch.int32, device=dev),
            "geom": torch.full((cap, 20), float("nan"), dtype=torch.float64, device=dev),
            "info": torch.full((cap, 4), -1, dtype=torch.int32, device=dev)}


@pytest.mark.parametrize("levels,npairs,depth", [((1, 2, 2, 3, 3), 200, 0.1), ((1, 4), 24, 0.05)],
                         ids=["to1280", "to5120"])
def test_noalloc_matches_allocating_call_twice(levels, npairs, depth):
    import torch

    from zdemx import _lib

    meshes, pairs, npairs = _setup(levels, npairs, depth)
    ctx = _lib.Context(0)
    try:
        cap = 16 * npairs
        ref = _outputs(npairs, cap)
        torch.cuda.synchronize()
        tot_ref = _lib.pair_contacts_device(ctx, meshes, pairs, ref, k=1e7, split=True)
        assert tot_ref[0] > npairs // 2
        # within the no-allocation call's per-pair segment limit, so both calls must agree
        assert int(ref["stats"][:, 0].max()) <= 1024
        for call in range(2):
            got = _outputs(npairs, cap)
            torch.cuda.synchronize()
            free_before = torch.cuda.mem_get_info()[0]
            tot = _lib.pair_contacts_noalloc(ctx, meshes, pairs, got, k=1e7, split=True)
            torch.cuda.synchronize()
            if call == 1:
                # the point of the entry: nothing on the device was allocated (or freed) by the call
                assert torch.cuda.mem_get_info()[0] == free_before
            assert tot[:3] == tot_ref[:3], (call, tot, tot_ref)
            n = int(tot[0])
            for key in ("ncontact", "contact_off", "stats"):
                assert torch.equal(got[key], ref[key]), (call, key)
            # bit-exact, which is within every tolerance the suite uses
            assert torch.equal(got["geom"][:n], ref["geom"][:n]), call
            assert torch.equal(got["info"][:n], ref["info"][:n]), call
    finally:
        ctx.close()


def test_noalloc_rejects_sizes_beyond_its_limits():
    import torch

    from zdemx import _lib

    meshes, pairs, npairs = _setup()
    ctx = _lib.Context(0)
    try:
        too_many = {"mesh": pairs["mesh"].repeat(30, 1).contiguous(), "pose": pairs["pose"].repeat(30, 1).contiguous()}
        assert too_many["mesh"].shape[0] > 4096
        out = _outputs(too_many["mesh"].shape[0], 16)
        torch.cuda.synchronize()
        with pytest.raises(_lib.ZdxError) as ei:
            _lib.pair_contacts_noalloc(ctx, meshes, too_many, out, k=1e7)
        assert ei.value.status == _lib.ZDX_ERR_INVALID and "at most 4096" in str(ei.value)
        big = _outputs(npairs, 20000)
        with pytest.raises(_lib.ZdxError) as ei:
            _lib.pair_contacts_noalloc(ctx, meshes, pairs, big, k=1e7)
        assert "contact_cap" in str(ei.value)
    finally:
        ctx.close()
