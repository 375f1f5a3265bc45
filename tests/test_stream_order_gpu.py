"""The pair calls read the caller's mesh offsets (and, without allocation, the pair meshes) back to the
host to size their work.  They must read them in the order of the context's stream: a caller may queue
the writes of those buffers on that stream (zdx_get_stream) and call the library without waiting.

Here the offsets start out invalid (-1, which the calls reject), a few dense products on the context
stream hold it busy for some milliseconds, and the valid offsets are copied in behind them; the calls
then run at once.  Both must see the valid offsets and give the host call's results."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _busy_then_copy(stream, dst, src):
    import torch

    with torch.cuda.stream(stream):
        a = torch.randn(2048, 2048, dtype=torch.float64, device=dst.device)
        for _ in range(8):
            a = (a @ a) * 1e-3
        dst.copy_(src)


@pytest.mark.parametrize("entry", ["pair_contacts_device", "pair_contacts_noalloc"])
def test_offsets_written_on_the_context_stream_are_read_in_order(entry):
    import torch

    from zdemx import _lib, synth
    from zdemx.contact import MeshLibrary

    rng = np.random.default_rng(404)
    lib = MeshLibrary.build([synth.noised_icosphere(s, 1e-3, 0.15, rng) for s in (1, 2, 3)])
    npairs = 64
    pm = rng.integers(0, lib.n_mesh, size=(npairs, 2)).astype(np.int32)
    pp = synth.pair_poses(rng, npairs, 1e-3, 0.0, 0.1)
    ctx = _lib.Context(0)
    try:
        ref = _lib.pair_contacts_raw(ctx, lib.tris, lib.tri_off, lib.mean_edge, lib.bbox_diag, pm, pp, k=1e7)
        dev = torch.device("cuda", 0)
        meshes = {"tris": torch.from_numpy(lib.tris).to(dev),
                  "tri_off": torch.full((lib.n_mesh + 1,), -1, dtype=torch.int64, device=dev),
                  "mean_edge": torch.from_numpy(lib.mean_edge).to(dev),
                  "bbox_diag": torch.from_numpy(lib.bbox_diag).to(dev)}
        pairs = {"mesh": torch.from_numpy(pm).to(dev), "pose": torch.from_numpy(pp).to(dev)}
        good_off = torch.from_numpy(lib.tri_off).to(dev)
        cap = 16 * npairs
        out = {"ncontact": torch.zeros(npairs, dtype=torch.int32, device=dev),
               "contact_off": torch.zeros(npairs + 1, dtype=torch.int64, device=dev),
               "stats": torch.zeros((npairs, 4), dtype=torch.int32, device=dev),
               "geom": torch.zeros((cap, 20), dtype=torch.float64, device=dev),
               "info": torch.zeros((cap, 4), dtype=torch.int32, device=dev)}
        torch.cuda.synchronize()
        ext = torch.cuda.ExternalStream(ctx.stream_ptr())
        _busy_then_copy(ext, meshes["tri_off"], good_off)
        # no synchronisation here: the call itself must order its read-back after the copy
        tot = getattr(_lib, entry)(ctx, meshes, pairs, out, k=1e7, split=True)
        torch.cuda.synchronize()
        n = int(tot[0])
        assert n == len(ref["geom"]) and n > 0
        assert np.array_equal(out["contact_off"].cpu().numpy(), ref["contact_off"])
        assert np.array_equal(out["stats"].cpu().numpy(), ref["stats"])
        assert np.array_equal(out["geom"][:n].cpu().numpy(), ref["geom"])
    finally:
        ctx.close()
