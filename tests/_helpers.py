"""Shared helpers of the test suite: expected contacts from an oracle / reference pair result."""
from __future__ import annotations

import numpy as np

ACCEPT = 3
DEGEN = 5


def expected_contacts(r: dict, k: float = 1.0, polyline: bool = False):
    """Contacts (in contact_id order) of one pair result of the oracle or of oracle/_ref.

    Returns dict: geom (n,13) Sn Gn xc0 nA area, nvert (n,), comp (n,), points list of (m,3)."""
    geom, nvert, comp, pts = [], [], [], []
    for l in range(r["nloop"]):
        st = r["loop_status"][l]
        if st != ACCEPT and not (polyline and st == DEGEN):
            continue
        c = int(r["loop_comp"][l])
        vids = r["loop_vid"][r["loop_off"][l]: r["loop_off"][l + 1]]
        V = r["V"][r["v_off"][c]: r["v_off"][c + 1]]
        geom.append(r["loop_geom"][l])
        nvert.append(len(vids))
        comp.append(c)
        pts.append(V[vids])
    g = np.asarray(geom, float).reshape(-1, 13)
    return {"geom": g, "nvert": np.asarray(nvert, np.int64), "comp": np.asarray(comp, np.int64), "points": pts}


def gpu_pair_slice(res: dict, p: int):
    """Contacts of pair p from the CSR result of zdemx._lib.pair_contacts_raw."""
    a, b = res["contact_off"][p], res["contact_off"][p + 1]
    out = {"geom": res["geom"][a:b], "info": res["info"][a:b], "stats": res["stats"][p]}
    if res.get("points") is not None:
        po = res["point_off"]
        out["points"] = [res["points"][po[c]: po[c + 1]] for c in range(a, b)]
    return out


def compare_gpu_to_expected(g: dict, e: dict, r: dict, exact: bool = True, rtol: float = 1e-9) -> list[str]:
    """Differences between one pair's GPU contacts and the expected ones; [] when they agree."""
    bad = []
    st = g["stats"]
    if st[0] != r["nseg"]:
        bad.append(f"segments {st[0]} != {r['nseg']}")
    if st[1] != r["ncomp"]:
        bad.append(f"components {st[1]} != {r['ncomp']}")
    if st[2] != r["nloop"]:
        bad.append(f"raw loops {st[2]} != {r['nloop']}")
    if st[3] != 0:
        bad.append(f"status {st[3]}")
    n = len(e["geom"])
    if len(g["geom"]) != n:
        bad.append(f"contacts {len(g['geom'])} != {n}")
        return bad
    if n == 0:
        return bad
    if not np.array_equal(g["info"][:, 1], np.arange(n)):
        bad.append("contact ids not 0..n-1")
    if not np.array_equal(g["info"][:, 2], e["nvert"]):
        bad.append("loop vertex counts differ")
    if not np.array_equal(g["info"][:, 3], e["comp"]):
        bad.append("components of contacts differ")
    gg = g["geom"][:, :13]
    if exact:
        if not np.array_equal(gg, e["geom"]):
            bad.append(f"geometry not bit-exact (max abs diff {np.max(np.abs(gg - e['geom']))})")
    else:
        scale = np.maximum(np.abs(e["geom"]), 1e-300)
        rel = np.max(np.abs(gg - e["geom"]) / np.maximum(scale, np.max(np.abs(e["geom"]), axis=0, keepdims=True)))
        if rel > rtol:
            bad.append(f"geometry rel err {rel} > {rtol}")
    if "points" in g:
        for c in range(n):
            if not (np.array_equal(g["points"][c], e["points"][c]) if exact else
                    np.allclose(g["points"][c], e["points"][c], rtol=rtol, atol=0)):
                bad.append(f"loop points of contact {c} differ")
                break
    return bad
