"""The FP64 tangent's DMMA tile table (igab_warp_tiles8.inc, written by
gen_warp_tiles.py): over the 8 consumer warps every upper 8x8 tile of the 88x88
element matrix and of the 32x32 geometric block is computed exactly once, and each
warp's fragment indices stay inside its fragment lists.  CPU only."""
import os
import re

INC = os.path.join(os.path.dirname(__file__), "..", "igap4standard_b200", "csrc", "igab_warp_tiles8.inc")


def _tables():
    text = open(INC).read()
    warps = {}
    for m in re.finditer(r"template <> struct warp_tiles8<(\d+)> \{(.*?)\n\};", text, re.S):
        w, body = int(m.group(1)), m.group(2)
        consts = dict((k, int(v)) for k, v in re.findall(r"(NB|NT|NGA|NGB|NGT) = (\d+)", body))

        def fn(name):
            f = re.search(r"constexpr int %s\(int k\) \{ switch \(k\) \{(.*?)default" % name, body)
            return [int(v) for v in re.findall(r"case \d+: return (\d+);", f.group(1))]
        warps[w] = (consts, {n: fn(n) for n in ("blk", "ti", "tj", "gablk", "gbblk", "gti", "gtj")})
    return warps


def test_every_tile_once():
    warps = _tables()
    assert sorted(warps) == list(range(8))
    k_tiles, g_tiles = [], []
    for w, (c, f) in warps.items():
        assert len(f["blk"]) == c["NB"] and len(f["ti"]) == c["NT"] and len(f["tj"]) == c["NT"]
        assert len(f["gablk"]) == c["NGA"] and len(f["gbblk"]) == c["NGB"]
        assert len(f["gti"]) == c["NGT"] and len(f["gtj"]) == c["NGT"]
        for i, j in zip(f["ti"], f["tj"]):
            assert 0 <= i < c["NB"] and 0 <= j < c["NB"]
            k_tiles.append((f["blk"][i], f["blk"][j]))
        for i, j in zip(f["gti"], f["gtj"]):
            assert 0 <= i < c["NGA"] and 0 <= j < c["NGB"]
            g_tiles.append((f["gablk"][i], f["gbblk"][j]))
    assert sorted(k_tiles) == [(i, j) for i in range(11) for j in range(i, 11)]
    assert sorted(g_tiles) == [(i, j) for i in range(4) for j in range(i, 4)]
