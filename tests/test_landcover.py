"""Land-cover lookup (FloodCA prep/floodca_prep/landcover.py:35-70) against
fixtures generated by running the reference's own lookup functions and
table (tests/golden/landcover/make_landcover.py): WorldCover codes (and codes
absent from the table) to Manning n and runoff C with k_n / k_C scaling, C
clipped to [0, 1], and the 3 x 3 aggregation to 90 m, bit for bit."""
import numpy as np
import pytest

from conftest import GOLDEN
from floodca_b200 import landcover, synth


@pytest.fixture(scope="module")
def fx():
    return np.load(GOLDEN / "landcover" / "worldcover.npz")


def test_builtin_table_is_the_reference_table(fx):
    codes = [int(c) for c in fx["table_codes"]]
    assert sorted(landcover.WORLDCOVER) == codes
    for c, n, C in zip(codes, fx["table_n"], fx["table_C"]):
        assert landcover.WORLDCOVER[c] == (n, C)


@pytest.mark.parametrize("tag", ["k1", "k2", "k3"])
def test_lookup_matches_reference(fx, tag):
    k_n, k_c = (float(x) for x in fx[f"{tag}_kn_kc"])
    n, C = landcover.lookup(fx["lc30"], None, k_n, k_c)
    assert n.dtype == C.dtype == np.float32
    assert np.array_equal(n, fx[f"{tag}_n30"]) and np.array_equal(C, fx[f"{tag}_c30"])
    lc90, n90, c90 = landcover.lookup_90m(fx["lc30"], None, k_n, k_c)
    assert np.array_equal(lc90, fx[f"{tag}_lc90"])
    assert np.array_equal(n90, fx[f"{tag}_n90"]) and np.array_equal(c90, fx[f"{tag}_c90"])


def test_table_file_round_trip(tmp_path):
    p = tmp_path / "lc.csv"
    rows = ["worldcover_code,class,manning_n,runoff_C", "10,Tree,0.1,0.2", "-1,default,0.05,0.5"]
    p.write_text("\n".join(rows) + "\n")
    t = landcover.load_table(p)
    assert t == {10: (0.1, 0.2), -1: (0.05, 0.5)}
    n, C = landcover.lookup(np.array([[10, 99]], np.uint8), t, 2.0, 3.0)
    assert n.tolist() == [[np.float32(0.1) * np.float32(2.0), np.float32(0.05) * np.float32(2.0)]]
    assert C.tolist() == [[np.float32(0.2) * np.float32(3.0), 1.0]]


def test_apply_feeds_a_domain(fx):
    dom = synth.make_terrain(synth.TerrainSpec(48, 63, seed=2))
    out = landcover.apply(dom, fx["lc30"], k_n=1.3, k_c=1.6)
    assert np.array_equal(out.n, fx["k2_n30"]) and np.array_equal(out.C, fx["k2_c30"])
    assert np.array_equal(out.z, dom.z)
    with pytest.raises(ValueError):
        landcover.apply(dom, fx["lc30"][:10])
