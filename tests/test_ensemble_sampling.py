"""The batched-ensemble workload generator: seeded, within its ranges."""
import numpy as np

from imex_sflow2d_v2_b200 import configs


def test_members_seeded_and_in_range():
    a = configs.ensemble_members(n_members=6, side_min=24, side_max=40)
    b = configs.ensemble_members(n_members=6, side_min=24, side_max=40)
    for (pa, sa, qa, da), (pb, sb, qb, db) in zip(a, b):
        assert da == db
        np.testing.assert_array_equal(sa["B_cent"], sb["B_cent"])
        assert 24 <= da["side"] <= 40 and pa.nx == pa.ny == da["side"]
        assert 1e6 <= da["mfr"] <= 1e8 and 600 <= da["T_source"] <= 1200
        assert 1e-5 <= da["diam"] <= 1e-3 and pa.diam_s[0] == da["diam"]
        assert pa.n_solid == 1 and pa.radial_source_flag == 1
        assert (sa["source_cell"] == 1).any()
    assert len({d["side"] for *_, d in a}) > 1
