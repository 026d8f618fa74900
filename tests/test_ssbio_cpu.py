"""The reference's column-file layout (src/ssb/ssb_utils.h:106-171): names of the
files, and a round trip of synthetic columns written and read back in it, which
then answers Q3.3 and Q4.1 like the in-memory columns."""
import numpy as np
import pytest



def test_file_names_follow_ssb_column_order(sj):
    assert sj.ssb_file_name("lo_custkey") == "LINEORDER2"
    assert sj.ssb_file_name("lo_orderdate") == "LINEORDER5"
    assert sj.ssb_file_name("lo_revenue") == "LINEORDER12"
    assert sj.ssb_file_name("lo_supplycost") == "LINEORDER13"
    assert sj.ssb_file_name("d_datekey") == "DDATE0"
    assert sj.ssb_file_name("d_year") == "DDATE4"
    assert sj.ssb_file_name("s_region") == "SUPPLIER5"
    assert sj.ssb_file_name("c_nation") == "CUSTOMER4"
    assert sj.ssb_file_name("p_brand1") == "PART4"
    with pytest.raises(sj.StarJoinError) as e:
        sj.ssb_file_name("lo_nothing")
    assert e.value.status == sj.SJ_ERR_INVALID_ARGUMENT


def test_round_trip_answers_queries(sj, oracle, tmp_path):
    sc = sj.StarSchema(seed=21, fact_rows=250_003, cust_rows=3000, supp_rows=200, part_rows=20_000)
    cols = sj.gen_host(sc)
    sj.store_ssb_columns(str(tmp_path), cols)
    assert (tmp_path / "LINEORDER2").stat().st_size == 4 * sc.fact_rows  # headerless int32
    lengths = {k: len(v) for k, v in cols.items() if k in sj.SSB_NAMES}
    back = sj.load_ssb_columns(str(tmp_path), lengths)
    for k in lengths:
        np.testing.assert_array_equal(back[k], cols[k], k)
    for q in (sj.q33_query(sc), sj.q41_query(sc)):
        assert oracle.run(q, back) == oracle.run(q, cols)
    with pytest.raises(sj.StarJoinError):  # a file shorter than asked for
        sj.load_ssb_columns(str(tmp_path), {"fk_cust": sc.fact_rows + 1})
    with pytest.raises(sj.StarJoinError):
        sj.load_ssb_columns(str(tmp_path / "missing"), {"fk_cust": 1})
