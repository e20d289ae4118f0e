"""Failure paths on the GPU, without a GPU fault.

The partitioned and sort-merge joins wait on mbarriers for their bulk copies
with an iteration bound; a wait that runs out sets the call's error word and
the call returns ADB_ERR_TIMEOUT.  adb_join_params.test_flags =
ADB_TEST_WAITS_RUN_OUT makes every such wait report "ran out" after it has
really completed, so the host path is exercised while no kernel spins and
nothing is left in flight.  The context must stay usable: the next call
without the flag returns the oracle's result.
"""
import pytest

import alliancedb_b200 as adb

pytestmark = pytest.mark.gpu

ADB_TEST_WAITS_RUN_OUT = 1


@pytest.mark.parametrize("algo", ["PRO", "PRH", "m-way"])
def test_wait_run_out_returns_timeout_then_recovers(oracle, algo):
    R = adb.gen_pk(1 << 16, 31)
    S = adb.gen_fk(1 << 16, R, 0.0, 32)
    with pytest.raises(adb.AdbError) as ei:
        adb.join(algo, R, S, adb.default_params(test_flags=ADB_TEST_WAITS_RUN_OUT))
    assert ei.value.status == adb.ADB_ERR_TIMEOUT
    assert "bounded device wait" in adb.lib().adb_last_error().decode()
    got = adb.join(algo, R, S)
    assert (got.count, got.checksum) == oracle.by_name(algo, R, S)


def test_wait_flag_is_ignored_where_no_bounded_wait_exists(oracle):
    """NPO has no bulk-copy waits: the flag changes nothing there."""
    R = adb.gen_pk(1 << 14, 33)
    S = adb.gen_fk(1 << 14, R, 0.0, 34)
    got = adb.join("NPO", R, S, adb.default_params(test_flags=ADB_TEST_WAITS_RUN_OUT))
    assert (got.count, got.checksum) == oracle.npo(R, S)
