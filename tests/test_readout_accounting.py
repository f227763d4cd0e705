"""The learned readout's fallback accounting (surrogate_workflow.readout_accounting)
without a GPU: how many FDTD runs the rejected pairs cost and the IRs/s of the
readout with its fallback against the FDTD alone, for queries known before
the runs and for query pairs arriving one at a time after them."""
import numpy as np
import pytest


def acct(pkg, accept, t_pred=0.01, fd_s=(2.0, 2.0), t_plain=None):
    import ancfield_b200.surrogate_workflow as SW
    return SW.readout_accounting(np.asarray(accept, bool), t_pred, list(fd_s), t_plain)


def test_every_pair_accepted(pkg):
    a = acct(pkg, np.ones((2, 4, 8)))
    assert a["query_pairs"] == 64 and a["fallback_runs"] == 0 and a["rejected_pairs"] == 0
    # before the runs: two batched runs (4 s) against 0.01 s of predictions
    assert a["irs_fdtd"] == pytest.approx(64 / 4.0)
    assert a["irs_readout"] == pytest.approx(64 / 0.01)
    # after the runs: each pair costs one source's share of a batched run (0.5 s)
    assert a["t_pair"] == pytest.approx(0.5)
    assert a["irs_fdtd_after"] == pytest.approx(2.0)
    assert a["gain_after"] == pytest.approx((64 / 0.01) / 2.0)


def test_one_rejected_pair_per_source_costs_every_run_before_the_runs(pkg):
    acc = np.ones((2, 4, 8), bool)
    acc[:, :, 3] = False  # one rejected query position per (wall set, source)
    a = acct(pkg, acc)
    assert a["fallback_runs"] == 8 and a["rejected_pairs"] == 8
    # eight single-source runs at the batched share (0.5 s each): 4 s, no gain over two batched runs
    assert a["irs_readout"] == pytest.approx(64 / (0.01 + 8 * 0.5))
    assert a["gain"] < 1.0
    # after the runs only the 8 rejected pairs pay: 56 of 64 pairs answered by the readout
    assert a["irs_readout_after"] == pytest.approx(64 / (0.01 + 8 * 0.5))
    assert a["gain_after"] == pytest.approx((64 / 4.01) / 2.0)
    assert a["gain_after"] > 7.9


def test_plain_run_time_prices_the_fallback_runs(pkg):
    acc = np.ones((1, 2, 4), bool)
    acc[0, 1, 0] = False
    a = acct(pkg, acc, fd_s=(1.0,), t_plain=0.8)
    assert a["fallback_runs"] == 1
    assert a["irs_readout"] == pytest.approx(8 / (0.01 + 0.8))
    # the after-the-runs setting prices a pair at the batched share in both arms
    assert a["t_pair"] == pytest.approx(0.5)
    assert a["irs_readout_after"] == pytest.approx(8 / (0.01 + 0.5))


def test_nothing_accepted_is_slower_than_the_fdtd(pkg):
    a = acct(pkg, np.zeros((1, 4, 16)))
    assert a["rejected_pairs"] == 64 and a["fallback_runs"] == 4
    assert a["gain_after"] < 1.0
