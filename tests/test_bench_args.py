"""bench.py's command line on the CPU: the defaults (learned + batched in
batch mode, the plain kernel in single mode) and every strategy the C ABI
offers for each mode."""
import sys

import pytest

import bench
from kites_b200 import capi


def parse(monkeypatch, *argv):
    monkeypatch.setattr(sys, "argv", ["bench.py", *argv])
    return bench.parse()


def test_defaults(monkeypatch):
    a = parse(monkeypatch)
    assert a.mode == "batch" and a.strategy == "auto" and a.gpus == 1
    assert a.warmup >= 3
    assert parse(monkeypatch, "--mode", "single").strategy == "plain"


def test_strategy_table_matches_the_abi():
    assert bench.STRATEGIES == {"plain": capi.STRATEGY_PLAIN, "auto": capi.STRATEGY_AUTO,
                                "push": capi.STRATEGY_PUSH, "pull_all": capi.STRATEGY_PULL_ALL,
                                "tpv1": capi.STRATEGY_TPV1, "tpv4": capi.STRATEGY_TPV4,
                                "tpv8": capi.STRATEGY_TPV8, "tpv32": capi.STRATEGY_TPV32,
                                "pull_changed": capi.STRATEGY_PULL_CHANGED,
                                "mip": capi.STRATEGY_MIP}


@pytest.mark.parametrize("strategy", ["plain", "auto", "push", "pull_all", "pull_changed"])
def test_batch_strategies_parse(monkeypatch, strategy):
    assert parse(monkeypatch, "--strategy", strategy).strategy == strategy


def test_gather_margin_and_coarse_options(monkeypatch):
    a = parse(monkeypatch, "--batch-gather", "async", "--margin", "0.05")
    assert a.batch_gather == "async" and abs(a.margin - 0.05) < 1e-12
    a = parse(monkeypatch, "--mode", "single", "--strategy", "mip", "--mip-block", "1024")
    assert a.strategy == "mip" and a.mip_block == 1024 and a.coarse == "pull_all"
    assert parse(monkeypatch, "--mode", "single", "--strategy", "auto",
                 "--coarse", "mip").coarse == "mip"
