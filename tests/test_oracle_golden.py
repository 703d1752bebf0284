"""The CPU oracle against the reference unit test's seeded inputs and its
closed-form expectations (all 11 scenarios x 4 shapes, 1024 keys)."""
import pytest

from indexes import OracleIndex
from scenarios import SCENARIOS, SHAPES, run_scenario


@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("scenario", list(SCENARIOS))
def test_oracle_scenario(scenario, shape):
    run_scenario(scenario, shape, lambda: OracleIndex())


@pytest.mark.parametrize("shape", ["k1-200_v1-200"])
@pytest.mark.parametrize("scenario", ["FindExist", "RangeQuery", "ConcurrentMix", "EraseAllTwice"])
def test_sharded_oracle_scenario(scenario, shape):
    # The range-partitioned, multi-threaded oracle (the CPU baseline) must agree.
    run_scenario(scenario, shape, lambda: OracleIndex(shards=8, threads=8))
