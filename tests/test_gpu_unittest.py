"""The reference unit test's 11 scenarios x 4 shapes on the CUDA library at
every tile size, and on the reference's own gpu_masstree (which pins the
restated expectations to the real reference)."""
import pytest

from indexes import GpuIndex, RefIndex
from scenarios import SCENARIOS, SHAPES, run_scenario
from oracle.pyoracle import RefMasstree

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("tile", [4, 8, 16, 32])
@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("scenario", list(SCENARIOS))
def test_b200_scenario(scenario, shape, tile):
    made = []

    def make():
        made.append(GpuIndex(tile_size=tile, pool_bytes=256 << 20))
        return made[-1]
    try:
        run_scenario(scenario, shape, make)
    finally:
        for m in made:
            m.close()


@pytest.mark.skipif(not RefMasstree.available(), reason="reference build absent")
@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("scenario", list(SCENARIOS))
def test_reference_scenario(scenario, shape):
    made = []

    def make():
        made.append(RefIndex(pool_ratio=0.02))
        return made[-1]
    try:
        run_scenario(scenario, shape, make)
    finally:
        for m in made:
            m.close()
