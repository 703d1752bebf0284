"""The reference unit test's 11 scenarios x 4 shapes on the CUDA library at
every tile size, against the reference test's own expectations."""
import pytest

from indexes import GpuIndex
from scenarios import SCENARIOS, SHAPES, run_scenario

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
