"""Device memory of destroyed contexts: kept in the library's pool for the
next context until relax_release_cached_memory returns it to the device."""
import pytest

from relax_b200.api import Relax, release_cached_memory
from relax_b200.config import powerlaw_thrust

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def test_release_cached_memory_returns_the_pool_to_the_device():
    sim = powerlaw_thrust(sx=256, sz=128, dx=0.5)
    with Relax(sim) as r:
        r.coseismic()
        r.step()
    torch.cuda.synchronize()
    held = torch.cuda.mem_get_info()[0]
    release_cached_memory(0)
    freed = torch.cuda.mem_get_info()[0] - held
    # the context holds ~0.6 GB of fields and spectrum (256 x 256 x 128 box)
    assert freed > 4e8, freed
    # a context created afterwards allocates again and runs
    with Relax(sim) as r:
        r.coseismic()
        assert r.step()[0] == 1
    # releasing twice, or with nothing pooled, is harmless
    release_cached_memory(0)
    release_cached_memory(0)


def test_release_cached_memory_rejects_a_missing_device():
    from relax_b200 import _lib
    with pytest.raises(_lib.RelaxError):
        release_cached_memory(torch.cuda.device_count() + 3)
