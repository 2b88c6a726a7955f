"""The round-end smoke check (one small Bjorken run per precision against the oracle)
runs as part of the GPU tests too."""
import pytest

pytestmark = pytest.mark.gpu


def test_smoke():
    import __graft_entry__ as ge
    ge.smoke()
