"""The build entry's smoke run (a small DI + PT frame sequence on cuda:0
against the oracle) stays runnable."""
import pytest


@pytest.mark.gpu
def test_smoke():
    import __graft_entry__
    __graft_entry__.smoke()
