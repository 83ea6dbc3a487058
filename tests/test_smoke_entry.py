"""The build entry's smoke run: one small factorization + refined solve on
cuda:0, checked against the oracle's inertia and the backward-error bound."""
import pytest

pytestmark = pytest.mark.gpu


def test_graft_entry_smoke_passes():
    import __graft_entry__ as entry

    entry.smoke()
