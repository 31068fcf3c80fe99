"""The build entry's smoke check (QV-12 through the backend vs the oracle,
gates through blackwell_kernels, shots) runs on the GPU suite too."""
import pytest

pytestmark = pytest.mark.gpu


def test_graft_entry_smoke():
    import __graft_entry__
    __graft_entry__.smoke()
