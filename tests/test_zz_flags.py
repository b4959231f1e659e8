"""After the GPU suite: no bounded wait of the TMA-pipelined kernels ran out
(the flag word the kernels raise when a wait gives up is still 0)."""
import pytest

from cuhelmholtz_b200 import api

pytestmark = pytest.mark.gpu


def test_no_wait_ran_out():
    assert api.debug_flags(reset=True) == 0
