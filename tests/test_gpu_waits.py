"""Failure detection without a GPU fault: the bounded waits of the streaming
kernel (fused.cuh) and of the tensor-core GEMM kernels (tc.cuh) give up at
their 2 s limit when nothing completes the barrier, report it to the host as
a status, and leave the context usable (afd_wait_selftest)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("which", [0, 1])
def test_bounded_wait_gives_up_and_reports(pkg, which):
    gave_up, waited = pkg.afd.wait_selftest(which, complete=False)
    assert gave_up
    assert 2.0 <= waited < 4.0
    gave_up, waited = pkg.afd.wait_selftest(which, complete=True)
    assert not gave_up
    assert waited < 0.1
    # the context still runs a simulation
    sim = pkg.Simulation(mode=1)
    sim.SetMinSize(0.3, 0.3, 0.3)
    sim.AddSourceCell((5, 5, 5), np.ones(4, np.float32))
    sim.AddMicCell((8, 8, 8))
    sim.Run(20)
    assert np.all(np.isfinite(sim.mics())) and np.any(sim.mics() != 0)
    sim.close()


def test_selftest_arguments(pkg):
    with pytest.raises(pkg.AfdError):
        pkg.afd.wait_selftest(2, complete=True)
    with pytest.raises(pkg.AfdError):
        pkg.afd.wait_selftest(0, complete=True, device=99)
