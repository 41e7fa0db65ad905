"""Failure detection of the staged voxel kernel's bounded waits, without a GPU fault.

Every mbarrier wait of the staged kernel has a time limit.  The test hook
csp_test_wait_timeout makes one thread of the first CTA (not its issuing thread) wait on
an mbarrier that nothing completes, with a 1 ms limit, so the real timeout path runs: the
CTA takes one decision at its end-of-plane barrier, drains its own bulk copies, sets the
timeout bit of the device error word and returns.  Every bulk copy that was issued
completes, so nothing is left writing shared memory.  The host reads the error word:
csp_advance returns CSP_EDEVICE and csp_status names the timeout, where the reference
aborts the process (fvm_mpi/src/utils.h:21-27).  The context stays usable: a fresh
handle runs and matches the FP64 oracle.
"""
import numpy as np
import pytest

from parity import assert_close

pytestmark = pytest.mark.gpu

CSP_EDEVICE = -5


def test_bounded_wait_timeout_is_reported(pkg, oracle_mod, synth):
    spec = synth.tiny((16, 14, 20))
    opts = dict(h=6.0, tstop=5.0, seed=1, open_states={"ryr": [0, 3], "p_ryr": [1]})
    sim = pkg.Simulation(spec, opts)
    sim.set_kernel(0)
    sim.advance(5)
    assert sim.lib.csp_test_wait_timeout(sim.h, 1) == 0
    with pytest.raises(pkg.CspError) as e:
        sim.advance(3)
    assert e.value.code == CSP_EDEVICE
    assert "bounded wait timed out" in str(e.value)
    sim.close()

    fresh = pkg.Simulation(spec, opts)
    fresh.set_kernel(0)
    orc = oracle_mod.Oracle(spec, opts)
    fresh.advance(60)
    orc.step(60)
    assert_close(fresh.state(), orc.state(), what="after a reported timeout")
    fresh.close()


def test_hook_needs_the_staged_kernel(pkg, synth):
    sim = pkg.Simulation(synth.tiny((12, 12, 16)), dict(h=6.0, tstop=1.0, seed=1))
    sim.set_kernel(1)
    assert sim.lib.csp_test_wait_timeout(sim.h, 1) == -1
    sim.set_kernel(0)
    assert sim.lib.csp_test_wait_timeout(sim.h, 1) == 0
    assert sim.lib.csp_test_wait_timeout(sim.h, 0) == 0
    flags = sim.advance(10)
    assert not flags.any() and sim.info().step == 10
    sim.close()
