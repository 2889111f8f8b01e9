"""fn_observe_noalloc: the observables reduction for callers that cannot
allocate device memory at the point of the call (a loop or callback that must
not synchronise the device, as cudaMalloc and cudaFree may, or an application
whose device memory all belongs to its own allocator).  It must give fn_observe's
results, call after call, with its scratch in the library's static array and
without any device allocation.  Collected last so that a failure here leaves
every other test already run."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_observe_noalloc_matches_observe():
    import torch

    from fibrenet_b200 import generate as g
    from fibrenet_b200.native import Simulation

    m = g.tensile_network(seed=5, fibres=40, beads=20, box=(40.0, 30.0, 8.0), z_range=(1.0, 7.0),
                          clamp_lo=2.0, clamp_hi=38.0, pull=0.5, cell=2.5,
                          fail_mu=np.log(0.5), fail_sigma=0.4)
    with Simulation(m, list_capacity=64) as s:
        outs = [torch.full((5,), -1.0, dtype=torch.float64, device="cuda") for _ in range(2)]
        torch.cuda.synchronize()
        s.observe_noalloc(outs[0].data_ptr(), 0, reaction_type=2)  # first call: set-up
        s.sync()
        broke_seen = False
        for round_ in range(2):
            s.step(60)
            want = s.observe(0, reaction_type=2)
            for out in outs:
                out.fill_(-1.0)
            torch.cuda.synchronize()
            free_before = torch.cuda.mem_get_info()[0]
            for out in outs:  # two calls in a row, sharing the static scratch
                s.observe_noalloc(out.data_ptr(), 0, reaction_type=2)
            s.sync()
            assert torch.cuda.mem_get_info()[0] == free_before
            for out in outs:
                got = out.cpu().numpy()
                np.testing.assert_array_equal(got[:3], want["reaction"])  # same partial sums
                assert int(got[3]) == want["broken"]
                assert int(got[4]) == want["angles_dead"]
            broke_seen |= want["broken"] > 0
        assert broke_seen


def test_observe_noalloc_large_network_bit_identical():
    """A 375,000-bead network: its reduction needs more than 1,024 blocks'
    worth of items, so both entry points loop inside their 1,024 blocks and
    must still agree bit for bit, call after call."""
    import torch

    from fibrenet_b200 import generate as g
    from fibrenet_b200.native import Simulation

    F = 7500
    side = 1000.0 * np.sqrt(F / 20000.0)
    m = g.tensile_network(seed=9, fibres=F, box=(side, side, 20.0), clamp_lo=2.0, clamp_hi=side - 2.0,
                          pull=0.5, fail_mu=np.log(0.5), fail_sigma=0.4)
    assert m.n_beads > 1024 * 256
    with Simulation(m, list_capacity=64) as s:
        out = torch.full((5,), -1.0, dtype=torch.float64, device="cuda")
        for _ in range(2):
            s.step(40)
            want = s.observe(0, reaction_type=2)
            torch.cuda.synchronize()
            free_before = torch.cuda.mem_get_info()[0]
            s.observe_noalloc(out.data_ptr(), 0, reaction_type=2)
            s.observe_noalloc(out.data_ptr(), 0, reaction_type=2)
            s.sync()
            assert torch.cuda.mem_get_info()[0] == free_before
            got = out.cpu().numpy()
            np.testing.assert_array_equal(got[:3], want["reaction"])
            assert int(got[3]) == want["broken"]
            assert int(got[4]) == want["angles_dead"]
        assert want["broken"] > 0
