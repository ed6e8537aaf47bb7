"""The key sort's bounded wait as a tested failure path.

Each digit pass of the onesweep radix sort resolves a tile's offsets by a
look-back over earlier tiles that polls an unpublished tile a bounded number
of times.  With the bound set to 0 a look-back gives up at the first tile it
finds unpublished, which on a multi-tile sort happens in practice on every
pass.  The force pass must then return PT_E_DEVICE naming the sort, stop
before it permutes the particles (a look-back cut short writes in bounds but
not a permutation), and leave the handle usable: with the default bound the
next pass equals a fresh handle's bit for bit.  No wait in this test is left
to run out on its own; the bound only cuts waits short."""
import numpy as np
import pytest

from paratreet_b200 import ics

pytestmark = pytest.mark.gpu


def test_sort_lookback_limit_reports_and_recovers():
    from paratreet_b200._lib import PtError
    from paratreet_b200.gravity import GravitySimulation

    n = 1 << 22  # 1024 tiles of 4096 keys per digit pass
    p = ics.plummer(n, seed=5, soft=1e-3)
    with GravitySimulation(max_particles_per_leaf=32, theta=0.7, precision="fp64") as ref:
        ref.set_particles(p)
        ref.start_down()
        want = ref.accelerations()
    with GravitySimulation(max_particles_per_leaf=32, theta=0.7, precision="fp64") as s:
        s.set_particles(p)
        s.set_sort_spin_limit(0)
        msgs = []
        for _ in range(5):  # each pass of 8 x 1024 tiles x 256 digits races many times
            try:
                s.start_down()
            except PtError as e:
                msgs.append(str(e))
                break
        assert msgs, "no look-back gave up in 5 passes with a spin limit of 0"
        assert "radix sort look-back timed out" in msgs[0]
        s.set_sort_spin_limit()
        s.start_down()
        got = s.accelerations()
    for k in ("ax", "ay", "az", "pot", "pot_full"):
        assert np.array_equal(got[k], want[k]), k
