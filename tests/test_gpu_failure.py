"""The failure path of the device waits, exercised without a GPU fault: with a short spin
limit and the copy-timeout test hook (the sweeps neither arrive on their mbarriers nor issue
a copy, so nothing is in flight), every wait on the staging copies runs out, the evaluation fails with
engine_err_cuda and the copy-timeout message, and the device stays usable: the next
evaluation with copies restored matches the FP64 oracle."""
import time

import pytest

import mdcore_b200 as M
import oracle as O
from helpers import force_errors, load_golden

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("form", ["tuned", "plain"])
def test_copy_wait_runs_out_and_the_device_stays_usable(form):
    sysm, ref = load_golden("water_3000.npz")
    o = O.nonbond(sysm, ref["tables"])
    e = M.Engine.from_system(sysm)
    if form == "plain":
        e.tune(0, plain=True)
    e.set_spin(2000)
    e.copytimeout_test(True)
    try:
        t0 = time.time()
        with pytest.raises(M.MdcoreError, match="timed out") as info:
            e.nonbond()
        assert "-21" in str(info.value)                     # engine_err_cuda
        assert time.time() - t0 < 30.0
        assert e.stats().status & 1                          # kStatusCopyTimeout
    finally:
        e.copytimeout_test(False)
        e.set_spin(0)
        M.lib().errs_clear()
    e.nonbond()
    st = e.stats()
    assert st.status == 0 and st.pairs == o["pairs"] and st.excluded == o["excluded"]
    assert force_errors(e.forces(), o["f"])["global_rel"] <= 2e-6
    e.close()
