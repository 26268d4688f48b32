"""Failure path of the stage kernels: a bounded wait that runs out is reported, not hung on.

Every TMA wait in the stage kernels gives up after 200 ms of global time, records the error in
the device scalars, drains its own copies (bounded) and returns; CTAs that start later leave at
once, and the step returns R3D_ECUDA with the reason.  The test makes the waits run out with the
r3d_gpu_debug_tma_extra hook (each transaction then expects more bytes than its copies carry:
the data lands, the barrier never completes) - no fault, no trap, no unbounded wait - and checks
the status, the time it takes and that the same context then runs a correct step.
"""
import time

import numpy as np
import pytest

import r3d_b200 as R


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "fp32bulk"])
def test_bounded_tma_wait_reports_error_and_context_recovers(precision):
    p = R.parse(["--npx", "64", "--npy", "32", "--npz", "32", "--seed", "3", "--precision", precision])
    st = R.HostState.setup(p)
    ref = st.copy()
    with R.GpuSim(p) as sim:
        sim.upload(ref)
        sim.step()
        sim.download(ref)
    with R.GpuSim(p) as sim:
        sim.upload(st)
        sim.debug_tma_extra(16)
        t0 = time.time()
        with pytest.raises(R.R3dError) as e:
            sim.step()
        took = time.time() - t0
        assert e.value.code == R.R3D_ECUDA and "bounded TMA wait" in str(e.value)
        assert took < 30.0, took
        # the context is still usable: switch the hook off, upload again, step
        sim.debug_tma_extra(0)
        got = R.HostState.setup(p)
        sim.upload(got)
        sim.step()
        sim.download(got)
    for n in ref.fields:
        assert np.array_equal(ref.fields[n], got.fields[n]), n
