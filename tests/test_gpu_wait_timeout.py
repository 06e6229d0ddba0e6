"""Failure detection on the GPU without a fault: the tcgen05 kernel's waits are
bounded; with the bound set to 1 ns the first wait that finds its barrier
not yet complete runs out, the kernel stops, releases its tensor memory and the
call reports DD_ERR_TIMEOUT.  The same context then computes a correct
histogram."""
import pytest

import coding_reliability_b200 as dd

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("epilogue", ["paired", "single"])
def test_wait_timeout_is_reported_and_the_context_recovers(epilogue):
    """Both tcgen05 epilogues: the paired one also waits at its epilogue-wide
    barriers around the table flushes, which give up the same way."""
    q = dd.Request(dd.CODE_AN, dd.MODE_EXHAUSTIVE, 58659, 18, kernel=dd.KERNEL_MMA)
    with dd.Context(0) as ctx:
        e = dd.MMA_EPILOGUE_PAIRED if epilogue == "paired" else dd.MMA_EPILOGUE_SINGLE
        ctx.set_mma_epilogue(e)
        good = ctx.histogram(q)
        assert good.kernel_used == dd.KERNEL_MMA and good.mma_epilogue == e
        ctx.set_wait_timeout(1)
        for _ in range(2):
            with pytest.raises(dd.DDError) as e:
                ctx.histogram(q)
            assert e.value.status == 7 and "timed out" in str(e.value)
        ctx.set_wait_timeout(0)
        again = ctx.histogram(q)
        assert again.counts == good.counts and again.raw == good.raw
        popc = ctx.histogram(dd.Request(dd.CODE_AN, dd.MODE_EXHAUSTIVE, 58659, 18, kernel=dd.KERNEL_POPC))
        assert popc.counts == good.counts
