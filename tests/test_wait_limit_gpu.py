"""The error path of the mixed-precision tensor-core Coulomb kernel, exercised
without a GPU fault: every wait between its roles (producers, MMA issue,
epilogue) has a poll limit, and flosic_sic_set_wait_limit lowers it so that
the waits give up.  The kernel then stops its roles, drains its own copies and
tensor-core operations, frees its tensor memory and returns; the cycle reports
FLOSIC_ERR_CUDA.  With the default limit restored, the same context runs the
next cycle to the same results bit for bit as before the failure."""
import numpy as np
import pytest

from publicrelease_2020_b200 import sic as S
from publicrelease_2020_b200 import workloads as W

pytestmark = pytest.mark.gpu

FLOSIC_ERR_CUDA = 7


def test_short_wait_limit_fails_cleanly_and_context_recovers():
    import torch

    sysm = W.small_synthetic(seed=5, natoms=3, nbasis=24, nmsh=5000, nfo=4)
    ctx = S.open_system(sysm)
    try:
        ctx.set_precision("mixed")
        ref = ctx.cycle()
        ctx.set_orbitals(sysm.psi, sysm.nwfs, sysm.fods)  # drop the cached potentials
        ctx.set_wait_limit(1)
        with pytest.raises(S.FlosicError) as e:
            ctx.cycle()
        assert e.value.code == FLOSIC_ERR_CUDA
        assert "limit" in str(e.value)
        torch.cuda.synchronize()  # the device is still usable
        ctx.set_wait_limit(0)
        again = ctx.cycle()
        assert again["esic"] == ref["esic"]
        for k in ("results", "sic", "debdax"):
            assert np.array_equal(again[k], ref[k]), k
    finally:
        ctx.close()
