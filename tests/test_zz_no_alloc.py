"""Allocation-free GETVLXC (flosic_sic_getvlxc_device) against the allocating
entry point (flosic_sic_getvlxc), both through the C ABI.

The device buffers belong to the caller (torch CUDA tensors here); the entry
point keeps its block partial sums in a file-scope device array.  Two calls in
a row must both agree with the allocating path: the scratch is reused without
being cleared, and every output entry must be written (outputs start as NaN).
The device's free memory, read before the first call on a new context and
after each call with torch's allocator idle, must not change: the scratch and
the kernels' code are placed on the device when the context is created.
The per-point potential comes from the same XC kernel in both paths, so it
agrees to rounding; the energies are summed over a different block partition,
so they agree to 1e-12 relative."""
import numpy as np
import pytest

from publicrelease_2020_b200 import sic as S
from publicrelease_2020_b200 import workloads as W

pytestmark = pytest.mark.gpu

CAPACITY = 4_194_304  # points held by the file-scope scratch


def _system(name):
    if name == "water_lda":
        return W.water(seed=0, nrad=16)
    return W.small_synthetic(seed=5, natoms=3, nbasis=24, nmsh=5000, nfo=4)


@pytest.mark.parametrize("name", ["water_lda", "synthetic_pbe"])
def test_getvlxc_device_matches_getvlxc(name):
    import torch

    sysm = _system(name)
    ctx = S.open_system(sysm)
    try:
        _, rho = ctx.coupot_sic(1, 1)  # FO density channels, reference point order
        n = sysm.nmsh
        v_ref, e_ref = ctx.getvlxc(rho)
        v_ref = np.asarray(v_ref).reshape(-1)
        ldr = n + 3  # a leading dimension above NPTS
        r_dev = torch.zeros((10, ldr), dtype=torch.float64, device="cuda")
        r_dev[:, :n] = torch.from_numpy(np.ascontiguousarray(rho))
        w_dev = torch.from_numpy(np.ascontiguousarray(sysm.wmsh, dtype=np.float64)).to("cuda")
        v_devs = [torch.full((2 * n,), float("nan"), dtype=torch.float64, device="cuda") for _ in range(2)]
        torch.cuda.synchronize()
        free = [torch.cuda.mem_get_info()[0]]
        for call in range(2):
            v_dev = v_devs[call]
            e = ctx.getvlxc_device(n, r_dev.data_ptr(), ldr, w_dev.data_ptr(), v_dev.data_ptr())
            torch.cuda.synchronize()
            free.append(torch.cuda.mem_get_info()[0])
            # no device memory taken by the call, the first one on this context included
            assert free[-1] == free[0], (name, call, free)
            v = v_dev.cpu().numpy()
            assert np.all(np.isfinite(v)), (name, call)
            assert np.max(np.abs(v - v_ref)) <= 1e-13 * np.abs(v_ref).max(), (name, call)
            assert np.max(np.abs(e - e_ref)) <= 1e-12 * max(1.0, np.abs(e_ref).max()), (name, call, e, e_ref)
    finally:
        ctx.close()


def test_getvlxc_device_rejects_bad_sizes():
    """Sizes beyond the scratch capacity and a short leading dimension are
    refused on the host before any device work."""
    import torch

    sysm = _system("water_lda")
    ctx = S.open_system(sysm)
    try:
        buf = torch.zeros(16, dtype=torch.float64, device="cuda")
        p = buf.data_ptr()
        with pytest.raises(S.FlosicError) as e:
            ctx.getvlxc_device(CAPACITY + 1, p, CAPACITY + 1, p, p)
        assert e.value.code == 2  # FLOSIC_ERR_CAPACITY
        assert "capacity" in str(e.value)
        with pytest.raises(S.FlosicError) as e:
            ctx.getvlxc_device(8, p, 7, p, p)
        assert e.value.code == 1  # FLOSIC_ERR_ARG
        with pytest.raises(S.FlosicError) as e:
            ctx.getvlxc_device(0, p, 1, p, p)
        assert e.value.code == 1
    finally:
        ctx.close()
