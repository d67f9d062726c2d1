"""thx_rhs_host: right-hand sides of states held in host memory, with the
transfers of neighbouring states overlapping the kernels.  Each rate must
equal the device-resident Mult of the same state bit for bit, in FP64 and in
FP32-mixed mode, whatever the number of states, and the call must be
ordered on the given stream."""
import numpy as np
import pytest

import theseus_b200 as T
from _helpers import box, smooth_state


def test_rhs_host_rejects_bad_arguments():
    lib = T.library()
    from theseus_b200._abi import THX_ERR_INVALID_ARGUMENT
    assert lib.thx_rhs_host(None, 1, None, None, None) == THX_ERR_INVALID_ARGUMENT


@pytest.mark.gpu
@pytest.mark.parametrize("precision,n", [("fp64", 1), ("fp64", 5), ("fp32", 4)])
def test_rhs_host_equals_device_mult(cuda, precision, n):
    import torch
    m = box(3, 3, (4, 3, 3))
    op = T.NSOperator(m, numerical_flux="ranocha", surface_flux="hll", mu=0.01, Pr=0.72, precision=precision)
    states = [torch.as_tensor(smooth_state(m, seed=s), dtype=torch.float64).pin_memory() for s in range(n)]
    rates = [torch.full_like(x, np.nan).pin_memory() for x in states]
    s = torch.cuda.Stream()
    op.mult_host(states, rates, stream=s)
    s.synchronize()
    for x, r in zip(states, rates):
        ud = x.to("cuda").to(op.dtype)
        du = torch.empty_like(ud)
        op.Mult(ud, du)
        torch.cuda.synchronize()
        assert torch.equal(r, du.to(torch.float64).cpu())
    assert op.read_status() == 0


@pytest.mark.gpu
def test_rhs_host_is_stream_ordered(cuda):
    """An event recorded on the call's stream after it completes only once
    every rate has been copied out."""
    import torch
    m = box(2, 3, (6, 5))
    op = T.EulerOperator(m, numerical_flux="chandrashekar", surface_flux="llf")
    x = torch.as_tensor(smooth_state(m, seed=1), dtype=torch.float64).pin_memory()
    r = torch.zeros_like(x).pin_memory()
    s = torch.cuda.Stream()
    op.mult_host([x, x, x], [r, r, r], stream=s)
    marker = torch.cuda.Event()
    marker.record(s)
    marker.synchronize()
    ud = x.to("cuda")
    du = torch.empty_like(ud)
    op.Mult(ud, du)
    torch.cuda.synchronize()
    assert torch.equal(r, du.cpu())
