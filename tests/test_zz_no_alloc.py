"""The allocation-free measure product (``cdftb_measure_cross_static_f64``) against the scratch one.

This file is collected last on purpose: the static variant's first call on a device does its
set-up, and the test must pass both alone and after every other test has used the library.
"""

from __future__ import annotations

import pytest
import torch


def _static_cross(pkg, a, b, q, groups):
    lib = pkg._lib
    n = a.shape[-1]
    a2 = a.reshape(groups, -1, n).contiguous()
    b2 = b.reshape(groups, -1, n).contiguous()
    ma, mb = a2.shape[1], b2.shape[1]
    out = torch.empty((groups, ma, mb), dtype=torch.float64, device=a.device)
    lib.call("cdftb_measure_cross_static_f64", lib.ptr(a2), ma, a2.stride(0), lib.ptr(b2), mb, b2.stride(0),
             lib.ptr(q), n, groups, lib.ptr(out), lib.stream_handle(a.device))
    return out


# (rows a, rows b, columns, groups): the 6x6-tile, 4x4-tile and 1x1-tile (row-wise) reductions.
CASES = [(6, 6, 65 ** 3, 1), (12, 12, 65 ** 3, 1), (5, 9, 33 ** 3, 3), (1, 1, 17 ** 3, 40)]


@pytest.mark.gpu
@pytest.mark.parametrize("ma,mb,n,groups", CASES)
def test_static_matches_scratch_two_calls(pkg, cuda, ma, mb, n, groups):
    gen = torch.Generator(device="cpu").manual_seed(ma * 1000 + groups)
    q = torch.rand(n, generator=gen, dtype=torch.float64).to(cuda)
    for call in range(2):
        a = torch.randn(groups, ma, n, generator=gen, dtype=torch.float64).to(cuda)
        b = torch.randn(groups, mb, n, generator=gen, dtype=torch.float64).to(cuda)
        weights = q if call == 0 else None
        want = pkg.measure_cross(a, b, weights, groups)
        got = _static_cross(pkg, a, b, weights, groups)
        torch.cuda.synchronize()
        assert torch.equal(got, want), f"call {call}: max diff {(got - want).abs().max().item()}"


@pytest.mark.gpu
def test_static_rejects_sizes_above_capacity(pkg, cuda):
    lib = pkg._lib
    capacity = lib.library().cdftb_measure_cross_static_capacity_bytes()
    assert capacity == 4 << 20
    ma = mb = 12
    n = 64
    groups = 4000
    need = lib.library().cdftb_measure_cross_scratch_bytes(ma, mb, n, groups)
    assert need > capacity
    a = torch.zeros(groups, ma, n, dtype=torch.float64, device=cuda)
    out = torch.empty(groups, ma, mb, dtype=torch.float64, device=cuda)
    with pytest.raises(lib.CdftbError, match="compiled limit"):
        lib.call("cdftb_measure_cross_static_f64", lib.ptr(a), ma, a.stride(0), lib.ptr(a), mb, a.stride(0), None, n,
                 groups, lib.ptr(out), lib.stream_handle(cuda))
