"""Host-resident batches (sht_forward_host / sht_inverse_host /
sht_round_trip_host): chunked copies pipelined with the transforms give the
same numbers as the device calls, for any chunk size, plane count and
precision, from page-locked or pageable host memory."""
from __future__ import annotations

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", ["float64", "float32", "split16"])
@pytest.mark.parametrize("planes,chunk", [(7, 0), (7, 3), (6, 1), (12, 12)])
def test_host_calls_match_device_calls(precision, planes, chunk):
    from b200sht import SphericalHarmonicTransform
    from b200sht.synthetic import red_spectrum

    t = SphericalHarmonicTransform.create(21, precision=precision)
    coeff = torch.as_tensor(red_spectrum(21, planes)).to(t.backend.complex_dtype)
    grid_dev = t.inverse(coeff.to(t.backend.device))
    grid_host = grid_dev.cpu().pin_memory()
    # device reference
    spec_dev = t.forward(grid_dev).cpu()
    rt_dev = t.inverse(t.forward(grid_dev)).cpu()
    inv_dev = grid_dev.cpu()
    torch.cuda.synchronize()
    spec = t.forward_host(grid_host, chunk=chunk)
    assert spec.device.type == "cpu" and spec.is_pinned()
    assert torch.equal(spec, spec_dev)
    assert torch.equal(t.inverse_host(coeff, chunk=chunk), inv_dev)
    out = torch.empty_like(grid_host).pin_memory()
    got = t.round_trip_host(grid_host, out=out, chunk=chunk)
    assert got.data_ptr() == out.data_ptr()
    assert torch.equal(got, rt_dev)
    # pageable input: same result, no overlap
    assert torch.equal(t.round_trip_host(grid_host.clone(), chunk=chunk), rt_dev)
    t.check_device()


def test_host_call_errors():
    from b200sht import SphericalHarmonicTransform

    t = SphericalHarmonicTransform.create(9, precision="float32")
    with pytest.raises(ValueError, match="host"):
        t.forward_host(torch.zeros((2, *t.grid.shape), device="cuda"))
    with pytest.raises(ValueError, match="trailing shape"):
        t.forward_host(torch.zeros((2, 3, 3)))
    with pytest.raises(ValueError, match="out must be"):
        t.round_trip_host(torch.zeros((2, *t.grid.shape)), out=torch.zeros((3, *t.grid.shape)))
    with pytest.raises(ValueError, match="chunk"):
        t.forward_host(torch.zeros((2, *t.grid.shape)), chunk=-1)


def test_round_trip_host_at_t511_meets_the_bar():
    from b200sht import SphericalHarmonicTransform
    from b200sht.synthetic import red_spectrum

    f64 = SphericalHarmonicTransform.create(511, precision="float64")
    t = SphericalHarmonicTransform.create(511, precision="split16")
    coeff = red_spectrum(511, 4)
    grid = f64.inverse(coeff)
    ref = f64.inverse(f64.forward(grid)).cpu().numpy()
    got = t.round_trip_host(grid.float().cpu().pin_memory(), chunk=2).numpy()
    assert np.max(np.abs(got - ref)) / np.max(np.abs(ref)) < 2e-6
    t.check_device()


@pytest.mark.parametrize("precision", ["float32", "split16"])
@pytest.mark.parametrize("planes", [57, 200])
def test_default_chunk_schedule_on_a_register_fft_grid(precision, planes):
    """The default schedule (chunks ramped 2, 4, ... at both ends, an odd
    chunk where the plane count is odd) on a grid the register-resident FFTs
    serve (T62 on 94 x 192): the same numbers as the whole-batch device
    calls."""
    from b200sht import SphericalHarmonicTransform
    from b200sht.synthetic import red_spectrum

    t = SphericalHarmonicTransform.create(62, nlat=94, nlon=192, dealias_factor=1.49,
                                          precision=precision)
    coeff = torch.as_tensor(red_spectrum(62, planes, seed=3)).to(t.backend.complex_dtype)
    grid_dev = t.inverse(coeff.to(t.backend.device))
    rt_dev = t.inverse(t.forward(grid_dev)).cpu()
    got = t.round_trip_host(grid_dev.cpu().pin_memory())
    assert torch.equal(got, rt_dev)
    assert torch.equal(t.forward_host(grid_dev.cpu().pin_memory()), t.forward(grid_dev).cpu())
    t.check_device()
