"""nadia_shrinkwrap_noalloc_f32: the shrinkwrap for callers that cannot
allocate device memory when they update a support (concurrent streams that a
cudaMalloc would stall, or device memory already committed to a budget or
another allocator).  It works on the caller's device buffers and keeps its
working memory in an array built into the library.

Checked through the C ABI against the existing entry point
(nadia_apply_shrinkwrap on an FP32 handle, read back with nadia_get_support)
on two calls in a row that reuse the same caller buffers and the same
built-in array, with the tolerance of the other shrinkwrap tests: at most
0.1% of pixels may differ by more than 1e-5 (pixels that sit on the
threshold can flip)."""
import numpy as np
import pytest

import pynadia
from pynadia import synth

pytestmark = pytest.mark.gpu


def handle_support(esw, sigma, threshold):
    nx, ny = esw.shape
    s = pynadia.Solver("planar", nx, ny, precision=pynadia.FP32)
    s.set_exit_surface_wave(esw)
    s.apply_shrinkwrap(sigma, threshold)
    return s.get_support()


def estimate(nx, ny, seed):
    c = synth.PlanarCase(nx, nx * 0.16, 2, 1e8, seed=seed, support_side=int(nx * 0.4), ny=ny)
    g = np.random.default_rng(seed)
    noise = 0.05 * (g.standard_normal((nx, ny)) + 1j * g.standard_normal((nx, ny)))
    return (c.obj + noise).astype(np.complex64)


def test_two_calls_match_the_handle_shrinkwrap():
    import torch

    dev = torch.device("cuda", 0)
    esw_d = torch.empty(512 * 512 * 2, dtype=torch.float32, device=dev)
    sup_d = torch.empty(512 * 512, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    for (nx, ny, sigma, t, seed) in ((512, 512, 1.5, 0.1, 21), (256, 512, 2.0, 0.2, 22)):
        esw = estimate(nx, ny, seed)
        flat = np.stack([esw.real, esw.imag], axis=-1).reshape(-1)
        esw_d[: flat.size].copy_(torch.from_numpy(flat))
        pynadia.shrinkwrap_noalloc_f32(esw_d.data_ptr(), sup_d.data_ptr(), nx, ny, sigma, t,
                                       stream)
        torch.cuda.synchronize(dev)
        got = sup_d[: nx * ny].cpu().numpy().astype(np.float64).reshape(nx, ny)
        ref = handle_support(esw.astype(np.complex128), sigma, t)
        assert np.mean(np.abs(got - ref) > 1e-5) < 1e-3
        assert np.abs(got - ref).max() <= 1.0


def test_rejects_grids_beyond_its_array():
    # checked on the host before any work is queued
    with pytest.raises(pynadia.NadiaError) as e:
        pynadia.shrinkwrap_noalloc_f32(16, 16, 4128, 4128)
    assert e.value.code == 1 and "4096" in str(e.value)
