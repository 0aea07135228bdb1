"""nadia_shrinkwrap_noalloc_f32: the shrinkwrap for callers that cannot
allocate device memory when they update a support (concurrent streams that a
cudaMalloc would stall, or device memory already committed to a budget or
another allocator).  It works on the caller's device buffers and keeps its
working memory in an array built into the library.

Checked through the C ABI against the existing entry point
(nadia_apply_shrinkwrap, read back with nadia_get_support) on calls in a row
that reuse the same caller buffers and the same built-in array, with the
tolerance of the other shrinkwrap tests: at most 0.1% of pixels may differ by
more than 1e-5 (pixels that sit on the threshold can flip).  Grids the FP32
form has tiles for are compared with an FP32 handle; ragged grids (partial
32x32 tiles at the edges, nx > ny and nx < ny, so both branches of the
reference's `j < nx` threshold bound) with an FP64 handle.  Device memory is
checked unchanged across calls after the first (which may load the module
that holds the array)."""
import numpy as np
import pytest

import pynadia
from pynadia import synth

pytestmark = pytest.mark.gpu


def handle_support(esw, sigma, threshold, precision):
    nx, ny = esw.shape
    s = pynadia.Solver("planar", nx, ny, precision=precision)
    s.set_exit_surface_wave(esw)
    s.apply_shrinkwrap(sigma, threshold)
    return s.get_support()


def estimate(nx, ny, seed):
    c = synth.PlanarCase(nx, min(nx, ny) * 0.16, 2, 1e8, seed=seed,
                         support_side=int(min(nx, ny) * 0.4), ny=ny)
    g = np.random.default_rng(seed)
    noise = 0.05 * (g.standard_normal((nx, ny)) + 1j * g.standard_normal((nx, ny)))
    return (c.obj + noise).astype(np.complex64)


def close(got, ref):
    # nx > ny: the reference's threshold loop zeroes every row after the
    # first and the support becomes 0/0 (NaN) in every form
    assert np.array_equal(np.isnan(got), np.isnan(ref))
    both = np.isnan(got) & np.isnan(ref)
    got, ref = np.where(both, 0, got), np.where(both, 0, ref)
    assert np.mean(np.abs(got - ref) > 1e-5) < 1e-3
    assert np.abs(got - ref).max() <= 1.0


# (nx, ny, sigma, threshold, seed, precision of the handle compared with)
CASES = ((512, 512, 1.5, 0.1, 21, pynadia.FP32), (256, 512, 2.0, 0.2, 22, pynadia.FP32),
         (328, 200, 1.5, 0.1, 23, pynadia.FP64), (200, 328, 1.5, 0.15, 24, pynadia.FP64),
         (72, 40, 1.0, 0.1, 25, pynadia.FP64), (40, 72, 1.5, 0.1, 26, pynadia.FP64))


def test_calls_in_a_row_match_the_handle_shrinkwrap():
    import torch

    dev = torch.device("cuda", 0)
    esw_d = torch.empty(512 * 512 * 2, dtype=torch.float32, device=dev)
    sup_d = torch.empty(512 * 512, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    free_after_first = None
    for k, (nx, ny, sigma, t, seed, prec) in enumerate(CASES):
        esw = estimate(nx, ny, seed)
        flat = np.stack([esw.real, esw.imag], axis=-1).reshape(-1)
        esw_d[: flat.size].copy_(torch.from_numpy(flat))
        torch.cuda.synchronize(dev)
        pynadia.shrinkwrap_noalloc_f32(esw_d.data_ptr(), sup_d.data_ptr(), nx, ny, sigma, t,
                                       stream)
        torch.cuda.synchronize(dev)
        free = torch.cuda.mem_get_info(dev)[0]
        if free_after_first is None:
            free_after_first = free
        else:
            # nothing allocated on the device by this call
            assert free == free_after_first, (k, free, free_after_first)
        got = sup_d[: nx * ny].cpu().numpy().astype(np.float64).reshape(nx, ny)
        ref = handle_support(esw.astype(np.complex128), sigma, t, prec)
        close(got, ref)
        torch.cuda.synchronize(dev)
        free_after_first = torch.cuda.mem_get_info(dev)[0]


def test_rejects_grids_beyond_its_array():
    # checked on the host before any work is queued
    with pytest.raises(pynadia.NadiaError) as e:
        pynadia.shrinkwrap_noalloc_f32(16, 16, 4128, 4128)
    assert e.value.code == 1 and "4096" in str(e.value)
