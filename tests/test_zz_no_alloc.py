"""The no-allocation stage entry point against the allocating one.

nssb_bm3d_plane_stage_noalloc serves callers that cannot allocate device
memory while they run (a host whose device memory belongs to its own frame
pool, or a loop where cudaMalloc/cudaFree would stall the device). It must
give what nssb_bm3d_plane_stage gives on the same planes, call after call,
although every call reuses one fixed device array left over from the last
call. The buffers below are the test's own; the library allocates nothing.

Both entry points run the same matching, group and finish kernels on the same
planes, and the sums are exact integers, so the outputs must be equal bit for
bit: a sum left over from the previous call would show as a difference.
"""
import importlib

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu



@pytest.fixture(scope="module")
def dev():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda:0")


def run_stage(nssb, fn, src, ref, sigma, block, group, step, rng_):
    h, w = src.shape
    out = torch.empty_like(src)
    nssb.check(getattr(nssb.lib(), fn)(src.data_ptr(), ref.data_ptr() if ref is not None else None, out.data_ptr(),
                                       w, w, h, sigma, block, group, step, rng_, None))
    torch.cuda.synchronize()
    return out.cpu().numpy()


def device_free_bytes():
    torch.cuda.synchronize()
    return torch.cuda.mem_get_info()[0]


@pytest.mark.parametrize("block,group,step,rng_", [(8, 8, 8, 9), (4, 16, 3, 6)])
def test_noalloc_matches_allocating_stage_twice(nssb, dev, block, group, step, rng_):
    synth = importlib.import_module("vapoursynth-nssfactory_b200.synth")
    sigma = (10.0 / 255.0) * 0.75
    # two calls in a row on different planes: the second must not see the first's sums
    for seed, (w, h) in ((11, (256, 192)), (12, (200, 136))):
        noisy, _ = synth.gray_frame(seed, w, h, sigma=10)
        src = torch.from_numpy(noisy).to(dev)
        basic_ref = run_stage(nssb, "nssb_bm3d_plane_stage", src, None, sigma, block, group, step, rng_)
        basic_new = run_stage(nssb, "nssb_bm3d_plane_stage_noalloc", src, None, sigma, block, group, step, rng_)
        assert np.array_equal(basic_new, basic_ref)
        ref = torch.from_numpy(basic_ref).to(dev)
        final_ref = run_stage(nssb, "nssb_bm3d_plane_stage", src, ref, sigma, block, group, step, rng_)
        final_new = run_stage(nssb, "nssb_bm3d_plane_stage_noalloc", src, ref, sigma, block, group, step, rng_)
        assert np.array_equal(final_new, final_ref)


def test_noalloc_allocates_nothing(nssb, dev):
    """After a first call has loaded the kernels, further calls leave the
    device's free memory exactly as it was (no library pool growth, no
    cudaMalloc); the output buffers are allocated before the measurement."""
    synth = importlib.import_module("vapoursynth-nssfactory_b200.synth")
    sigma = (10.0 / 255.0) * 0.75
    noisy, _ = synth.gray_frame(21, 320, 240, sigma=10)
    src = torch.from_numpy(noisy).to(dev)
    outs = [torch.empty_like(src) for _ in range(4)]
    lib = nssb.lib()

    def call(out, ref):
        nssb.check(lib.nssb_bm3d_plane_stage_noalloc(src.data_ptr(), ref.data_ptr() if ref is not None else None,
                                                     out.data_ptr(), 320, 320, 240, sigma, 8, 8, 8, 9, None))

    call(outs[0], None)
    call(outs[1], outs[0])
    before = device_free_bytes()
    call(outs[2], None)
    call(outs[3], outs[2])
    after = device_free_bytes()
    assert after == before, (before, after)
    assert torch.equal(outs[2], outs[0]) and torch.equal(outs[3], outs[1])


def test_noalloc_rejects_oversized_planes(nssb, dev):
    w, h = 2048, 1100  # 2,252,800 elements: beyond the fixed scratch
    src = torch.zeros((h, w), dtype=torch.float32, device=dev)
    out = torch.empty_like(src)
    rc = nssb.lib().nssb_bm3d_plane_stage_noalloc(src.data_ptr(), None, out.data_ptr(), w, w, h, 0.01, 8, 8, 8, 9,
                                                  None)
    assert rc == nssb.ERR_STATE
    assert "at most 2097152 plane elements" in nssb.last_error()
