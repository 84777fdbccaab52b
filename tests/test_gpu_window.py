"""The opt-in Kaiser aggregation window (nssb_bm3d_set_window).

The reference's BM3D weights every pixel of a group's patches by one flat
per-group weight; it has no windowed mode (only its BM4D windows). This
build's opt-in mode multiplies each patch pixel's weight by the block's
separable Kaiser window, in num and den alike. It is checked against the
oracle's windowed pass (oracle/bm3d_oracle.c om_bm3d_plane_window, the same
matcher and group filter with the window in the aggregation), not against
the reference. beta = 0 must give the default output bit for bit.
"""
import importlib

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

MIN_PSNR = 60.0


@pytest.fixture(scope="module")
def dev():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda:0")


@pytest.fixture(scope="module")
def synth():
    return importlib.import_module("vapoursynth-nssfactory_b200.synth")


def gray_node(nssb, plane, **kw):
    return nssb.BM3D(nssb.Clip.from_frames([(plane,)], nssb.GRAY), **kw)


@pytest.mark.parametrize("block,group,step,final", [(8, 8, 8, 0), (8, 16, 4, 1), (8, 32, 3, 0), (8, 4, 8, 1),
                                                    (4, 8, 4, 0), (16, 8, 8, 1)])
@pytest.mark.parametrize("beta", [2.0, 6.0])
def test_window_vs_oracle(nssb, oracle, dev, synth, block, group, step, final, beta):
    noisy, _ = synth.gray_frame(31 + block, 112, 88, sigma=15)
    node = gray_node(nssb, noisy, sigma=15, block_size=block, group_size=group, block_step=step, final=final)
    node.set_window(beta)
    got = node.get_frame(0)[0]
    node.close()
    st = oracle.stage(oracle.effective_sigma(15.0), block=block, group=group, step=step)
    win = oracle.kaiser_window(block, beta)
    if final:
        basic = oracle.bm3d_plane_window(noisy, st, win)
        want = oracle.bm3d_plane_window(noisy, st, win, ref=basic)
    else:
        want = oracle.bm3d_plane_window(noisy, st, win)
    p = oracle.psnr(got, want)
    print(f"block {block} group {group} step {step} final {final} beta {beta}: {p:.1f} dB vs the windowed oracle")
    assert p >= MIN_PSNR
    # and it is a different estimate from the flat weights
    flat = oracle.bm3d_plane(noisy, st) if not final else oracle.bm3d_plane_two_stage(noisy, st, st)[0]
    assert not np.array_equal(got, flat)


def test_beta_zero_is_the_default_bit_for_bit(nssb, dev, synth):
    frames = synth.yuv420_clip(8, 160, 96, frames=1, sigma=10)
    node = nssb.BM3D(nssb.Clip.from_frames(frames, nssb.YUV, 1, 1), sigma=10, final=1)
    want = [np.array(p) for p in node.get_frame(0)]
    node.set_window(3.0)
    windowed = [np.array(p) for p in node.get_frame(0)]
    node.set_window(0.0)
    got = [np.array(p) for p in node.get_frame(0)]
    node.close()
    assert all(np.array_equal(a, b) for a, b in zip(got, want))
    assert not all(np.array_equal(a, b) for a, b in zip(windowed, want))


def test_window_rejected_where_it_does_not_apply(nssb, dev, synth):
    clip = [(synth.gray_frame(s, 64, 48, sigma=10)[0],) for s in range(3)]
    tnode = nssb.BM3D(nssb.Clip.from_frames(clip, nssb.GRAY), sigma=10, radius=1)
    with pytest.raises(nssb.Error, match="radius-0"):
        tnode.set_window(2.0)
    tnode.close()
    node = nssb.BM3D(nssb.Clip.from_frames(clip, nssb.GRAY), sigma=10)
    with pytest.raises(nssb.Error, match="finite and non-negative"):
        node.set_window(-1.0)
    node.set_window(2.0)
    batch = nssb.Batch()
    with pytest.raises(nssb.Error, match="Kaiser window"):
        batch.run([(node, 0)])
    batch.close()
    node.close()
