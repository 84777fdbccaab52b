"""The serving form (nssb_server_*): requests of differing resolution, sigma,
radius and length, admitted by device footprint and rendered in continuous
batches (radius 0) or on pooled engines (radius > 0).

- each result is the same alone and in the mix, bit for bit, and equals the
  per-frame drop-in (BM3D(...).get_frame) on the same clip;
- a small memory budget bounds what is admitted at once, and everything
  still completes;
- a served temporal request agrees with the oracle (>= 60 dB);
- argument errors come back at submission with the filter's messages.
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


def requests(nssb, synth):
    """(clip, kwargs) pairs: YUV420 and Gray, 1-4 frames, radius 0-2, sigma 3-20."""
    out = []
    specs = [(96, 64, 3, 0, 10, True), (128, 72, 2, 1, 5, True), (80, 48, 4, 2, 20, False), (64, 48, 1, 0, 3, False),
             (112, 80, 3, 2, 10, True), (96, 64, 2, 0, 20, True), (72, 56, 4, 1, 10, False), (160, 96, 1, 0, 5, True)]
    for i, (w, h, n, r, s, yuv) in enumerate(specs):
        frames = synth.panning_clip(50 + i, w, h, frames=n, sigma=s, yuv420=yuv)
        clip = nssb.Clip.from_frames(frames, nssb.YUV if yuv else nssb.GRAY, 1 if yuv else 0, 1 if yuv else 0)
        out.append((clip, dict(sigma=s, radius=r, final=1)))
    return out


def planes_equal(a, b):
    return all(np.array_equal(np.asarray(x), np.asarray(y)) for x, y in zip(a, b))


def test_alone_equals_in_the_mix(nssb, synth, dev):
    reqs = requests(nssb, synth)
    srv = nssb.Server()
    alone = []
    for clip, kw in reqs:
        outs, res = srv.wait(srv.submit(clip, **kw))
        assert res.status == 0 and res.frames == clip.vi.num_frames
        alone.append([tuple(p.copy() for p in f) for f in outs])
    tickets = [srv.submit(clip, **kw) for clip, kw in reqs]
    mixed = [srv.wait(t)[0] for t in tickets]
    for a, m in zip(alone, mixed):
        for fa, fm in zip(a, m):
            assert planes_equal(fa, fm)
    st = srv.stats()
    assert st.completed == 2 * len(reqs) and st.failed == 0
    assert st.ticks >= 1 and st.temporal_frames > 0
    assert st.engines_reused > 0  # the second round reuses the first round's engines
    srv.close()
    # the per-frame drop-in on the same clips gives the same frames
    for (clip, kw), a in zip(reqs, alone):
        node = nssb.BM3D(clip, **kw)
        for n in range(clip.vi.num_frames):
            assert planes_equal(node.get_frame(n), a[n])
        node.close()


def test_budget_bounds_admission(nssb, synth, dev):
    reqs = requests(nssb, synth)
    srv = nssb.Server(memory_budget_mb=8, workers=2)
    tickets = [srv.submit(clip, **kw) for clip, kw in reqs for _ in range(2)]
    for t in tickets:
        _, res = srv.wait(t)
        assert res.status == 0 and res.latency_ms >= res.queue_ms >= 0
    st = srv.stats()
    assert st.completed == len(tickets)
    budget = 8 << 20
    assert st.budget_bytes == budget
    # oversized requests run alone; otherwise the reservations stay inside the budget
    assert st.peak_reserved_bytes <= budget or st.peak_active == 1
    srv.close()


def test_served_temporal_vs_oracle(nssb, oracle, synth, dev):
    frames = [f[0] for f in synth.panning_clip(77, 64, 48, frames=4, sigma=12, yuv420=False)]
    clip = nssb.Clip.from_frames([(f,) for f in frames], nssb.GRAY)
    srv = nssb.Server()
    outs, res = srv.wait(srv.submit(clip, sigma=12, radius=1, final=1))
    srv.close()
    st = oracle.stage(oracle.effective_sigma(12.0))
    basic = oracle.bm3d_clip_plane(frames, st, 1)
    want = oracle.bm3d_clip_plane(frames, st, 1, ref_frames=basic)
    for o, w in zip(outs, want):
        assert oracle.psnr(o[0], w) >= MIN_PSNR


def test_device_request(nssb, synth, dev):
    frames = synth.panning_clip(88, 96, 64, frames=3, sigma=10)
    dclip = nssb.Clip.from_frames([tuple(torch.from_numpy(p).to(dev) for p in f) for f in frames], nssb.YUV, 1, 1)
    hclip = nssb.Clip.from_frames(frames, nssb.YUV, 1, 1)
    srv = nssb.Server()
    for r in (0, 1):
        d, _ = srv.wait(srv.submit(dclip, sigma=10, radius=r, final=1))
        h, _ = srv.wait(srv.submit(hclip, sigma=10, radius=r, final=1))
        for fd, fh in zip(d, h):
            assert planes_equal([p.cpu().numpy() for p in fd], fh)
    srv.close()


def test_submit_errors(nssb, synth, dev):
    clip = nssb.Clip.from_frames([(synth.gray_frame(1, 64, 48)[0],)], nssb.GRAY)
    srv = nssb.Server()
    with pytest.raises(nssb.Error, match="nss_cuda.BM3D: radius must be"):
        srv.submit(clip, radius=99)
    with pytest.raises(nssb.Error, match="legacy"):
        srv.submit(clip, radius=1, temporal_mode="legacy")
    srv.close()
