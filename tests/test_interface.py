"""Creation-time interface of nss_cuda.BM3D through the C ABI (no device needed).

The 900 BM3D cases of the reference's interface golden (CPU plugin, "nss."
prefix) are checked the way the reference checks its CUDA plugin
(tests/test_plugin_interface.py with --namespace nss_cuda --backend-args
device_id,num_streams --default-temporal rolling --rolling-cache adaptive):
the prefix becomes "nss_cuda.", a probe that leaves temporal_mode unset runs
in legacy mode, and the CPU's "use only one of rolling_cache_limit and
rolling_cache_chunks" error must instead be accepted.
"""
import json
from pathlib import Path

import pytest

GOLDEN = Path(__file__).resolve().parent / "golden" / "bm3d_interface_cases.json"
CASES = json.loads(GOLDEN.read_text())
FORMAT_NAMES = {"GRAYS": "GrayS", "RGBS": "RGBS", "YUV420PS": "YUV420PS"}


def clip_info(nssb, fmt):
    c = CASES["clip"]
    return nssb.format_info(fmt, c["width"], c["height"], c["frames"])


def run(nssb, fmt, kwargs):
    vi = clip_info(nssb, fmt)
    try:
        out = nssb.check_args(vi, None, **kwargs)
    except nssb.Error as e:
        return {"error": str(e)}
    return {"ok": {"format": FORMAT_NAMES[fmt], "frames": out.num_frames, "height": out.height, "width": out.width}}


def expected(case):
    exp = case["expect"]
    if "error" in exp:
        return {"error": exp["error"].replace("nss.BM3D:", "nss_cuda.BM3D:", 1)}
    return exp


def test_signature_matches_reference(nssb):
    assert nssb.SIGNATURE == CASES["signature"] + "device_id:int:opt;num_streams:int:opt;"


@pytest.mark.parametrize("case", CASES["cases"], ids=[c["key"] for c in CASES["cases"]])
def test_golden_case(nssb, case):
    kwargs = dict(case["kwargs"])
    if "temporal_mode" not in kwargs:
        kwargs["temporal_mode"] = "legacy"
    got = run(nssb, case["format"], kwargs)
    want = expected(case)
    if "use only one of rolling_cache_limit and rolling_cache_chunks" in want.get("error", ""):
        assert "ok" in got, got
        return
    if want.get("error", "").startswith("nss: ") and "error" in got:
        assert got["error"] in (want["error"], "nss_cuda" + want["error"][3:])
        return
    assert got == want


def test_default_temporal_mode_is_rolling(nssb):
    out = nssb.check_args(clip_info(nssb, "GRAYS"), None, radius=1)
    assert out.height == 40


def test_cache_limit_below_chunks_rejected(nssb):
    with pytest.raises(nssb.Error, match="rolling_cache_limit must be at least rolling_cache_chunks"):
        nssb.check_args(clip_info(nssb, "GRAYS"), None, radius=1, temporal_mode="rolling", rolling_cache_chunks=4,
                        rolling_cache_limit=2)


def test_ref_rules(nssb):
    vi = clip_info(nssb, "GRAYS")
    other = nssb.format_info("GRAYS", 40, 40, 4)
    with pytest.raises(nssb.Error, match="^nss_cuda.BM3D: ref must match clip$"):
        nssb.check_args(vi, other)
    with pytest.raises(nssb.Error, match="^nss_cuda.BM3D: use only one of final and ref$"):
        nssb.check_args(vi, vi, final=1)
    assert nssb.check_args(vi, vi).height == 40


def test_format_rules(nssb):
    bad = nssb.video_info(nssb.GRAY, 48, 40, 4)
    bad.bits_per_sample = 16
    bad.sample_float = 0
    with pytest.raises(nssb.Error, match="constant Gray/YUV/RGB 32-bit float required"):
        nssb.check_args(bad)
    yuv444 = nssb.format_info("YUV444PS", 48, 40, 4)
    assert nssb.check_args(yuv444, None, chroma=1).width == 48


def test_backend_args(nssb):
    vi = clip_info(nssb, "GRAYS")
    with pytest.raises(nssb.Error, match="device_id must be >= 0"):
        nssb.check_args(vi, None, device_id=-1)
    with pytest.raises(nssb.Error, match=r"num_streams must be in \[1, 16\]"):
        nssb.check_args(vi, None, num_streams=17)
    nssb.check_args(vi, None, device_id=3, num_streams=16)


def test_numeric_representability(nssb):
    vi = clip_info(nssb, "GRAYS")
    with pytest.raises(nssb.Error, match=r"nss: parameter block_size\[0\] is not representable as a finite int"):
        nssb.check_args(vi, None, block_size=2 ** 40)
    with pytest.raises(nssb.Error, match=r"nss: parameter sigma\[1\] is not representable as a finite float"):
        nssb.check_args(vi, None, sigma=[3.0, float("inf")])
