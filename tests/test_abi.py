"""The C-ABI library loads without a GPU and exports every entry point the
public header declares; calls that need no device behave."""
import ctypes as C
import re
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def declared_functions():
    names = set()
    for header in (ROOT / "include").glob("*.h"):
        text = re.sub(r"/\*.*?\*/", "", header.read_text(), flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[a-z_0-9]+\s*\**\s*(nssb_[a-z_0-9]+)\s*\(", text, flags=re.M):
            names.add(m.group(1))
    return names


def test_header_declares_entry_points():
    names = declared_functions()
    for n in ("nssb_last_error", "nssb_bm3d_create", "nssb_bm3d_get_frame", "nssb_match_spatial",
              "nssb_bm3d_plane_stage", "nssb_bm3d_check"):
        assert n in names


def test_library_exports_every_declared_symbol(nssb):
    lib = nssb.lib()
    missing = [n for n in sorted(declared_functions()) if not hasattr(lib, n)]
    assert not missing, missing


def test_version_and_error_without_device(nssb):
    assert "sm_100a" in nssb.version()
    assert nssb.last_error() == ""


def test_create_without_device_is_a_creation_error(nssb):
    import torch

    if torch.cuda.is_available():
        return
    vi = nssb.format_info("GRAYS", 48, 40, 4)
    clip = nssb.Clip([(None,)] * 4, vi)
    try:
        nssb.BM3D(clip)
    except nssb.Error as e:
        assert str(e).startswith("nss_cuda.BM3D: no CUDA device available")
    else:
        raise AssertionError("creation without a device must fail")


def test_batch_create_checks_arguments_then_device(nssb):
    import pytest
    import torch

    with pytest.raises(nssb.Error, match="unknown argument bogus"):
        nssb.Batch(bogus=1)
    with pytest.raises(nssb.Error, match="match_parts must be 1, 2 or 4"):
        nssb.Batch(autotune=False, match_parts=3)
    with pytest.raises(nssb.Error, match="group_warps must be 2, 4 or 8"):
        nssb.Batch(autotune=False, group_warps=16)
    if not torch.cuda.is_available():
        with pytest.raises(nssb.Error, match="nss_batch: no CUDA device available"):
            nssb.Batch()


def test_server_create_checks_arguments_then_device(nssb):
    import pytest
    import torch

    with pytest.raises(nssb.Error, match="unknown argument bogus"):
        nssb.Server(bogus=1)
    with pytest.raises(nssb.Error, match="workers out of range"):
        nssb.Server(workers=0)
    if not torch.cuda.is_available():
        with pytest.raises(nssb.Error, match="nss_server: no CUDA device available"):
            nssb.Server()
