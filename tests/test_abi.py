"""The C ABI library loads and exports every symbol include/vkb.h declares (no GPU calls)."""
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


def declared_symbols():
    text = (ROOT / "include" / "vkb.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(vkb_[a-z_]+)\s*\(", text)))


def test_header_declares_the_boundary():
    syms = declared_symbols()
    for s in ["vkb_open", "vkb_close", "vkb_scene_create", "vkb_scene_destroy", "vkb_scene_update_instances", "vkb_render"]:
        assert s in syms


def test_library_builds_and_exports_every_symbol():
    from vork_b200 import abi
    from vork_b200.build import build
    build()
    lib = abi.load()
    for s in declared_symbols():
        assert hasattr(lib, s), s
    assert set(declared_symbols()) == set(abi.SIGNATURES)
    assert lib.vkb_abi_version() == 7


def test_product_package_does_not_import_the_oracle():
    for p in (ROOT / "vork_b200").rglob("*.py"):
        src = p.read_text()
        assert "oracle" not in re.sub(r"#.*", "", src).replace("oracle is the oracle", ""), p
    for p in (ROOT / "vork_b200" / "csrc").glob("*"):
        assert "oracle" not in p.read_text().lower(), p


def test_errors_without_a_device_are_status_codes():
    # No GPU here: vkb_open reports a status instead of crashing; null arguments are INVALID_ARG.
    import ctypes as C
    from vork_b200 import abi
    lib = abi.load()
    assert lib.vkb_open(0, None) == abi.VKB_INVALID_ARG
    assert lib.vkb_render(None, None, None, None) == abi.VKB_INVALID_ARG
    assert lib.vkb_scene_create(None, None, None) == abi.VKB_INVALID_ARG
    assert lib.vkb_close(None) == abi.VKB_OK
