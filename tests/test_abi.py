"""The C-ABI library loads without a GPU and exports every entry point include/sr_cuda.h declares; the Python
mirror of the config struct has the C layout."""
import ctypes as C
import os
import re

from sandbox_reactions_b200 import build
from sandbox_reactions_b200.abi import Config, sr_config
from sandbox_reactions_b200.engine import load_library

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for f in os.listdir(os.path.join(ROOT, "include")):
        if f.endswith(".h"):
            text = open(os.path.join(ROOT, "include", f)).read()
            text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
            names |= set(re.findall(r"\b(sr_[a-z0-9_]+)\s*\(", text))
    return names


def test_the_library_exports_every_declared_entry_point():
    build.build()
    lib = load_library()
    names = declared_symbols()
    assert {"sr_create", "sr_step", "sr_upload", "sr_readback", "sr_last_error"} <= names
    for name in sorted(names):
        assert hasattr(lib, name), name


def test_the_config_defaults_match_the_library():
    lib = load_library()
    c = sr_config()
    lib.sr_config_default(C.byref(c))
    assert c.struct_size == C.sizeof(sr_config)
    py = Config().to_c()
    for name, _ in sr_config._fields_:
        if name.startswith("reserved") or name in ("width", "height"):
            continue
        assert getattr(c, name) == getattr(py, name), name
    assert lib.sr_abi_version() == 3


def test_create_refuses_a_bad_world_without_touching_a_device():
    lib = load_library()
    c = Config(width=100).to_c()
    h = C.c_void_p()
    st = lib.sr_create(C.byref(c), C.byref(h))
    assert st == 1 and not h.value
    assert b"multiple of 8" in lib.sr_last_error(None)
