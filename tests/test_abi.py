"""The C-ABI library loads and exports every function include/natsel_gpu.h declares; the
product fails loudly instead of falling back to the CPU. No compute calls."""
import ctypes
import os
import re

import pytest

from conftest import HAS_GPU, ROOT
from natsel_b200 import world as nw

HEADER = os.path.join(ROOT, "include", "natsel_gpu.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(ns_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_the_step_api():
    names = declared_functions()
    for required in ("ns_world_create", "ns_world_step", "ns_world_get_bodies", "ns_world_state_hash",
                     "ns_collide_pairs"):
        assert required in names


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(nw.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_the_header():
    assert sorted(nw.EXPORTED) == declared_functions()


def test_library_is_built_for_sm100a():
    # the fatbinary carries sm_100a code: the build records the arch in its flags
    from natsel_b200 import _build
    assert "arch=compute_100a,code=sm_100a" in " ".join(_build.NVCC_FLAGS)
    assert os.path.getsize(nw.LIB_PATH) > 0


def test_struct_layouts_match_header():
    assert ctypes.sizeof(nw.WorldDef) == 4 * 3 + 4 * 3 + 4 * 5 + 4 + 4 * 2 + 4 * 3
    assert ctypes.sizeof(nw.BodyDef) == 8 + 24 + 16 + 12 + 12 + 12 + 4
    from natsel_b200 import narrowphase
    assert narrowphase.PAIR_JOB_DTYPE.itemsize == 152


@pytest.mark.skipif(HAS_GPU, reason="checks the no-GPU failure path")
def test_world_without_gpu_raises():
    with pytest.raises(nw.NsError):
        nw.World()


def test_sleeping_is_rejected():
    d = nw.default_world_def(enable_sleep=1)
    with pytest.raises(nw.NsError):
        nw.World(d)
