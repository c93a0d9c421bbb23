"""The C-ABI library loads and exports every function include/natsel_gpu.h declares; the
product fails loudly instead of falling back to the CPU. No compute calls."""
import ctypes
import os
import re

import numpy as np
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
    assert ctypes.sizeof(nw.BodyDef) == 8 + 24 + 16 + 12 + 12 + 12 + 4 + 4 + 4  # tail padding to 8
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


def _c_layout():
    """Field offsets and struct sizes of the header's structs, as a C99 compiler lays them out."""
    import shutil
    import subprocess
    import tempfile
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    structs = {
        "ns_world_def": [f[0] for f in nw.WorldDef._fields_],
        "ns_body_def": [f[0] for f in nw.BodyDef._fields_],
        "ns_shape_def": [f[0] for f in nw.ShapeDef._fields_],
    }
    from natsel_b200 import narrowphase
    structs["ns_pair_job"] = list(narrowphase.PAIR_JOB_DTYPE.names)
    structs["ns_pair_result"] = list(narrowphase.PAIR_RESULT_DTYPE.names)
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "natsel_gpu.h"', 'int main(void) {']
    for s, fields in structs.items():
        lines.append('  printf("%s size %%zu\\n", sizeof(%s));' % (s, s))
        for f in fields:
            lines.append('  printf("%s %s %%zu\\n", offsetof(%s, %s));' % (s, f, s, f))
    lines += ['  return 0;', '}']
    with tempfile.TemporaryDirectory() as d:
        src, exe = os.path.join(d, "layout.c"), os.path.join(d, "layout")
        open(src, "w").write("\n".join(lines) + "\n")
        subprocess.run([cc, "-std=c99", "-Wall", "-Wextra", "-Werror", "-pedantic", "-I",
                        os.path.join(ROOT, "include"), src, "-o", exe], check=True)
        out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout
    layout = {}
    for line in out.splitlines():
        s, f, v = line.split()
        layout[(s, f)] = int(v)
    return layout


def test_header_compiles_as_c99_with_the_mirrored_layouts():
    from natsel_b200 import narrowphase
    layout = _c_layout()
    for name, cls in (("ns_world_def", nw.WorldDef), ("ns_body_def", nw.BodyDef), ("ns_shape_def", nw.ShapeDef)):
        assert layout[(name, "size")] == ctypes.sizeof(cls)
        for f in cls._fields_:
            assert layout[(name, f[0])] == getattr(cls, f[0]).offset, (name, f[0])
    for name, dt in (("ns_pair_job", narrowphase.PAIR_JOB_DTYPE), ("ns_pair_result", narrowphase.PAIR_RESULT_DTYPE)):
        assert layout[(name, "size")] == dt.itemsize
        for f in dt.names:
            assert layout[(name, f)] == dt.fields[f][1], (name, f)


def _bad_jobs():
    """One valid batch with a single bad job planted in it, for every check the host makes."""
    import _pairgen
    from natsel_b200 import narrowphase
    cases = []

    def plant(idx, **fields):
        jobs = _pairgen.make_jobs(narrowphase.PAIR_JOB_DTYPE, 12, 3, 1.0)
        for k, v in fields.items():
            jobs[idx][k] = v
        return jobs

    # idx 0 is hull-hull, 1 hull-sphere, 2 hull-capsule, 3 sphere-sphere, 4 capsule-sphere
    cases.append(("unknown type", plant(3, type_a=7)))
    cases.append(("secondary type first", plant(3, type_a=5, type_b=0)))
    cases.append(("sphere with a box", plant(3, type_b=3)))
    cases.append(("sat type", plant(0, sat_type=9)))
    cases.append(("sat hit", plant(0, sat_hit=2)))
    cases.append(("face index", plant(0, sat_type=2, sat_index_a=6)))
    cases.append(("face b index", plant(0, sat_type=3, sat_index_b=200)))
    cases.append(("odd edge", plant(0, sat_type=4, sat_index_a=3, sat_index_b=2)))
    cases.append(("edge past the end", plant(0, sat_type=4, sat_index_a=0, sat_index_b=24)))
    cases.append(("negative index", plant(0, sat_index_a=-1)))
    cases.append(("simplex count", plant(1, simplex_count=65535)))
    cases.append(("simplex count negative", plant(1, simplex_count=-1)))
    ia = np.array([0, 8, 0, 0], np.int32)
    cases.append(("simplex vertex of the box", plant(1, simplex_count=2, simplex_ia=ia)))
    ib = np.array([0, 1, 0, 0], np.int32)
    cases.append(("simplex vertex of the sphere", plant(1, simplex_count=2, simplex_ib=ib)))
    ib2 = np.array([2, 0, 0, 0], np.int32)
    cases.append(("simplex vertex of the capsule", plant(2, simplex_count=1, simplex_ib=ib2)))
    return cases



@pytest.mark.parametrize("entry", ["ns_collide_pairs", "ns_collide_pairs_noalloc"])
def test_bad_pair_jobs_are_rejected_on_the_host_before_any_gpu_work(entry):
    """Every job is checked before a copy or launch: a batch with one bad job returns
    NS_ERR_INVALID and leaves the jobs as they were (no device is needed to see it)."""
    from natsel_b200 import narrowphase
    lib = nw.load_library()
    fn = getattr(lib, entry)
    for what, jobs in _bad_jobs():
        before = jobs.tobytes()
        results = np.zeros(len(jobs), narrowphase.PAIR_RESULT_DTYPE)
        status = fn(jobs.ctypes.data_as(ctypes.c_void_p), results.ctypes.data_as(ctypes.c_void_p), len(jobs))
        assert status == 1, what
        assert b"job" in lib.ns_last_error(None), what
        assert jobs.tobytes() == before and not results.tobytes().strip(b"\0"), what
    # the untouched batch passes the checks (without a GPU it then fails on the device instead)
    import _pairgen
    jobs = _pairgen.make_jobs(narrowphase.PAIR_JOB_DTYPE, 12, 3, 1.0)
    results = np.zeros(len(jobs), narrowphase.PAIR_RESULT_DTYPE)
    status = fn(jobs.ctypes.data_as(ctypes.c_void_p), results.ctypes.data_as(ctypes.c_void_p), len(jobs))
    assert status == (0 if HAS_GPU else 2)


def _rust_source():
    return open(os.path.join(ROOT, "natsel-gpu-sys", "src", "lib.rs")).read()


def _c_params(name):
    text = re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)
    m = re.search(r"\b%s\s*\(([^)]*)\)" % name, text)
    args = [a for a in m.group(1).split(",") if a.strip() and a.strip() != "void"]
    return len(args)


def test_rust_ffi_crate_declares_every_header_function():
    """natsel-gpu-sys/src/lib.rs (the reference-side binding; cargo is not in this image) declares
    every function of include/natsel_gpu.h, with the same number of parameters."""
    src = _rust_source()
    block = src[src.index('extern "C" {'):]
    block = block[:block.index("\n}\n")]
    decls = dict((m.group(1), m.group(2)) for m in re.finditer(r"pub fn (ns_[a-z0-9_]+)\(([^)]*)\)", block, re.S))
    assert sorted(decls) == declared_functions()
    for name, params in decls.items():
        n = len([p for p in params.split(",") if p.strip()])
        assert n == _c_params(name), name


def test_rust_ffi_structs_mirror_the_header_layouts():
    """Each #[repr(C)] struct of the crate lists the header struct's fields in the same order with
    types of the same size (checked against the offsets a C99 compiler gives the header)."""
    src = _rust_source()
    sizes = {"c_int": 4, "f32": 4, "i32": 4, "u32": 4, "u64": 8, "f64": 8}

    def rust_fields(name):
        body = re.search(r"pub struct %s \{(.*?)\n\}" % name, src, re.S).group(1)
        out = []
        for fname, ftype in re.findall(r"pub (\w+): ([^,\n]+),", body):
            ftype = ftype.strip()
            n, base = 1, ftype
            while base.startswith("["):
                inner, count = re.match(r"\[(.*); (\d+)\]$", base).groups()
                n *= int(count)
                base = inner
            out.append((fname.rstrip("_") if fname == "type_" else fname, sizes[base] * n, sizes[base]))
        return out

    layout = _c_layout()
    for name in ("ns_world_def", "ns_body_def", "ns_shape_def", "ns_pair_job", "ns_pair_result"):
        off = 0
        for fname, size, align in rust_fields(name):
            off = (off + align - 1) // align * align
            assert layout[(name, fname)] == off, (name, fname)
            off += size
        assert (off + 7) // 8 * 8 >= layout[(name, "size")] >= off
