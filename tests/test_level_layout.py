"""The level-order pressure solve's staging layout, checked on the CPU.

Each level's records and input values reach shared memory by bulk copies (cp.async.bulk), which
must start and end on 16-byte boundaries; an unaligned copy loses the GPU context.  The layout
header the kernels use (ressim_b200/csrc/rf_level_layout.hpp) is compiled here with g++
(tests/native/level_layout_host.cpp), and every level placement (first position, width up to the
plan's widest level) of arrays of n positions is replayed for FP64 and FP32: the copies are
aligned, stay inside their source arrays (the scratch vectors padded to four values) and fit their
shared-memory slots, and the long rows' shared-memory regions are aligned and disjoint.
"""
import ctypes as C
import os
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def layout_lib(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("layout") / "level_layout_host.so")
    subprocess.run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-o", out,
                    os.path.join(HERE, "native", "level_layout_host.cpp")], check=True)
    lib = C.CDLL(out)
    lib.rfh_level_layout_check.argtypes = [C.c_int32, C.c_int32, C.c_char_p, C.c_size_t]
    lib.rfh_level_layout_check.restype = C.c_int32
    return lib


@pytest.mark.parametrize("n,W", [(n, W) for n in (1, 2, 3, 5, 8, 17, 40) for W in (1, 2, 3, 7, 16)]
                         + [(3300, 110), (18921, 380), (64512, 952), (72000, 1000)])
def test_bulk_copies_aligned_and_in_bounds(layout_lib, n, W):
    W = min(W, n)
    err = C.create_string_buffer(256)
    assert layout_lib.rfh_level_layout_check(n, W, err, len(err)) == 1, err.value.decode()
