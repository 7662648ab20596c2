"""The C ABI: library loads, exports every declared entry point, and its
host-only functions behave as specified (no GPU needed)."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

from marigold_b200 import _lib
from marigold_b200.bvh import NODE_DTYPE, encode_gpu_bytes, sah_cost

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include",
                      "mgbvh.h")


def declared_functions():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"MGBVH_API\s+[\w\s\*]+?\b(mgbvh_\w+)\s*\(", text)))


def test_header_and_binding_agree():
    assert declared_functions() == sorted(_lib.EXPORTED)


def test_library_exports_every_declared_symbol():
    L = _lib.load()
    for name in declared_functions():
        assert hasattr(L, name), name


def test_struct_layouts_match_header(tmp_path):
    # compile the header with the host C compiler and compare sizes/offsets
    src = tmp_path / "sz.c"
    src.write_text(
        '#include <stdio.h>\n#include <stddef.h>\n#include "mgbvh.h"\n'
        'int main(void){printf("%zu %zu %zu %zu %zu %zu\\n", sizeof(mgbvh_node), '
        'sizeof(mgbvh_settings), sizeof(mgbvh_stats), offsetof(mgbvh_settings, bins), '
        'offsetof(mgbvh_stats, total_object_count), offsetof(mgbvh_stats, feasible));return 0;}\n')
    exe = tmp_path / "sz"
    subprocess.run(["gcc", "-I", os.path.dirname(HEADER), str(src), "-o", str(exe)], check=True)
    got = [int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True,
                                          check=True).stdout.split()]
    assert got == [ctypes.sizeof(_lib.Node), ctypes.sizeof(_lib.Settings),
                   ctypes.sizeof(_lib.Stats), _lib.Settings.bins.offset,
                   _lib.Stats.total_object_count.offset, _lib.Stats.feasible.offset]
    assert got[0] == 32 == NODE_DTYPE.itemsize


def test_scene_record_layouts(tmp_path):
    # the two-level scene records: 16-byte mesh table rows, 80-byte instances
    # (marigold_b200.bvh.Scene writes them as int32 [M, 4] and [I, 20])
    src = tmp_path / "sc.c"
    src.write_text(
        '#include <stdio.h>\n#include <stddef.h>\n#include "mgbvh.h"\n'
        'int main(void){printf("%zu %zu %zu %zu\\n", sizeof(mgbvh_scene_mesh), sizeof(mgbvh_scene_instance), '
        'offsetof(mgbvh_scene_mesh, vertex_offset), offsetof(mgbvh_scene_instance, mesh));return 0;}\n')
    exe = tmp_path / "sc"
    subprocess.run(["gcc", "-I", os.path.dirname(HEADER), str(src), "-o", str(exe)], check=True)
    got = [int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    assert got == [16, 80, 12, 64]


def test_default_settings_are_the_reference_profile():
    s = _lib.Settings()
    _lib.load().mgbvh_default_settings(ctypes.byref(s))
    assert (s.min_leaf_objects, s.max_leaf_objects, s.max_depth) == (1, 1, 32)
    assert (s.bins, s.adaptive_max_n, s.adaptive_steps, s.has_bounds) == (0, 32, 0, 0)


def test_status_strings():
    for rc in (0, 1, 2, -1, -2, -3, -4, -5, -6, -7, -8):
        assert _lib.status_string(rc) != "unknown status"


def _nodes(rows):
    a = np.zeros(len(rows), NODE_DTYPE)
    for i, (mn, start, mx, child) in enumerate(rows):
        a[i] = (mn, start, mx, child)
    return a


def test_gpu_bytes_max_one_is_identity():
    nd = _nodes([((0, 0, 0), 0, (1, 1, 1), 1), ((0, 0, 0), 1, (1, 1, 1), 0),
                 ((0, 0, 0), 0, (1, 1, 1), 0)])
    w = encode_gpu_bytes(nd, np.array([2, 1, 1], np.uint32), 1)
    assert np.array_equal(w, nd.view(np.uint32).reshape(-1, 8))


def test_gpu_bytes_packing_matches_reference_formula():
    # bvh/src/lib.rs:170-195 with MAX = 6: len_bits = ilog2(8) = 3,
    # packed = (len & 7) << 29 | (child & !7)
    nd = _nodes([((0, 0, 0), 0, (1, 1, 1), 13), ((0, 0, 0), 4, (1, 1, 1), 0)])
    w = encode_gpu_bytes(nd, np.array([9, 5], np.uint32), 6)
    assert w[0, 7] == ((9 & 7) << 29) | (13 & ~7 & 0xFFFFFFFF)
    assert w[1, 7] == (5 << 29)
    assert w[1, 3] == 4


def test_gpu_bytes_reference_assert_on_overflowing_leaf():
    # a leaf with len >= next_power_of_two(MAX) panics in the reference
    nd = _nodes([((0, 0, 0), 0, (1, 1, 1), 0)])
    with pytest.raises(_lib.MgbvhError):
        encode_gpu_bytes(nd, np.array([4], np.uint32), 4)


def test_sah_cost_of_hand_tree():
    # root [0,3]x[0,1]x[0,1] (SA 14) with two unit-box leaves (SA 6 each):
    # 1 * 14/14 + 8 * 1 * 6/14 * 2
    nd = _nodes([((0, 0, 0), 0, (3, 1, 1), 1), ((2, 0, 0), 1, (3, 1, 1), 0),
                 ((0, 0, 0), 0, (1, 1, 1), 0)])
    c = sah_cost(nd, np.array([2, 1, 1], np.uint32))
    assert abs(c - (1.0 + 16.0 * 6.0 / 14.0)) < 1e-12


def test_no_device_means_an_error_not_a_fallback():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(_lib.MgbvhError) as e:
        _lib.Context(0)
    assert e.value.status == _lib.ERR_NO_DEVICE
