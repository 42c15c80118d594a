"""C ABI checks that need no GPU: symbols, struct layouts, argument
validation and the host-side flattening (hlrc_plan_info_*)."""
import ctypes as C
import re
import subprocess

import numpy as np
import pytest

import hlr_b200 as hlr
from hlr_b200 import _capi
from hlr_b200._capi import HLRCError

from conftest import ROOT


def declared_functions():
    text = (ROOT / "include" / "hlrc.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(hlrc_[a-z_0-9]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    L = _capi.lib()
    names = declared_functions()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    # and the Python binding declares a prototype for each
    assert set(names) <= set(_capi.PROTOTYPES), set(names) - set(_capi.PROTOTYPES)


def test_abi_version():
    assert _capi.lib().hlrc_abi_version() == 1


def test_struct_layouts_match_header(tmp_path):
    structs = ["hlrc_block", "hlrc_h_desc", "hlrc_basis", "hlrc_uniform_block", "hlrc_uniform_desc",
               "hlrc_options", "hlrc_info", "hlrc_problem", "hlrc_tuning",
               "hlrc_h2_cluster", "hlrc_h2_desc"]
    # the size of every struct and the offset of every field of the ctypes
    # mirror, as the C compiler lays out the header
    fields = [(s, f) for s in structs for f, *_ in getattr(_capi, s)._fields_]
    src = tmp_path / "sz.c"
    src.write_text('#include <stddef.h>\n#include <stdio.h>\n#include "hlrc.h"\nint main(void){\n' +
                   "".join(f'printf("{s} %zu\\n", sizeof({s}));\n' for s in structs) +
                   "".join(f'printf("{s}.{f} %zu\\n", offsetof({s}, {f}));\n' for s, f in fields) +
                   "return 0;}\n")
    exe = tmp_path / "sz"
    subprocess.run(["gcc", f"-I{ROOT / 'include'}", str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()
    sizes = dict(zip(out[0::2], map(int, out[1::2])))
    for s in structs:
        assert C.sizeof(getattr(_capi, s)) == sizes[s], s
    for s, f in fields:
        assert getattr(getattr(_capi, s), f).offset == sizes[f"{s}.{f}"], (s, f)


def _ll_desc(n=8):
    rng = np.random.default_rng(0)
    ll = hlr.LeafList(n, n)
    h = n // 2
    ll.add_dense(0, 0, rng.standard_normal((h, h)))
    ll.add_lowrank(0, h, rng.standard_normal((h, 2)), rng.standard_normal((n - h, 2)))
    ll.add_lowrank(h, 0, rng.standard_normal((n - h, 0)), rng.standard_normal((h, 0)))
    ll.add_dense(h, h, rng.standard_normal((n - h, n - h)))
    return ll


def test_plan_info_accounting_matches_reference_formulas():
    ll = _ll_desc(8)
    info = hlr.plan_info(ll)
    # mul_vec_datasize: data bytes + 2*8*(nrows+ncols); FLOPS_DGEMV(m,n) = 2mn + 2m
    data = 8 * (16 + 16) + 8 * 2 * (4 + 4)
    assert info["algorithmic_bytes"] == data + 2 * 8 * 16
    fl = lambda m, n: 2 * m * n + 2 * m
    assert info["flops"] == fl(4, 4) * 2 + fl(4, 2) + fl(4, 2) + fl(4, 0) + fl(4, 0)
    assert info["n_dense"] == 2 and info["n_lowrank"] == 2
    assert info["n_row_tiles"] == 2 and info["n_col_tiles"] == 2


def test_plan_info_of_built_matrix(c1_small):
    info = hlr.plan_info(c1_small)
    d = c1_small.h_desc()
    dense = sum(d.blocks[i].nrows * d.blocks[i].ncols for i in range(d.nblocks) if d.blocks[i].kind == 0)
    lr = sum(d.blocks[i].rank * (d.blocks[i].nrows + d.blocks[i].ncols) for i in range(d.nblocks)
             if d.blocks[i].kind == 1)
    assert info["matrix_bytes"] == 8 * (dense + lr)
    assert info["n_dense"] + info["n_lowrank"] == c1_small.nleaves
    assert info["n_row_tiles"] == 2048 // 64
    assert info["device_bytes"] >= info["matrix_bytes"]


def test_rejects_gap_and_overlap():
    rng = np.random.default_rng(1)
    ll = hlr.LeafList(8, 8)
    ll.add_dense(0, 0, rng.standard_normal((8, 4)))  # right half missing
    with pytest.raises(HLRCError) as e:
        hlr.plan_info(ll)
    assert e.value.status == 2
    ll.add_dense(0, 3, rng.standard_normal((8, 5)))  # overlap by one column, area too large
    with pytest.raises(HLRCError):
        hlr.plan_info(ll)


def test_rejects_out_of_range_and_bad_args():
    rng = np.random.default_rng(1)
    ll = hlr.LeafList(4, 4)
    ll.add_dense(2, 2, rng.standard_normal((4, 4)))
    with pytest.raises(HLRCError) as e:
        hlr.plan_info(ll)
    assert e.value.status == 2
    with pytest.raises(HLRCError) as e:
        hlr.plan_info(_ll_desc(8), precision=99)
    assert e.value.status == 1
    L = _capi.lib()
    assert L.hlrc_upload_h(None, None, None) == 1
    assert L.hlrc_mvm(None, 1.0, 0, None, None, 1, 1, 1, None) == 1
    assert b"NULL" in L.hlrc_last_error()
    assert L.hlrc_free(None) == 0


def test_batch_upload_validates_members_before_any_device_work():
    L = _capi.lib()
    a, b = _ll_desc(8), _ll_desc(8)
    da, db = a.h_desc(), b.h_desc()
    arr = (_capi.hlrc_h_desc * 2)(da, db)
    out = C.c_void_p()
    overlap = (C.c_int64 * 3)(0, 4, 12)   # member 0 (n = 8) does not fit in [0, 4)
    assert L.hlrc_upload_h_batch(arr, 2, overlap, None, C.byref(out)) == 2
    assert b"does not fit" in L.hlrc_last_error()
    ll = hlr.LeafList(8, 8)
    ll.add_dense(0, 0, np.ones((8, 4)))  # member with a gap
    arr2 = (_capi.hlrc_h_desc * 2)(da, ll.h_desc())
    offs = (C.c_int64 * 3)(0, 8, 16)
    assert L.hlrc_upload_h_batch(arr2, 2, offs, None, C.byref(out)) == 2
    assert b"cover" in L.hlrc_last_error()
    assert L.hlrc_upload_h_batch(arr, 0, offs, None, C.byref(out)) == 1


def test_uniform_basis_mismatch_is_rejected(c3_small):
    u = c3_small.uniform_desc()
    # find an admissible block and corrupt its basis index
    for i in range(u.nblocks):
        if u.blocks[i].kind == 1:
            old = u.blocks[i].row_basis
            u.blocks[i].row_basis = 0  # root cluster: index set differs
            try:
                with pytest.raises(HLRCError) as e:
                    hlr.plan_info(u, uniform=True)
                assert e.value.status == 2
            finally:
                u.blocks[i].row_basis = old
            break
    info = hlr.plan_info(u, uniform=True)
    assert info["kind"] == 1 and info["n_lowrank"] > 0
