"""The C ABI boundary on a machine without a GPU: libspk.so loads, exports
every entry point include/spk.h declares, rejects bad k exactly like the
CLI (src/main.rs:11-30), and fails loudly (no CPU fallback) without a device."""
import ctypes as C
import os
import re
import subprocess

import pytest

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "spk.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(spk_[a-z0-9_]+)\s*\(", src)))


def test_header_declares_the_boundary():
    names = declared_functions()
    for required in ("spk_ctx_create", "spk_bloom_create", "spk_bloom_insert_u64",
                     "spk_bloom_is_solid_k256", "spk_count", "spk_result_solid",
                     "spk_result_edges", "spk_result_table_view", "spk_submit", "spk_wait"):
        assert required in names


def test_library_exports_every_declared_symbol(spk_lib):
    from spk import _lib
    path = _lib.lib_path()
    out = subprocess.run(["nm", "-D", "--defined-only", path], capture_output=True, text=True,
                         check=True).stdout
    exported = set(re.findall(r"\bT (spk_[a-z0-9_]+)", out))
    missing = [n for n in declared_functions() if n not in exported]
    assert not missing, missing
    # the ctypes layer declares exactly the header's functions
    assert sorted(_lib.EXPORTED) == declared_functions()
    L = C.CDLL(path)
    for n in declared_functions():
        assert getattr(L, n)


@pytest.mark.parametrize("k,ok,msg", [
    (10, False, "too small"), (11, True, ""), (31, True, ""), (32, False, "even"),
    (127, True, ""), (128, False, "exceeds maximum of 127"), (150, False, "exceeds"),
    (0, False, "too small"),
])
def test_validate_k_matches_cli(spk_lib, k, ok, msg):
    import spk
    if ok:
        spk.validate_k(k)
    else:
        with pytest.raises(spk.SpkError) as e:
            spk.validate_k(k)
        assert e.value.code == 2 and msg in str(e.value)


def test_count_opts_defaults(spk_lib):
    from spk._lib import CountOpts, lib
    o = CountOpts()
    lib().spk_count_opts_default(C.byref(o))
    assert o.bloom_bits == 512 * 1024 * 1024   # src/assemble.rs:84
    assert o.min_coverage == 5.0               # src/assemble.rs:82
    assert o.min_count == 0 and o.list_min_count == 2


def test_no_device_fails_loudly(spk_lib):
    """Without a usable GPU the library refuses to run (there is no CPU path)."""
    import spk
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    with pytest.raises(spk.SpkError) as e:
        spk.Context(0)
    assert e.value.code == 7  # SPK_E_NO_DEVICE


def test_struct_layouts_match_the_header(tmp_path):
    """The ctypes mirrors of the header's structs have the C sizes and field
    offsets (a compiled probe of include/spk.h against spk._lib)."""
    import ctypes as C
    from spk import _lib
    structs = {"spk_count_opts": _lib.CountOpts, "spk_result_info": _lib.ResultInfo,
               "spk_table_view": _lib.TableView, "spk_job": _lib.JobC}
    lines = ["#include <stdio.h>", "#include <stddef.h>", f'#include "{HEADER}"', "int main(void) {"]
    for cname, py in structs.items():
        lines.append(f'printf("{cname} size %zu\\n", sizeof({cname}));')
        for fname, _ in py._fields_:
            lines.append(f'printf("{cname} {fname} %zu\\n", offsetof({cname}, {fname}));')
    lines += ["return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    got = {}
    for line in out:
        if line:
            cname, what, v = line.split()
            got[(cname, what)] = int(v)
    for cname, py in structs.items():
        assert got[(cname, "size")] == C.sizeof(py), cname
        for fname, _ in py._fields_:
            assert got[(cname, fname)] == getattr(py, fname).offset, (cname, fname)


def test_solid_out_options_are_checked(spk_lib):
    """make_opts(solid_out=...) takes C-contiguous u64 keys and u32 counts of
    one length, and points the options at them (no device needed)."""
    import numpy as np
    from spk import SpkError
    from spk.api import make_opts
    keys = np.zeros((10, 2), dtype=np.uint64)
    counts = np.zeros(10, dtype=np.uint32)
    o = make_opts(solid_out=(keys, counts))
    assert o.solid_keys_out == keys.ctypes.data and o.solid_counts_out == counts.ctypes.data
    assert o.solid_capacity == 10
    assert make_opts().solid_keys_out is None and make_opts().solid_capacity == 0
    for bad in ((keys.astype(np.int64), counts), (keys, counts[:9]), (keys[:, :1][::2], counts[:5]),
                (keys, counts.astype(np.uint64))):
        with pytest.raises(SpkError):
            make_opts(solid_out=bad)
