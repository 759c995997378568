"""The C-ABI library loads and exports every entry point include/*.h declares (no GPU needed)."""
import ctypes as C
import glob
import os
import re

import pytest

from nndex_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        names |= set(re.findall(r"NNDEX_API\s+[\w\s\*]+?\b(nndex_cuda_\w+)\s*\(", text))
    return names


def test_header_declares_entry_points():
    names = _declared_symbols()
    assert {"nndex_cuda_create", "nndex_cuda_search", "nndex_cuda_search_batch", "nndex_cuda_destroy",
            "nndex_cuda_last_error", "nndex_cuda_info", "nndex_cuda_list_devices"} <= names


def test_library_exports_every_declared_symbol():
    L = C.CDLL(_lib.LIB_PATH)
    missing = [n for n in sorted(_declared_symbols()) if not hasattr(L, n)]
    assert not missing, missing


def test_ctypes_signatures_cover_the_header():
    assert set(_lib.SIGNATURES) == _declared_symbols()
    _lib.lib()  # binds every signature


def test_structs_match_header_layout():
    # sizes of the C structs as the header lays them out (x86-64)
    assert C.sizeof(_lib.Opts) == 4 + 4 * 5 + 8 + 4 + 4 * 7
    assert C.sizeof(_lib.DevInfo) == 8 + 256 + 64 + 64 + 32 + 32 + 4 * 3 + 4 + 8 + 8
    assert C.sizeof(_lib.SearchStats) == 4 * 6 + 8 + 8 + 8 + 8 + 8 + 4 * 4 + 8 + 8 + 4 * 2 + 8 + 4 * 2


def test_last_error_is_empty_string_initially():
    assert isinstance(_lib.last_error(), str)


STRUCTS = {
    "nndex_cuda_opts": "Opts",
    "nndex_cuda_devinfo": "DevInfo",
    "nndex_cuda_search_stats": "SearchStats",
    "nndex_cuda_ivf_stats": "IvfStats",
    "nndex_cuda_server_opts": "ServerOpts",
    "nndex_cuda_request_info": "RequestInfo",
    "nndex_cuda_server_stats": "ServerStats",
}


def test_ctypes_structs_match_the_c_compiler(tmp_path):
    # sizeof and every field offset as gcc lays the header out, against the ctypes mirrors
    import shutil
    import subprocess
    gcc = shutil.which("gcc")
    if gcc is None:
        pytest.skip("no C compiler")
    lines = ["#include <stdio.h>", "#include <stddef.h>", f'#include "{ROOT}/include/nndex_cuda.h"', "int main(void) {"]
    for cname, pyname in STRUCTS.items():
        lines.append(f'printf("{cname} sizeof %zu\\n", sizeof({cname}));')
        for field, _ in getattr(_lib, pyname)._fields_:
            lines.append(f'printf("{cname} {field} %zu\\n", offsetof({cname}, {field}));')
    lines += ["return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run([gcc, "-o", str(exe), str(src)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    got = {tuple(l.split()[:2]): int(l.split()[2]) for l in out if l.strip()}
    for cname, pyname in STRUCTS.items():
        cls = getattr(_lib, pyname)
        assert got[(cname, "sizeof")] == C.sizeof(cls), cname
        for field, _ in cls._fields_:
            assert got[(cname, field)] == getattr(cls, field).offset, (cname, field)



def test_null_index_is_refused_without_touching_the_device():
    # Every entry point that takes an index checks it before any CUDA call, so a wrapper that
    # passes NULL gets NNDEX_ERR_INVALID_ARGUMENT and a message, also on a machine without a GPU.
    L = _lib.lib()
    u64, f32 = C.c_uint64(), C.c_float()
    st = _lib.SearchStats()
    calls = [
        ("search", lambda: L.nndex_cuda_search(None, None, 0, 1, None, None, None)),
        ("search_batch", lambda: L.nndex_cuda_search_batch(None, None, 0, 0, 1, None, None, None)),
        ("search_batch_device", lambda: L.nndex_cuda_search_batch_device(None, None, 0, 0, 1, None, None, None,
                                                                         None, 1)),
        ("set_precision", lambda: L.nndex_cuda_set_precision(None, 0, 0)),
        ("stream_status", lambda: L.nndex_cuda_stream_status(None)),
        ("last_search_stats", lambda: L.nndex_cuda_last_search_stats(None, C.byref(st))),
        ("rows", lambda: L.nndex_cuda_rows(None, C.byref(u64), C.byref(u64), C.byref(u64))),
        ("base_checksum", lambda: L.nndex_cuda_base_checksum(None, C.byref(u64))),
        ("set_nprobe", lambda: L.nndex_cuda_set_nprobe(None, 8)),
        ("set_graphs", lambda: L.nndex_cuda_set_graphs(None, 1)),
        ("set_scan_timing", lambda: L.nndex_cuda_set_scan_timing(None, 1)),
        ("set_error_report", lambda: L.nndex_cuda_set_error_report(None, 1)),
        ("last_score_errors", lambda: L.nndex_cuda_last_score_errors(None, 1, 1, None)),
        ("server_start", lambda: L.nndex_cuda_server_start(None, None, C.byref(C.c_void_p()))),
        ("server_submit", lambda: L.nndex_cuda_server_submit(None, None, 1, 1, 1, 0, 0, C.byref(u64))),
        ("server_poll", lambda: L.nndex_cuda_server_poll(None, 1, 0, None, None, None, None)),
        ("server_stats", lambda: L.nndex_cuda_server_stats_get(None, C.byref(_lib.ServerStats()))),
    ]
    L.nndex_cuda_server_stop(None)  # a no-op
    for name, call in calls:
        code = call()
        assert code == _lib.NNDEX_ERR_INVALID_ARGUMENT, (name, code, _lib.last_error())
        assert "null" in _lib.last_error(), (name, _lib.last_error())
