"""The C ABI library: it loads without a GPU, exports every function that
include/knn.h declares, agrees with the ctypes struct layouts, and rejects bad
arguments before touching a device.  No compute call runs here."""
from __future__ import annotations

import ctypes
import re
import subprocess
import textwrap

import numpy as np
import pytest

from conftest import PKG_DIR, ROOT, load_package

HEADERS = sorted((ROOT / "include").glob("*.h"))


def _declared_functions():
    names = []
    for h in HEADERS:
        text = h.read_text()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^\s*[A-Za-z_][\w\s\*]*?\b(knn_\w+)\s*\(", text, flags=re.M):
            names.append(m.group(1))
    return sorted(set(names))


def test_header_declares_functions():
    names = _declared_functions()
    assert "knn_build" in names and "knn_build_ex" in names
    assert len(names) >= 14


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(str(PKG_DIR / "libacknn.so"))
    missing = [n for n in _declared_functions() if not hasattr(lib, n)]
    assert not missing, f"declared but not exported: {missing}"


def test_python_binding_covers_header():
    acknn = load_package()
    assert set(_declared_functions()) <= set(acknn.EXPORTS), "ctypes table misses a symbol"


def test_struct_layout_matches_c(tmp_path):
    """Every field offset and every struct size of the ctypes mirror equals
    the C compiler's for the header's structs."""
    acknn = load_package()
    structs = {"knn_options": acknn.KnnOptions, "knn_stats": acknn.KnnStats,
               "knn_dataset": acknn.KnnDataset}
    lines, want = [], []
    for cname, py in structs.items():
        lines.append(f'printf("%zu\\n", sizeof({cname}));')
        want.append(ctypes.sizeof(py))
        for fname, _ in py._fields_:
            lines.append(f'printf("%zu\\n", offsetof({cname}, {fname}));')
            want.append(getattr(py, fname).offset)
    src = tmp_path / "probe.c"
    body = "\n          ".join(lines)
    src.write_text(textwrap.dedent(f"""
        #include <stdio.h>
        #include <stddef.h>
        #include "{ROOT / 'include' / 'knn.h'}"
        int main(void) {{
          {body}
          return 0;
        }}"""))
    exe = tmp_path / "probe"
    subprocess.run(["/usr/bin/gcc", str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()
    assert [int(v) for v in out] == want


def test_status_strings_and_version():
    acknn = load_package()
    lib = acknn.load_library()
    assert lib.knn_version() >= 100
    for code, text in acknn.STATUS.items():
        assert lib.knn_status_string(code).decode() == text


def test_default_options():
    acknn = load_package()
    o = acknn.default_options()
    assert o.struct_size == ctypes.sizeof(acknn.KnnOptions)
    assert o.device == -1 and o.dtype == 0 and o.precision == 0 and o.points_on_device == 0


@pytest.mark.parametrize("n,d,k,metric,expect", [
    (10, 4, 10, 0, -2),    # n <= k
    (10, 4, 0, 0, -1),     # k < 1
    (10, 0, 3, 0, -1),     # d < 1
    (10, 4, 3, 7, -1),     # unknown metric
    (10, 4, 200, 0, -1),   # k > KNN_MAX_K
])
def test_argument_errors_before_device(n, d, k, metric, expect):
    acknn = load_package()
    lib = acknn.load_library()
    x = np.zeros((max(n, 1), max(d, 1)), dtype=np.float32)
    idx = np.zeros((max(n, 1), max(k, 1)), dtype=np.int32)
    dist = np.zeros((max(n, 1), max(k, 1)), dtype=np.float32)
    rc = lib.knn_build(x.ctypes.data, n, d, k, 2, 8, 1, metric, 0, idx.ctypes.data, dist.ctypes.data)
    assert rc == expect
    assert lib.knn_last_error()


def test_null_pointers_rejected():
    acknn = load_package()
    lib = acknn.load_library()
    assert lib.knn_build(None, 10, 2, 3, 1, 4, 1, 0, 0, None, None) == -1


def test_missing_library_fails_loudly(tmp_path):
    acknn = load_package()
    with pytest.raises(RuntimeError, match="no CPU fallback"):
        acknn.load_library(tmp_path / "libacknn.so")


def test_batch_argument_errors_before_device():
    """knn_build_batch rejects bad batches before touching a device."""
    acknn = load_package()
    x = np.zeros((10, 4), dtype=np.float32)
    small = np.zeros((3, 4), dtype=np.float32)
    with pytest.raises(acknn.KnnError) as e:
        acknn.knn_build_batch([x, small], 5, 2, 8, 1, 0)
    assert e.value.status == -2  # a set with n <= k
    with pytest.raises(acknn.KnnError) as e:
        acknn.knn_build_batch([x], 5, 0, 8, 1, 0)
    assert e.value.status == -1
    with pytest.raises(acknn.KnnError) as e:
        acknn.knn_build_batch([x], 5, 2, 8, 1, 7)
    assert e.value.status == -1
    with pytest.raises(acknn.KnnError) as e:
        acknn.knn_build_batch([], 5, 2, 8, 1, 0)
    assert e.value.status == -1
