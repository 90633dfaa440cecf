"""The CLI's CSV reader (cli/hello.cpp load_csv: one read into one buffer,
newline-aligned byte ranges per thread, lines counted then parsed into their
rows) against the reference's reading rules as restated by
formats.read_csv (loadData, euclideandistancematrixgpu.cu:2712-2757: strtok on
',', space trim, atof, optional trailing cluster id, at most N lines).  A small
harness is compiled around the CLI source; no GPU is needed."""
from __future__ import annotations

import subprocess
import textwrap

import numpy as np
import pytest

from conftest import PKG_DIR, ROOT, load_package

HARNESS = textwrap.dedent("""
    #define main hello_main
    #include "{src}"
    #undef main
    int main(int argc, char** argv) {{
      std::vector<float> x;
      const int64_t n = std::atoll(argv[2]);
      const int d = std::atoi(argv[3]);
      if (!load_csv(argv[1], n, d, argv[4][0] == 'T', x)) return 1;
      std::FILE* f = std::fopen(argv[5], "wb");
      std::fwrite(x.data(), 4, x.size(), f);
      std::fclose(f);
      return 0;
    }}
""")


@pytest.fixture(scope="module")
def loader(tmp_path_factory):
    tmp = tmp_path_factory.mktemp("csv")
    src = tmp / "harness.cpp"
    src.write_text(HARNESS.format(src=PKG_DIR / "cli" / "hello.cpp"))
    exe = tmp / "harness"
    subprocess.run(["/usr/bin/g++", "-O1", "-std=c++17", f"-I{ROOT / 'include'}", str(src), f"-L{PKG_DIR}",
                    "-lacknn", f"-Wl,-rpath,{PKG_DIR}", "-pthread", "-o", str(exe)], check=True)
    return exe


def _check(loader, tmp_path, text, n, d, klaster):
    f = load_package().formats
    path = tmp_path / "in.csv"
    path.write_text(text)
    out = tmp_path / "out.bin"
    subprocess.run([str(loader), str(path), str(n), str(d), "T" if klaster else "F", str(out)], check=True)
    got = np.fromfile(out, dtype=np.float32).reshape(n, d)
    want, _ = f.read_csv(str(path), n, d, klaster)
    np.testing.assert_array_equal(got, want)


@pytest.mark.parametrize("text,n,d,klaster", [
    ("3\n2\n1,2\n3,4\n5,6\n", 3, 2, False),
    ("3\n2\n1,2\n\n5,6", 3, 2, False),                       # empty line, no final newline
    ("4\n2\n 1 , 2 ,7\n,,3,,4,\n5x,abc\n", 4, 2, True),      # blanks, empty tokens, junk, cluster ids
    ("2\n3\n1,2\r\n3,4,5,6,7\r\n", 2, 3, False),             # CRLF, short and long lines
    ("5\n1\n1\n2\n", 5, 1, False),                           # fewer lines than N
    ("2\n2\n1e3,-2.5e-3\n.5,+7\n9,9\n", 2, 2, False),        # exponents, signs, more lines than N
])
def test_edge_cases(loader, tmp_path, text, n, d, klaster):
    _check(loader, tmp_path, text, n, d, klaster)


@pytest.mark.parametrize("seed", range(6))
def test_random_files(loader, tmp_path, seed):
    f = load_package().formats
    rng = np.random.default_rng(seed)
    n, d = int(rng.integers(1, 3000)), int(rng.integers(1, 40))
    x = rng.standard_normal((n, d)).astype(np.float32)
    path = tmp_path / "r.csv"
    f.write_csv(str(path), x, labels=rng.integers(0, 9, n) if seed % 2 else None)
    _check(loader, tmp_path, path.read_text(), n, d, bool(seed % 2))


def test_fast_writers_round_trip(loader, tmp_path):
    """The bench's fast CSV writers produce files both readers parse back to
    the values they report."""
    acknn = load_package()
    f = acknn.formats
    x = acknn.workloads.integer_mixture(n=3000, d=16)
    p = tmp_path / "ints.csv"
    f.write_csv_integers(str(p), x)
    _check(loader, tmp_path, p.read_text(), 3000, 16, False)
    np.testing.assert_array_equal(f.read_csv(str(p))[0], x)
    y = acknn.workloads.sparse_prototypes(n=500, d=60)
    q = tmp_path / "fixed.csv"
    parsed = f.write_csv_fixed(str(q), y)
    _check(loader, tmp_path, q.read_text(), 500, 60, False)
    np.testing.assert_array_equal(f.read_csv(str(q))[0], parsed)
    assert np.abs(parsed - y).max() <= 1e-9
