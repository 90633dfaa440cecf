"""The drop-in `hello` CLI (approximate-cuda-knn_b200/cli/hello.cpp): argument
order, messages and exit codes of the reference's main.cpp, its CSV input and
its binary output layout."""
from __future__ import annotations

import subprocess

import numpy as np
import pytest

from conftest import PKG_DIR, load_package

HELLO = PKG_DIR / "hello"


@pytest.fixture(scope="module")
def hello():
    if not HELLO.exists():
        subprocess.run(["make", "-C", str(PKG_DIR), "hello"], check=True, capture_output=True)
    return str(HELLO)


def _run(hello, *args):
    return subprocess.run([hello, *map(str, args)], capture_output=True, text=True, timeout=600)


def test_wrong_argument_count(hello):
    r = _run(hello, "a", "b")
    assert r.returncode == 1
    assert r.stdout.startswith("Wrong number of arguments!")


def test_unknown_metric(hello):
    r = _run(hello, "in.csv", "out", 3, 2, 8, 1, "MANHATTAN", 0, "F")
    assert r.returncode == 2
    assert "Wrong distance algorithm!" in r.stdout


def test_device_not_present(hello):
    r = _run(hello, "in.csv", "out", 3, 2, 8, 1, "EUCLIDEAN", 97, "F")
    assert r.returncode == 3
    assert "Device with id 97 is not located in this computer" in r.stdout


def _points(n, d, seed):
    rng = np.random.Generator(np.random.PCG64(seed))
    c = rng.uniform(-5, 5, size=(6, d))
    return (c[rng.integers(0, 6, n)] + rng.standard_normal((n, d))).astype(np.float32)


@pytest.mark.gpu
def test_missing_input(hello, tmp_path):
    r = _run(hello, tmp_path / "nope.csv", tmp_path / "out", 3, 2, 8, 1, "EUCLIDEAN", 0, "F")
    assert r.returncode == 7
    assert "Error opening the file" in r.stdout


@pytest.mark.gpu
@pytest.mark.parametrize("metric", ["EUCLIDEAN", "TAXICAB", "COSINE"])
def test_cli_matches_library_and_mirror(hello, tmp_path, metric):
    acknn = load_package()
    f = acknn.formats
    n, d, k = 3000, 9, 7
    x = _points(n, d, 5)
    lab = np.arange(n) % 6
    csv = tmp_path / "in.csv"
    f.write_csv(str(csv), x, lab)
    out = tmp_path / "out.bin"
    r = _run(hello, csv, out, k, 4, 32, 2, metric, 0, "T", "--debug")
    assert r.returncode == 0, r.stdout
    assert "The end" in r.stdout
    nn, kk, ids, stored = f.read_result(str(out))
    assert (nn, kk) == (n, k)
    # the same build through the library, on the reference-normalised points
    m = acknn.METRICS[metric]
    xn = acknn.normalize_reference(f.read_csv(str(csv), klaster=True)[0])
    idx, dist = acknn.knn_build(xn, k, 4, 32, 2, m, seed=0)
    np.testing.assert_array_equal(ids, idx)
    np.testing.assert_array_equal(stored, f.stored_distance(dist, m))
    assert (tmp_path / "out.binVALIDATION").read_text() == "Everything is OK."
    assert (tmp_path / "out.binDEBUG").read_text().startswith("NEAR: <0, ")
    # the Python mirror of the reference class writes the same bytes
    edm = acknn.EuclideanDistanceMatrixGPU(debugMode=True)
    edm.setDataFile(str(csv))
    edm.setResultsFile(str(tmp_path / "mirror.bin"))
    assert edm.initialize(n, d, k, 0, m, True, 4, 2, 32) is False
    assert edm.calculate() is False
    assert edm.saveResultToResultFile() is False
    assert edm.deinitialize() is False
    assert (tmp_path / "mirror.bin").read_bytes() == out.read_bytes()
    assert (tmp_path / "mirror.binDEBUG").read_text() == (tmp_path / "out.binDEBUG").read_text()


@pytest.mark.gpu
@pytest.mark.parametrize("env, kw", [
    ({"ACKNN_PRECISION": "bf16", "ACKNN_SEED": "11"}, {"precision": 1, "seed": 11}),
    ({"ACKNN_PRECISION": "f16", "ACKNN_TIMING": "1"}, {"precision": 2}),
    ({"ACKNN_SPLITS": "reference", "ACKNN_SEED": "3"}, {"split_rule": 1, "seed": 3}),
])
def test_cli_environment_knobs(hello, tmp_path, env, kw):
    """Precision, split rule and seed come from ACKNN_* variables; the
    positional command line is unchanged and the graph is the library's with
    the same options."""
    import os

    acknn = load_package()
    f = acknn.formats
    n, d, k = 4000, 12, 8
    x = _points(n, d, 8)
    csv = tmp_path / "in.csv"
    f.write_csv(str(csv), x)
    out = tmp_path / "out.bin"
    r = subprocess.run([hello, str(csv), str(out), str(k), "4", "64", "1", "EUCLIDEAN", "0", "F"],
                       capture_output=True, text=True, timeout=600, env={**os.environ, **env})
    assert r.returncode == 0, r.stdout
    _, _, ids, stored = f.read_result(str(out))
    xn = acknn.normalize_reference(f.read_csv(str(csv), klaster=False)[0])
    idx, dist = acknn.knn_build(xn, k, 4, 64, 1, 0, **kw)
    np.testing.assert_array_equal(ids, idx)
    np.testing.assert_array_equal(stored, f.stored_distance(dist, 0))


@pytest.mark.gpu
@pytest.mark.parametrize("env", [{"ACKNN_PRECISION": "fp8"}, {"ACKNN_SPLITS": "sideways"}, {"ACKNN_SEED": "-1"}])
def test_cli_rejects_unknown_knob_values(hello, tmp_path, env):
    import os

    acknn = load_package()
    csv = tmp_path / "in.csv"
    acknn.formats.write_csv(str(csv), _points(100, 4, 1))
    r = subprocess.run([hello, str(csv), str(tmp_path / "o"), "3", "2", "16", "1", "EUCLIDEAN", "0", "F"],
                       capture_output=True, text=True, timeout=600, env={**os.environ, **env})
    assert r.returncode == 8
    assert "Initialization failed." in r.stdout
