"""The reference's file formats, byte for byte.

Input CSV (README.md:31-47, loadData euclideandistancematrixgpu.cu:2712-2757,
main.cpp:84-101):
    line 1: number of points N; line 2: number of dimensions d;
    then one point per line, features separated by ',', each token trimmed of
    spaces and parsed with atof; with the cluster flag the last token is an
    integer cluster id.  Tokens are cut with strtok, so empty tokens vanish.

Binary result (saveResultToResultFile, .cu:2908-2978):
    text header "<N>;<k>;8\\n" (the README says dimensions, the code writes k),
    the 8-byte little-endian long 0x01020304,
    then for every point its k records of 8 bytes each, written from a
    DataPoint{int id; float distance} (.h:45-48) as sizeof(long) bytes: the low
    4 bytes are the int32 id, the high 4 bytes the float32 stored distance.
    Stored distance: L2 for EUCLIDEAN, sqrt(L1) for TAXICAB (.cu:567-570) and the
    cosine similarity 1 - (1 - cos) for COSINE (.cu:1007), records ordered by
    distance ascending (similarity descending for COSINE, .cu:2938-2942).
Side files: "<out>VALIDATION" holding "Everything is OK." (.cu:2967-2971) and,
with --debug, "<out>DEBUG" lines "NEAR: <i, j>(dist) ... ;" (.cu:2946-2961).
"""
from __future__ import annotations

import numpy as np

MAGIC = 0x01020304


def _atof(tok: str) -> float:
    """C atof: the longest numeric prefix, 0.0 when there is none."""
    tok = tok.strip()
    try:
        return float(tok)
    except ValueError:
        pass
    best = 0.0
    for end in range(len(tok), 0, -1):
        try:
            best = float(tok[:end])
            break
        except ValueError:
            continue
    return best


def _atoi(tok: str) -> int:
    tok = tok.strip()
    sign, i = 1, 0
    if tok[:1] in "+-":
        sign = -1 if tok[0] == "-" else 1
        i = 1
    j = i
    while j < len(tok) and tok[j].isdigit():
        j += 1
    return sign * int(tok[i:j]) if j > i else 0


def read_header(path: str) -> tuple[int, int]:
    """N and d from the first two lines (main.cpp:88-101, atoi semantics)."""
    with open(path, "r") as f:
        n = _atoi(f.readline())
        d = _atoi(f.readline())
    return n, d


def read_csv(path: str, n: int | None = None, d: int | None = None, klaster: bool = False):
    """Points float32 [n, d] and cluster ids int32 [n] (zeros without the flag)."""
    hn, hd = read_header(path)
    n = hn if n is None else n
    d = hd if d is None else d
    x = np.zeros((n, d), dtype=np.float32)
    labels = np.zeros(n, dtype=np.int32)
    with open(path, "r") as f:
        f.readline()
        f.readline()
        row = 0
        for line in f:
            if row >= n:
                break
            toks = [t for t in line.rstrip("\r\n").split(",") if t != ""]
            toks = [t.strip(" ") for t in toks]
            if klaster and toks:
                labels[row] = _atoi(toks[-1])
                toks = toks[:-1]
            vals = [_atof(t) for t in toks[:d]]
            x[row, : len(vals)] = vals
            row += 1
    return x, labels


def write_csv(path: str, x: np.ndarray, labels: np.ndarray | None = None) -> None:
    """CSV in the reference's input format (float32 values, repr precision)."""
    x = np.asarray(x, dtype=np.float32)
    with open(path, "w") as f:
        f.write(f"{x.shape[0]}\n{x.shape[1]}\n")
        for i in range(x.shape[0]):
            line = ", ".join(repr(float(v)) for v in x[i])
            if labels is not None:
                line += f", {int(labels[i])}"
            f.write(line + "\n")


def write_csv_integers(path: str, x: np.ndarray) -> None:
    """CSV in the reference's input format for non-negative integer values
    below 1000 (the integer-mixture points), written without per-value
    formatting: every value takes three characters, left-padded with spaces,
    which the reference's reader trims before atof (trim, .cu:1987-1995)."""
    x = np.asarray(x)
    n, d = x.shape
    v = np.rint(x).astype(np.int64)
    if v.size and (v.min() < 0 or v.max() > 999 or not np.array_equal(v, x)):
        raise ValueError("write_csv_integers takes integers in [0, 999]")
    table = np.frombuffer(b"".join(b"%3d" % i for i in range(1000)), dtype=np.uint8).reshape(1000, 3)
    with open(path, "wb") as f:
        f.write(f"{n}\n{d}\n".encode())
        step = 1 << 16
        for s in range(0, n, step):
            blk = v[s:s + step]
            out = np.empty((blk.shape[0], d, 4), dtype=np.uint8)
            out[:, :, :3] = table[blk]
            out[:, :, 3] = ord(",")
            out[:, -1, 3] = ord("\n")
            f.write(out.tobytes())


def write_csv_fixed(path: str, x: np.ndarray, decimals: int = 9) -> np.ndarray:
    """CSV in the reference's input format for values in (-1000, 1000): exact
    zeros as "0", every other value in fixed point, with a sign when negative
    and ``decimals`` digits after the point (no per-value formatting, so a
    multi-GB file takes seconds).  Returns the float32 values a reader parses
    back (the written decimals, rounded)."""
    x = np.asarray(x, dtype=np.float32)
    n, d = x.shape
    if x.size and (x.min() <= -1000 or x.max() >= 1000):
        raise ValueError("write_csv_fixed takes values in (-1000, 1000)")
    scale = 10 ** decimals
    parsed = np.empty_like(x)
    with open(path, "wb") as f:
        f.write(f"{n}\n{d}\n".encode())
        step = 4096
        for s in range(0, n, step):
            blk = x[s:s + step].astype(np.float64)
            m = np.rint(blk * scale).astype(np.int64)
            zero = m == 0
            parsed[s:s + step] = (m / scale).astype(np.float32)
            neg = m < 0
            am = np.abs(m)
            ip = am // scale
            ndig = 1 + (ip >= 10) + (ip >= 100)
            w = np.where(zero, 1, neg + ndig + 1 + decimals) + 1  # token + separator
            ends = np.cumsum(w, axis=1)
            starts = ends - w
            row_len = ends[:, -1]
            row_off = np.concatenate(([0], np.cumsum(row_len)[:-1]))
            buf = np.empty(int(row_len.sum()), dtype=np.uint8)
            pos = row_off[:, None] + starts
            buf[pos[zero]] = ord("0")
            nz = ~zero
            pz, iz, dz, gz = pos[nz], ip[nz], ndig[nz], neg[nz]
            buf[pz[gz]] = ord("-")
            p0 = pz + gz  # first digit
            for j in range(3):  # integer digits, most significant first
                has = dz > j
                digit = (iz // (10 ** (dz - 1 - j).clip(0))) % 10
                buf[(p0 + j)[has]] = (digit[has] + ord("0")).astype(np.uint8)
            pdot = p0 + dz
            buf[pdot] = ord(".")
            frac = am[nz] % scale
            for j in range(decimals):
                buf[pdot + decimals - j] = (frac % 10 + ord("0")).astype(np.uint8)
                frac //= 10
            sep = row_off[:, None] + ends - 1
            buf[sep] = ord(",")
            buf[sep[:, -1]] = ord("\n")
            f.write(buf.tobytes())
    return parsed


def stored_distance(dist: np.ndarray, metric: int) -> np.ndarray:
    """Value the reference stores for a returned distance (see module doc)."""
    dist = np.asarray(dist, dtype=np.float32)
    if metric == 1:
        return np.sqrt(dist).astype(np.float32)
    if metric == 2:
        return (1.0 - dist.astype(np.float64)).astype(np.float32)
    return dist


def _fmt_g(v: float) -> str:
    """C++ ostream default float formatting (%g, 6 significant digits)."""
    return "%g" % v


def write_result(path: str, idx: np.ndarray, dist: np.ndarray, metric: int,
                 debug: bool = False) -> None:
    """Binary result file plus VALIDATION (and DEBUG) side files."""
    idx = np.ascontiguousarray(idx, dtype=np.int32)
    n, k = idx.shape
    stored = stored_distance(dist, metric)
    rec = np.empty((n, k, 2), dtype=np.uint32)
    rec[:, :, 0] = idx.view(np.uint32)
    rec[:, :, 1] = stored.view(np.uint32)
    with open(path, "wb") as f:
        f.write(f"{n};{k};8\n".encode())
        f.write(np.int64(MAGIC).tobytes())
        f.write(rec.astype("<u4").tobytes())
    with open(path + "VALIDATION", "wb") as f:
        f.write(b"Everything is OK.")
    if debug:
        with open(path + "DEBUG", "wb") as f:
            for i in range(n):
                parts = [f"NEAR: <{i}, {int(idx[i, j])}>({_fmt_g(float(stored[i, j]))}) "
                         for j in range(k)]
                f.write(("".join(parts) + ";\n").encode())


def read_result(path: str):
    """(N, k, idx int32 [N, k], stored float32 [N, k]) from a binary result file."""
    with open(path, "rb") as f:
        data = f.read()
    nl = data.index(b"\n")
    n_s, k_s, sz_s = data[:nl].decode().split(";")
    n, k, sz = int(n_s), int(k_s), int(sz_s)
    if sz != 8:
        raise ValueError(f"record size {sz} != 8")
    magic = int(np.frombuffer(data[nl + 1: nl + 9], dtype="<i8")[0])
    if magic != MAGIC:
        raise ValueError(f"bad magic {magic:#x}")
    body = np.frombuffer(data[nl + 9: nl + 9 + n * k * 8], dtype="<u4").reshape(n, k, 2)
    return n, k, body[:, :, 0].view(np.int32).copy(), body[:, :, 1].view(np.float32).copy()
