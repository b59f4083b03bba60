"""Gauge configurations in openQCD's exported format (the files ms10 reads,
main/ms10.c:709-718): byte layout, round trip, and the reader's checks.
The format is openQCD's (not part of the reference); no real exported file
is available here, so the layout is checked against its written definition."""
import os
import struct

import numpy as np
import pytest

from wloop_b200 import generate_links
from wloop_b200._native import WlgError
from wloop_b200 import measure as M


def lex(n, x):
    return x[3] + n[3] * (x[2] + n[2] * (x[1] + n[1] * x[0]))


def tagged_field(n):
    """entry (0,0) of U(s, mu) = 4 s + mu, the rest random"""
    vol = int(np.prod(n))
    u = generate_links(n, 3, 7, 0.3).copy()
    for s in range(vol):
        for mu in range(4):
            u[s, mu, 0, 0] = 4 * s + mu + 0.5j
    return u


def test_layout_and_round_trip(tmp_path):
    n = (4, 2, 4, 6)
    u = tagged_field(n)
    path = str(tmp_path / "runn1")
    M.export_cnfg(path, u, n, 0.625)
    raw = open(path, "rb").read()
    vol = int(np.prod(n))
    assert len(raw) == 16 + 8 + 4 * vol * 144
    assert struct.unpack("<4i", raw[:16]) == n
    assert struct.unpack("<d", raw[16:24])[0] == 0.625
    body = np.frombuffer(raw[24:], dtype="<f8").reshape(-1, 18)
    # file order: odd points lexicographically, 8 links each
    r = 0
    for x0 in range(n[0]):
        for x1 in range(n[1]):
            for x2 in range(n[2]):
                for x3 in range(n[3]):
                    x = [x0, x1, x2, x3]
                    if sum(x) % 2 == 0:
                        continue
                    for mu in range(4):
                        y = list(x)
                        y[mu] = (y[mu] - 1) % n[mu]
                        assert body[r, 0] == 4 * lex(n, x) + mu
                        assert body[r + 1, 0] == 4 * lex(n, y) + mu
                        r += 2
    assert r == 4 * vol
    v = M.import_cnfg(path)
    assert np.array_equal(v, u)
    assert M.cnfg_head(path) == (n, 0.625)


def test_reader_checks(tmp_path):
    n = (2, 2, 2, 4)
    u = generate_links(n, 0, 3, 0.2)
    path = str(tmp_path / "c")
    M.export_cnfg(path, u, n, 1.0)
    with pytest.raises(WlgError, match="expected"):
        M.import_cnfg(path, (2, 2, 4, 2))
    with open(path, "r+b") as f:
        f.truncate(os.path.getsize(path) - 8)
    with pytest.raises(WlgError, match="bytes"):
        M.import_cnfg(path, n)
    with pytest.raises(WlgError, match="even"):
        M.export_cnfg(str(tmp_path / "odd"), generate_links((3, 2, 2, 2), 3, 1, 0.1), (3, 2, 2, 2), 1.0)


def test_cnfg_source_naming(tmp_path):
    n = (2, 2, 2, 2)
    for nc in (4, 8):
        M.export_cnfg(str(tmp_path / f"runAn{nc}"), generate_links(n, 3, nc, 0.2), n, 1.0)
    src = M.cnfg_source(str(tmp_path), "runA", n)
    assert np.array_equal(src(8), generate_links(n, 3, 8, 0.2))
