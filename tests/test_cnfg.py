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


# ---------------------------------------------------------------------------
# import into a context: the stored plaquette is checked (openQCD's import_cnfg)
# ---------------------------------------------------------------------------
@pytest.mark.gpu
@pytest.mark.parametrize("bc,prec", [(3, "fp64"), (0, "fp64"), (3, "mixed")])
def test_context_import_checks_the_plaquette(tmp_path, bc, prec):
    from tests import oracle as O
    from wloop_b200 import Context
    from wloop_b200.api import plaquette_count
    n = (8, 4, 6, 4)
    u = generate_links(n, bc, 31, 0.3)
    want = O.plaq_sum(n, bc, u) / plaquette_count(n, bc)
    good = str(tmp_path / "goodn1")
    M.export_cnfg(good, u, n, want)
    with Context(n, bc, prec) as c:
        got = c.import_cnfg(good)
        assert abs(got - want) <= 1e-14
        if prec == "fp64":
            assert np.array_equal(c.download(), u)
        # a head whose plaquette differs from the field's by more than
        # sqrt(nplaq) DBL_EPSILON is refused
        bad = str(tmp_path / "badn1")
        M.export_cnfg(bad, u, n, want + 1e-11)
        with pytest.raises(WlgError, match="Incorrect average plaquette"):
            c.import_cnfg(bad)
        # as is a field whose links were changed after the head was written
        v = u.copy()
        v[5, 2] = v[5, 2] @ v[9, 1]
        M.export_cnfg(bad, v, n, want)
        with pytest.raises(WlgError, match="Incorrect average plaquette"):
            c.import_cnfg(bad)
        # export writes the field's own plaquette, and it imports again
        out = str(tmp_path / "outn1")
        c.import_cnfg(good)
        p = c.export_cnfg(out)
        assert abs(p - want) <= (1e-14 if prec == "fp64" else 1e-6)
        assert abs(c.import_cnfg(out) - p) <= 1e-14


@pytest.mark.gpu
def test_run_imports_exported_files_and_logs_plaquettes(tmp_path):
    """measure.run on exported files (ms10's cnfg_dir naming): .dat records
    equal Context.measure, the .par has the bc record then the wloop record,
    and the log holds the average plaquette after HYP and after every level."""
    from tests import oracle as O
    from wloop_b200 import Context
    from wloop_b200.api import APE, WloopParms, plaquette_count
    n, bc = (8, 4, 4, 4), 0
    p = WloopParms(msl=3, nss=[0, 2, 2], mwlt=3, mwlr=2, op_smear=APE, alpha_ape=0.5,
                   proj_iter=4)
    cdir = tmp_path / "cnfg"
    cdir.mkdir()
    fields = {}
    for nc in (1, 2):
        fields[nc] = generate_links(n, bc, 40 + nc, 0.3)
        M.export_cnfg(str(cdir / f"runn{nc}"), fields[nc], n,
                      O.plaq_sum(n, bc, fields[nc]) / plaquette_count(n, bc))
    r = M.Run("run", n, bc, p, first=1, last=2, precision="fp64")
    M.run(r, str(tmp_path), cnfg_dir=str(cdir))
    _, ncs, wl = M.read(M.dat_path(str(tmp_path), "run"))
    M.check_par(M.par_path(str(tmp_path), "run"), p, bc=bc)
    log = open(M.log_path(str(tmp_path), "run")).read().splitlines()
    with Context(n, bc, "fp64") as c:
        for k, nc in enumerate(ncs):
            c.upload(fields[nc])
            assert np.array_equal(c.measure(p), wl[k])
    nplaq = plaquette_count(n, bc)
    uh = O.hyp_links(n, bc, fields[2], *p.alpha_action, p.proj, p.proj_iter)
    _, pl = O.wloop_sum(n, bc, uh, p, want_plaq=True)
    hyp_line = [ln for ln in log if ln.startswith("Average plaquette after HYP")][1]
    assert abs(float(hyp_line.split("=")[1]) - O.plaq_sum(n, bc, uh) / nplaq) < 1e-13
    lv = [ln for ln in log if ln.startswith("Average plaquette at smearing level")][3:6]
    for sl, ln in enumerate(lv):
        assert abs(float(ln.split("=")[1]) - pl[sl] / nplaq) < 1e-13
    assert sum(ln.startswith("Configuration no") and "fully processed" in ln for ln in log) == 2
