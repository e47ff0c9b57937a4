"""The CUDA library on a machine without a GPU: it loads, exports every entry
point include/pimc_b200.h declares, and its host-side .dm reader agrees
bitwise with the oracle's and with the golden arrays."""
import os
import re

import numpy as np
import pytest

import oracle as O
import pimcplusplus_b200 as P
from helpers import ROOT, coulomb_fit2_tables, write_testcoul_dm
from pimcplusplus_b200 import workloads as W


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "pimc_b200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(pimc_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    syms = declared_symbols()
    assert len(syms) >= 25
    for s in syms:
        assert hasattr(P.lib(), s), s
    assert set(syms) <= set(P.EXPORTED) | {"pimc_stream"}


def test_status_strings():
    assert P.lib().pimc_status_string(0) == b"ok"
    assert P.lib().pimc_version() >= 100


def test_product_dm_reader_matches_oracle_lj(tmp_path):
    cfg = W.CONFIGS["C1"]
    tau, box = W.derived(cfg)
    dm = W.make_dm_for(cfg, str(tmp_path))
    t = P.read_dm(dm, tau)
    pa = O.PairAction.from_dm(dm, tau, 0)
    assert t["tau_pos"] == pa.info()["tau_pos"] == 0
    for lev in range(t["num_tau"]):
        for w, k in ((0, "ukj"), (1, "ukj_d2"), (2, "dukj"), (3, "dukj_d2")):
            assert np.array_equal(pa.table(w, lev), t[k][lev])


def test_product_dm_reader_matches_golden(tmp_path):
    p = write_testcoul_dm(str(tmp_path / "tc.dm"))
    t = P.read_dm(p, 1.0 / 32)
    g, u, du = coulomb_fit2_tables()
    assert t["tau_pos"] == 1 and t["grid_type"] == P.GRID_LOG
    assert np.array_equal(t["ukj"], u) and np.array_equal(t["dukj"], du)


def test_product_dm_reader_errors(tmp_path):
    with pytest.raises(P.PimcError):
        P.read_dm(str(tmp_path / "missing.dm"), 0.01)
    bad = tmp_path / "bad.dm"
    bad.write_text(" SQUARER 1. 7 3 3 60 14\n RANK 2 10 1\n")
    with pytest.raises(P.PimcError):
        P.read_dm(str(bad), 0.01)
    p = write_testcoul_dm(str(tmp_path / "tc.dm"))
    with pytest.raises(P.PimcError):  # tau not on the file's tau grid
        P.read_dm(p, 0.3)
