"""The squarer .dm reader on damaged files: truncated, with flipped bytes,
with header numbers replaced by nonsense (negative, zero, huge, NaN, text),
with chunks removed or repeated.  Every file either reads, with tables of
the shape the info call reports, or gives a status code; none crashes the
process (the reference's reader would abort or read past its arrays)."""
import random

import numpy as np

import pimcplusplus_b200 as P
from helpers import write_testcoul_dm


def _mutate(text, rng):
    t = list(text)
    kind = rng.randrange(5)
    if kind == 0:
        t = t[:rng.randrange(len(t))]
    elif kind == 1:
        for _ in range(rng.randrange(1, 50)):
            t[rng.randrange(len(t))] = chr(rng.randrange(32, 127))
    elif kind == 2:
        lines = "".join(t).split("\n")
        i = rng.randrange(min(12, len(lines)))
        toks = lines[i].split()
        if toks:
            toks[rng.randrange(len(toks))] = rng.choice(["-5", "0", "999999999", "1e308", "nan", "-1", "2147483647", "x"])
            lines[i] = " " + " ".join(toks)
        t = list("\n".join(lines))
    elif kind == 3:
        a = rng.randrange(len(t))
        del t[a:a + rng.randrange(1, 2000)]
    else:
        a = rng.randrange(len(t))
        t[a:a] = t[a:a + rng.randrange(1, 2000)]
    return "".join(t)


def test_damaged_dm_files_read_or_fail_cleanly(tmp_path):
    text = open(write_testcoul_dm(str(tmp_path / "tc.dm"))).read()
    rng = random.Random(11)
    outcomes = {"read": 0, "error": 0}
    for i in range(60):
        p = tmp_path / f"m{i}.dm"
        p.write_text(_mutate(text, rng))
        try:
            t = P.read_dm(str(p), 1.0 / 32)
        except P.PimcError:
            outcomes["error"] += 1
            continue
        outcomes["read"] += 1
        assert t["ukj"].shape == (t["num_tau"], t["num_grid"], t["num_cols"])
        assert 0 <= t["tau_pos"] < t["num_tau"]
    assert outcomes["error"] > 0 and outcomes["read"] > 0, outcomes


def test_dm_header_fields_out_of_range(tmp_path):
    """Every number on the SQUARER, RANK, GRID and BEGIN lines replaced by a
    value no table has (huge counts, negatives, zero, NaN, infinities): the
    reader returns a status code (huge counts once made it throw bad_alloc
    across the C ABI) or reads a table of sane shape."""
    lines = open(write_testcoul_dm(str(tmp_path / "tc.dm"))).read().split("\n")
    heads = [i for i, ln in enumerate(lines) if ln.split() and ln.split()[0] in ("SQUARER", "RANK", "GRID", "BEGIN")]
    p = tmp_path / "x.dm"
    errors = 0
    for i in heads:
        for k in range(1, len(lines[i].split())):
            for val in ("2147483647", "99999999999999", "-3", "0", "nan", "-inf"):
                toks = lines[i].split()
                toks[k] = val
                p.write_text("\n".join(lines[:i] + [" " + " ".join(toks)] + lines[i + 1:]))
                try:
                    t = P.read_dm(str(p), 1.0 / 32)
                except P.PimcError:
                    errors += 1
                    continue
                assert t["num_grid"] <= 1 << 24 and t["num_tau"] <= 64 and np.all(np.isfinite(t["ukj"][:, :-1]))
    assert errors > 100
