"""Profile comparison/validation tool (the reference's compare_profile_indices.py
and validate_profiles.py behaviour): file formats, index-difference counting,
distance-tie acceptance and folder validation."""
from __future__ import annotations

import io

import numpy as np

from thesiscode_b200 import validate, workloads


def _profile(oracle, n=3000, m=50, seed=7):
    x = workloads.random_walk(n, seed)
    d2, idx = oracle.selfjoin(x, m)
    return x, m, d2, idx


def test_ascii_and_binary_round_trip(oracle, tmp_path):
    x, m, d2, idx = _profile(oracle)
    a, b = tmp_path / "p.ascii", tmp_path / "p.bin"
    validate.write_profile_ascii(str(a), d2, idx)
    validate.write_profile_bin(str(b), d2, idx)
    da, ia = validate.read_profile(str(a))
    db, ib = validate.read_profile(str(b))
    assert np.array_equal(ia, idx) and np.array_equal(ib, idx)
    assert np.array_equal(da, db)  # 17 significant digits round-trip the distance exactly
    rep = validate.compare_profiles((da, ia), (db, ib))
    assert rep["index_differences"] == 0 and rep["max_abs_diff"] == 0.0
    assert validate.main(["compare", str(a), str(b), "--silent"]) == 0


def test_differing_indices_are_counted(oracle, tmp_path, capsys):
    x, m, d2, idx = _profile(oracle)
    bad = idx.copy()
    bad[[3, 17, 400]] += 1
    a, b = tmp_path / "a.ascii", tmp_path / "b.ascii"
    validate.write_profile_ascii(str(a), d2, idx)
    validate.write_profile_ascii(str(b), d2, bad)
    assert validate.main(["compare", str(a), str(b)]) == 3
    out = capsys.readouterr().out
    assert "ERROR: Profile indices differ in 3 entries" in out
    assert f"l 4 has differing indices, id1: {idx[3]} id2: {bad[3]}" in out


def test_length_mismatch_fails(oracle, tmp_path, capsys):
    x, m, d2, idx = _profile(oracle)
    a, b = tmp_path / "a.ascii", tmp_path / "b.ascii"
    validate.write_profile_ascii(str(a), d2, idx)
    validate.write_profile_ascii(str(b), d2[:-5], idx[:-5])
    assert validate.main(["compare", str(a), str(b), "--silent"]) == 5
    assert "FATAL: file 2 is shorter than file 1!" in capsys.readouterr().out
    assert validate.main(["compare", str(b), str(a), "--silent"]) == 5
    assert "FATAL: file 1 is shorter than file 2!" in capsys.readouterr().out


def test_reference_conversion_flags_are_accepted(oracle, tmp_path):
    x, m, d2, idx = _profile(oracle)
    a, b = tmp_path / "a.ascii", tmp_path / "b.bin"
    validate.write_profile_ascii(str(a), d2, idx)
    validate.write_profile_bin(str(b), d2, idx)
    assert validate.main(["compare", str(a), str(b), "--silent", "--keep_converted",
                          "--cvt_prof_path", "./cvt_matprof"]) == 0


def test_equal_distance_neighbours_are_ties(oracle, tmp_path):
    rng = np.random.default_rng(3)
    base = np.cumsum(rng.standard_normal(300))
    x = np.concatenate([base, np.cumsum(rng.standard_normal(200)) + 50, base,
                        np.cumsum(rng.standard_normal(200)) - 50, base])
    m = 40
    d2, idx = oracle.selfjoin(x, m)
    # window 10 has exact copies at +500 and +1000: either is a correct neighbour
    other = idx.copy()
    other[10] = 1010 if idx[10] != 1010 else 510
    s, a, b = tmp_path / "ts.ascii", tmp_path / "a.ascii", tmp_path / "b.ascii"
    np.savetxt(s, x)
    validate.write_profile_ascii(str(a), d2, idx)
    validate.write_profile_ascii(str(b), d2, other)
    assert validate.main(["compare", str(a), str(b), "--silent"]) == 1
    assert validate.main(["compare", str(a), str(b), "--silent", "--series", str(s),
                          "--window", str(m)]) == 0
    # a non-tie stays an error
    other[20] = idx[20] + 7
    validate.write_profile_ascii(str(b), d2, other)
    assert validate.main(["compare", str(a), str(b), "--silent", "--series", str(s),
                          "--window", str(m)]) == 1


def test_folder_validation(oracle, tmp_path):
    x, m, d2, idx = _profile(oracle)
    n = x.size
    stem = f"matprof_v1_l{n}m{m}"
    validate.write_profile_ascii(str(tmp_path / f"{stem}_alg#scrimp_sequ#_p1_.ascii"), d2, idx)
    validate.write_profile_bin(str(tmp_path / f"{stem}_alg#gpu_vert_blocked_fp64#_p1_.bin"), d2, idx)
    validate.write_profile_bin(str(tmp_path / f"{stem}_alg#scrimp_triv_par#_p8_.bin"), d2, idx)
    out = io.StringIO()
    assert validate.validate_folder(str(tmp_path), out=out) == 0
    text = out.getvalue()
    assert "VALIDATION SUCCESSFUL" in text and "compared 2 pairs" in text
    assert "[1, 8]" in text
    # the orig-baseline requirement fails without a scrimppp_orig file
    assert validate.validate_folder(str(tmp_path), force_orig_baseline=True, out=io.StringIO()) == 1
    # a differing index fails the group
    bad = idx.copy()
    bad[0] += 1
    validate.write_profile_bin(str(tmp_path / f"{stem}_alg#scrimp_triv_par#_p8_.bin"), d2, bad)
    assert validate.validate_folder(str(tmp_path), out=io.StringIO()) == 1
