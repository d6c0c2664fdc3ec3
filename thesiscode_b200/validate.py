"""Profile comparison and validation, with the reference's two utilities'
behaviour and summaries:

  compare   two profile files entry by entry, as
            scrimppp/utils/compare_profile_indices.py does: counts entries
            whose neighbour indices differ, reports the largest absolute
            difference of the profile values (distances), and exits with the
            number of differing entries (capped at 255 so that a count never
            wraps to a "success" exit status).
  folder    every group of result files of one experiment in a directory, as
            scrimppp/utils/validate_profiles.py does: files are named
            ``matprof_v<data-id>_l<length>m<window>...alg#<algorithm>#..._p<workers>_...``;
            each group is compared against the scrimppp_orig result (or
            scrimp_sequ, unless --force_orig_baseline) or pairwise in order.

Both read ASCII profiles (``distance index`` per line,
scrimppp/src/ScrimpSequ.cpp:275-276) and binary profiles (format 1: a 100-byte
header {u32 format, u32 data offset, u64 count} and {f64 squared distance,
u64 index} records, scrimppp/src/binproffile.cpp:49-127) directly; binary
squared distances are compared as distances, like the reference's converted
files.  No conversion utility is needed.

Ties: with ``--series FILE --window M`` an index difference is accepted when
the two neighbours' distances, computed directly from the series (centred
two-pass FP64 dot products), agree within ``--rel-tol`` (default 1e-9, the
FP64 form's tolerance).  The reference breaks exact ties by its shuffled
block order, so equal-distance neighbours legitimately differ between runs.

    python -m thesiscode_b200.validate compare a.matprof.ascii b.matprof.bin
    python -m thesiscode_b200.validate compare a b --series ts.ascii --window 400
    python -m thesiscode_b200.validate folder results/
"""
from __future__ import annotations

import argparse
import math
import os
import re
import struct
import sys

import numpy as np

from thesiscode_b200.error_report import pair_distance

HEADER_BYTES = 100
FMT_PROFILE = 1
FMT_SERIES = 2


def _is_binary(path: str, fmt: int) -> bool:
    if path.endswith(".bin"):
        return True
    with open(path, "rb") as f:
        head = f.read(16)
    if len(head) < 16:
        return False
    f0, off, _ = struct.unpack("<IIQ", head)
    return f0 == fmt and off == HEADER_BYTES


def _read_binary(path: str, fmt_want: int, dtype, what: str) -> np.ndarray:
    """The payload of a binary file in the reference's format, its header's
    count checked against the file's size before anything is read."""
    with open(path, "rb") as f:
        head = f.read(16)
        if len(head) < 16:
            raise ValueError(f"{path}: no binary header")
        fmt, off, count = struct.unpack("<IIQ", head)
        if fmt != fmt_want or off != HEADER_BYTES:
            raise ValueError(f"{path}: not a binary {what} file (format {fmt}, offset {off})")
        width = np.dtype(dtype).itemsize
        have = max(os.path.getsize(path) - off, 0) // width
        if count > have:
            raise ValueError(f"{path}: truncated ({have} of {count} {what} entries)")
        f.seek(off)
        return np.frombuffer(f.read(width * count), dtype=dtype).copy()


def read_profile(path: str):
    """(distances, indices) of an ASCII or binary (format 1) profile file."""
    if _is_binary(path, FMT_PROFILE):
        rec = _read_binary(path, FMT_PROFILE, [("d2", "<f8"), ("idx", "<u8")], "profile")
        return np.sqrt(np.abs(rec["d2"])), rec["idx"].astype(np.int64)
    dist, idx = [], []
    with open(path) as f:
        for line in f:
            parts = line.split()
            if not parts:
                continue
            dist.append(float(parts[0]))
            idx.append(int(parts[1]))
    return np.array(dist, dtype=np.float64), np.array(idx, dtype=np.int64)


def read_series(path: str) -> np.ndarray:
    """A time series from an ASCII file (whitespace-separated values) or a
    binary series file (format 2)."""
    if _is_binary(path, FMT_SERIES):
        return _read_binary(path, FMT_SERIES, "<f8", "series")
    with open(path) as f:
        return np.array(f.read().split(), dtype=np.float64)


def write_profile_ascii(path: str, d2, idx) -> None:
    """ASCII profile: sqrt(|d2|) with 17 significant digits and the index."""
    with open(path, "w") as f:
        for v, i in zip(np.asarray(d2, dtype=np.float64), np.asarray(idx)):
            f.write(f"{math.sqrt(abs(v)):.17g} {int(i)}\n")


def write_profile_bin(path: str, d2, idx) -> None:
    """Binary profile, format 1 (squared distances)."""
    d2 = np.asarray(d2, dtype=np.float64)
    rec = np.empty(d2.size, dtype=[("d2", "<f8"), ("idx", "<u8")])
    rec["d2"] = d2
    rec["idx"] = np.asarray(idx).astype(np.int64).astype(np.uint64)
    with open(path, "wb") as f:
        f.write(struct.pack("<IIQ", FMT_PROFILE, HEADER_BYTES, d2.size).ljust(HEADER_BYTES, b"\0"))
        f.write(rec.tobytes())


def compare_profiles(a, b, series=None, m: int | None = None, rel_tol: float = 1e-9):
    """Compares two (distances, indices) profiles entry by entry."""
    da, ia = a
    db, ib = b
    n = min(da.size, db.size)
    length_diff = abs(da.size - db.size)
    diff = np.nonzero(ia[:n] != ib[:n])[0]
    ties = 0
    if series is not None and diff.size:
        for i in diff:
            ea = pair_distance(series, m, int(i), int(ia[i]))
            eb = pair_distance(series, m, int(i), int(ib[i]))
            if np.isfinite(ea) and np.isfinite(eb) and abs(ea - eb) <= rel_tol * max(ea, eb):
                ties += 1
    with np.errstate(invalid="ignore"):
        delta = np.abs(da[:n] - db[:n])
    max_diff = float(np.nanmax(delta)) if n else 0.0
    return {"entries": n + length_diff, "index_differences": int(diff.size) - ties + length_diff,
            "ties_within_tolerance": ties, "length_difference": length_diff,
            "shorter": 0 if da.size == db.size else (2 if db.size < da.size else 1),
            "max_abs_diff": max_diff, "differing_entries": diff,
            "index_pairs": [(int(ia[i]), int(ib[i])) for i in diff[:1000]]}


def _print_compare(rep, silent: bool) -> None:
    # the messages of the reference's compare_profile_indices.py
    if not silent:
        for i, (x, y) in zip(rep["differing_entries"][:1000], rep["index_pairs"]):
            print(f"l {i + 1} has differing indices, id1: {x} id2: {y}")
    if rep["shorter"] == 2:
        print("FATAL: file 2 is shorter than file 1!")
    elif rep["shorter"] == 1:
        print("FATAL: file 1 is shorter than file 2!")
    if rep["index_differences"] == 0:
        print("SUCCESS: The profile indices coincide in all %d entries" % rep["entries"])
    else:
        print("ERROR: Profile indices differ in %d entries" % rep["index_differences"])
    if rep["ties_within_tolerance"]:
        print("index differences accepted as distance ties within tolerance: %d"
              % rep["ties_within_tolerance"])
    print("maximum absolute difference in profile values: %r" % rep["max_abs_diff"])


_NAME = re.compile(r"matprof_v(\d+)_l(\d+)m(\d+)")


def experiment_of(fname: str):
    m = _NAME.search(fname)
    if not m:
        raise ValueError(f"{fname}: file name does not match the validation job pattern")
    return int(m.group(1)), int(m.group(2)), int(m.group(3))


def _algo_of(fname: str) -> str:
    m = re.search(r"alg#(\S+?)#", fname)
    return m.group(1) if m else "?"


def _procs_of(fname: str):
    m = re.search(r"_p(\d+)_", fname)
    return int(m.group(1)) if m else None


def validate_folder(folder: str, force_orig_baseline: bool = False, out=sys.stdout) -> int:
    """Returns 0 when every group's indices coincide, 1 otherwise."""
    files = sorted(f for f in os.listdir(folder) if _NAME.search(f))
    groups = {}
    for f in files:
        groups.setdefault(experiment_of(f), []).append(f)
    max_diff, ncmp = 0.0, 0
    for exp, members in sorted(groups.items()):
        cfg = "data-id %d, time-series length %d, window-length %d" % exp
        print("Processing set of result files with the configuration: " + cfg, file=out)
        if len(members) < 2:
            print(f"VALIDATION FAILED: {members[0]} has no other profile of the same configuration",
                  file=out)
            return 1
        base = next((f for f in members if _algo_of(f) == "scrimppp_orig"), None)
        if base is None and not force_orig_baseline:
            base = next((f for f in members if _algo_of(f) == "scrimp_sequ"), None)
        if base is None and force_orig_baseline:
            print("VALIDATION FAILED: no required baseline from original algorithm for "
                  "configuration " + cfg, file=out)
            return 1
        pairs = ([(base, f) for f in members if f != base] if base
                 else list(zip(members[:-1], members[1:])))
        for f1, f2 in pairs:
            rep = compare_profiles(read_profile(os.path.join(folder, f1)),
                                   read_profile(os.path.join(folder, f2)))
            print(f"comparing profiles {f1} and {f2}: {rep['index_differences']} index "
                  f"differences, max value difference {rep['max_abs_diff']:.3E}", file=out)
            if rep["index_differences"]:
                print(f"COMPARISON FAILED: comparing the profiles {f1} and {f2} failed.", file=out)
                return 1
            max_diff = max(max_diff, rep["max_abs_diff"])
            ncmp += 1
    print("-----------------------------------------------------------", file=out)
    print("VALIDATION SUCCESSFUL, SUMMARY:", file=out)
    print("All profile indices coincide", file=out)
    print("Overall maximum difference in profile values {:.3E}".format(max_diff), file=out)
    print("compared %d pairs of matrix profile result files" % ncmp, file=out)
    print("total number of result files used: %d" % len(files), file=out)
    print("number of different experiments (groups with same profile): %d" % len(groups), file=out)
    print("Various algorithms encountered: " + str(sorted({_algo_of(f) for f in files})), file=out)
    print("Various numbers of workers used for profile generation: "
          + str(sorted({p for p in map(_procs_of, files) if p is not None})), file=out)
    print("Various time series lengths used: " + str(sorted({e[1] for e in groups})), file=out)
    print("various window length used: " + str(sorted({e[2] for e in groups})), file=out)
    return 0


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description="compare or validate matrix profile files")
    sub = ap.add_subparsers(dest="cmd", required=True)
    c = sub.add_parser("compare", help="compare the profile indices of two profile files")
    c.add_argument("file1")
    c.add_argument("file2")
    c.add_argument("--silent", action="store_true")
    c.add_argument("--series", help="time series file: accept index differences between "
                                    "neighbours of equal distance")
    c.add_argument("--window", type=int, help="window length m (with --series)")
    c.add_argument("--rel-tol", type=float, default=1e-9)
    # accepted for command-line compatibility with compare_profile_indices.py;
    # binary profiles are read directly, so nothing is converted or kept
    c.add_argument("--keep_converted", action="store_true", help=argparse.SUPPRESS)
    c.add_argument("--cvt_prof_path", nargs=1, help=argparse.SUPPRESS)
    v = sub.add_parser("folder", help="validate all profiles of a validation job directory")
    v.add_argument("directory")
    v.add_argument("--force_orig_baseline", action="store_true")
    v.add_argument("--cvt_prof_path", nargs=1, help=argparse.SUPPRESS)  # as in validate_profiles.py
    a = ap.parse_args(argv)
    if a.cmd == "compare":
        if a.series and not a.window:
            ap.error("--series needs --window")
        series = read_series(a.series) if a.series else None
        rep = compare_profiles(read_profile(a.file1), read_profile(a.file2), series, a.window,
                               a.rel_tol)
        _print_compare(rep, a.silent)
        return min(rep["index_differences"], 255)
    if not os.path.isdir(a.directory):
        print("specified folder not existing, aborting")
        return 1
    print("operating on folder: " + a.directory)
    return validate_folder(a.directory, a.force_orig_baseline)


if __name__ == "__main__":
    sys.exit(main())
