"""PreSCRIMP on the GPU (mp_prescrimp) against the reference's own PreSCRIMP
(golden outputs of ScrimpppOrig.cpp, tests/golden/prescrimp_ref.npz) and
against the CPU restatement (oracle/prescrimp.py, itself pinned to those
outputs): same queries, same exclusion rule, same diagonal walks.  Values are
compared within 1e-9 relative (direct dot products on both sides, summed in
different orders; the reference's FFT rows where its tolerance says so) and a
differing index must tie in distance."""
from __future__ import annotations

import os
import subprocess

import numpy as np
import pytest

import thesiscode_b200 as mp
from oracle.prescrimp import prescrimp as ref_prescrimp
from thesiscode_b200 import workloads
from thesiscode_b200.error_report import pair_distance

pytestmark = pytest.mark.gpu


def _check(x, m, got, want):
    d_g, i_g = np.sqrt(np.abs(got.dist2)), got.index
    d_w, i_w = np.sqrt(np.abs(want[0])), want[1]
    fin = np.isfinite(d_w)
    assert np.array_equal(np.isfinite(d_g), fin)
    assert np.allclose(d_g[fin], d_w[fin], rtol=1e-9, atol=1e-12)
    for w in np.nonzero(i_g != i_w)[0]:
        a = pair_distance(x, m, int(w), int(i_g[w]))
        b = pair_distance(x, m, int(w), int(i_w[w]))
        assert a == pytest.approx(b, rel=1e-9, abs=1e-12), (w, i_g[w], i_w[w])


def test_prescrimp_matches_reference_golden(gpu_ctx, golden_prescrimp):
    from test_prescrimp_oracle import check_against_reference, golden_rtol
    for name, c in golden_prescrimp.items():
        m, stride = int(c["m"]), int(c["stride"])
        got = gpu_ctx.prescrimp(c["x"], m, float(stride))
        check_against_reference(c["x"], m, got.dist2, got.index, c["dist"],
                                c["index"].astype(np.int64), rtol=golden_rtol(name))


@pytest.mark.parametrize("n,m,stride", [(5000, 64, 0.25), (8000, 100, 1.0), (3000, 50, 100.0),
                                        (20000, 128, 0.5), (4096, 17, 2.0)])
def test_prescrimp_matches_restatement(gpu_ctx, n, m, stride):
    x = workloads.random_walk(n, n + m)
    got = gpu_ctx.prescrimp(x, m, stride)
    _check(x, m, got, ref_prescrimp(x, m, stride))


def test_prescrimp_device_buffers(gpu_ctx):
    import torch
    x = workloads.random_walk(6000, 11)
    m = 80
    host = gpu_ctx.prescrimp(x, m, 0.5)
    xd = torch.from_numpy(x).cuda()
    d2 = torch.empty(x.size - m + 1, dtype=torch.float64, device="cuda")
    ix = torch.empty(x.size - m + 1, dtype=torch.int64, device="cuda")
    gpu_ctx.prescrimp(xd, m, 0.5, out=(d2, ix))
    assert np.array_equal(d2.cpu().numpy(), host.dist2)
    assert np.array_equal(ix.cpu().numpy(), host.index)


def test_prescrimp_rejects_zero_step(gpu_ctx):
    with pytest.raises(mp.MpError):
        gpu_ctx.prescrimp(workloads.random_walk(1000, 1), 64, 0.001)


def test_cli_scrimppp_writes_prescrimp_and_exact_profiles(tmp_path, golden_ascii):
    from thesiscode_b200 import validate
    x = golden_ascii["series"]
    inp = tmp_path / "test.ascii"
    inp.write_text(" ".join(repr(float(v)) for v in x))
    out = tmp_path / "prof.ascii"
    r = subprocess.run([mp.CLI_PATH, "gpu_scrimppp", "64", "1", str(inp), "--output-file", str(out)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    pre = validate.read_profile(str(out) + "_prescrimp")
    want = ref_prescrimp(x, 64, 1.0)
    assert np.allclose(pre[0], np.sqrt(np.abs(want[0])), rtol=1e-9)
    exact = validate.read_profile(str(out))
    assert np.array_equal(exact[1], golden_ascii["idx_m64"])
    assert np.array_equal(exact[0], np.sqrt(np.abs(golden_ascii["d2_m64"])))
    assert os.path.getsize(str(out) + "_prescrimp") > 0


@pytest.mark.parametrize("case", ["chirp_n2048_m64_s1", "walk_n1500_m50_s1",
                                  "readme_test_ascii_m400_s100"])
def test_cli_scrimppp_final_profile_is_the_reference(tmp_path, golden_prescrimp, case):
    # gpu_scrimppp's two files against the reference scrimppp_orig's; on the
    # chirped sine hundreds of neighbours lie exactly m/4 away, where only
    # PreSCRIMP looks
    from test_prescrimp_oracle import check_against_reference, golden_rtol
    from thesiscode_b200 import validate
    c = golden_prescrimp[case]
    x, m, stride = c["x"], int(c["m"]), int(c["stride"])
    inp = tmp_path / "series.ascii"
    inp.write_text(" ".join(repr(float(v)) for v in x))
    out = tmp_path / "prof.ascii"
    r = subprocess.run([mp.CLI_PATH, "gpu_scrimppp", str(m), str(stride), str(inp),
                        "--output-file", str(out)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    for path, dist, index in ((str(out) + "_prescrimp", c["dist"], c["index"]),
                              (str(out), c["exact_dist"], c["exact_index"])):
        d, i = validate.read_profile(path)
        check_against_reference(x, m, d * d, i, dist, index.astype(np.int64), rtol=golden_rtol(case))
