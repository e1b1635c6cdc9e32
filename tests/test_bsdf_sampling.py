"""Sampling statistics of the CUDA StandardBSDF lobes, with the reference's own
BSDF unit test (Tools/FalcorTest/Tests/Scene/Material/BSDFTests.cpp:242-470)
as the specification: for each lobe and incident direction, 64 M samples
binned over 130 (phi) x 65 (cos theta) cells are compared with the integral of
evalPdf over each cell by a chi^2 test (cells below an expected count of 5
pooled, significance 0.01 with the Sidak correction over the lobe's
configurations), and every sample's weight and pdf must agree with eval /
evalPdf within 1e-3 relative.  The chi^2 test restates
hypothesis::chi2_test (external/include/hypothesis/hypothesis.h:143-240 in the
reference tree, a third-party header-only library) with scipy's chi^2
distribution.  The same test, compiled unmodified, passes against the CPU
oracle (tests/test_oracle_pinning.py).
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

PERP = (0.0, 0.0, 1.0)
OBLIQUE = tuple(np.array([0.5, 0.0, 0.5]) / np.linalg.norm([0.5, 0.0, 0.5]))
GRAZING = tuple(np.array([0.0, 1.0, 0.01]) / np.linalg.norm([0.0, 1.0, 0.01]))
DIRS = {"perp": PERP, "oblique": OBLIQUE, "grazing": GRAZING}

# (lobe id, name, [(config name, wi, params)]) as BSDFTests.cpp:300-470 sets them.
CASES = [
    (0, "FrostbiteDiffuseBRDF", [(n, d, (0.5, 0, 0, 0)) for n, d in DIRS.items()]),
    (1, "LambertDiffuseBRDF", [(n, d, (0, 0, 0, 0)) for n, d in DIRS.items()]),
    (2, "LambertDiffuseBTDF", [(n, d, (0, 0, 0, 0)) for n, d in DIRS.items()]),
    (3, "SpecularMicrofacetBRDF", [(f"{r}_{n}", d, (a, 0, 0, 0)) for r, a in (("smooth", 0.05), ("rough", 0.5))
                                   for n, d in DIRS.items()]),
]
PHI_BINS, COS_BINS = 128 + 2, 64 + 1
SAMPLES, THREAD_SAMPLES, BIN_SAMPLES = 64 * 1024 * 1024, 128 * 1024, 128


def chi2_test(obs, exp, sample_count, min_exp=5.0, significance=0.01, num_tests=1):
    """hypothesis::chi2_test: cells sorted by expected count, low ones pooled."""
    from scipy.stats import chi2
    order = np.argsort(exp, kind="stable")
    pooled_obs = pooled_exp = chsq = 0.0
    dof = 0
    for i in order:
        e, o = exp[i], obs[i]
        if e < 0:
            return False, "negative expected frequency"
        if e == 0:
            if o > sample_count * 1e-5:
                return False, f"{o} samples in a cell with expected frequency 0"
        elif e < min_exp or (0 < pooled_exp < min_exp):
            pooled_obs += o
            pooled_exp += e
        else:
            chsq += (o - e) ** 2 / e
            dof += 1
    if pooled_exp > 0 or pooled_obs > 0:
        chsq += (pooled_obs - pooled_exp) ** 2 / pooled_exp
        dof += 1
    dof -= 1
    if dof <= 0:
        return False, f"dof {dof}"
    pval = float(chi2.sf(chsq, dof))
    alpha = 1.0 - (1.0 - significance) ** (1.0 / num_tests)
    return (pval >= alpha and np.isfinite(pval)), f"chi2 {chsq:.1f} dof {dof} p {pval:.4f} alpha {alpha:.5f}"


@pytest.mark.parametrize("lobe,name,configs", CASES, ids=[c[1] for c in CASES])
def test_bsdf_lobe_sampling_statistics(fpt, lobe, name, configs):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from falcor_b200 import _ffi
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    bins = PHI_BINS * COS_BINS
    report = []
    for cname, wi, params in configs:
        p = _ffi.fpt_bsdf_probe(lobe=lobe, sample_count=SAMPLES, thread_sample_count=THREAD_SAMPLES, phi_bins=PHI_BINS,
                                cos_bins=COS_BINS, bin_sample_count=BIN_SAMPLES)
        for k in range(3):
            p.wi[k] = wi[k]
        for k in range(4):
            p.params[k] = params[k]
        hist = torch.zeros(bins, dtype=torch.int32, device="cuda")
        werr = torch.zeros(bins, dtype=torch.int32, device="cuda")
        perr = torch.zeros(bins, dtype=torch.int32, device="cuda")
        pdf = torch.zeros(bins, dtype=torch.float64, device="cuda")
        _ffi.check(fpt.fpt_bsdf_probe_run(C.byref(p), hist.data_ptr(), werr.data_ptr(), perr.data_ptr(), pdf.data_ptr(), stream))
        torch.cuda.synchronize()
        obs = hist.cpu().numpy().view(np.uint32).astype(np.float64)
        exp = pdf.cpu().numpy()
        ok, msg = chi2_test(obs, exp, SAMPLES, num_tests=len(configs))
        max_w = float(werr.cpu().numpy().view(np.float32).max())
        max_p = float(perr.cpu().numpy().view(np.float32).max())
        report.append(f"{name}_{cname}: {msg}, max weight error {max_w:.2e}, max pdf error {max_p:.2e}")
        assert ok, report[-1]
        assert max_w <= 1e-3, report[-1]
        assert max_p <= 1e-3, report[-1]
        assert obs.sum() > 0.1 * SAMPLES
    print("\n".join(report))
