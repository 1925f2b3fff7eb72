"""The grid_search command-line driver (bbrcit_kde_b200/grid_search/grid_search.cc):
the reference driver's configuration keys, steps and output files over the C ABI.

Tolerances: the driver writes numbers with 6 significant digits (as the
reference does), so values are compared at 1e-5 relative; the bandwidth it
selects must be the oracle's argmin of the same grid."""
from __future__ import annotations

import os
import subprocess

import numpy as np
import pytest

from bbrcit_kde_b200 import build
from bbrcit_kde_b200 import workloads as W


def _has_gpu() -> bool:
    import torch
    return torch.cuda.is_available()


HAS_GPU = _has_gpu()


def _exe():
    return build.build_grid_search()


def _write_cfg(path, **over):
    keys = dict(
        rel_tol="1e-7", abs_tol="1e-8", cuda_device_number="0", gpu_block_size="128",
        refpt_max_leaf_size="32768", qgrid_max_leaf_size="32768", use_adaptive_cv="false",
        cv_method="lsq_conv", skip_cross_validation="false", input_refpts_fname="points.dat",
        output_scatter_fname="scatter.csv", base_bwx="0.3", base_bwy="0.25", alpha="0.5",
        adapted_base_bwx="0.3", adapted_base_bwy="0.3", use_manual_bwgrid="false",
        output_gridsearch_fname="gridsearch.csv", manual_bwx="0.2 0.3 0.5",
        manual_bwy="0.25 0.4", start_bwx="0.1", end_bwx="0.8", steps_bwx="7",
        start_bwy="0.15", end_bwy="0.9", steps_bwy="5", start_qix="-4.0", end_qix="4.0",
        steps_qix="160", start_qiy="-4.0", end_qiy="4.0", steps_qiy="160",
        use_gridsearch_best="true", start_qx="-3.0", end_qx="3.0", steps_qx="30",
        start_qy="-2.5", end_qy="2.5", steps_qy="20", output_eval_fname="kde.csv",
        output_adaptive_eval_fname="akde.csv")
    keys.update(over)
    with open(path, "w") as f:
        f.write("# test configuration\n")
        for k, v in keys.items():
            f.write(f"{k} = {v}   # {k}\n")
    return keys


def _read_grid(path):
    with open(path) as f:
        lines = [ln.split() for ln in f if ln.strip()]
    xs = np.array(lines[0], float)
    ys = np.array(lines[1], float)
    vals = np.array([[float(v) for v in row] for row in lines[2:]])
    return xs, ys, vals


def test_help_and_missing_key(tmp_path):
    exe = _exe()
    r = subprocess.run([exe, "--help"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0 and "Usage: grid_search" in r.stdout
    cfg = tmp_path / "bad.cfg"
    cfg.write_text("abs_tol = 1e-8\n")
    r = subprocess.run([exe, str(cfg)], capture_output=True, text=True, timeout=60)
    assert r.returncode == 1 and "missing option 'rel_tol'" in r.stderr


@pytest.mark.skipif(HAS_GPU, reason="a GPU is present")
def test_fails_loudly_without_gpu(tmp_path):
    _write_cfg(tmp_path / "c.cfg")
    r = subprocess.run([_exe(), "c.cfg"], capture_output=True, text=True, cwd=tmp_path,
                       timeout=60)
    assert r.returncode == 1 and "no CUDA device" in r.stderr


def _data(tmp_path, n=2000):
    wl = W.config2(n=n, m=1)
    with open(tmp_path / "points.dat", "w") as f:
        for (x, y), w in zip(wl.refs, wl.weights):
            f.write(f"{float(x)!r} {float(y)!r} {float(w)!r}\n")
    return wl.refs, wl.weights


@pytest.mark.gpu
def test_conv_grid_search_matches_oracle(tmp_path, oracle):
    refs, w = _data(tmp_path)
    keys = _write_cfg(tmp_path / "c.cfg")
    r = subprocess.run([_exe(), "c.cfg"], capture_output=True, text=True, cwd=tmp_path,
                       timeout=600)
    assert r.returncode == 0, r.stderr
    assert "found 2000 points" in r.stdout
    assert "one batched launch" in r.stdout
    xs, ys, scores = _read_grid(tmp_path / "gridsearch.csv")
    assert scores.shape == (6, 8)
    wn = w / w.sum()
    want = np.empty_like(scores)
    for j, hy in enumerate(ys):
        for i, hx in enumerate(xs):
            want[j, i] = oracle.lsq_conv_cv(W.EPAN_PROD2D, W.EPAN_PROD_CONV2D, 2, (hx, hy), refs,
                                            wn, wn)
    np.testing.assert_allclose(scores, want, rtol=1e-5)
    j, i = np.unravel_index(np.argmin(want), want.shape)
    assert f"best bandwidth: ({xs[i]:g}, {ys[j]:g})" in r.stdout
    # densities on the plotting grid at the selected bandwidth (end points included)
    qx, qy, dens = _read_grid(tmp_path / "kde.csv")
    assert dens.shape == (21, 31)
    q = np.stack(np.meshgrid(qx, qy), -1).reshape(-1, 2)
    f = oracle.direct(W.EPAN_PROD2D, 2, (xs[i], ys[j]), refs, wn, q).reshape(dens.shape)
    np.testing.assert_allclose(dens, f, rtol=1e-5, atol=1e-8)
    # the adaptive density: pilot at the selected bandwidth, alpha 0.5
    _, abw, mass, _ = oracle.adapt(W.EPAN_PROD2D, 2, (xs[i], ys[j]), refs, wn, 0.5)
    _, _, adens = _read_grid(tmp_path / "akde.csv")
    fa = oracle.direct(W.EPAN_PROD2D, 2, (xs[i], ys[j]), refs, mass, q, abw=abw)
    np.testing.assert_allclose(adens, fa.reshape(adens.shape), rtol=1e-5, atol=1e-8)
    # the scatter file repeats the input coordinates
    sc = np.loadtxt(tmp_path / "scatter.csv")
    np.testing.assert_allclose(sc, refs, rtol=1e-5)
    assert float(keys["rel_tol"]) == 1e-7


@pytest.mark.gpu
def test_numint_and_manual_grid_match_oracle(tmp_path, oracle):
    refs, w = _data(tmp_path, n=1500)
    _write_cfg(tmp_path / "c.cfg", cv_method="lsq_numint", use_manual_bwgrid="true")
    r = subprocess.run([_exe(), "c.cfg", "--steps_qix=120", "--steps_qiy", "100"],
                       capture_output=True, text=True, cwd=tmp_path, timeout=600)
    assert r.returncode == 0, r.stderr
    assert "one bandwidth at a time" in r.stdout
    assert not (tmp_path / "gridsearch.csv").exists()   # manual grids write no grid file
    wn = w / w.sum()
    lines = [ln.split() for ln in r.stdout.splitlines() if ln.startswith("  (")]
    assert len(lines) == 6
    for ln in lines:   # "  (hx, hy) score"
        hx, hy, got = float(ln[0].strip("(,")), float(ln[1].strip(")")), float(ln[2])
        want = oracle.lsq_numint_cv(W.EPAN_PROD2D, (hx, hy), refs, wn, wn,
                                    (120, 100, -4.0, 4.0, -4.0, 4.0))
        assert got == pytest.approx(want, rel=1e-5), (hx, hy)
