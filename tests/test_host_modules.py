"""Host-side pieces of the learned settings and the batched ensemble (no GPU)."""
import os

import numpy as np

import saplibrary_b200 as sap
from saplibrary_b200 import ensemble, learned


def test_band_features_are_finite_and_scale_aware():
    f1 = learned.band_features(sap.generate_band_host(20000, 20, 1.0, 1, seed=1), 20000, 20)
    f2 = learned.band_features(sap.generate_band_host(20000, 80, 0.6, 2, seed=1), 20000, 80)
    assert f1.shape == (learned.NUM_FEATURES,) and np.all(np.isfinite(f1)) and np.all(np.isfinite(f2))
    assert f2[1] > f1[1]          # log10 K
    assert f2[4] < f1[4]          # mean dominance follows d
    assert f1[15] <= 1.0 and f2[15] > 0.9  # rows below dominance 1


def test_gain_and_labels_from_a_time_table():
    T = np.array([[3.0, 1.0, 2.0, 9, 9, 9, 9], [1.0, 2.0, 3.0, 9, 9, 9, 9], [np.inf, 4.0, 5.0, 9, 9, 9, 9]])
    assert list(learned.labels_from_times(T)) == [1, 0, 1]
    g = learned.gain(T, np.array([1, 0, 1]))
    assert g["total_chosen_s"] == 6.0 and g["total_default_s"] == 10.0 and g["picked_best"] == 1.0


def test_ensemble_generator_shapes_and_seeds():
    bands, ks, bs = ensemble.make_ensemble(12, seed=4, n_min=2000, n_max=8000, ks=(8, 16))
    assert len(bands) == len(ks) == len(bs) == 12
    for band, K, b in zip(bands, ks, bs):
        assert K in (8, 16) and 2000 <= len(b) <= 8000 and band.size == len(b) * (2 * K + 1)
    again = ensemble.make_ensemble(12, seed=4, n_min=2000, n_max=8000, ks=(8, 16))
    assert all(np.array_equal(a, c) for a, c in zip(bands, again[0]))


def test_sweep_bytes_counts_triangles_vectors_and_scales():
    # algorithmic bytes of one block sweep (the roofline numerator)
    import bench
    bs, nb, P = 64, 3, 2
    tri = bs * (bs + 1) // 2
    mats = (4 * nb - 2) * tri
    vecs = (4 * nb - 2) * 2 * bs + (2 * nb - 2) * bs
    assert bench.sweep_bytes(bs, nb, P, 4) == P * (mats + vecs) * 4
    assert bench.sweep_bytes(bs, nb, P, 8) == P * (mats + vecs) * 8
    # FP16 copies: 2-byte factor values, FP32 vectors and one FP32 scale per column
    assert bench.sweep_bytes(bs, nb, P, 2) == P * (mats * 2 + vecs * 4 + (4 * nb - 2) * bs * 4)
    # the full-size workload's FP16 sweep reads about half of the FP32 one
    r = bench.sweep_bytes(3168, 20, 16, 2) / bench.sweep_bytes(3168, 20, 16, 4)
    assert 0.5 < r < 0.51


def test_numpy_band_generator_matches_the_library_generator():
    # the CPU reference side of the bench generates the banded workloads with
    # numpy (without loading the CUDA library): the same matrices as the
    # library's generator, bit for bit for uniform values
    from saplibrary_b200 import problems
    for n, k, d in ((1000, 7, 1.0), (3000, 50, 0.8), (300, 200, 1.2)):
        a = problems.banded_rowmajor(n, k, d, dist=1, seed=11, rows_per_chunk=997)
        b = sap.generate_band_host(n, k, d, 1, seed=11).reshape(n, 2 * k + 1)
        assert np.array_equal(a, b)
        a2 = problems.banded_rowmajor(n, k, d, dist=2, seed=3)
        b2 = sap.generate_band_host(n, k, d, 2, seed=3).reshape(n, 2 * k + 1)
        assert np.allclose(a2, b2, rtol=1e-13, atol=1e-13)


def test_bench_reference_arm_reports_unavailable_without_the_cuda_library():
    # the CPU reference arm must not load libsap_b200 (checked in a fresh
    # process) and reports why no complete CPU solve of the 1M-row workload runs
    import json
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    code = ("import runpy, sys; sys.argv = ['bench.py', '--impl', 'reference'];\n"
            "runpy.run_path('bench.py', run_name='__main__');\n"
            "maps = open('/proc/self/maps').read(); print('LOADED' if 'libsap_b200' in maps else 'CLEAN')")
    out = subprocess.run([sys.executable, "-c", code], cwd=root, capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    lines = out.stdout.strip().splitlines()
    line = json.loads(lines[0])
    assert line["impl"] == "reference" and "tens of minutes" in line["unavailable"]
    assert lines[-1] == "CLEAN"
