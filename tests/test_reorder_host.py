"""The host reordering pipeline (DB, RCM, drop-off, coupling split, second
level, composed permutations) through `sap_reorder_host`, on the CPU, against
the oracle's restatement of sap/graph.h: every output bit-exact, for any
number of host threads (the stages run in parallel with outputs that must
not depend on the thread count)."""
import numpy as np
import pytest

import oracle
import saplibrary_b200 as sap
from saplibrary_b200.problems import convection_diffusion_csr

ARRAYS = ("dbRowPerm", "finalPerm", "finalReordering", "first_rows", "ks")


def check_against_oracle(rp, ci, v, P, dtype, drop, threads, **opt):
    o = oracle.SparsePrecond(P, dtype=dtype, dropFrac=drop, **{k: opt[k] for k in opt if k in ("doDB", "scale")})
    rc_o = o.setup(rp, ci, v, factor=False, band=False)
    opts = sap.Options(dropOffFraction=drop, performDB=opt.get("doDB", True), applyScaling=opt.get("scale", True))
    if rc_o != 0:  # the reference's failures are sap::system_error with its Reason
        with pytest.raises(sap.SystemError) as ei:
            sap.reorder_host(rp, ci, v, P, opts, prec=dtype, threads=threads)
        assert ei.value.reason == rc_o
        return None
    r = sap.reorder_host(rp, ci, v, P, opts, prec=dtype, threads=threads)
    inf = o.info()
    assert (r["K"], r["P"], r["k_db"], r["k_reorder"]) == (inf.K, inf.P, inf.k_db, inf.k_reorder)
    assert r["drop_actual"] == inf.drop_actual
    for name in ARRAYS:
        assert np.array_equal(r[name], o.ints(name)), name
    return r


@pytest.mark.parametrize("dtype", ["float", "double"])
@pytest.mark.parametrize("m,P,drop", [(30, 4, 0.0), (60, 8, 1e-4), (100, 16, 1e-4), (101, 7, 1e-3)])
@pytest.mark.parametrize("threads", [1, 3, 8])
def test_reorder_matches_oracle(m, P, drop, dtype, threads):
    rp, ci, v, _ = convection_diffusion_csr(m=m, fill_reach=5 * m, seed=m)
    check_against_oracle(rp, ci, v, P, dtype, drop, threads)


def test_wide_bfs_levels_any_thread_count():
    # a grid wide enough that the RCM queue batches exceed the serial
    # threshold, so the level-synchronous BFS runs its parallel branch
    rp, ci, v, _ = convection_diffusion_csr(m=400, fill_reach=2000, seed=3)
    outs = [check_against_oracle(rp, ci, v, 16, "float", 1e-4, t) for t in (1, 4, 8)]
    for r in outs[1:]:
        for name in ARRAYS:
            assert np.array_equal(r[name], outs[0][name]), name


def block_diag_csr(parts):
    rps, cis, vs, off, nnz = [np.zeros(1, np.int32)], [], [], 0, 0
    for rp, ci, v in parts:
        rps.append(np.asarray(rp[1:], np.int64) + nnz)
        cis.append(np.asarray(ci, np.int64) + off)
        vs.append(np.asarray(v))
        off += len(rp) - 1
        nnz += len(ci)
    return (np.concatenate(rps).astype(np.int32), np.concatenate(cis).astype(np.int32), np.concatenate(vs))


def test_disconnected_graph_restarts():
    # independent blocks: the BFS restarts at the lowest unvisited node
    parts = [convection_diffusion_csr(m=m, fill_reach=3 * m, seed=m)[:3] for m in (20, 35, 27)]
    rp, ci, v = block_diag_csr(parts)
    for threads in (1, 5):
        check_against_oracle(rp, ci, v, 6, "double", 1e-4, threads)


def test_explicit_zeros_and_no_db():
    rp, ci, v, _ = convection_diffusion_csr(m=50, fill_reach=250, seed=9)
    v = v.copy()
    v[::17] = 0.0  # explicit zeros are removed before reordering
    check_against_oracle(rp, ci, v, 8, "float", 1e-4, 4)
    check_against_oracle(rp, ci, v, 8, "float", 1e-4, 4, doDB=False)
    check_against_oracle(rp, ci, v, 8, "double", 0.0, 2, scale=False)


def test_structurally_singular_matrix_is_reported():
    rp, ci, v, _ = convection_diffusion_csr(m=20, fill_reach=60, seed=4)
    v = v.copy()
    r = 7  # zero out one whole row: no matching can cover it
    v[rp[r]:rp[r + 1]] = 0.0
    check_against_oracle(rp, ci, v, 4, "double", 0.0, 3)


def random_sparse(n, seed, band=40, extra=3, far=0.02):
    """A nonsymmetric sparse pattern: a random band around the diagonal,
    `extra` random entries per row at any distance, some far outliers; a
    dominant diagonal keeps the DB matching well defined."""
    rng = np.random.default_rng(seed)
    rows, cols, vals = [], [], []
    for i in range(n):
        k = rng.integers(1, 6)
        cs = set(np.clip(i + rng.integers(-band, band + 1, size=k), 0, n - 1).tolist())
        cs |= set(rng.integers(0, n, size=extra).tolist()) if rng.random() < 0.5 else set()
        if rng.random() < far:
            cs.add(int(rng.integers(0, n)))
        cs.add(i)
        for c in sorted(cs):
            rows.append(i)
            cols.append(c)
            vals.append(10.0 if c == i else float(rng.uniform(-1, 1)))
    rp = np.zeros(n + 1, np.int32)
    np.add.at(rp, np.asarray(rows) + 1, 1)
    return np.cumsum(rp).astype(np.int32), np.asarray(cols, np.int32), np.asarray(vals)


@pytest.mark.parametrize("seed", [1, 2, 3])
@pytest.mark.parametrize("dtype", ["float", "double"])
def test_random_patterns_match_oracle(seed, dtype):
    rp, ci, v = random_sparse(3000 + 517 * seed, seed)
    for P, drop, threads in ((4, 0.0, 1), (7, 1e-3, 6), (12, 1e-2, 3)):
        check_against_oracle(rp, ci, v, P, dtype, drop, threads)


def test_invalid_csr_is_rejected():
    rp, ci, v, _ = convection_diffusion_csr(m=10, fill_reach=30, seed=1)
    bad_ci = ci.copy()
    bad_ci[5] = len(rp) + 3  # column out of range
    with pytest.raises(sap.LibraryError) as ei:
        sap.reorder_host(rp, bad_ci, v, 2)
    assert ei.value.code == -100 and "column index" in str(ei.value)
    bad_rp = rp.copy()
    bad_rp[3], bad_rp[4] = bad_rp[4], bad_rp[3]  # not monotone
    with pytest.raises(sap.LibraryError) as ei:
        sap.reorder_host(bad_rp, ci, v, 2)
    assert ei.value.code == -100
    with pytest.raises(ValueError):
        sap.reorder_host(rp, ci, v, 2, prec="tf32")


def random_unscaled(n, seed, reach=60, per=6):
    """Entries of random magnitude within +-reach of the diagonal, no
    dominant diagonal: several rows have their largest entry in the same
    column, so the DB's greedy pass leaves rows for the augmenting-path
    search."""
    rng = np.random.default_rng(seed)
    rows, cols, vals = [], [], []
    for i in range(n):
        cs = set(rng.integers(max(0, i - reach), min(n, i + reach + 1), size=per).tolist())
        cs.add(i)
        for c in sorted(cs):
            rows.append(i)
            cols.append(c)
            vals.append(float(rng.uniform(-1, 1)))
    rp = np.zeros(n + 1, np.int32)
    np.add.at(rp, np.asarray(rows) + 1, 1)
    return np.cumsum(rp).astype(np.int32), np.asarray(cols, np.int32), np.asarray(vals)


@pytest.mark.parametrize("seed", [0, 1])
def test_db_greedy_conflicts_match_oracle(seed):
    rp, ci, v = random_unscaled(4000 + 313 * seed, seed)
    for dtype, threads in (("float", 1), ("double", 5), ("float", 8)):
        check_against_oracle(rp, ci, v, 6, dtype, 1e-3, threads)


def symmetric_permuted(m, fill, reach, seed):
    """The convection-diffusion matrix under a random symmetric permutation
    (rows and columns alike): DB restores the diagonal but not the band, so
    RCM lowers the bandwidth and its order is kept."""
    rp, ci, v, _ = convection_diffusion_csr(m=m, fill_per_row=fill, fill_reach=reach, seed=seed,
                                            permute_rows=False)
    n = rp.size - 1
    p = np.random.default_rng(seed).permutation(n)
    rows = np.repeat(np.arange(n), np.diff(rp))
    nr, nc = p[rows], p[ci]
    order = np.lexsort((nc, nr))
    nr, nc, nv = nr[order], nc[order], v[order]
    out_rp = np.zeros(n + 1, np.int64)
    np.add.at(out_rp, nr + 1, 1)
    return np.cumsum(out_rp).astype(np.int32), nc.astype(np.int32), nv


@pytest.mark.parametrize("m,fill,reach,kept", [
    (90, 1, 30, True),      # RCM order kept (bandwidth 8,060 -> 168)
    (400, 0, 1, True),      # kept, batches above the serial threshold (parallel BFS)
    (200, 2, 3000, False),  # long-range fill: every trial gives its order up
    (400, 2, 2000, False),  # given up, parallel BFS, levels still drive the second trial
])
def test_rcm_orders_kept_and_given_up(m, fill, reach, kept):
    """The BFS trials track their bandwidth and give an order up as soon as
    it cannot be kept (only its levels are filled from then on); kept and
    given-up orders both match the oracle at any thread count."""
    if kept:
        rp, ci, v = symmetric_permuted(m, fill, reach, m)
    else:
        rp, ci, v, _ = convection_diffusion_csr(m=m, fill_per_row=fill, fill_reach=reach, seed=m)
    for threads in (1, 4, 8):
        r = check_against_oracle(rp, ci, v, 8, "double", 1e-4, threads)
        assert (r["k_reorder"] < r["k_db"]) == kept


@pytest.mark.parametrize("place", ["all", "none"])
def test_drop_off_group_placement_modes(place, monkeypatch):
    """Drop-off places the values of the distance groups its walk is
    predicted to reach (from double sums) and the rest when the exact walk
    goes further; placing all groups first, or none (every group placed on
    demand), gives the same outputs, equal to the oracle's."""
    monkeypatch.setenv("SAPB_DROPOFF_PLACE", place)
    rp, ci, v, _ = convection_diffusion_csr(m=120, fill_reach=600, seed=12)
    for drop, dtype, threads in ((1e-4, "float", 4), (1e-2, "double", 3), (0.0, "float", 1)):
        check_against_oracle(rp, ci, v, 8, dtype, drop, threads)


def test_stage_times_are_reported():
    """sap_reorder_host_stages returns the last call's stage times in order."""
    rp, ci, v, _ = convection_diffusion_csr(m=80, fill_reach=400, seed=8)
    r = sap.reorder_host(rp, ci, v, 6, sap.Options(dropOffFraction=1e-4), prec="float", threads=2)
    assert list(r["stage_ms"]) == ["db", "rcm", "drop_off", "coupling", "second_level", "assemble", "compose"]
    assert all(t >= 0.0 for t in r["stage_ms"].values())
    assert sap._lib.sap_reorder_host_stages(-1, None, None, None) == -100  # SAP_ERR_INVALID_ARGUMENT


def test_seeded_mix_with_bandwidth_caps():
    """A seeded mix of the families above with drop-off fractions up to 5 %,
    maximum bandwidths that cut (first drop-off phase) or skip RCM (<= 64),
    1 to 19 partitions and 1 to 8 host threads, all against the oracle."""
    rng = np.random.default_rng(123)
    for it in range(24):
        kind, seed = it % 4, int(rng.integers(1 << 30))
        if kind == 0:
            m = int(rng.integers(10, 90))
            rp, ci, v, _ = convection_diffusion_csr(m=m, fill_per_row=int(rng.integers(0, 3)),
                                                    fill_reach=int(rng.integers(8, 6 * m)), seed=seed)
        elif kind == 1:
            rp, ci, v = random_sparse(int(rng.integers(200, 3000)), seed, band=int(rng.integers(5, 80)))
        elif kind == 2:
            rp, ci, v = random_unscaled(int(rng.integers(200, 2500)), seed, reach=int(rng.integers(5, 100)))
        else:
            m = int(rng.integers(10, 60))
            rp, ci, v = symmetric_permuted(m, int(rng.integers(0, 3)), int(rng.integers(8, 3 * m)), seed)
        P, dtype = int(rng.integers(1, 20)), ["float", "double"][it % 2]
        drop = float(rng.choice([0.0, 1e-5, 1e-4, 1e-3, 1e-2, 0.05]))
        threads = int(rng.integers(1, 9))
        maxbw = int(rng.choice([2**31 - 1, 2**31 - 1, int(rng.integers(1, 200)), 64, 65, 300]))
        o = oracle.SparsePrecond(P, dtype=dtype, dropFrac=drop, maxBandwidth=maxbw)
        rc = o.setup(rp, ci, v, factor=False, band=False)
        opts = sap.Options(dropOffFraction=drop, maxBandwidth=maxbw)
        if rc != 0:
            with pytest.raises(sap.SystemError) as ei:
                sap.reorder_host(rp, ci, v, P, opts, prec=dtype, threads=threads)
            assert ei.value.reason == rc
            continue
        r = sap.reorder_host(rp, ci, v, P, opts, prec=dtype, threads=threads)
        inf = o.info()
        assert (r["K"], r["P"], r["k_db"], r["k_reorder"]) == (inf.K, inf.P, inf.k_db, inf.k_reorder), it
        assert r["drop_actual"] == inf.drop_actual, it
        for name in ARRAYS:
            assert np.array_equal(r[name], o.ints(name)), (it, name)

