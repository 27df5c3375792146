"""wcg_pcg_solve_csr against the reference's own robertbridson::PCGSolver<double>
(libWetCloth/Core/PCGSolver/PCGSolver.h:245-330), run through the compiled
reference (oracle/_ref, wcref_pcg_solve_csr) on the same CSR matrices:

* the assembled pressure systems of two seeded scenes (7-point, bucket-major
  DOF order: no dropped fill-in), and the implicit viscosity system (cross
  terms: the MIC(0) dropped-entry rule applies);
* seeded random symmetric, diagonally dominant matrices with irregular
  sparsity (a grid Laplacian plus long-range couplings), with and without an
  empty row.

The iteration counts are equal and the solutions agree to 1e-10 of their
largest entry (the iterates differ only by the summation order of the dot
products); on the singular viscosity system the counts agree within one and
A x agrees to the solve's tolerance.  Edge cases: a zero right-hand side (no iteration), the iteration
limit (WCG_ERR_NOT_CONVERGED, as the reference's false), and malformed
matrices (WCG_ERR_ARG before any device work)."""
import numpy as np
import pytest

from libwetcloth_b200 import _capi, scenes
from oracle import ref as oref

DT = 1e-3


def random_spd(n_side, extra, seed, empty_row=False):
    """Symmetric, strictly diagonally dominant CSR matrix on an n_side^3 grid
    (7-point couplings with random weights) plus `extra` random long-range
    symmetric couplings; columns sorted in each row."""
    rng = np.random.default_rng(seed)
    n = n_side ** 3
    ent = {}

    def add(i, j, v):
        ent[(i, j)] = ent.get((i, j), 0.0) + v
        ent[(j, i)] = ent.get((j, i), 0.0) + v

    idx = np.arange(n).reshape(n_side, n_side, n_side)
    for ax in range(3):
        a = np.moveaxis(idx, ax, 0)
        for i, j in zip(a[:-1].ravel(), a[1:].ravel()):
            add(int(i), int(j), -rng.uniform(0.2, 1.0))
    for _ in range(extra):
        i, j = rng.integers(0, n, 2)
        if i != j:
            add(int(i), int(j), -rng.uniform(0.05, 0.5))
    skip = n // 3 if empty_row else -1
    rows = [[] for _ in range(n)]
    for (i, j), v in ent.items():
        if i == skip or j == skip:
            continue
        rows[i].append((j, v))
    rowstart, col, val = [0], [], []
    for i in range(n):
        if i != skip:
            diag = sum(abs(v) for _, v in rows[i]) + rng.uniform(0.1, 1.0)
            rows[i].append((i, diag))
        for j, v in sorted(rows[i]):
            col.append(j)
            val.append(v)
        rowstart.append(len(col))
    b = rng.standard_normal(n)
    if empty_row:
        b[skip] = 0.0
    return (np.array(rowstart, np.int64), np.array(col, np.int64), np.array(val), b)


def csr_matvec(rowstart, col, val, x):
    rows = np.repeat(np.arange(len(rowstart) - 1), np.diff(rowstart))
    return np.bincount(rows, weights=val * x[col], minlength=len(rowstart) - 1)


def _pressure_system(kind):
    sc = scenes.dam_break(16, 8, 0) if kind == "dam16" else \
        scenes.half_box(32, 2, 5, amplitude=0.5, sigma_cells=2.0)
    r = oref.RefScene(sc, mic=True)
    r.step(DT, snapshot=True)
    out = (r.get("A_rowstart"), r.get("A_col"), r.get("A_val"), r.get("b"),
           sc.params.criterion, sc.params.maxiters)
    r.close()
    return out


def _viscosity_system():
    sc = scenes.dam_break(16, 8, 0)
    sc.params.viscosity = 0.5
    sc.params.viscosity_substeps = 1
    sc.params.viscosity_implicit = True
    sc.params.viscosity_criterion = 1e-10
    sc.params.maxiters = 5000
    r = oref.RefScene(sc, mic=True)
    r.step(DT, snapshot=True)
    out = (r.get("V_rowstart"), r.get("V_col"), r.get("V_val"), r.get("V_rhs"), 1e-10, 5000)
    r.close()
    return out


def _system(kind):
    if kind in ("dam16", "curl32"):
        return _pressure_system(kind)
    if kind == "viscosity":
        return _viscosity_system()
    seed = {"random_a": 1, "random_b": 2, "random_empty": 3}[kind]
    rs, col, val, b = random_spd(9, 400, seed, empty_row=(kind == "random_empty"))
    return rs, col, val, b, 1e-10, 2000


def test_reference_csr_entry_matches_its_own_solve():
    """The harness entry rebuilds the SparseMatrix from CSR: on the assembled
    pressure system it reproduces the iterations and solution of the
    reference's MIC(0) solve inside the step."""
    if not oref.available():
        pytest.skip("oracle/_ref not built")
    sc = scenes.dam_break(16, 8, 0)
    r = oref.RefScene(sc, mic=True)
    r.step(DT, snapshot=True)
    it_ref, _ = r.solver_stats()
    x, res, it, ok = oref.pcg_solve_csr(r.get("A_rowstart"), r.get("A_col"), r.get("A_val"),
                                        r.get("b"), sc.params.criterion, sc.params.maxiters)
    assert ok and it == it_ref
    p = r.get("pressure")
    di = r.get("dof_index")
    m = di >= 0
    xr = np.zeros(int(m.sum()))
    xr[di[m]] = p[m]
    assert np.array_equal(x, xr)
    r.close()


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["dam16", "curl32", "viscosity", "random_a", "random_b",
                                  "random_empty"])
def test_pcg_solve_csr_matches_reference(kind, wcg):
    if not oref.available():
        pytest.skip("oracle/_ref not built")
    rs, col, val, b, tol, maxit = _system(kind)
    xr, res_r, it_r, ok_r = oref.pcg_solve_csr(rs, col, val, b, tol, maxit)
    assert ok_r
    x, res, it, st = _capi.pcg_solve_csr(rs, col, val, b, tol, maxit)
    assert st == _capi.WCG_OK
    if kind == "viscosity":
        # the viscosity matrix is singular (unknowns that touch liquid only
        # across an edge): the Krylov iterates drift apart in its null space
        # with the dot products' rounding, so the stop may come one iteration
        # apart; compare A x, which the null-space components do not touch,
        # to the solve's own tolerance
        assert abs(it - it_r) <= 1, (it, it_r)
        ax, axr = csr_matvec(rs, col, val, x), csr_matvec(rs, col, val, xr)
        err = np.abs(ax - axr).max() / max(np.abs(b).max(), 1e-300)
        assert err <= 10 * tol, f"{kind}: A x differs by {err:.3e} of max|b|"
        assert res <= tol * np.abs(b).max()
    else:
        assert it == it_r, (it, it_r)
        err = np.abs(x - xr).max() / max(np.abs(xr).max(), 1e-300)
        assert err <= 1e-10, f"{kind}: solution differs by {err:.3e} of max"
        assert res <= tol * np.abs(b).max()
        assert abs(res - res_r) <= 1e-6 * max(res_r, 1e-300) + 1e-12 * np.abs(b).max()


@pytest.mark.gpu
def test_pcg_solve_csr_edges(wcg):
    rs, col, val, b = random_spd(5, 40, 7)
    # zero right-hand side: no iteration, zero solution (PCGSolver.h:268-271)
    x, res, it, st = _capi.pcg_solve_csr(rs, col, val, np.zeros_like(b), 1e-8, 100)
    assert st == _capi.WCG_OK and it == 0 and res == 0.0 and not x.any()
    # the iteration limit: the reference's false, with its iterate
    xr, res_r, it_r, ok_r = oref.pcg_solve_csr(rs, col, val, b, 1e-14, 3)
    x, res, it, st = _capi.pcg_solve_csr(rs, col, val, b, 1e-14, 3)
    assert not ok_r and st == _capi.WCG_ERR_NOT_CONVERGED and it == it_r == 3
    assert np.abs(x - xr).max() <= 1e-10 * np.abs(xr).max()


def test_pcg_solve_csr_rejects_malformed(wcg):
    """Argument checks that need no device: negative size, null arrays."""
    import ctypes
    L = wcg
    res = ctypes.c_double(0)
    it = ctypes.c_int(0)
    assert L.wcg_pcg_solve_csr(None, None, None, -1, None, None, 1e-6, 10,
                               ctypes.byref(res), ctypes.byref(it)) == _capi.WCG_ERR_ARG
    assert L.wcg_pcg_solve_csr(None, None, None, 4, None, None, 1e-6, 10,
                               ctypes.byref(res), ctypes.byref(it)) == _capi.WCG_ERR_ARG
    assert L.wcg_pcg_solve_csr(None, None, None, 0, None, None, 1e-6, 10,
                               ctypes.byref(res), ctypes.byref(it)) == _capi.WCG_OK
    assert it.value == 0


@pytest.mark.gpu
def test_pcg_solve_csr_rejects_unsorted_rows(wcg):
    rs = np.array([0, 2, 4], np.int32)
    col = np.array([1, 0, 0, 1], np.int32)  # row 0 not ascending
    val = np.array([-1.0, 4.0, -1.0, 4.0])
    with pytest.raises(_capi.WcgError) as e:
        _capi.pcg_solve_csr(rs, col, val, np.ones(2), 1e-8, 10)
    assert e.value.code == _capi.WCG_ERR_ARG
