"""The SuiteSparse sweep driver (the counterpart of test.sh): dataset parsing,
matrix lookup, result-line parsing, and a GPU run over generated matrices."""
import importlib.util
import os

import numpy as np
import pytest

_spec = importlib.util.spec_from_file_location(
    "mf_sweep", os.path.join(os.path.dirname(__file__), "..", "mille-feillue_b200", "sweep.py"))
sweep = importlib.util.module_from_spec(_spec)
_spec.loader.exec_module(sweep)


def _write_mtx(path, n, rp, ci, v):
    with open(path, "w") as f:
        f.write("%%MatrixMarket matrix coordinate real general\n")
        f.write(f"{n} {n} {len(v)}\n")
        for i in range(n):
            for k in range(rp[i], rp[i + 1]):
                f.write(f"{i + 1} {ci[k] + 1} {v[k]:.17g}\n")


def test_dataset_and_result_parsing(tmp_path):
    ds = tmp_path / "CG_dataset.csv"
    ds.write_text("name,nnz\n494_bus,16\nmesh3e1,16\n\n")
    assert sweep.read_dataset(str(ds)) == [("494_bus", "16"), ("mesh3e1", "16")]
    (tmp_path / "MM" / "a").mkdir(parents=True)
    (tmp_path / "MM" / "a" / "mesh3e1.mtx").write_text("")
    assert sweep.find_matrices(str(tmp_path / "MM"), "mesh3e1") == [str(tmp_path / "MM" / "a" / "mesh3e1.mtx")]
    assert sweep.find_matrices(str(tmp_path / "MM"), "494_bus") == []
    r = sweep.parse_result("x\niter=123,time_cg=4.500000 ms,rel_residual=9.1e-11,true_rel_residual=9.2e-11\n")
    assert r == {"iterations": 123, "time_ms": 4.5, "rel_residual": 9.1e-11, "true_rel_residual": 9.2e-11}
    assert sweep.parse_result("nothing") is None


def test_missing_matrices_are_recorded(tmp_path, monkeypatch):
    ds = tmp_path / "d.csv"
    ds.write_text("name,nnz\nnot_there,16\n")
    monkeypatch.setattr(sweep, "DRIVERS", {"cg": str(ds), "bicgstab": str(ds)})  # existing paths, never run
    rows = sweep.sweep(str(ds), str(tmp_path), ["cg", "bicgstab"], str(tmp_path / "out.csv"))
    assert [r["status"] for r in rows] == ["missing", "missing"]
    assert (tmp_path / "out.csv").read_text().splitlines()[0].startswith("name,nnz_class,solver,status")


@pytest.mark.gpu
def test_sweep_runs_the_drivers(mf, tmp_path):
    root = tmp_path / "MM"
    root.mkdir()
    A = mf.Matrix.poisson2d(48)
    rp, ci, v = A.csr()
    _write_mtx(str(root / "pois48.mtx"), A.n, rp, ci, v)
    B = mf.Matrix.convdiff3d(16)
    rp, ci, v = B.csr()
    _write_mtx(str(root / "cd16.mtx"), B.n, rp, ci, v)
    ds = tmp_path / "CG_dataset.csv"
    ds.write_text("name,nnz\npois48,16\ncd16,16\nabsent,16\n")
    rows = sweep.sweep(str(ds), str(root), ["cg", "bicgstab"], str(tmp_path / "out.csv"))
    by = {(r["name"], r["solver"]): r for r in rows}
    assert by[("absent", "cg")]["status"] == "missing"
    assert by[("pois48", "cg")]["status"] == "ok" and by[("pois48", "cg")]["true_rel_residual"] <= 2e-10
    assert by[("cd16", "bicgstab")]["status"] == "ok" and by[("cd16", "bicgstab")]["true_rel_residual"] <= 2e-10
    assert all(np.isfinite(r["time_ms"]) for r in rows if r["status"] == "ok")
