"""The C++ drop-in layer on the GPU: drivers written against the reference's
class API (tests/cpp/*.cpp), built with include/aifmm/ over libaifmm_b200.so,
run on the reference's 78-triangle sphere and their outputs are compared with
the committed golden fixture and the CPU oracle.

Bars: the right-hand side and the matrix entries bit-for-bit against the
fixture's values to 1e-14; the AIFMM solution to the oracle's AIFMM solution
at 1e-10 (as the Python-API parity test); the dense solve at 1e-10; the RRQR
rank and pivots exactly, Q and R to 1e-10; the ACA pivots exactly; the far
field against the reference's formulas restated in tests/physics.py (currents
to 1e-12, RCS to 1e-10: the sums run in another order);
capacitance by AIFMM against dense LU to 1e-8.
"""
import os
import subprocess

import numpy as np
import pytest

import oracle
from rcs_b200 import dropin
from rcs_b200 import mesh as M

from tests import physics

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CPP = os.path.join(ROOT, "tests", "cpp")


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def _vec(path):
    d = np.loadtxt(path, ndmin=2)
    return d[:, 0] + 1j * d[:, 1]


def _mat(path):
    with open(path) as f:
        r, c = (int(x) for x in f.readline().split())
        d = np.loadtxt(f, ndmin=2) if r * c else np.zeros((0, 2))
    return (d[:, 0] + 1j * d[:, 1]).reshape((c, r)).T if r * c else np.zeros((r, c), dtype=complex)


def _summary(path):
    out = {}
    for line in open(path):
        k, *v = line.split()
        out[k] = [float(x) for x in v]
    return out


@pytest.fixture(scope="module")
def golden():
    return np.load(os.path.join(ROOT, "tests", "golden", "sphere78.npz"))


@pytest.fixture(scope="module")
def mesh_files(tmp_path_factory, golden):
    d = tmp_path_factory.mktemp("mesh")
    m = M.Mesh(golden["nodes"], golden["tris"].astype(np.int32))  # 3 columns: no conductor, as shipped
    nf, pf = str(d / "nodeList78.txt"), str(d / "patchList78.txt")
    M.write_mesh(m, nf, pf)
    return nf, pf, m


@pytest.fixture(scope="module")
def run(tmp_path_factory, mesh_files):
    d = tmp_path_factory.mktemp("dropin")
    exe = str(d / "dropin_driver")
    r = dropin.compile_driver([os.path.join(CPP, "dropin_driver.cpp")], exe)
    assert r.returncode == 0, r.stderr
    nf, pf, _ = mesh_files
    out = d / "out"
    out.mkdir()
    p = subprocess.run([exe, nf, pf, str(out), "8", "10", "8"], capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stdout[-2000:] + p.stderr[-2000:]
    s = _summary(str(out / "summary.txt"))
    assert s["done"] == [1.0]
    return out, s


def test_kernel_rhs_and_dense_solution(run, golden):
    out, s = run
    assert s["N"] == [117.0] and s["conductors"] == [1.0]
    rhs = _vec(out / "rhs.txt")
    assert np.abs(rhs - golden["rhs"]).max() <= 1e-14 * np.abs(golden["rhs"]).max()
    assert s["rhs_entry_5"][0] == 0.0
    z37 = complex(*s["entry_3_7"])
    assert abs(z37 - golden["A"][3, 7]) <= 1e-14 * abs(golden["A"][3, 7])
    assert _rel(_vec(out / "x_lu.txt"), golden["x_lu"]) < 1e-10


def test_aifmm_solution_and_stats(run, golden):
    out, s = run
    phi = _vec(out / "phi.txt")
    assert _rel(phi, golden["x_aifmm"]) < 1e-10
    assert s["backward_error"][0] < 1e-10
    assert s["reorder_diff"][0] == 0.0
    tree = _vec(out / "phi_tree.txt")  # solve() keeps tree order: a permutation of phi
    assert np.array_equal(np.sort_complex(tree), np.sort_complex(phi))
    assert s["levels"][0] >= 2 and s["avg_leaf"][0] > 0 and s["avg_rank"][0] > 0
    assert s["mem"][0] > 0 and s["mem_after"][0] > 0


def test_far_field_matches_reference_formulas(run, golden, mesh_files):
    out, _ = run
    _, _, m = mesh_files
    x = _vec(out / "x_lu.txt")
    J_ref, cen, area = physics.centroid_currents(m, golden["rwg"], golden["length"], x)
    J = _mat(out / "J.txt")
    assert J.shape == (78, 3)
    assert _rel(J, J_ref) < 1e-12
    th_rcs = np.loadtxt(out / "rcs.txt", ndmin=2)
    k = 2 * np.pi * float(golden["freq"]) / 3.0e8
    ref = physics.rcs_one_point(J_ref, cen, area, k, th_rcs[:, 0], 0.0)
    assert np.allclose(th_rcs[:, 1], ref, rtol=1e-10, atol=1e-12 * ref.max())


def test_rrqr_class_matches_oracle(run):
    out, s = run
    B = _mat(out / "block.txt")
    Qo, Ro, permo, mpo, erro = oracle.rrqr(B, 8, 10, 0, 1.0, B.shape[1])
    Q, R = _mat(out / "rrqr_q.txt"), _mat(out / "rrqr_r.txt")
    perm = np.loadtxt(out / "rrqr_perm.txt", dtype=int, ndmin=1)
    r = Q.shape[1]
    assert r == Qo.shape[1] == int(s["rrqr_rank"][0])
    assert abs(s["rrqr_maxpivot"][0] - mpo) <= 1e-12 * mpo
    assert _rel(Q, Qo) < 1e-10
    assert np.array_equal(perm[:r], permo[:r])  # the pivots, in order
    assert sorted(perm.tolist()) == list(range(B.shape[1]))
    # R columns by original column index: the non-pivot order differs by design
    Rc, Roc = np.zeros_like(R), np.zeros_like(Ro)
    Rc[:, perm], Roc[:, permo] = R, Ro
    assert _rel(Rc, Roc) < 1e-10
    assert s["rrqr_error"][0] < 1e-8


def test_aca_class_matches_oracle(run, mesh_files):
    out, s = run
    _, _, m = mesh_files
    N = 117
    rows, cols = np.arange(N // 2), np.arange(N // 2, N)
    rb, cb, Ac, _ = oracle.aca(oracle.EFIE(m, 1.0e7), rows, cols, 1e-8)
    assert int(s["aca_rank"][0]) == len(rb)
    assert [int(x) for x in s["aca_rows"]] == rb.tolist()
    assert [int(x) for x in s["aca_cols"]] == cb.tolist()
    assert _rel(_mat(out / "aca_ac.txt"), Ac) < 1e-12


def test_electrostatics_capacitance(run, mesh_files):
    _, s = run
    _, _, m = mesh_files
    C_lu, C_h = s["capacitance_lu"][0], s["capacitance_aifmm"][0]
    assert abs(C_h - C_lu) <= 1e-8 * abs(C_lu)
    assert abs(s["capacitance_matrix"][0] - C_lu) <= 1e-12 * abs(C_lu)
    E = oracle.Electrostatics(m)
    q = np.real(E.dense_solve(np.ones(E.N)))
    v = m.nodes[m.tris - 1]
    area = 0.5 * np.linalg.norm(np.cross(v[:, 1] - v[:, 0], v[:, 2] - v[:, 0]), axis=1)
    assert abs(C_lu - q @ area) <= 1e-10 * abs(C_lu)


def test_real_mode_driver(tmp_path, mesh_files):
    exe = str(tmp_path / "es_double")
    r = dropin.compile_driver([os.path.join(CPP, "dropin_es_double.cpp")], exe, defines=("USE_DOUBLE", "USE_THREE"))
    assert r.returncode == 0, r.stderr
    nf, pf, _ = mesh_files
    p = subprocess.run([exe, nf, pf, "8", "10", "8"], capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stdout[-2000:] + p.stderr[-2000:]
    s = {}
    for line in p.stdout.splitlines():
        k, *v = line.split()
        s[k] = [float(x) for x in v]
    assert s["done"] == [1.0] and s["N"] == [78.0]
    assert abs(s["capacitance_aifmm"][0] - s["capacitance_lu"][0]) <= 1e-8 * abs(s["capacitance_lu"][0])
    assert s["charge_diff"][0] < 1e-8
    assert s["rrqr_rank"][0] >= 1 and s["rrqr_error"][0] < 1e-8
