"""Matrix Market reader (hpb_mm_read_csr, host code): every accepted case of
the format against scipy.io.mmread converted to CSR with sorted indices
(files without duplicate entries), duplicates kept in stable order (a
file with repeated (row, column) pairs), and the refused files with the
reference's messages.  The fixtures are hand-made small matrices written
by tests/golden/mm/make_mm_fixtures.py; a larger case is generated here
(a seeded random matrix written with scipy.io.mmwrite)."""
import numpy as np
import pytest
import scipy.io
import scipy.sparse as sp

from conftest import GOLDEN
from high_precision_blas1_b200 import problems

MM = GOLDEN / "mm"


def as_scipy(A):
    return sp.csr_matrix((A.val, A.col_ind, A.row_ptr), shape=(A.n, A.n))


@pytest.mark.parametrize("name", ["general_real", "symmetric_real", "pattern", "integer_amgx", "complex_general"])
def test_matches_scipy(name):
    A = problems.read_matrix_market(MM / f"{name}.mtx")
    ref = sp.csr_matrix(scipy.io.mmread(str(MM / f"{name}.mtx")))
    ref.sort_indices()
    assert A.row_ptr.dtype == np.int32 and A.col_ind.dtype == np.int32
    assert np.array_equal(A.row_ptr, ref.indptr) and np.array_equal(A.col_ind, ref.indices)
    assert np.array_equal(A.val, ref.data.astype(A.val.dtype))
    assert np.all(np.diff(A.col_ind[A.row_ptr[0]:A.row_ptr[1]]) > 0)


def test_duplicates_kept_in_stable_order():
    A = problems.read_matrix_market(MM / "duplicates.mtx")
    assert A.row_ptr.tolist() == [0, 3, 4]
    assert A.col_ind.tolist() == [0, 1, 1, 1]
    assert A.val.tolist() == [2.0, 1.0, 3.0, 4.0]  # the two (1, 2) entries in file order


def test_larger_random_roundtrip(tmp_path):
    rng = np.random.default_rng(17)
    M = sp.random(500, 500, density=0.02, random_state=3, format="coo") + sp.eye(500)
    M = sp.coo_matrix(M)
    M.data = rng.standard_normal(M.nnz)
    f = tmp_path / "r.mtx"
    scipy.io.mmwrite(str(f), M, precision=17)
    A = problems.read_matrix_market(f)
    ref = sp.csr_matrix(M)
    ref.sum_duplicates()
    ref.sort_indices()
    assert np.array_equal(A.row_ptr, ref.indptr) and np.array_equal(A.col_ind, ref.indices)
    assert np.array_equal(A.val, ref.data)


@pytest.mark.parametrize("name,msg", [("bad_hermitian", "hermitian"), ("bad_banner", "banner"),
                                      ("bad_index", "invalid row index"), ("bad_array", "not supported"),
                                      ("bad_truncated", "unexpected end of file")])
def test_rejected(name, msg):
    with pytest.raises(ValueError, match=msg):
        problems.read_matrix_market(MM / f"{name}.mtx")


def test_missing_file():
    with pytest.raises(ValueError, match="cannot open"):
        problems.read_matrix_market(MM / "no_such_file.mtx")
