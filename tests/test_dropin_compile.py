"""CPU test: the reference's own solver headers compile unchanged against the
C++ drop-in (include/hpblas1_dropin), for real and complex scalar types.

The reference's source tree comes from HPB_REF_SOURCE, else from the path the
oracle build recorded in oracle/_ref/source_path; skipped where neither names
an existing directory."""
import os
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


def _ref_source() -> Path | None:
    env = os.environ.get("HPB_REF_SOURCE")
    if env:
        return Path(env)
    rec = ROOT / "oracle" / "_ref" / "source_path"
    if rec.exists():
        return Path(rec.read_text().strip())
    return None


REF = _ref_source()

SRC = r'''
#include <common/gpu_vector_operations.h>
#include <common/csr/gpu_matrix.h>
#include <common/csr/linear_operator.h>
#include <common/csr/preconditioner.h>
#include <common/csr/gpu_ilu0_preconditioner.h>
#include <common/csr/matrix_market_reader.h>
#include <common/ogita/gpu_reduction_ogita.h>
#include <numerical_algos/lin_solvers/default_monitor.h>
#include <numerical_algos/lin_solvers/bicgstabl.h>
#include <numerical_algos/lin_solvers/bicgstab.h>
#include <numerical_algos/lin_solvers/gmres.h>
#include <utils/log.h>
#include <thrust/complex.h>
template <class T> int run(int n) {
    using vec_ops_t = gpu_vector_operations<T>;
    using mat_t = csr::gpu_matrix<vec_ops_t, cublas_wrap>;
    using lin_op_t = csr::linear_operator<vec_ops_t, mat_t>;
    using prec_t = csr::preconditioner<vec_ops_t, lin_op_t, mat_t>;
    using log_t = utils::log_std;
    using mon_t = numerical_algos::lin_solvers::default_monitor<vec_ops_t, log_t>;
    cublas_wrap cublas(true);
    vec_ops_t vec_ops(n, &cublas);
    mat_t mat(&cublas);
    lin_op_t lin_op(&vec_ops, &mat);
    prec_t prec(&vec_ops);
    log_t log;
    numerical_algos::lin_solvers::bicgstabl<lin_op_t, prec_t, vec_ops_t, mon_t, log_t> s1(&vec_ops, &log);
    numerical_algos::lin_solvers::gmres<lin_op_t, prec_t, vec_ops_t, mon_t, log_t, 300> s2(&vec_ops, &log);
    numerical_algos::lin_solvers::bicgstab<lin_op_t, prec_t, vec_ops_t, mon_t, log_t> s3(&vec_ops, &log);
    s1.set_preconditioner(&prec); s1.set_basis_size(4); s1.monitor().init(1e-10, 0, 100);
    s2.set_preconditioner(&prec); s2.set_restarts(30); s2.monitor().init(1e-10, 0, 100);
    s3.set_preconditioner(&prec); s3.monitor().init(1e-10, 0, 100);
    T *x, *b; vec_ops.init_vector(x); vec_ops.start_use_vector(x); vec_ops.init_vector(b); vec_ops.start_use_vector(b);
    vec_ops.use_high_precision();
    bool ok = s1.solve(lin_op, b, x) && s2.solve(lin_op, b, x) && s3.solve(lin_op, b, x);
    // triangular factors: csr::preconditioner with L/U set, the ILU(0) preconditioner
    using ilu_t = csr::gpu_ilu0_preconditioner<vec_ops_t, lin_op_t, mat_t>;
    prec_t lu_prec(&vec_ops);
    lu_prec.set_matrix(&mat, &mat);
    ilu_t ilu(&vec_ops);
    ilu.set_matrix(mat);
    numerical_algos::lin_solvers::bicgstabl<lin_op_t, ilu_t, vec_ops_t, mon_t, log_t> s4(&vec_ops, &log);
    s4.set_preconditioner(&ilu); s4.set_basis_size(2); s4.monitor().init(1e-10, 0, 100);
    ok = ok && s4.solve(lin_op, b, x);
    mat.triangular_solve_lower(b, x);
    mat.triangular_solve_upper(x, b, T(2.0));
    mat.axpy(T(1.0), x, T(0.0), b, true);
    mat.triangular_solve_lower(b, x, T(1.0), true);
    mat.triangular_solve_upper(x, b, T(1.0), true);
    // Matrix Market reader (test_csr_matrix.cpp's use of csr::matrix_market_reader)
    csr::matrix_market_reader<T> reader(true);
    mat_t mm_mat(&cublas);
    reader.read_file_2_csr_marix("m.mtx", &mm_mat);
    int rp_n, ci_n, nnz, rows, cols; int *rp = nullptr, *ci = nullptr; T* val = nullptr;
    reader.get_matrix_dim(rows, cols);
    reader.allocate_set_csr_pointers(rp_n, ci_n, nnz, rp, ci, val);
    free(rp); free(ci); free(val);
    // the reducer class the reference's drivers instantiate directly
    // (test_vector_operations.cpp:61, :100, :211, :304; obtain_condition_precision.cpp:81)
    using gpu_reduction_ogita_t = gpu_reduction_ogita<T, T*>;
    gpu_reduction_ogita_t reduciton_ogita(n);
    T d = reduciton_ogita.dot(x, b);
    T s = reduciton_ogita.sum(b);
    typename gpu_reduction_ogita_type::type_complex_cast<T>::T a = reduciton_ogita.asum(b), nr = reduciton_ogita.norm(x);
    ok = ok && (d == d) && (s == s) && (a == a) && (nr == nr);
    vec_ops.free_vector(x); vec_ops.free_vector(b);
    return ok;
}
int main() { return run<double>(10) + run<float>(10) + run<thrust::complex<double> >(10) + run<thrust::complex<float> >(10); }
'''


@pytest.mark.skipif(REF is None or not REF.is_dir(), reason="reference sources not present")
def test_reference_solvers_compile_against_dropin(tmp_path):
    src = tmp_path / "dropin_driver.cu"
    src.write_text(SRC)
    cmd = ["nvcc", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-w", "-c",
           "-I", str(ROOT / "include" / "hpblas1_dropin"), "-I", str(ROOT / "include"), "-I", str(REF),
           str(src), "-o", str(tmp_path / "d.o")]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
