"""bench.py's byte model of the fused GMRES(m) restart cycle, counted by
hand for a tiny case (n = 4 rows, 10 nonzeros, m = 2, 4-byte values and
indices)."""
import bench


def test_gmres_cycle_bytes_by_hand():
    vec = 4 * 4
    spmv = 8 * 10 + 4 * 5 + 2 * vec       # values + indices, row pointers, u, w
    step0 = spmv + 2 * vec + 3 * vec      # reduction (u, w); update (u, w read, next written)
    step1 = spmv + 3 * vec + 5 * vec      # reduction (V_0, u, w); update (+ q_1 and next written)
    closing = 3 * vec                     # <V_k, V_2>, <V_2, V_2>
    solution = 4 * vec                    # V_0, V_1, x read, x written
    residual = spmv + 2 * vec
    assert bench.gmres_cycle_bytes(4, 10, 2) == step0 + step1 + closing + solution + residual


def test_gmres_cycle_bytes_grows_with_the_basis():
    a = bench.gmres_cycle_bytes(1000, 5000, 10)
    b = bench.gmres_cycle_bytes(1000, 5000, 20)
    assert b > 2 * a * 0.9
