"""bench.py's byte models of the fused GMRES(m) restart cycle and the fused
BiCGStab(l) cycle, counted by hand for tiny cases (n = 4 rows, 10
nonzeros)."""
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


def test_bicgstabl_cycle_bytes_by_hand():
    """The fused BiCGStab(l) cycle counted kernel by kernel (n = 4 rows,
    10 nonzeros, binary64 values, int32 indices)."""
    vec = 8 * 4
    spmv = 12 * 10 + 4 * 5 + 2 * vec      # values + indices, row pointers, the gathered operand, y
    # l = 2.  Step 0: A (r_0 - beta u_0) + <rt, .> (r_0 gathered too, rt);
    # update + A r_0' + <rt, .> (u_1 gathered, u_0 and x read and written, rt).
    # Step 1: the same product; update + A r_1' + the first sweep's sums
    # (u_2 gathered, r_0, u_0, u_1, x read; u_0, u_1, r_0, x written).
    # Sweep 2: r_1, r_2, r_0 read, r_2 written, plus the deferred r_1 update
    # (u_2 read, r_1 written).  Closing update: r_0, x, r_1, r_2, u_1, u_2,
    # u_0, rt read; x, r_0, u_0 written.
    l2 = (spmv + 2 * vec) + (spmv + 6 * vec) + (spmv + 2 * vec) + (spmv + 9 * vec) + 6 * vec + 11 * vec
    assert bench.bicgstabl_cycle_bytes(4, 10, 2) == l2
    # l = 1: the step's product + <rt, .>, then update + A r_0' + the sweep's
    # sums (no rt); the closing update applies the deferred r_0 update with
    # the u_1 and r_0 it reads and writes anyway
    l1 = (spmv + 2 * vec) + (spmv + 5 * vec) + 9 * vec
    assert bench.bicgstabl_cycle_bytes(4, 10, 1) == l1
