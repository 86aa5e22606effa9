"""Writes the small Matrix Market fixtures of tests/test_mm.py (hand-made
matrices exercising the format's cases; run from this directory)."""
from pathlib import Path

HERE = Path(__file__).resolve().parent

FILES = {
    "general_real.mtx": """%%MatrixMarket matrix coordinate real general
% a 4 x 4 nonsymmetric matrix, entries out of order, a blank line below

4 4 7
3 1 -2.5
1 1 4.0
2 2 5.0e0
1 4 1.0e-3
4 4 6.25
2 3 -1
4 2 0.5
""",
    "symmetric_real.mtx": """%%MatrixMarket matrix coordinate real symmetric
% lower triangle of a symmetric 3 x 3 matrix
3 3 5
1 1 2.0
2 1 -1.0
2 2 2.0
3 2 -1.0
3 3 2.0
""",
    "pattern.mtx": """%%MatrixMarket matrix coordinate pattern general
3 3 4
1 1
2 1
2 3
3 3
""",
    "integer_amgx.mtx": """%%MatrixMarket matrix coordinate integer general
%%AMGX 1 1 sorted
2 2 3
1 1 3
2 1 -7
2 2 9
""",
    "complex_general.mtx": """%%MatrixMarket matrix coordinate complex general
2 2 3
1 1 1.5 -0.5
2 1 0.0 2.0
2 2 -3.0 1.0
""",
    "duplicates.mtx": """%%MatrixMarket matrix coordinate real general
2 2 4
1 2 1.0
1 1 2.0
1 2 3.0
2 2 4.0
""",
    "bad_hermitian.mtx": """%%MatrixMarket matrix coordinate complex hermitian
1 1 1
1 1 1.0 0.0
""",
    "bad_banner.mtx": """%%MatrixMarket matrix coordinate real
1 1 1
1 1 1.0
""",
    "bad_index.mtx": """%%MatrixMarket matrix coordinate real general
2 2 2
1 1 1.0
3 1 1.0
""",
    "bad_array.mtx": """%%MatrixMarket matrix array real general
2 2
1.0
2.0
3.0
4.0
""",
    "bad_truncated.mtx": """%%MatrixMarket matrix coordinate real general
2 2 3
1 1 1.0
2 2 2.0
""",
}

if __name__ == "__main__":
    for name, text in FILES.items():
        (HERE / name).write_text(text)
