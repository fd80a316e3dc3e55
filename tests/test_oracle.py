"""Pins the C restatement (oracle/sparse_oracle.c) before anything trusts it:
against the reference's known answers (tests/golden/known_answers.npz), the
reference's outputs on seeded random cases (tests/golden/random_cases.npz) and,
where the reference harness is built, bit-exactly against it directly."""

import numpy as np
import pytest

from asc_cpp_b200 import synthetic
from oracle import CSC, CSR, COL_MAJOR, OP_NONE, OP_TRANSPOSE, ROW_MAJOR


def _bits_equal(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return a.dtype == b.dtype and a.shape == b.shape and a.tobytes() == b.tobytes()


@pytest.mark.parametrize("tag,dt", [("f64", np.float64), ("f32", np.float32)])
def test_known_answers_compat(restatement, known_answers, tag, dt):
    ptr = np.array([0, 2, 4, 5], np.int64)
    idx = np.array([1, 3, 0, 2, 1], np.int64)
    val = np.array([2, -1, 4, 5, 3], dt)
    x = np.array([2, -1, 3, 4], dt)
    y = np.array([7, -90, 11, -91, 13, -92], dt)
    restatement.compat_spmv(ptr, idx, val, 2.0, x, -0.5, y, 1, 2)
    assert _bits_equal(y, known_answers[f"blas_compat_a2_bm05_{tag}"])
    np.testing.assert_array_equal(y[::2], np.array([-15.5, 40.5, -12.5], dt))
    y2 = np.array([np.nan, -90, np.nan, -91, np.nan, -92], dt)
    restatement.compat_spmv(ptr, idx, val, 1.0, x, 0.0, y2, 1, 2)
    assert _bits_equal(y2, known_answers[f"blas_compat_a1_b0_{tag}"])
    # zero columns: y = beta * y
    yz = np.array([2, -3, 4], dt)
    restatement.compat_spmv(np.zeros(4, np.int64), np.zeros(0, np.int64), np.zeros(0, dt),
                            7.0, np.zeros(0, dt), 2.0, yz)
    assert _bits_equal(yz, known_answers[f"blas_zero_columns_{tag}"])


def test_known_answer_order(restatement, known_answers):
    y = np.array([-1.0], np.float32)
    restatement.compat_spmv(np.array([0, 3], np.int64), np.array([0, 1, 2], np.int64),
                            np.array([1e20, 1, -1e20], np.float32), 1.0,
                            np.ones(3, np.float32), 0.0, y)
    assert y[0] == 0.0 and _bits_equal(y, known_answers["blas_order_f32"])


@pytest.mark.parametrize("tag,dt", [("f64", np.float64), ("f32", np.float32)])
def test_known_answers_cuda_cases(restatement, known_answers, tag, dt):
    ptr = np.array([0, 2, 3, 6, 8], np.int64)
    idx = np.array([0, 3, 1, 0, 2, 4, 1, 4], np.int64)
    val = np.array([2, -1, 4, 7, 3, 5, -2, 6], dt)
    x = np.array([1, 91, -2, 91, 3, 91, 4, 91, -1], dt)
    y = np.array([10, 91, 91, 20, 91, 91, 30, 91, 91, 40], dt)
    restatement.compat_spmv(ptr, idx, val, 2.0, x, -0.5, y, 2, 3)
    assert _bits_equal(y, known_answers[f"cuda_strided_{tag}"])
    np.testing.assert_array_equal(y[::3], np.array([-9, -26, 7, -24], dt))
    yu = np.array([1, 1], dt)
    restatement.compat_spmv(np.array([0, 1, 2], np.int64), np.array([0, 1], np.int64),
                            np.array([2, 3], dt), 2.0, np.array([4, 5], dt), -1.0, yu)
    assert list(yu) == [15, 29]


@pytest.mark.parametrize("tag,dt", [("f64", np.float64), ("f32", np.float32)])
def test_known_answers_standard(restatement, known_answers, tag, dt):
    ptr = np.array([0, 1, 3], np.int64)
    idx = np.array([0, 0, 1], np.int64)
    cptr = np.array([0, 2, 3], np.int64)
    cidx = np.array([0, 1, 1], np.int64)
    val = np.array([2.0, 1.0, 3.0], dt)
    x = np.array([1.0, -1.0], dt)
    for op, name in ((OP_NONE, "none"), (OP_TRANSPOSE, "transpose")):
        y = np.zeros(2, dt)
        restatement.standard_spmv(CSR, op, 2, 2, ptr, idx, val, 1.0, x, y)
        assert _bits_equal(y, known_answers[f"std_spmv_csr_{name}_{tag}"])
        y = np.zeros(2, dt)
        restatement.standard_spmv(CSC, op, 2, 2, cptr, cidx, val, 1.0, x, y)
        assert _bits_equal(y, known_answers[f"std_spmv_csc_{name}_{tag}"])
    c = np.zeros(4, dt)
    restatement.standard_spmm(CSR, OP_NONE, 2, 2, ptr, idx, val, 1.0,
                              np.array([1, 2, 3, 4], dt), ROW_MAJOR, 2, c, ROW_MAJOR, 2, 2)
    assert _bits_equal(c, known_answers[f"std_spmm_row_{tag}"])
    c = np.zeros(4, dt)
    restatement.standard_spmm(CSC, OP_TRANSPOSE, 2, 2, cptr, cidx, val, 1.0,
                              np.array([1, 3, 2, 4], dt), COL_MAJOR, 2, c, COL_MAJOR, 2, 2)
    assert _bits_equal(c, known_answers[f"std_spmm_csc_col_t_{tag}"])


def test_random_cases_match_reference_outputs(restatement, random_cases):
    n = int(random_cases["count"][0])
    for case in range(n):
        p = f"c{case}_"
        rows, cols = (int(v) for v in random_cases[p + "shape"])
        ptr, idx, val = random_cases[p + "ptr"], random_cases[p + "idx"], random_cases[p + "val"]
        alpha, beta = (float(v) for v in random_cases[p + "ab"])
        y = random_cases[p + "y0"].copy()
        restatement.compat_spmv(ptr, idx, val, alpha, random_cases[p + "x"], beta, y)
        assert _bits_equal(y, random_cases[p + "compat"]), case
        y = random_cases[p + "y0"].copy()
        restatement.standard_spmv(CSR, OP_NONE, rows, cols, ptr, idx, val, alpha,
                                  random_cases[p + "x"], y)
        assert _bits_equal(y, random_cases[p + "std_none"]), case
        y = random_cases[p + "yt0"].copy()
        restatement.standard_spmv(CSR, OP_TRANSPOSE, rows, cols, ptr, idx, val, alpha,
                                  random_cases[p + "xt"], y)
        assert _bits_equal(y, random_cases[p + "std_t"]), case
        c = random_cases[p + "c0"].copy()
        k = c.size // max(rows, 1)
        restatement.standard_spmm(CSR, OP_NONE, rows, cols, ptr, idx, val, alpha,
                                  random_cases[p + "b"], ROW_MAJOR, k, c, ROW_MAJOR, k, k)
        assert _bits_equal(c, random_cases[p + "spmm"]), case


def test_restatement_matches_reference_directly(restatement, reference):
    """Fresh seeds each run: restatement and reference agree bit for bit,
    including negative strides and CSC."""
    from asc_cpp_b200 import synthetic
    rng = np.random.default_rng()
    for _ in range(20):
        dt = rng.choice([np.float32, np.float64])
        rows, cols = int(rng.integers(1, 120)), int(rng.integers(1, 120))
        a = synthetic.random_csr(rng, rows, cols, int(rng.integers(1, 30)), dt, 0.2)
        alpha, beta = float(rng.normal()), float(rng.choice([0.0, rng.normal()]))
        x = rng.uniform(-1, 1, cols * 2).astype(dt)
        y1 = rng.uniform(-1, 1, rows * 3).astype(dt)
        y2 = y1.copy()
        assert reference.compat_spmv(rows, cols, a.ptr, a.idx, a.val, alpha, x, beta, y1, 2, 3) == 0
        restatement.compat_spmv(a.ptr, a.idx, a.val, alpha, x, beta, y2, 2, 3)
        assert _bits_equal(y1, y2)
        # standard, transpose, negative increments on both vectors
        xt = rng.uniform(-1, 1, rows * 2).astype(dt)
        yt1 = rng.uniform(-1, 1, cols).astype(dt)
        yt2 = yt1.copy()
        assert reference.standard_spmv(CSR, OP_TRANSPOSE, rows, cols, a.ptr, a.idx, a.val,
                                       alpha, xt, yt1, incx=-2, incy=-1,
                                       x_offset=2 * (rows - 1), y_offset=cols - 1) == 0
        restatement.standard_spmv(CSR, OP_TRANSPOSE, rows, cols, a.ptr, a.idx, a.val, alpha,
                                  xt, yt2, incx=-2, incy=-1, x_offset=2 * (rows - 1),
                                  y_offset=cols - 1)
        assert _bits_equal(yt1, yt2)
        # CSC view of the same arrays (a is then cols x rows)
        xc = rng.uniform(-1, 1, rows).astype(dt)
        yc1 = rng.uniform(-1, 1, cols).astype(dt)
        yc2 = yc1.copy()
        assert reference.standard_spmv(CSC, OP_NONE, cols, rows, a.ptr, a.idx, a.val, alpha,
                                       xc, yc1) == 0
        restatement.standard_spmv(CSC, OP_NONE, cols, rows, a.ptr, a.idx, a.val, alpha, xc, yc2)
        assert _bits_equal(yc1, yc2)


def test_transpose_structure_is_stable_csc(restatement):
    from asc_cpp_b200 import synthetic
    rng = np.random.default_rng(5)
    a = synthetic.random_csr(rng, 300, 200, 25, np.float64, 0.1)
    t_ptr, t_idx, perm = restatement.transpose_structure(a.rows, a.cols, a.ptr, a.idx)
    rows_of = np.repeat(np.arange(a.rows), np.diff(a.ptr))
    order = np.lexsort((rows_of, a.idx))  # by column, then row
    np.testing.assert_array_equal(perm, order)
    np.testing.assert_array_equal(t_idx, rows_of[order])
    np.testing.assert_array_equal(np.diff(t_ptr), np.bincount(a.idx, minlength=a.cols))


def test_merge_path_split_properties(restatement):
    from asc_cpp_b200 import synthetic
    rng = np.random.default_rng(6)
    a = synthetic.random_csr(rng, 500, 100, 30, np.float64, 0.3)
    total = a.rows + a.nnz
    prev = (0, 0)
    for d in range(0, total + 1, 7):
        r, z = restatement.merge_path_split(a.ptr, d)
        assert r + z == d and r >= prev[0] and z >= prev[1]
        # every row before r has ended by nonzero z; row r has not ended before z
        if r > 0:
            assert a.ptr[r] <= z
        if r < a.rows:
            assert a.ptr[r + 1] >= z
        prev = (r, z)


CONVERSION_CASES = ("ka", "r1", "r2", "r3", "r4")


@pytest.mark.parametrize("name", CONVERSION_CASES)
def test_conversions_match_reference_fixtures(restatement, conversions, name):
    """The oracle's stable bucket sort reproduces the reference's conversions
    (compressed.h:1082-1221) on the committed fixtures."""
    g = conversions
    r, c = (int(v) for v in g[f"{name}_shape"])
    ptr, idx, val = g[f"{name}_csr_ptr"], g[f"{name}_csr_idx"], g[f"{name}_csr_val"]
    got = restatement.convert_compressed(1, r, c, ptr, idx, val)
    for k, arr in zip(("ptr", "idx", "val"), got):
        assert _bits_equal(arr, g[f"{name}_csc_{k}"])
    back = restatement.convert_compressed(0, r, c, g[f"{name}_csc_ptr"], g[f"{name}_csc_idx"],
                                          g[f"{name}_csc_val"])
    for k, arr in zip(("ptr", "idx", "val"), back):
        assert _bits_equal(arr, g[f"{name}_csc_to_csr_{k}"])
        assert _bits_equal(arr, g[f"{name}_csr_{k}"])
    for fmt, to_csc in (("csr", 0), ("csc", 1)):
        got = restatement.convert_coordinates(to_csc, r, c, g[f"{name}_coo"], val)
        for k, arr in zip(("ptr", "idx", "val"), got):
            assert _bits_equal(arr, g[f"{name}_coo_to_{fmt}_{k}"])


def test_conversion_known_answer_values(conversions):
    """compressed_conversion_test.cc:28-36 expected CSC arrays."""
    assert conversions["ka_csc_ptr"].tolist() == [0, 1, 3, 4, 5]
    assert conversions["ka_csc_idx"].tolist() == [1, 0, 2, 1, 0]
    assert conversions["ka_csc_val"].tolist() == [4.0, 2.0, 3.0, 5.0, -1.0]


def test_conversion_matches_reference_directly(restatement, reference):
    from asc_cpp_b200 import synthetic
    rng = np.random.default_rng(22)
    a = synthetic.random_csr(rng, 150, 90, 20, np.float64, 0.3)
    for to_csc in (1,):
        got = restatement.convert_compressed(to_csc, a.rows, a.cols, a.ptr, a.idx, a.val)
        want = reference.convert_compressed(to_csc, a.rows, a.cols, a.ptr, a.idx, a.val)
        for x, y in zip(got, want):
            assert _bits_equal(x, y)


@pytest.mark.parametrize("tag", ["z", "c"])
def test_complex_restatement_matches_reference_fixtures(restatement, complex_cases, tag):
    """Complex standard SpMV / SpMM of the oracle equal the reference's
    (standard_blas_test.cc:177-345 known answers and random cases)."""
    from oracle import CSC, CSR, COL_MAJOR, OP_NONE, ROW_MAJOR
    g = complex_cases
    dt = np.complex128 if tag == "z" else np.complex64
    ptr, idx = np.array([0, 1, 3], np.int64), np.array([0, 0, 1], np.int64)
    val = np.array([2 + 1j, 1 - 1j, 3 + 0.5j], dt)
    x = np.array([1 + 2j, -1 + 1j], dt)
    for name, op in (("csr_none", OP_NONE), ("csr_conjt", 2)):
        y = np.zeros(2, dt)
        restatement.standard_spmv(CSR, op, 2, 2, ptr, idx, val, 1.0, x, y)
        assert _bits_equal(y, g[f"ka_spmv_{name}_{tag}"])
    y = np.zeros(2, dt)
    restatement.standard_spmv(CSC, OP_NONE, 2, 2, np.array([0, 2, 3]), np.array([0, 1, 1]), val,
                              1.0, x, y)
    assert _bits_equal(y, g[f"ka_spmv_csc_none_{tag}"])
    c = np.zeros(4, dt)
    restatement.standard_spmm(CSR, OP_NONE, 2, 2, ptr, idx, val, 1.0, np.array([1, 2, 3, 4], dt),
                              ROW_MAJOR, 2, c, ROW_MAJOR, 2, 2)
    assert _bits_equal(c, g[f"ka_spmm_row_{tag}"])
    c = np.zeros(4, dt)
    restatement.standard_spmm(CSC, 2, 2, 2, np.array([0, 2, 3]), np.array([0, 1, 1]), val, 1.0,
                              np.array([1, 3, 2, 4], dt), COL_MAJOR, 2, c, COL_MAJOR, 2, 2)
    assert _bits_equal(c, g[f"ka_spmm_csc_col_conjt_{tag}"])
    rows, cols = (int(v) for v in g[f"rand_shape_{tag}"])
    p, i, v = g[f"rand_ptr_{tag}"], g[f"rand_idx_{tag}"], g[f"rand_val_{tag}"]
    for op in (0, 1, 2):
        y = g[f"rand_y0_op{op}_{tag}"].copy()
        restatement.standard_spmv(CSR, op, rows, cols, p, i, v, 0.75 - 1.25j,
                                  g[f"rand_x_op{op}_{tag}"], y)
        assert _bits_equal(y, g[f"rand_y_op{op}_{tag}"])
        c = g[f"rand_c0_op{op}_{tag}"].copy()
        restatement.standard_spmm(CSR, op, rows, cols, p, i, v, 0.75 - 1.25j,
                                  g[f"rand_b_op{op}_{tag}"], ROW_MAJOR, 5, c, ROW_MAJOR, 5, 5)
        assert _bits_equal(c, g[f"rand_c_op{op}_{tag}"])


def test_mlp_oracle_gradient_matches_finite_differences():
    """The CPU restatement's analytic MLP gradient (the checker of the CUDA
    backward kernels) agrees with central differences of its own loss."""
    from oracle import mlp_oracle
    rng = np.random.default_rng(3)
    v = 5
    p = rng.standard_normal(mlp_oracle.param_count(v)) * 0.3
    x = rng.standard_normal((9, 12))
    t = rng.standard_normal((9, v))
    g = mlp_oracle.backward(p, x, t, v)
    h = 1e-6
    for i in rng.choice(p.size, 60, replace=False):
        d = np.zeros_like(p)
        d[i] = h
        fd = (mlp_oracle.loss(p + d, x, t, v) - mlp_oracle.loss(p - d, x, t, v)) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 + 1e-4 * abs(g[i]), (i, fd, g[i])


def test_feature_oracle_on_a_known_matrix():
    """Features of a 4 x 4 matrix worked out by hand."""
    from oracle import mlp_oracle
    # rows: [0, 1], [], [2, 3, 9?] -> use 16 columns: row 2 has cols 2, 3, 9
    ptr = np.array([0, 2, 2, 5, 6])
    idx = np.array([0, 1, 2, 3, 9, 3])
    f = mlp_oracle.features(4, 16, ptr, idx, 8)
    assert f[2] == np.log2(7.0)            # nnz = 6
    assert f[4] == np.log2(4.0)            # longest row 3
    assert f[6] == 7 / 16                  # |9 - 2| / columns
    assert f[8] == 3 / 4                   # (0,0), (2,2), (3,3) on the diagonal
    assert f[9] == 6 / (8 * 4)             # runs: row0 {0,1}, row2 {2,3}, {9}, row3 {3}
    assert f[10] == 1 / 4 and f[11] == 1.0


@pytest.mark.parametrize("tag", ["f64", "f32", "z", "c"])
def test_level1_restatement_matches_reference_fixtures(restatement, level1_cases, tag):
    """Dot, axpy, gather, gather-zero and scatter of the oracle equal the
    reference's on standard_blas_test.cc:69-173 and a random case."""
    g = level1_cases
    for name in ("ka", "rand"):
        idx, val, x = g[f"{name}_idx_{tag}"], g[f"{name}_val_{tag}"], g[f"{name}_x_{tag}"]
        alpha = (0.75 - 1.5j) if np.iscomplexobj(val) else 2.0
        for op in range(5):
            for conj in ((0, 1) if op == 0 else (0,)):
                v, xx, r = restatement.level1(op, conj, idx, val, alpha, x)
                key = f"{name}_op{op}_conj{conj}_{tag}"
                assert _bits_equal(v, g[key + "_val"]) and _bits_equal(xx, g[key + "_x"])
                if op == 0:
                    assert _bits_equal(np.array([r], val.dtype), g[key + "_res"])


def test_level1_known_answer_values(level1_cases):
    """standard_blas_test.cc:69-173 expectations, literally: the dot of
    {1, -2} at {0, 2} with {3, 9, 2} is -1; axpy with alpha 2 gives {5, 9, -2}."""
    assert level1_cases["ka_op0_conj0_f64_res"][0] == -1.0
    assert level1_cases["ka_op1_conj0_f64_x"].tolist() == [5.0, 9.0, -2.0]
    assert level1_cases["ka_op3_conj0_f64_x"].tolist() == [0.0, 9.0, 0.0]


TRSV_TAGS = {"f64": np.float64, "f32": np.float32, "z": np.complex128, "c": np.complex64}
TRSV_SHAPES = ((1, 1), (1, 3), (0, 3))  # (layout: 1 row major / 0 column major, k)


def trsv_fixture_cases(g, tag):
    """(key, op, triangle, diagonal, layout, k, alpha, ptr, idx, val, b, x) of
    the random triangular-solve fixtures of one element kind."""
    dt = TRSV_TAGS[tag]
    alpha = (0.5 - 1.25j) if np.iscomplexobj(dt(0)) else -1.5
    for triangle in (0, 1):
        for diagonal in (0, 1):
            base = f"rand_{tag}_{triangle}{diagonal}"
            ptr, idx, val = g[base + "_ptr"], g[base + "_idx"], g[base + "_val"]
            for op in (0, 1, 2):
                for s_, (layout, k) in enumerate(TRSV_SHAPES):
                    key = f"{base}{op}_{s_}"
                    yield (key, op, triangle, diagonal, layout, k, alpha, ptr, idx, val,
                           g[key + "_b"], g[key + "_x"])


@pytest.mark.parametrize("tag", list(TRSV_TAGS))
def test_trsv_restatement_matches_reference_fixtures(restatement, trsv_cases, tag):
    """The C restatement reproduces the reference's triangular solves bit for
    bit, except complex FP32 division by a non-unit diagonal: the reference's
    CPU build divides std::complex<float> with libgcc's routine, the
    restatement (like the CUDA facet, kernels.cu:58-72) with Smith's method;
    there the two agree to a few ulps."""
    for (key, op, tri, diag, layout, k, alpha, ptr, idx, val, b,
         x) in trsv_fixture_cases(trsv_cases, tag):
        got = restatement.triangular_solve(op, tri, diag, 48, ptr, idx, val, alpha, b, layout,
                                           None, k)
        if tag == "c" and diag == 0:
            np.testing.assert_allclose(got, x, rtol=2e-5, atol=2e-6, err_msg=key)
        else:
            assert _bits_equal(got, x), key


@pytest.mark.parametrize("tag", list(TRSV_TAGS))
def test_trsv_known_answers(restatement, trsv_cases, tag):
    """standard_blas_test.cc:336-420 and standard_blas_cuda_test.cc:542-680:
    (2, -1) for the vector and its conjugate transpose, [[2, 1], [-1, 3]] for
    two right-hand sides, zeros for alpha = 0 over NaN values, 1 for the huge
    1 x 1 complex division."""
    g = trsv_cases
    ptr = np.array([0, 1, 3], np.int64)
    idx = np.array([0, 0, 1], np.int64)
    v = g[f"ka_{tag}_val"]
    for name, op, k, want in (("vec", 0, 1, [2, -1]), ("ct", 2, 1, [2, -1]),
                              ("multi", 0, 2, [2, 1, -1, 3])):
        x = g[f"ka_{name}_{tag}_x"]
        assert np.allclose(x, want, rtol=1e-6)
        got = restatement.triangular_solve(op, 1, 0, 2, ptr, idx, v, 1.0, g[f"ka_{name}_{tag}_b"],
                                           1, k, k)
        assert np.allclose(got, want, rtol=1e-6)
    zero = restatement.triangular_solve(0, 1, 0, 2, ptr, idx, g[f"ka_zero_{tag}_val"], 0.0,
                                        np.array([4, 5], v.dtype), 1, 1, 1)
    assert _bits_equal(zero, g[f"ka_zero_{tag}_x"]) and not zero.any()
    if f"ka_large_{tag}_val" in g:
        lv = g[f"ka_large_{tag}_val"]
        got = restatement.triangular_solve(0, 1, 0, 1, np.array([0, 1], np.int64),
                                           np.array([0], np.int64), lv, 1.0, lv, 1, 1, 1)
        assert got[0] == 1 and g[f"ka_large_{tag}_x"][0] == 1


def test_trsv_restatement_matches_reference_larger(restatement, reference):
    """A 300 x 300 case per kind against the compiled reference (its solve
    scans every stored entry per lookup, so larger ones take long)."""
    rng = np.random.default_rng(3)
    for dt in TRSV_TAGS.values():
        for triangle, op in ((1, 0), (0, 2)):
            m = synthetic.triangular(rng, 300, lower=triangle == 1, dtype=dt)
            b = synthetic._values(rng, 600, dt)
            rc, want = reference.triangular_solve(op, triangle, 1, 300, m.ptr, m.idx, m.val,
                                                  1.0, b, 1, None, 2)
            assert rc == 0
            got = restatement.triangular_solve(op, triangle, 1, 300, m.ptr, m.idx, m.val, 1.0,
                                               b, 1, None, 2)
            assert _bits_equal(got, want)


def test_trsv_edge_cases_against_reference(restatement, reference):
    """Shapes at the edges of the solve, each through both the restatement
    and the reference's own SparseTriangularSolveMultiple: a 1 x 1 system,
    a diagonal-only matrix (empty strict triangle), alpha = 0 over NaN
    entries (zeros without reading B), one and five right-hand sides with a
    leading dimension larger than the matrix needs, all four kinds."""
    rng = np.random.default_rng(91)
    for dt in TRSV_TAGS.values():
        cplx = np.iscomplexobj(dt(0))
        one = (np.array([2.5 - 1j]) if cplx else np.array([2.5])).astype(dt)
        cases = [(1, np.array([0, 1], np.int64), np.array([0], np.int64), one)]
        d = synthetic._values(rng, 7, dt) + dt(3)
        cases.append((7, np.arange(8, dtype=np.int64), np.arange(7, dtype=np.int64), d))
        m = synthetic.triangular(rng, 30, lower=False, dtype=dt)
        cases.append((30, m.ptr, m.idx, m.val))
        for n, ptr, idx, val in cases:
            for op in (0, 1, 2):
                for triangle in (0, 1):
                    for diagonal in (0, 1):
                        if n == 30 and triangle == 1:
                            continue  # the upper matrix is not lower triangular
                        for layout, k, ld in ((1, 1, 1), (1, 5, 7), (0, 5, n + 3)):
                            size = (n * ld) if layout == 1 else (k * ld)
                            b = synthetic._values(rng, size, dt)
                            alpha = (0.5 + 2j) if cplx else -0.75
                            rc, want = reference.triangular_solve(op, triangle, diagonal, n, ptr,
                                                                  idx, val, alpha, b, layout, ld,
                                                                  k)
                            assert rc == 0
                            got = restatement.triangular_solve(op, triangle, diagonal, n, ptr,
                                                               idx, val, alpha, b, layout, ld, k)
                            if cplx and dt == np.complex64 and diagonal == 0:
                                np.testing.assert_allclose(got, want, rtol=2e-5, atol=2e-6)
                            else:
                                assert _bits_equal(got, want), (n, op, triangle, diagonal, k)
        # alpha = 0: zeros, whatever the matrix holds
        nan_val = np.full(7, np.nan, dt)
        b = synthetic._values(rng, 7, dt)
        rc, want = reference.triangular_solve(0, 1, 1, 7, np.arange(8, dtype=np.int64),
                                              np.arange(7, dtype=np.int64), nan_val, 0.0, b)
        got = restatement.triangular_solve(0, 1, 1, 7, np.arange(8, dtype=np.int64),
                                           np.arange(7, dtype=np.int64), nan_val, 0.0, b)
        assert rc == 0 and _bits_equal(got, want) and not got.any()


def test_triangular_generators_are_canonical():
    """synthetic.triangular and triangle_of give canonical CSR (sorted,
    unique columns per row) inside the requested triangle, diagonal included."""
    rng = np.random.default_rng(5)
    for lower in (True, False):
        m = synthetic.triangular(rng, 5000, lower=lower, near=5, far=3, span=40)
        rows = np.repeat(np.arange(m.rows), np.diff(m.ptr))
        same_row = rows[1:] == rows[:-1]
        assert (np.diff(m.idx)[same_row] > 0).all()
        assert ((m.idx <= rows) if lower else (m.idx >= rows)).all()
        diag = m.idx == rows
        assert np.bincount(rows[diag], minlength=m.rows).tolist() == [1] * m.rows
        off = np.bincount(rows[~diag], weights=np.abs(m.val[~diag]), minlength=m.rows)
        assert (np.abs(m.val[diag]) >= off + 1 - 1e-12).all()  # diagonally dominant
    lap = synthetic.laplacian_2d(20)
    for lower in (True, False):
        t = synthetic.triangle_of(lap, lower)
        rows = np.repeat(np.arange(t.rows), np.diff(t.ptr))
        assert ((t.idx <= rows) if lower else (t.idx >= rows)).all()
        full_rows = np.repeat(np.arange(lap.rows), np.diff(lap.ptr))
        keep = (lap.idx <= full_rows) if lower else (lap.idx >= full_rows)
        assert _bits_equal(t.idx, lap.idx[keep]) and _bits_equal(t.val, lap.val[keep])


from hypothesis import HealthCheck, given, settings, strategies as st  # noqa: E402


@st.composite
def _small_csr(draw):
    rows = draw(st.integers(0, 12))
    cols = draw(st.integers(0, 12))
    seed = draw(st.integers(0, 2**31 - 1))
    rng = np.random.default_rng(seed)
    lengths = rng.integers(0, cols + 1, size=rows) if cols else np.zeros(rows, np.int64)
    ptr = np.zeros(rows + 1, np.int64)
    np.cumsum(lengths, out=ptr[1:])
    idx = np.concatenate([np.sort(rng.choice(cols, int(n), replace=False))
                          for n in lengths]).astype(np.int64) if ptr[-1] else np.zeros(0, np.int64)
    val = rng.standard_normal(int(ptr[-1]))
    return rows, cols, ptr, idx, val


@settings(max_examples=150, deadline=None, suppress_health_check=[HealthCheck.too_slow])
@given(_small_csr())
def test_conversion_restatement_matches_reference_on_random_shapes(restatement, reference, m):
    """CSR -> CSC and back through the restatement equal the reference's
    ConvertToCsc / ConvertToCsr on random small shapes, empty rows, columns
    and matrices included."""
    rows, cols, ptr, idx, val = m
    got = restatement.convert_compressed(True, rows, cols, ptr, idx, val)
    want = reference.convert_compressed(True, rows, cols, ptr, idx, val)
    for g, w in zip(got, want):
        assert _bits_equal(np.asarray(g, w.dtype), w)
    back = restatement.convert_compressed(False, rows, cols, *got)
    assert _bits_equal(back[0], ptr) and _bits_equal(np.asarray(back[1], np.int64), idx)
    assert _bits_equal(np.asarray(back[2]), val)


@settings(max_examples=120, deadline=None, suppress_health_check=[HealthCheck.too_slow])
@given(st.integers(1, 24), st.integers(0, 2**31 - 1), st.sampled_from([0, 1, 2]),
       st.sampled_from([0, 1]), st.sampled_from([0, 1]),
       st.sampled_from([np.float64, np.float32, np.complex128]))
def test_trsv_restatement_matches_reference_on_random_systems(restatement, reference, n, seed,
                                                              op, triangle, diagonal, dt):
    rng = np.random.default_rng(seed)
    m = synthetic.triangular(rng, n, lower=triangle == 1, near=2, far=1, span=4, dtype=dt)
    b = synthetic._values(rng, 2 * n, dt)
    alpha = (1.5 - 0.5j) if np.iscomplexobj(dt(0)) else 1.5
    rc, want = reference.triangular_solve(op, triangle, diagonal, n, m.ptr, m.idx, m.val, alpha,
                                          b, 1, 2, 2)
    assert rc == 0
    got = restatement.triangular_solve(op, triangle, diagonal, n, m.ptr, m.idx, m.val, alpha, b,
                                       1, 2, 2)
    assert _bits_equal(got, want)
