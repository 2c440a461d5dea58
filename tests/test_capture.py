"""The captured-linear-system format (reader, writer, v3 companion checks, block conversion).

Mirrors the reference's own capture tests (src/lib/ressim/src/fim/linear/capture.rs:645-833):
the same 3x3 sample system, round trips with and without equation scaling, a v3 round trip
and the rejection of a tampered true-IMPES weight, and the rejection of a wrong header and of
truncated triplets.  The expected file text is what the reference writer produces for the
sample system: Rust `{:e}` numbers, rows in CSR order.
"""
import numpy as np
import pytest

from ressim_b200 import capture as cap


def sample_system():
    trip = [(0, 0, 4.0), (0, 2, -1.5e-8), (1, 1, 2.0), (2, 0, 1e12), (2, 2, 8.0)]
    return cap.csr_from_triplets(3, 3, trip), np.array([1.0, -2.5, 3e-4])


def sample_flow(jac):
    empty = lambda r, c: cap.csr_from_triplets(r, c, [])  # noqa: E731
    storage = np.array([[[1.0, 0.0, 0.0], [0.0, 2.0, 0.0], [0.0, 0.0, 3.0]]])
    return cap.FlowLifecycle(cap.FLOW_SOURCE_TAG, cap.FLOW_SOURCE_COMMIT, cap.DUNE_ISTL_VERSION,
                             cap.TRUE_IMPES_PRESSURE_SCALE_BAR, storage, np.array([[1.0, 0.0, 0.0]]), 3,
                             jac, empty(3, 0), empty(0, 3), empty(0, 0))


ONE_CELL = cap.Layout(1, 3, 0, 3)

EXPECTED_V2 = """fim-capture-v2
newton_iteration 7
failure_reason dead-state
dominant_family water
dominant_item_index 405
layout 1 3 0 3
equation_scaling 1
water 1 1e1
oil_component 1 1e1
gas_component 1 1e1
well_constraint 0
perforation_flow 0
rows 3
cols 3
nnz 5
rhs
1e0
-2.5e0
3e-4
triplets
0 0 4e0
0 2 -1.5e-8
1 1 2e0
2 0 1e12
2 2 8e0
"""


def scaling():
    return {"water": np.array([10.0]), "oil_component": np.array([10.0]), "gas_component": np.array([10.0]),
            "well_constraint": np.array([]), "perforation_flow": np.array([])}


def test_rust_exp_formatting():
    cases = [(4.0, "4e0"), (-1.5e-8, "-1.5e-8"), (1e12, "1e12"), (3e-4, "3e-4"), (0.1, "1e-1"),
             (123.456, "1.23456e2"), (0.0, "0e0"), (-0.0, "-0e0"), (1.0 / 3.0, "3.333333333333333e-1"),
             (5e-324, "5e-324"), (1.7976931348623157e308, "1.7976931348623157e308"), (float("inf"), "inf"),
             (float("-inf"), "-inf")]
    for v, s in cases:
        assert cap.rust_exp(v) == s, (v, cap.rust_exp(v), s)
        assert float(s) == v
    assert cap.rust_exp(float("nan")) == "NaN"


def test_round_trip_metadata_layout_rhs_and_triplets(tmp_path):
    jac, rhs = sample_system()
    s = cap.CapturedSystem(7, "dead-state", "water", 405, ONE_CELL, jac, rhs, scaling())
    path = cap.write_capture(tmp_path, 3, s)
    assert path.endswith("fim_capture_00003.txt")
    with open(path) as f:
        assert f.read() == EXPECTED_V2
    loaded = cap.load_captures(tmp_path)
    assert len(loaded) == 1
    t = loaded[0]
    assert (t.newton_iteration, t.failure_reason, t.dominant_family, t.dominant_item_index) == \
        (7, "dead-state", "water", 405)
    assert t.layout == ONE_CELL
    assert np.array_equal(t.rhs, rhs)
    assert np.array_equal(t.jacobian.to_dense(), jac.to_dense())
    for k, v in scaling().items():
        assert np.array_equal(t.equation_scaling[k], v)
    assert t.flow_lifecycle is None


def test_round_trip_none_equation_scaling(tmp_path):
    jac, rhs = sample_system()
    cap.write_capture(tmp_path, 0, cap.CapturedSystem(1, "max-iters", "water", 0, None, jac, rhs))
    loaded = cap.load_captures(tmp_path)
    assert len(loaded) == 1
    assert loaded[0].equation_scaling is None and loaded[0].layout is None
    assert loaded[0].flow_lifecycle is None


def test_flow_lifecycle_round_trip(tmp_path):
    jac, rhs = sample_system()
    s = cap.CapturedSystem(0, "y2d6a-proof", "water", 0, ONE_CELL, jac, rhs, None, sample_flow(jac))
    path = cap.write_capture(tmp_path, 0, s)
    text = open(path).read()
    assert text.startswith("fim-capture-v3\n")
    assert "\nflow_lifecycle 1\nflow_source_tag release/2026.04/final\n" in text
    assert "\npressure_scale_bar 5e1\nstorage_blocks 1\n1e0 0e0 0e0 0e0 2e0 0e0 0e0 0e0 3e0\n" in text
    assert "\nmatrix_j_rr 3 3 5\n0 0 4e0\n" in text and "\nmatrix_j_ww 0 0 0\nrows 3\n" in text
    f = cap.load_captures(tmp_path)[0].flow_lifecycle
    assert np.array_equal(f.storage_blocks, s.flow_lifecycle.storage_blocks)
    assert np.array_equal(f.true_impes_weights, s.flow_lifecycle.true_impes_weights)
    assert np.array_equal(f.j_rr.to_dense(), jac.to_dense())


def test_flow_lifecycle_rejects_mismatched_true_impes_weight(tmp_path):
    jac, rhs = sample_system()
    flow = sample_flow(jac)
    flow.true_impes_weights[0, 0] = 0.5
    cap.write_capture(tmp_path, 0, cap.CapturedSystem(0, "y2d6a-reject", "water", 0, ONE_CELL, jac, rhs,
                                                      None, flow))
    with pytest.raises(cap.CaptureError, match="true-IMPES weight mismatch at cell 0: 5e-1"):
        cap.load_captures(tmp_path)


def test_flow_lifecycle_rejects_fingerprint_and_partition_errors():
    jac, rhs = sample_system()
    flow = sample_flow(jac)
    flow.dune_istl_version = "2.10.0"
    text = cap.format_capture(cap.CapturedSystem(0, "x", "water", 0, ONE_CELL, jac, rhs, None, flow))
    with pytest.raises(cap.CaptureError, match="fingerprint mismatch"):
        cap.parse_capture(text)
    flow = sample_flow(jac)
    flow.j_rr = cap.csr_from_triplets(3, 3, [(0, 0, 4.0), (1, 1, 2.0), (2, 0, 1e12), (2, 2, 8.0)])
    text = cap.format_capture(cap.CapturedSystem(0, "x", "water", 0, ONE_CELL, jac, rhs, None, flow))
    with pytest.raises(cap.CaptureError, match=r"partition mismatch at \(0,2\)"):
        cap.parse_capture(text)


def test_true_impes_weight_of_a_coupled_block():
    block = np.array([[2.0, 1.0, 0.0], [0.5, 3.0, 0.2], [0.1, 0.0, 4.0]])
    w = cap.true_impes_weight(block)
    t = block.T.copy()
    t[0] *= 50.0
    raw = np.linalg.solve(t, [1.0, 0.0, 0.0])
    assert np.allclose(w, raw / np.max(np.abs(raw)), rtol=0, atol=1e-15)
    assert np.max(np.abs(w)) == 1.0


def test_parse_rejects_wrong_header_and_truncated_triplets():
    with pytest.raises(cap.CaptureError, match="unexpected header"):
        cap.parse_capture("not-a-capture")
    with pytest.raises(cap.CaptureError, match="empty file"):
        cap.parse_capture("")
    lines = EXPECTED_V2.splitlines()
    with pytest.raises(cap.CaptureError, match="expected 5 triplets, found 4"):
        cap.parse_capture("\n".join(lines[:-1]))


@pytest.mark.parametrize("edit, message", [
    (lambda L: L[:4], "missing dominant_item_index"),
    (lambda L: L[:5] + ["layout 1 3 0"] + L[6:], "layout expects 4 fields, got 3"),
    (lambda L: L[:7] + ["water 2 1e1"] + L[8:], "water expects 2 values, got 1"),
    (lambda L: L[:6] + ["equation_scaling 2"] + L[7:], "unexpected equation_scaling flag '2'"),
    (lambda L: L[:4] + ["dominant_family water", "layout none"] + L[6:], "expected dominant_item_index"),
    (lambda L: L[:15] + ["rhs_values"] + L[16:], "expected rhs section"),
    (lambda L: L[:18], "rhs truncated"),
    (lambda L: L[:19] + ["triplet"] + L[20:], "expected triplets section"),
    (lambda L: L[:20] + ["0 0"] + L[21:], "triplet missing value"),
    (lambda L: L[:20] + ["0 x 4e0"] + L[21:], "invalid digit"),
])
def test_parse_error_messages(edit, message):
    lines = EXPECTED_V2.splitlines()
    with pytest.raises(cap.CaptureError, match=message):
        cap.parse_capture("\n".join(edit(lines)) + "\n")


def test_duplicate_triplets_are_summed_and_rows_sorted():
    text = EXPECTED_V2.replace("nnz 5", "nnz 6").replace("2 2 8e0\n", "2 2 8e0\n0 0 1e0\n")
    text = text.replace("0 0 4e0\n0 2 -1.5e-8\n", "0 2 -1.5e-8\n0 0 4e0\n")
    s = cap.parse_capture(text)
    assert s.jacobian.nnz == 5
    assert s.jacobian.get(0, 0) == 5.0
    assert list(s.jacobian.col[:2]) == [0, 2]
    assert cap.format_capture(s).count("\n0 0 5e0\n") == 1


def test_crlf_and_blank_triplet_lines_are_accepted():
    text = EXPECTED_V2.replace("\n", "\r\n").replace("1 1 2e0\r\n", "1 1 2e0\r\n\r\n   \r\n")
    s = cap.parse_capture(text)
    assert np.array_equal(s.jacobian.to_dense(), sample_system()[0].to_dense())


def test_to_bsr_blocks_and_tail_rejection():
    rng = np.random.default_rng(3)
    n = 4
    dense = np.zeros((3 * n, 3 * n))
    for i, j in [(0, 0), (0, 1), (1, 0), (1, 1), (1, 3), (2, 2), (3, 1), (3, 3)]:
        dense[3 * i:3 * i + 3, 3 * j:3 * j + 3] = rng.standard_normal((3, 3))
    trip = [(r, c, dense[r, c]) for r, c in zip(*np.nonzero(dense))]
    jac = cap.csr_from_triplets(3 * n, 3 * n, trip)
    s = cap.CapturedSystem(0, "x", "water", 0, cap.Layout(n, 3, 0, 3 * n), jac, np.arange(3.0 * n))
    rp, cols, vals, rhs = cap.to_bsr(s)
    assert list(rp) == [0, 2, 5, 6, 8]
    assert list(cols) == [0, 1, 0, 1, 3, 2, 1, 3]
    rebuilt = np.zeros_like(dense)
    for i in range(n):
        for k in range(rp[i], rp[i + 1]):
            rebuilt[3 * i:3 * i + 3, 3 * cols[k]:3 * cols[k] + 3] = vals[9 * k:9 * k + 9].reshape(3, 3)
    assert np.array_equal(rebuilt, dense)
    assert np.array_equal(rhs, s.rhs)
    tail = cap.CapturedSystem(0, "x", "water", 0, cap.Layout(n - 1, 3, 1, 3 * n), jac, s.rhs)
    with pytest.raises(cap.CaptureError, match="tail-free"):
        cap.to_bsr(tail)
    with pytest.raises(cap.CaptureError, match="block layout"):
        cap.to_bsr(cap.CapturedSystem(0, "x", "water", 0, None, jac, s.rhs))
    # replay routes tail systems to the full-system seam only when the tail follows the cells and
    # the well BHP unknowns; these checks run before the device is touched
    with pytest.raises(cap.CaptureError, match="perforation tail"):
        cap.replay(None, tail)
    with pytest.raises(cap.CaptureError, match="block layout"):
        cap.replay(None, cap.CapturedSystem(0, "x", "water", 0, None, jac, s.rhs))


def oracle_capture(dims=(10, 9, 3), seed=11):
    """A tail-free Newton system assembled by the oracle, as a captured system."""
    from oracle.oracle_py import OracleSimulator
    from ressim_b200 import decks

    deck = decks.waterflood_3d(*dims, seed=seed, rate_per_perf=20.0)
    deck.wells = []
    deck.pressure = deck.pressure + np.linspace(0.0, 30.0, deck.n_cells)
    res, ptr, col, val = OracleSimulator(deck).assemble_current(2.0)
    n = deck.n_cells
    jac = cap.csr_from_arrays(3 * n, 3 * n, ptr, col, val)
    return deck, cap.CapturedSystem(0, "none", "water", 0, cap.Layout(n, 3, 0, 3 * n), jac, -res)


def test_oracle_system_round_trips_bit_exactly(tmp_path):
    deck, s = oracle_capture()
    cap.write_capture(tmp_path, 12, s)
    t = cap.load_captures(tmp_path)[0]
    assert np.array_equal(t.rhs.view(np.uint64), s.rhs.view(np.uint64))
    assert np.array_equal(t.jacobian.ptr, s.jacobian.ptr) and np.array_equal(t.jacobian.col, s.jacobian.col)
    assert np.array_equal(t.jacobian.val.view(np.uint64), s.jacobian.val.view(np.uint64))
    assert cap.format_capture(t) == cap.format_capture(s)
