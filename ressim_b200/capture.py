"""Reader and writer of the reference's captured linear systems, and their replay on the device.

The reference dumps the Jacobian, right-hand side and block layout of a Newton linear solve to a
text file (`fim-capture-v2`, or `fim-capture-v3` with a source-pinned companion section), so that
linear solvers can be compared offline on identical systems (src/lib/ressim/src/fim/linear/
capture.rs: writer `try_write_capture` :198-349, parser `parse_capture` :380-643, v3 companion
checks `validate_capture_data` in flow_lifecycle.rs:153-224).

- `parse_capture` / `read_capture` accept both versions with the reference parser's checks and
  error messages, including the v3 companion checks.
- `format_capture` / `write_capture` write byte-for-byte what the reference writes for the same
  system: numbers in Rust's shortest `{:e}` form, matrix rows in CSR order.
- `replay` solves a captured system on a simulator of the deck it came from: a tail-free system
  (reservoir cells only, three unknowns per cell) through `rf_linear_solve_bsr`, a system with a
  well tail (one BHP per well, one rate per perforation) through `rf_linear_solve_csr`, which
  eliminates the wells, solves and recovers the tail on the device as a Newton step does.
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass, field
from decimal import Decimal

import numpy as np

# Fingerprint of the v3 companion section (flow_lifecycle.rs:20-26).
FLOW_SOURCE_TAG = "release/2026.04/final"
FLOW_SOURCE_COMMIT = "b82f21dba405286c4c4446614dd3bf9cdebf7a2c"
DUNE_ISTL_VERSION = "2.11.0"
TRUE_IMPES_PRESSURE_SCALE_BAR = 50.0

SCALING_ROWS = ("water", "oil_component", "gas_component", "well_constraint", "perforation_flow")
PARTITIONS = ("j_rr", "j_rw", "j_wr", "j_ww")


class CaptureError(ValueError):
    """A capture file that the reference parser would also reject; the message is its message."""


@dataclass
class Layout:
    """`FimLinearBlockLayout` (fim/linear/mod.rs): cell blocks first, then the well tail."""
    cell_block_count: int
    cell_block_size: int
    well_bhp_count: int
    perforation_tail_start: int

    def cell_unknown_count(self) -> int:
        return self.cell_block_count * self.cell_block_size


@dataclass
class Csr:
    rows: int
    cols: int
    ptr: np.ndarray
    col: np.ndarray
    val: np.ndarray

    @property
    def nnz(self) -> int:
        return len(self.val)

    def get(self, r: int, c: int) -> float:
        lo, hi = int(self.ptr[r]), int(self.ptr[r + 1])
        k = lo + int(np.searchsorted(self.col[lo:hi], c))
        return float(self.val[k]) if k < hi and self.col[k] == c else 0.0

    def to_dense(self) -> np.ndarray:
        d = np.zeros((self.rows, self.cols))
        for r in range(self.rows):
            for k in range(int(self.ptr[r]), int(self.ptr[r + 1])):
                d[r, self.col[k]] = self.val[k]
        return d


@dataclass
class FlowLifecycle:
    """The v3 companion section (`FimFlowLifecycleCapture`, capture.rs)."""
    source_tag: str
    source_commit: str
    dune_istl_version: str
    pressure_scale_bar: float
    storage_blocks: np.ndarray  # (cells, 3, 3)
    true_impes_weights: np.ndarray  # (cells, 3)
    reservoir_unknown_count: int
    j_rr: Csr
    j_rw: Csr
    j_wr: Csr
    j_ww: Csr


@dataclass
class CapturedSystem:
    newton_iteration: int
    failure_reason: str
    dominant_family: str
    dominant_item_index: int
    layout: Layout | None
    jacobian: Csr
    rhs: np.ndarray
    equation_scaling: dict | None = None
    flow_lifecycle: FlowLifecycle | None = field(default=None)


def rust_exp(v: float) -> str:
    """Rust's `{:e}` for an f64: the shortest digits that round-trip, as d[.ddd]e<exp>."""
    if math.isnan(v):
        return "NaN"
    if math.isinf(v):
        return "inf" if v > 0 else "-inf"
    if v == 0.0:
        return "-0e0" if math.copysign(1.0, v) < 0 else "0e0"
    sign, digits, exponent = Decimal(repr(v)).normalize().as_tuple()
    ds = "".join(str(d) for d in digits)
    mantissa = ds[0] + ("." + ds[1:] if len(ds) > 1 else "")
    return ("-" if sign else "") + f"{mantissa}e{exponent + len(ds) - 1}"


def csr_from_triplets(rows: int, cols: int, trip) -> Csr:
    """Triplets to CSR like sprs `TriMat::to_csr`: columns sorted within a row, duplicates summed
    in the order they were added."""
    by_row = [dict() for _ in range(rows)]
    for r, c, v in trip:
        d = by_row[r]
        d[c] = d[c] + v if c in d else v
    ptr = np.zeros(rows + 1, dtype=np.int64)
    col_l, val_l = [], []
    for r in range(rows):
        cs = sorted(by_row[r])
        col_l.extend(cs)
        val_l.extend(by_row[r][c] for c in cs)
        ptr[r + 1] = len(col_l)
    return Csr(rows, cols, ptr, np.array(col_l, dtype=np.int64), np.array(val_l, dtype=np.float64))


def csr_from_arrays(rows: int, cols: int, ptr, col, val) -> Csr:
    """A CSR matrix from arrays whose columns are sorted and unique within each row."""
    return Csr(rows, cols, np.asarray(ptr, dtype=np.int64), np.asarray(col, dtype=np.int64),
               np.asarray(val, dtype=np.float64))


def _lines(text: str):
    """Rust `str::lines`: split on '\\n', drop one trailing empty line and a '\\r' before '\\n'."""
    parts = text.split("\n")
    if parts and parts[-1] == "":
        parts.pop()
    return iter(p[:-1] if p.endswith("\r") else p for p in parts)


def _uint(s: str) -> int:
    if not s.isdigit():
        raise CaptureError(f"invalid digit found in string {s!r}" if s else "cannot parse integer from empty string")
    return int(s)


def _float(s: str) -> float:
    try:
        return float(s)
    except ValueError:
        raise CaptureError(f"invalid float literal {s!r}") from None


def _field(line, key):
    if line is None:
        raise CaptureError(f"missing {key}")
    if not line.startswith(key):
        raise CaptureError(f"expected {key}, got {line!r}")
    return line[len(key):].strip()


def true_impes_weight(block) -> np.ndarray:
    """True-IMPES weight of one cell (flow_lifecycle.rs:32-59): solve S^T w = e_0, where S is the
    3x3 storage block with its pressure column scaled by 50 bar, then divide by max |w|."""
    t = np.array(block, dtype=np.float64).T.copy()
    t[0, :] *= TRUE_IMPES_PRESSURE_SCALE_BAR
    try:
        w = np.linalg.solve(t, np.array([1.0, 0.0, 0.0]))
    except np.linalg.LinAlgError:
        raise CaptureError("singular true-IMPES storage block") from None
    if not np.all(np.isfinite(w)):
        raise CaptureError("non-finite true-IMPES storage solve")
    scale = float(np.max(np.abs(w)))
    if not math.isfinite(scale) or scale <= np.finfo(np.float64).eps:
        raise CaptureError("degenerate true-IMPES normalization")
    return w / scale


def validate_flow_lifecycle(flow: FlowLifecycle, layout: Layout, jacobian: Csr) -> None:
    """The v3 companion checks (flow_lifecycle.rs:153-224): source fingerprint, cardinalities,
    recomputed true-IMPES weights within 1e-12, partition shapes, and a bit-exact partition of
    the full Jacobian into reservoir/well blocks."""
    if (flow.source_tag != FLOW_SOURCE_TAG or flow.source_commit != FLOW_SOURCE_COMMIT
            or flow.dune_istl_version != DUNE_ISTL_VERSION
            or abs(flow.pressure_scale_bar - TRUE_IMPES_PRESSURE_SCALE_BAR) > np.finfo(np.float64).eps):
        raise CaptureError("Y2d6 source/config fingerprint mismatch")
    if (layout.cell_block_size != 3 or len(flow.storage_blocks) != layout.cell_block_count
            or len(flow.true_impes_weights) != layout.cell_block_count
            or flow.reservoir_unknown_count != layout.cell_unknown_count()):
        raise CaptureError("Y2d6 storage/layout cardinality mismatch")
    for cell, (block, captured) in enumerate(zip(flow.storage_blocks, flow.true_impes_weights)):
        gap = float(np.max(np.abs(true_impes_weight(block) - np.asarray(captured))))
        if gap > 1e-12:
            raise CaptureError(f"Y2d6 true-IMPES weight mismatch at cell {cell}: {rust_exp(gap)}")
    res = flow.reservoir_unknown_count
    well = max(jacobian.rows - res, 0)
    want = {"j_rr": (res, res), "j_rw": (res, well), "j_wr": (well, res), "j_ww": (well, well)}
    for name in PARTITIONS:
        m = getattr(flow, name)
        if (m.rows, m.cols) != want[name]:
            raise CaptureError("Y2d6 reservoir/well partition dimensions mismatch")
    full = jacobian.to_dense()
    parts = {n: getattr(flow, n).to_dense() for n in PARTITIONS}
    stitched = np.zeros_like(full)
    stitched[:res, :res] = parts["j_rr"]
    stitched[:res, res:] = parts["j_rw"]
    stitched[res:, :res] = parts["j_wr"]
    stitched[res:, res:] = parts["j_ww"]
    bad = np.argwhere(stitched.view(np.uint64) != full.view(np.uint64))
    if len(bad):
        r, c = (int(v) for v in bad[0])
        raise CaptureError(f"Y2d6 partition mismatch at ({r},{c})")


def parse_capture(text: str) -> CapturedSystem:
    """Parse one capture file's text (capture.rs:380-643)."""
    lines = _lines(text)
    nxt = lambda: next(lines, None)  # noqa: E731
    header = nxt()
    if header is None:
        raise CaptureError("empty file")
    if header not in ("fim-capture-v2", "fim-capture-v3"):
        raise CaptureError(f"unexpected header {header!r}")
    newton_iteration = _uint(_field(nxt(), "newton_iteration"))
    failure_reason = _field(nxt(), "failure_reason")
    dominant_family = _field(nxt(), "dominant_family")
    dominant_item_index = _uint(_field(nxt(), "dominant_item_index"))
    lay = _field(nxt(), "layout")
    if lay == "none":
        layout = None
    else:
        parts = [_uint(p) for p in lay.split()]
        if len(parts) != 4:
            raise CaptureError(f"layout expects 4 fields, got {len(parts)}")
        layout = Layout(*parts)

    def scale_row(key):
        rest = _field(nxt(), key).split()
        if not rest:
            raise CaptureError(f"{key} missing count")
        count, values = _uint(rest[0]), [_float(p) for p in rest[1:]]
        if len(values) != count:
            raise CaptureError(f"{key} expects {count} values, got {len(values)}")
        return np.array(values, dtype=np.float64)

    flag = _field(nxt(), "equation_scaling")
    if flag == "0":
        scaling = None
    elif flag == "1":
        scaling = {k: scale_row(k) for k in SCALING_ROWS}
    else:
        raise CaptureError(f"unexpected equation_scaling flag {flag!r}")

    def dense_rows(key, ncols):
        count = _uint(_field(nxt(), key))
        out = np.zeros((count, ncols))
        for i in range(count):
            line = nxt()
            if line is None:
                raise CaptureError(f"{key} truncated at row {i}")
            vals = [_float(p) for p in line.split()]
            if len(vals) != ncols:
                raise CaptureError(f"{key} row {i} expects {ncols} values, got {len(vals)}")
            out[i] = vals
        return out

    def sparse(name):
        dims = [_uint(p) for p in _field(nxt(), f"matrix_{name}").split()]
        if len(dims) != 3:
            raise CaptureError(f"matrix_{name} expects rows cols nnz")
        r, c, nz = dims
        trip = []
        for e in range(nz):
            line = nxt()
            if line is None:
                raise CaptureError(f"matrix_{name} truncated at entry {e}")
            p = line.split()
            for i, what in enumerate(("row", "column", "value")):
                if len(p) <= i:
                    raise CaptureError(f"matrix_{name} missing {what}")
            row, col, v = _uint(p[0]), _uint(p[1]), _float(p[2])
            if len(p) > 3 or row >= r or col >= c:
                raise CaptureError(f"matrix_{name} invalid entry {e}")
            trip.append((row, col, v))
        return csr_from_triplets(r, c, trip)

    flow = None
    if header == "fim-capture-v3":
        if _field(nxt(), "flow_lifecycle") != "1":
            raise CaptureError("fim-capture-v3 requires flow_lifecycle 1")
        tag = _field(nxt(), "flow_source_tag")
        commit = _field(nxt(), "flow_source_commit")
        dune = _field(nxt(), "dune_istl_version")
        pscale = _float(_field(nxt(), "pressure_scale_bar"))
        storage = dense_rows("storage_blocks", 9).reshape(-1, 3, 3)
        weights = dense_rows("true_impes_weights", 3)
        res_count = _uint(_field(nxt(), "reservoir_unknown_count"))
        mats = [sparse(n) for n in PARTITIONS]
        flow = FlowLifecycle(tag, commit, dune, pscale, storage, weights, res_count, *mats)

    rows = _uint(_field(nxt(), "rows"))
    cols = _uint(_field(nxt(), "cols"))
    nnz = _uint(_field(nxt(), "nnz"))
    if nxt() != "rhs":
        raise CaptureError("expected rhs section")
    rhs = np.zeros(rows)
    for r in range(rows):
        line = nxt()
        if line is None:
            raise CaptureError("rhs truncated")
        rhs[r] = _float(line.strip())
    if nxt() != "triplets":
        raise CaptureError("expected triplets section")
    trip = []
    for line in lines:
        line = line.strip()
        if not line:
            continue
        p = line.split()
        for i, what in enumerate(("row", "col", "value")):
            if len(p) <= i:
                raise CaptureError(f"triplet missing {what}")
        r, c, v = _uint(p[0]), _uint(p[1]), _float(p[2])
        if r >= rows or c >= cols:
            raise CaptureError(f"triplet ({r},{c}) outside a {rows}x{cols} matrix")
        trip.append((r, c, v))
    if len(trip) != nnz:
        raise CaptureError(f"expected {nnz} triplets, found {len(trip)}")
    system = CapturedSystem(newton_iteration, failure_reason, dominant_family, dominant_item_index, layout,
                            csr_from_triplets(rows, cols, trip), rhs, scaling, flow)
    if flow is not None:
        if layout is None:
            raise CaptureError("fim-capture-v3 requires a block layout")
        validate_flow_lifecycle(flow, layout, system.jacobian)
    return system


def read_capture(path) -> CapturedSystem:
    with open(path) as f:
        text = f.read()
    try:
        return parse_capture(text)
    except CaptureError as e:
        raise CaptureError(f"{path}: {e}") from None


def load_captures(directory) -> list[CapturedSystem]:
    """Every `fim_capture_*.txt` in `directory`, sorted by file name (capture.rs:351-378)."""
    names = sorted(n for n in os.listdir(directory) if n.startswith("fim_capture_") and n.endswith(".txt"))
    return [read_capture(os.path.join(directory, n)) for n in names]


def _matrix_lines(out, m: Csr, prefix=""):
    for r in range(m.rows):
        for k in range(int(m.ptr[r]), int(m.ptr[r + 1])):
            out.append(f"{prefix}{r} {int(m.col[k])} {rust_exp(float(m.val[k]))}")


def format_capture(s: CapturedSystem) -> str:
    """The text the reference writes for this system (capture.rs:198-349): v3 when it carries a
    companion section, else v2."""
    out = ["fim-capture-v3" if s.flow_lifecycle is not None else "fim-capture-v2",
           f"newton_iteration {s.newton_iteration}", f"failure_reason {s.failure_reason}",
           f"dominant_family {s.dominant_family}", f"dominant_item_index {s.dominant_item_index}"]
    if s.layout is None:
        out.append("layout none")
    else:
        lay = s.layout
        out.append(f"layout {lay.cell_block_count} {lay.cell_block_size} {lay.well_bhp_count} "
                   f"{lay.perforation_tail_start}")
    if s.equation_scaling is None:
        out.append("equation_scaling 0")
    else:
        out.append("equation_scaling 1")
        for k in SCALING_ROWS:
            v = s.equation_scaling[k]
            out.append(f"{k} {len(v)}" + "".join(" " + rust_exp(float(x)) for x in v))
    f = s.flow_lifecycle
    if f is not None:
        out += ["flow_lifecycle 1", f"flow_source_tag {f.source_tag}", f"flow_source_commit {f.source_commit}",
                f"dune_istl_version {f.dune_istl_version}", f"pressure_scale_bar {rust_exp(f.pressure_scale_bar)}"]
        for key, rows in (("storage_blocks", np.asarray(f.storage_blocks).reshape(-1, 9)),
                          ("true_impes_weights", np.asarray(f.true_impes_weights).reshape(-1, 3))):
            out.append(f"{key} {len(rows)}")
            out += [" ".join(rust_exp(float(v)) for v in row) for row in rows]
        out.append(f"reservoir_unknown_count {f.reservoir_unknown_count}")
        for name in PARTITIONS:
            m = getattr(f, name)
            out.append(f"matrix_{name} {m.rows} {m.cols} {m.nnz}")
            _matrix_lines(out, m)
    j = s.jacobian
    out += [f"rows {j.rows}", f"cols {j.cols}", f"nnz {j.nnz}", "rhs"]
    out += [rust_exp(float(v)) for v in s.rhs]
    out.append("triplets")
    _matrix_lines(out, j)
    return "\n".join(out) + "\n"


def write_capture(directory, sequence: int, s: CapturedSystem) -> str:
    """Write `<directory>/fim_capture_<sequence:05>.txt` (capture.rs:208-210); returns the path."""
    os.makedirs(directory, exist_ok=True)
    path = os.path.join(directory, f"fim_capture_{sequence:05d}.txt")
    with open(path, "w") as fh:
        fh.write(format_capture(s))
    return path


def to_bsr(s: CapturedSystem):
    """A tail-free captured system as 3x3 block CSR: (block row pointers, block columns, row-major
    3x3 block values, right-hand side)."""
    lay = s.layout
    if lay is None or lay.cell_block_size != 3:
        raise CaptureError("replay needs a block layout with 3 unknowns per cell")
    n = lay.cell_block_count
    j = s.jacobian
    if lay.well_bhp_count != 0 or j.rows != 3 * n or j.cols != 3 * n:
        raise CaptureError(
            f"replay takes tail-free systems of 3 x {n} rows; this one has {j.rows} rows and "
            f"{lay.well_bhp_count} well BHP unknowns (systems with a well tail replay through "
            f"rf_linear_solve_csr)")
    blocks = [dict() for _ in range(n)]
    for r in range(j.rows):
        for k in range(int(j.ptr[r]), int(j.ptr[r + 1])):
            c = int(j.col[k])
            b = blocks[r // 3].setdefault(c // 3, np.zeros(9))
            b[3 * (r % 3) + (c % 3)] = j.val[k]
    rp, cols, vals = [0], [], []
    for i in range(n):
        for c in sorted(blocks[i]):
            cols.append(c)
            vals.append(blocks[i][c])
        rp.append(len(cols))
    return (np.array(rp, dtype=np.int32), np.array(cols, dtype=np.int32),
            np.concatenate(vals) if vals else np.zeros(0), s.rhs.copy())


def replay(sim, s: CapturedSystem):
    """Solve a captured system on the device, on `sim`, a ReservoirSimulator of the deck the
    capture came from.  Tail-free systems go through `rf_linear_solve_bsr`; systems with a well
    tail through `rf_linear_solve_csr`, whose unknowns must follow the layout's order (cells,
    well BHPs from `perforation_tail_start - well_bhp_count`, perforation rates from
    `perforation_tail_start`) with `sim`'s wells and perforations.  Returns (x, report)."""
    from .simulator import linear_solve_bsr, linear_solve_csr

    lay = s.layout
    if lay is None or lay.cell_block_size != 3:
        raise CaptureError("replay needs a block layout with 3 unknowns per cell")
    j = s.jacobian
    n = lay.cell_block_count
    if lay.well_bhp_count == 0 and j.rows == 3 * n:
        rp, cols, vals, rhs = to_bsr(s)
        return linear_solve_bsr(sim, rp, cols, vals, rhs)
    if j.rows != j.cols or lay.perforation_tail_start != 3 * n + lay.well_bhp_count:
        raise CaptureError(
            f"replay needs a square system whose perforation tail starts after the cells and the "
            f"{lay.well_bhp_count} well BHP unknowns; this one is {j.rows} x {j.cols} with the "
            f"tail at {lay.perforation_tail_start}")
    return linear_solve_csr(sim, j.ptr, j.col, j.val, s.rhs)
