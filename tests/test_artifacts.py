"""The reference's binary artifacts of an estimate (cellwise_error.bin,
cellwise_error_components.bin, x_indicator_components.bin), written by the library through the C ABI from host
arrays (no GPU): byte for byte against the files the reference's own writers produced
for the golden cases, 2+1D and 1+1D (fixtures ``bin_*``, by ``tests/golden/make_golden.py``).  The values
are taken from the reference's files, given to the writer in mesh-cell order, so the
comparison pins the header, the block layout and the entry order (decreasing value,
ties by increasing cell id)."""
import os

import numpy as np
import pytest

from conftest import GOLDEN, GOLDEN_CASES, GOLDEN_CASES_1D


def _parse(raw: np.ndarray, n_header: int, n_cols: int):
    b = raw.tobytes()
    head = np.frombuffer(b, dtype=np.int32, count=n_header)
    n = int(head[1])
    ids = np.frombuffer(b, dtype=np.int32, count=n, offset=4 * n_header)
    cols = [np.frombuffer(b, dtype=np.float64, count=n, offset=4 * n_header + 4 * n + 8 * n * k)
            for k in range(n_cols)]
    assert len(b) == 4 * n_header + 4 * n + 8 * n * n_cols
    return head, ids, cols


@pytest.mark.parametrize("name", GOLDEN_CASES + GOLDEN_CASES_1D)
def test_cellwise_error_binaries_match_reference_bytes(name, tmp_path):
    from doubleadapparabolicfem_b200.estimator import (write_cellwise_error_binary,
                                                       write_cellwise_error_components_binary)
    z = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    ref = z["bin_cellwise_error"]
    head, ids, (vals,) = _parse(ref, 2, 1)
    assert head[0] == 1
    order = np.argsort(ids, kind="stable")  # hand the writer the cells in mesh order
    out = tmp_path / "cellwise_error.bin"
    write_cellwise_error_binary(out, ids[order], vals[order])
    assert out.read_bytes() == ref.tobytes()

    refc = z["bin_cellwise_error_components"]
    headc, idsc, colsc = _parse(refc, 3, 4)
    assert list(headc) == [1, len(idsc), 4]
    order = np.argsort(idsc, kind="stable")
    cells = {k: c[order] for k, c in zip(("flux", "reconstruction", "divergence", "eta"), colsc)}
    outc = tmp_path / "cellwise_error_components.bin"
    write_cellwise_error_components_binary(outc, idsc[order], cells)
    assert outc.read_bytes() == refc.tobytes()
    # sort_descending = False keeps the given order
    write_cellwise_error_binary(out, ids[order], vals[order], sort_descending=False)
    _, ids2, (vals2,) = _parse(np.fromfile(out, dtype=np.uint8), 2, 1)
    assert np.array_equal(ids2, ids[order]) and np.array_equal(vals2, vals[order])


def test_cellwise_error_binary_ties_break_by_cell_id(tmp_path):
    from doubleadapparabolicfem_b200.estimator import write_cellwise_error_binary
    ids = np.array([7, 3, 5, 1], dtype=np.int32)
    vals = np.array([1.0, 2.0, 1.0, 2.0])
    out = tmp_path / "e.bin"
    write_cellwise_error_binary(out, ids, vals)
    _, ids2, (vals2,) = _parse(np.fromfile(out, dtype=np.uint8), 2, 1)
    assert list(ids2) == [1, 3, 5, 7] and list(vals2) == [2.0, 2.0, 1.0, 1.0]


@pytest.mark.parametrize("name", GOLDEN_CASES + GOLDEN_CASES_1D)
def test_x_indicator_components_binary_matches_reference_bytes(name, tmp_path):
    from doubleadapparabolicfem_b200.estimator import write_x_indicator_components_binary
    z = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    ref = z["bin_x_indicator_components"]
    head, ids, (lam, trace, eta) = _parse(ref, 3, 3)
    assert list(head) == [1, len(ids), 3]
    order = np.argsort(ids, kind="stable")
    out = tmp_path / "x_indicator_components.bin"
    write_x_indicator_components_binary(out, ids[order], lam[order], trace[order], eta[order])
    assert out.read_bytes() == ref.tobytes()
