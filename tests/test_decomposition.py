"""The row-strip decomposition of the reference's multi-GPU driver
(HP/MultiGPU_CatchFlood_main.py ave_loadStep / ave_overlapMask), as
baseline/ref_loop.py restates it for running the reference's Parallel_SWE
class, against tests/golden/multigpu/decomposition.npz (made by
tests/golden/make_decomposition.py from the reference's own functions):
square urban rasters and ragged masks with holes, 2 to 4 ranks, and the
masks on which the reference itself raises IndexError."""
import os

import numpy as np
import pytest

from baseline import ref_loop

Z = np.load(os.path.join(os.path.dirname(__file__), "golden", "multigpu",
                         "decomposition.npz"))
CASES = range(int(Z["n_cases"]))


@pytest.mark.parametrize("k", CASES)
def test_decomposition_matches_reference(k):
    mask, size = Z[f"mask_{k}"], int(Z[f"size_{k}"])
    if f"raises_{k}" in Z:
        with pytest.raises(IndexError):
            ref_loop.row_splits(mask, size)
        return
    splits = ref_loop.row_splits(mask, size)
    assert splits == [int(v) for v in Z[f"splits_{k}"]]
    np.testing.assert_array_equal(ref_loop.overlap_mask(mask, splits, size).numpy(),
                                  Z[f"overlap_{k}"])
    # every valid row in exactly one rank's own rows, two overlap rows per edge
    spans = [ref_loop.rank_rows(splits, r, size, mask.shape[0]) for r in range(size)]
    assert spans[0][0] == 0 and spans[-1][1] == mask.shape[0]
    for (a0, b0), (a1, b1) in zip(spans, spans[1:]):
        assert b0 - a1 == 4
