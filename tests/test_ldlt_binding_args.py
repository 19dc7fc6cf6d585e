"""Host-side argument handling of `rslab_b200.ldlt` (no GPU needed): the
reference's validation of method / memory and square, supported-dtype input
(python/src/lib.rs:74-118, :930-947)."""
import numpy as np
import pytest
import scipy.sparse as sp

from rslab_b200 import InvalidInput, ldlt
from rslab_b200.ldlt import _lower_csc


def test_lower_triangle_extraction_sums_duplicates():
    A = sp.coo_matrix(([1.0, 2.0, 3.0, 4.0], ([0, 1, 1, 0], [0, 0, 1, 0])), shape=(2, 2)).tocsc()
    a = _lower_csc(A)
    assert a.n == 2
    assert list(a.col_ptr) == [0, 2, 3]
    assert list(a.row_idx) == [0, 1, 1]
    assert list(a.values) == [5.0, 2.0, 3.0]


@pytest.mark.parametrize("kw", [{"method": "banded"}, {"memory": "huge"}, {"threads": -1}])
def test_bad_keywords(kw):
    with pytest.raises(ValueError):
        ldlt(sp.eye(3, format="csc"), **kw)


def test_non_square_and_dtype_rejected():
    with pytest.raises(InvalidInput):
        ldlt(sp.random(3, 4, density=0.5, format="csc"))
    with pytest.raises(InvalidInput):
        ldlt(sp.eye(3, format="csc", dtype=np.int64))
