"""Connected components on the B200: the label fixpoint equals the
oracle's (labels[v] = min id reaching v), the partition equals the
oracle's after min-id canonicalisation, and it matches the reference's CC
kernel on the same BVSS."""
import numpy as np
import pytest

import oracle as O
from blest_b200 import Graph, relabel_dense
from graphs import golden_cases, small_cases

pytestmark = pytest.mark.gpu

CASES = small_cases() + golden_cases()


@pytest.fixture(params=CASES, ids=[c[0] for c in CASES])
def case(request, gpu):
    csc, bvss, csr = request.param[1]()
    return csc, bvss, csr, Graph(bvss, csr)


def test_labels_equal_oracle(case):
    csc, bvss, csr, g = case
    want = O.cc_csc(csc.n, csc.col_ptrs, csc.rows)
    lab, st = g.cc()
    np.testing.assert_array_equal(lab, want)
    assert st.no_components == int(np.unique(want).size)
    np.testing.assert_array_equal(O.canonical_min_labels(lab), O.canonical_min_labels(want))
    dense, k = relabel_dense(lab)
    assert k == st.no_components
    # repeated run is identical
    lab2, _ = g.cc()
    np.testing.assert_array_equal(lab, lab2)


@pytest.mark.skipif(not O.ref_available(), reason="reference harness not built")
def test_matches_reference_cc_kernel(case):
    csc, bvss, csr, g = case
    if csc.nnz == 0:
        pytest.skip("the reference kernels need at least one slice")
    ref = O.RefGraph.from_bvss(csc.n, bvss.arrays(), bvss.full_padding, bvss.update_divergence,
                               csr.col_ptrs, csr.rows)
    raw, _ = ref.cc_raw(csc.n)
    lab, st = g.cc()
    np.testing.assert_array_equal(lab, raw)
    # the reference's own hostCode result: same component count
    _, _, k = ref.cc(csc.n)
    assert k == st.no_components
