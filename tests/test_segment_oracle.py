"""The oracle's segmented solves (padding as geometry/segment.py, one padded
solve per segment) reproduce the reference's own tools/segment_sinkhorn.py
run (golden vectors) to 1e-12 in float64."""
import numpy as np
import pytest

from oracle import sinkhorn_np as o
from tests import golden_cases


@pytest.mark.parametrize("name", golden_cases.segment_names())
def test_oracle_segments_match_reference(name):
  data, kw = golden_cases.load_segment(name, "f64")
  got = o.segment_sinkhorn(data["x"], data["y"], **kw)
  np.testing.assert_allclose(got, data["costs"], rtol=1e-12)
