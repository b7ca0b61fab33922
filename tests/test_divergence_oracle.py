"""The oracle's Sinkhorn divergence (three solves; symmetric terms with
parallel updates and momentum 1/2) reproduces the reference's own
tools/sinkhorn_divergence.py run (golden vectors) to 1e-12 in float64."""
import numpy as np
import pytest

from oracle import sinkhorn_np as o
from tests import golden_cases


@pytest.mark.parametrize("name", golden_cases.divergence_names())
def test_oracle_divergence_matches_reference(name):
  data, geom, dkw, weights = golden_cases.load_divergence(name, "f64")
  a, b = (data["a"], data["b"]) if weights else (None, None)
  div, res = o.sinkhorn_divergence(data["x"], data["y"], a, b, **geom, **dkw)
  np.testing.assert_allclose(div, float(data["divergence"]), rtol=1e-12, atol=1e-15)
  assert [r.n_iters for r in res] == data["n_iters"].tolist()
  for r, tag in zip(res, ("xy", "xx", "yy")):
    np.testing.assert_allclose(r.f, data["f_" + tag], rtol=0, atol=1e-11)
    np.testing.assert_allclose(r.g, data["g_" + tag], rtol=0, atol=1e-11)
