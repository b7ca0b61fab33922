"""Re-runs the reference's own code over the NumPy stand-in for jax on one
golden case and checks the committed vectors are what it produces (skipped
where the reference source tree is absent, e.g. on the GPU machine)."""
import os
import warnings

import numpy as np
import pytest

from oracle import reference_loader
from tests import golden_cases

ROOT = reference_loader.DEFAULT_ROOT


@pytest.mark.skipif(not os.path.isdir(os.path.join(ROOT, "ott")),
                    reason="reference source tree not present")
def test_golden_vectors_regenerate_from_reference():
  warnings.filterwarnings("ignore")
  ref = reference_loader.load(ROOT, x64=True)
  data, _, _, _ = golden_cases.load("refprob_eps0.1", "f64")
  geom = ref.pointcloud.PointCloud(data["x"], data["y"], epsilon=0.1)
  out = ref.solve(geom, data["a"], data["b"])
  np.testing.assert_array_equal(np.asarray(out.f), data["f"])
  np.testing.assert_array_equal(np.asarray(out.g), data["g"])
  np.testing.assert_array_equal(np.asarray(out.errors), data["errors"])
  assert float(out.reg_ot_cost) == float(data["reg_ot_cost"])
