"""Segmented solves (tools/segment_sinkhorn.py) on the GPU against the
reference's own run (golden vectors: every segment padded, one padded solve
per segment). reg_ot_cost within 1e-5 relative (FP32 path)."""
import numpy as np
import pytest

from tests import golden_cases

pytestmark = pytest.mark.gpu


def _clouds(seed, nx, ny, d):
  rng = np.random.default_rng(seed)
  return (rng.uniform(size=(nx, d)).astype(np.float32),
          rng.uniform(size=(ny, d)).astype(np.float32))


@pytest.mark.parametrize("name", golden_cases.segment_names())
def test_segments_match_reference_golden(name):
  """The reference's own segment_sinkhorn (padded segments, vmapped solves)."""
  import torch
  from ott_b200.tools import segment_sinkhorn as ss
  data, kw = golden_cases.load_segment(name, "f64")
  kw = dict(kw)
  for k in ("weights_x", "weights_y"):
    if k in kw:
      kw[k] = torch.as_tensor(kw[k], dtype=torch.float32).cuda()
  for k in ("segment_ids_x", "segment_ids_y"):
    if k in kw:
      kw[k] = torch.as_tensor(kw[k])
  got = ss.segment_sinkhorn(torch.as_tensor(data["x"], dtype=torch.float32).cuda(),
                            torch.as_tensor(data["y"], dtype=torch.float32).cuda(), **kw)
  np.testing.assert_allclose(got.detach().cpu().numpy(), data["costs"], rtol=1e-5)


def test_segment_gradient_matches_single_solves():
  """d(sum of segment costs)/dx on a segment's rows equals the gradient of
  that segment's own solve."""
  import torch
  from ott_b200.geometry import pointcloud
  from ott_b200.solvers import linear
  from ott_b200.tools import segment_sinkhorn as ss
  npx, npy = (50, 70), (60, 40)
  x, y = _clouds(5, 120, 100, 3)
  xt = torch.as_tensor(x).cuda().requires_grad_()
  ss.segment_sinkhorn(xt, torch.as_tensor(y).cuda(), num_per_segment_x=npx,
                      num_per_segment_y=npy, epsilon=0.05).sum().backward()
  x0 = torch.as_tensor(x[:50]).cuda().requires_grad_()
  linear.reg_ot_cost(pointcloud.PointCloud(x0, torch.as_tensor(y[:60]).cuda(), epsilon=0.05),
                     torch.full((50,), 1 / 50, device="cuda"),
                     torch.full((60,), 1 / 60, device="cuda")).backward()
  np.testing.assert_allclose(xt.grad[:50].cpu().numpy(), x0.grad.cpu().numpy(), rtol=1e-5,
                             atol=1e-7)
