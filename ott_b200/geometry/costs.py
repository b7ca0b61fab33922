"""Cost functions (ott/geometry/costs.py). Only the squared Euclidean cost is
on this path; the others of the reference are outside it."""


class CostFn:
  """Base class of cost functions (costs.py:37)."""


class SqEuclidean(CostFn):
  """Squared Euclidean distance, ``|x|^2 + |y|^2 - 2 <x, y>`` (costs.py:548-573)."""

  def __eq__(self, other):
    return isinstance(other, SqEuclidean)

  def __hash__(self):
    return hash("SqEuclidean")

  def __repr__(self):
    return "SqEuclidean()"
