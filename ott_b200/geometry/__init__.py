from ott_b200.geometry import costs, epsilon_scheduler, geometry, pointcloud  # noqa: F401
