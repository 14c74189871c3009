"""Substrate part of the reference's ``prrtc`` extension module.

The planner plugins reach the collision–kinematics substrate through three
names of ``prrtc`` (``python/gpu_planning/plugins/_substrate_planner_base.py``:
``prrtc.RobotModelBuilder``, ``prrtc.SceneCollisionDataBuilder`` and
``prrtc.check_collision_scene``, bound in ``cpp/src/python/bindings.cpp``).
This module provides those names with the same fields, keywords and results,
backed by ``libprism_b200.so``, so a plugin can ``import prismplan_b200.prrtc
as prrtc``. The planners themselves (``solve_scene``, ``*_solve_scene`` and
their settings and buffer types) are not part of the substrate and are not
provided: asking for one raises AttributeError with that explanation.
"""
from .api import check_collision_scene  # noqa: F401
from .robot import RobotModelBuilder  # noqa: F401
from .scene import SceneCollisionDataBuilder  # noqa: F401

__all__ = ["RobotModelBuilder", "SceneCollisionDataBuilder", "check_collision_scene"]


def __getattr__(name):
    raise AttributeError(
        f"prrtc.{name} is not part of the collision–kinematics substrate; this module provides only "
        + ", ".join(__all__))
