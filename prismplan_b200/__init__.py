"""B200-native (sm_100a) collision-kinematics substrate for PrismPlan's planners.

Drop-in surface (names of the reference ``prrtc`` module and substrate):
``RobotModelBuilder``, ``SceneCollisionDataBuilder``, ``PlanningScene``,
``check_collision_scene``, ``EdgeEvalGpu``, ``load_robot_asset``,
``build_robot_model``; device-resident torch ops ``check_configs``,
``check_edges``, ``traj_cost``, ``rollout_costs``, ``hinge_cost``; the
batched optimisers ``chomp_solve`` / ``chomp_optimize`` and
``stomp_solve`` / ``stomp_optimize``; the mixed-request batch
``MixedBatch``; the launch-shape tuners ``tune_edges`` / ``tune_configs``.
The compute path is the CUDA library ``libprism_b200.so``; importing this
package does not load it (so CPU-only tooling works), the first call does and
fails loudly if it is missing.
"""
from ._lib import PrismError  # noqa: F401
from .api import (  # noqa: F401
    ChompResult,
    ChompSettings,
    CostParams,
    EdgeEvalGpu,
    EdgeEvalParams,
    MixedBatch,
    StompSettings,
    check_collision_scene,
    check_configs,
    check_edges,
    chomp_linear_init,
    chomp_optimize,
    chomp_solve,
    chomp_workspace,
    edges_workspace,
    fk_spheres,
    hinge_cost,
    rollout_costs,
    stomp_optimize,
    stomp_solve,
    stomp_workspace,
    traj_cost,
    tune_configs,
    tune_edges,
)
from .robot import RobotModelBuilder, build_robot_model, load_robot_asset  # noqa: F401
from .scene import PlanningScene, SceneCollisionDataBuilder, SceneTensors  # noqa: F401
