"""Scene and solver constants with the reference's defaults (wp_sph/main.py:13-61).

Unlike the reference, nothing is baked in at import: ``wp_sph.solver.IISPH``
reads these module attributes when it is constructed, so a caller may change
them first.
"""
import math
from enum import Enum, auto
from pathlib import Path

MODEL_DIR = Path(__file__).parents[1] / "models"


def model_dir(filename):
    return MODEL_DIR / filename


class SceneType(Enum):
    HOUSE = auto()
    PLANE = auto()
    HAND = auto()
    EMPTY = auto()


scene_type = SceneType.EMPTY
DYNAMIC_SCENE = scene_type in [SceneType.PLANE, SceneType.HAND]

GRAVITY = 9.8
DIAMETER = 0.05
OMEGA = 0.5
ETA = 1.0e-3
RHO_0 = 1.0e3
INV_SMALL = 1.0e-6
FPS = 60

# Scene settings (main.py:34-53): the box of each scene type, no gravity for
# the plane; the mesh models each scene adds (IISPH.py:966-984) and the
# velocity its rigid body moves with (IISPH.py:1061-1081).
SCENE_BOX = {
    SceneType.HOUSE: (8.0, 10.0, 12.0),
    SceneType.PLANE: (8.0, 8.0, 8.0),
    SceneType.HAND: (8.0, 50.0, 8.0),
    SceneType.EMPTY: (4.0, 4.0, 4.0),
}
_C, _S = math.cos(math.radians(160)), math.sin(math.radians(160))
SCENE_MODELS = {
    SceneType.HOUSE: [("house.obj", 2e-2, (3.0, 0.0, 4.0), ((1, 0, 0), (0, 1, 0), (0, 0, 1)))],
    SceneType.PLANE: [("plane.obj", 3e-3, (0.0, 4.0, 4.0), ((1, 0, 0), (0, 0, -1), (0, 1, 0)))],
    SceneType.HAND: [("hand.obj", 0.3, (4.5, 2.0, 1.0), ((_C, -_S, 0), (_S, _C, 0), (0, 0, 1)))],
    SceneType.EMPTY: [],
}
RIGID_VELOCITY = {SceneType.PLANE: (2.0, 0.0, 0.0), SceneType.HAND: (0.0, 0.1, 0.0)}

BOX_WIDTH, BOX_HEIGHT, BOX_LENGTH = SCENE_BOX[scene_type]
if scene_type == SceneType.PLANE:
    GRAVITY = 0.0  # no gravity for the plane scene

SMOOTHING_LENGTH = 2 * DIAMETER
TIME_STEP_MAX = 5e-2 * DIAMETER
FLUID_MASS = RHO_0 * DIAMETER**3
SIGMA = 8 / (math.pi * SMOOTHING_LENGTH**3)
VIS_MU = 0.0 * RHO_0
