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

BOX_WIDTH = 4.0
BOX_HEIGHT = 4.0
BOX_LENGTH = 4.0

SMOOTHING_LENGTH = 2 * DIAMETER
TIME_STEP_MAX = 5e-2 * DIAMETER
FLUID_MASS = RHO_0 * DIAMETER**3
SIGMA = 8 / (math.pi * SMOOTHING_LENGTH**3)
VIS_MU = 0.0 * RHO_0
