"""The drop-in module under the reference's names.  The compiled module is
``pyopenlpt`` (pyopenlpt_b200/pyopenlpt*.so), so with ``pyopenlpt_b200/`` on
``sys.path`` both ``import pyopenlpt as lpt`` and ``import openlpt as lpt`` work
unchanged; ``import pyopenlpt_b200.openlpt as lpt`` works from the repository root.
Classes: Camera, Image, ImageIO, ObjectFinder2D, StereoMatch, Shake, IPR, STB,
BasicSetting, ObjectConfig, TracerConfig, run, ... backed by the B200 library."""
import os
import sys

try:
    import pyopenlpt  # noqa: F401
except ImportError:
    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    import pyopenlpt  # noqa: F401
from pyopenlpt import *  # noqa: F401,F403,E402
from pyopenlpt import run  # noqa: F401,E402
