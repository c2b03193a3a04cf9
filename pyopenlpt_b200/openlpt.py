"""The drop-in module under the reference's shim name: ``import
pyopenlpt_b200.openlpt as lpt`` gives the classes of the reference's ``openlpt``
(Camera, Image, ImageIO, ObjectFinder2D, StereoMatch, Shake, IPR, STB, BasicSetting,
TracerConfig, run, ...) backed by the B200 library."""
from ._openlpt import *  # noqa: F401,F403
from ._openlpt import run  # noqa: F401
