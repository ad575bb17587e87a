"""heatflow_mpm on B200: the Eulerian air substep of Heatflow-MPM as sm_100a CUDA behind the reference's Python API."""
from .grid import GridConfig, AirGrid  # noqa: F401
from .heat import HeatField  # noqa: F401
from .heater import Heater, BoxHeater  # noqa: F401
from .mpm import DLPackBody, Material, ThermalMPM, FrozenBody  # noqa: F401
from .solver import HeatflowMPM, KAPPA_AIR  # noqa: F401
from .batch import AirScenario, AirBatch, autotune, ensemble, shard_scenarios  # noqa: F401
from .serve import AirServer, Request, poisson_trace  # noqa: F401
from .frames import FrameWriter  # noqa: F401
from .shapes import load_mesh, sample_interior, mesh_particles, BUNNY  # noqa: F401

__version__ = "0.3.0"
