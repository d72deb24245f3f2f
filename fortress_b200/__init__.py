"""fortress_b200 -- B200-native split-step Fourier propagator for the coupled
Gross-Pitaevskii equations of spin-orbit-coupled spin-1 / spin-2 condensates
(the path of FORTRESS's cgpe{1,2,3}d programs), behind a C ABI
(include/fgpe.h, libfgpe.so)."""
from ._abi import FgpeError
from .config import RunConfig
from .propagator import Propagator, device_ok

__all__ = ["FgpeError", "RunConfig", "Propagator", "device_ok"]
