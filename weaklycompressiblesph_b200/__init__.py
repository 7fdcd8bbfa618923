"""B200-native weakly-compressible SPH hydro force path.

* ``fdps``   FDPS multiwalk plugin mirror (HydrDispatchKernel / HydrRetrieveKernel)
* ``sim``    device-resident solver (``Solver``): cell binning, density, EoS,
             hydro, KDK and CFL dt on the device, many instances at once
* ``cases``  seeded problem setups (dam break, periodic lattice, ensembles, requests)
* ``serving`` continuous-batching request loop over a ``Solver``

The compute path is libwcsph.so (csrc/, sm_100a); there is no CPU fallback.
"""
from . import _native  # noqa: F401
from .cases import Case, Physics, dam_break, ensemble_cases, periodic_lattice, serving_requests  # noqa: F401

__all__ = ["Case", "Physics", "dam_break", "periodic_lattice", "ensemble_cases", "serving_requests"]
