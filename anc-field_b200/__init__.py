"""B200 FDTD core of anc-field: C-ABI library bindings, the Python mirror
of the reference Simulation class, and seeded workloads.

Import as a package from its directory (the directory name carries a
hyphen), e.g. through importlib; see load() in __graft_entry__.py.
"""
from . import afd, lms, sharding, slabs, surrogate, workloads  # noqa: F401
from .afd import AfdError, Model, Simulation, check_filters, default_params, library  # noqa: F401
