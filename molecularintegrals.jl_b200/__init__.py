"""molints_b200: a B200-native (sm_100a) two-electron repulsion integral engine.

Drop-in for the ERI hot path of MolecularIntegrals.jl (``all_twoe_ints`` /
``all_twoe_ints_chrr`` / ``all_twoe_ints_rys``): the packed output uses the reference's
``iindex`` layout and normalised functions.  The compute runs in ``libmolints_cuda.so``
(hand-written CUDA for sm_100a behind a C ABI); this package is its Python host side.

The directory is named ``molecularintegrals.jl_b200``; since that is not an importable
identifier the package is registered as ``molints_b200`` by ``load_package`` in the
repository's ``__graft_entry__.py``.
"""
from . import basis  # noqa: F401
from .basis import (Shells, atom, build_basis, config0, config1, config2, config3,  # noqa: F401
                    config3_molecule, config4_arrivals, config4_request, h2, ethane_staggered)
