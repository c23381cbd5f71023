"""jfli_b200 — the jax-fli particle-mesh force step and lightcone painting on one B200.

Same public names as jax_fli for this path (`lpt`, `nbody`, the solver classes,
`PaintingOptions`, the field containers, `power`); arrays are CUDA torch tensors and
every operation on them runs in libjfli_b200's sm_100a kernels.
"""

from . import cosmology, ops, utils
from . import io_api as io
from . import fields as units
from .catalog import CATALOG_VERSION, Catalog
from .cosmology import Cosmology, Planck18
from .fields import (
    AbstractField,
    DensityField,
    DensityUnit,
    FieldStatus,
    PaintingOptions,
    ParticleField,
    PhysicalUnit,
    PositionUnit,
    ConvergenceUnit,
    FieldMetadata,
    FlatDensity,
    FlatKappaField,
    FlatShearField,
    PowerSpectrum,
    SphericalDensity,
    SphericalKappaField,
    SphericalShearField,
    convert_units,
    uniform_particles,
)
from .initial import gaussian_initial_conditions, interpolate_initial_conditions, white_noise
from .lensing import RedshiftDistribution, born, kde_nz, smail_nz, tophat_nz
from .pm import (
    AbstractNBodySolver,
    DriftInterp,
    EfficientDriftDoubleKick,
    InterpTilerState,
    NoCorrection,
    NoInterp,
    OnionTiler,
    PGDKernel,
    ReversibleDoubleKickDrift,
    SharpeningKernel,
    TelephotoInterp,
    get_all_47_symmetries,
    lpt,
    nbody,
)
from .power import (angular_cl_flat, angular_cl_spherical, coherence, cross_angular_cl_spherical, power,
                    transfer)
from .utils import (
    centers,
    compute_box_size_from_redshift,
    compute_lightcone_shells,
    compute_max_redshift_from_box_size,
    compute_particle_scale_factors,
    distances,
    edges,
)

__version__ = "0.1.0"
