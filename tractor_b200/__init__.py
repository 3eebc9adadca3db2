"""tractor_b200: the Tractor's forward-model hot path on NVIDIA B200 (sm_100a).

Rendering of point sources and exp / deV / Sersic / composite galaxies with
mixture-of-Gaussians or pixelized PSFs, their parameter derivatives and the
least-squares step, behind the reference Tractor's object API (same class
and method names, arguments and return conventions).  The pixel work runs in
hand-written CUDA kernels (libtractor_b200.so, C ABI in
include/tractor_b200.h); there is no CPU implementation.
"""
__version__ = '0.1.0'

from .params import (BaseParams, ScalarParam, NamedParams, ParamList, MultiParams,
                     GaussianPriors, GaussianPriorsMixin)
from .patch import Patch, ModelMask, add_patches, get_overlapping_region
from .basics import (PixPos, NullWCS, Flux, Mag, Mags, Fluxes, NanoMaggies, MultiBandBrightness,
                     NullPhotoCal, LinearPhotoCal, FluxesPhotoCal, MagsPhotoCal, NullSky,
                     ConstantSky, Image)
from .ellipses import GalaxyShape, EllipseE, EllipseESoft
from .profiles import MixtureOfGaussians, SersicMixture
from .psf import (HybridPSF, HybridPixelizedPSF, GaussianMixturePSF, GaussianMixtureEllipsePSF,
                  NCircularGaussianPSF,
                  PixelizedPSF, NormalizedPixelizedPsf, MogParams)
from .sources import (BasicSource, SingleProfileSource, PointSource, Galaxy, ProfileGalaxy,
                      HoggGalaxy, GaussianGalaxy, ExpGalaxy, DevGalaxy, SersicGalaxy, SersicIndex,
                      CompositeGalaxy,
                      FracDev, SoftenedFracDev, FixedCompositeGalaxy)
from .engine import Tractor, Catalog, Images
from .optimizer import (B200Optimizer, B200ConstrainedOptimizer, LsqrOptimizer,
                        ConstrainedOptimizer)

__all__ = [
    'BaseParams', 'ScalarParam', 'NamedParams', 'ParamList', 'MultiParams', 'GaussianPriors',
    'Patch', 'ModelMask', 'add_patches', 'get_overlapping_region',
    'PixPos', 'NullWCS', 'Flux', 'Mag', 'Fluxes', 'NanoMaggies', 'NullPhotoCal', 'LinearPhotoCal',
    'NullSky', 'ConstantSky', 'Image', 'Mags', 'FluxesPhotoCal', 'MagsPhotoCal',
    'LsqrOptimizer', 'ConstrainedOptimizer',
    'GalaxyShape', 'EllipseE', 'EllipseESoft',
    'MixtureOfGaussians', 'SersicMixture',
    'HybridPSF', 'HybridPixelizedPSF', 'GaussianMixturePSF', 'GaussianMixtureEllipsePSF',
    'NCircularGaussianPSF', 'PixelizedPSF',
    'NormalizedPixelizedPsf',
    'PointSource', 'Galaxy', 'ProfileGalaxy', 'HoggGalaxy', 'GaussianGalaxy', 'ExpGalaxy',
    'DevGalaxy', 'SersicGalaxy', 'SersicIndex', 'FracDev', 'SoftenedFracDev',
    'FixedCompositeGalaxy', 'CompositeGalaxy',
    'Tractor', 'Catalog', 'Images', 'B200Optimizer', 'B200ConstrainedOptimizer',
]
