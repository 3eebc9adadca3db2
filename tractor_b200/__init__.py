"""tractor_b200: the Tractor's forward-model hot path on NVIDIA B200 (sm_100a).

Rendering of point sources and exp / deV / Sersic / composite galaxies with
mixture-of-Gaussians or pixelized PSFs, their parameter derivatives and the
least-squares step, behind the reference Tractor's object API.
"""
__version__ = '0.1.0'
