"""B200 engine for the propagate-and-retrieve path of Ziggyware/DiffractiveOpticalElement.

The public names mirror the reference's ES-module exports (src/index.js:13-21)
for the functions on that path. Every numerical routine runs in hand-written
sm_100a CUDA kernels behind the C ABI in include/doe_b200.h
(``libdoe_b200.so``); there is no CPU implementation to fall back to.
"""
from ._lib import DOEError, EngineUnavailable, Context, context, load_library
from .fft import fft2d, fft2dOut, isPow2, nextPow2
from .field import ComplexField, discMask, rectMask, ringMask
from .doe import (DEFAULT_DESIGN, blurRaster, designDOE, errorDiffusionQuantize, flatPhase, fourierCgh, gerchbergSaxton,
                  gerchbergSaxtonMultiPlane, illuminationProfile, kinoformLens, makeRng, prepareTargetAmp,
                  randomPhase, weightedGerchbergSaxton, wrapPhase)
from .interference import (modalIntensity, partiallyCoherentModes, propagatedModalIntensity, reconstructHologram,
                           recordHologram)
from .projector import DEFAULT_PROJECTOR, ProjectorSystem, autoRoi, makeTarget
from .propagate import (
    DEFAULT_WAVELENGTH,
    angularSpectrumTransferFunction,
    focalPlaneSpectrum,
    focusSweep,
    fresnelMinDistance,
    localFrequencyLimit,
    propagate,
    propagateAngularSpectrum,
    propagateAngularSpectrumInPlace,
    propagateFraunhofer,
    propagateFresnelFFT,
    propagateFresnelFFTInverse,
)

__all__ = [
    "DOEError", "EngineUnavailable", "Context", "context", "load_library",
    "fft2d", "fft2dOut", "isPow2", "nextPow2", "ComplexField",
    "DEFAULT_WAVELENGTH", "angularSpectrumTransferFunction", "focalPlaneSpectrum", "focusSweep",
    "fresnelMinDistance", "localFrequencyLimit", "propagate", "propagateAngularSpectrum",
    "propagateAngularSpectrumInPlace", "propagateFraunhofer", "propagateFresnelFFT", "propagateFresnelFFTInverse",
    "discMask", "rectMask", "ringMask", "DEFAULT_DESIGN", "blurRaster",
    "designDOE", "errorDiffusionQuantize", "flatPhase", "fourierCgh", "gerchbergSaxton", "gerchbergSaxtonMultiPlane", "illuminationProfile",
    "kinoformLens", "makeRng", "prepareTargetAmp", "randomPhase", "weightedGerchbergSaxton", "wrapPhase",
    "DEFAULT_PROJECTOR", "ProjectorSystem", "autoRoi", "makeTarget",
    "modalIntensity", "partiallyCoherentModes", "propagatedModalIntensity", "reconstructHologram", "recordHologram",
]
