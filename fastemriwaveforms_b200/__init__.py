"""B200-native interpolated mode summation for FastEMRIWaveforms.

Drop-in for ``few.summation.interpolatedmodesum.InterpolatedModeSum`` and its
``CubicSplineInterpolant`` (and, around it, ``FDInterpolatedModeSum``,
``get_fundamental_frequencies``, ``AmpInterp2D`` and the dense output of
``DOPR853``): Python host code over hand-written sm_100a CUDA
kernels reached through the C ABI of ``libfew_b200.so`` (include/few_b200.h).
"""
from .aakwave import AAKSummation
from .amplitude import AmpInterp2D
from .directmodesum import DirectModeSum
from .dopr853 import DOPR853
from .fdinterp import FDInterpolatedModeSum
from .geodesic import get_fundamental_frequencies
from .modeselector import ModeSelector
from .summation import CubicSplineInterpolant, InterpolatedModeSum, SummationBase
from .utility import get_mismatch, get_overlap
from .ylm import GetYlms

__all__ = ["AAKSummation", "AmpInterp2D", "CubicSplineInterpolant", "DOPR853", "DirectModeSum", "FDInterpolatedModeSum", "GetYlms", "InterpolatedModeSum",
           "ModeSelector", "SummationBase", "get_fundamental_frequencies", "get_mismatch", "get_overlap"]
