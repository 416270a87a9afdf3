"""B200-native EFIE method-of-moments hot path (drop-in for the CUDA MEX
entry points of mahmut26/Matlab-cuda-efief-vs-cpu).

The package directory name contains hyphens, so import it with
``importlib.import_module("matlab-cuda-efief-vs-cpu_b200")`` after putting the
repository root on ``sys.path``.
"""
from .api import *  # noqa: F401,F403
from .api import __all__  # noqa: F401
from ._native import MexError, lib, context  # noqa: F401
