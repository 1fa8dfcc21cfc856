"""B200-native engine for the AIR Tools II SIRT/ART hot path.

Public API mirrors the reference MATLAB toolbox: ``sirt``/``art`` and the
method wrappers, the ``paralleltomo``/``fanlineartomo`` test problems and the
afun operator handle.  All iterations run in libairt.so (hand-written CUDA for
sm_100a); the package raises on import if the library is missing.
"""
from ._lib import AirtError, lib as _load_lib
from .afun import AirtOperator, afun_matrix, as_operator
from .batch import ParallelBatch
from .analytic import fbp
from .unet import UNet
from .solvers import (art, calczeta, cart, cav, cimmino, columnaction, drop, kaczmarz, landweber,
                      randkaczmarz, sart, sirt, symkaczmarz)
from .testprobs import (add_noise, cosd, fancurvedtomo, fanlineartomo, paralleltomo, phantomgallery,
                        random_ellipses, seismictomo, sind, sphericaltomo)

_load_lib()

__all__ = ["AirtError", "AirtOperator", "ParallelBatch", "UNet", "afun_matrix", "as_operator", "art", "calczeta", "cart", "cav", "columnaction", "fbp",
           "cimmino", "drop", "kaczmarz", "landweber", "randkaczmarz", "sart", "sirt",
           "symkaczmarz", "add_noise", "cosd", "fancurvedtomo", "fanlineartomo", "paralleltomo", "seismictomo",
           "sphericaltomo",
           "phantomgallery", "random_ellipses", "sind"]
