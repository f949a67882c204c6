"""pyyrtpet_b200: YRT-PET's projection hot path on B200 (sm_100a).

Drop-in Python surface for the reference's projector / OSEM API
(``import pyyrtpet_b200 as yrt``).  All projection work runs in libyrtb.so
(yrt-pet_b200/lib), reached through the C ABI of include/yrt_b200.h.
"""
from ._lib import YrtbError, lib  # noqa: F401
from .core import (BinIteratorChronologicalInterleaved,  # noqa: F401
                   BinIteratorRangeHistogram3D, DeviceEvents, DeviceProjector,
                   Histogram3D, ImageParams, ListModeLUT,
                   OperatorProjectorDevice, ProjectionList,
                   ProjectionListOwned, ProjectionOper, ProjectorParams,
                   Scanner, UniformHistogram, convertToHistogram3D,
                   histo3d_bins, histo3d_detpairs, read_psf_csv,
                   release_cached_memory, write_psf_csv)
from .osem import OSEM_GPU, createOSEM  # noqa: F401
from .psf import (ConvolutionKernel, ConvolutionKernelGaussian,  # noqa: F401
                  ConvolutionKernelGaussianMixture, OperatorPsfDevice,
                  OperatorVarPsfDevice, write_image_psf_csv)
from .lrem import LREM_GPU, LowRankProjector  # noqa: F401
from .ranges import RangeList  # noqa: F401

ListModeLUTOwned = ListModeLUT
ListModeLUTAlias = ListModeLUT
Histogram3DOwned = Histogram3D
