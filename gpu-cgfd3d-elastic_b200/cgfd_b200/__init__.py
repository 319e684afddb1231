"""Python bindings of libcgfd_b200 (the B200-native CGFD3D elastic time loop).

The product is the C ABI declared in include/cgfd_b200.h; this package only builds the
problem description from numpy arrays, calls the library through ctypes and generates the
seeded synthetic inputs used by the tests and the benchmark.
"""
from .abi import (  # noqa: F401
    CGFD_MEDIUM_ACOUSTIC_ISO, CGFD_MEDIUM_ELASTIC_ISO, CGFD_MEDIUM_ELASTIC_VTI, CGFD_MEDIUM_ELASTIC_ANISO,
    CGFD_MEDIUM_VISCO_ISO, visco_gmb,
    CGFD_PREC_FP32, CGFD_PREC_BF16_COEF, CGFD_PREC_FP16_COEF, CGFD_PREC_U16_COEF, CGFD_PREC_FP16_WAVE, CGFD_PREC_FP64,
    CGFD_MEDIA_LOC, CGFD_MEDIA_HAR, CGFD_MEDIA_ARI, media_layer_gpu, media_layer_any_gpu, media_bin_gpu, media_grid_gpu,
    WAVELETS, Problem, Simulation, Server, problem_bytes, lib, lib_path, CgfdError, ref_shape, medium_ncmp,
)
