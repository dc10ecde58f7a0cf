"""B200-native hash GROUP BY aggregation (sm_100a CUDA kernels behind a C ABI).

A drop-in for the tiled group-by path of PneNPproof/cpu_gpu_coprocess_groupby_agg
(``groupby_agg_partition`` + ``groupby_agg_intra_partition``).  The product is
``lib/libgba.so`` (C ABI in ``include/gba.h``, C++ drop-ins in
``include/tiled_groupby_agg_partition.hpp``); this package is its Python host
binding.
"""
from .api import Context, Result, Server, gen_device, gen_host, gen_spec, make_knobs  # noqa: F401
from . import _abi  # noqa: F401
