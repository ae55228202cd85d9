"""B200 static priority search tree: Python host mirror of the reference's interface.

The compute path is libpst_b200.so (hand-written sm_100a CUDA behind a C ABI,
include/pst_c.h); this package only binds it with ctypes.  torch provides device
memory and streams.  There is no CPU fallback: every call raises PSTError when the
library or a CUDA device is missing.

Names follow the reference (arraylistnumstring/static-priority-search-tree):
StaticPSTGPU with threeSidedSearch / twoSidedLeftSearch / twoSidedRightSearch
(pst/static-pst-gpu.h:103-128), intervalParallelSearch
(interval-parallel-search/interval-parallel-search.h:29), formMetacellTags
(helpers/isosurface-data-processing.h:69) and calcNumMetacells (:23).
"""
from .pst import (  # noqa: F401
    BatchEngine,
    PSTError,
    Server,
    StaticPSTGPU,
    StaticPSTGPUArr,
    calcNumMetacells,
    formMetacellTags,
    formMetacellTagsFromFile,
    free_device,
    intervalParallelSearch,
    lib,
    library_path,
    make_queries,
    marchingCubes,
    marchingCubesTables,
    point_dtype,
    points_to_device,
    readInVertices,
)
