"""B200-native LBLRTM layer optical-depth and radiance-merge path.

* ``lblrtm_b200.gpu``      -- binding of the CUDA library (include/lblgpu.h)
* ``lblrtm_b200.abi``      -- ctypes structs of the C ABI
* ``lblrtm_b200.configs``  -- seeded synthetic inputs of the benchmark cases
* ``lblrtm_b200.tape3``    -- TAPE3 line-file writer/reader
* ``lblrtm_b200.build``    -- in-tree build of the sm_100a library
"""
from . import abi, configs  # noqa: F401

__all__ = ["abi", "configs", "gpu", "tape3", "build"]
