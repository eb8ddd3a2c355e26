"""B200-native exhaustive War enumerator: a drop-in for the gpu/war_gpu.py path of
OrygnsCode/endless-games-of-war.  The modules of this directory import each other as top-level modules
(the directory name is not a Python identifier), so importing the package puts the directory on
sys.path first.

  warlib   ctypes binding of libwar.so (C ABI: include/war.h)
  war_gpu  the drop-in CLI and run()
  autotune launch-shape sweeps with a JSON cache
  serve    Python face of the continuous-batching job server
  shard    rank-range sharding and result reduction across processes
  build    nvcc build of libwar.so for sm_100a
"""
import os
import sys

_HERE = os.path.dirname(os.path.abspath(__file__))
if _HERE not in sys.path:
    sys.path.insert(0, _HERE)

import warlib  # noqa: E402,F401
from war_gpu import run  # noqa: E402,F401
