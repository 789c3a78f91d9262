"""B200 (sm_100a) execution core for MiniLake's hot path: filter/expression
kernels over selection vectors and dictionary codes, hash aggregation, hash-join
build/probe and top-N, behind MiniLake's Operator / Sink / LocalSink contract.

``minilake_b200.gpu`` loads the CUDA library (``_lib/libminilake_gpu.so``) and
fails loudly when it is missing; there is no CPU execution path.
"""
from . import abi, columns, datagen  # noqa: F401
