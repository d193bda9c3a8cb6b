"""zkmetal_b200: B200-native (sm_100a CUDA) multi-scalar multiplication.

A drop-in for zkMetal's G1 MSM path (BN254 and BLS12-381): the C ABI in
``include/zkmsm.h`` keeps the reference FFI's entry points; ``msm`` mirrors
the Swift engine API.  All arithmetic runs in ``libzkmsm.so``.
"""
from . import lib  # noqa: F401  (raises ImportError when the CUDA library is missing)
from .msm import (BLS12377MSM, BLS12381MSM, BN254G2MSM, CommitmentServer, CommitmentServerPool,  # noqa: F401
                  CommitmentTable, KZGEngine, route_pick,
                  MetalMSM, MSMError, MSMTask, PointProjective, batchMSMAsync, innerProductMSM,
                  innerProductMSMHalves, multiMSM, multiMSMPipelined)

__all__ = ["MetalMSM", "BLS12381MSM", "BLS12377MSM", "BN254G2MSM", "MSMError", "PointProjective", "multiMSM",
           "multiMSMPipelined", "innerProductMSM", "innerProductMSMHalves", "MSMTask", "batchMSMAsync",
           "CommitmentTable", "CommitmentServer", "CommitmentServerPool", "route_pick", "KZGEngine", "lib"]
