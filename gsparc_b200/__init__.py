"""gsparc_b200 -- B200-native sparse tensor contraction (SpTC) engine.

A drop-in for the SpTC path of seohyeon0322/GSPARC: linearise -> sort ->
match -> accumulate (dense window | on-chip ESC) -> memory-aware output
chunking, as hand-written sm_100a CUDA behind a C ABI (include/gsparc_b200.h).
"""
from .synth import CooTensor  # noqa: F401
from .api import (  # noqa: F401
    ACCUM_AUTO, ACCUM_DENSE, ACCUM_ESC, Context, DeviceTensor, GsparcError, SpTC, SpTCResult,
    decode_keys, digest_chunk, splitmix64, index_match, layout, lib, linearize, plan_shards, read_tns, read_quantum, sort_pairs, sptc,
    sptc_batch, sptc_host, Server, ServerTensor, sptc_resident, ResidentResult, autotune, Plan,
    version, write_tns, LIB_PATH, CLI_PATH, EXPORTS,
)
