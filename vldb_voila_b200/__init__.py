"""voila-b200: the CUDA flavor of VOILA's data-parallel hot path (selections, hash-join
build/probe and hash group-by) for one NVIDIA B200, behind a C ABI (include/voila_cuda.h)."""
from .engine import (Engine, Query, VoilaError, Workload, batch_specs, generate_host, generate_workload_host, lib,
                     workload, zipf_cdf)

__all__ = ["Engine", "Query", "VoilaError", "Workload", "batch_specs", "generate_host", "generate_workload_host",
           "lib", "workload", "zipf_cdf"]
