"""gmkbe_b200: maximal k-biplex enumeration on NVIDIA B200 (sm_100a).

A drop-in for the enumeration path of the GMkBPE reference: same .graph.bin
input, same -f/-k/-r/-d command line (gmkbe_b200/gmk, `python -m gmkbe_b200`),
and a C ABI (include/gmk.h, libgmk.so) for embedding.  The search runs only
on the GPU; without the built library every entry point raises.
"""
from .api import (EXPORTS, LIB_PATH, Graph, GmkError, Stats, enumerate_batch,  # noqa: F401
                  load_library, plan_tasks, result_hash)

__all__ = ["Graph", "GmkError", "Stats", "enumerate_batch", "load_library", "plan_tasks",
           "result_hash",
           "EXPORTS", "LIB_PATH"]
