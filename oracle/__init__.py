"""Oracles for the maximal k-biplex enumerator -- TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU legs import this
package.  It holds:
  * liboracle.so   -- our C restatement (kbiplex_oracle.c), dense adjacency;
  * _ref/bppivot   -- the reference's own CPU enumerator (BPPivot), compiled
                      from its sources by oracle/Makefile;
  * _ref/gmkbpe    -- the reference's own GPU enumerator (make -C oracle refgpu),
                      run on a machine with a GPU as a second reference;
  * brute_force    -- exhaustive definition check for graphs of <= 16 vertices;
  * result_hash    -- the canonical per-result hash shared with the CUDA code.
"""
from .oracle import (  # noqa: F401
    MASK64, OracleStats, brute_force, classify, enumerate_oracle, liboracle_path,
    parse_bppivot_sets, result_hash, run_bppivot, set_summary, bppivot_path,
    parse_reference_results, refgpu_path, run_reference_gpu,
)
