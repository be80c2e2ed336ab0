"""B200 CFPQ closure engine: Python plumbing around libcfpq_b200.so.

The engine is the C ABI library (csrc/, include/cfpq_b200.h) and the C++
drop-in backend (cpp/cfpq/B200Matrix.h, bin/b200GPU).  This package exposes
  capi       ctypes binding of the C ABI
  query      grammar / graph text formats and a one-call query runner
  workloads  seeded synthetic workloads in the reference's text formats
  shard      LPT sharding of query batches over ranks
  rowblock   row-block closure of one large query over several GPUs
The directory name contains hyphens; import it with
importlib.import_module("cfpq-on-gpgpu_b200").
"""
from . import capi, query, rowblock, shard, workloads  # noqa: F401

__all__ = ["capi", "query", "rowblock", "shard", "workloads"]
