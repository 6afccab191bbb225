"""vecruntime_b200 -- a B200 (sm_100a) backend for VecRuntime's grouped aggregate.

The product is libvrgpu.so (C ABI, include/vrgpu.h) with hand-written CUDA
kernels; this package is its Python host mirror of the reference's operator
interface. Importing it does not touch the GPU; creating an aggregate loads
the library and fails loudly when it was not built.
"""
from .aggregate import (AggFunction, AggregateServer, AverageAgg, AverageMergeAgg, CountAgg, CountMergeAgg,
                        DecimalProduct, GpuBatchedAggregate, GpuHashAggregate, MinMaxAgg, Spec, SumDoubleAgg, SumLongAgg, WideDecimalAvgAgg,
                        WideDecimalAvgMergeAgg, WideDecimalSumAgg, WideDecimalSumMergeAgg)
from .columns import (Col, DeviceBatch, HostBatch, bools, decimals, decimals128, dict_ids, doubles, host_batch,
                      ints, longs, pack_bits, unpack_bits)
from .native import VrError, lib

__all__ = [
    "AggFunction", "AggregateServer", "AverageAgg", "AverageMergeAgg", "CountAgg", "CountMergeAgg", "DecimalProduct",
    "GpuBatchedAggregate", "GpuHashAggregate", "MinMaxAgg", "Spec", "SumDoubleAgg", "SumLongAgg", "WideDecimalAvgAgg",
    "WideDecimalAvgMergeAgg", "WideDecimalSumAgg", "WideDecimalSumMergeAgg", "Col", "DeviceBatch", "HostBatch",
    "bools", "decimals", "decimals128", "dict_ids", "doubles", "host_batch", "ints", "longs", "pack_bits",
    "unpack_bits", "VrError", "lib",
]
