"""The measurement kernels behind the tensor-pipe and warp-shuffle decisions
compute what they claim: one radix-16 DFT stage (butterflies and DFT-as-GEMM)
and one 384-point transform (exchange through shared memory and as a lane
transpose with warp shuffles), each checked inside the library against an
FP64 DFT, to FP32 accuracy."""

import ctypes as ct

import pytest

from azeban_b200 import _lib

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("method", [0, 1])
def test_radix16_stage_bench(method):
    ns, err = ct.c_double(), ct.c_double()
    _lib.check(_lib.lib.az_bench_radix16_stage(method, 4, ct.byref(ns), ct.byref(err)))
    assert err.value < 1e-6, err.value
    assert ns.value > 0


@pytest.mark.parametrize("method", [0, 1, 2])
def test_exchange384_bench(method):
    ns, err = ct.c_double(), ct.c_double()
    _lib.check(_lib.lib.az_bench_exchange384(method, 4, ct.byref(ns), ct.byref(err)))
    assert err.value < 1e-6, err.value
    assert ns.value > 0


def test_bench_entry_points_reject_bad_arguments():
    ns, err = ct.c_double(), ct.c_double()
    assert _lib.lib.az_bench_exchange384(3, 4, ct.byref(ns), ct.byref(err)) == _lib.AZ_ERR_INVALID
    assert _lib.lib.az_bench_radix16_stage(2, 4, ct.byref(ns), ct.byref(err)) == _lib.AZ_ERR_INVALID
