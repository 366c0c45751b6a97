"""The allocation-free G1 MSM entry point (g16_msm_g1_device_noalloc).

Some callers of this library cannot call cudaMalloc, because their device
memory belongs to another allocator or because an allocation in their request
path is not acceptable.  For them the library offers one MSM that runs inside a
fixed scratch array built into the library.  This file checks, through the C
ABI, that it returns exactly what the allocating entry point returns: on two
calls in a row (the second sees the first call's leftovers in the shared
scratch), at the largest size it accepts, and that it refuses a larger input.
At that largest size both results are also compared with the oracle's.  The
library's device-allocation counter must not move across these calls (after the
allocating entry point's own calls), and the refused call must launch nothing.
It sorts last so that a failure here leaves every other test already run.
"""
import ctypes

import pytest

import oracle as O
import snarkrs_b200 as S

pytestmark = pytest.mark.gpu

MAX_POINTS = 16384


def _on_device(backend, data):
    d = backend.alloc(len(data))
    backend.upload(d, data)
    return d


def _noalloc(device, d_bases, d_scalars, n, form=S.SCALARS_STANDARD):
    out = ctypes.create_string_buffer(64)
    rc = S.lib().g16_msm_g1_device_noalloc(ctypes.c_int(device), ctypes.c_void_p(d_bases),
                                           ctypes.c_void_p(d_scalars), ctypes.c_size_t(n), ctypes.c_int(form), out)
    return rc, out.raw


def test_noalloc_msm_matches_the_allocating_entry_point():
    backend = S.CudaBackend(0)
    msm = S.CudaMsm(backend)
    buffers = []
    try:
        cases = [(1000, 0), (MAX_POINTS, 1), (MAX_POINTS, 0), (37, 1)]
        inputs = []
        for n, dist in cases:
            bases = S.synth_points(1, 900 + n + dist, n)
            scal = S.synth_scalars(901 + n + dist, n, dist)
            db, ds = _on_device(backend, bases), _on_device(backend, scal)
            buffers += [db, ds]
            want = msm.msm_g1_device(db, ds, n)
            if n == MAX_POINTS:
                assert want == O.msm_g1(bases, scal)
            inputs.append((n, db, ds, want))
        allocs = S.device_alloc_count()
        for n, db, ds, want in inputs:
            for _ in range(2):          # two calls in a row on the shared scratch
                rc, got = _noalloc(backend.ordinal, db, ds, n)
                assert rc == S.G16_OK, S.last_error()
                assert got == want
        assert S.device_alloc_count() == allocs, "the allocation-free MSM called cudaMalloc"
        # Montgomery-form scalars through both entry points
        n = 512
        want = msm.msm_g1_device(buffers[0], buffers[1], n, S.SCALARS_MONTGOMERY)
        allocs = S.device_alloc_count()
        rc, got = _noalloc(backend.ordinal, buffers[0], buffers[1], n, S.SCALARS_MONTGOMERY)
        assert rc == S.G16_OK, S.last_error()
        assert got == want
        # beyond the fixed scratch: refused, nothing launched, nothing allocated
        launches = S.launch_count()
        rc, _ = _noalloc(backend.ordinal, buffers[2], buffers[3], MAX_POINTS + 1)
        assert rc == S.InvalidArgumentError.code
        assert "16384" in S.last_error()
        assert S.launch_count() == launches
        assert S.device_alloc_count() == allocs
    finally:
        for d in buffers:
            backend.free(d)
        backend.close()
