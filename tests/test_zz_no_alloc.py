"""lfts_dots_static (the allocation-free, context-free inner products) against
lfts_dots, the context entry point it mirrors.  The file name sorts last so
that the static scratch array is exercised after every other test has run;
the test also passes on its own."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MAX_JOBS = 256  # LFTS_DOTS_STATIC_MAX_JOBS


def _job_set(ctx, rng, nj, dtype):
    """nj dot jobs over a pool of eight vectors, every third job with a weight."""
    from langevinfts_b200.capi import DotJob
    pool = [rng.random(ctx.M).astype(dtype) + (0.5 if k >= 6 else 0.0) for k in range(8)]
    ptr = [ctx.upload(v) for v in pool]
    jobs, ref = [], []
    for j in range(nj):
        ia, ib = j % 6, (5 * j + 1) % 6
        iw = 6 + j % 2 if j % 3 == 0 else None
        scale = 0.5 + 0.01 * j
        jobs.append(DotJob(ptr[ia], ptr[ib], ptr[iw] if iw is not None else None, scale))
        v = pool[ia].astype(np.float64) * pool[ib].astype(np.float64)
        if iw is not None:
            v = v / pool[iw].astype(np.float64)
        ref.append(scale * v.sum())
    arr = (DotJob * nj)(*jobs)
    return ctx.upload(np.frombuffer(arr, dtype=np.uint8)), np.array(ref)


@pytest.mark.parametrize("precision", [8, 4])
def test_dots_static_matches_context_dots_twice(precision):
    from langevinfts_b200.capi import Context, check
    ctx = Context([16, 12, 10], precision=precision)
    lib = ctx.lib
    stream = lib.lfts_ctx_stream(ctx.h)
    rng = np.random.default_rng(11 + precision)
    dtype = np.float64 if precision == 8 else np.float32
    tol = 1e-12 if precision == 8 else 1e-6
    # two calls in a row: the full scratch size, then a smaller set on new data
    for nj in (MAX_JOBS, 37):
        jp, ref = _job_set(ctx, rng, nj, dtype)
        out_ctx, out_static = ctx.malloc(8 * nj), ctx.malloc(8 * nj)
        check(lib.lfts_memset_async(ctx.h, out_static, 0xFF, 8 * nj))
        check(lib.lfts_dots(ctx.h, jp, nj, out_ctx))
        check(lib.lfts_dots_static(precision, ctx.M, jp, nj, out_static, stream))
        ctx.sync()
        a = ctx.d2h(out_ctx, (nj,), np.float64)
        b = ctx.d2h(out_static, (nj,), np.float64)
        assert np.max(np.abs(b - a) / np.abs(a)) < 1e-12
        assert np.max(np.abs(b - ref) / np.abs(ref)) < tol
    ctx.close()


def test_dots_static_rejects_oversize_and_bad_arguments():
    from langevinfts_b200.capi import Context, lib
    L = lib()
    ctx = Context([16, 12, 10], precision=8)
    dummy = ctx.malloc(64)
    assert L.lfts_dots_static(8, ctx.M, dummy, MAX_JOBS + 1, dummy, None) < 0
    assert b"static scratch" in L.lfts_last_error()
    assert L.lfts_dots_static(3, ctx.M, dummy, 1, dummy, None) < 0
    assert L.lfts_dots_static(8, 0, dummy, 1, dummy, None) < 0
    assert L.lfts_dots_static(8, ctx.M, None, 1, dummy, None) < 0
    assert L.lfts_dots_static(8, ctx.M, dummy, 0, dummy, None) == 0
    ctx.close()
