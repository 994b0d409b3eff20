"""PCG64 streams on the device (lfts_pcg64_raw, lfts_pcg64_normal) against
numpy's PCG64: the raw 64-bit outputs and the advanced states bit for bit,
the normals N(0, sigma^2) by their moments and a Kolmogorov-Smirnov test
(the normal transform is Box-Muller, not numpy's ziggurat), and a batched
L-FTS run with device noise resumed from its checkpoint."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

M64 = (1 << 64) - 1


def states_of(gens):
    st = np.zeros([len(gens), 4], dtype=np.uint64)
    for r, g in enumerate(gens):
        s = g.state["state"]
        st[r] = [s["state"] >> 64, s["state"] & M64, s["inc"] >> 64, s["inc"] & M64]
    return st


def test_raw_stream_matches_numpy_bit_for_bit():
    from langevinfts_b200.capi import Context, check
    ctx = Context([8, 8, 8], precision=8)
    gens = [np.random.PCG64(s) for s in (5, 6, 7)]
    dst = ctx.upload(states_of(gens))
    for n in (1001, 37, 16, 1):  # calls continue the streams
        out = ctx.malloc(len(gens) * n * 8)
        check(ctx.lib.lfts_pcg64_raw(ctx.h, dst, len(gens), n, out))
        got = ctx.d2h(out, (len(gens), n), np.uint64)
        for r, g in enumerate(gens):
            assert np.array_equal(got[r], g.random_raw(n)), (n, r)
        assert np.array_equal(ctx.d2h(dst, (len(gens), 4), np.uint64), states_of(gens))
    ctx.close()


def test_normals_are_standard_normal_and_advance_the_stream():
    from scipy import stats
    from langevinfts_b200.capi import Context, check
    ctx = Context([8, 8, 8], precision=8)
    gens = [np.random.PCG64(s) for s in (11, 12)]
    dst = ctx.upload(states_of(gens))
    n, sigma = 2_000_001, 0.7
    out = ctx.malloc(len(gens) * n * 8)
    check(ctx.lib.lfts_pcg64_normal(ctx.h, dst, len(gens), n, sigma, out))
    z = ctx.d2h(out, (len(gens), n), np.float64) / sigma
    for r in range(len(gens)):
        x = z[r]
        assert abs(x.mean()) < 5 / np.sqrt(n)
        assert abs(x.var() - 1) < 5 * np.sqrt(2 / n)
        assert abs(stats.skew(x)) < 5 * np.sqrt(6 / n) and abs(stats.kurtosis(x)) < 5 * np.sqrt(24 / n)
        assert stats.kstest(x[:200_000], "norm").pvalue > 1e-4
        gens[r].random_raw(n + 1)  # 2 * ceil(n / 2) raw outputs were used
    assert abs(np.corrcoef(z[0][:100_000], z[1][:100_000])[0, 1]) < 5 / np.sqrt(100_000)
    assert np.array_equal(ctx.d2h(dst, (len(gens), 4), np.uint64), states_of(gens))
    ctx.close()


def test_batched_lfts_with_device_noise_resumes_from_checkpoint(tmp_path):
    from langevinfts_b200.lfts import BatchedLFTS
    from tests.test_checkpoint_gpu import params
    a = BatchedLFTS(params(), random_seeds=[31, 32], noise="device")
    rng = np.random.Generator(np.random.PCG64(4))
    a.start([{"A": rng.normal(0, 1, a.M), "B": rng.normal(0, 1, a.M)} for _ in range(a.R)])
    a.step()
    paths = [str(tmp_path / f"dev_r{r}.mat") for r in range(a.R)]
    a.save_simulation_data(paths)
    cont = [a.step() for _ in range(2)]
    assert not any(any(s["failed"]) for s in cont)
    b = BatchedLFTS(params(), random_seeds=[0, 0], noise="device")
    b.continue_run(paths)
    resumed = [b.step() for _ in range(2)]
    for s_a, s_b in zip(cont, resumed):
        assert list(s_a["iterations"]) == list(s_b["iterations"])
    w_a, w_b = a.fields(), b.fields()
    assert np.max(np.abs(w_b - w_a)) <= 1e-9 * np.max(np.abs(w_a))
    # the device streams moved on by the draws of the steps
    assert a.engine.get_noise_streams().tolist() == b.engine.get_noise_streams().tolist()
