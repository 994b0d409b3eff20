"""Engine kernels through the C ABI (liblfts_b200.so) against the CPU oracle.

FP64 tolerance: relative 1e-12 per step (FFT round-off), FP32: 2e-5.
"""
import ctypes as C

import numpy as np
import pytest

from oracle import lfts_oracle as orc

pytestmark = pytest.mark.gpu

GRIDS = [((5, 4, 3), (4.0, 3.0, 2.0)), ((8, 8, 8), (3.0, 3.0, 3.0)), ((32, 32, 32), (4.0, 4.0, 4.0)),
         ((23, 27, 25), (3.2, 3.3, 3.4)), ((64,), (5.0,)), ((16, 12), (3.0, 2.5)), ((48, 48, 48), (5.0, 5.0, 5.0)),
         ((31, 49, 23), (4.0, 4.5, 3.5)), ((16, 16, 16), (3.0, 3.0, 3.0)), ((64, 64, 64), (7.3, 7.3, 7.3)),
         ((96, 96, 96), (8.0, 8.0, 8.0))]
GRID_IDS = ["x".join(map(str, nx)) for nx, _ in GRIDS]


def _ctx(nx, prec=8):
    from langevinfts_b200.capi import Context
    return Context(nx, precision=prec)


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def _tables(ctx, nx, lx, b2, ds, dt):
    from langevinfts_b200.capi import check
    Mc = ctx.Mc
    bond = ctx.malloc(Mc * dt.itemsize)
    bondh = ctx.malloc(Mc * dt.itemsize)
    lxa = (C.c_double * len(lx))(*lx)
    check(ctx.lib.lfts_bond_tables(ctx.h, b2, ds, lxa, bond, bondh))
    return bond, bondh


def _jobs(ctx, jobs):
    from langevinfts_b200.capi import StepJob
    arr = (StepJob * len(jobs))(*jobs)
    p = ctx.malloc(C.sizeof(arr))
    ctx.h2d(p, np.frombuffer(arr, dtype=np.uint8))
    return p


@pytest.mark.parametrize("nx,lx", GRIDS, ids=GRID_IDS)
@pytest.mark.parametrize("prec", [8, 4])
def test_step_continuous(nx, lx, prec, autotune=False):
    from langevinfts_b200.capi import StepJob, check
    dt = np.dtype(np.float64 if prec == 8 else np.float32)
    ctx = _ctx(nx, prec)
    if autotune:
        report = C.create_string_buffer(512)
        check(ctx.lib.lfts_autotune(ctx.h, 4, 3, report, 512))
        text = report.value.decode()
        assert "generic" in text and " -> " in text, text
    M = ctx.M
    rng = np.random.default_rng(7)
    ds, b2, nsteps, njobs = 0.01, 1.3, 4, 3
    g = orc.Grid(nx, lx)
    w = [rng.normal(0, 2.0, M) for _ in range(njobs)]
    q0 = [1.0 + 0.3 * rng.random(M) for _ in range(njobs)]
    bond, bondh = _tables(ctx, nx, lx, b2, ds, dt)
    jobs = []
    for j in range(njobs):
        wd = ctx.upload(w[j])
        fac = ctx.malloc(M * dt.itemsize)
        check(ctx.lib.lfts_field_factors(ctx.h, wd, -ds / 4, fac))
        q = ctx.malloc((nsteps + 1) * M * dt.itemsize)
        ctx.h2d(q, q0[j].astype(dt))
        spec = ctx.malloc(2 * ctx.Mc * 2 * dt.itemsize)
        jobs.append(StepJob(q, M, q + M * dt.itemsize, M, fac, bond, bondh, spec))
    jp = _jobs(ctx, jobs)
    for s in range(nsteps):
        check(ctx.lib.lfts_step_continuous(ctx.h, jp, njobs, s))
    ctx.sync()
    bo = orc.boltz_bond(nx, lx, b2, ds)
    bh = orc.boltz_bond(nx, lx, b2 / 2, ds)
    for j in range(njobs):
        got = ctx.d2h(jobs[j].in_, (nsteps + 1, M), dt)
        ref = q0[j].copy()
        e, eh = np.exp(-w[j] * ds / 2), np.exp(-w[j] * ds / 4)
        for s in range(nsteps):
            ref = orc.step_continuous(g, ref, e, eh, bo, bh)
            tol = 1e-12 if prec == 8 else 2e-5
            assert _rel(got[s + 1].astype(float), ref) < tol * (s + 1), (j, s, _rel(got[s + 1], ref))
    ctx.close()


@pytest.mark.parametrize("nx,lx", [GRIDS[9], GRIDS[10], GRIDS[2], GRIDS[3]], ids=["64x64x64", "96x96x96", "32x32x32", "23x27x25"])
@pytest.mark.parametrize("prec", [8, 4])
def test_step_after_autotune(nx, lx, prec):
    """lfts_autotune times every step implementation the grid has (register,
    cubic, generic) and keeps one; the step still matches the oracle."""
    test_step_continuous(nx, lx, prec, autotune=True)


MASK_GRIDS = [((64, 64, 64), (7.3, 7.3, 7.3)), ((96, 96, 96), (8.0, 8.0, 8.0)), ((32, 32, 32), (4.0, 4.0, 4.0)),
              ((23, 27, 25), (3.2, 3.3, 3.4))]


@pytest.mark.parametrize("nx,lx", MASK_GRIDS, ids=["x".join(map(str, nx)) for nx, _ in MASK_GRIDS])
@pytest.mark.parametrize("prec", [8, 4])
def test_step_active_mask(nx, lx, prec):
    """Jobs of inactive replicas leave their output untouched; the others step
    as usual (the batched saddle loop stops converged replicas this way)."""
    from langevinfts_b200.capi import StepJob, check
    dt = np.dtype(np.float64 if prec == 8 else np.float32)
    ctx = _ctx(nx, prec)
    M = ctx.M
    rng = np.random.default_rng(11)
    ds, b2, R = 0.01, 1.0, 3
    g = orc.Grid(nx, lx)
    bond, bondh = _tables(ctx, nx, lx, b2, ds, dt)
    active = np.array([1, 0, 1], dtype=np.int32)
    act = ctx.upload(active)
    jobs, w, q0 = [], [], []
    for r in range(R):
        w.append(rng.normal(0, 1.0, M))
        q0.append(1.0 + 0.3 * rng.random(M))
        wd = ctx.upload(w[r])
        fac = ctx.malloc(M * dt.itemsize)
        check(ctx.lib.lfts_field_factors(ctx.h, wd, -ds / 4, fac))
        q = ctx.malloc(2 * M * dt.itemsize)
        ctx.h2d(q, np.concatenate([q0[r], np.full(M, -7.0)]).astype(dt))  # slice 1 holds a sentinel
        spec = ctx.malloc(2 * ctx.Mc * 2 * dt.itemsize)
        jobs.append(StepJob(q, M, q + M * dt.itemsize, M, fac, bond, bondh, spec, act, r, 0))
    jp = _jobs(ctx, jobs)
    check(ctx.lib.lfts_step_continuous(ctx.h, jp, R, 0))
    ctx.sync()
    bo, bh = orc.boltz_bond(nx, lx, b2, ds), orc.boltz_bond(nx, lx, b2 / 2, ds)
    for r in range(R):
        got = ctx.d2h(jobs[r].in_, (2, M), dt)[1].astype(float)
        if active[r]:
            ref = orc.step_continuous(g, q0[r], np.exp(-w[r] * ds / 2), np.exp(-w[r] * ds / 4), bo, bh)
            assert _rel(got, ref) < (1e-12 if prec == 8 else 2e-5)
        else:
            assert np.all(got == -7.0)
    ctx.close()


@pytest.mark.parametrize("nx,lx,prec", [(n, l, 8) for n, l in GRIDS[:4] + GRIDS[5:6] + GRIDS[9:10]] +
                         [(n, l, 4) for n, l in GRIDS[2:3] + GRIDS[9:10]])
@pytest.mark.parametrize("half,with_fac", [(0, 1), (1, 0), (1, 1)])
def test_step_discrete(nx, lx, prec, half, with_fac):
    from langevinfts_b200.capi import StepJob, check
    dt = np.dtype(np.float64 if prec == 8 else np.float32)
    ctx = _ctx(nx, prec)
    M = ctx.M
    rng = np.random.default_rng(3)
    ds, b2 = 1 / 20, 0.8
    g = orc.Grid(nx, lx)
    w = rng.normal(0, 1.0, M)
    q0 = 1.0 + 0.3 * rng.random(M)
    bond, bondh = _tables(ctx, nx, lx, b2, ds, dt)
    wd = ctx.upload(w)
    fac = ctx.malloc(M * dt.itemsize)
    check(ctx.lib.lfts_field_factors(ctx.h, wd, -ds, fac))
    q = ctx.upload(q0.astype(dt))
    out = ctx.malloc(M * dt.itemsize)
    spec = ctx.malloc(2 * ctx.Mc * 2 * dt.itemsize)
    jp = _jobs(ctx, [StepJob(q, 0, out, 0, fac, bond, bondh, spec)])
    check(ctx.lib.lfts_step_discrete(ctx.h, jp, 1, 0, half, with_fac))
    got = ctx.d2h(out, (M,), dt).astype(float)
    b = orc.boltz_bond(nx, lx, b2 / 2 if half else b2, ds)
    ref = orc.half_bond_step(g, q0, b)
    if with_fac:
        ref = ref * np.exp(-w * ds)
    assert _rel(got, ref) < (1e-12 if prec == 8 else 2e-5)
    ctx.close()


def test_dots_phi_am():
    from langevinfts_b200.capi import DotJob, PhiJob, check
    nx = (16, 12, 10)
    ctx = _ctx(nx)
    M = ctx.M
    rng = np.random.default_rng(5)
    a, b, w = rng.random(M), rng.random(M), 0.5 + rng.random(M)
    pa, pb, pw = ctx.upload(a), ctx.upload(b), ctx.upload(w)
    jobs = (DotJob * 2)(DotJob(pa, pb, None, 0.25), DotJob(pa, pb, pw, 2.0))
    jp = ctx.upload(np.frombuffer(jobs, dtype=np.uint8))
    out = ctx.malloc(16)
    check(ctx.lib.lfts_dots(ctx.h, jp, 2, out))
    got = ctx.d2h(out, (2,), np.float64)
    assert abs(got[0] - 0.25 * np.sum(a * b)) < 1e-12 * abs(got[0])
    assert abs(got[1] - 2.0 * np.sum(a * b / w)) < 1e-12 * abs(got[1])
    # continuous Simpson phi and discrete phi
    NL, NR = 9, 7
    ql, qr = rng.random((NL + 1, M)), rng.random((NR + 2, M))
    pql, pqr = ctx.upload(ql), ctx.upload(qr)
    coef = orc.simpson_coeff(NR)
    pc = ctx.upload(coef)
    phi = ctx.malloc(2 * M * 8)
    pj = (PhiJob * 1)(PhiJob(pql, pqr, None, phi, 1.7, None, NL, NR, 0, 0))
    check(ctx.lib.lfts_phi_blocks(ctx.h, 0, ctx.upload(np.frombuffer(pj, dtype=np.uint8)), 1, pc))
    ref = 1.7 * sum(coef[n] * ql[NL - n] * qr[n] for n in range(NR + 1))
    assert np.max(np.abs(ctx.d2h(phi, (M,), np.float64) - ref)) < 1e-12 * np.max(ref)
    pj = (PhiJob * 1)(PhiJob(pql, pqr, pw, phi + M * 8, 0.3, None, NL, NR, 0, 0))
    check(ctx.lib.lfts_phi_blocks(ctx.h, 1, ctx.upload(np.frombuffer(pj, dtype=np.uint8)), 1, pc))
    ref = 0.3 * sum(ql[NL - n + 1] * qr[n] for n in range(1, NR + 1)) / w
    assert np.max(np.abs(ctx.d2h(phi + M * 8, (M,), np.float64) - ref)) < 1e-12 * np.max(ref)
    # Anderson-mixing dots and update
    nh = 5
    hist = rng.random((nh, M))
    d = rng.random(M)
    ph, pd = ctx.upload(hist), ctx.upload(d)
    dots = ctx.malloc(nh * 8)
    check(ctx.lib.lfts_am_dots(ctx.h, pd, ph, M, nh, M, dots, nh - 1, nh))
    # ring: newest is the last slot, i-th newest is slot nh-1-i
    hist = hist[::-1]
    assert np.allclose(ctx.d2h(dots, (nh,), np.float64), hist @ d, rtol=1e-13)
    wh, dh = rng.random((nh, M)), rng.random((nh, M))
    av = rng.random(nh - 1)
    pwh, pdh, pa2 = ctx.upload(wh), ctx.upload(dh), ctx.upload(av)
    wn = ctx.malloc(M * 8)
    check(ctx.lib.lfts_am_update(ctx.h, wn, pwh, pdh, M, nh - 1, pa2, M, 0, nh))
    # head = 0: the k-th newest history is ring slot (-k) mod nh
    ref = wh[0] + dh[0] + sum(av[i] * (wh[(-(i + 1)) % nh] + dh[(-(i + 1)) % nh] - wh[0] - dh[0]) for i in range(nh - 1))
    assert np.allclose(ctx.d2h(wn, (M,), np.float64), ref, rtol=1e-13, atol=1e-13)
    ctx.close()


@pytest.mark.parametrize("nx,lx", [((8, 6, 10), (3.0, 2.0, 4.0)), ((32, 32, 32), (4.0, 4.0, 4.0)), ((23, 27, 25), (3.2, 3.3, 3.4))])
def test_stress(nx, lx):
    from langevinfts_b200.capi import StressJob, check
    ctx = _ctx(nx)
    M, Mc = ctx.M, ctx.Mc
    rng = np.random.default_rng(11)
    g = orc.Grid(nx, lx)
    nj = 5
    q1, q2 = rng.random((nj, M)), rng.random((nj, M))
    p1, p2 = ctx.upload(q1), ctx.upload(q2)
    basis = ctx.malloc(3 * Mc * 8)
    check(ctx.lib.lfts_fourier_basis(ctx.h, (C.c_double * 3)(*lx), basis))
    bond, bondh = _tables(ctx, nx, lx, 1.4, 0.05, np.dtype(np.float64))
    jobs = (StressJob * nj)(*[StressJob(p1 + j * M * 8, p2 + j * M * 8, bond if j % 2 else None, 0.5 + j) for j in range(nj)])
    jp = ctx.upload(np.frombuffer(jobs, dtype=np.uint8))
    spec = ctx.malloc(2 * 2 * Mc * 16)
    out = ctx.malloc(3 * nj * 8)
    check(ctx.lib.lfts_stress(ctx.h, jp, nj, basis, spec, 2, out))
    got = ctx.d2h(out, (nj, 3), np.float64)
    bas = orc.fourier_basis(nx, lx)
    bo = orc.boltz_bond(nx, lx, 1.4, 0.05)
    for j in range(nj):
        ref = orc.segment_stress(g, q1[j], q2[j], 1.0, bas, bo if j % 2 else None) * (0.5 + j)
        assert np.allclose(got[j], ref, rtol=1e-11, atol=1e-9 * np.max(np.abs(ref))), (j, got[j], ref)
    ctx.close()


@pytest.mark.parametrize("prec", [4, 8])
def test_step_implementations_agree_64cubed(prec):
    """The step implementations of the 64^3 grid agree: the register-resident
    kernels and the compile-time cubic kernels to round-off, 13 jobs with two
    inactive replicas, whose outputs stay untouched; an implementation the grid
    lacks is refused."""
    from langevinfts_b200.capi import StepJob, check
    nx, lx = (64, 64, 64), (7.3, 7.3, 7.3)
    dt = np.dtype(np.float64 if prec == 8 else np.float32)
    ctx = _ctx(nx, prec)
    M = ctx.M
    rng = np.random.default_rng(23)
    ds, b2, nj = 1 / 90, 1.0, 13
    bond, bondh = _tables(ctx, nx, lx, b2, ds, dt)
    active = np.ones(nj, dtype=np.int32)
    active[[3, 10]] = 0
    act = ctx.upload(active)
    jobs, q0 = [], []
    for r in range(nj):
        wd = ctx.upload(rng.normal(0, 1.0, M))
        fac = ctx.malloc(M * dt.itemsize)
        check(ctx.lib.lfts_field_factors(ctx.h, wd, -ds / 4, fac))
        q0.append((1.0 + 0.3 * rng.random(M)).astype(dt))
        q = ctx.malloc(2 * M * dt.itemsize)
        spec = ctx.malloc(2 * ctx.Mc * 2 * dt.itemsize)
        jobs.append(StepJob(q, M, q + M * dt.itemsize, M, fac, bond, bondh, spec, act, r, 0))
    jp = _jobs(ctx, jobs)
    names = ["register-64", "cubic"]
    out = {}
    for name in names:
        check(ctx.lib.lfts_set_step_impl(ctx.h, name.encode()))
        got = C.create_string_buffer(64)
        check(ctx.lib.lfts_step_impl(ctx.h, got, 64))
        assert got.value.decode() == name
        for r in range(nj):
            ctx.h2d(jobs[r].in_, np.concatenate([q0[r], np.full(M, -7.0, dtype=dt)]))
        check(ctx.lib.lfts_step_continuous(ctx.h, jp, nj, 0))
        ctx.sync()
        out[name] = np.array([ctx.d2h(jobs[r].in_, (2, M), dt)[1] for r in range(nj)])
    for r in np.flatnonzero(active == 0):
        assert np.all(out["register-64"][r] == -7.0)
    tol = 1e-12 if prec == 8 else 2e-5
    assert _rel(out["cubic"].astype(float), out["register-64"].astype(float)) < tol
    with pytest.raises(RuntimeError):
        check(ctx.lib.lfts_set_step_impl(ctx.h, b"register-96"))
    ctx.close()
