"""Device-resident SCFT (langevinfts_b200.scft.SCFT) against the reference
driver's iteration (examples/scft/scft.py:617-736) written out on the host
through the langevinfts API: the error level of every iteration, the box and
the final fields agree."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

NX, LX0, F, CHIN = [16, 16, 16], [3.6, 3.6, 3.6], 0.36, 20.0


def params(optimizer, box, iters):
    return {
        "nx": NX, "lx": LX0, "chain_model": "continuous", "ds": 0.01,
        "segment_lengths": {"A": 1.0, "B": 1.0}, "chi_n": {"A,B": CHIN},
        "distinct_polymers": [{"volume_fraction": 1.0, "blocks": [{"type": "A", "length": F}, {"type": "B", "length": 1 - F}]}],
        "box_is_altering": box, "scale_stress": 0.1, "optimizer": optimizer, "max_iter": iters, "tolerance": 0.0,
    }


def initial_fields():
    M = int(np.prod(NX))
    x = np.arange(NX[0]) * 2 * np.pi / NX[0]
    X, Y, Z = np.meshgrid(x, x, x, indexing="ij")
    g = (np.sin(X) * np.cos(Y) + np.sin(Y) * np.cos(Z) + np.sin(Z) * np.cos(X)).reshape(-1)
    rng = np.random.Generator(np.random.PCG64(2))
    return {"A": CHIN * g + 0.1 * rng.normal(0, 1, M), "B": -CHIN * g + 0.1 * rng.normal(0, 1, M)}


def host_loop(p, iters):
    """scft.py:617-736 with the solver on the GPU and everything else in numpy."""
    from langevinfts_b200.scft import SCFT
    ref = SCFT(p)  # for the factory, box, solver objects and matrices only
    f, cb, mpt = ref.factory, ref.cb, ref.mpt
    solver = f.create_pseudospectral_solver(cb, ref.molecules, ref.analyzer)
    M, S = cb.get_n_grid(), 2
    dv = cb.get_volume() / M
    box = p["box_is_altering"]
    opt = p["optimizer"]
    n_var = S * M + (3 if box else 0)
    if opt["name"] == "am":
        am = f.create_anderson_mixing(n_var, opt["max_hist"], opt["start_error"], opt["mix_min"], opt["mix_init"])
    else:
        m, v, count = np.zeros(n_var), np.zeros(n_var), 1
    init = initial_fields()
    w = np.array([init["A"], init["B"]])
    w -= w.mean(axis=1, keepdims=True)
    err, errs = 1e20, []
    for _ in range(iters):
        solver.compute_statistics({"A": w[0], "B": w[1]})
        phi = np.array([solver.get_total_concentration(t) for t in "AB"])
        wd = mpt.matrix_chi @ phi - mpt.matrix_p @ w
        wd -= wd.mean(axis=1, keepdims=True)
        old, err = err, np.sqrt(dv * np.sum(wd ** 2) / (1.0 + dv * np.sum(w ** 2)))
        if box:
            solver.compute_stress()
            st = np.array(solver.get_stress())
            err += np.sqrt(np.sum(st ** 2))
            cur = np.concatenate([w.reshape(-1), cb.get_lx()])
            dif = np.concatenate([wd.reshape(-1), -0.1 * st])
        else:
            cur, dif = w.reshape(-1), wd.reshape(-1)
        errs.append(err)
        if opt["name"] == "am":
            new = am.calculate_new_fields(cur, dif, old, err)
        else:
            lr = opt["lr"] * opt["gamma"] ** (count - 1)
            m = 0.9 * m + (1.0 - 0.9) * dif
            v = 0.999 * v + (1.0 - 0.999) * dif ** 2
            new = cur + lr * (m / (1.0 - 0.9 ** count)) / (np.sqrt(v / (1.0 - 0.999 ** count)) + 1e-8)
            count += 1
        if box:
            lx0 = np.array(cb.get_lx())
            cb.set_lx(list((1 + np.clip((new[-3:] - lx0) / lx0, -0.1, 0.1)) * lx0))
            solver.update_laplacian_operator()
        w = new[:S * M].reshape(S, M).copy()
        w -= w.mean(axis=1, keepdims=True)
    return np.array(errs), w, np.array(cb.get_lx())


@pytest.mark.parametrize("optimizer,box", [
    ({"name": "am", "max_hist": 20, "start_error": 1e-1, "mix_min": 0.1, "mix_init": 0.1}, True),
    ({"name": "adam", "lr": 1e-1, "gamma": 0.9993}, False),
])
def test_device_scft_follows_reference_iteration(optimizer, box):
    from langevinfts_b200.scft import SCFT
    iters = 12
    p = params(optimizer, box, iters)
    errs_h, w_h, lx_h = host_loop(p, iters)
    sim = SCFT(p)
    st = sim.run(initial_fields())
    errs_d = np.array([e for e, _ in st["history"]])
    assert len(errs_d) == iters
    np.testing.assert_allclose(errs_d, errs_h, rtol=1e-9)
    # both loops updated the fields (and box) after their last evaluation
    assert np.isfinite(st["energy"]) and np.isfinite(st["mass_error"])
    assert np.max(np.abs(sim.w - w_h)) <= 1e-8 * np.max(np.abs(w_h))
    np.testing.assert_allclose(sim.cb.get_lx(), lx_h, rtol=1e-10)
    if box:
        assert np.max(np.abs(lx_h - LX0)) > 1e-6  # the box moved
