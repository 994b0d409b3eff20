"""Learned saddle-point start (langevinfts_b200.learned): the U-Net respects
the periodic box, an untrained network (zero last layer) leaves the batched
L-FTS trajectory exactly as the plain warm start gives it, training pairs
are the solver's own fields, and training lowers the loss."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_unet_is_shift_equivariant_on_the_periodic_grid():
    import torch
    from langevinfts_b200.learned import UNet3D
    torch.manual_seed(0)
    net = UNet3D(cin=2, cout=1, base=8).cuda().double()
    for p in net.parameters():  # a non-trivial last layer
        torch.nn.init.normal_(p, 0, 0.1)
    x = torch.randn(1, 2, 16, 16, 16, device="cuda", dtype=torch.float64)
    shift = (4, 8, 12)  # multiples of 4: both pooling levels commute with the shift
    with torch.no_grad():
        a = torch.roll(net(x), shift, dims=(2, 3, 4))
        b = net(torch.roll(x, shift, dims=(2, 3, 4)))
    assert float((a - b).abs().max()) < 1e-12 * float(a.abs().max())


def test_untrained_start_reproduces_the_plain_step():
    from langevinfts_b200.learned import LearnedStart, UNet3D
    from langevinfts_b200.lfts import BatchedLFTS
    from tests.test_checkpoint_gpu import params
    sims = [BatchedLFTS(params(), random_seeds=[41, 42]) for _ in range(2)]
    rng = np.random.Generator(np.random.PCG64(5))
    init = [{"A": rng.normal(0, 1, sims[0].M), "B": rng.normal(0, 1, sims[0].M)} for _ in range(2)]
    for s in sims:
        s.start(init)
    start = LearnedStart(UNet3D(base=8).cuda(), 1.0, 1.0)
    for _ in range(2):
        a = sims[0].step()
        b = sims[1].step(start=start)
        assert list(a["iterations"]) == list(b["iterations"])
    assert np.array_equal(sims[0].fields(), sims[1].fields())


def test_generate_pairs_and_training_lowers_the_loss():
    from langevinfts_b200.learned import generate_pairs, train
    from langevinfts_b200.lfts import BatchedLFTS
    from tests.test_checkpoint_gpu import params
    sim = BatchedLFTS(params(), random_seeds=[51, 52, 53, 54])
    rng = np.random.Generator(np.random.PCG64(6))
    sim.start([{"A": rng.normal(0, 1, sim.M), "B": rng.normal(0, 1, sim.M)} for _ in range(sim.R)])
    w_before = sim.fields()
    X, Y, iters = generate_pairs(sim, 3)
    assert X.shape == (12, 3, 16, 16, 16) and Y.shape == (12, 1, 16, 16, 16) and len(iters) == 12
    w_after = sim.fields()
    ri, ii = sim.mpt.aux_fields_real_idx[0], sim.mpt.aux_fields_imag_idx[0]
    # the last step's pairs: inputs (w_- now, w_+ of the step before), target w_+ now
    last = X[-sim.R:], Y[-sim.R:]
    np.testing.assert_allclose(last[0][:, 0].reshape(sim.R, -1), w_after[:, ri].astype(np.float32), rtol=0, atol=0)
    np.testing.assert_allclose(last[1][:, 0].reshape(sim.R, -1), w_after[:, ii].astype(np.float32), rtol=0, atol=0)
    first = X[:sim.R]
    np.testing.assert_allclose(first[:, 1].reshape(sim.R, -1), w_before[:, ii].astype(np.float32), rtol=0, atol=0)
    # third channel: the update's change of w_- (w_- now minus w_- before the step), in FP32
    np.testing.assert_allclose((first[:, 0].astype(np.float64) - first[:, 2]).reshape(sim.R, -1), w_before[:, ri],
                               rtol=0, atol=1e-5)
    np.testing.assert_allclose(last[0][:, 2], last[0][:, 0] - X[-2 * sim.R:-sim.R, 0], rtol=0, atol=1e-5)
    # the network can fit a handful of pairs: 150 AdamW steps on 4 of them
    start, hist = train(X[:4], Y[:4], base=8, seconds=120, epochs=150, batch=4, lr=3e-3)
    assert hist[-1][1] < 0.6 * hist[0][1], hist[:: max(1, len(hist) // 6)]


def gain_params():
    """The benchmark system (f = 0.5, chiN = 17, nbar = 100, N = 90, dt = 0.8,
    tolerance 1e-4) on a 32^3 box of the same grid spacing (3.65)."""
    return {
        "nx": [32, 32, 32], "lx": [3.65, 3.65, 3.65], "chain_model": "continuous", "ds": 1 / 90,
        "segment_lengths": {"A": 1.0, "B": 1.0}, "chi_n": {"A,B": 17.0},
        "distinct_polymers": [{"volume_fraction": 1.0, "blocks": [{"type": "A", "length": 0.5}, {"type": "B", "length": 0.5}]}],
        "langevin": {"dt": 0.8, "nbar": 100}, "saddle": {"max_iter": 100, "tolerance": 1e-4},
        "am": {"max_hist": 20, "start_error": 5e-1, "mix_min": 0.01, "mix_init": 0.01},
    }


def test_trained_start_cuts_saddle_iterations():
    """What the trained network gains: 16 replicas at 32^3, pairs from 12 plain
    steps, 60 s of training on the tensor cores (convolutions forward and
    backward, AdamW kernel), then the same 6 Langevin steps (same state, same
    noise) from the plain warm start and from the network's prediction.  The
    learned start needs at least 10 % fewer saddle-point iterations and every
    step still reaches the 1e-4 tolerance."""
    from langevinfts_b200.learned import ablation, generate_pairs, train
    from langevinfts_b200.lfts import BatchedLFTS
    seeds = list(range(300, 316))
    sim = BatchedLFTS(gain_params(), random_seeds=seeds)
    rng = np.random.Generator(np.random.PCG64(8))
    sim.start([{"A": rng.normal(0, 1, sim.M), "B": rng.normal(0, 1, sim.M)} for _ in seeds])
    for _ in range(3):
        sim.step()
    X, Y, it_pairs = generate_pairs(sim, 12)
    start, hist = train(X, Y, seconds=60.0)
    assert start.net is not None  # inference on the tensor cores
    plain, learned = ablation(sim, [None, start], 6)
    assert plain["failed"] == 0 and learned["failed"] == 0
    assert learned["mean_iterations"] <= 0.9 * plain["mean_iterations"], (plain["mean_iterations"],
                                                                          learned["mean_iterations"], hist[-1])
