"""The learned effective action and the global block moves on the GPU.

* forward S and parameter gradients of the tensor-core network kernels
  against the numpy restatement (oracle/nn_oracle.py, which rounds to bf16 at
  the same points and is itself checked by finite differences in
  tests/test_oracle.py): relative 2e-4 on S, 2e-3 on the gradient norm;
* training on recorded pairs lowers the loss;
* the recorded pairs are the chains' fields and log weights;
* block moves are exact: with local updates off, the change of the log weight
  over a learned sweep equals the sum of the accepted blocks' log ratios, and
  the wrap error stays at rounding level;
* learned and plain sweeps sample the same double occupancy.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HUB = dict(lattice=1, l1=4, l2=4, beta=2.0, dtau=0.1, rhub=4.0, nflr=2, kinetic=0, update=1, hs=0, nwrap=10,
           nublock=8)


@pytest.fixture(scope="module")
def sb():
    import sunhubbardmy_b200 as sb
    return sb


def rand_theta(nn_oracle, seed, scale=1.0):
    rng = np.random.default_rng(seed)
    th = np.zeros(nn_oracle.NP)
    C = nn_oracle.C
    th[:27 * C] = rng.uniform(-1, 1, 27 * C) * np.sqrt(3 / 27) * scale
    k = 27 * C
    th[k:k + C] = rng.uniform(-0.2, 0.2, C); k += C
    th[k:k + 27 * C * C] = rng.uniform(-1, 1, 27 * C * C) * np.sqrt(3 / 864) * scale; k += 27 * C * C
    th[k:k + C] = rng.uniform(-0.2, 0.2, C); k += C
    th[k:k + C] = rng.uniform(-1, 1, C) * np.sqrt(3 / 32); k += C
    th[k] = 0.25
    return th.astype(np.float32)


@pytest.mark.parametrize("shape", [(8, 4), (12, 20), (6, 5)])
def test_nn_forward_and_gradient_match_oracle(sb, shape):
    from oracle import nn_oracle as no
    from sunhubbardmy_b200.learned import EffectiveAction
    Lt, L = shape
    th = rand_theta(no, 3)
    nn = EffectiveAction(Lt, L, max_batch=4)
    nn.set_params(th)
    rng = np.random.default_rng(1)
    fields = rng.choice(np.array([-1, 1], np.int8), size=(3, Lt, L, L))
    S = nn.forward(fields)
    So = np.array([no.forward(th.astype(np.float64), f) for f in fields])
    assert np.max(np.abs(S - So)) < 2e-4 * np.max(np.abs(So))
    r = np.array([0.5, -1.25, 0.75])
    S2, g = nn.gradient(fields, r)
    So2, go = no.gradient(th.astype(np.float64), fields, r)
    assert np.allclose(S2, So, rtol=0, atol=2e-4 * np.max(np.abs(So)))
    assert np.linalg.norm(g - go) < 2e-3 * np.linalg.norm(go)
    # per block of parameters as well (W1, b1, W2, b2, w3, b3)
    k = 0
    for size in (27 * 32, 32, 27 * 32 * 32, 32, 32, 1):
        a, b = g[k:k + size], go[k:k + size]
        assert np.linalg.norm(a - b) <= 3e-3 * np.linalg.norm(b) + 1e-6, k
        k += size


def test_nn_training_reduces_loss(sb):
    """Fit a randomly initialised network to a teacher network's values."""
    from oracle import nn_oracle as no
    from sunhubbardmy_b200.learned import EffectiveAction
    Lt, L = 8, 4
    teacher = rand_theta(no, 11, scale=1.5)
    rng = np.random.default_rng(2)
    fields = rng.choice(np.array([-1, 1], np.int8), size=(64, Lt, L, L))
    y = np.array([no.forward(teacher.astype(np.float64), f, emulate_bf16=False) for f in fields])
    nn = EffectiveAction(Lt, L, max_batch=32, seed=5)
    losses = [nn.train_step(fields[i % 2 * 32:(i % 2 + 1) * 32], y[i % 2 * 32:(i % 2 + 1) * 32], lr=3e-3)
              for i in range(60)]
    assert np.mean(losses[-10:]) < 0.5 * np.mean(losses[:5])


def test_recorded_pairs_are_fields_and_weights(sb):
    p = sb.DqmcParams.make(**HUB)
    g = sb.Dqmc(p, n_chains=3)
    g.sweep_start()
    g.record(1000)
    g.sweeps(1, False)
    n = g.record_count()
    assert n == 3 * 2 * p.nst
    f, v = g.record_get(n - 1)            # the last stabilisation of chain 2
    assert np.array_equal(f.reshape(p.ltrot, -1), 2 * g.conf(2) - 3)
    assert abs(v - p.nflr * g.diag(2)["logweight"].real) < 1e-9 * max(1.0, abs(v))
    g.record(0)


def test_record_with_new_capacity_after_stop(sb):
    """record(a), sweeps, record(0), record(b != a), sweeps: the captured sweep
    must write into the new buffers, which then hold the new pairs."""
    p = sb.DqmcParams.make(**HUB)
    g = sb.Dqmc(p, n_chains=2)
    g.sweep_start()
    g.record(100)
    g.sweeps(1, False)
    assert g.record_count() == 2 * 2 * p.nst
    g.record(0)
    g.record(300)
    assert g.record_count() == 0
    g.sweeps(1, False)
    n = g.record_count()
    assert n == 2 * 2 * p.nst
    f, v = g.record_get(n - 1)
    assert np.array_equal(f.reshape(p.ltrot, -1), 2 * g.conf(1) - 3)
    assert abs(v - p.nflr * g.diag(1)["logweight"].real) < 1e-9 * max(1.0, abs(v))
    g.record(0)


def test_block_moves_are_exact(sb):
    """Local updates off: every change of the field comes from accepted
    blocks, so nflr * (Re log W_end - Re log W_start) must equal the sum of
    the accepted blocks' Re log R (a zero network passes every proposal to
    the exact second stage)."""
    from sunhubbardmy_b200.learned import EffectiveAction
    p = sb.DqmcParams.make(**HUB)
    g = sb.Dqmc(p, n_chains=8)
    nn = EffectiveAction(p.ltrot, p.l1, max_batch=16)
    nn.set_params(np.zeros(nn.nparams, np.float32))
    g.sweep_start()
    w0 = np.array([g.diag(c)["logweight"].real for c in range(8)])
    g.reset_diag()
    g.sweeps_learned(nn, 3, lmeasure=False, seed=77, lupdate=False)
    for c in range(8):
        d = g.diag(c)
        assert d["blk_proposed"] == d["blk_stage1"] > 0
        assert d["max_wrap_error"] < 1e-8
        w1 = d["logweight"].real
        assert abs(p.nflr * (w1 - w0[c]) - d["blk_sum_logratio"]) < 1e-7 * max(1.0, abs(w1))
    assert sum(g.diag(c)["blk_accepted"] for c in range(8)) > 0


def test_learned_and_plain_sample_the_same_double_occupancy(sb):
    from sunhubbardmy_b200.learned import EffectiveAction
    from sunhubbardmy_b200.stats import double_occupancy
    kw = dict(HUB, beta=1.0, rhub=4.0)
    p = sb.DqmcParams.make(**kw)
    nch = 32
    Ns = np.full(nch, p.ndim, float)
    res = {}
    for mode in ("plain", "learned"):
        g = sb.Dqmc(p, n_chains=nch, seeds=[sb.test_seed(c + (0 if mode == "plain" else 1000)) for c in range(nch)])
        g.sweep_start()
        nn = EffectiveAction(p.ltrot, p.l1, max_batch=2 * nch)
        nn.set_params(np.zeros(nn.nparams, np.float32))
        series = []
        for s in range(30):
            g.obser_init()
            if mode == "plain":
                g.sweeps(1, True)
            else:
                g.sweeps_learned(nn, 1, lmeasure=True)
            if s >= 5:
                series.append(double_occupancy(g.energy_all(), Ns))
        x = np.array(series)              # [sweep, chain]
        m = x.mean(axis=0)                # per-chain means: independent
        res[mode] = (m.mean(), m.std(ddof=1) / np.sqrt(nch))
    (a, ea), (b, eb) = res["plain"], res["learned"]
    assert abs(a - b) < 5 * np.hypot(ea, eb) + 1e-12


def test_training_on_recorded_pairs_learns_the_weight(sb):
    """Training on pairs recorded from the plain chains (slot-aligned targets)
    lowers the held-out residual of -log|W| below its variance."""
    from sunhubbardmy_b200.learned import EffectiveAction, collect, train
    kw = dict(HUB, beta=4.0, rhub=6.0)
    p = sb.DqmcParams.make(**kw)
    g = sb.Dqmc(p, n_chains=32)
    g.sweep_start()
    g.sweeps(3, False)
    y = collect(g, 20, 4096)
    n = len(y)
    rng = np.random.default_rng(0)
    perm = rng.permutation(n)
    val, tr = perm[:256], perm[256:]
    vf = np.stack([g.record_get(int(i))[0] for i in val])
    nn = EffectiveAction(p.ltrot, p.l1, max_batch=32, seed=2)
    train(nn, g, y[tr], 600, batch=32, lr=3e-3, seed=1, slots=tr)
    S = np.concatenate([nn.forward(vf[i:i + 32]) for i in range(0, len(vf), 32)])
    r2 = 1 - np.var(S - y[val]) / np.var(y[val])
    assert r2 > 0.2, r2


def test_training_on_record_differences_lowers_its_loss(sb):
    """dqmc_nn_train_recorded_pairs: fitting the change of -log|W| between a
    chain's consecutive records lowers the pair loss."""
    from sunhubbardmy_b200.learned import EffectiveAction, collect, train
    kw = dict(HUB, beta=2.0, rhub=6.0)
    p = sb.DqmcParams.make(**kw)
    nch = 16
    g = sb.Dqmc(p, n_chains=nch)
    g.sweep_start()
    g.sweeps(2, False)
    y = collect(g, 8, 4096)
    nn = EffectiveAction(p.ltrot, p.l1, max_batch=32, seed=3)
    losses = train(nn, g, y, 400, batch=32, lr=1e-3, seed=2, pair_lag=nch, diff_every=1)
    assert np.mean(losses[-40:]) < 0.7 * np.mean(losses[:40])
