"""The learned cost model: GPU gradients against a float64 numpy oracle,
training, save/load, and that it never changes a join's pair set."""
import numpy as np
import pytest

import new_fgssjoin_b200 as F
from new_fgssjoin_b200 import datagen
from oracle import oracle as O

pytestmark = pytest.mark.gpu

NF, NH, NO = 8, 32, 2
IN_SCALE, OUT_SCALE = 0.125, 8.0


def _unpack(p):
    p = p.astype(np.float64)
    i = 0
    W1 = p[i:i + NH * NF].reshape(NH, NF); i += NH * NF
    b1 = p[i:i + NH]; i += NH
    W2 = p[i:i + NO * NH].reshape(NO, NH); i += NO * NH
    b2 = p[i:i + NO]
    return W1, b1, W2, b2


def _np_loss_grad(feat, target, p):
    """Float64 reference: mean over rows of the Poisson loss sum_j exp(r_j) - y_j r_j,
    with log-rates r = 8 * output clamped to [-30, 30] (zero gradient outside)."""
    W1, b1, W2, b2 = _unpack(p)
    x = feat.astype(np.float64) * IN_SCALE
    y = target.astype(np.float64)
    hp = x @ W1.T + b1
    h = np.maximum(hp, 0)
    o = h @ W2.T + b2
    n = x.shape[0]
    r = o * OUT_SCALE
    rc = np.clip(r, -30.0, 30.0)
    e = np.exp(rc)
    loss = (e - y * rc).sum() / n
    dO = np.where((r > -30.0) & (r < 30.0), (e - y) * OUT_SCALE, 0.0) / n
    gW2 = dO.T @ h
    gb2 = dO.sum(0)
    dh = (dO @ W2) * (hp > 0)
    gW1 = dh.T @ x
    gb1 = dh.sum(0)
    return loss, np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2])


def test_num_params():
    assert F.load_library().fgss_model_num_params() == NH * NF + NH + NO * NH + NO


@pytest.mark.parametrize("n", [1, 37, 5000])
def test_gradients_match_float64_oracle(ctx, n):
    rng = np.random.default_rng(n)
    feat = rng.uniform(0, 12, (n, NF)).astype(np.float32)
    target = np.floor(rng.exponential(20.0, (n, NO))).astype(np.float32)  # counts
    params = (rng.standard_normal(NH * NF + NH + NO * NH + NO) * 0.1).astype(np.float32)
    g, loss = ctx.model_grad(feat, target, params)
    rl, rg = _np_loss_grad(feat, target, params)
    assert abs(loss - rl) <= 1e-4 * max(1.0, abs(rl))
    np.testing.assert_allclose(g, rg, rtol=2e-3, atol=2e-5 * max(1.0, np.abs(rg).max()))


@pytest.fixture(scope="module")
def titles(ctx):
    return ctx.tokenize(datagen.titles(8000, seed=41), **datagen.TITLE_TOK)


def test_training_reduces_loss_and_roundtrips(ctx, titles, tmp_path):
    ts = [0.6, 0.8]
    l_short = ctx.model_train([titles, titles], ts, epochs=5, lr=0.01, seed=3)
    l_long = ctx.model_train([titles, titles], ts, epochs=300, lr=0.01, seed=3)
    assert l_long < l_short
    p = tmp_path / "m.bin"
    ctx.model_save(str(p))
    ctx.model_load(str(p))
    raw = bytearray(p.read_bytes())
    raw[20:24] = np.array([np.nan], np.float32).tobytes()  # corrupt one weight: rejected, not used
    (tmp_path / "bad.bin").write_bytes(bytes(raw))
    with pytest.raises(F.FgssError) as e:
        ctx.model_load(str(tmp_path / "bad.bin"))
    assert e.value.status == 4
    with pytest.raises(F.FgssError):
        ctx.model_load(str(tmp_path / "missing.bin"))


@pytest.mark.parametrize("t", [0.5, 0.7, 0.9])
def test_model_never_changes_the_pairs(ctx, titles, t):
    ctx.model_train([titles], [t], epochs=100, lr=0.01, seed=5)
    a = ctx.selfjoin(titles, t, method="batched", use_model=True)
    b = ctx.selfjoin(titles, t, method="plain")
    ref, st = O.join(titles.pos, titles.len, titles.tokens, titles.n_terms, t)
    for got in (a, b):
        assert np.array_equal(got.q, ref["q"]) and np.array_equal(got.s, ref["s"])
        assert got.stats["candidates"] == st["candidates"]


def test_undersized_result_buffer_reruns_exactly(ctx, titles):
    """A presized result buffer that is too small is detected on the device and
    the join re-runs with the exact size; the pair set is unchanged."""
    ref, st = O.join(titles.pos, titles.len, titles.tokens, titles.n_terms, 0.5)
    assert len(ref) > 10
    got = ctx.selfjoin(titles, 0.5, method="batched", result_capacity=3)
    assert got.stats["overflow_retries"] == 1
    assert np.array_equal(got.q, ref["q"]) and np.array_equal(got.s, ref["s"])
    assert got.stats["candidates"] == st["candidates"]


def _dup_titles(n_distinct, copies, seed):
    """Title records, each line repeated `copies` times in a row."""
    lines = datagen.titles(n_distinct, seed=seed).split(b"\n")[:-1]
    return b"\n".join(x for x in lines for _ in range(copies)) + b"\n"


def test_trained_model_gains_one_filter_pass(ctx):
    """What the trained network gains over the method without it: on records with
    many duplicates the result pairs outnumber the records, so the model-free
    result buffer (records + 4096 slots) overflows and the join runs its filter
    a second time with the exact size; with the trained model the presized
    buffer fits and the filter runs once.  The pair set is the same."""
    train = ctx.tokenize(_dup_titles(3000, 6, 51), **datagen.TITLE_TOK)
    test = ctx.tokenize(_dup_titles(3000, 6, 52), **datagen.TITLE_TOK)
    ref, st = O.join(test.pos, test.len, test.tokens, test.n_terms, 0.8)
    assert st["results"] > test.n_sets + 4096
    outs = {}
    for learned in (False, True):
        with F.Context(device=0) as fresh:  # nothing remembered from earlier calls
            if learned:
                fresh.model_train([train], [0.8], epochs=300, lr=0.01, seed=1)
            outs[learned] = fresh.selfjoin(test, 0.8, method="batched", use_model=learned)
    assert outs[False].stats["overflow_retries"] == 1
    assert outs[True].stats["overflow_retries"] == 0
    pred = outs[True].stats["predicted_results"]
    assert 0.5 * st["results"] <= pred <= 2.0 * st["results"], (pred, st["results"])
    for got in outs.values():
        assert np.array_equal(got.q, ref["q"]) and np.array_equal(got.s, ref["s"])
        assert got.stats["candidates"] == st["candidates"]
