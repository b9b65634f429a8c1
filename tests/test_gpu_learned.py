"""The learned part on the GPU: the row-nnz MLP's CUDA inference and
gradient against the FP64 restatement in oracle/mlp.py, training, and the
learned product (predicted cut, one numeric pass, exact redo of mispredicted
rows) — whose output must stay bit-identical to the oracle whatever the
predictor says."""
import numpy as np
import pytest

from bcl_b200 import gen
from oracle import mlp as M
from oracle import oracle as O

from gpu_util import assert_csr_identical

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _samples(n=3000, seed=0):
    rng = np.random.default_rng(seed)
    X = np.column_stack([rng.uniform(0, 8, n), rng.uniform(0, 16, n), rng.uniform(0, 12, n),
                         rng.uniform(0, 1, n), rng.uniform(0, 1, n)]).astype(np.float32)
    y = (0.7 * X[:, 1] + 0.1 * X[:, 0] + np.sin(3 * X[:, 3])).astype(np.float32)
    return X, y


def test_mlp_forward_matches_fp64():
    import torch
    from bcl_b200.learned import RowNnzPredictor
    X, _ = _samples()
    m = RowNnzPredictor(seed=3)
    got = m.predict(torch.from_numpy(X).cuda()).cpu().numpy()
    want, _ = M.forward(m.params.cpu().numpy(), X)
    np.testing.assert_allclose(got, want, rtol=1e-4, atol=1e-4)


def test_mlp_gradient_matches_fp64():
    """FP32 kernels (per-sample backward, block reductions, atomics) against
    the FP64 gradient: relative L2 error of the whole gradient < 1e-4."""
    import torch
    from bcl_b200.learned import RowNnzPredictor
    X, y = _samples(2000, seed=1)
    m = RowNnzPredictor(seed=4)
    g = m.gradient(torch.from_numpy(X).cuda(), torch.from_numpy(y).cuda()).cpu().numpy()
    loss, want = M.loss_and_grad(m.params.cpu().numpy(), X, y)
    rel = np.linalg.norm(g[:M.NPARAMS] - want) / np.linalg.norm(want)
    print(f"\ngradient relative error vs FP64: {rel:.2e}")
    assert rel < 1e-4
    np.testing.assert_allclose(g[M.NPARAMS] / X.shape[0], loss, rtol=1e-4)


def test_mlp_training_reduces_loss():
    import torch
    from bcl_b200.learned import RowNnzPredictor
    X, y = _samples(4000, seed=2)
    m = RowNnzPredictor(seed=5)
    losses = m.fit(torch.from_numpy(X).cuda(), torch.from_numpy(y).cuda(), steps=300, lr=3e-3)
    assert losses[-1] < 0.1 * losses[0]
    # the trained model's loss agrees with the FP64 evaluation of the same weights
    l64, _ = M.loss_and_grad(m.params.cpu().numpy(), X, y)
    assert l64 < 0.1 * losses[0]


def _small_predictor():
    from bcl_b200.containers import BlockCustom, SPMatrix
    from bcl_b200.learned import RowNnzPredictor, row_samples
    Xs, ys = [], []
    for s in range(6):
        a = gen.rmat(12 + s % 2, seed=500 + s)
        A = SPMatrix.from_csr(a, BlockCustom((1024 * (1 + s % 2), 1024 * (1 + s % 2))))
        X, y = row_samples(A, A)
        Xs.append(X)
        ys.append(y)
    import torch
    m = RowNnzPredictor(seed=6)
    m.fit(torch.cat(Xs), torch.cat(ys), steps=400, lr=3e-3)
    return m


@pytest.fixture(scope="module")
def predictor():
    return _small_predictor()


@pytest.mark.parametrize("which", ["trained", "none", "poor"])
@pytest.mark.parametrize("value_type", ["f32", "i32"])
def test_learned_product_bit_identical(predictor, which, value_type):
    from bcl_b200.containers import BlockCustom, SPMatrix, learned_stats, spgemm_learned
    from bcl_b200.learned import RowNnzPredictor
    if which == "poor":  # predicts ~1 output per row: every heavy item overflows -> exact redo
        p = predictor.params.cpu().numpy().copy()
        p[-1] = -50.0
        p[-65:-1] = 0.0
        pred = RowNnzPredictor(p)
    else:
        pred = predictor if which == "trained" else None
    a = gen.rmat(13, seed=77, value_type=value_type)
    A = SPMatrix.from_csr(a, BlockCustom((2048, 2048)))
    C, plan = spgemm_learned(A, A, predictor=pred, keep_plan=True)
    st = learned_stats(plan)
    plan.close()
    rp, ci, cv = O.gemm_tiled(a, a, 2048, 2048, 2048, mode=value_type)
    assert_csr_identical(C.get(), rp, ci, cv)
    assert st["heavy_rows"] > 0
    if which == "poor":
        assert st["rows_redone"] > 0


def test_learned_gain_over_predictor_free_cut():
    """What the network buys: heavy rows cut and their temporary slots sized
    from predicted counts give fewer items and less temporary space than
    when both come from product counts (the predictor-free upper bound),
    while mispredicting few rows."""
    from bcl_b200.containers import BlockCustom, SPMatrix, learned_stats, spgemm_learned
    # a 27-point stencil squared: 729 products per row for 125 outputs, so
    # the product-count bound is loose and a good prediction pays
    a = gen.stencil27(32)
    A = SPMatrix.from_csr(a, BlockCustom((4096, 4096)))
    from bcl_b200 import learned
    trained = learned.get_default(train_if_missing=False)  # the packaged network
    _, p1 = spgemm_learned(A, A, predictor=trained, keep_plan=True)
    with_net = learned_stats(p1)
    p1.close()
    _, p0 = spgemm_learned(A, A, predictor=None, keep_plan=True)
    without = learned_stats(p0)
    p0.close()
    print(f"\nwith network: {with_net}\nwithout:      {without}")
    assert with_net["heavy_items"] < 0.8 * without["heavy_items"]
    assert with_net["temp_entries"] < 0.7 * without["temp_entries"]
    assert with_net["rows_redone"] <= 0.05 * with_net["heavy_rows"]
