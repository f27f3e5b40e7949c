"""The picker MLP's GPU kernels against the CPU reference (oracle/mlp_ref.py):
forward outputs and gradients of the masked MSE, with bf16 rounding at the
same points; and a short training run that lowers the loss."""
import numpy as np
import pytest
import torch

import bine_trees_fugaku_b200 as bine
from oracle import mlp_ref

pytestmark = pytest.mark.gpu


def test_forward_and_gradients_match_cpu_reference():
    m = bine.MLP(32, 256, 64, 256, seed=1)
    rng = np.random.default_rng(1)
    n = 128
    x = rng.standard_normal((n, 32)).astype(np.float32)
    t = rng.standard_normal((n, 64)).astype(np.float32)
    mask = (rng.random((n, 64)) < 0.6).astype(np.float32)
    p = m.get_params()
    lay = m.layout()
    xd, td, md = (torch.from_numpy(a).cuda() for a in (x, t, mask))
    y = m.forward(xd).cpu().numpy()
    pres, _ = mlp_ref.forward(p, lay, x)
    ref_y = pres[-1]
    assert np.abs(y - ref_y).max() <= 2e-2 * np.abs(ref_y).max()
    g, loss = m.gradients(xd, td, md)
    ref_loss, ref_g = mlp_ref.loss_and_grads(p, lay, x, t, mask)
    assert abs(loss - ref_loss) <= 1e-3 * ref_loss
    for w, b, nout, nin in lay:
        for lo, hi in ((w, w + nout * nin), (b, b + nout)):
            a, r = g[lo:hi].astype(np.float64), ref_g[lo:hi]
            rel = np.linalg.norm(a - r) / max(1e-30, np.linalg.norm(r))
            cos = float(a @ r / max(1e-30, np.linalg.norm(a) * np.linalg.norm(r)))
            assert rel < 2e-2 and cos > 0.9995, (lo, rel, cos)
    m.close()


def test_training_lowers_the_loss():
    m = bine.MLP(16, 256, 16, 256, seed=2)
    rng = np.random.default_rng(2)
    x = rng.standard_normal((256, 16)).astype(np.float32)
    t = np.tanh(x @ rng.standard_normal((16, 16))).astype(np.float32)
    mask = np.ones_like(t)
    xd, td, md = (torch.from_numpy(a).cuda() for a in (x, t, mask))
    first = m.train_step(xd, td, md, 1e-3)
    for _ in range(300):
        last = m.train_step(xd, td, md, 1e-3)
    assert last < 0.2 * first
    m.close()


@pytest.mark.parametrize("nmodels,din,dout,n", [(5, 16, 144, 16), (1, 32, 64, 48), (8, 16, 256, 32), (3, 256, 16, 16)])
def test_fused_ensemble_forward_matches_the_reference_and_the_layered_path(nmodels, din, dout, n):
    """bine_mlp_ensemble_forward (one launch for every model and layer)
    against the CPU reference's mean over the models, and against the
    layered per-model path: the same bf16 rounding points, fp32 sums in
    another order."""
    rng = np.random.default_rng(nmodels * 100 + din)
    models = [bine.MLP(din, 256, dout, 64, seed=s) for s in range(nmodels)]
    for m in models:  # nonzero biases exercise the fused epilogue
        p = m.get_params()
        for w, b, nout, nin in m.layout():
            p[b:b + nout] = rng.standard_normal(nout).astype(np.float32) * 0.1
        m.set_params(p)
    x = rng.standard_normal((n, din)).astype(np.float32)
    xd = torch.from_numpy(x).cuda()
    ens = bine.Ensemble(models)
    y = ens.forward(xd).cpu().numpy()
    ref = np.mean([mlp_ref.forward(m.get_params(), m.layout(), x)[0][-1] for m in models], axis=0)
    assert np.abs(y - ref).max() <= 2e-2 * np.abs(ref).max()
    layered = np.mean([m.forward(xd).cpu().numpy() for m in models], axis=0)
    assert np.abs(y - layered).max() <= 2e-2 * np.abs(layered).max()
    # Deterministic: the models' outputs are summed in model order.
    assert np.array_equal(ens.forward(xd).cpu().numpy(), y)
    ens.close()
    for m in models:
        m.close()
