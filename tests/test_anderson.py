"""Anderson acceleration of the finishing blocks (glide_b200.physics._Anderson)
on CPU: on a linear contraction x -> A x + b its host-side bookkeeping
reproduces the textbook stacked-history formulation step by step and
converges far faster than the plain iteration.  The two device products
(multi-dot, combination; the library's kernels on the GPU, checked in
tests/test_gpu_krylov.py) are replaced here by plain torch products."""
import numpy as np
import torch


class _TorchProducts:
    def dots(self, rows, w):
        return (rows @ w).numpy()

    def combine(self, rows, coef, out):
        out.copy_(rows.T @ torch.as_tensor(coef, dtype=rows.dtype))


def _reference_aa(g, x0, m, iters):
    """x_{k+1} = G_k - dG gam, gam = argmin |f_k - dF gam| over the last m+1 pairs."""
    Fs, Gs, x, out = [], [], x0.copy(), []
    for _ in range(iters):
        Gx = g(x)
        Fs.append(Gx - x)
        Gs.append(Gx)
        Fs, Gs = Fs[-(m + 1):], Gs[-(m + 1):]
        if len(Fs) > 1:
            dF = np.stack([Fs[k + 1] - Fs[k] for k in range(len(Fs) - 1)], 1)
            dG = np.stack([Gs[k + 1] - Gs[k] for k in range(len(Gs) - 1)], 1)
            Gm = dF.T @ dF
            Gm = Gm + 1e-12 * np.trace(Gm) * np.eye(Gm.shape[0])
            x = Gx - dG @ np.linalg.solve(Gm, dF.T @ Fs[-1])
        else:
            x = Gx
        out.append(x.copy())
    return out


def test_anderson_matches_reference_and_accelerates():
    from glide_b200.physics import _Anderson
    rng = np.random.default_rng(0)
    n = 200
    Q, _ = np.linalg.qr(rng.standard_normal((n, n)))
    A = Q @ np.diag(np.linspace(0.5, 0.97, n)) @ Q.T
    b = rng.standard_normal(n)
    g = lambda x: A @ x + b
    x_star = np.linalg.solve(np.eye(n) - A, b)
    ref = _reference_aa(g, np.zeros(n), 3, 25)
    aa = _Anderson(3, n, torch.float64, "cpu", products=_TorchProducts())
    x = torch.zeros(n, dtype=torch.float64)
    before = torch.empty_like(x)
    for k in range(25):
        before.copy_(x)
        x.copy_(torch.as_tensor(g(x.numpy())))
        aa.step(before, x)
        assert np.allclose(x.numpy(), ref[k], rtol=1e-9, atol=1e-9), k
    plain = np.zeros(n)
    for _ in range(25):
        plain = g(plain)
    assert np.linalg.norm(x.numpy() - x_star) < 0.05 * np.linalg.norm(plain - x_star)  # measured 0.006
