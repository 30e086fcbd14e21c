"""The steady glucose field and its adjoint (bcg_steady_*; no counterpart in
the reference).  CPU: the scipy FP64 reference's adjoint gradients against
central finite differences (h = 1e-6 relative).  GPU: the CUDA solve and
VJP against that reference, the torch.autograd wrapper, and central finite
differences of the CUDA solve itself.

Loss: squared L2 distance of the radial mean concentration profile on the
agar surface row to a seeded target profile."""
import numpy as np
import pytest

from baccolonygrowth_b200 import steady as st

from steady_ref import SteadyRef

THETA = np.array([0.8, 0.3, 1.0, 0.05])      # d_agar, d_colony, vmax, km


def small_case(nx=17, nz=9, nz_agar=5, n=60, seed=3):
    cells, w, x0 = st.synthetic_problem(nx=nx, nz=nz, nz_agar=nz_agar, h=2.0, n_cells=n, seed=seed)
    return dict(nx=nx, nz=nz, nz_agar=nz_agar, h=2.0, c0=20.0), cells, w, x0


def loss_and_grad(C, h, x0, nbins, row, target):
    b, cnt = st.radial_bins(C.shape[1], h, x0, nbins, row)
    prof = np.bincount(b, weights=C[row], minlength=nbins) / cnt
    diff = prof - target
    g = np.zeros_like(C)
    g[row] = 2 * diff[b] / cnt[b]
    return float((diff ** 2).sum()), g


def test_reference_adjoint_matches_finite_differences():
    g0, cells, w, x0 = small_case()
    ref = SteadyRef(g0["nx"], g0["nz"], g0["nz_agar"], g0["h"], g0["c0"], cells)
    row, nbins = g0["nz_agar"] - 1, 4
    target = np.linspace(19.0, 19.9, nbins)
    C = ref.solve(THETA, w)
    L0, dLdC = loss_and_grad(C, g0["h"], x0, nbins, row, target)
    gt, gw = ref.gradients(dLdC)
    for j in range(4):
        e = 1e-6 * THETA[j]
        tp, tm = THETA.copy(), THETA.copy()
        tp[j] += e; tm[j] -= e
        fd = (loss_and_grad(ref.solve(tp, w), g0["h"], x0, nbins, row, target)[0]
              - loss_and_grad(ref.solve(tm, w), g0["h"], x0, nbins, row, target)[0]) / (2 * e)
        assert abs(fd - gt[j]) <= 1e-5 * max(abs(fd), 1e-3 * abs(L0)), (j, fd, gt[j])
    for c in (0, 7, 31):
        wp, wm = w.copy(), w.copy()
        e = 1e-6 * w[c]
        wp[c] += e; wm[c] -= e
        fd = (loss_and_grad(ref.solve(THETA, wp), g0["h"], x0, nbins, row, target)[0]
              - loss_and_grad(ref.solve(THETA, wm), g0["h"], x0, nbins, row, target)[0]) / (2 * e)
        assert abs(fd - gw[c]) <= 1e-5 * max(abs(fd), 1e-6 * abs(L0)), (c, fd, gw[c])


@pytest.mark.gpu
def test_cuda_steady_matches_reference(gpu):
    g0, cells, w, x0 = small_case(nx=33, nz=17, nz_agar=9, n=400, seed=5)
    ref = SteadyRef(g0["nx"], g0["nz"], g0["nz_agar"], g0["h"], g0["c0"], cells)
    s = st.Steady(max_cells=len(cells), **g0)
    s.set_cells(cells)
    row, nbins = g0["nz_agar"] - 1, 6
    target = np.linspace(18.0, 19.9, nbins)
    Cr = ref.solve(THETA, w)
    Cg = s.solve(THETA, w)
    assert np.abs(Cg - Cr).max() <= 1e-10 * np.abs(Cr).max()
    _, dLdC = loss_and_grad(Cr, g0["h"], x0, nbins, row, target)
    gtr, gwr = ref.gradients(dLdC)
    gtg, gwg = s.vjp(dLdC)
    assert np.abs(gtg - gtr).max() <= 1e-7 * np.abs(gtr).max(), (gtg, gtr)
    assert np.abs(gwg - gwr).max() <= 1e-7 * np.abs(gwr).max()
    s.close()


@pytest.mark.gpu
def test_cuda_steady_torch_autograd_and_fd(gpu):
    torch = pytest.importorskip("torch")
    g0 = dict(nx=129, nz=65, nz_agar=33, h=2.0, c0=20.0)
    cells, w, x0 = st.synthetic_problem(n_cells=50000, **{k: g0[k] for k in ("nx", "nz", "nz_agar", "h")})
    s = st.Steady(max_cells=len(cells), **g0)
    s.set_cells(cells)
    row, nbins = g0["nz_agar"] - 1, 16
    target = np.linspace(15.0, 19.9, nbins)
    Field = st.make_steady_field(torch)
    theta = torch.tensor(THETA, dtype=torch.float64, requires_grad=True)
    wt = torch.tensor(w, dtype=torch.float64, requires_grad=True)
    C = Field.apply(theta, wt, s, 1e-13)
    loss = st.radial_profile_loss(torch, C, g0["h"], x0, nbins, row, target)
    loss.backward()
    # the same gradients as the VJP entry with the numpy loss gradient
    L0, dLdC = loss_and_grad(C.detach().numpy(), g0["h"], x0, nbins, row, target)
    gt, gw = s.vjp(dLdC)
    assert np.allclose(theta.grad.numpy(), gt, rtol=1e-12, atol=0)
    assert np.allclose(wt.grad.numpy(), gw, rtol=1e-12, atol=1e-300)
    # central finite differences of the CUDA solve (h = 1e-6 relative)
    for j in range(4):
        e = 1e-6 * THETA[j]
        tp, tm = THETA.copy(), THETA.copy()
        tp[j] += e; tm[j] -= e
        fd = (loss_and_grad(s.solve(tp, w), g0["h"], x0, nbins, row, target)[0]
              - loss_and_grad(s.solve(tm, w), g0["h"], x0, nbins, row, target)[0]) / (2 * e)
        assert abs(fd - gt[j]) <= 1e-4 * max(abs(fd), 1e-6 * abs(L0)), (j, fd, gt[j])
    s.close()
