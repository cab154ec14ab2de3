"""g2oc_backward: implicit-function-theorem gradients of a loss on the
converged bundle adjustment with respect to the measured pixel coordinates
and the per-edge log-information weights.

Loss: L = sum_i |c_i - c_i^truth|^2 over the camera centres c_i = -R_i^T t_i.
Checked two ways:
  - against a dense FP64 reference on 20 cameras / 500 points: the exact
    Hessian built column by column from central differences of the oracle's
    FP64 gradient, a dense solve, and the analytic dG/dtheta from the oracle's
    errors and Jacobians (tolerance 1e-6 relative to the largest gradient);
  - against central finite differences of L through re-optimization (FP64,
    step 1e-4) on random coordinates, to 1e-4 relative, with the gradient
    taken through a torch.autograd.Function whose backward calls the C-ABI.
"""
import numpy as np
import pytest

from g2o_b200 import synth
from g2o_b200.abi import PREC_MIXED

pytestmark = pytest.mark.gpu

FD_STEP = 1e-4
FD_TOL = 1e-4
REOPT_ITERATIONS = 30
DENSE_TOL = 1e-6


@pytest.fixture(scope="module")
def backend():
    from g2o_b200 import backend as B
    B.library()
    return B


def converge(backend, g):
    """Estimates at the optimum: LM, then Gauss-Newton with exact (Cholesky) solves."""
    fac = backend.OptimizationAlgorithmFactory.instance()
    c = backend.CudaProblem(g, fac.construct("lm_cuda_chol"))
    c.optimize(30)
    c.set_params(fac.construct("gn_cuda_chol"))
    c.optimize(REOPT_ITERATIONS)
    pose, point = c.estimates()
    return c, pose, point


def adjoint(backend, g, pose, point, params):
    c = backend.CudaProblem(g, params)
    c.set_estimates(pose, point)
    L, dpose = synth.centre_loss(pose, g.extra["truth_pose"])
    dmeas, dlogw, st = c.backward(dpose, np.zeros((g.num_points, 3)))
    c.close()
    return L, dmeas, dlogw, st


# ------------------------------------------------------------ dense reference
def _se3_left_update(pose, u):
    """exp(u) * T for (t, q) 7-vectors; u = [omega, upsilon]."""
    from oracle import oracle as O
    E = O.se3quat_exp(u)
    Re = synth._quat_to_rot(E[3:7])
    R = synth._quat_to_rot(pose[3:7])
    Rn = Re @ R
    tn = Re @ pose[:3] + E[:3]
    return np.concatenate([tn, synth._rot_to_quat(Rn)])


def dense_reference(g, pose, point, dl_dpose, h=1e-6):
    from oracle import oracle as O
    o = O.OracleProblem(g)
    free_pose = [i for i in range(g.num_poses) if not g.pose_fixed[i]]
    Cf, P = len(free_pose), g.num_points
    n = Cf * 6 + P * 3

    def grad_at(j, step):
        """G = grad F = -b at x* with tangent coordinate j moved by step"""
        ps, pt = pose.copy(), point.copy()
        if j < Cf * 6:
            u = np.zeros(6)
            u[j % 6] = step
            ps[free_pose[j // 6]] = _se3_left_update(pose[free_pose[j // 6]], u)
        else:
            pt[(j - Cf * 6) // 3, (j - Cf * 6) % 3] += step
        o.set_estimates(ps, pt)
        o.build_system()
        return -o.hessian()[3]

    H = np.empty((n, n))
    for j in range(n):
        H[:, j] = (grad_at(j, h) - grad_at(j, -h)) / (2 * h)
    H = 0.5 * (H + H.T)
    gvec = np.concatenate([dl_dpose[free_pose].reshape(-1), np.zeros(P * 3)])
    v = np.linalg.solve(H, gvec)
    o.set_estimates(pose, point)
    e = o.errors()
    j0, j1 = o.jacobians()
    hidx = {i: k for k, i in enumerate(free_pose)}
    dmeas = np.zeros((g.num_edges, 2))
    dlogw = np.zeros(g.num_edges)
    for k in range(g.num_edges):
        pt, cam = g.edge_vertex[k]
        u = j0[k] @ v[Cf * 6 + 3 * pt: Cf * 6 + 3 * pt + 3]
        if cam in hidx:
            u = u + j1[k] @ v[6 * hidx[cam]: 6 * hidx[cam] + 6]
        Om = g.information[k].reshape(2, 2)
        dmeas[k] = -(Om @ u)
        dlogw[k] = -(e[k] @ Om @ u)
    return dmeas, dlogw


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_adjoint_matches_dense_fp64_reference(backend, precision):
    g = synth.adjoint_problem(num_cameras=20, num_points=500, seed=77)
    c, pose, point = converge(backend, g)
    c.close()
    _, dpose = synth.centre_loss(pose, g.extra["truth_pose"])
    rm, rw = dense_reference(g, pose, point, dpose)
    prm = backend.default_params(precision=PREC_MIXED) if precision == "mixed" else backend.default_params()
    _, dm, dw, st = adjoint(backend, g, pose, point, prm)
    assert np.abs(dm - rm).max() <= DENSE_TOL * np.abs(rm).max()
    assert np.abs(dw - rw).max() <= DENSE_TOL * np.abs(rw).max()


class ConvergedLoss:
    """torch.autograd.Function factory: forward = the loss at the optimum for
    given measurements and log-information weights (the optimum itself taken
    from the converged estimates); backward = g2oc_backward."""

    @staticmethod
    def make(backend, g, pose, point, params):
        import torch

        class F(torch.autograd.Function):
            @staticmethod
            def forward(ctx, meas, logw):
                L, _ = synth.centre_loss(pose, g.extra["truth_pose"])
                return torch.tensor(L, dtype=torch.float64)

            @staticmethod
            def backward(ctx, grad_out):
                _, dm, dw, _ = adjoint(backend, g, pose, point, params)
                s = float(grad_out)
                return torch.from_numpy(dm * s), torch.from_numpy(dw * s)

        return F


def loss_after_reopt(backend, c, g2, pose, point):
    # Gauss-Newton on a robust cost converges linearly (its Hessian keeps
    # rho' where the exact one has rho' + 2 rho'' s along the residual of an
    # edge in Huber's linear regime), so the shift of the optimum is resolved
    # to the finite-difference accuracy only after a few tens of iterations
    c.upload(g2)  # same topology: values only
    c.set_estimates(pose, point)
    c.optimize(REOPT_ITERATIONS)
    p, _ = c.estimates()
    return synth.centre_loss(p, g2.extra["truth_pose"])[0]


def fd_check(backend, g, precision, ncoords, seed):
    import torch
    c, pose, point = converge(backend, g)
    prm = backend.default_params(precision=PREC_MIXED) if precision == "mixed" else backend.default_params()
    F = ConvergedLoss.make(backend, g, pose, point, prm)
    meas = torch.tensor(g.measurement, requires_grad=True)
    logw = torch.zeros(g.num_edges, dtype=torch.float64, requires_grad=True)
    L = F.apply(meas, logw)
    dm, dw = torch.autograd.grad(L, [meas, logw])
    dm, dw = dm.numpy(), dw.numpy()
    # coordinates: edges of free cameras, half measurements, half weights
    rng = np.random.default_rng(seed)
    free_edges = np.nonzero(~g.pose_fixed[g.edge_vertex[:, 1]].astype(bool))[0]
    picks = rng.choice(free_edges, ncoords, replace=False)
    fac = backend.OptimizationAlgorithmFactory.instance()
    c.set_params(fac.construct("gn_cuda_chol"))
    scale_m, scale_w = np.abs(dm).max(), np.abs(dw).max()
    worst = 0.0
    for k, e in enumerate(picks):
        Ls = []
        if k % 2 == 0:
            comp = int(rng.integers(2))
            for sgn in (1, -1):
                g2 = g.copy()
                g2.measurement[e, comp] += sgn * FD_STEP
                Ls.append(loss_after_reopt(backend, c, g2, pose, point))
            ad, scale = dm[e, comp], scale_m
        else:
            for sgn in (1, -1):
                g2 = g.copy()
                g2.information[e] *= np.exp(sgn * FD_STEP)
                Ls.append(loss_after_reopt(backend, c, g2, pose, point))
            ad, scale = dw[e], scale_w
        fd = (Ls[0] - Ls[1]) / (2 * FD_STEP)
        err = abs(fd - ad) / max(abs(fd), abs(ad), 1e-2 * scale)
        worst = max(worst, err)
        assert err <= FD_TOL, (k, e, fd, ad)
    c.close()
    return worst


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_adjoint_matches_finite_differences(backend, precision):
    fd_check(backend, synth.adjoint_problem(num_cameras=40, num_points=3000, seed=78), precision, 16, 5)


def test_adjoint_config_instance_matches_finite_differences(backend):
    """The adjoint configuration itself: 200 cameras / 40k points, mixed
    precision, 64 random coordinates."""
    fd_check(backend, synth.adjoint_problem(), "mixed", 64, 6)


def test_backward_rejects_pose_graphs(backend):
    g = synth.pose_graph_2d(num_poses=50, num_closures=10, seed=4)
    c = backend.CudaProblem(g)
    with pytest.raises(Exception):
        c.backward(np.zeros((g.num_poses, 3)), np.zeros((0, 3)))
