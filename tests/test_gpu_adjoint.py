"""The adjoint pass (nd_march_backward) against FP64 central finite differences.

Workload: the differentiation view -- Mandelbulb (12 iterations, escape radius as a
parameter) with Lambert shading from one directional light, orbit camera;
theta = (power, bailout, yaw, pitch, distance); loss: mean squared difference to a
target rendered at power 8 with the camera yawed 2 degrees.  The hit bisection runs
its whole budget (ND_VIEW_EXACT_HIT) so that the hit distance is a smooth function
of theta; with the reference's stop at eps(t) it is a step function of theta.

What the adjoint differentiates: the shade of every ray that hits, the hit point
moving on its surface sheet (implicit differentiation of DE = eps(t)) through the
central-difference normal and the Lambert term.  Visibility changes are not
differentiated, nor are hits on a jump of the DE (a Mandelbulb of non-integer power
jumps across the preimages of atan2's branch cut; a hit there follows the jump, not
the level set): the test finds those rays itself, from the FP64 residual
|DE(p) - eps(t)| at the hit, and leaves them out.  A 12-iteration Mandelbulb's shade is not smooth at the scale of a
1e-3 step in theta on most rays (the normal field turns over at the scale of the
normal taps, h = 1e-4 t), so the checks use the rays on which the FP64 central
difference itself has converged: hit in every render, and the difference at step 1e-5
agrees to 1e-4 relative with those at steps 3e-5 and 1e-6.  The reference value is the
difference at step 1e-5.

The finite differences are taken of an FP64 shade: the FP64 forward's hit distance
(depth64), the six normal taps evaluated with the FP64 DE (nd_de_points) and the
Lambert term in FP64 -- the G-buffer's f32 normal and shade would put rounding steps
of ~1e-7 into every difference.  Formula parameters are stored as f32, so their
differences divide by the step the f32 value really took.  The loss difference at step
1e-3 over all hit rays is printed beside the adjoint for the record.

torch.autograd.Function wraps the forward/backward pair here, in the test harness only.
"""

import math

import numpy as np
import pytest
import torch

from numericdream_b200 import abi, runtime, workloads

pytestmark = pytest.mark.gpu

SIZE = 128
PROBLEMS = 2
STEPS = (1e-5, 3e-5, 1e-6)  # the reference step first
CONVERGED = 1e-4      # FD(1e-5) vs FD(3e-5) and FD(1e-6), relative
PER_RAY_TOL = 1e-3    # adjoint vs converged FD, relative, per ray
SUM_TOL = 1e-3        # sum over converged rays, relative to the sum of |FD|
# The FP32 adjoint (the one the differentiation benchmark times) is held to the
# same 1e-3 relative target on its median and on the sum over converged rays; its DE
# carries ~1e-3 relative rounding near the surface, so single rays may exceed it
SUM_TOL_FP32 = 1e-3
NAMES = ("power", "bailout", "yaw", "pitch", "dist")


def _views(theta):
    views, cams = [], []
    for th in theta:
        v, c = workloads.mandelbulb_512(runtime.find_formula, power=float(th[0]), bailout=float(th[1]),
                                        yaw=float(th[2]), pitch=float(th[3]), dist=float(th[4]), size=SIZE)
        views.append(v)
        cams.append(c)
    return views, cams


def _render(ctx, theta, de_precision=64):
    views, cams = _views(theta)
    g = runtime.GBuffer.allocate(workloads.rays(views))
    ctx.forward(views, g, runtime.make_opts(kernel=abi.ND_KERNEL_PERSISTENT, de_precision=de_precision))
    torch.cuda.synchronize()
    return views, cams, g


def _shade64(ctx, views, g, residual=False):
    """FP64 Lambert shade of the rays of an FP64 forward: normal by central differences
    (h = normal_h_coef t) of the FP64 DE at the depth64 hit point, light in FP64.
    With residual=True also |DE(p) - eps(t)| / eps(t) at the hit."""
    out = torch.zeros((len(views), SIZE * SIZE), dtype=torch.float64, device="cuda")
    res = torch.zeros_like(out)
    t_all = g.depth64.view(len(views), -1)
    hit_all = _hit(g)
    for i, v in enumerate(views):
        j = torch.arange(SIZE * SIZE, device="cuda", dtype=torch.float64)
        px, py = j % SIZE, torch.div(j, SIZE, rounding_mode="floor")
        ux = (2.0 * (px + 0.5) / SIZE - 1.0) * (v.width / v.height)
        uy = -(1.0 - 2.0 * (py + 0.5) / SIZE)
        f, r, u = (torch.tensor(list(a), dtype=torch.float64, device="cuda") for a in (v.fwd, v.right, v.up))
        w = f[None, :] + ux[:, None] * r[None, :] + uy[:, None] * u[None, :]
        d = w / torch.linalg.norm(w, dim=1, keepdim=True)
        t = torch.where(hit_all[i], t_all[i], torch.ones_like(t_all[i]))
        p = torch.tensor(list(v.cam_pos), dtype=torch.float64, device="cuda")[None, :] + d * t[:, None]
        h = float(np.float32(v.normal_h_coef)) * t
        if residual:
            eps = float(np.float32(v.eps_coef)) * t + float(np.float32(v.eps_floor))
            de0, _, _ = ctx.de_points(v, p, 64)
            res[i] = (torch.as_tensor(de0, device="cuda") - eps).abs() / eps
        taps = []
        for ax in range(3):
            e = torch.zeros(3, dtype=torch.float64, device="cuda")
            e[ax] = 1.0
            taps += [p + h[:, None] * e, p - h[:, None] * e]
        de, _, _ = ctx.de_points(v, torch.stack(taps, 1).reshape(-1, 3), 64)
        de = torch.as_tensor(de, device="cuda").view(-1, 6)
        D = torch.stack([de[:, 0] - de[:, 1], de[:, 2] - de[:, 3], de[:, 4] - de[:, 5]], 1)
        n = D / torch.linalg.norm(D, dim=1, keepdim=True)
        L = torch.tensor([float(np.float32(x)) for x in v.light_dir], dtype=torch.float64, device="cuda")
        L = L / torch.linalg.norm(L)
        lam = torch.clamp(n @ L, min=0.0)
        out[i] = torch.where(hit_all[i], 0.18 + 0.82 * lam, torch.zeros_like(lam))
    return (out, res) if residual else out


def _hit(g):
    return (g.normal[:, 3] > 0.5).view(PROBLEMS, -1)


def _theta0():
    rng = np.random.default_rng(11)
    # powers exact in f32, so that the f32 steps either side are symmetric
    return np.stack([np.array([float(np.float32(rng.uniform(6.0, 10.0))), 2.0, 0.01, 0.02, 2.5])
                     for _ in range(PROBLEMS)])


def _target_theta():
    return np.tile([8.0, 2.0, math.radians(2.0), 0.0, 2.5], (PROBLEMS, 1))


def _step_taken(theta, k, h):
    """(theta + h, theta - h, the denominator of the central difference)."""
    tp, tm = theta.copy(), theta.copy()
    tp[:, k] += h
    tm[:, k] -= h
    if k < 2:  # formula parameters are f32 in the view
        tp[:, k] = tp[:, k].astype(np.float32)
        tm[:, k] = tm[:, k].astype(np.float32)
    return tp, tm, torch.tensor(tp[:, k] - tm[:, k], dtype=torch.float64, device="cuda")[:, None]


def _shade_of(ctx, theta):
    views, _, g = _render(ctx, theta, 64)
    return _shade64(ctx, views, g), _hit(g)


def _fd(ctx, theta, k, h):
    tp, tm, den = _step_taken(theta, k, h)
    sp, hp = _shade_of(ctx, tp)
    sm, hm = _shade_of(ctx, tm)
    return (sp - sm) / den, hp & hm


@pytest.fixture(scope="module")
def study(ctx):
    """Per-ray FP64 finite differences of the shade at two steps, for every theta."""
    theta = _theta0()
    views, cams, g64 = _render(ctx, theta, 64)
    _, _, g32 = _render(ctx, theta, 32)
    hit = _hit(g64)
    s64, resid = _shade64(ctx, views, g64, residual=True)
    root = hit & (resid <= 1e-6)
    print(f"hit rays {int(hit.sum())}, of which on a jump of the DE (residual > 1e-6 eps): "
          f"{int((hit & ~root).sum())}")
    fds, masks = [], []
    for k in range(5):
        f1, m1 = _fd(ctx, theta, k, STEPS[0])
        conv = root & m1 & (f1 != 0)
        for h in STEPS[1:]:
            f2, m2 = _fd(ctx, theta, k, h)
            conv &= m2 & ((f1 - f2).abs() <= CONVERGED * f1.abs())
        fds.append(f1)
        masks.append(conv)
    return {"ctx": ctx, "theta": theta, "views": views, "cams": cams, "g64": g64, "g32": g32, "hit": hit,
            "root": root, "s64": s64, "fd": fds, "conv": masks}


def _per_ray(s, g, prec):
    _, per = s["ctx"].backward(s["views"], s["cams"], g, None, param_idx=(0, 2), de_precision=prec, per_ray=True)
    torch.cuda.synchronize()
    # columns: power, bailout, yaw, pitch, dist
    return [per[:, j].view(PROBLEMS, -1) for j in range(5)]


def _compare(s, adj, label):
    rows = []
    for k in (0, 2, 3, 4):
        m = s["conv"][k]
        fd = s["fd"][k][m]
        a = adj[k][m]
        rel = ((a - fd).abs() / fd.abs()).cpu().numpy()
        within = float((rel <= PER_RAY_TOL).mean()) if rel.size else 0.0
        sum_err = float((a.sum() - fd.sum()).abs() / fd.abs().sum()) if rel.size else float("inf")
        rows.append((NAMES[k], int(m.sum()), within, float(np.median(rel)) if rel.size else 0.0, sum_err))
        print(f"{label} {NAMES[k]:6s} converged rays {int(m.sum()):5d}  within {PER_RAY_TOL:g}: {within:.3f}  "
              f"median rel {rows[-1][3]:.2e}  sum rel {sum_err:.2e}")
    return rows


def test_adjoint_fp64_matches_converged_fd_per_ray(study):
    rows = _compare(study, _per_ray(study, study["g64"], 64), "fp64 adjoint")
    for name, n, within, _, sum_err in rows:
        assert n >= 100, f"{name}: only {n} rays with a converged finite difference"
        assert within >= 0.9, f"{name}: {within:.3f} of converged rays within {PER_RAY_TOL}"
        assert sum_err <= SUM_TOL, f"{name}: sum over converged rays off by {sum_err:.2e}"


def test_adjoint_fp32_matches_converged_fd_sum(study):
    rows = _compare(study, _per_ray(study, study["g64"], 32), "fp32 adjoint at the fp64 hit")
    for name, n, within, median, sum_err in rows:
        assert median <= 1e-3, f"{name}: median relative error {median:.2e}"
        assert sum_err <= SUM_TOL_FP32, f"{name}: sum over converged rays off by {sum_err:.2e}"
    # the production path: FP32 forward, FP32 adjoint (hit distances differ by the FP32 DE's error)
    rows = _compare(study, _per_ray(study, study["g32"], 32), "fp32 forward + fp32 adjoint")
    for name, n, within, median, sum_err in rows:
        assert median <= 1e-3, f"fp32 forward: {name}: median relative error {median:.2e}"
        assert sum_err <= SUM_TOL_FP32, f"fp32 forward: {name}: sum over converged rays off by {sum_err:.2e}"


def test_bailout_gradient_is_zero(study):
    adj = _per_ray(study, study["g64"], 64)
    assert bool((adj[1] == 0).all())
    m = study["conv"][1]
    print(f"bailout: {int(m.sum())} rays with a converged nonzero FD; "
          f"hit rays with FD exactly 0 at step 1e-5: {float(((study['fd'][1] == 0) & study['hit']).sum())}")


def test_loss_gradient_matches_fd_on_converged_rays(study):
    """dLoss/dtheta from nd_march_backward for the mean-L2 loss over the converged rays
    of each theta, against the FP64 central difference of that loss at step 1e-5."""
    ctx, theta = study["ctx"], study["theta"]
    target, _ = _shade_of(ctx, _target_theta())
    for k in (0, 2, 3, 4):
        m = study["conv"][k].double()
        npx = float(m.sum())

        def loss_of(shade):
            return (((shade - target) ** 2) * m).sum(1) / npx

        tp, tm, den = _step_taken(theta, k, STEPS[0])
        fd = ((loss_of(_shade_of(ctx, tp)[0]) - loss_of(_shade_of(ctx, tm)[0])) / den[:, 0]).cpu().numpy()
        g64 = study["g64"]
        img = study["s64"]
        w = 2.0 * (img - target) * m / npx
        grad = ctx.backward(study["views"], study["cams"], g64, w.float().reshape(-1), param_idx=(0, 2),
                            de_precision=64)
        adj = grad[:, k].cpu().numpy()
        # scale: the sum over rays of |dLoss/dshade * dshade/dtheta|
        scale = (w.abs() * study["fd"][k].abs() * m).sum(1).cpu().numpy()
        rel = np.abs(adj - fd) / np.maximum(scale, 1e-30)
        print(f"loss {NAMES[k]:6s} fd {fd} adjoint {adj} rel {rel}")
        assert (rel <= SUM_TOL).all()


def test_autograd_function_and_step_1e3_record(study):
    """The C-ABI pair behind torch.autograd.Function (FP32 forward and adjoint), and
    for the record the FP64 loss difference at step 1e-3 over every hit ray."""
    ctx = study["ctx"]

    class MarchShade(torch.autograd.Function):
        @staticmethod
        def forward(fctx, th):
            views, cams, g = _render(ctx, th.detach().cpu().numpy(), 32)
            fctx.state = (views, cams, g)
            return g.shade.view(len(views), -1).clone()

        @staticmethod
        def backward(fctx, grad_shade):
            views, cams, g = fctx.state
            gr = ctx.backward(views, cams, g, grad_shade.reshape(-1).float().contiguous(), param_idx=(0, 2))
            return gr.to(grad_shade.device)

    target = torch.tensor(_target_theta(), dtype=torch.float64, device="cuda")
    with torch.no_grad():
        t_img = MarchShade.apply(target).double()
    theta = torch.tensor(study["theta"], dtype=torch.float64, device="cuda", requires_grad=True)
    img = MarchShade.apply(theta)
    loss = ((img.double() - t_img) ** 2).mean()
    loss.backward()
    g = theta.grad
    assert g is not None and torch.isfinite(g).all()
    assert (g[:, 1] == 0).all()
    print("autograd dLoss/dtheta (power, bailout, yaw, pitch, dist):", g.cpu().numpy())

    # the 1e-3 secant of the loss over rays that hit in all three renders, beside the adjoint
    theta0 = study["theta"]
    target_img, _ = _shade_of(ctx, _target_theta())
    for k in (0, 2, 3, 4):
        tp, tm, den = _step_taken(theta0, k, 1e-3)
        sp, hp = _shade_of(ctx, tp)
        sm, hm = _shade_of(ctx, tm)
        m = (study["hit"] & hp & hm).double()
        n = m.sum(1)
        fd = ((((sp - target_img) ** 2 - (sm - target_img) ** 2) * m).sum(1) / n / den[:, 0])
        dl = (2.0 * (study["s64"] - target_img) * m / n[:, None]).float().reshape(-1)
        adj = ctx.backward(study["views"], study["cams"], study["g64"], dl, param_idx=(0, 2), de_precision=64)[:, k]
        print(f"step 1e-3 {NAMES[k]:6s} loss FD {fd.cpu().numpy()} adjoint {adj.cpu().numpy()}")
