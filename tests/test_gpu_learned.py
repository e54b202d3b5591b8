"""Learned min-sum training kernels: the hand-written backward against a
float reference gradient (the same unrolled layered decoder written with
torch operations and differentiated by autograd) and against finite
differences of the CUDA forward; a few optimiser steps lower the loss."""
import numpy as np
import pytest
import torch

import dvbrx_b200 as D
from dvbrx_b200 import learned as Lm

pytestmark = pytest.mark.gpu


def reference_loss(short, rate, llr, bits, beta, alpha, iters, cod, weights=None):
    """The learned decoder in torch (float64): same schedule (steps of the
    library's wavefront levels), same saturations, autograd gradients."""
    step, links = Lm.schedule(short, rate)
    K = D.code_info(short, rate).K
    kl = D.fec_lookup(short, rate).kldpc
    n, N = llr.shape
    R, DS = links.shape
    P = llr.clamp(-128, 127)
    M = torch.zeros((n, R, DS), dtype=llr.dtype, device=llr.device)
    groups = [np.nonzero(step == s)[0] for s in range(int(step.max()) + 1)]
    b = torch.from_numpy(bits).to(llr.device)
    sgnb = 1.0 - 2.0 * b.double()
    total = 0.0
    w = np.ones(iters) if weights is None else np.asarray(weights, np.float64)
    for t in range(iters):
        Mn = M.clone()
        for chk in groups:
            L = links[chk]
            valid = torch.from_numpy(L >= 0).to(llr.device)
            idx = torch.from_numpy(np.where(L >= 0, L, 0)).long().to(llr.device)
            deg = valid.sum(dim=1)
            cls = torch.from_numpy(cod[(L >= 0).sum(axis=1)].astype(np.int64)).to(llr.device)
            ck = torch.from_numpy(chk.astype(np.int64)).to(llr.device)
            x = P[:, idx] - (Mn[:, ck, :] if t > 0 else 0.0)
            x = x.clamp(-128, 127)
            a = torch.where(valid, x.abs(), torch.full_like(x, 1e30))
            vals, inds = torch.topk(a, 2, dim=-1, largest=False)
            slot = torch.arange(DS, device=llr.device)
            mu = torch.where(slot == inds[..., :1], vals[..., 1:2], vals[..., 0:1]).clamp(max=127)
            mag = torch.relu(beta[t][cls][None, :, None] * mu - alpha[t][cls][None, :, None])
            negs = ((x < 0) & valid).sum(dim=-1, keepdim=True) % 2
            sneg = (negs + (x < 0).long()) % 2
            m = torch.where(sneg == 1, -mag, mag)
            newp = (x + m).clamp(-128, 127)
            P = P.clone()
            vi = idx[valid]
            P[:, vi] = newp[:, valid]
            Mn = Mn.clone()
            Mn[:, ck, :] = torch.where(valid, m.clamp(-32, 31), torch.zeros_like(m))
            del deg
        M = Mn
        total = total + float(w[t]) * torch.nn.functional.softplus(-sgnb * P[:, :kl] / 2).sum()
    del K
    return total / (float(w.sum()) * n * kl)


def small_case(short, rate, n, es, iters, seed):
    p = D.fec_lookup(short, rate)
    dec = D.Ldpc(p, rate)
    _, info, llr16 = dec.generate(n, es, seed=seed, info=True, llr=False, llr_f16=True)
    bits = np.unpackbits(info.cpu().numpy(), axis=1)[:, : p.kldpc]
    return dec, llr16, info, bits


@pytest.mark.parametrize("weights", [None, [0.0, 0.5, 2.0]])
def test_backward_matches_float_reference(weights):
    short, rate, iters = 1, "1_2", 3
    dec, llr16, info, bits = small_case(short, rate, 3, 1.2, iters, 5)
    degs, cod = Lm.degree_classes(short, rate)
    nclass = len(degs)
    g = torch.Generator(device="cpu").manual_seed(0)
    beta0 = (0.75 + 0.5 * torch.rand((iters, nclass), generator=g)).half().float().cuda()
    alpha0 = (0.25 + 1.5 * torch.rand((iters, nclass), generator=g)).half().float().cuda()

    beta = beta0.clone().requires_grad_(True)
    alpha = alpha0.clone().requires_grad_(True)
    work = Lm._Work(dec, llr16.shape[0], iters, cod, weights)
    loss = Lm.LearnedMinSum.apply(beta, alpha, dec, llr16, info, iters, cod, work)
    loss.backward()

    rb = beta0.double().clone().requires_grad_(True)
    ra = alpha0.double().clone().requires_grad_(True)
    rl = reference_loss(short, rate, llr16.double(), bits, rb, ra, iters, cod, weights)
    rl.backward()
    assert abs(float(loss.detach()) - float(rl.detach())) <= 1e-4 * abs(float(rl.detach())) + 1e-6
    for got, want in ((beta.grad, rb.grad), (alpha.grad, ra.grad)):
        want = want.float()
        err = (got - want).norm() / want.norm()
        assert err < 1e-3, float(err)


def test_backward_matches_finite_differences():
    short, rate, iters = 0, "2_3", 4
    dec, llr16, info, bits = small_case(short, rate, 8, 6.3, iters, 9)
    degs, cod = Lm.degree_classes(short, rate)
    nclass = len(degs)
    beta = torch.ones((iters, nclass), device="cuda") * 0.875
    alpha = torch.ones((iters, nclass), device="cuda") * 0.5
    work = Lm._Work(dec, llr16.shape[0], iters, cod)
    b = beta.clone().requires_grad_(True)
    a = alpha.clone().requires_grad_(True)
    Lm.LearnedMinSum.apply(b, a, dec, llr16, info, iters, cod, work).backward()
    k = degs.index(max(degs))  # the class every check but one has
    eps = 1.0 / 32  # exact steps of the FP16 parameters near 1
    for t in range(iters):
        for grad, base, which in ((b.grad, beta, "beta"), (a.grad, alpha, "alpha")):
            up, dn = base.clone(), base.clone()
            up[t, k] += eps
            dn[t, k] -= eps
            lu = Lm.LearnedMinSum.apply(up if which == "beta" else beta, up if which == "alpha" else alpha, dec,
                                        llr16, info, iters, cod, work)
            ld = Lm.LearnedMinSum.apply(dn if which == "beta" else beta, dn if which == "alpha" else alpha, dec,
                                        llr16, info, iters, cod, work)
            fd = (float(lu) - float(ld)) / (2 * eps)
            g = float(grad[t, k])
            assert abs(fd - g) <= 0.1 * max(abs(fd), abs(g)) + 1e-6, (which, t, fd, g)


def test_training_lowers_the_loss():
    model = Lm.LearnedDecoder(0, "2_3", iters=8)
    opt = torch.optim.Adam(model.parameters(), lr=0.02)
    rng = np.random.default_rng(3)
    first = last = None
    for stepi in range(12):
        es = float(rng.uniform(6.0, 7.5))
        _, info, llr16 = model.dec.generate(64, es, seed=100 + stepi, info=True, llr=False, llr_f16=True)
        loss = model(llr16, info)
        opt.zero_grad()
        loss.backward()
        opt.step()
        if first is None:
            first = float(loss)
        last = float(loss)
    # the same frames before and after training
    _, info, llr16 = model.dec.generate(64, 6.75, seed=999, info=True, llr=False, llr_f16=True)
    trained = float(model(llr16, info))
    plain = Lm.LearnedDecoder(0, "2_3", iters=8)
    base = float(plain(llr16, info))
    assert trained < base, (trained, base)
