"""Shared checks of the test suite (the oracle is the checker; nothing here computes a distance map)."""
import numpy as np
import torch


def assert_images_eq(got, ref, what=""):
    """Bit-exact comparison (reference tests/helpers.hpp:25-33 compares with !=), with a useful message."""
    got = got.detach().cpu().numpy() if isinstance(got, torch.Tensor) else np.asarray(got)
    ref = np.asarray(ref)
    assert got.shape == ref.shape, "%s: shape %s != %s" % (what, got.shape, ref.shape)
    bad = got.view(np.uint32) != ref.view(np.uint32)
    if bad.any():
        ys, xs = np.nonzero(bad)
        k = 0
        raise AssertionError("%s: %d of %d values differ; first at (x=%d, y=%d): got %r, expected %r" % (
            what, int(bad.sum()), bad.size, xs[k], ys[k], float(got[ys[k], xs[k]]), float(ref[ys[k], xs[k]])))


def ns_weights_torch(img, gamma):
    """Edge weights of the ns-mode graph on the GPU (float32, every operation rounded):
    returns (wx, wy) with wx[y, x] = w((x, y), (x+1, y)) and wy[y, x] = w((x, y), (x, y+1))."""
    g = torch.tensor(np.float32(gamma), dtype=torch.float32, device=img.device)
    g2 = g * g
    I = img.to(torch.int32)
    if I.dim() == 2:
        I = I[..., None]
    dx = ((I[:, 1:] - I[:, :-1]) ** 2).sum(-1).to(torch.float32)
    dy = ((I[1:] - I[:-1]) ** 2).sum(-1).to(torch.float32)
    return torch.sqrt(1.0 + g2 * dx), torch.sqrt(1.0 + g2 * dy)


def ns_fixpoint_violations(img, mask, gamma, v, D):
    """Size-independent exactness check of an ns-mode map.

    D is the greatest fixpoint iff (a) no edge can lower it: D(p) <= fl(D(q) + w) for every edge, and
    (b) every value is realised: D(p) == min(init(p), min_q fl(D(q) + w)).  For values below 2^23, (a) and (b)
    together imply equality with the greatest fixpoint (a smaller fixpoint would need a value supported only by
    smaller values, which strictly positive weights >= 1 rule out).  Returns (#violations of a, #of b, max D)."""
    wx, wy = ns_weights_torch(img, gamma)
    inf = torch.tensor(float("inf"), device=D.device)
    best = torch.where(mask != 0, torch.zeros_like(D), torch.full_like(D, float(v)))
    cand_l = torch.full_like(D, float("inf")); cand_l[:, 1:] = D[:, :-1] + wx
    cand_r = torch.full_like(D, float("inf")); cand_r[:, :-1] = D[:, 1:] + wx
    cand_u = torch.full_like(D, float("inf")); cand_u[1:, :] = D[:-1, :] + wy
    cand_d = torch.full_like(D, float("inf")); cand_d[:-1, :] = D[1:, :] + wy
    m = torch.minimum(torch.minimum(cand_l, cand_r), torch.minimum(cand_u, cand_d))
    viol_a = int((D > m).sum())
    viol_b = int((D != torch.minimum(best, m)).sum())
    del inf
    return viol_a, viol_b, float(D.max())
