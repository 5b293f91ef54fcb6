"""Size-independent exactness check of an ns-mode distance map, computed with torch on the map's device.

A map D of the C4 graph with weights w = sqrt(1 + g2 * dI2) is the greatest fixpoint of single-edge relaxations
from init = (mask != 0 ? 0 : v) iff
  (a) no edge can lower it:        D(p) <= fl(D(q) + w(p, q)) for every edge (p, q), and
  (b) every value is realised:     D(p) == min(init(p), min_q fl(D(q) + w(p, q))).
For values below 2^23, (a) and (b) together imply equality with the greatest fixpoint: a smaller fixpoint would
need a value supported only by smaller values, which strictly positive weights >= 1 rule out.  The check needs
no second implementation of the transform, so it runs at any image size.
"""
import numpy as np
import torch


def ns_weights(img, gamma):
    """Edge weights of the ns-mode graph (float32, every operation rounded separately, square root correctly
    rounded): returns (wx, wy) with wx[y, x] = w((x, y), (x+1, y)) and wy[y, x] = w((x, y), (x, y+1))."""
    g = torch.tensor(np.float32(gamma), dtype=torch.float32, device=img.device)
    g2 = g * g
    I = img.to(torch.int32)
    if I.dim() == 2:
        I = I[..., None]
    dx = ((I[:, 1:] - I[:, :-1]) ** 2).sum(-1).to(torch.float32)
    dy = ((I[1:] - I[:-1]) ** 2).sum(-1).to(torch.float32)
    return torch.sqrt(1.0 + g2 * dx), torch.sqrt(1.0 + g2 * dy)


def ns_fixpoint_violations(img, mask, gamma, v, D):
    """Returns (#pixels violating (a), #pixels violating (b), max D) for the map D of image `img` ([H, W] or
    [H, W, 3] uint8), seed mask `mask` ([H, W] uint8, non-zero = seed), gamma and unreached value v.  All
    tensors on one device; rows may be padded."""
    wx, wy = ns_weights(img, gamma)
    best = torch.where(mask != 0, torch.zeros_like(D), torch.full_like(D, float(v)))
    cand_l = torch.full_like(D, float("inf"))
    cand_l[:, 1:] = D[:, :-1] + wx
    cand_r = torch.full_like(D, float("inf"))
    cand_r[:, :-1] = D[:, 1:] + wx
    cand_u = torch.full_like(D, float("inf"))
    cand_u[1:, :] = D[:-1, :] + wy
    cand_d = torch.full_like(D, float("inf"))
    cand_d[:-1, :] = D[1:, :] + wy
    m = torch.minimum(torch.minimum(cand_l, cand_r), torch.minimum(cand_u, cand_d))
    viol_a = int((D > m).sum())
    viol_b = int((D != torch.minimum(best, m)).sum())
    return viol_a, viol_b, float(D.max()) if D.numel() else 0.0
