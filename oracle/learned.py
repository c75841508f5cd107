"""Float64 CPU restatement of the learned momentum proposal's network (TEST INFRASTRUCTURE ONLY).

The reference has no learned component; this oracle restates the network of base/learnedProposal.py -- a ReLU MLP,
squared-error loss on the first `nout` outputs -- in float64 torch on the CPU:
  * `mlp_loss_and_grads`: exact-arithmetic gradients from torch.autograd (the ideal network);
  * `mlp_loss_and_grads_bf16`: the same network with the device's rounding points restated -- hidden activations
    stored in bf16, output in f32, backward deltas stored in bf16 -- with a hand-written backward pass, so that the
    device kernels are compared with an oracle that differs only in summation order.
"""
import torch


def _bf16(t):
    return t.to(torch.bfloat16).to(torch.float64)


def mlp_loss_and_grads(F, W, b, target, nout, weight):
    """F (M, d0), W[i] (d_i, d_{i+1}), b[i] (d_{i+1}), target (M, nout): returns (loss, y, [dW..., db...])."""
    F = F.to(torch.float64).cpu()
    Ws = [w.to(torch.float64).cpu().clone().requires_grad_(True) for w in W]
    bs = [v.to(torch.float64).cpu().clone().requires_grad_(True) for v in b]
    h = F
    for i in range(len(Ws)):
        h = h @ Ws[i] + bs[i]
        if i < len(Ws) - 1:
            h = torch.relu(h)
    y = h
    loss = weight * ((y[:, :nout] - target.to(torch.float64).cpu()) ** 2).sum()
    loss.backward()
    return loss.detach(), y.detach(), [w.grad for w in Ws] + [v.grad for v in bs]


def mlp_loss_and_grads_bf16(F, W, b, target, nout, weight):
    """As `mlp_loss_and_grads` with bf16 storage of activations and deltas (the device's rounding points)."""
    F = F.to(torch.float64).cpu()
    Ws = [w.to(torch.float64).cpu() for w in W]
    bs = [v.to(torch.float64).cpu() for v in b]
    L = len(Ws)
    acts = [_bf16(F)]
    h = acts[0]
    for i in range(L - 1):
        h = _bf16(torch.relu(h @ Ws[i] + bs[i]))
        acts.append(h)
    y = h @ Ws[L - 1] + bs[L - 1]
    t = target.to(torch.float64).cpu()
    diff = y[:, :nout] - t
    loss = weight * (diff ** 2).sum()
    dy = torch.zeros_like(y)
    dy[:, :nout] = 2.0 * weight * diff
    dy = _bf16(dy)
    dW, db = [None] * L, [None] * L
    for i in range(L - 1, -1, -1):
        dW[i] = acts[i].t() @ dy
        db[i] = dy.sum(dim=0)
        if i > 0:
            dy = _bf16((dy @ Ws[i].t()) * (acts[i] > 0))
    return loss, y, dW + db
