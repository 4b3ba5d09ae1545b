"""torch.autograd binding of the differentiable step (pbf_batch_forward_record /
pbf_batch_backward over ctypes).

``step(batch, pos, vel, sdf_offsets)`` advances every scene of ``batch`` by
one step (all substeps and iterations) from the given state and returns the
final positions and velocities; gradients flow back to ``pos``, ``vel`` (n,3)
and ``sdf_offsets`` (num_scenes,3), the translation of each scene's SDF
obstacle.  The backward is the hand-written adjoint of the engine
(k_adjoint.cu) with per-substep checkpoints; when other steps were recorded
in between, the step is recorded again from the saved inputs first.
"""
import itertools

import numpy as np
import torch

_tokens = itertools.count(1)


def _pad4(x):
    out = torch.zeros((x.shape[0], 4), dtype=torch.float32, device=x.device)
    out[:, :3] = x.detach()
    return out


class _Step(torch.autograd.Function):
    @staticmethod
    def forward(ctx, batch, pos, vel, offsets):
        dev = pos.device
        off = offsets.detach().to("cpu", torch.float32).numpy()
        for k in range(batch.num_scenes):
            batch.set_sdf_offset(k, off[k])
        p4, v4 = _pad4(pos), _pad4(vel)
        torch.cuda.synchronize(dev)
        batch.set_state(p4.data_ptr(), v4.data_ptr())
        batch.forward_record()
        op, ov = torch.empty_like(p4), torch.empty_like(v4)
        batch.get_state(op.data_ptr(), ov.data_ptr())
        token = next(_tokens)
        batch._diff_token = token
        ctx.batch = batch
        ctx.token = token
        ctx.save_for_backward(pos.detach(), vel.detach(), offsets.detach())
        return op[:, :3].clone(), ov[:, :3].clone()

    @staticmethod
    def backward(ctx, gpos, gvel):
        batch = ctx.batch
        pos, vel, offsets = ctx.saved_tensors
        dev = pos.device
        if getattr(batch, "_diff_token", None) != ctx.token:  # re-record this step
            off = offsets.to("cpu", torch.float32).numpy()
            for k in range(batch.num_scenes):
                batch.set_sdf_offset(k, off[k])
            p4, v4 = _pad4(pos), _pad4(vel)
            torch.cuda.synchronize(dev)
            batch.set_state(p4.data_ptr(), v4.data_ptr())
            batch.forward_record()
            batch._diff_token = ctx.token
        n = pos.shape[0]
        g4p = torch.zeros((n, 4), dtype=torch.float32, device=dev)
        g4v = torch.zeros((n, 4), dtype=torch.float32, device=dev)
        if gpos is not None:
            g4p[:, :3] = gpos
        if gvel is not None:
            g4v[:, :3] = gvel
        op, ov = torch.empty_like(g4p), torch.empty_like(g4v)
        torch.cuda.synchronize(dev)
        gt = batch.backward(g4p.data_ptr(), g4v.data_ptr(), op.data_ptr(), ov.data_ptr())
        gt_t = torch.from_numpy(np.ascontiguousarray(gt)).to(offsets.device, offsets.dtype)
        return None, op[:, :3].clone(), ov[:, :3].clone(), gt_t


def step(batch, pos, vel, sdf_offsets):
    """One differentiable step of every scene of `batch` (see module doc)."""
    return _Step.apply(batch, pos, vel, sdf_offsets)
