"""CG-SENSE with the coils of one problem split across ranks.

``qpwls_pcg1_coil_sharded`` runs the iteration of wls/qpwls_pcg1.m:94-189
(Fletcher-Reeves directions, real step) for the SENSE system of
systems/Asense.m:53-56 when each rank holds only some of the coils: rank r
applies A_r x = [G (s_c .* x)]_{c in its coils} and A_r' and keeps its own
rows of the data; the image, the direction and the regulariser are
replicated.  The only exchange is one all-reduce per iteration (a SUM over
``torch.distributed``, NCCL between GPUs): the rank's part of A'W(A ddir)
packed with its part of the data-domain inner product <A ddir, W A ddir>,
both in FP64 -- the image-size vector and the scalar that the coil sum
needs (qpwls_pcg1.m:145 forms A'(W (yi - Ax)) from all coils, :163 the
denominator's data term).

The reference recomputes ngrad = A'(W (yi - Ax)) - R x every iteration from
the running Ax (:145, :166).  Here g = A'(W (yi - Ax)) runs alongside x, and
g <- g - step A'(W A ddir) uses the same all-reduce as the denominator, so an
iteration needs one collective instead of two; by linearity of A' the two
are the same iterates up to rounding.  Every rank takes the same steps from
the same replicated quantities, so the iterates agree on all ranks.

The system object needs forward(x) -> this rank's data rows, adjoint(r) ->
the image summed over this rank's coils, and reg(x) -> the regulariser's
gradient R x (image domain, not split).  torch tensors; the images are
complex (complex64 on the GPU, complex128 in FP64 tests).
"""
from __future__ import annotations

import torch


def _dot(a, b) -> torch.Tensor:
    """Re <a, b> in FP64 (a FP64 scalar tensor on a's device)."""
    return torch.vdot(a.reshape(-1).to(torch.complex128), b.reshape(-1).to(torch.complex128)).real


def qpwls_pcg1_coil_sharded(x, A, yi, niter, W=None, precon=None, group=None, iterates=False):
    """niter iterations of qpwls_pcg1 from x with this rank's coils of the
    system A and data yi (rows [M, C_rank]); W: data weights [M] or None;
    precon: a function of the gradient image or None.  group: the process
    group whose ranks share the problem (None: the default group, or no
    exchange when torch.distributed is not initialised).  Returns x, or with
    iterates=True the list [x_0, ..., x_niter]."""
    dist = torch.distributed
    sharded = dist.is_available() and dist.is_initialized() and dist.get_world_size(group) > 1

    def allreduce_(buf):
        if sharded:
            dist.all_reduce(buf, op=dist.ReduceOp.SUM, group=group)
        return buf

    def weight(r):
        return r if W is None else r * W.reshape(-1, *([1] * (r.dim() - 1)))

    x = x.clone()
    shape = x.shape
    n = x.numel()
    cdt = x.dtype
    # g = A'(W (yi - A x)) over all coils: one all-reduce before the loop
    g = A.adjoint(weight(yi - A.forward(x)))
    gbuf = allreduce_(torch.view_as_real(g.reshape(-1).to(torch.complex128)).reshape(-1).clone())
    g = torch.view_as_complex(gbuf.reshape(-1, 2)).reshape(shape)
    Rx = A.reg(x).to(torch.complex128)
    xs = [x.clone()] if iterates else None
    ddir = None
    oldinprod = 0.0
    for it in range(1, niter + 1):
        ngrad = g - Rx
        pregrad = ngrad if precon is None else precon(ngrad.to(cdt)).to(torch.complex128)
        newinprod = float(_dot(ngrad, pregrad))
        if it == 1:
            ddir = pregrad
        else:
            gamma = 0.0 if oldinprod == 0 else newinprod / oldinprod
            ddir = pregrad + gamma * ddir
        oldinprod = newinprod
        ddir_c = ddir.to(cdt)
        Adir = A.forward(ddir_c)
        WAdir = weight(Adir)
        # the iteration's one exchange: [this rank's A'(W A ddir), <A ddir, W A ddir>]
        part = A.adjoint(WAdir).reshape(-1).to(torch.complex128)
        buf = torch.empty(2 * n + 1, dtype=torch.float64, device=part.device)
        buf[:2 * n] = torch.view_as_real(part).reshape(-1)
        buf[2 * n] = _dot(Adir, WAdir)
        allreduce_(buf)
        AtWAdir = torch.view_as_complex(buf[:2 * n].reshape(-1, 2)).reshape(shape)
        Rdir = A.reg(ddir_c).to(torch.complex128)
        denom = float(buf[2 * n]) + float(_dot(ddir, Rdir))
        step = 0.0 if denom == 0 else float(_dot(ddir, ngrad)) / denom
        x = (x.to(torch.complex128) + step * ddir).to(cdt)
        Rx = Rx + step * Rdir
        g = g - step * AtWAdir
        if iterates:
            xs.append(x.clone())
    return xs if iterates else x
