"""The discrete adjoint of the batched solve behind torch.autograd.

    from krome_x_b200 import krome, autograd
    net = krome.load("primordial")
    n, T, flags = autograd.solve(net, n0, T0, lnm, dt, par, opts)
    loss = (n[:, iH2] / nH).sum() + T.sum()
    loss.backward()        # n0.grad, T0.grad, lnm.grad

n0[N, nspec], T0[N], lnm ([nrea] shared by every cell, or [N, nrea]), dt[N]
and par (one row or [N, npar]) are float64 CUDA tensors. The forward is the
lane-per-cell solve with every rate coefficient multiplied by exp(lnm),
recording each cell's tape of Nordsieck operations on the device
(krome_b200_adjoint_record_device); the backward is the reverse sweep over
the tapes (krome_b200_adjoint_device), one lane per cell. Both run on the
current torch stream. A cell that fails (flags != 0, including -120 when
its tape outgrows tape_cap doubles) gets zero gradients and keeps its
inputs. The gradients are those of the discrete solution: the step sizes,
orders and Newton decisions of the forward solve are held fixed.
"""
import torch

from . import krome

DEFAULT_TAPE_CAP = 32768


class _Solve(torch.autograd.Function):
    @staticmethod
    def forward(ctx, n0, T0, lnm, dt, par, net, opts, tape_cap):
        lib = net._lib
        N = int(n0.shape[0])
        neq = net.nspec + (1 if opts["evolve_T"] else 0)
        dev = n0.device
        n = n0.detach().to(torch.float64).contiguous().clone()
        T = T0.detach().to(torch.float64).contiguous().clone()
        T0c = T.clone()
        dtv = dt.detach().to(torch.float64).contiguous()
        P = par.detach().to(torch.float64).contiguous()
        pstride = 0 if P.numel() == net.npar else net.npar
        mult = lnm.detach().to(torch.float64).exp().contiguous()
        mstride = 0 if mult.dim() == 1 else net.nrea
        flags = torch.zeros(N, dtype=torch.int32, device=dev)
        cursor = torch.zeros(1, dtype=torch.int32, device=dev)
        tape = torch.empty(N * tape_cap, dtype=torch.float64, device=dev)
        tlen = torch.zeros(N, dtype=torch.int64, device=dev)
        yfin = torch.empty(N * neq, dtype=torch.float64, device=dev)
        stream = torch.cuda.current_stream(dev).cuda_stream
        r = lib.krome_b200_adjoint_record_device(
            N, n.data_ptr(), T.data_ptr(), dtv.data_ptr(), P.data_ptr(),
            pstride, mult.data_ptr(), mstride, flags.data_ptr(), None,
            cursor.data_ptr(), tape.data_ptr(), tape_cap, tlen.data_ptr(),
            yfin.data_ptr(), opts._h, stream)
        if r != 0:
            raise krome.KromeError("adjoint forward: %d (%s)"
                                   % (r, net.flag_message(r)))
        ctx.save_for_backward(T0c, P, mult, flags, tape, tlen, yfin, cursor)
        ctx.net, ctx.opts, ctx.cap = net, opts, tape_cap
        ctx.pstride, ctx.mstride = pstride, mstride
        ctx.mark_non_differentiable(flags)
        return n, T, flags

    @staticmethod
    def backward(ctx, gn, gT, _gflags):
        T0c, P, mult, flags, tape, tlen, yfin, cursor = ctx.saved_tensors
        net = ctx.net
        N = int(T0c.shape[0])
        dev = T0c.device
        gn = (torch.zeros(N, net.nspec, dtype=torch.float64, device=dev)
              if gn is None else gn.to(torch.float64).contiguous())
        gT = (torch.zeros(N, dtype=torch.float64, device=dev)
              if gT is None else gT.to(torch.float64).contiguous())
        dn0 = torch.empty(N, net.nspec, dtype=torch.float64, device=dev)
        dT0 = torch.empty(N, dtype=torch.float64, device=dev)
        dm = torch.empty(N, net.nrea, dtype=torch.float64, device=dev)
        stream = torch.cuda.current_stream(dev).cuda_stream
        r = net._lib.krome_b200_adjoint_device(
            N, T0c.data_ptr(), P.data_ptr(), ctx.pstride, mult.data_ptr(),
            ctx.mstride, gn.data_ptr(), gT.data_ptr(), flags.data_ptr(),
            tape.data_ptr(), ctx.cap, tlen.data_ptr(), yfin.data_ptr(),
            dn0.data_ptr(), dT0.data_ptr(), dm.data_ptr(), cursor.data_ptr(),
            ctx.opts._h, stream)
        if r != 0:
            raise krome.KromeError("adjoint backward: %d" % r)
        dlnm = dm if ctx.mstride else dm.sum(0)
        return dn0, dT0, dlnm, None, None, None, None, None


def solve(net, n0, T0, lnm, dt, par, opts=None, tape_cap=DEFAULT_TAPE_CAP):
    """(n, Tgas, flags) after dt, differentiable in n0, T0 and lnm"""
    opts = net._options(opts)
    # the required-parameter rule, checked before any work
    row = par.detach().cpu().numpy().reshape(-1, net.npar)
    net._params(row if row.shape[0] > 1 else row[0], int(n0.shape[0]))
    return _Solve.apply(n0, T0, lnm, dt, par, net, opts, int(tape_cap))
