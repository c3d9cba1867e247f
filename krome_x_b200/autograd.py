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

Memory. The tapes take N x tape_cap doubles (256 KB per cell by default:
17 GB for 65,536 cells). With max_tape_bytes set below that, the solve
keeps no tape: the forward is a counting solve (the rate multipliers
applied, each cell's tape length counted, nothing recorded), and the
backward recomputes the tapes from the stored initial states -- the one
checkpoint a cell needs, as every cell is independent -- in chunks of
cells sorted by tape length, each chunk's tapes as long as its longest and
the chunk as large as max_tape_bytes allows, each chunk's reverse sweep
right after its recording. The results and gradients are the same bit for
bit; the cost is one more solve (~3.4 forward solves against ~2.5).
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


def _record(net, opts, n, T, dtv, P, pstride, mult, mstride, flags, cursor,
            tape, cap, tlen, yfin, c0, c1, count=False):
    """the recording solve of cells [c0, c1) (rows of the per-cell arrays;
    broadcast par / mult rows stay whole), in place in n and T; count: no
    tape, tlen gets the length each cell's tape needs"""
    stream = torch.cuda.current_stream(n.device).cuda_stream
    neq = yfin.numel() // max(int(n.shape[0]), 1) if c1 > c0 else 0
    r = net._lib.krome_b200_adjoint_record_device(
        c1 - c0, n[c0:c1].data_ptr(), T[c0:c1].data_ptr(),
        dtv[c0:c1].data_ptr(), P[c0:c1].data_ptr() if pstride else P.data_ptr(),
        pstride, mult[c0:c1].data_ptr() if mstride else mult.data_ptr(),
        mstride, flags[c0:c1].data_ptr(), None, cursor.data_ptr(),
        None if count else tape.data_ptr(), cap, tlen[c0:c1].data_ptr(),
        yfin[c0 * neq:c1 * neq].data_ptr(), opts._h, stream)
    if r != 0:
        raise krome.KromeError("adjoint forward: %d (%s)"
                               % (r, net.flag_message(r)))


class _SolveChunked(torch.autograd.Function):
    """the same solve and gradients without keeping the tapes: a counting
    forward, then chunks of length-sorted cells recorded and swept back in
    the backward through one buffer of at most max_bytes"""

    @staticmethod
    def forward(ctx, n0, T0, lnm, dt, par, net, opts, tape_cap, max_bytes):
        N = int(n0.shape[0])
        neq = net.nspec + (1 if opts["evolve_T"] else 0)
        dev = n0.device
        n = n0.detach().to(torch.float64).contiguous().clone()
        T = T0.detach().to(torch.float64).contiguous().clone()
        n0c, T0c = n.clone(), T.clone()
        dtv = dt.detach().to(torch.float64).contiguous()
        P = par.detach().to(torch.float64).contiguous()
        pstride = 0 if P.numel() == net.npar else net.npar
        if pstride:
            P = P.reshape(N, net.npar)
        mult = lnm.detach().to(torch.float64).exp().contiguous()
        mstride = 0 if mult.dim() == 1 else net.nrea
        flags = torch.zeros(N, dtype=torch.int32, device=dev)
        cursor = torch.zeros(1, dtype=torch.int32, device=dev)
        tlen = torch.zeros(N, dtype=torch.int64, device=dev)
        yfin = torch.empty(N * neq, dtype=torch.float64, device=dev)
        # the counting solve: the results, and each cell's tape length
        _record(net, opts, n, T, dtv, P, pstride, mult, mstride, flags,
                cursor, None, 0, tlen, yfin, 0, N, count=True)
        # a cell whose tape would outgrow tape_cap fails as with a tape:
        # -120, its input kept
        over = (flags == 0) & (tlen > tape_cap)
        if bool(over.any()):
            flags[over] = -120
            n[over], T[over] = n0c[over], T0c[over]
        ctx.save_for_backward(n0c, T0c, dtv, P, mult, flags, tlen)
        ctx.net, ctx.opts, ctx.max_bytes = net, opts, max_bytes
        ctx.pstride, ctx.mstride, ctx.neq = pstride, mstride, neq
        ctx.mark_non_differentiable(flags)
        return n, T, flags

    @staticmethod
    def backward(ctx, gn, gT, _gflags):
        n0c, T0c, dtv, P, mult, flags, tlen = ctx.saved_tensors
        net, neq = ctx.net, ctx.neq
        N = int(T0c.shape[0])
        dev = T0c.device
        gn = (torch.zeros(N, net.nspec, dtype=torch.float64, device=dev)
              if gn is None else gn.to(torch.float64).contiguous())
        gT = (torch.zeros(N, dtype=torch.float64, device=dev)
              if gT is None else gT.to(torch.float64).contiguous())
        ps, ms = ctx.pstride, ctx.mstride
        # the cells sorted by tape length; chunks as large as the budget
        # allows with tapes as long as each chunk's longest
        lens = torch.where(flags == 0, tlen, torch.zeros_like(tlen))
        order = torch.argsort(lens)
        sl = lens[order].cpu().tolist()
        budget = max(int(ctx.max_bytes) // 8, 1)
        chunks, c0 = [], 0
        while c0 < N:
            c1 = c0 + 1
            while c1 < N and (c1 + 1 - c0) * max(sl[c1], 1) <= budget:
                c1 += 1
            chunks.append((c0, c1, max(sl[c1 - 1], 1)))
            c0 = c1
        # every per-cell array in the sorted order
        n_s, T_s = n0c[order].contiguous(), T0c[order].contiguous()
        T0_s = T_s.clone()
        dt_s = dtv[order].contiguous()
        P_s = P[order].contiguous() if ps else P
        m_s = mult[order].contiguous() if ms else mult
        gn_s, gT_s = gn[order].contiguous(), gT[order].contiguous()
        dn0 = torch.empty(N, net.nspec, dtype=torch.float64, device=dev)
        dT0 = torch.empty(N, dtype=torch.float64, device=dev)
        dm = torch.empty(N, net.nrea, dtype=torch.float64, device=dev)
        fl = torch.zeros(N, dtype=torch.int32, device=dev)
        cursor = torch.zeros(1, dtype=torch.int32, device=dev)
        tl = torch.zeros(N, dtype=torch.int64, device=dev)
        yfin = torch.empty(N * neq, dtype=torch.float64, device=dev)
        need = max((c1 - c0) * cap for c0, c1, cap in chunks)
        tape = torch.empty(need, dtype=torch.float64, device=dev)
        stream = torch.cuda.current_stream(dev).cuda_stream
        for c0, c1, cap in chunks:
            # the chunk's tapes again, from its cells' initial states
            _record(net, ctx.opts, n_s, T_s, dt_s, P_s, ps, m_s, ms, fl,
                    cursor, tape, cap, tl, yfin, c0, c1)
            r = net._lib.krome_b200_adjoint_device(
                c1 - c0, T0_s[c0:c1].data_ptr(),
                P_s[c0:c1].data_ptr() if ps else P_s.data_ptr(), ps,
                m_s[c0:c1].data_ptr() if ms else m_s.data_ptr(), ms,
                gn_s[c0:c1].data_ptr(), gT_s[c0:c1].data_ptr(),
                fl[c0:c1].data_ptr(), tape.data_ptr(), cap,
                tl[c0:c1].data_ptr(), yfin[c0 * neq:c1 * neq].data_ptr(),
                dn0[c0:c1].data_ptr(), dT0[c0:c1].data_ptr(),
                dm[c0:c1].data_ptr(), cursor.data_ptr(), ctx.opts._h, stream)
            if r != 0:
                raise krome.KromeError("adjoint backward: %d" % r)
        # back to the caller's order
        inv = torch.empty_like(order)
        inv[order] = torch.arange(N, device=dev)
        dn0, dT0, dm = dn0[inv], dT0[inv], dm[inv]
        dlnm = dm if ms else dm.sum(0)
        return dn0, dT0, dlnm, None, None, None, None, None, None


def solve(net, n0, T0, lnm, dt, par, opts=None, tape_cap=DEFAULT_TAPE_CAP,
          max_tape_bytes=None):
    """(n, Tgas, flags) after dt, differentiable in n0, T0 and lnm;
    max_tape_bytes bounds the device memory of the tapes (the backward then
    recomputes them chunk by chunk)"""
    opts = net._options(opts)
    # the required-parameter rule, checked before any work
    row = par.detach().cpu().numpy().reshape(-1, net.npar)
    net._params(row if row.shape[0] > 1 else row[0], int(n0.shape[0]))
    N = int(n0.shape[0])
    cap = int(tape_cap)
    if max_tape_bytes is not None and N * cap * 8 > max_tape_bytes:
        return _SolveChunked.apply(n0, T0, lnm, dt, par, net, opts, cap,
                                   int(max_tape_bytes))
    return _Solve.apply(n0, T0, lnm, dt, par, net, opts, cap)
