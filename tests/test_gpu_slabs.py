"""Two z slabs of one periodic box on one GPU, exchanging their interface
ghosts through the library's exchange hook (stx_set_exchange at
STX_BC_EXCHANGE faces, the hook the NCCL z-slab decomposition uses), against
the same box run whole.

Each slab is a Solver driven by its own host thread, as an MPI rank drives its
GPU in the reference; the hook of each slab waits for the other at every swap
(a barrier with a timeout, so a mismatch fails instead of hanging), then copies
the neighbour's top / bottom ng interior planes into its ghosts and waits again
before either slab goes on.  Unlike the one-rank test of the hook, the field
here is not the same on both sides of an interface, so the exchange must move
the right planes to the right ghosts in every swap of the step (conserved
variables, Ducros sensor, div/3).

The reference's swaps send only the interior (i, j) columns of a ghost plane
(bcswap, base_gpu.F90:1132-1196); the x / y ghost edges of the z ghost planes
are exchanged only with immersed boundaries on (bcswap_edges_corners,
multideal_gpu.F90:573-577), yet the viscous fluxes at the first face read them.
A decomposed run therefore differs from the whole box at those edges, in the
reference as here: at an interior interface the whole box has live x / y
ghosts (its periodic x and y swaps fill them), at the periodic wrap it has
never-exchanged ones.  Likewise the temperature at a ghost point comes from
eval_aux there, whose Newton iteration starts from that point's previous
result: a ghost point's history of evaluations differs from an interior
point's (the central-only compute_aux of every step skips ghosts), so its last
bits can too.  To compare bit for bit, the hook gives each slab exactly the
ghosts the whole box sees: across the interior interface the whole plane, x / y
ghosts included (the neighbour's own x and y swaps of the same call have filled
them), and with the conserved variables the neighbour's temperature there (the
Newton guess of the interior points it stands for); across the wrap only the
interior columns."""
import threading

import numpy as np
import pytest
import torch

import helpers as H

pytestmark = pytest.mark.gpu
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

from stx import dist as D  # noqa: E402
from stx.native import EXCHANGE_FN, check  # noqa: E402
from stx.solver import Solver  # noqa: E402

NX, NY, NZ, STEPS = 16, 12, 20, 3


def full_case():
    # periodic in every direction; fixed dt so that both runs take the same steps
    return H.synthetic_case(n=(NX, NY, NZ), seed=41, L=(0.01, 0.008, 0.012), T0=1250.0, amp_T=180.0, amp_u=80.0,
                            cfl=-4e-9)


def slab_case(k0, k1):
    """The box's cells k0..k1 (1-based) as a z slab with exchange faces."""
    full = full_case()
    c = H.synthetic_case(n=(NX, NY, k1 - k0 + 1), seed=41, L=(0.01, 0.008, 0.012 * (k1 - k0 + 1) / NZ),
                         T0=1250.0, amp_T=180.0, amp_u=80.0, cfl=-4e-9)
    ng = c.ng
    c.w[:] = full.w[:, k0 - 1:k1 + 2 * ng, :, :]
    c.w_aux[:] = full.w_aux[:, k0 - 1:k1 + 2 * ng, :, :]
    # the whole box's z coordinates and metrics of these planes: a slab's own
    # grid starts at z = 0, and its finite-difference metrics then round
    # differently from the box's in the last bit
    assert np.allclose(c.dzitdz, full.dzitdz[k0 - 1:k1])
    c.z[:] = full.z[k0 - 1:k1 + 2 * ng]
    c.dzitdz[:] = full.dzitdz[k0 - 1:k1]
    c.dzitdzs[:] = full.dzitdzs[k0 - 1:k1]
    return D.make_z_slab(c)


class PairExchange:
    """The exchange hook of slab `me` of two slabs on one GPU."""

    def __init__(self, sols, me, barrier):
        self.sols, self.me, self.bar = sols, me, barrier
        self._fn = EXCHANGE_FN(self._call)
        self.calls = 0
        self.error = None

    def _view(self, s, ptr, nvar):
        base = s.w_aux if s.w_aux.data_ptr() <= ptr < s.w_aux.data_ptr() + s.w_aux.numel() * 8 else s.w
        first = (ptr - base.data_ptr()) // (8 * base[0].numel())
        return base, first

    def _call(self, user, stream, field, nvar):
        try:
            s, o = self.sols[self.me], self.sols[1 - self.me]
            base, first = self._view(s, int(field), int(nvar))
            F = base[first:first + int(nvar)]
            G = (o.w_aux if base is s.w_aux else o.w)[first:first + int(nvar)]
            ng = s.case.ng
            nz = s.case.nz
            interior = (slice(ng, ng + s.case.ny), slice(ng, ng + s.case.nx))
            whole = (slice(None), slice(None))
            # slab 0 is the lower half: its bottom faces the wrap, its top the
            # interior interface; slab 1 the other way round
            lo_ij, hi_ij = (interior, whole) if self.me == 0 else (whole, interior)
            torch.cuda.synchronize()
            self.bar.wait()                      # both slabs' fields are current
            # the periodic pair: each slab's neighbour below and above is the other slab
            lo = G[(slice(None), slice(G.shape[1] - 2 * ng, G.shape[1] - ng)) + lo_ij].clone()
            hi = G[(slice(None), slice(ng, 2 * ng)) + hi_ij].clone()
            F[(slice(None), slice(0, ng)) + lo_ij] = lo
            F[(slice(None), slice(nz + ng, nz + 2 * ng)) + hi_ij] = hi
            if base is s.w:
                # the Newton guess of T across the interior interface (see above)
                jT = s.case.J("T")
                FT, GT = s.w_aux[jT], o.w_aux[jT]
                if self.me == 0:
                    FT[nz + ng:nz + 2 * ng] = GT[ng:2 * ng].clone()
                else:
                    FT[0:ng] = GT[GT.shape[0] - 2 * ng:GT.shape[0] - ng].clone()
            torch.cuda.synchronize()
            self.bar.wait()                      # both have read before either moves on
            self.calls += 1
            return 0
        except Exception as e:
            self.error = e
            self.bar.abort()
            return -2


def test_two_slabs_equal_the_whole_box():
    whole = Solver(full_case())
    whole.prepare()
    for _ in range(STEPS):
        whole.step()
    torch.cuda.synchronize()
    ref_w, ref_wa = whole.case.interior(whole.host_w()), whole.case.interior(whole.host_w_aux())
    whole.close()

    half = NZ // 2
    sols = [Solver(slab_case(1, half)), Solver(slab_case(half + 1, NZ))]
    bar = threading.Barrier(2, timeout=120)
    hooks = [PairExchange(sols, r, bar) for r in range(2)]
    for s, h in zip(sols, hooks):
        check(s.lib.stx_set_exchange(s.ctx, h._fn, None), "stx_set_exchange")
    errors = []

    def rank(r):
        try:
            sols[r].prepare()
            for _ in range(STEPS):
                sols[r].step()
            torch.cuda.synchronize()
        except Exception as e:
            errors.append(e)
            bar.abort()

    th = [threading.Thread(target=rank, args=(r,)) for r in range(2)]
    for t in th:
        t.start()
    for t in th:
        t.join(timeout=600)
    assert not any(t.is_alive() for t in th)
    assert not errors and all(h.error is None for h in hooks), (errors, [h.error for h in hooks])
    assert hooks[0].calls == hooks[1].calls > 0
    got_w = np.concatenate([s.case.interior(s.host_w()) for s in sols], axis=1)
    got_wa = np.concatenate([s.case.interior(s.host_w_aux()) for s in sols], axis=1)
    for s in sols:
        s.close()
    diff = np.argwhere(got_w != ref_w)
    rel = float(np.max(np.abs(got_w - ref_w) / np.maximum(np.abs(ref_w), 1e-300)))
    assert diff.size == 0, f"{len(diff)} values differ (max rel {rel:.3g}), z planes " \
                           f"{sorted(set(diff[:, 1].tolist()))[:10]}"
    assert np.array_equal(got_wa, ref_wa)
