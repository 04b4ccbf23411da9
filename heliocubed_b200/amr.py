"""Two-level synchronous AMR RK4 step of the fourth-order scheme on the
device (CubedSphereAMR::advanceRungeKuttaSynchronous with prepareFourthOrder
and evaluate, src/MHD_AMRRungeKutta.H:5-41, src/MHD_AMRFourthOrder.H:5-100,
src/MHD_AMR.H:1417-1499).

The coarse level covers the shell (a `Shell`); the fine level is a set of
boxes of a `Shell` refined by 2 in every direction.  Per stage, in the
reference's order:

1. stage states of every box of both levels (hc_amr_rk_stage), the fine
   stage restricted onto the coarse cells it covers;
2. the coarse level's stage preparation, keeping its Cartesian averages
   (hc_level_prepare_cartesian);
3. the fine boxes' preparation: donor zeroed, coarse-fine fourth-order
   interpolation of the ghosts from the coarse Cartesian averages
   (hc_amr_cf_interpolate), <JU> of the ghosts (hc_amr_cf_mapped), the
   same-level exchange, <U> of the valid cells (hc_amr_cf_quotient), the
   donor's valid cells and same-level exchange, native averages and radial
   ghosts (hc_amr_native);
4. evaluation: the coarse operator with the panel seams reconciled and its
   face fluxes (hc_level_rhs_fluxes), the fine boxes' operator in one batch
   with their face fluxes (hc_o4_batch_rhs);
5. the coarse-fine flux correction of the coarse cells next to the fine
   boxes (hc_amr_reflux, one launch per face direction and side), the fine
   rhs restricted onto the coarse cells it covers, and the stage rhs kept.

After the fourth stage: the state update of both levels and the fine state
restricted onto the coarse cells it covers (averageDown).

Scope: fine boxes aligned to the refinement (even low, odd high indices),
disjoint, inside one panel with the six donor ghost layers inside it (no
fine panel-seam interpolation is needed), and at least 10 fine cells from
both radial boundaries (every ghost's coarse interpolation stencil inside
the coarse level).  The coarse level is prepared by the uniform level's
Cartesian conversion.  All arrays are allocated when the step is built; the
first step also builds the coarse level's operator batch.
"""
from __future__ import annotations

import numpy as np
import torch

from .level import AmrPlan, O4Batch, Shell, amr_exchange_copies, make_box

RATIO = 2
C4 = (0.0, 0.5, 0.5, 1.0)


def _cells(n) -> int:
    return int(n[0] * n[1] * n[2])


class AmrStep:
    """The device step of one coarse level (whole shell) and one fine level
    of boxes (see the module docstring).  boxes: (panel, lo, hi) in the
    fine level's index space, inclusive."""

    def __init__(self, coarse: Shell, fine: Shell, boxes):
        pc, pf = coarse.params, fine.params
        if pc.spatial_order != 4 or pf.spatial_order != 4:
            raise ValueError("the AMR step is fourth order")
        if pf.nr != RATIO * pc.nr or pf.na != RATIO * pc.na:
            raise ValueError("the fine level refines the coarse one by 2 in every direction")
        self.coarse, self.fine = coarse, fine
        self.boxes = [(int(b), tuple(int(x) for x in lo), tuple(int(x) for x in hi)) for b, lo, hi in boxes]
        nrf, naf = pf.nr, pf.na
        for b, lo, hi in self.boxes:
            if not 0 <= b < 6 or any(lo[d] % RATIO or (hi[d] + 1) % RATIO or hi[d] < lo[d] for d in range(3)):
                raise ValueError(f"box {lo}..{hi} on panel {b}: not aligned to the refinement")
            if lo[0] < 10 or hi[0] > nrf - 11:
                raise ValueError(f"box {lo}..{hi}: closer than 10 fine cells to a radial boundary")
            if any(lo[d] < 6 or hi[d] > naf - 7 for d in (1, 2)):
                raise ValueError(f"box {lo}..{hi}: its donor ghosts would cross a panel edge")
        for a in range(len(self.boxes)):
            for c in range(a):
                (ba, la, ha), (bc, lc, hc) = self.boxes[a], self.boxes[c]
                if ba == bc and all(la[d] <= hc[d] and lc[d] <= ha[d] for d in range(3)):
                    raise ValueError("fine boxes overlap")
        self._alloc()
        self._build()

    # --- storage -------------------------------------------------------
    def _alloc(self) -> None:
        dev = self.fine._dev
        z = lambda n: torch.zeros(int(n), dtype=torch.float64, device=dev)  # noqa: E731
        c = self.coarse
        nv = c.nv // 6
        self.nv_c = nv
        self.state_c = c.new_state()
        self.stage_c = c.new_state()
        self.rk_c = [c.new_state() for _ in range(4)]
        self.k_c = c.new_state()
        self.usph_c = c.new_primitive()
        self.cart_c = z(self.coarse._lib.hc_level_cartesian_size(self.coarse._ctx))
        nr, na = c.params.nr, c.params.na
        self.cflux_n = [(nr + 1, na, na), (nr, na + 1, na), (nr, na, na + 1)]
        self.flux_c = [z(6 * 8 * _cells(n)) for n in self.cflux_n]
        # fine boxes: one contiguous tensor per kind, a view per box
        self.valid_n = [tuple(hi[d] - lo[d] + 1 for d in range(3)) for _, lo, hi in self.boxes]
        grow = lambda n, g: tuple(x + 2 * g for x in n)  # noqa: E731
        kinds = {"state": 0, "stage": 0, "k": 0, "rk0": 0, "rk1": 0, "rk2": 0, "rk3": 0, "out": 0,
                 "mapped": 2, "jac": 3, "usph": 5, "donor": 6}
        self.f = {}
        for kind, g in kinds.items():
            comps = 1 if kind == "jac" else 8
            sizes = [comps * _cells(grow(n, g)) for n in self.valid_n]
            whole = z(sum(sizes))
            views, off = [], 0
            for s in sizes:
                views.append(whole[off:off + s])
                off += s
            self.f[kind] = (whole, views)
        self.fflux = []
        for n in self.valid_n:
            self.fflux.append([z(8 * _cells(tuple(n[e] + (e == d) for e in range(3)))) for d in range(3)])
        self._jacobians()

    def _jacobians(self) -> None:
        """<J> = dVolr(i) <det A>(j, k) of the fine level on valid.grow(3)."""
        fp = self.fine.params
        det = self.fine.geometry(4).reshape(6, fp.na, fp.na)
        vol = self.fine.geometry(0).reshape(fp.nr + 1, 4)[:fp.nr, 3]
        for q, (b, lo, hi) in enumerate(self.boxes):
            i = np.arange(lo[0] - 3, hi[0] + 4)
            j = np.arange(lo[1] - 3, hi[1] + 4)
            k = np.arange(lo[2] - 3, hi[2] + 4)
            jac = det[b][np.ix_(k, j)][:, :, None] * vol[i][None, None, :]
            self.f["jac"][1][q].copy_(torch.from_numpy(np.ascontiguousarray(jac).reshape(-1)))

    def _panel(self, t: torch.Tensor, b: int) -> torch.Tensor:
        return t.view(6, -1)[b]

    # --- plan ----------------------------------------------------------
    def _build(self) -> None:
        c, nf = self.coarse, len(self.boxes)
        nr, na = c.params.nr, c.params.na
        V = lambda kind, q: self.f[kind][1][q]  # noqa: E731
        rk_boxes = [(self._panel(self.state_c, b), self._panel(self.stage_c, b),
                     [self._panel(r, b) for r in self.rk_c]) for b in range(6)]
        rk_boxes += [(V("state", q), V("stage", q), [V(f"rk{s}", q) for s in range(4)]) for q in range(nf)]
        restricts = []
        for fine_kind, coarse_arr in (("stage", self.stage_c), ("k", self.k_c), ("state", self.state_c)):
            for q, (b, lo, hi) in enumerate(self.boxes):
                restricts.append({"fine": V(fine_kind, q), "coarse": self._panel(coarse_arr, b),
                                  "fine_lo": lo, "fine_n": self.valid_n[q], "coarse_lo": (0, 0, 0),
                                  "coarse_n": (nr, na, na), "lo": [x // RATIO for x in lo],
                                  "hi": [x // RATIO for x in hi], "ratio": (RATIO,) * 3})
        self.plan = AmrPlan(self.fine, rk_boxes, restricts)
        self.r_stage, self.r_rhs, self.r_state = (0, nf), (nf, nf), (2 * nf, nf)
        # coarse-fine interpolation of every fine box's donor ghosts
        clo, cn = (0, -6, -6), (nr, na + 12, na + 12)
        self.plan.set_cf_interp([
            {"coarse": self._panel(self.cart_c, b), "fine": V("donor", q), "coarse_lo": clo, "coarse_n": cn,
             "fine_lo": [x - 6 for x in lo], "fine_n": [n + 12 for n in self.valid_n[q]], "valid_lo": lo,
             "valid_hi": hi, "ratio": (RATIO,) * 3, "ncomp": 8} for q, (b, lo, hi) in enumerate(self.boxes)])
        fp = self.fine.params
        block_hi = (fp.nr - 1, fp.na - 1, fp.na - 1)
        g = lambda lo, q, w: ([x - w for x in lo], [n + 2 * w for n in self.valid_n[q]])  # noqa: E731
        fine_boxes = []
        for q, (b, lo, hi) in enumerate(self.boxes):
            jl, jn = g(lo, q, 3)
            dl, dn = g(lo, q, 6)
            ml, mn = g(lo, q, 2)
            fine_boxes.append({"jac": V("jac", q), "donor": V("donor", q), "state": V("stage", q),
                               "mapped": V("mapped", q), "out": V("out", q), "jac_lo": jl, "jac_n": jn,
                               "donor_lo": dl, "donor_n": dn, "state_lo": lo, "state_n": self.valid_n[q],
                               "mapped_lo": ml, "mapped_n": mn, "out_lo": lo, "out_n": self.valid_n[q],
                               "valid_lo": lo, "valid_hi": hi, "block_lo": (0, 0, 0), "block_hi": block_hi})
        self.plan.set_cf_fine(fine_boxes)
        # region copies: the mapped exchange, <U> into the donor's valid
        # cells, the donor exchange
        triples = [(b, lo, hi) for b, lo, hi in self.boxes]
        copies = []

        def exchange(kind, w):
            for cp in amr_exchange_copies(triples, w):
                s, d = cp["src_box"], cp["dst_box"]
                sl, sn = g(self.boxes[s][1], s, w)
                dl2, dn2 = g(self.boxes[d][1], d, w)
                copies.append(dict(cp, src=V(kind, s), dst=V(kind, d), src_lo=sl, src_n=sn, dst_lo=dl2,
                                   dst_n=dn2, ncomp=8))

        exchange("mapped", 2)
        n_mapped = len(copies)
        for q, (b, lo, hi) in enumerate(self.boxes):
            dl, dn = g(lo, q, 6)
            copies.append({"src": V("out", q), "dst": V("donor", q), "src_lo": lo, "src_n": self.valid_n[q],
                           "dst_lo": dl, "dst_n": dn, "lo": lo, "hi": hi, "perm": (0, 1, 2), "sign": (1, 1, 1),
                           "shift": (0, 0, 0), "ncomp": 8})
        n_out = len(copies) - n_mapped
        exchange("donor", 6)
        self.cp_mapped, self.cp_out = (0, n_mapped), (n_mapped, n_out)
        self.cp_donor = (n_mapped + n_out, len(copies) - n_mapped - n_out)
        self.plan.set_copies(copies)
        self.plan.set_native([
            {"cart": V("donor", q), "usph": V("usph", q), "cart_lo": g(lo, q, 6)[0], "cart_n": g(lo, q, 6)[1],
             "usph_lo": g(lo, q, 5)[0], "usph_n": g(lo, q, 5)[1], "block": b}
            for q, (b, lo, hi) in enumerate(self.boxes)])
        # the fine operator: one batch over the boxes, rhs k, face fluxes
        works = [(make_box(lo, hi, 5, b), V("usph", q), V("k", q), self.fflux[q])
                 for q, (b, lo, hi) in enumerate(self.boxes)]
        self.batch = O4Batch(self.fine, works)
        self._reflux_patches()

    def _reflux_patches(self) -> None:
        """Coarse faces between a fine box and an uncovered coarse cell,
        grouped by face direction and side (one launch per group: no coarse
        cell is corrected twice in a launch)."""
        c = self.coarse
        nr, na = c.params.nr, c.params.na
        covered = np.zeros((6, nr, na, na), dtype=bool)
        for b, lo, hi in self.boxes:
            covered[b, lo[0] // 2:hi[0] // 2 + 1, lo[1] // 2:hi[1] // 2 + 1, lo[2] // 2:hi[2] // 2 + 1] = True
        dxi = (nr, na, na)
        groups = {}
        for q, (b, lo, hi) in enumerate(self.boxes):
            clo = [x // 2 for x in lo]
            chi = [x // 2 for x in hi]
            for d in range(3):
                t1, t2 = [e for e in range(3) if e != d]
                for side in (0, 1):
                    # the fine cells are above the face (fine_side 1) at the
                    # box's low face, below it (0) at the high face
                    face = clo[d] if side == 0 else chi[d] + 1
                    cell = face - 1 if side == 0 else face
                    lim = (nr, na, na)[d]
                    if not 0 <= cell < lim:
                        continue
                    for a2 in range(clo[t2], chi[t2] + 1):
                        run = None
                        for a1 in range(clo[t1], chi[t1] + 2):
                            idx = [0, 0, 0]
                            idx[d], idx[t1], idx[t2] = cell, a1, a2
                            free = a1 <= chi[t1] and not covered[b, idx[0], idx[1], idx[2]]
                            if free and run is None:
                                run = a1
                            if not free and run is not None:
                                plo, phi = [0, 0, 0], [0, 0, 0]
                                plo[d] = phi[d] = face
                                plo[t1], phi[t1] = run, a1 - 1
                                plo[t2] = phi[t2] = a2
                                groups.setdefault((d, side), []).append({
                                    "fine_flux": self.fflux[q][d],
                                    "coarse_flux": self._panel(self.flux_c[d], b),
                                    "rhs": self._panel(self.k_c, b),
                                    "fine_lo": lo, "fine_n": tuple(self.valid_n[q][e] + (e == d) for e in range(3)),
                                    "coarse_lo": (0, 0, 0), "coarse_n": self.cflux_n[d],
                                    "rhs_lo": (0, 0, 0), "rhs_n": (nr, na, na), "lo": plo, "hi": phi,
                                    "ratio": (RATIO,) * 3, "dir": d, "fine_side": 1 - side,
                                    "scale": float(dxi[d]), "box": q, "panel": b})
                                run = None
        patches, self.reflux_groups = [], []
        for key in sorted(groups):
            self.reflux_groups.append((len(patches), len(groups[key])))
            patches += groups[key]
        self.patches = patches
        self.plan.set_reflux(patches)

    # --- the step ------------------------------------------------------
    def load(self, ju_coarse: torch.Tensor, fine_states) -> None:
        """Coarse level state (level layout) and each fine box's valid <JU>."""
        self.state_c.copy_(ju_coarse)
        for q, s in enumerate(fine_states):
            self.f["state"][1][q].copy_(s.reshape(-1))

    def fine_state(self, q: int) -> torch.Tensor:
        return self.f["state"][1][q]

    def step(self, dt: float, t: float = 0.0) -> None:
        """One RK4 step of both levels with dt from the host."""
        P = self.plan
        nf = len(self.boxes)
        for s in range(4):
            P.rk_stage(4, s, dt)
            P.restrict(*self.r_stage)
            ts = t + C4[s] * dt
            self.coarse.prepare_cartesian(self.stage_c, ts, self.usph_c, self.cart_c)
            self.f["donor"][0].zero_()
            P.cf_interpolate(0, nf)
            P.cf_mapped(0, nf)
            P.copy(*self.cp_mapped)
            P.cf_quotient(0, nf)
            P.copy(*self.cp_out)
            P.copy(*self.cp_donor)
            P.native(0, nf, ts)
            self.coarse.rhs_fluxes(self.usph_c, self.k_c, self.flux_c)
            self.f["k"][0].zero_()
            self.batch.rhs()
            for first, count in self.reflux_groups:
                P.reflux(first, count)
            P.restrict(*self.r_rhs)
            self.rk_c[s].copy_(self.k_c)
            self.f[f"rk{s}"][0].copy_(self.f["k"][0])
        P.rk_stage(4, 4, dt)
        P.restrict(*self.r_state)

    def close(self) -> None:
        self.batch.close()
        self.plan.close()
