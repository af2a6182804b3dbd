"""Lock-step comparison of the CUDA path (through the C ABI) with the oracle."""
import math

import numpy as np

from imex_sflow2d_v2_b200.solver import ImexSolver
from oracle import Oracle


def rel_l1(a, b):
    den = np.abs(a).sum()
    return float(np.abs(a - b).sum() / den) if den > 0 else float(np.abs(a - b).sum())


def lockstep(p, st, q, nsteps, erosion=False, threads=8, mass=False):
    """Runs check_solve / timestep / imex_RK_solver (/ erosion) step by step on
    both sides with the oracle's dt.  Returns per-step records; with `mass`
    each record carries the relative residual of the mass budget of the GPU
    state (the oracle's border/inlet face fluxes, fixes and exchange)."""
    o = Oracle(p, st, threads=threads)
    o.set_state(q, 0.0)
    g = ImexSolver(p, st)
    g.set_state(q, 0.0)
    t = 0.0
    recs = []
    m0 = math.fsum(np.asarray(q[0]).ravel().tolist()) if mass else 0.0
    for s in range(nsteps):
        n_o = o.check_solve(t)
        n_g = g.check_solve(t)
        mo, mg = o.get_masks(), g.get_masks()
        dto = o.timestep()
        dtg = g.timestep()
        eo = o.rk_step(t, dto)
        eg = g.imex_RK_solver(t, dto)
        if erosion:
            eo |= o.erosion_deposition(dto)
            eg2 = g.update_erosion_deposition_cell(dto)
            eg = eg or eg2
        o.post_step()
        so, sg = o.stats(), g.stats()
        errs = ((so.error_mask, so.first_error_code, so.first_error_j, so.first_error_k),
                (sg.error_mask, sg.first_error_code, sg.first_error_j, sg.first_error_k))
        qo, qg = o.get_state(), g.get_state()
        recs.append(dict(step=s, cells=(n_o, n_g),
                         mask_equal=all(np.array_equal(a, b) for a, b in zip(mo, mg)),
                         dt=(dto, dtg), q_equal=bool(np.array_equal(qo, qg)),
                         rel_l1=rel_l1(qo, qg), err=errs, stale=o.stale_wet_reads()))
        if mass:
            b = o.mass_budget()
            m = math.fsum(qg[0].ravel().tolist())
            recs[-1]["mass_resid"] = (m - m0 - b[0] - b[1] - b[2]) / max(abs(m), 1e-300)
        t = t + dto
    return recs, o, g
