"""TEST INFRASTRUCTURE ONLY: a second, independent restatement of the
reference's point functions in numpy, written from the Fortran source
without reference to the C++ oracle, to cross-check the oracle.

Covered (the branches the workloads reach: gas carrier, no liquid, no
additional gas, no stochastic or pore-pressure variables, no vertical
profiles):
  mixt_var             src/constitutive_2d.f90:1333-1483
  r_phys_var/qc_to_qp  src/constitutive_2d.f90:541-967, 1628-1681
  qp_to_qc             src/constitutive_2d.f90:1709-2140
  eval_local_speeds_x/y src/constitutive_2d.f90:2194-2298
  eval_fluxes          src/constitutive_2d.f90:2316-2509
  one KT interface     src/solver_2d.f90:2862-2923 (x), 2932-2990 (y),
                       average_KT :3017-3047
  Voellmy implicit terms (real arithmetic)
                       src/constitutive_2d.f90:1145-1313 (c_phys_var),
                       3327-3497, 3806-3818

Every expression keeps the Fortran evaluation order (left to right,
parentheses kept, x**2 = x*x, x**4 = (x*x)*(x*x), SUM and DOT_PRODUCT as
sequential sums from 0).  numpy rounds each elementwise operation once, so
the results can be compared with the oracle bit for bit.  States are
columns: arrays of shape (n_vars, N) or (n_vars+2, N).
"""
import numpy as np

EPS = np.finfo(np.float64).eps


class Consts:
    """The module constants the routines read (from an ImexParams)."""

    def __init__(self, p):
        self.ns = p.n_solid
        self.nv = 4 + self.ns
        self.alpha_flag = bool(p.alpha_flag)
        self.energy_flag = bool(p.energy_flag)
        self.slope_correction = bool(p.slope_correction_flag)
        self.pres = p.pres
        self.Ra = p.sp_gas_const_a
        self.cpa = p.sp_heat_a
        self.T_amb = p.T_ambient
        self.grav = p.grav
        self.xi = p.xi
        self.rho_s = [p.rho_s[i] for i in range(self.ns)]
        self.cps = [p.sp_heat_s[i] for i in range(self.ns)]
        # src/inpout_2d.f90:1330,1353,1882; src/geometry_2d.f90:286-290
        self.inv_pres = 1.0 / self.pres
        self.rho_a_amb = self.pres / (self.Ra * self.T_amb)
        self.inv_rho_s = [1.0 / r for r in self.rho_s]
        self.eps_sing = p.eps_sing
        self.eps_sing4 = (p.eps_sing * p.eps_sing) * (p.eps_sing * p.eps_sing)


def _seqsum(terms):
    s = 0.0
    for t in terms:
        s = s + t
    return s


def mixt_var(K, qp):
    """(Ri, rho_m, rho_c, red_grav)."""
    h = qp[0]
    dry = h <= EPS
    hs = np.where(dry, 1.0, h)
    u, v, T = qp[K.nv], qp[K.nv + 1], np.where(dry, K.T_amb, qp[3])
    if K.alpha_flag:
        al = [qp[4 + i] for i in range(K.ns)]
    else:
        al = [qp[4 + i] / hs for i in range(K.ns)]
    at = _seqsum(al)
    rho_a = K.pres / (K.Ra * T)
    # ((1 - alphal - alphas_tot - SUM(alphag)) * rho_a + DOT(alphag, rho_g)) /
    # (1 - alphal - alphas_tot), alphal = 0, no additional gas
    rho_c = ((((1.0 - 0.0) - at) - 0.0) * rho_a + 0.0) / ((1.0 - 0.0) - at)
    rho_m = (1.0 - at) * rho_c + _seqsum(al[i] * K.rho_s[i] for i in range(K.ns))
    red_grav = (rho_m - K.rho_a_amb) / rho_m * K.grav
    vel2 = u * u + v * v
    with np.errstate(divide="ignore", invalid="ignore"):
        Ri = np.where(vel2 > 0.0, np.minimum(1.0e15, red_grav * h / np.where(vel2 > 0, vel2, 1.0)),
                      0.0)
    Ri = np.where(dry, 0.0, Ri)
    rho_m = np.where(dry, K.rho_a_amb, rho_m)
    rho_c = np.where(dry, K.rho_a_amb, rho_c)
    red_grav = np.where(dry, 0.0, red_grav)
    return Ri, rho_m, rho_c, red_grav


def qc_to_qp(K, qc):
    """r_phys_var + qc_to_qp: physical variables (n_vars+2, N)."""
    q1 = qc[0]
    wet = q1 > EPS
    inv = 1.0 / np.where(wet, q1, 1.0)
    xs = [qc[4 + i] * inv for i in range(K.ns)]
    same = _seqsum(qc[4 + i] for i in range(K.ns)) == q1
    xsum = _seqsum(xs)
    with np.errstate(divide="ignore", invalid="ignore"):
        xs = [np.where(same, x / xsum, x) for x in xs]
    xs_tot = _seqsum(xs)
    xc = 1.0 - xs_tot
    cp_c_by_xc = (xc - 0.0) * K.cpa + 0.0
    cp_mix = _seqsum(xs[i] * K.cps[i] for i in range(K.ns)) + cp_c_by_xc
    big = q1 > K.eps_sing
    with np.errstate(divide="ignore", invalid="ignore"):
        if K.energy_flag:
            T = (qc[3] - 0.5 * (qc[1] * qc[1] + qc[2] * qc[2]) * inv) / (q1 * cp_mix)
        else:
            T = qc[3] / (q1 * cp_mix)
    T = np.where(big, np.where(T <= 0.0, K.T_amb, T), K.T_amb)
    with np.errstate(divide="ignore", invalid="ignore"):
        Rc = np.where(xc > EPS, ((xc - 0.0) * K.Ra + 0.0) / xc, K.Ra)
    inv_rho_c = Rc * T * K.inv_pres
    inv_rhom = _seqsum(xs[i] * K.inv_rho_s[i] for i in range(K.ns)) + xc * inv_rho_c
    rho_m = 1.0 / inv_rhom
    alphas = [xs[i] * rho_m * K.inv_rho_s[i] for i in range(K.ns)]
    h = q1 * inv_rhom
    with np.errstate(divide="ignore", invalid="ignore"):
        den = np.sqrt((q1 * q1) * (q1 * q1) + K.eps_sing4)
        u = np.where(big, qc[1] * inv, np.sqrt(2.0) * q1 * qc[1] / den)
        v = np.where(big, qc[2] * inv, np.sqrt(2.0) * q1 * qc[2] / den)
    qp = np.empty((K.nv + 2,) + q1.shape)
    qp[0] = h
    qp[1] = h * u
    qp[2] = h * v
    qp[3] = T
    for i in range(K.ns):
        qp[4 + i] = alphas[i] if K.alpha_flag else alphas[i] * h
    qp[K.nv] = u
    qp[K.nv + 1] = v
    dry = ~wet
    qp[:, dry] = 0.0
    qp[3, dry] = K.T_amb
    return qp


def qp_to_qc(K, qp):
    h = qp[0]
    wet = h > EPS
    hs = np.where(wet, h, 1.0)
    hu, hv, u, v, T = qp[1], qp[2], qp[K.nv], qp[K.nv + 1], qp[3]
    if K.alpha_flag:
        al = [qp[4 + i] for i in range(K.ns)]
    else:
        al = [qp[4 + i] / hs for i in range(K.ns)]
    at = _seqsum(al)
    ars = [al[i] * K.rho_s[i] for i in range(K.ns)]
    with np.errstate(divide="ignore", invalid="ignore"):
        rho_a = K.pres / (K.Ra * T)
        rho_c = ((((1.0 - 0.0) - at) - 0.0) * rho_a + 0.0) / ((1.0 - 0.0) - at)
    # the volume-fraction corrections (at > 1, at < 0) change r_alphas only,
    # which nothing below reads: alphas_tot and alphas*rho_s are used as
    # computed above
    ac = 1.0 - at
    rho_m = ac * rho_c + _seqsum(ars)
    inv_rhom = 1.0 / rho_m
    xs = [ars[i] * inv_rhom for i in range(K.ns)]
    xc = ac * rho_c * inv_rhom
    with np.errstate(divide="ignore", invalid="ignore"):
        cp_c = np.where(xc > EPS, ((xc - 0.0) * K.cpa + 0.0) / xc, K.cpa)
    cp_mix = _seqsum(xs[i] * K.cps[i] for i in range(K.ns)) + xc * cp_c
    qc = np.empty((K.nv,) + h.shape)
    qc[0] = rho_m * h
    qc[1] = rho_m * hu
    qc[2] = rho_m * hv
    if K.energy_flag:
        qc[3] = np.where(h > 0.0, h * rho_m * (cp_mix * T + 0.5 * (u * u + v * v)), 0.0)
    else:
        qc[3] = h * rho_m * cp_mix * T
    for i in range(K.ns):
        qc[4 + i] = xs[i] * qc[0]
    qc[:, ~wet] = 0.0
    return qc


def local_speeds(K, qp, gcf, d):
    """eval_local_speeds_x (d = 1) / _y (d = 2): (vel_min, vel_max)."""
    _, _, _, red_grav = mixt_var(K, qp)
    h = qp[0]
    w = qp[K.nv] if d == 1 else qp[K.nv + 1]
    neg = red_grav * h < 0.0
    with np.errstate(invalid="ignore"):
        if d == 1:
            c = np.sqrt(red_grav * h * gcf)
        else:
            c = np.sqrt(gcf * red_grav * h)
    return np.where(neg, w, w - c), np.where(neg, w, w + c)


def eval_fluxes(K, qc, qp, gcf, d):
    h = qp[0]
    wet = h > EPS
    u, v = qp[K.nv], qp[K.nv + 1]
    _, rho_m, _, red_grav = mixt_var(K, qp)
    w = u if d == 1 else v
    press = 0.5 * rho_m * gcf * red_grav * (h * h)
    f = np.empty_like(qc)
    f[0] = w * qc[0]
    if d == 1:
        f[1] = w * qc[1] + press
        f[2] = w * qc[2]
    else:
        f[1] = w * qc[1]
        f[2] = w * qc[2] + press
    f[3] = w * (qc[3] + press) if K.energy_flag else w * qc[3]
    for i in range(K.ns):
        f[4 + i] = w * qc[4 + i]
    s = _seqsum(f[4 + i] for i in range(K.ns))
    with np.errstate(divide="ignore", invalid="ignore"):
        cap = (f[0] > 0.0) & (s / f[0] > 1.0)
        for i in range(K.ns):
            f[4 + i] = np.where(cap, f[4 + i] / s * f[0], f[4 + i])
    f[:, ~wet] = 0.0
    return f


def kt_interface(K, qcL, qpL, qcR, qpR, gcf, d):
    """H of one interface and (a-, a+)."""
    lmin, lmax = local_speeds(K, qpL, gcf, d)
    rmin, rmax = local_speeds(K, qpR, gcf, d)
    aN = np.minimum(np.minimum(lmin, rmin), 0.0)
    aP = np.maximum(np.maximum(lmax, rmax), 0.0)
    fL = eval_fluxes(K, qcL, qpL, gcf, d)
    fR = eval_fluxes(K, qcR, qpR, gcf, d)
    same = aN == aP
    den = np.where(same, 1.0, aP - aN)
    H = np.empty_like(qcL)
    for i in range(K.nv):
        avg = (aP * fL[i] - aN * fR[i]) / den
        H[i] = np.where(same, 0.0, avg + (aP * aN) / den * (qcR[i] - qcL[i]))
    s = _seqsum(H[4 + i] for i in range(K.ns))
    with np.errstate(divide="ignore", invalid="ignore"):
        if d == 1:
            cap = s / H[0] >= 1.0
            r = _seqsum(H[4 + i] / H[0] for i in range(K.ns))
            for i in range(K.ns):
                H[4 + i] = np.where(cap, H[4 + i] / r, H[4 + i])
            zero = (qpL[1] == 0.0) & (qpR[1] == 0.0)
        else:
            cap = s / H[0] > 1.0
            r = s / H[0]
            for i in range(K.ns):
                H[4 + i] = np.where(cap, H[4 + i] / r, H[4 + i])
            zero = (qcL[2] == 0.0) & (qcR[2] == 0.0)
    H[0] = np.where(zero, 0.0, H[0])
    for i in range(3, K.nv):
        H[i] = np.where(zero, 0.0, H[i])
    return H, aN, aP


def voellmy_implicit(K, q, bx=0.0, by=0.0):
    """Real part of eval_implicit_terms for the Voellmy-Salm model with
    real input (zero imaginary parts): (n_vars, N)."""
    q1 = q[0]
    wet = q1 > EPS
    inv = 1.0 / np.where(wet, q1, 1.0)
    xs = [q[4 + i] * inv for i in range(K.ns)]
    xs_tot = _seqsum(xs)
    xc = 1.0 - xs_tot
    with np.errstate(divide="ignore", invalid="ignore"):
        cp_c = ((xc - 0.0) * K.cpa + 0.0) / xc
        cp_mix = _seqsum(xs[i] * K.cps[i] for i in range(K.ns)) + xc * cp_c
        big = q1 > K.eps_sing
        if K.energy_flag:
            T = (q[3] - 0.5 * (q[1] * q[1] + q[2] * q[2]) * inv) / (q1 * cp_mix)
        else:
            T = q[3] / (q1 * cp_mix)
        T = np.where(big, np.where(T <= 0.0, K.T_amb, T), K.T_amb)
        Rc = ((xc - 0.0) * K.Ra + 0.0) / xc
        inv_rho_c = Rc * T * K.inv_pres
        inv_rhom = _seqsum(xs[i] * K.inv_rho_s[i] for i in range(K.ns)) + xc * inv_rho_c
        rho_m = 1.0 / inv_rhom
        den = np.sqrt((q1 * q1) * (q1 * q1) + K.eps_sing4)
        u = np.where(big, q[1] * inv, np.sqrt(2.0) * q1 * q[1] / den)
        v = np.where(big, q[2] * inv, np.sqrt(2.0) * q1 * q[2] / den)
    u = np.where(wet, u, 0.0)
    v = np.where(wet, v, 0.0)
    rho_m = np.where(wet, rho_m, K.rho_a_amb)
    red_grav = (rho_m - K.rho_a_amb) / rho_m * K.grav
    w = (u * bx + v * by) if K.slope_correction else 0.0
    mod_vel2 = u * u + v * v + w * w
    mod_vel = np.sqrt(mod_vel2)
    nh = np.zeros_like(q)
    moving = mod_vel != 0.0
    mv = np.where(moving, mod_vel, 1.0)
    ts = rho_m * red_grav / K.xi * mod_vel2
    nh[1] = np.where(moving, 0.0 - ts * (u / mv), 0.0)
    nh[2] = np.where(moving, 0.0 - ts * (v / mv), 0.0)
    return nh
