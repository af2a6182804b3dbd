"""Small run set-ups shared by the parity tests (seeded, synthetic)."""
import numpy as np

from imex_sflow2d_v2_b200 import configs


def dambreak(rheology=None, n=40, **kw):
    return configs.dambreak(nx=n, ny=n, dx=0.25, rheology=rheology, **kw)


def dambreak_variants():
    out = {}
    out["dambreak"] = dambreak()
    out["dambreak_voellmy"] = dambreak(rheology=1)
    out["dambreak_quadratic"] = dambreak(rheology=6)
    p, st, q = dambreak(rheology=1)
    p.alpha_flag = 1
    qp = np.zeros((7, p.nx, p.ny))
    _, xc, _, _ = configs.grid(p)
    h = np.where(np.repeat(xc[:, None], p.ny, axis=1) < 5.0, 1.0, 0.1)
    qp[0] = h
    qp[3] = 300.0
    qp[4] = 0.01
    out["dambreak_alpha_flag"] = (p, st, configs.qp_to_qc_grid(p, qp))
    p, st, q = dambreak(rheology=1)
    p.energy_flag = 0
    qp = np.zeros((7, p.nx, p.ny))
    qp[0] = h
    qp[3] = 300.0
    qp[4] = 0.01 * h
    out["dambreak_no_energy"] = (p, st, configs.qp_to_qc_grid(p, qp))
    for lim in (2, 3, 4):
        p, st, q = dambreak(rheology=1)
        for i in range(7):
            p.limiter[i] = lim
        p.theta = 1.3
        out["dambreak_limiter%d" % lim] = (p, st, q)
    p, st, q = dambreak(rheology=1)
    for side in "WESN":  # closed walls: reflective Dirichlet on hu/hv
        configs.set_bc(p, side, 1, 0, 0.0)
        configs.set_bc(p, side, 2, 0, 0.0)
    out["dambreak_dirichlet"] = (p, st, q)
    return out


def sloped(n=48, dx=4.0, rheology=1, slope=True, curvature=True, seed=7):
    """Wet slab on a seeded rough incline with the slope and curvature
    corrections switched on."""
    p = configs.default_params(n, n, 2, dx)
    for i in range(2):
        p.rho_s[i] = 2500.0
        p.diam_s[i] = (1e-4, 1e-3)[i]
        p.sp_heat_s[i] = 1617.0
    p.rheology_flag = 1
    p.rheology_model = rheology
    p.mu, p.xi, p.friction_factor = 0.1, 500.0, 1e-3
    p.max_dt = 1.0
    configs.transmissive_bcs(p)
    B = configs.fractal_dem(n, dx, 0.8, 30.0, 10.0, seed)
    st = {"B_cent": B, "solve_mask_time": np.zeros((n, n))}
    geom = configs.topography_geom(B, dx, dx)
    st.update(geom)
    if slope:
        p.slope_correction_flag = 1
        gc = 1.0 / (1.0 + geom["B_prime_x_geom"] ** 2 + geom["B_prime_y_geom"] ** 2)
        st["grav_coeff"] = gc
        st["d_grav_coeff_dx"] = -2.0 * gc ** 2 * (geom["B_prime_x_geom"] * geom["B_second_xx_geom"]
                                                  + geom["B_prime_y_geom"] * geom["B_second_xy_geom"])
        gsx = np.ones((n + 1, n))
        gsx[1:n] = 0.5 * (gc[:-1] + gc[1:])
        gsx[0] = gc[0]
        gsx[n] = gc[-1]
        gsy = np.ones((n, n + 1))
        gsy[:, 1:n] = 0.5 * (gc[:, :-1] + gc[:, 1:])
        gsy[:, 0] = gc[:, 0]
        gsy[:, n] = gc[:, -1]
        st["grav_coeff_stag_x"] = gsx
        st["grav_coeff_stag_y"] = gsy
    if curvature:
        p.curvature_term_flag = 1
    rng = np.random.default_rng(seed)
    qp = np.zeros((8, n, n))
    _, xc, _, yc = configs.grid(p)
    X, Y = np.meshgrid(xc, yc, indexing="ij")
    blob = np.exp(-((X - 0.3 * n * dx) ** 2 + (Y - 0.5 * n * dx) ** 2) / (2 * (0.15 * n * dx) ** 2))
    h = 2.0 * blob * (blob > 0.05)
    qp[0] = h
    qp[1] = h * 1.0
    qp[3] = 600.0 + 50.0 * rng.random((n, n))
    qp[4] = 0.01 * h
    qp[5] = 0.005 * h
    qp[6] = np.where(h > 0, 1.0, 0.0)
    return p, st, configs.qp_to_qc_grid(p, qp)


def radial(n=64):
    return configs.radial_current(nx=n, ny=n, dx=2.0, r_source=8.0, bump_sigma=30.0, mfr=5e5)


def fractal_small(n=64, layer=1.0, seed=20261203):
    """Third workload's physics (3 classes, settling + erosion, inlet) on a
    small fractal DEM with an initial layer."""
    return configs.fractal_inlet(n=n, dx=10.0, relief=120.0, seed=seed, r_source=25.0,
                                 mfr=2e5, initial_layer=layer)


def test2d():
    """The reference's TESTS/TEST_2D run (100x68, quadratic friction, settling
    and entrainment) from the committed input fixture."""
    import os
    d = np.load(os.path.join(os.path.dirname(__file__), "golden", "test2d_inputs.npz"))
    nx, ny = int(d["nx"]), int(d["ny"])
    p = configs.default_params(nx, ny, 1, float(d["cell_size"]), x0=float(d["x0"]),
                               y0=float(d["y0"]))
    p.rho_s[0] = 2000.0
    p.diam_s[0] = 1e-4
    p.sp_heat_s[0] = 1617.0
    p.settling_flag = 1
    p.entrainment_flag = 1
    p.erosion_coeff = 0.0
    p.erodible_porosity = 0.0
    p.erodible_fract[0] = 1.0
    p.T_erodible = 300.0
    p.rho_c_sub = p.pres / (p.sp_gas_const_a * p.T_erodible)
    p.coeff_porosity = 0.0
    p.rheology_flag = 1
    p.rheology_model = 6
    p.friction_factor = 1.0e-3
    p.max_dt = 1.0
    p.theta = 1.3
    for side in "WESN":
        for i in range(5):
            configs.set_bc(p, side, i, 1, 0.0)
    B = np.asfortranarray(d["B_cent"])
    st = {"B_cent": B, "solve_mask_time": np.zeros((nx, ny)),
          "erodible": np.zeros((1, nx, ny)), "deposit": np.zeros((nx, ny, 1)),
          "erosion": np.zeros((nx, ny, 1))}
    st.update(configs.topography_geom(B, p.cell_size, p.cell_size))
    return p, st, np.asfortranarray(d["q"])


def dambreak_ns(ns, nx=40, ny=40, dx=0.25, rheology=1):
    """Dam break with `ns` solid classes (diameters 1e-5..1e-3 m)."""
    p = configs.default_params(nx, ny, ns, dx)
    for i in range(ns):
        p.rho_s[i] = 2500.0 - 200.0 * i
        p.diam_s[i] = 10.0 ** (-5 + 2.0 * i / max(ns - 1, 1))
        p.sp_heat_s[i] = 1617.0
    p.max_dt = 1.0e-2
    configs.transmissive_bcs(p)
    p.rheology_flag = 1
    p.rheology_model = rheology
    p.mu, p.xi = 0.1, 500.0
    _, xc, _, _ = configs.grid(p)
    h = np.where(np.repeat(xc[:, None], ny, axis=1) < 0.5 * nx * dx, 1.0, 0.1)
    qp = np.zeros((4 + ns + 2, nx, ny))
    qp[0] = h
    qp[3] = 300.0
    for i in range(ns):
        qp[4 + i] = 0.01 / ns * h
    zeros = np.zeros((nx, ny))
    st = {"B_cent": zeros, "B_prime_x_geom": zeros, "B_prime_y_geom": zeros,
          "solve_mask_time": zeros}
    return p, st, configs.qp_to_qc_grid(p, qp)


def edge_variants():
    """Options and shapes beyond the workloads: the remaining limiters,
    four solid classes, a rectangular grid with per-cell release times and a
    Neumann slope on one side, no-data cells, an all-dry grid, the smallest
    grid."""
    out = {}
    for lim in (0, 5, 6, 7):
        p, st, q = dambreak(rheology=1)
        for i in range(7):
            p.limiter[i] = lim
        out["limiter%d" % lim] = (p, st, q)
    out["four_classes"] = dambreak_ns(4)
    out["two_classes_quadratic"] = dambreak_ns(2, rheology=6)
    # rectangular grid with ragged tiles; the dry strip east of x = 9.2 m is
    # released at t = 0.05 s, as the front arrives; Neumann slope on h at E
    p2, st2, q2 = configs.dambreak(nx=70, ny=33, dx=0.25, rheology=1, x_split=8.0)
    _, xc, _, _ = configs.grid(p2)
    X = np.repeat(xc[:, None], 33, axis=1)
    st2 = dict(st2)
    st2["solve_mask_time"] = np.asfortranarray(np.where(X > 9.2, 0.05, 0.0))
    q2 = q2.copy()
    q2[:, X > 9.2] = 0.0
    configs.set_bc(p2, "E", 0, 1, 0.01)      # h: Neumann with a non-zero slope
    out["rect_release_neumann"] = (p2, st2, q2)
    # no-data patch inside the flow (the reference zeroes it after each step)
    p, st, q = dambreak(rheology=1)
    nd = np.zeros((p.nx, p.ny), np.int8)
    nd[12:18, 20:30] = 1
    st = dict(st)
    st["B_nodata"] = nd
    q = q.copy()
    q[:, nd == 1] = 0.0
    out["nodata_patch"] = (p, st, q)
    # all dry: only the border rows are solved
    p, st, q = dambreak(rheology=1)
    out["all_dry"] = (p, st, np.zeros_like(q))
    # a 3x5 grid; one-row and one-column grids (no fluxes, divergence or
    # CFL limit across the one-cell direction, whose spacing is 1)
    out["tiny_3x5"] = configs.dambreak(nx=3, ny=5, dx=0.25, rheology=1, x_split=0.4)
    out["one_row_60x1"] = configs.dambreak(nx=60, ny=1, dx=0.25, rheology=1, x_split=7.0)
    p, st, q = configs.dambreak(nx=1, ny=60, dx=0.25, rheology=6)
    _, _, _, yc = configs.grid(p)
    qp = np.zeros((7, 1, 60))
    qp[0, 0] = np.where(yc < 7.0, 1.0, 0.1)
    qp[3] = 300.0
    qp[4] = 0.01 * qp[0]
    out["one_column_1x60"] = (p, st, configs.qp_to_qc_grid(p, qp))
    out["single_cell_1x1"] = configs.dambreak(nx=1, ny=1, dx=0.25, rheology=1)
    return out


def fractal_topo(n=48):
    """The fractal workload with a moving bed: erosion and deposition change
    B_cent (topo_change_flag), the slopes and, with slope correction and
    curvature on, grav_coeff and the curvatures are rebuilt after every step."""
    p, st, q = configs.fractal_inlet(n=n, initial_layer=1.0, erosion_coeff=5.0e-3)
    p.topo_change_flag = 1
    p.slope_correction_flag = 1
    p.curvature_term_flag = 1
    st = dict(st)
    geo = configs.topography_geom(np.asarray(st["B_cent"]), p.cell_size, p.cell_size)
    st.update(geo)
    st.update(configs.slope_correction_planes(geo))
    return p, st, q


def _one_row_case(name):
    """The reference's TESTS/TEST_BW or TESTS/TEST_BOX run (400 x 1 cells of
    125 m; quadratic friction 1e-3, settling and entrainment, one solid
    class of 2000 kg/m^3, minmod, theta 1.3, CFL 0.24, MAX_DT 0.2, DT0 1e-4)
    from the committed fixture (restart and DEM sampled at the cell
    centres).  TEST_BW: a 400 m deep current enters through a Dirichlet west
    boundary at 25 m/s over a ramp; TEST_BOX: a 9-cell box released on a
    flat bed.  The east boundary is zero-gradient.  Returns (p, st, q,
    t_end)."""
    import os
    d = np.load(os.path.join(os.path.dirname(__file__), "golden", "bw_box_inputs.npz"))
    nx, ny, cs = int(d["nx"]), int(d["ny"]), float(d["cell_size"])
    p = configs.default_params(nx, ny, 1, cs, x0=float(d["x0"]), y0=float(d["y0"]))
    p.rho_s[0] = 2000.0
    p.diam_s[0] = 1e-3 if name == "bw" else 1e-4
    p.sp_heat_s[0] = 1617.0
    p.settling_flag = 1
    p.entrainment_flag = 1
    p.erosion_coeff = 0.0
    p.erodible_porosity = 0.0
    p.erodible_fract[0] = 1.0
    p.T_erodible = 300.0
    p.rho_c_sub = p.pres / (p.sp_gas_const_a * p.T_erodible)
    p.coeff_porosity = 0.0
    p.rheology_flag = 1
    p.rheology_model = 6
    p.friction_factor = 1.0e-3
    p.cfl = 0.23999999463558197
    p.max_dt = 0.2
    p.theta = 1.3
    # boundary variables: h, hu, hv, T, h*alpha_s (src/inpout_2d.f90:2304-2306,2876,2895)
    if name == "bw":
        for i, v in enumerate((400.0, 10000.0, 0.0, 900.0, 0.1)):
            configs.set_bc(p, "W", i, 0, v)
    else:
        for i in range(5):
            configs.set_bc(p, "W", i, 1, 0.0)
        configs.set_bc(p, "W", 2, 0, 0.0)
    for i in range(5):
        configs.set_bc(p, "E", i, 1, 0.0)
    configs.set_bc(p, "E", 2, 0, 0.0)
    for side in "SN":              # not read for a one-row grid; never used
        for i in range(5):
            configs.set_bc(p, side, i, 1, 0.0)
    B = np.asfortranarray(d[name + "_B_cent"])
    st = {"B_cent": B, "solve_mask_time": np.zeros((nx, ny)),
          "erodible": np.zeros((1, nx, ny)), "deposit": np.zeros((nx, ny, 1)),
          "erosion": np.zeros((nx, ny, 1))}
    st.update(configs.topography_geom(B, cs, 1.0))
    t_end = 400.0 if name == "bw" else 200.0
    return p, st, np.asfortranarray(d[name + "_q"]), t_end


def test_bw():
    return _one_row_case("bw")


def test_box():
    return _one_row_case("box")
