"""Host setup (C++, no GPU) against the reference's own arrays dumped by the oracle harness.

The reference builds these in code/src/main.cc:273-860 (basis, quadrature, Jacobians, inverse
mass matrices, maps, neighbours, limiter transforms).  Integer arrays must match exactly;
floating-point arrays to 1e-13 relative (the reference inverts with LAPACK, this code with its
own LU).
"""
import numpy as np
import pytest

from conftest import golden_cases, load_golden, problem_for

INT_ARRAYS = ("map", "invmap", "boundaryMap", "neighbors")
FLOAT_ARRAYS = ("phi", "dphi", "phi_w", "dphi_w", "psi", "psi_w", "weight", "J", "invJac", "JF", "normals",
                "Minv", "Lag2Mono", "Mono2Lag", "Lag2MonoX", "MonoX2MonoY", "MonoY2Lag", "MonoX2Lag", "Lag2MonoY")


@pytest.mark.parametrize("name", golden_cases())
def test_setup_arrays_match_reference(name):
    meta, d = load_golden(name)
    prob = problem_for(meta)
    checked = 0
    for k in INT_ARRAYS + FLOAT_ARRAYS:
        if "ref_" + k not in d:
            continue
        ref = d["ref_" + k]
        if k not in INT_ARRAYS and not np.any(ref):
            continue  # allocated but never filled by the reference for this limiter
        if k in ("MonoX2Lag", "Lag2MonoY") and meta["limiter"] not in ("m2l", "hri", "m2i", "pri"):
            continue  # the 2D Limiting constructor forms these only for those methods (limiting.h:318-319)
        mine = prob.array(k)
        assert mine.shape == ref.shape, k
        if k in INT_ARRAYS:
            assert np.array_equal(mine, ref), k
        else:
            scale = max(np.abs(ref).max(), 1e-300)
            # the reference's p = 3 metric and face normals sum 16 (4) geometric-node derivative
            # terms whose cancellation leaves entries of ~1e-13 relative where the exact value is 0
            tol = 5e-13 if k in ("invJac", "normals", "JF", "J") and meta["order"] == 3 else 1e-13
            assert np.abs(mine - ref).max() <= tol * scale, (k, np.abs(mine - ref).max() / scale)
        checked += 1
    assert checked >= 12


@pytest.mark.parametrize("name", golden_cases())
def test_sizes_match_reference(name):
    meta, _ = load_golden(name)
    rm = meta["ref_meta"]
    i = problem_for(meta).info
    assert (i.n_elem, i.n_s, i.n_g, i.n_ifaces, i.m_s, i.m_g, i.n_n) == \
        (rm["N_E"], rm["N_s"], rm["N_G"], rm["M_T"], rm["M_s"], rm["M_G"], rm["N_N"])
    assert i.limiter == rm["limiter"]
    if meta["dim"] == 2:  # the 1D Limiting constructor leaves its cartesian flag unset
        assert i.cartesian == rm["cartesian"]
    # the fixtures' decks carry CFL = -1: cfl_scaled = CFL * Dx / (2p+1) (main.cc:896-897)
    assert abs(i.cfl_scaled / meta["cfl"] - rm["cfl_scaled"] / -1.0) <= 1e-15 * abs(rm["cfl_scaled"])


def test_msh_roundtrip_equals_in_memory_mesh(tmp_path):
    import dg_b200 as dgb
    dgb.write_msh(tmp_path / "mesh.msh", 2, 2, 6, 3, 0.0, 2.0, 0.0, 1.0,
                  ("reflective", "transmissive", "reflective", "transmissive"))
    (tmp_path / "deck.inp").write_text(
        "#Make options\nFLUX=RUS\n#Code options\n#time integration\nrk4\n#output time array\n0 0.1\n"
        "#final time\n0.1\n#Courant-Friedrichs-Lewy condition\n0.3\n#order\n2\n#mesh file\nmesh.msh\nqua\n"
        "#limiter\nm2l\n#initial condition\nsodcirc\n")
    a = dgb.Problem.from_deck(tmp_path / "deck.inp")
    b = dgb.Problem.structured(2, 2, 6, 3, 0.0, 2.0, 0.0, 1.0,
                               ("reflective", "transmissive", "reflective", "transmissive"),
                               flux="rusanov", limiter="m2l", cfl=0.3)
    assert a.info.flux == 0 and a.info.limiter == 2 and a.info.n_output_times == 2
    for k in ("map", "invmap", "neighbors", "normals", "Minv", "J", "JF", "xyz_nodes"):
        assert np.array_equal(a.array(k), b.array(k)), k


def test_pos_roundtrip(tmp_path):
    import dg_b200 as dgb
    p = dgb.Problem.structured(2, 2, 4, 3, flux="rusanov", limiter="m2l")
    U = p.init_state("quadrants", seed=5)
    p.write_pos(U, 3, 0.125, tmp_path)
    assert sorted(f.name for f in tmp_path.iterdir()) == \
        ["g0000000003.pos", "p0000000003.pos", "rho0000000003.pos", "ux0000000003.pos", "uy0000000003.pos"]
    V, t = p.read_pos(3, tmp_path)
    assert t == 0.125
    assert np.abs(U - V).max() <= 1e-14 * np.abs(U).max()


def test_mass_fraction_state_and_pos_round_trip(tmp_path):
    """One passive mass fraction: N_F grows by one, the initial states carry rho Y = rho times the
    region marker, and the .pos output (field y0 = Y, printer.cc:65-71) reads back exactly."""
    import dg_b200 as dgb
    prob = dgb.Problem.structured(2, 2, 8, 4, 0.0, 2.0, 0.0, 1.0, ("transmissive",) * 4, flux="roe", limiter="m2l",
                                  cfl=0.3, n_mass=1)
    i = prob.info
    assert i.n_fields == 6
    U = prob.init_state("shock_bubble", seed=3)
    V = U.reshape(i.n_elem, i.n_fields, i.n_s)
    Y = V[:, 5] / V[:, 0]
    assert set(np.unique(Y)) <= {0.0, 1.0} and Y.max() == 1.0 and Y.min() == 0.0
    prob.write_pos(U, 7, 0.25, tmp_path)
    assert (tmp_path / "y00000000007.pos").exists()
    assert '"Y0"' in (tmp_path / "y00000000007.pos").read_text()
    U2, t = prob.read_pos(7, tmp_path)
    assert t == 0.25
    assert np.abs(U2 - U).max() <= 1e-15 * np.abs(U).max()


def test_deck_mass_option(tmp_path):
    """MASS=1 in the deck's "#Make options" block gives one mass fraction."""
    import dg_b200 as dgb
    dgb.write_msh(tmp_path / "mesh.msh", 1, 2, 20, 1, 0.0, 1.0, 0.0, 1.0, ("transmissive",) * 4)
    (tmp_path / "deck.inp").write_text(
        "#Make options\nFLUX=RUS\nMASS=1\n#Code options\n#time integration\nrk4\n#output time step size\n0.1\n"
        "#final time\n0.1\n#Courant-Friedrichs-Lewy condition\n0.4\n#order\n2\n#mesh file\nmesh.msh\nlin\n"
        "#limiter\nm2l\n#initial condition\nsodtube\n")
    prob = dgb.Problem.from_deck(tmp_path / "deck.inp")
    assert prob.info.n_fields == 5
    assert prob.info.cons_output == 0 and prob.info.error_output == 0
    (tmp_path / "deck.inp").write_text((tmp_path / "deck.inp").read_text().replace("MASS=1", "CONS=CONS\nERRR=ERROR"))
    i = dgb.Problem.from_deck(tmp_path / "deck.inp").info
    assert (i.n_fields, i.cons_output, i.error_output) == (4, 1, 1)


def test_gamcons_state_pos_and_deck(tmp_path):
    """GAMCONS: the gamma-model field holds rho/(gamma-1) in every initial state, the .pos output
    (g = 1 + rho/field, printer_twod_multifluid.cu:48-52) reads back exactly, and GAMM=GAMCONS in
    the deck's "#Make options" block selects the model."""
    import dg_b200 as dgb
    a = dgb.Problem.structured(2, 2, 8, 4, 0.0, 2.0, 0.0, 1.0, ("transmissive",) * 4, flux="roe", limiter="hrl")
    b = dgb.Problem.structured(2, 2, 8, 4, 0.0, 2.0, 0.0, 1.0, ("transmissive",) * 4, flux="roe", limiter="hrl",
                               gamma_model="gamcons")
    assert (a.info.gamma_model, b.info.gamma_model) == (0, 1)
    i = b.info
    for ic in ("shock_bubble", "quadrants", "sinegam"):
        Ua = a.init_state(ic, seed=3).reshape(i.n_elem, i.n_fields, i.n_s)
        Ub = b.init_state(ic, seed=3).reshape(i.n_elem, i.n_fields, i.n_s)
        assert np.array_equal(Ua[:, :4], Ub[:, :4])
        assert np.allclose(Ub[:, 4], Ua[:, 0] * Ua[:, 4], rtol=1e-15, atol=0)
    U = b.init_state("shock_bubble", seed=3)
    b.write_pos(U, 2, 0.5, tmp_path)
    g = a.init_state("shock_bubble", seed=3)
    (tmp_path / "a").mkdir()
    a.write_pos(g, 2, 0.5, tmp_path / "a")
    for f in ("g0000000002.pos", "p0000000002.pos"):  # the same physical fields in both models
        assert (tmp_path / f).read_text() == (tmp_path / "a" / f).read_text()
    U2, t = b.read_pos(2, tmp_path)
    assert t == 0.5
    assert np.abs(U2 - U).max() <= 1e-14 * np.abs(U).max()
    dgb.write_msh(tmp_path / "mesh.msh", 1, 2, 20, 1, 0.0, 1.0, 0.0, 1.0, ("transmissive",) * 4)
    deck = ("#Make options\nFLUX=RUS\nGAMM={}\n#Code options\n#time integration\nrk4\n#output time step size\n"
            "0.1\n#final time\n0.1\n#Courant-Friedrichs-Lewy condition\n0.4\n#order\n2\n#mesh file\nmesh.msh\n"
            "lin\n#limiter\nhrl\n#initial condition\nsodtube\n")
    (tmp_path / "deck.inp").write_text(deck.format("GAMCONS"))
    assert dgb.Problem.from_deck(tmp_path / "deck.inp").info.gamma_model == 1
    (tmp_path / "deck.inp").write_text(deck.format("GAMNCON"))
    assert dgb.Problem.from_deck(tmp_path / "deck.inp").info.gamma_model == 0
    (tmp_path / "deck.inp").write_text(deck.format("OTHER"))
    with pytest.raises(dgb.DGBError):
        dgb.Problem.from_deck(tmp_path / "deck.inp")


def test_error_norms_match_the_oracle():
    """dgb_problem_error_norms (the reference driver's ERROR block) against its numpy restatement,
    on the smooth advection state and a perturbed copy."""
    import dg_b200 as dgb
    from oracle import dg_oracle as O
    for dim, nx, ny, gm in ((1, 24, 1, "gamncon"), (2, 8, 6, "gamncon"), (1, 24, 1, "gamcons")):
        prob = dgb.Problem.structured(dim, 2, nx, ny, 0.0, 1.0, 0.0, 1.0, ("periodic",) * 4, flux="rusanov",
                                      limiter="none", cfl=0.2, gamma_model=gm)
        Uex = prob.init_state("sinegam")
        rng = np.random.default_rng(4)
        U = Uex * (1 + 1e-3 * rng.uniform(-1, 1, Uex.shape))
        mine = prob.error_norms(U, Uex)
        S = O.Setup.from_problem(prob)
        xyz = prob.array("xyz_nodes")
        ref = O.error_norms(S, U, Uex, (xyz[0], xyz[1]))
        assert abs(mine["dx"] - ref[0]) == 0
        nf = prob.info.n_fields
        got = np.concatenate([mine["l1"], mine["l2"], mine["linf"]])
        assert np.allclose(got, ref[1:], rtol=1e-12, atol=0), (got, ref[1:])
        assert mine["l1"][0] > 0


def test_sinegam_initial_state():
    """The reference's smooth advection test: uniform velocity and pressure, rho and gamma perturbed."""
    import dg_b200 as dgb
    prob = dgb.Problem.structured(1, 2, 16, 1, 0.0, 1.0, 0.0, 1.0, ("periodic",) * 2, flux="rusanov", limiter="none")
    i = prob.info
    V = prob.init_state("sinegam").reshape(i.n_elem, i.n_fields, i.n_s)
    rho, u = V[:, 0], V[:, 1] / V[:, 0]
    gam = 1 + 1 / V[:, 3]
    p = (gam - 1) * (V[:, 2] - 0.5 * rho * u * u)
    assert np.allclose(u, 1.0, atol=1e-15) and np.allclose(p, 1.0, atol=1e-14)
    assert 0.79 < rho.min() < 0.81 and 1.19 < rho.max() < 1.21 and 1.19 < gam.min() and gam.max() < 1.61
