"""The CPU oracle against the reference's own outputs (tests/golden/, made by
tests/golden/make_golden.py from the reference's impl='c' host core).

These pin the oracle: every GPU parity test trusts it only because these pass."""
from pathlib import Path

import numpy as np
import pytest

from oracle import oracle as O

GOLD = Path(__file__).resolve().parent / "golden"


def rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def _args(d):
    return float(d["dh"]), float(d["dt"]), int(d["abcn"])


@pytest.mark.parametrize("case", ["acoustic2d_c1", "acoustic2d_multi", "acoustic2d_pershot"])
def test_acoustic2d_oracle_matches_reference(case):
    d = np.load(GOLD / f"{case}.npz")
    obs = O.acoustic_forward(d["vp_true"], d["wavelet"], d["src"], d["rec"], *_args(d))
    assert rel(obs, d["obs"]) < 2e-5
    pred, loss, g, gw = O.acoustic_gradient(d["vp_init"], d["wavelet"], d["src"], d["rec"], d["obs"], *_args(d))
    assert rel(pred, d["pred"]) < 2e-5
    assert abs(loss - float(d["loss"])) <= 1e-4 * abs(float(d["loss"]))
    assert rel(g, d["grad_vp"]) < 1e-5
    if "grad_wavelet" in d:
        assert rel(gw, d["grad_wavelet"]) < 1e-5


def test_acoustic2d_memory_modes_agree_in_reference():
    """The reference's own memory modes agree; so one backward (boundary
    saving) stands for all of them."""
    d = np.load(GOLD / "acoustic2d_multi.npz")
    assert rel(d["grad_vp_full"], d["grad_vp"]) < 1e-5
    assert rel(d["grad_vp_ckpt"], d["grad_vp"]) < 1e-5


def test_acoustic2d_fp64_oracle_close_to_fp32():
    d = np.load(GOLD / "acoustic2d_multi.npz")
    p32, _, g32, _ = O.acoustic_gradient(d["vp_init"], d["wavelet"], d["src"], d["rec"], d["obs"], *_args(d), prec="f32")
    p64, _, g64, _ = O.acoustic_gradient(d["vp_init"], d["wavelet"], d["src"], d["rec"], d["obs"], *_args(d), prec="f64")
    assert rel(p32, p64) < 1e-5
    assert rel(g32, g64) < 1e-4


def test_off_grid_receivers_record_zero():
    d = np.load(GOLD / "acoustic2d_multi.npz")
    obs = O.acoustic_forward(d["vp_true"], d["wavelet"], d["src"], d["rec"], *_args(d))
    # shot 1 has 7 receivers; the padding (x = -1000) lands off the grid
    assert np.all(obs[1, :, 7:, 0] == 0)
    assert np.all(d["obs"][1, :, 7:, 0] == 0)


def test_coefficient_tables_zero_sum():
    """The float32 Laplacian taps sum to exactly zero and equal the reference
    kernels' compile-time constants (operators/laplace.cuh:331-335)."""
    from fractions import Fraction
    lap, grad = O.fd_tables(4)
    assert Fraction(float(lap[0])) == 2 * sum(Fraction(float(x)) for x in lap[1:])
    f = np.float32
    c0, c1, c2, c3 = f(205 / 72), f(8 / 5), f(-1 / 5), f(8 / 315)
    c4 = ((f(0.5) * c0 - c1) - c2) - c3
    assert list(lap[1:]) == [c1, c2, c3, c4]
    assert list(grad[1:]) == [f(4 / 5), f(-1 / 5), f(4 / 105), f(-1 / 280)]


def test_acoustic3d_oracle_matches_reference():
    d = np.load(GOLD / "acoustic3d.npz")
    obs = O.acoustic_forward(d["vp_true"], d["wavelet"], d["src"], d["rec"], *_args(d))
    assert rel(obs, d["obs"]) < 2e-5
    run = O.Acoustic3D(d["vp_init"], d["wavelet"], d["src"], d["rec"], *_args(d))
    pred = run.forward()
    assert rel(pred, d["pred"]) < 2e-5
    g, gw = run.backward(pred - d["obs"])
    assert rel(g, d["grad_vp"]) < 1e-5
    assert rel(d["grad_vp_full"], d["grad_vp"]) < 1e-5
    # The reference's 3-D wavelet gradient holds shot 0 only: its kernel takes
    # the shot from the y launch axis while the launch puts shots on x
    # (reference acoustic3d/kernels.cu:256-257, launch/config.h:65-70).  Shot
    # 0 is exact; the oracle keeps every shot.
    assert rel(gw[0], d["grad_wavelet"]) < 1e-5
    assert np.abs(gw[1]).max() > 0


def _el_args(d):
    return float(d["dh"]), float(d["dt"]), int(d["abcn"]), int(d["order"])


@pytest.mark.parametrize("prec,tol", [("f32", 2e-6), ("f64", 5e-6)])
def test_elastic2d_oracle_matches_reference(prec, tol):
    """Records and vp / vs / rho gradients of the reference's boundary-saving
    elastic path (explosive sources, (vx, vz) receivers)."""
    d = np.load(GOLD / "elastic2d.npz")
    obs = O.elastic_forward(d["vp_true"], d["vs_true"], d["rho_true"], d["wavelet"], d["src"],
                            d["rec"], *_el_args(d), prec=prec)
    assert obs.shape == d["obs"].shape
    assert rel(obs, d["obs"]) < tol
    pred, loss, (gvp, gvs, grho) = O.elastic_gradient(
        d["vp_init"], d["vs_init"], d["rho_init"], d["wavelet"], d["src"], d["rec"], d["obs"],
        *_el_args(d), prec=prec)
    assert rel(pred, d["pred"]) < tol
    assert abs(loss - float(d["loss"])) < 1e-5 * float(d["loss"])
    assert rel(gvp, d["grad_vp"]) < 5 * tol
    assert rel(gvs, d["grad_vs"]) < 5 * tol
    assert rel(grho, d["grad_rho"]) < 5 * tol


@pytest.mark.parametrize("prec,tol", [("f32", 2e-6), ("f64", 5e-6)])
def test_elastic2d_velocity_sources_oracle_matches_reference(prec, tol):
    """Body-force sources on vx and vz (one inside the boundary strips, a
    receiver on its cell), (vx, vz, sxx) receivers: records and vp / vs / rho
    gradients, the rho one with the source correction of common.cu:40-75."""
    d = np.load(GOLD / "elastic2d_vsrc.npz")
    kw = dict(source_fields=("vx", "vz"), receiver_fields=("vx", "vz", "sxx"))
    obs = O.elastic_forward(d["vp_true"], d["vs_true"], d["rho_true"], d["wavelet"], d["src"],
                            d["rec"], *_el_args(d), prec=prec, **kw)
    assert obs.shape == d["obs"].shape
    assert rel(obs, d["obs"]) < tol
    pred, loss, (gvp, gvs, grho) = O.elastic_gradient(
        d["vp_init"], d["vs_init"], d["rho_init"], d["wavelet"], d["src"], d["rec"], d["obs"],
        *_el_args(d), prec=prec, **kw)
    assert rel(pred, d["pred"]) < tol
    assert rel(gvp, d["grad_vp"]) < 5 * tol
    assert rel(gvs, d["grad_vs"]) < 5 * tol
    assert rel(grho, d["grad_rho"]) < 5 * tol


@pytest.mark.parametrize("prec,tol", [("f32", 2e-6), ("f64", 5e-6)])
def test_elastic2d_free_surface_oracle_matches_reference(prec, tol):
    """Traction-free top face (image method, order-2 band, Robertsson sxx
    correction, szz = 0 on the surface row): a shot on the surface row
    recorded on it and a shot below it; records and vp / vs / rho gradients
    of the reference's boundary-saving run.  Without the free surface the
    records differ at order one, so the fixture pins the surface terms."""
    d = np.load(GOLD / "elastic2d_free_surface.npz")
    obs = O.elastic_forward(d["vp_true"], d["vs_true"], d["rho_true"], d["wavelet"], d["src"],
                            d["rec"], *_el_args(d), prec=prec, free_surface=True)
    assert obs.shape == d["obs"].shape
    assert rel(obs, d["obs"]) < tol
    plain = O.elastic_forward(d["vp_true"], d["vs_true"], d["rho_true"], d["wavelet"], d["src"],
                              d["rec"], *_el_args(d), prec=prec)
    assert rel(plain, d["obs"]) > 0.1
    pred, loss, (gvp, gvs, grho) = O.elastic_gradient(
        d["vp_init"], d["vs_init"], d["rho_init"], d["wavelet"], d["src"], d["rec"], d["obs"],
        *_el_args(d), prec=prec, free_surface=True)
    assert rel(pred, d["pred"]) < tol
    assert abs(loss - float(d["loss"])) < 1e-5 * float(d["loss"])
    assert rel(gvp, d["grad_vp"]) < 5 * tol
    assert rel(gvs, d["grad_vs"]) < 5 * tol
    assert rel(grho, d["grad_rho"]) < 5 * tol
    # the reference's checkpointed run gives the boundary-saving gradient
    for k in ("vp", "vs", "rho"):
        assert rel(d[f"grad_{k}_ckpt"], d[f"grad_{k}"]) < 2e-6


@pytest.mark.parametrize("tag,faces", [("br", ["bottom", "right"]), ("tl", ["top", "left"]),
                                       ("all", ["top", "bottom", "left", "right"])])
def test_elastic2d_free_faces_oracle_matches_reference(tag, faces):
    """Traction-free faces per edge: the high-side images (a half field's
    surface node is air; zeroed shear), the x-normal Robertsson correction of
    szz, corners where two surfaces meet; (vx, vz, sxx) receivers on the
    surface rows and columns."""
    d = np.load(GOLD / "elastic2d_free_faces.npz")
    kw = dict(free_surface=faces, receiver_fields=("vx", "vz", "sxx"))
    obs = O.elastic_forward(d["vp_true"], d["vs_true"], d["rho_true"], d["wavelet"], d["src"],
                            d["rec"], *_el_args(d), **kw)
    assert rel(obs, d[f"obs_{tag}"]) < 2e-6
    pred, loss, (gvp, gvs, grho) = O.elastic_gradient(
        d["vp_init"], d["vs_init"], d["rho_init"], d["wavelet"], d["src"], d["rec"], d[f"obs_{tag}"],
        *_el_args(d), **kw)
    assert rel(pred, d[f"pred_{tag}"]) < 2e-6
    assert rel(gvp, d[f"grad_vp_{tag}"]) < 1e-5
    assert rel(gvs, d[f"grad_vs_{tag}"]) < 1e-5
    assert rel(grho, d[f"grad_rho_{tag}"]) < 1e-5


def test_elastic2d_reference_full_and_boundary_modes_agree():
    """The reference's full-storage gradient adds the it = 0 image the
    boundary-saving reverse skips; the two differ at the 1e-6 level."""
    d = np.load(GOLD / "elastic2d.npz")
    for k in ("vp", "vs", "rho"):
        assert rel(d[f"grad_{k}_full"], d[f"grad_{k}"]) < 1e-5


def test_staggered_coefficients_match_compiled_constants():
    """Order 8 gives the compile-time constants of operators/staggered.cuh:351-354."""
    from fractions import Fraction
    c = O.staggered_coefficients(4)
    assert c == [Fraction(1225, 1024), Fraction(-245, 3072), Fraction(49, 5120), Fraction(-5, 7168)]
    assert O.staggered_coefficients(1) == [Fraction(1)]
    assert O.staggered_coefficients(2) == [Fraction(9, 8), Fraction(-1, 24)]


@pytest.mark.parametrize("case", ["acoustic2d_illum", "acoustic3d_illum"])
def test_illumination_oracle_matches_reference(case):
    """Source and receiver illumination (sum_t u_tt^2, sum_t lambda^2 on the
    physical box, summed over shots) of the reference's boundary-saving run
    with solver.compute_illumination = True; its full-storage run agrees, and
    turning illumination on left the reference's gradient bit-identical."""
    d = np.load(GOLD / f"{case}.npz")
    pred, loss, g, gw, i_s, i_r = O.acoustic_gradient(d["vp_init"], d["wavelet"], d["src"], d["rec"], d["obs"],
                                                      *_args(d), illum=True)
    assert rel(pred, d["pred_bs"]) < 2e-5
    assert rel(g, d["grad_vp_bs"]) < 1e-5
    assert rel(i_s, d["src_illum_bs"]) < 1e-5
    assert rel(i_r, d["rec_illum_bs"]) < 1e-5
    assert np.array_equal(d["grad_vp_bs"], d["grad_vp_off"])
    assert rel(d["src_illum_full"], d["src_illum_bs"]) < 1e-4
    assert rel(d["rec_illum_full"], d["rec_illum_bs"]) < 1e-4
    # the same gradient with illumination off in the oracle
    _, _, g_off, _ = O.acoustic_gradient(d["vp_init"], d["wavelet"], d["src"], d["rec"], d["obs"], *_args(d))
    assert np.array_equal(g, g_off)


def test_acoustic3d_clean_box_oracle_matches_reference():
    """A 3-D grid whose clear box spans several 32 x 8 column blocks."""
    d = np.load(GOLD / "acoustic3d_clean.npz")
    pred, loss, g, gw = O.acoustic_gradient(d["vp_init"], d["wavelet"], d["src"], d["rec"], d["obs"], *_args(d))
    assert rel(pred, d["pred"]) < 2e-5
    assert rel(g, d["grad_vp"]) < 1e-5
    # reference 3-D wavelet gradient: shot 0 only (see above)
    assert rel(gw[0], d["grad_wavelet"][0]) < 1e-5


def test_acoustic2d_many_shots_oracle_matches_reference():
    d = np.load(GOLD / "acoustic2d_many.npz")
    pred, loss, g, gw = O.acoustic_gradient(d["vp_init"], d["wavelet"], d["src"], d["rec"], d["obs"], *_args(d))
    assert rel(pred, d["pred"]) < 2e-5
    assert rel(g, d["grad_vp"]) < 1e-5
    assert rel(gw, d["grad_wavelet"]) < 1e-5


def test_elastic2d_interior_tiles_oracle_matches_reference():
    d = np.load(GOLD / "elastic2d_interior.npz")
    pred, loss, (gvp, gvs, grho) = O.elastic_gradient(
        d["vp_init"], d["vs_init"], d["rho_init"], d["wavelet"], d["src"], d["rec"], d["obs"], *_el_args(d))
    assert rel(pred, d["pred"]) < 2e-6
    assert rel(gvp, d["grad_vp"]) < 1e-5
    assert rel(gvs, d["grad_vs"]) < 1e-5
    assert rel(grho, d["grad_rho"]) < 1e-5


def test_library_tables_equal_the_oracle_restatement():
    """The library derives its float32 tables in closed form; the oracle
    restates the reference's own derivation.  They agree bit for bit."""
    from sweep_b200.scalars import centred_tables
    for M in range(1, 7):
        lib, ora = centred_tables(M), O.fd_tables(M)
        assert np.array_equal(lib[0], ora[0]) and np.array_equal(lib[1], ora[1]), M


@pytest.mark.parametrize("prec,tol", [("f32", 2e-6), ("f64", 5e-6)])
@pytest.mark.parametrize("tag,kw", [("", {}),
                                    ("_vsrc", dict(source_fields=("vx", "vz"), receiver_fields=("vx", "vz", "syy")))])
def test_elastic3d_oracle_matches_reference(prec, tol, tag, kw):
    """3-D isotropic elastic (reference Elastic3D, order 8, boundary saving):
    explosive sources with (vx, vy, vz) receivers, and body-force sources on
    (vx, vz) with (vx, vz, syy) receivers; records and vp / vs / rho
    gradients."""
    d = np.load(GOLD / "elastic3d.npz")
    args = (float(d["dh"]), float(d["dt"]), int(d["abcn"]))
    obs = O.elastic3d_forward(d["vp_true"], d["vs_true"], d["rho_true"], d["wavelet"], d["src"], d["rec"],
                              *args, prec=prec, **kw)
    assert obs.shape == d[f"obs{tag}"].shape
    assert rel(obs, d[f"obs{tag}"]) < tol
    pred, loss, (gvp, gvs, grho) = O.elastic3d_gradient(
        d["vp_init"], d["vs_init"], d["rho_init"], d["wavelet"], d["src"], d["rec"], d[f"obs{tag}"],
        *args, prec=prec, **kw)
    assert rel(pred, d[f"pred{tag}"]) < tol
    assert abs(loss - float(d[f"loss{tag}"])) < 1e-5 * float(d[f"loss{tag}"])
    assert rel(gvp, d[f"grad_vp{tag}"]) < 5 * tol
    assert rel(gvs, d[f"grad_vs{tag}"]) < 5 * tol
    assert rel(grho, d[f"grad_rho{tag}"]) < 5 * tol


@pytest.mark.parametrize("prec,tol", [("f32", 2e-6), ("f64", 5e-6)])
def test_elastic3d_free_surface_oracle_matches_reference(prec, tol):
    """3-D traction-free top face (the full stencil over image values, the
    Robertsson sxx / syy correction, szz = 0 on the surface row): a shot on
    the surface row, (vx, vy, vz, sxx) receivers on it and two rows below.
    Without the surface terms the records differ at order one."""
    d = np.load(GOLD / "elastic3d_free_surface.npz")
    args = (float(d["dh"]), float(d["dt"]), int(d["abcn"]))
    kw = dict(receiver_fields=("vx", "vy", "vz", "sxx"))
    obs = O.elastic3d_forward(d["vp_true"], d["vs_true"], d["rho_true"], d["wavelet"], d["src"], d["rec"],
                              *args, prec=prec, free_surface=True, **kw)
    assert rel(obs, d["obs"]) < tol
    plain = O.elastic3d_forward(d["vp_true"], d["vs_true"], d["rho_true"], d["wavelet"], d["src"], d["rec"],
                                *args, prec=prec, **kw)
    assert rel(plain, d["obs"]) > 0.1
    pred, loss, (gvp, gvs, grho) = O.elastic3d_gradient(
        d["vp_init"], d["vs_init"], d["rho_init"], d["wavelet"], d["src"], d["rec"], d["obs"],
        *args, prec=prec, free_surface=True, **kw)
    assert rel(pred, d["pred"]) < tol
    assert rel(gvp, d["grad_vp"]) < 5 * tol
    assert rel(gvs, d["grad_vs"]) < 5 * tol
    assert rel(grho, d["grad_rho"]) < 5 * tol


@pytest.mark.parametrize("order", [2, 4, 6, 12])
def test_acoustic2d_orders_oracle_matches_reference(order):
    """Spatial orders other than 8: the oracle reproduces the reference's
    records and gradients bit for bit in float32 (order 4 with the forward's
    summed Laplacian)."""
    d = np.load(GOLD / "acoustic_orders.npz")
    a = (float(d["dh"]), float(d["dt"]), int(d["abcn"]))
    obs = O.acoustic_forward(d["vp_true"], d["wavelet"], d["src"], d["rec"], *a, order=order)
    assert np.array_equal(obs.astype(np.float32), d[f"obs_o{order}"])
    pred, loss, g, gw = O.acoustic_gradient(d["vp_init"], d["wavelet"], d["src"], d["rec"], d[f"obs_o{order}"], *a,
                                            order=order)
    assert rel(pred, d[f"pred_o{order}"]) < 1e-6
    assert rel(g, d[f"grad_vp_o{order}"]) < 1e-6
    assert rel(gw, d[f"grad_wavelet_o{order}"]) < 1e-6


@pytest.mark.parametrize("order", [4, 6])
def test_acoustic3d_orders_oracle_matches_reference(order):
    d = np.load(GOLD / "acoustic_orders.npz")
    a = (float(d["dh"]), float(d["dt3"]), int(d["abcn3"]))
    run = O.Acoustic3D(d["vp3_init"], d["wavelet3"], d["src3"], d["rec3"], *a, order=order)
    pred = run.forward()
    assert rel(pred, d[f"pred3_o{order}"]) < 1e-6
    g, gw = run.backward(pred - d[f"obs3_o{order}"])
    assert rel(g, d[f"grad3_vp_o{order}"]) < 1e-6
    assert rel(gw[0], d[f"grad3_wavelet_o{order}"]) < 1e-6     # shot 0: the reference's 3-D defect


@pytest.mark.parametrize("tag,order,kw", [("o2", 2, {}), ("o4", 4, {}), ("o6", 6, {}),
                                          ("o4_fs", 4, dict(free_surface=True, receiver_fields=("vx", "vz", "sxx")))])
def test_elastic_orders_oracle_matches_reference(tag, order, kw):
    """2-D elastic at orders 2, 4, 6 (and 4 with a traction-free top face):
    records bit for bit in float32, gradients within 1e-6 of the reference."""
    d = np.load(GOLD / "elastic_orders.npz")
    a = (float(d["dh"]), float(d["dt"]), int(d["abcn"]))
    obs = O.elastic_forward(d["vp_true"], d["vs_true"], d["rho_true"], d["wavelet"], d["src"], d["rec"], *a,
                            order=order, **kw)
    assert np.array_equal(obs.astype(np.float32), d[f"obs_{tag}"])
    pred, loss, grads = O.elastic_gradient(d["vp_init"], d["vs_init"], d["rho_init"], d["wavelet"], d["src"],
                                           d["rec"], d[f"obs_{tag}"], *a, order=order, **kw)
    assert rel(pred, d[f"pred_{tag}"]) < 1e-6
    for g, n in zip(grads, ("vp", "vs", "rho")):
        assert rel(g, d[f"grad_{n}_{tag}"]) < 1e-6


@pytest.mark.parametrize("tag,order,kw", [("o2", 2, {}), ("o4", 4, {}), ("o6", 6, {}),
                                          ("o4_fs", 4, dict(free_surface=True))])
def test_elastic3d_orders_oracle_matches_reference(tag, order, kw):
    """3-D elastic at orders 2, 4, 6 (and 4 with a traction-free top face):
    records bit for bit in float32, gradients within 1e-6 of the reference."""
    d = np.load(GOLD / "elastic3d_orders.npz")
    a = (float(d["dh"]), float(d["dt"]), int(d["abcn"]))
    obs = O.elastic3d_forward(d["vp_true"], d["vs_true"], d["rho_true"], d["wavelet"], d["src"], d["rec"], *a,
                              order=order, **kw)
    assert np.array_equal(obs.astype(np.float32), d[f"obs_{tag}"])
    pred, loss, grads = O.elastic3d_gradient(d["vp_init"], d["vs_init"], d["rho_init"], d["wavelet"], d["src"],
                                             d["rec"], d[f"obs_{tag}"], *a, order=order, **kw)
    assert rel(pred, d[f"pred_{tag}"]) < 1e-6
    for g, n in zip(grads, ("vp", "vs", "rho")):
        assert rel(g, d[f"grad_{n}_{tag}"]) < 1e-6


@pytest.mark.parametrize("tag,order,kw", [("o8", 8, {}), ("o4", 4, {}),
                                          ("o8_rec", 8, dict(receiver_fields=("vx", "vz", "sH")))])
def test_vti2d_oracle_matches_reference(tag, order, kw):
    """First-order acoustic VTI (AcousticVTI1st): records bit for bit in
    float32, vp / epsilon / delta / rho gradients within 1e-6 of the
    reference, at orders 8 and 4 and with stress receivers."""
    d = np.load(GOLD / "vti2d.npz")
    a = (float(d["dh"]), float(d["dt"]), int(d["abcn"]))
    names = ("vp", "eps", "dlt", "rho")
    obs = O.vti2d_forward(*[d[f"{n}_true"] for n in names], d["wavelet"], d["src"], d["rec"], *a, order=order, **kw)
    assert np.array_equal(obs.astype(np.float32), d[f"obs_{tag}"])
    pred, loss, grads = O.vti2d_gradient(*[d[f"{n}_init"] for n in names], d["wavelet"], d["src"], d["rec"],
                                         d[f"obs_{tag}"], *a, order=order, **kw)
    assert rel(pred, d[f"pred_{tag}"]) < 1e-6
    for g, n in zip(grads, names):
        assert rel(g, d[f"grad_{n}_{tag}"]) < 1e-6


@pytest.mark.parametrize("tag,order,kw", [("o4", 4, {}), ("o8", 8, {}),
                                          ("o4_rec", 4, dict(receiver_fields=("vx", "vy", "sH")))])
def test_vti3d_oracle_matches_reference(tag, order, kw):
    """3-D first-order acoustic VTI (AcousticVTI1st3D): records bit for bit
    in float32, vp / epsilon / delta / rho gradients within 1e-6 of the
    reference, at orders 4 and 8 and with (vx, vy, sH) receivers."""
    d = np.load(GOLD / "vti3d.npz")
    a = (float(d["dh"]), float(d["dt"]), int(d["abcn"]))
    names = ("vp", "eps", "dlt", "rho")
    obs = O.vti3d_forward(*[d[f"{n}_true"] for n in names], d["wavelet"], d["src"], d["rec"], *a, order=order, **kw)
    assert np.array_equal(obs.astype(np.float32), d[f"obs_{tag}"])
    pred, loss, grads = O.vti3d_gradient(*[d[f"{n}_init"] for n in names], d["wavelet"], d["src"], d["rec"],
                                         d[f"obs_{tag}"], *a, order=order, **kw)
    errs = [rel(g, d[f"grad_{n}_{tag}"]) for g, n in zip(grads, names)]
    print(f"vti3d oracle {tag}: record {rel(pred, d[f'pred_{tag}']):.2e}, grads " + " / ".join(f"{e:.2e}" for e in errs))
    assert rel(pred, d[f"pred_{tag}"]) < 1e-6
    assert max(errs) < 1e-6
