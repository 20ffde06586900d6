"""The FLOP model of the roofline (3t_rh_b200/flops.py) against the
operation-counting instantiation of the oracle's templated physics."""
import importlib


def test_flop_constants_match_op_counts(O):
    fl = importlib.import_module("3t_rh_b200.flops")
    c = O.flop_counts()
    assert c["flux_x"] == fl.FACE_FLUX and c["flux_y"] == fl.FACE_FLUX
    assert c["derived"] == fl.DERIVED
    assert c["noncon_dir"] == fl.NONCON_DIR
    assert c["diffusion"] == fl.DIFFUSION
    assert c["source"] == fl.SOURCE
    assert c["local_dt"] == fl.LOCAL_DT
    assert c["build_l"] == fl.BUILD_L and c["build_r"] == fl.BUILD_R
    # reconstruction_fast = L + R + 6 physical fluxes + 72 projections of
    # length 6 + 72 splits + 12 WENO5 + 6 sums + R.g
    assert c["flux_x"] == (c["build_l"] + c["build_r"] + 6 * c["phys_flux"] + 72 * 11 + 6 + 72 * 3 +
                           12 * c["weno5"] + 6 + 6 * 11)


def test_face_counts(rh):
    fl = importlib.import_module("3t_rh_b200.flops")
    f = rh.cases.init_cylinder()
    nxf, nyf = fl.face_counts(f.fluid, f.grid.nx, f.grid.ny)
    assert nxf > f.fluid.sum() and nyf > f.fluid.sum()
    assert fl.step_flops(int(f.fluid.sum()), nxf, nyf, 4914, 4480) > 0
