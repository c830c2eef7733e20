"""libbnb's MSLD lambda maps, biases and split Langevin step against the
golden vectors from the reference's own CUDA code (see
tests/test_golden_msld.py for what each file holds).  The step is run as the
batched MSLD step runs it: bnb_theta_force_f32 on the FP32 mirrors,
bnb_langevin_half phase 0, bnb_holonomic_position, phase 1,
bnb_holonomic_position, bnb_lambda_from_theta."""
import ctypes as C
import os

import numpy as np
import pytest
import torch

from blade_b200 import _lib, msld
from blade_b200.holonomic import Constraints
from oracle import update_oracle as U

from test_golden_msld import BIAS_TOL, LAMBDA_TOL, MAPS, STEP_TOL, THETA_FORCE_TOL, step_errors

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))


def _load(name):
    return np.load(os.path.join(HERE, "golden", name + ".npz"))


def _t(a, dt):
    return torch.from_numpy(np.ascontiguousarray(a, dt)).cuda()


@pytest.mark.parametrize("name", MAPS)
def test_maps_and_biases_match_reference(cuda, name):
    g = _load(name)
    sb, ls = _t(g["site_bound"], np.int32), _t(g["lambda_site"], np.int32)
    fixed = _t(g["fixed"], np.uint8)
    fb32 = _t(g["fixed_bias"], np.float32)
    vb = _t(g["var_bias"], np.uint8)
    nvar = g["var_bias"].size // msld.VARBIAS_DTYPE.itemsize
    fnex = float(g["fnex"])
    nL = len(g["lambda_site"])
    for k in range(len(g["theta"])):
        th = _t(g["theta"][k], np.float64)
        lam = torch.zeros(nL, dtype=torch.float64, device="cuda")
        lamf = torch.zeros(nL, dtype=torch.float32, device="cuda")
        msld.lambda_from_theta(sb, fnex, th, lam, lamf, fixed)
        assert np.abs(lam.cpu().numpy() - g["lambda_ref"][k]).max() <= LAMBDA_TOL
        assert torch.equal(lamf, lam.float())
        lam_ref_f = _t(g["lambda_ref"][k], np.float32)
        tf = torch.zeros(nL, dtype=torch.float32, device="cuda")
        msld.theta_force_f32(ls, sb, fnex, lam_ref_f, th.float(), _t(g["lambda_force"][k], np.float32), tf, fixed)
        ref = g["theta_force_ref"][k]
        assert (np.abs(tf.cpu().numpy() - ref) / (1 + np.abs(ref))).max() <= THETA_FORCE_TOL
        lf = torch.zeros(nL, dtype=torch.float32, device="cuda")
        e = torch.zeros(1, dtype=torch.float64, device="cuda")
        _lib.call("bnb_bias_f32", nL, C.c_void_p(lam_ref_f.data_ptr()), C.c_void_p(fb32.data_ptr()), nvar,
                  C.c_void_p(vb.data_ptr()), C.c_void_p(lf.data_ptr()), C.c_void_p(e.data_ptr()),
                  C.c_void_p(torch.cuda.current_stream().cuda_stream))
        ref = g["bias_lambda_force_ref"][k]
        assert (np.abs(lf.cpu().numpy() - ref) / (1 + np.abs(ref))).max() <= BIAS_TOL
        eref = g["bias_energy_ref"][k]
        assert abs(float(e.item()) - eref) / (1 + abs(eref)) <= BIAS_TOL


def test_split_langevin_step_matches_reference(cuda):
    g = _load("update_msld_water")
    inp = U.golden_inputs(g)
    ref = U.golden_outputs(g)
    lp = inp["lp"]
    nx, nt = len(inp["x"]), len(inp["theta"])
    f64 = np.float64
    x, th = _t(inp["x"], f64), _t(inp["theta"], f64)
    v, vt = _t(inp["v"], f64), _t(inp["vtheta"], f64)
    fx, ismx, ismt = _t(inp["fx"], f64), _t(inp["ismx"], f64), _t(inp["ismt"], f64)
    sb, ls = _t(inp["site_bound"], np.int32), _t(inp["lambda_site"], np.int32)
    fnex = inp["fnex"]
    lam = torch.zeros(nt, dtype=torch.float64, device="cuda")
    lamf = torch.zeros(nt, dtype=torch.float32, device="cuda")
    msld.lambda_from_theta(sb, fnex, th, lam, lamf)
    tf = torch.zeros(nt, dtype=torch.float32, device="cuda")
    msld.theta_force_f32(ls, sb, fnex, lamf, th.float(), _t(inp["lambda_force"], np.float32), tf)
    ftheta = tf.double()
    xprev = torch.zeros_like(x)
    xf = torch.zeros(nx, dtype=torch.float32, device="cuda")
    nan = torch.zeros(1, dtype=torch.int32, device="cuda")
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    cons = Constraints(tri=inp["tri"])
    dt = 2.0 * float(lp[2])
    assert float(lp[5]) == float(lp[2])
    P = lambda t: C.c_void_p(t.data_ptr())
    s = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    for phase in (0, 1):
        _lib.call("bnb_langevin_half", phase, nx, nt, P(x), P(v), P(xprev), P(fx), P(ismx), P(th), P(vt), P(ftheta),
                  P(ismt), dt, float(lp[0]), float(lp[1]), float(lp[3]), float(lp[4]), 1, 0, None, P(xf), P(nan), s)
        cons.position(xprev, x, v, ismx, 0.5 * dt, tolerance=1e-10, max_iter=10, x_f=xf, status=status)
    msld.lambda_from_theta(sb, fnex, th, lam, lamf)
    torch.cuda.synchronize()
    assert int(status.item()) == 0 and int(nan.item()) == 0
    out = {"x": x.cpu().numpy(), "v": v.cpu().numpy(), "theta": th.cpu().numpy(), "vtheta": vt.cpu().numpy(),
           "lambda": lam.cpu().numpy(), "theta_force": tf.double().cpu().numpy()}
    err = step_errors(out, ref, inp)
    for k, tol in STEP_TOL.items():
        assert err[k] <= tol, (k, err[k])
