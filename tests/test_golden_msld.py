"""The FP64 oracle of the MSLD lambda maps, biases and the Langevin step
against golden vectors from the reference's own CUDA code (built unmodified
into the comparison library; tests/golden/make_golden.py --msld-only):
  msld_maps*.npz        Msld::calc_lambda_from_theta,
                        calc_thetaForce_from_lambdaForce, getforce_fixedBias +
                        getforce_variableBias (src/msld/msld.cu:863-1153) on
                        3 sites x 4 substituents, every variable-bias type
                        1-12, with and without a fixed block;
  update_msld_water.npz one State::update (src/update/update.cu:233-305) of
                        the MSLD water box with rigid waters, friction on and
                        zero Gaussian numbers.
The reference computes the theta forces and biases in FP32 (lambda_fd,
theta_fd, FP32 atomics), so those are compared to FP32 rounding."""
import os

import numpy as np
import pytest

import oracle
from oracle import update_oracle as U

HERE = os.path.dirname(os.path.abspath(__file__))
MAPS = ["msld_maps", "msld_maps_fixed"]
LAMBDA_TOL = 1e-12        # FP64 in both
THETA_FORCE_TOL = 1e-5    # |diff| / (1 + |value|): FP32 reference
BIAS_TOL = 2e-6           # |diff| / (1 + |value|): FP32 reference
STEP_TOL = {"x_free": 1e-8, "x_cons": 5e-6, "v_free": 1e-6, "v_cons": 5e-4, "theta": 1e-8, "vtheta": 1e-6,
            "lambda": 1e-9, "theta_force": 1e-6}


def _load(name):
    return np.load(os.path.join(HERE, "golden", name + ".npz"))


@pytest.mark.parametrize("name", MAPS)
def test_lambda_from_theta(name):
    g = _load(name)
    for k in range(len(g["theta"])):
        lam = oracle.lambda_from_theta(g["site_bound"], float(g["fnex"]), g["theta"][k], g["fixed"].astype(np.int32))
        assert np.abs(lam - g["lambda_ref"][k]).max() <= LAMBDA_TOL


@pytest.mark.parametrize("name", MAPS)
def test_theta_force(name):
    g = _load(name)
    fx = g["fixed"].astype(np.int32)
    for k in range(len(g["theta"])):
        lam_f = g["lambda_ref"][k].astype(np.float32).astype(np.float64)
        th_f = g["theta"][k].astype(np.float32).astype(np.float64)
        tf = oracle.theta_force(g["lambda_site"], g["site_bound"], float(g["fnex"]), lam_f, th_f,
                                g["lambda_force"][k].astype(np.float64), fx)
        ref = g["theta_force_ref"][k]
        assert (np.abs(tf - ref) / (1 + np.abs(ref))).max() <= THETA_FORCE_TOL
        assert np.all(tf[g["fixed"].astype(bool)] == 0)


@pytest.mark.parametrize("name", MAPS)
def test_biases_every_type(name):
    g = _load(name)
    vb = g["var_bias"].view(oracle.VARBIAS_DTYPE)
    assert set(vb["type"]) == set(range(1, 13))
    for k in range(len(g["theta"])):
        lam_f = g["lambda_ref"][k].astype(np.float32).astype(np.float64)
        lf, e = oracle.bias(lam_f, g["fixed_bias"].astype(np.float64), vb)
        ref = g["bias_lambda_force_ref"][k]
        assert (np.abs(lf - ref) / (1 + np.abs(ref))).max() <= BIAS_TOL
        assert abs(e - g["bias_energy_ref"][k]) / (1 + abs(e)) <= BIAS_TOL


def step_errors(out, ref, inp):
    cons = np.zeros(len(inp["x"]) // 3, bool)
    cons[inp["tri"]["idx"].reshape(-1)] = True
    c3 = np.repeat(cons, 3)
    dx, dv = np.abs(out["x"] - ref["x"]), np.abs(out["v"] - ref["v"])
    return {"x_free": dx[~c3].max(), "x_cons": dx[c3].max(), "v_free": dv[~c3].max(), "v_cons": dv[c3].max(),
            "theta": np.abs(out["theta"] - ref["theta"]).max(), "vtheta": np.abs(out["vtheta"] - ref["vtheta"]).max(),
            "lambda": np.abs(out["lambda"] - ref["lambda"]).max(),
            "theta_force": np.abs(out["theta_force"] - ref["theta_force"]).max()}


def test_langevin_step_matches_reference():
    g = _load("update_msld_water")
    inp = U.golden_inputs(g)
    ref = U.golden_outputs(g)
    out = U.msld_step(**inp)
    err = step_errors(out, ref, inp)
    for k, tol in STEP_TOL.items():
        assert err[k] <= tol, (k, err[k])
    assert np.abs(ref["x"] - inp["x"]).max() > 0.05      # the step moved the atoms
