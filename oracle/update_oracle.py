"""FP64 CPU restatement of one MSLD Langevin step (test infrastructure only:
tests/ import it as the checker).

The step is State::update on a step that is not an energy step
(src/update/update.cu:233-305), in the reference's order:
  1. dU/dtheta from dU/dlambda (Msld::calc_thetaForce_from_lambdaForce,
     src/msld/msld.cu:937-998, on the FP32 mirrors of lambda and theta);
  2. update_VVhbpR (update.cu:107-135): v -= 2 (dt/2) ism^2 f; xPrev = x;
     x += (dt/2) v -- only where ism is finite;
  3. holonomic_position (src/holonomic/holonomic.cu) on the clusters;
  4. update_OOhbpR (update.cu:196-229): v = a v + b ism xi; xPrev = x;
     x += (dt/2) v -- (a, b) = (friction, noise) of the coordinates for the
     first 3N degrees of freedom and of theta for the rest;
  5. holonomic_position;
  6. lambda from theta (Msld::calc_lambda_from_theta, msld.cu:863-921).
"""
from __future__ import annotations

import numpy as np

import oracle
from oracle import holonomic_oracle as H


def msld_step(x, theta, v, vtheta, fx, lambda_force, ismx, ismt, lp, site_bound, lambda_site, fnex,
              xi=None, xi_theta=None, tri=(), b1=(), b2=(), b3=(), fixed=None):
    """One step; returns dict(x, theta, v, vtheta, lambda, theta_force).

    x, v, fx, ismx: [3N]; theta, vtheta, lambda_force, ismt: [nL];
    lp = (friction_x, noise_x, halfdt_x, friction_theta, noise_theta,
    halfdt_theta) as LeapParms2 for coordinates then theta; xi, xi_theta:
    the Gaussian numbers (zero when None)."""
    x = np.array(x, np.float64)
    th = np.array(theta, np.float64)
    v = np.array(v, np.float64)
    vt = np.array(vtheta, np.float64)
    ismx = np.asarray(ismx, np.float64)
    ismt = np.asarray(ismt, np.float64)
    lam0 = oracle.lambda_from_theta(site_bound, fnex, th, fixed)
    lam_f = lam0.astype(np.float32).astype(np.float64)
    th_f = th.astype(np.float32).astype(np.float64)
    tf = oracle.theta_force(lambda_site, site_bound, fnex, lam_f, th_f, np.asarray(lambda_force, np.float64), fixed)
    cl = H.clusters(tri, b1, b2, b3)
    fric = (lp[0], lp[3])
    noise = (lp[1], lp[4])
    half = (lp[2], lp[5])
    xi = np.zeros_like(x) if xi is None else np.asarray(xi, np.float64)
    xit = np.zeros_like(th) if xi_theta is None else np.asarray(xi_theta, np.float64)

    def drift(q, w, ism, h):
        ok = np.isfinite(ism)
        q = q.copy()
        q[ok] += h * w[ok]
        return q

    # update_VVhbpR
    okx, okt = np.isfinite(ismx), np.isfinite(ismt)
    v = np.where(okx, v - 2 * half[0] * ismx ** 2 * np.asarray(fx, np.float64), v)
    vt = np.where(okt, vt - 2 * half[1] * ismt ** 2 * tf, vt)
    xp = x.copy()
    x = drift(x, v, ismx, half[0])
    th = drift(th, vt, ismt, half[1])
    if cl:
        xn, vc, _ = H.constrain_position(cl, xp.reshape(-1, 3), x.reshape(-1, 3), ismx, half[0])
        x = xn.reshape(-1)
        for idx, _, _ in cl:
            for a in idx:
                v[3 * a:3 * a + 3] = vc[a]
    # update_OOhbpR
    v = np.where(okx, fric[0] * v + noise[0] * ismx * xi, v)
    vt = np.where(okt, fric[1] * vt + noise[1] * ismt * xit, vt)
    xp = x.copy()
    x = drift(x, v, ismx, half[0])
    th = drift(th, vt, ismt, half[1])
    if cl:
        xn, vc, _ = H.constrain_position(cl, xp.reshape(-1, 3), x.reshape(-1, 3), ismx, half[0])
        x = xn.reshape(-1)
        for idx, _, _ in cl:
            for a in idx:
                v[3 * a:3 * a + 3] = vc[a]
    lam = oracle.lambda_from_theta(site_bound, fnex, th, fixed)
    return {"x": x, "theta": th, "v": v, "vtheta": vt, "lambda": lam, "theta_force": tf}


def golden_inputs(g):
    """Unpacks update_msld_water.npz into msld_step's arguments."""
    N = int(g["n_atoms"])
    nL = len(g["lambda_site"])
    pos, vel, frc = g["pos_in"], g["vel_in"].astype(np.float64), g["frc_in"].astype(np.float64)
    ism = g["ism"].astype(np.float64)
    return dict(x=pos[nL:nL + 3 * N], theta=pos[nL + 3 * N:], v=vel[:3 * N], vtheta=vel[3 * N:],
                fx=frc[nL:nL + 3 * N], lambda_force=frc[:nL], ismx=ism[:3 * N], ismt=ism[3 * N:],
                lp=g["lp"].astype(np.float64), site_bound=g["site_bound"], lambda_site=g["lambda_site"],
                fnex=float(g["fnex"]), tri=g["tri"].view(H.TRI_DTYPE))


def golden_outputs(g):
    N = int(g["n_atoms"])
    nL = len(g["lambda_site"])
    pos, vel, frc = g["pos_ref"], g["vel_ref"].astype(np.float64), g["frc_ref"].astype(np.float64)
    return {"lambda": pos[:nL], "x": pos[nL:nL + 3 * N], "theta": pos[nL + 3 * N:], "v": vel[:3 * N],
            "vtheta": vel[3 * N:], "theta_force": frc[nL + 3 * N:]}
