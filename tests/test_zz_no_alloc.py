"""bnb_nbdirect_noalloc against bnb_compute on the same inputs.

bnb_nbdirect_noalloc serves callers that may not allocate device memory at
all (an engine that owns the whole device memory through its own pool, or
one that cannot take the device-wide synchronisation of cudaMalloc and
cudaFree while other streams run): it needs no handle and keeps its scratch
in a fixed array inside the library.

This file is collected last on purpose: it must also pass after every other
GPU test has run in the same process.  Two calls in a row must each match
bnb_compute within tolerance and match each other bit for bit (the second
call runs on the scratch the first one left behind).  Each case is also
checked against the FP64 oracle directly, since the all-pairs kernel has its
own minimum image and exclusion search; the output rule (force and energy
added to, force64 and energy64 overwritten) is checked on prefilled buffers,
and two calls on two streams ordered by an event must give the same bits.
"""
import ctypes as C

import numpy as np
import pytest
import torch

import oracle
from blade_b200 import _lib, systems
from blade_b200.nbdirect import NbDirect, params_for

pytestmark = pytest.mark.gpu

MAX_ATOMS = 4096                  # BNB_NOALLOC_MAX_ATOMS in include/bnb.h
FORCE_RMS_TOL = 2e-5              # relative RMS of dU/dx vs bnb_compute
ENERGY_TOL = 2e-5                 # energy difference vs bnb_compute, per max(|E|, N)
ORACLE_FORCE_TOL = 1e-5           # relative RMS of dU/dx vs the FP64 oracle
ORACLE_ENERGY_TOL = 1e-5          # energy difference vs the FP64 oracle, per max(|E|, N)


def _p(t):
    return None if t is None else C.c_void_p(t.data_ptr())


def _stream():
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def _handle_path(s):
    nb = NbDirect(s)
    pos = nb.positions_tensor()
    nb.update_domdec(pos, True)
    f64, _, e64 = nb.evaluate(pos, nb.lambdas_tensor())
    torch.cuda.synchronize()
    out = f64.cpu().numpy().reshape(-1), float(e64.cpu()[0])
    nb.close()
    return out


class _Inputs:
    def __init__(self, s):
        dev = torch.device("cuda")
        self.s = s
        self.params = params_for(s)
        self.box = np.ascontiguousarray(s.box, np.float32)
        self.pos = torch.from_numpy(np.ascontiguousarray(s.xyz, np.float32).reshape(-1)).to(dev)
        self.nbonds = torch.from_numpy(np.ascontiguousarray(s.nbonds).view(np.uint8).copy()).to(dev)
        self.vdw = torch.from_numpy(np.ascontiguousarray(s.vdw, np.float32).reshape(-1)).to(dev)
        start, partner = systems.excl_csr(s.N, s.excl)
        self.start = torch.from_numpy(start).to(dev)
        self.partner = torch.from_numpy(partner if len(partner) else np.zeros(1, np.int32)).to(dev)

    def call(self, force=None, force64=None, energy=None, energy64=None, calc_energy=True, n=None):
        out = _lib.Outputs(force=_p(force), lambdaForce=None, energy=_p(energy), force64=_p(force64),
                           lambdaForce64=None, energy64=_p(energy64))
        return _lib.lib().bnb_nbdirect_noalloc(
            C.byref(self.params), self.s.N if n is None else n, _p(self.pos),
            self.box.ctypes.data_as(C.c_void_p), _p(self.nbonds), self.s.nTypes, _p(self.vdw),
            _p(self.start), _p(self.partner), int(calc_energy), C.byref(out), _stream())


def _small_chain():
    return systems.chain_in_water(seed=5, box=30.0, n_chain=250, n_wat=780, name="chain_water_small")


def _water(elec, vdw):
    s = systems.water_box(4)
    s.elecMethod, s.vdwMethod = elec, vdw
    return s


CASES = {
    "water_pme_vfswitch": lambda: _water(1, 0),
    "water_fshift_vshift": lambda: _water(2, 2),
    "water_fswitch_vswitch": lambda: _water(0, 1),
    "chain_water_pme_vfswitch": _small_chain,
}


@pytest.mark.parametrize("case", list(CASES))
def test_two_calls_match_handle_path(cuda, case):
    s = CASES[case]()
    assert s.N <= MAX_ATOMS
    g_ref, e_ref = _handle_path(s)
    inp = _Inputs(s)
    results = []
    for _ in range(2):
        f32 = torch.zeros(3 * s.N, dtype=torch.float32, device="cuda")
        f64 = torch.zeros(3 * s.N, dtype=torch.float64, device="cuda")
        e = torch.zeros(1, dtype=torch.float64, device="cuda")
        e64 = torch.zeros(1, dtype=torch.float64, device="cuda")
        assert inp.call(force=f32, force64=f64, energy=e, energy64=e64) == 0
        torch.cuda.synchronize()
        g = f64.cpu().numpy()
        rel = np.sqrt(((g - g_ref) ** 2).sum() / (g_ref ** 2).sum())
        assert rel <= FORCE_RMS_TOL, (case, rel)
        en = float(e64.cpu()[0])
        assert abs(en - e_ref) <= ENERGY_TOL * max(abs(e_ref), s.N), (case, en, e_ref)
        assert float(e.cpu()[0]) == en
        np.testing.assert_allclose(f32.cpu().numpy(), g, rtol=1e-6, atol=1e-6)
        results.append((g, en))
    assert np.array_equal(results[0][0], results[1][0])
    assert results[0][1] == results[1][1]
    o = oracle.nbdirect(s)
    g_o = o["grad"].reshape(-1)
    rel = np.sqrt(((results[0][0] - g_o) ** 2).sum() / (g_o ** 2).sum())
    assert rel <= ORACLE_FORCE_TOL, (case, "oracle", rel)
    # energy scale: the larger of |E| and one kcal/mol per atom (a small net
    # energy is a difference of large pair sums)
    assert abs(results[0][1] - o["energy"]) <= ORACLE_ENERGY_TOL * max(abs(o["energy"]), s.N), (case, o["energy"])


@pytest.mark.parametrize("calc_energy", [True, False])
def test_outputs_added_and_overwritten(cuda, calc_energy):
    """force and energy are added to what the caller's buffers hold; force64
    and energy64 are overwritten (energy64 with 0 on a force-only call)."""
    s = _water(1, 0)
    inp = _Inputs(s)
    ref64 = torch.zeros(3 * s.N, dtype=torch.float64, device="cuda")
    refe = torch.zeros(1, dtype=torch.float64, device="cuda")
    assert inp.call(force64=ref64, energy64=refe, calc_energy=calc_energy) == 0
    g = torch.Generator(device="cuda").manual_seed(7)
    pre = torch.randn(3 * s.N, generator=g, device="cuda", dtype=torch.float32) * 3.0
    f32 = pre.clone()
    f64 = torch.full((3 * s.N,), 1.0e30, dtype=torch.float64, device="cuda")
    e = torch.full((1,), -123.25, dtype=torch.float64, device="cuda")
    e64 = torch.full((1,), 4.5e20, dtype=torch.float64, device="cuda")
    assert inp.call(force=f32, force64=f64, energy=e, energy64=e64, calc_energy=calc_energy) == 0
    torch.cuda.synchronize()
    assert torch.equal(f64, ref64)
    want = (pre.double() + ref64).float().cpu().numpy()
    np.testing.assert_allclose(f32.cpu().numpy(), want, rtol=1e-6, atol=1e-5)
    if calc_energy:
        assert float(e64.cpu()[0]) == float(refe.cpu()[0]) != 0.0
        assert float(e.cpu()[0]) == -123.25 + float(refe.cpu()[0])
    else:
        assert float(e64.cpu()[0]) == 0.0
        assert float(e.cpu()[0]) == -123.25


def test_two_streams_ordered_by_event(cuda):
    """Calls on two streams share the scratch array; ordered by an event they
    give the same bits as two calls on one stream."""
    s = _small_chain()
    inp = _Inputs(s)
    one = torch.zeros(3 * s.N, dtype=torch.float64, device="cuda")
    assert inp.call(force64=one) == 0
    torch.cuda.synchronize()
    a = torch.cuda.Stream()
    b = torch.cuda.Stream()
    fa = torch.zeros(3 * s.N, dtype=torch.float64, device="cuda")
    fb = torch.zeros(3 * s.N, dtype=torch.float64, device="cuda")
    ev = torch.cuda.Event()
    a.wait_stream(torch.cuda.current_stream())
    b.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(a):
        assert inp.call(force64=fa) == 0
        ev.record(a)
    b.wait_event(ev)
    with torch.cuda.stream(b):
        assert inp.call(force64=fb) == 0
    torch.cuda.synchronize()
    assert torch.equal(fa, one)
    assert torch.equal(fb, one)


def test_force_only_call_matches(cuda):
    s = _water(1, 0)
    g_ref, _ = _handle_path(s)
    inp = _Inputs(s)
    f64 = torch.zeros(3 * s.N, dtype=torch.float64, device="cuda")
    assert inp.call(force64=f64, calc_energy=False) == 0
    g = f64.cpu().numpy()
    assert np.sqrt(((g - g_ref) ** 2).sum() / (g_ref ** 2).sum()) <= FORCE_RMS_TOL


def test_rejects_sizes_above_limit(cuda):
    inp = _Inputs(_water(1, 0))
    f64 = torch.zeros(3, dtype=torch.float64, device="cuda")
    assert inp.call(force64=f64, n=MAX_ATOMS + 1) == 7          # BNB_ERR_TOO_LARGE, nothing launched
    with pytest.raises(_lib.BnbError, match="size above the fixed limit"):
        _lib.check("bnb_nbdirect_noalloc", 7)


def test_rejects_cutoff_beyond_half_box(cuda):
    s = _water(1, 0)
    inp = _Inputs(s)
    inp.params.rCut = float(s.box[0]) * 0.5 + 0.1
    f64 = torch.zeros(3 * s.N, dtype=torch.float64, device="cuda")
    assert inp.call(force64=f64) == 1                           # BNB_ERR_ARG
